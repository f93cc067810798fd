"""Small, fixed workloads for profiling one kernel under ncu.

    python -m demystification_dfn_b200.profile_case tc_kv [R]
        R realisations (default 64) of the 800-fault network sharing one
        kernel matrix: three K.V launches of the tensor-core GEMM (2.05 GB of
        BF16 hi + lo entries per launch).
    python -m demystification_dfn_b200.profile_case tc_shapes [R ...]
        for each R (default 64), the same batch: the autotuner's timing of the
        three GEMM shapes (persistent, one unit per CTA with the deepest or a
        2-stage ring), three calls, one JSON line per R; checks that K.V is
        unchanged bit for bit across the calls.
    python -m demystification_dfn_b200.profile_case tc_round [cg|tridiag]
        the same batch, six solve rounds launched one by one (launch list of
        a round: GEMM, pressure, friction, step control).
    python -m demystification_dfn_b200.profile_case hmatrix_kv [n_faults box_m]
        the 4000-fault network in 20 km x 20 km (N = 81 750; or n_faults in a
        box_m square) as an H-matrix (leaf 64, eta 2, ACA 1e-6, FP32
        factors): three K.V launches (several kernels each).
    python -m demystification_dfn_b200.profile_case hmatrix_autotune
        the same network with CG pressure: the autotuner's timing of the
        stage pressure systems by one CTA each and by a cluster of CTAs each
        (one JSON line).
    python -m demystification_dfn_b200.profile_case hmatrix_round
        the same network with shear loading (1e-9 m/s) and CG pressure: four
        solve steps launched one by one (launch list of a step: the H-matrix
        K.V kernels, the pressure solves, the stage kernel, step control).
    python -m demystification_dfn_b200.profile_case ensemble_round
        eight 120-fault networks (FP32 storage, tridiagonal pressure), forty
        solve rounds launched one by one.

Each case exits 0 after printing one line, so the same command can run once
without ncu and then under it.
"""
from __future__ import annotations

import sys

import numpy as np


def main(argv):
    from . import networks
    from .ensemble import Ensemble

    case = argv[0] if argv else "tc_kv"
    if case == "tc_kv":
        R = int(argv[1]) if len(argv) > 1 else 64
        base = networks.fault_network(n_faults=800, seed=0)
        e = Ensemble(networks.shared_geometry_ensemble(R, base=base, seed=0), storage="bf16x2_tc")
        rng = np.random.default_rng(0)
        N = e.n_elements[0]
        for _ in range(3):
            e.kernel([rng.normal(size=N) for _ in range(R)])
    elif case == "tc_shapes":
        import json

        base = networks.fault_network(n_faults=800, seed=0)
        for R in [int(x) for x in argv[1:]] or [64]:
            e = Ensemble(networks.shared_geometry_ensemble(R, base=base, seed=0), storage="bf16x2_tc")
            rng = np.random.default_rng(0)
            N = e.n_elements[0]
            slips = [rng.normal(size=N) for _ in range(R)]
            a = e.kernel(slips)
            tunes = [e.autotune() for _ in range(3)]
            b = e.kernel(slips)
            same = all(np.array_equal(x, y) for x, y in zip(a[0] + a[1], b[0] + b[1]))
            ms = {k: v for k, v in tunes[-1]["ms"].items() if k.startswith("kv_")}
            print(json.dumps({"R": R, "kv_bytes": e.kernel_bytes, "ms": ms, "pick": tunes[-1]["gemv_impl"],
                              "unchanged": same}))
            e.close()
            if not same:
                raise SystemExit("K.V changed across GEMM shapes")
        e = None
    elif case == "tc_round":
        pressure = argv[1] if len(argv) > 1 else "tridiag"
        base = networks.fault_network(n_faults=800, seed=0)
        e = Ensemble(networks.shared_geometry_ensemble(64, base=base, seed=0), storage="bf16x2_tc",
                     pressure=pressure)
        e.set_graphs(False)
        e.solve(n_steps=6, check=False)
    elif case == "hmatrix_kv":
        from .simulation import Simulation

        nf = int(argv[1]) if len(argv) > 1 else 4000
        box = float(argv[2]) if len(argv) > 2 else 20000.0
        p = networks.fault_network(n_faults=nf, box=box, seed=0, kernel="hmatrix", tol=1e-6)
        e = Simulation(p, storage="fp32", hmat_leaf=64, hmat_eta=2.0, hmat_eps=1e-6)
        rng = np.random.default_rng(0)
        for _ in range(3):
            e.kernel(rng.normal(size=e.N))
    elif case == "hmatrix_autotune":
        import json

        from .simulation import Simulation

        p = networks.fault_network(n_faults=4000, box=20000.0, seed=0, kernel="hmatrix", tol=1e-6)
        e = Simulation(p, storage="fp32", pressure="cg", hmat_leaf=64, hmat_eta=2.0, hmat_eps=1e-6)
        print(json.dumps(e.autotune()))
    elif case == "hmatrix_round":
        from .simulation import Simulation

        p = networks.fault_network(n_faults=4000, box=20000.0, seed=0, kernel="hmatrix", tol=1e-6, v_load=1e-9)
        e = Simulation(p, storage="fp32", pressure="cg", hmat_leaf=64, hmat_eta=2.0, hmat_eps=1e-6)
        e.set_graphs(False)
        e.solve_steps(4)
    elif case == "ensemble_round":
        e = Ensemble([networks.ensemble_member(s, n_faults=120) for s in range(64, 72)], storage="fp32",
                     pressure="tridiag")
        e.set_graphs(False)
        e.solve(n_steps=40, check=False)
    else:
        raise SystemExit(f"unknown case {case!r}")
    if e is not None:
        e.close()
    print("ok", case)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
