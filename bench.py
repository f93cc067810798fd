#!/usr/bin/env python
"""Benchmark: RK45 accepted steps/s of the earthquake-cycle hot path.

Workload: seeded random fault network of 800 faults (centres uniform in a
7 km x 7 km square, lengths log-uniform 50-500 m, strikes N(30, 10) deg,
10 m elements, ~16k elements with the fake ones), mode II dense shear+normal
kernel, aging-law rate-and-state friction, 10 MPa pore-pressure step on one
fault, RK45 with tol 1e-8. One "step" is one accepted Cash-Karp step of the
reference's solve() loop (6+ right-hand-side evaluations, each one K.V over
2 x N^2 stored kernel entries, a pressure solve and the friction update).

`value` is whole-job throughput (sum of accepted steps/s over ranks, each rank
integrating its own network realisation: weak scaling); `e2e` times the
same steps through the C ABI with host buffers on both sides (state in,
save_data snapshot out). The K.V matrix (4.3 GB in FP64) is larger than L2,
so every launch streams it from HBM.

`--impl reference` times the CPU restatement of the reference's own
algorithm (matrix-free directII, CG pressure, rkqs) with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(n_faults=800, box=7000.0, seed=0, tol=1e-8)


def make_problem(rank=0, n_faults=None):
    from demystification_dfn_b200 import networks

    kw = dict(WORKLOAD)
    if n_faults:
        kw["n_faults"] = n_faults
    kw["seed"] = kw["seed"] + rank
    return networks.fault_network(**kw)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes (read + write) per K.V launch of the headline workload from ncu:
# FP64 storage, the 800-fault network, scaled by matrix bytes from the
# capture of the N = 4 395 case (profiles/kv_gemv_tma_fp64_network800.md)
TRAFFIC = {"fp64": 4194000000}


def traffic_per_launch(storage):
    return TRAFFIC.get(storage)


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"dfn_bench_clocks_rank{index}_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_rhs_seconds(problem, threads=1):
    """Seconds of one right-hand-side evaluation (matrix-free directII K.V,
    pressure CG, friction law) of the CPU restatement on ``threads`` cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle
    from demystification_dfn_b200.layout import build_arrays

    o = Oracle(problem, threads=threads)
    Y = build_arrays(problem).Y0()
    t0 = time.perf_counter()
    o.friction_law(1.0, Y)
    dt = time.perf_counter() - t0
    o.close()
    return dt


def time_oracle_steps(problem, threads, warmup, steps, budget_s):
    """The CPU restatement of the reference path (matrix-free directII, CG,
    rkqs) on ``threads`` host cores: ``warmup`` untimed accepted steps from
    the initial state, then at most ``steps`` timed steps or ``budget_s``
    seconds. Both the GPU arm's cpu_baseline and the reference arm use it, so
    the two figures time the same sample. Returns (timed steps, seconds, N)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle

    o = Oracle(problem, threads=threads)
    for _ in range(warmup):
        o.lib.orc_solve_step(o.o)
    t0 = time.perf_counter()
    n = 0
    while n < steps:
        st = o.lib.orc_solve_step(o.o)
        n += 1
        if st != 0 or time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    N = o.N
    o.close()
    return n, dt, N


def bench_config(N):
    """The workload description printed by both arms (identical dicts)."""
    return {"workload": "fault network 800 faults 7x7 km, mode II dense kernel, FP64 (seeded synthetic)",
            "n_faults": WORKLOAD["n_faults"], "n_elements": int(N), "tol_solver": WORKLOAD["tol"],
            "l2": "K.V matrix %.2f GB > 126 MB L2, streamed from HBM each launch" % (16.0 * N * N / 1e9)}


def _timed(stream, fn):
    import torch

    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a0.record(stream)
    out = fn()
    a1.record(stream)
    torch.cuda.synchronize()
    return out, a0.elapsed_time(a1)


def leg_single_fault(args, local, stream):
    """One straight 40 km fault, 4000 x 10 m elements, mode II dense FP64
    kernel (256 MB), injection at the centre, tol 1e-8; CG (the reference's
    solver) and the exact tridiagonal pressure solve."""
    from demystification_dfn_b200 import networks
    from demystification_dfn_b200.simulation import Simulation

    from demystification_dfn_b200.networks import YEAR

    out = {"workload": "single fault 40 km, 4000 elements, 50 kg/s injection, tol 1e-8; modes II and III"}
    for mode in ("modeII", "modeIII"):
        p = networks.single_fault(mode=mode)
        for pressure in ("cg", "tridiag"):
            s = Simulation(p, pressure=pressure, device=local, gemv=args.gemv)
            s.set_stream(stream.cuda_stream)
            s.solve_steps(3)
            n = 200
            rep, ms = _timed(stream, lambda: s.solve_steps(n))
            res = {"steps_per_s": n / (ms / 1e3), "kv_ms": s.time_kernel(20), "kv_bytes": s.kernel_bytes,
                   "simulated_s": rep["time"], "cg_iterations": rep["cg_iterations"],
                   "probe_halvings": rep["probe_halvings"]}
            s.close()
            # the configuration's span: one simulated year from the start
            s = Simulation(p, pressure=pressure, device=local, gemv=args.gemv)
            s.set_stream(stream.cuda_stream)
            try:
                r1, ms1 = _timed(stream, lambda: s.solve_to(YEAR))
                res["one_year"] = {"wall_s": ms1 / 1e3, "accepted_steps": r1["it_count"], "status": r1["status"]}
            except Exception as exc:   # a stop of the reference's own rules (status code)
                res["one_year"] = {"stopped": str(exc)[:200], "state_time": s.state()["time"]}
            s.close()
            out[f"{mode}_{pressure}"] = res
    return out


def hmatrix_network(kernel="hmatrix"):
    """4000 seeded faults in 20 km x 20 km (~82k elements), tectonic shear
    loading of 1e-9 m/s (mu v / L per fault); kernel "direct" gives the same
    network with the dense kernel matrix."""
    from demystification_dfn_b200 import networks

    return networks.fault_network(n_faults=4000, box=20000.0, seed=0, kernel=kernel, tol=1e-6, v_load=1e-9)


def leg_hmatrix(args, local, stream):
    """4000 seeded faults in 20 km x 20 km (~82k elements), H-matrix with
    leaf 64, eta 2, ACA 1e-6, FP32 factors, FP64 sums."""
    from demystification_dfn_b200.simulation import Simulation

    hbm, _ = peaks()
    p = hmatrix_network()
    t0 = time.perf_counter()
    s = Simulation(p, storage="fp32", pressure=args.pressure, device=local, gemv=args.gemv, hmat_leaf=64,
                   hmat_eta=2.0, hmat_eps=1e-6)
    build_s = time.perf_counter() - t0
    s.set_stream(stream.cuda_stream)
    st = s.hmat_stats()
    tune = s.autotune()
    s.solve_steps(3)
    s.profile_kv(True)
    n = 10
    rep, ms = _timed(stream, lambda: s.solve_steps(n))
    kms, kn = s.profile_kv_read()
    s.profile_kv(False)
    kavg = kms / max(kn, 1)
    gbs = s.kernel_bytes / (kavg / 1e3) / 1e9
    dense_equiv = 2 * s.N * s.N * 4
    out = {"workload": "4000 faults 20x20 km, shear loading 1e-9 m/s, H-matrix leaf 64 eta 2 ACA 1e-6, FP32 factors",
           "n_elements": s.N,
           "build_s": build_s, "stats": st, "autotune": tune, "steps_per_s": n / (ms / 1e3), "kv_avg_ms": kavg,
           "kv_bytes": s.kernel_bytes, "kv_GBps": gbs, "kv_frac_of_measured_hbm": gbs / hbm,
           "compression_vs_dense_fp32": s.kernel_bytes / dense_equiv, "simulated_s": rep["time"]}
    st32 = s.state()
    vk = np.random.default_rng(11).normal(size=s.N) * 1e-9
    hk = s.kernel(vk)
    s.close()
    # the same 13 steps with FP64 factors (the FP64 H-matrix reference run)
    s = Simulation(p, storage="fp64", pressure=args.pressure, device=local, gemv=args.gemv, hmat_leaf=64,
                   hmat_eta=2.0, hmat_eps=1e-6)
    s.set_stream(stream.cuda_stream)
    s.solve_steps(3 + n)
    st64 = s.state()
    s.close()
    N = len(st64["P"])
    V32, V64 = st32["Y"][:N], st64["Y"][:N]
    out["fp32_vs_fp64_factors"] = {
        "rel_err_V": float(np.abs(V32 - V64).max() / np.abs(V64).max()),
        "rel_err_psi": float(np.abs(st32["Y"][N:2 * N] - st64["Y"][N:2 * N]).max() / np.abs(st64["Y"][N:2 * N]).max()),
        "rel_err_time": abs(st32["time"] - st64["time"]) / st64["time"],
        "compared_after": "13 accepted steps from the same start"}
    # the H-matrix K.V against the dense K.V of the same network (FP32
    # entries, 2 x N^2 x 4 B = 53 GB on the device)
    s = Simulation(hmatrix_network("direct"), storage="fp32", pressure=args.pressure, device=local, gemv=args.gemv)
    s.set_stream(stream.cuda_stream)
    dk = s.kernel(vk)
    s.close()
    out["kv_vs_dense_fp32"] = {
        "rel_err_shear": float(np.abs(hk[0] - dk[0]).max() / np.abs(dk[0]).max()),
        "rel_err_normal": float(np.abs(hk[1] - dk[1]).max() / np.abs(dk[1]).max()),
        "slip_rates": "seeded normal x 1e-9 m/s", "eps_aca": 1e-6}
    return out


def leg_learned(args, local, stream):
    """Newton slip formulation with the learned initial guess.

    Record the Newton solves that the analytic start does not settle on
    training networks (ensemble seeds 0-7, 120 faults each), train the MLP on
    the GPU, then deploy it on held-out seeds 64-71 up to the same simulated
    time as (i) the FP64 Newton run with the analytic start, the reference of
    this formulation, (ii) FP32 storage with the analytic start and (iii)
    FP32 storage with the learned guess; (ii') FP32 with the quasi-static
    start (radiation damping neglected) shows what the bounded analytic start
    already saves. The FP64 V formulation (the reference's own ODE) is run
    beside it for its step count and its slip rates at the same time."""
    from demystification_dfn_b200 import learned, networks
    from demystification_dfn_b200.ensemble import Ensemble
    from demystification_dfn_b200.layout import build_arrays
    from demystification_dfn_b200.simulation import Simulation

    kw = dict(n_faults=120)
    t_end, max_steps = 2.0e6, 6000
    train_nets = [networks.ensemble_member(s, **kw) for s in range(8)]
    test_nets = [networks.ensemble_member(s, **kw) for s in range(64, 72)]
    cap = 4_000_000
    ens = Ensemble(train_nets, storage="fp32", pressure="tridiag", device=local, formulation="newton")
    ens.set_stream(stream.cuda_stream)
    ens.record(cap)
    ens.solve(n_steps=max_steps, t_end=t_end, check=False)
    x, t = ens.record_read(cap)
    ens.close()
    t0 = time.perf_counter()
    w, loss = learned.train(x, t, epochs=20, batch=4096, lr=2e-3, seed=0)
    out = {"workload": "8 held-out networks (ensemble seeds 64-71, 120 faults, injection + diffusion), "
                       "to t = %.0e s" % t_end,
           "train_samples": int(len(t)), "train_loss_first_last": [float(loss[0]), float(loss[1])],
           "train_s": time.perf_counter() - t0, "networks": len(test_nets)}
    runs = (("newton_fp64_analytic", "newton", "analytic", "fp64", None),
            ("newton_fp32_quasistatic", "newton", "quasistatic", "fp32", None),
            ("newton_fp32_analytic", "newton", "analytic", "fp32", None),
            ("newton_fp32_mlp", "newton", "mlp", "fp32", None),
            ("newton_fp32_mlp_ungated", "newton", "mlp", "fp32", 0.0),
            ("newton_fp32_mlp_gate1e-2", "newton", "mlp", "fp32", 1e-2),
            ("newton_fp32_mlp_gate1e-3", "newton", "mlp", "fp32", 1e-3),
            ("newton_fp32_mlp_never", "newton", "mlp", "fp32", 1e300),
            ("v_fp64", "v", "analytic", "fp64", None))
    ref = None
    for name, form, guess, store, gate in runs:
        e = Ensemble(test_nets, storage=store, pressure="tridiag", device=local, formulation=form, guess=guess)
        e.set_stream(stream.cuda_stream)
        if guess == "mlp":
            e.set_mlp(w)
            if gate is not None:
                e.set_mlp_gate(gate)
        out["elements"] = int(sum(e.n_elements))
        reps, ms = _timed(stream, lambda: e.solve(n_steps=max_steps, t_end=t_end, check=False))
        steps = sum(r["it_count"] for r in reps)
        res = {"ms_to_t_end": ms, "accepted_steps": int(steps), "steps_per_s": steps / (ms / 1e3),
               "newton_solves": int(sum(r["newton_solves"] for r in reps)),
               "newton_iterations": int(sum(r["newton_iters"] for r in reps)),
               "newton_fail": int(sum(r["newton_fail"] for r in reps)),
               "mlp_warps": int(sum(r["mlp_warps"] for r in reps)),
               "reached_t_end": sum(1 for r in reps if abs(r["time"] - t_end) <= 1e-9 * t_end),
               "status_counts": {str(s): sum(1 for r in reps if r["status"] == s)
                                 for s in sorted({r["status"] for r in reps})}}
        states = [e.state(i) for i in range(len(test_nets))]
        e.close()
        # slip (Newton state) and slip rate of every network at t_end
        fin = []
        for i, p in enumerate(test_nets):
            st = states[i]
            if abs(st["time"] - t_end) > 1e-9 * t_end:
                fin.append(None)
                continue
            if form == "v":
                fin.append((None, st["Y"][:len(st["P"])]))
                continue
            with Simulation(p, storage="fp32", pressure="tridiag", device=local, formulation="newton") as s:
                s.set_stream(stream.cuda_stream)
                s.set_state(st["Y"], st["P"], st["time"], st["t_try"], st["it_count"])
                fin.append((st["Y"][:s.N].copy(), s.velocity()))
        if ref is None:
            ref = fin
            res["max_V_at_t_end"] = max(float(np.abs(f[1]).max()) for f in fin if f is not None)
        else:
            es, ev = 0.0, 0.0
            for i, p in enumerate(test_nets):
                if fin[i] is None or ref[i] is None:
                    continue
                real = ~build_arrays(p).fake_mask
                if fin[i][0] is not None:
                    d, dr = fin[i][0][real], ref[i][0][real]
                    es = max(es, float(np.abs(d - dr).max() / max(np.abs(dr).max(), 1e-300)))
                v, vr = fin[i][1][real], ref[i][1][real]
                ev = max(ev, float(np.abs(v - vr).max() / np.abs(vr).max()))
            if form != "v":
                res["max_rel_err_slip_vs_newton_fp64"] = es
            res["max_rel_err_V_vs_newton_fp64"] = ev
        out[name] = res
    m = out["newton_fp32_mlp"]
    per = lambda r: r["newton_iterations"] / max(r["newton_solves"], 1)
    for base in ("quasistatic", "analytic"):
        b = out["newton_fp32_" + base]
        if b["newton_iterations"]:
            out["newton_iterations_per_solve_saved_vs_" + base] = 1.0 - per(m) / per(b)
    out["time_to_t_end_newton_fp32_analytic_over_mlp"] = out["newton_fp32_analytic"]["ms_to_t_end"] / m["ms_to_t_end"]
    out["time_to_t_end_v_fp64_over_newton_fp32_mlp"] = out["v_fp64"]["ms_to_t_end"] / m["ms_to_t_end"]
    out["time_to_t_end_newton_fp64_over_newton_fp32_mlp"] = (out["newton_fp64_analytic"]["ms_to_t_end"]
                                                              / m["ms_to_t_end"])
    return out


def hmat_eps(name):
    """ACA tolerance of an H-matrix variant of the 64-network comparison
    (1e-7 unless its name says otherwise)."""
    for e in ("1e-5", "1e-6"):
        if "eps" + e in name:
            return float(e)
    return 1e-7


def hmat_leaf(name):
    """Leaf size of an H-matrix variant of the 64-network comparison (64
    unless its name says otherwise)."""
    for n in ("96", "128"):
        if "leaf" + n in name:
            return int(n)
    return 64


def leg_ensemble64(args, local, stream, t_end=3.0e5, n_steps=10):
    """The ensemble comparison the metric is quoted on: 64 seeded networks
    (seeds 0-63, 100-400 faults each, 2k-10k elements, distinct geometries,
    so one kernel matrix per network, 25 GB in FP64), injection and
    diffusion per network. For each variant (formulation, K storage, Newton
    start): RK45 network-steps/s over ``n_steps`` steps per network, time to
    ``t_end`` from the initial state, and the slip at t_end against the FP64
    run of the same formulation (V formulation: the reference's ODE, slip
    integrated as a passive component; Newton: slip is the state). The FP64
    GPU paths follow the oracle to 1e-8 in the parity tests. The learned
    guess is trained on solves recorded from eight held-out networks (seeds
    64-71). The H-matrix variants use eta 2, leaves of 64 (or 96, 128)
    elements and an ACA tolerance of 1e-7 (or 1e-6, 1e-5: fewer stored
    factors; their slip error is reported like the others')."""
    from demystification_dfn_b200 import learned, networks
    from demystification_dfn_b200.ensemble import Ensemble

    hbm, _ = peaks()
    members = networks.ensemble(64)
    variants = (("v_fp64", "v", "fp64", "analytic"), ("v_fp32", "v", "fp32", "analytic"),
                ("v_bf16x2", "v", "bf16x2", "analytic"), ("newton_fp64", "newton", "fp64", "analytic"),
                ("newton_fp32", "newton", "fp32", "analytic"), ("newton_fp32_mlp", "newton", "fp32", "mlp"),
                ("newton_bf16x2_mlp", "newton", "bf16x2", "mlp"), ("newton_hmat_fp32", "newton", "fp32", "analytic"),
                ("newton_hmat_eps1e-6_fp32", "newton", "fp32", "analytic"),
                ("newton_hmat_eps1e-5_fp32", "newton", "fp32", "analytic"),
                ("newton_hmat_leaf96_eps1e-5_fp32", "newton", "fp32", "analytic"),
                ("newton_hmat_leaf128_eps1e-5_fp32", "newton", "fp32", "analytic"))
    hmembers = networks.ensemble(64, kernel="hmatrix")
    # the learned guess: solves recorded on held-out networks, trained on the GPU
    held = [networks.ensemble_member(s) for s in range(64, 72)]
    rec = Ensemble(held, storage="fp32", pressure="tridiag", device=local, formulation="newton")
    rec.set_stream(stream.cuda_stream)
    cap = 4_000_000
    rec.record(cap)
    rec.solve(n_steps=60, check=False)
    xr, tr = rec.record_read(cap)
    rec.close()
    t0 = time.perf_counter()
    weights, loss = learned.train(xr, tr, epochs=20, batch=4096, lr=2e-3, seed=0)
    out = {"networks": len(members), "t_end_s": t_end, "timed_steps_per_network": n_steps,
           "learned": {"train_samples": int(len(tr)), "train_s": time.perf_counter() - t0,
                       "loss_first_last": [float(loss[0]), float(loss[1])]}}
    slips_ref = {}
    for name, form, store, guess in variants:
        hm = "hmat" in name
        t0 = time.perf_counter()
        e = Ensemble(hmembers if hm else members, storage=store, pressure="tridiag", device=local,
                     formulation=form, guess=guess,
                     **(dict(hmat_leaf=hmat_leaf(name), hmat_eta=2.0, hmat_eps=hmat_eps(name)) if hm else {}))
        create_s = time.perf_counter() - t0
        e.set_stream(stream.cuda_stream)
        if guess == "mlp":
            e.set_mlp(weights)
        tune = e.autotune()
        reps, ms_end = _timed(stream, lambda: e.solve(t_end=t_end, check=False))
        res = {"elements": int(sum(e.n_elements)), "kv_bytes": e.kernel_bytes, "ms_to_t_end": ms_end,
               "create_s": create_s,
               "steps_to_t_end": int(sum(r["it_count"] for r in reps)),
               "reached_t_end": sum(1 for r in reps if abs(r["time"] - t_end) <= 1e-9 * t_end),
               "status_counts": {str(c): sum(1 for r in reps if r["status"] == c)
                                 for c in sorted({r["status"] for r in reps})}}
        slips = [e.slip(i) for i in range(len(members))]
        ok = [i for i, r in enumerate(reps) if r["status"] == 0 and abs(r["time"] - t_end) <= 1e-9 * t_end]
        ref_name = form + "_fp64"
        if name == ref_name:
            slips_ref[form] = (slips, set(ok))
        elif form in slips_ref:
            ref, ref_ok = slips_ref[form]
            err = 0.0
            for i in ok:
                if i not in ref_ok:
                    continue
                real = ~e.arrays[i].fake_mask
                d, r = slips[i][real], ref[i][real]
                err = max(err, float(np.abs(d - r).max() / max(np.abs(r).max(), 1e-300)))
            res["slip_rel_err_vs_fp64"] = err
        e.profile_kv(True)
        reps2, ms = _timed(stream, lambda: e.solve(n_steps=n_steps, check=False))
        kms, kn = e.profile_kv_read()
        e.profile_kv(False)
        kavg = kms / max(kn, 1)
        live = sum(1 for r in reps2 if r["status"] == 0)
        # the K.V of all 64 networks back to back (launches inside the loop
        # skip the networks that sit out a round, so their mean understates
        # a full launch)
        kfull = e.time_kernel(10)
        res.update({"network_steps_per_s": len(members) * n_steps / (ms / 1e3), "networks_ok": live,
                    "kv_avg_ms_in_loop": kavg, "kv_ms_all_networks": kfull,
                    "kv_frac_of_measured_hbm": e.kernel_bytes / (kfull / 1e3) / 1e9 / hbm,
                    "kv_impl": tune["gemv_impl"],
                    "newton_iterations_per_solve": (sum(r["newton_iters"] for r in reps) /
                                                    max(sum(r["newton_solves"] for r in reps), 1))})
        e.close()
        out[name] = res
    base = out["v_fp64"]
    for name, *_ in variants:
        out[name]["steps_per_s_vs_v_fp64"] = out[name]["network_steps_per_s"] / base["network_steps_per_s"]
        out[name]["time_to_t_end_vs_v_fp64"] = base["ms_to_t_end"] / out[name]["ms_to_t_end"]
    return out


def leg_tensor_core(args, local, stream, t_end=200.0, n_steps=20):
    """Shared-geometry ensemble: 64 realisations of the 800-fault network
    (per-member a, b, initial V and stepped fault) sharing one kernel matrix,
    so the K.V of all members in a stage is one GEMM streaming K once. The
    FP64 shared-K batch (FP64 products and sums on the CUDA cores) against
    the BF16 hi+lo tcgen05 batch (FP32 accumulation), in the V formulation
    and the Newton formulation (with and without the learned guess, trained
    on solves recorded from eight members): network-steps/s, time to
    ``t_end`` and the slip of every member at t_end against the FP64
    shared-K run of the same formulation (which follows the per-network
    FP64 path to 1e-9 in the tests). Isolates the tensor-core arithmetic
    from the sharing of K."""
    from demystification_dfn_b200 import learned, networks
    from demystification_dfn_b200.ensemble import Ensemble

    hbm, _ = peaks()
    tc_peak = 1653.7
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        tc_peak = float(json.load(open(pk)).get("bf16_tflops", tc_peak))
    base = make_problem(0, args.n_faults)
    R = 64
    members = networks.shared_geometry_ensemble(R, base=base, seed=0)
    out = {"workload": f"{R} realisations of the {len(base.faults)}-fault network sharing one kernel matrix",
           "members": R, "pressure_solver": "tridiag (exact implicit step)", "t_end_s": t_end,
           "timed_steps_per_member": n_steps}
    pressure = "tridiag"
    rec = Ensemble(members[:8], storage="bf16x2_tc", pressure=pressure, device=local, formulation="newton")
    rec.set_stream(stream.cuda_stream)
    rec.record(2_000_000)
    rec.solve(n_steps=60, check=False)
    xr, tr = rec.record_read(2_000_000)
    rec.close()
    weights = learned.train(xr, tr, epochs=20, batch=4096, lr=2e-3, seed=0)[0] if len(tr) >= 4096 else None
    out["learned_train_samples"] = int(len(tr))
    runs = [("fp64_shared_v", "fp64_shared", "v", "analytic"), ("tc_v", "bf16x2_tc", "v", "analytic"),
            ("fp64_shared_newton", "fp64_shared", "newton", "analytic"),
            ("tc_newton", "bf16x2_tc", "newton", "analytic")]
    if weights is not None:
        runs.append(("tc_newton_learned", "bf16x2_tc", "newton", "mlp"))
    ref = {}
    for name, store, form, guess in runs:
        e = Ensemble(members, storage=store, pressure=pressure, device=local, formulation=form, guess=guess)
        e.set_stream(stream.cuda_stream)
        if guess == "mlp":
            e.set_mlp(weights)
        res_tune = e.autotune()
        N = e.n_elements[0]
        reps, ms_end = _timed(stream, lambda: e.solve(t_end=t_end, check=False))
        slips = [e.slip(i) for i in range(R)]
        ok = {i for i, r in enumerate(reps) if r["status"] == 0 and abs(r["time"] - t_end) <= 1e-9 * t_end}
        res = {"ms_to_t_end": ms_end, "steps_to_t_end": int(sum(r["it_count"] for r in reps)),
               "reached_t_end": len(ok)}
        if store == "fp64_shared":
            ref[form] = (slips, ok)
        else:
            rs, rok = ref[form]
            err = 0.0
            for i in ok & rok:
                real = ~e.arrays[i].fake_mask
                err = max(err, float(np.abs(slips[i][real] - rs[i][real]).max() / np.abs(rs[i][real]).max()))
            res["slip_rel_err_vs_fp64_shared_k"] = err
        e.profile_kv(True)
        reps2, ms = _timed(stream, lambda: e.solve(n_steps=n_steps, check=False))
        kms, kn = e.profile_kv_read()
        e.profile_kv(False)
        kavg = kms / max(kn, 1)
        res.update({"network_steps_per_s": R * n_steps / (ms / 1e3), "ms_per_round": ms / n_steps,
                    "kv_avg_ms": kavg, "kv_bytes": e.kernel_bytes,
                    "kv_GBps": e.kernel_bytes / (kavg / 1e3) / 1e9,
                    "kv_frac_of_measured_hbm": e.kernel_bytes / (kavg / 1e3) / 1e9 / hbm,
                    "status_counts": {str(c): sum(1 for r in reps2 if r["status"] == c)
                                      for c in sorted({r["status"] for r in reps2})},
                    "autotune": res_tune,
                    "newton_iterations_per_solve": (sum(r["newton_iters"] for r in reps) /
                                                    max(sum(r["newton_solves"] for r in reps), 1))})
        if store == "bf16x2_tc":
            flops = 3 * 2 * (2 * N) * N * R      # three BF16 products per entry, mode II rows
            res["tensor_TFLOPs"] = flops / (kavg / 1e3) / 1e12
            res["tensor_frac_of_measured_bf16"] = res["tensor_TFLOPs"] / tc_peak
        else:
            res["fp64_TFLOPs"] = 2 * (2 * N) * N * R / (kavg / 1e3) / 1e12
        e.close()
        out[name] = res
    for form in ("v", "newton"):
        a, b = out.get("fp64_shared_" + form), out.get("tc_" + form)
        if a and b:
            out["tc_over_fp64_shared_" + form] = {
                "network_steps_per_s": b["network_steps_per_s"] / a["network_steps_per_s"],
                "kv": a["kv_avg_ms"] / b["kv_avg_ms"], "time_to_t_end": a["ms_to_t_end"] / b["ms_to_t_end"]}
    return out


def leg_span(args, local, stream):
    """The benchmark network over the configuration's span (0.1 simulated
    year) from its initial state, FP64 plain path, in chunks of 500 accepted
    steps until the span is reached or 120 s of wall time have passed."""
    from demystification_dfn_b200 import _lib
    from demystification_dfn_b200.layout import DfnReport
    from demystification_dfn_b200.networks import YEAR
    from demystification_dfn_b200.simulation import Simulation

    span = 0.1 * YEAR
    s = Simulation(make_problem(0, args.n_faults), storage="fp64", pressure=args.pressure, device=local,
                   gemv=args.gemv)
    s.set_stream(stream.cuda_stream)
    reps = (DfnReport * 1)()
    t0 = time.perf_counter()
    while True:
        _lib.check(s.lib.dfn_solve_batch(s.h, 500, float(span), reps), s.lib)
        rep = reps[0].as_dict()
        done = rep["time"] >= span * (1 - 1e-12)
        if done or rep["status"] != 0 or time.perf_counter() - t0 > 120.0:
            break
    wall = time.perf_counter() - t0
    out = {"span_s": span, "reached_s": rep["time"], "accepted_steps": int(rep["it_count"]), "wall_s": wall,
           "status": int(rep["status"]), "complete": bool(done)}
    s.close()
    return out


def leg_ensemble_span(args, local, stream, storage="fp32", wall_limit=240.0):
    """The 64-network ensemble over its whole span (1 simulated year), FP32
    storage, one handle, in chunks of 1000 accepted steps per network until
    every network has reached the span or the wall-time limit has passed.
    Not in the default legs (about three minutes)."""
    from demystification_dfn_b200 import networks
    from demystification_dfn_b200.ensemble import Ensemble
    from demystification_dfn_b200.networks import YEAR

    members = networks.ensemble(64)
    e = Ensemble(members, storage=storage, pressure=args.pressure, device=local, gemv=args.gemv)
    e.set_stream(stream.cuda_stream)
    tune = e.autotune()
    t0 = time.perf_counter()
    while True:
        reps = e.solve(n_steps=1000, t_end=YEAR, check=False)
        times = np.array([r["time"] for r in reps])
        live = [r for r in reps if r["status"] == 0 and r["time"] < YEAR * (1 - 1e-12)]
        if not live or time.perf_counter() - t0 > wall_limit:
            break
    wall = time.perf_counter() - t0
    steps = int(sum(r["it_count"] for r in reps))
    out = {"networks": len(members), "storage": storage, "span_s": YEAR, "wall_s": wall,
           "networks_complete": int(sum(1 for r in reps if r["time"] >= YEAR * (1 - 1e-12))),
           "min_reached_s": float(times.min()), "median_reached_s": float(np.median(times)),
           "accepted_steps_total": steps, "network_steps_per_s": steps / wall,
           "rejected_total": int(sum(r["rejected"] for r in reps)),
           "status_counts": {str(st): sum(1 for r in reps if r["status"] == st) for st in sorted({r["status"] for r in reps})},
           "short_segments": tune["short_segments"], "kv_impl": tune["gemv_impl"]}
    e.close()
    return out


def leg_hmatrix_span(args, local, stream, wall_limit=300.0):
    """The H-matrix network (config of leg_hmatrix) toward its 100-year span:
    chunks of 500 accepted steps until 100 simulated years or the wall-time
    limit; reports the simulated time reached and the largest slip rate at
    the chunk ends (seismic phases: V > 1e-3 m/s). Not in the default legs."""
    from demystification_dfn_b200.networks import YEAR
    from demystification_dfn_b200.simulation import Simulation

    from demystification_dfn_b200 import _lib
    from demystification_dfn_b200.layout import DfnReport

    s = Simulation(hmatrix_network(), storage="fp32", pressure=args.pressure, device=local, gemv=args.gemv,
                   hmat_leaf=64, hmat_eta=2.0, hmat_eps=1e-6)
    s.set_stream(stream.cuda_stream)
    s.autotune()
    span = 100.0 * YEAR
    reps = (DfnReport * 1)()
    t0 = time.perf_counter()
    vmax, t_seismic = 0.0, None
    while True:
        _lib.check(s.lib.dfn_solve_batch(s.h, 500, float(span), reps), s.lib)
        rep = reps[0].as_dict()
        v = float(np.abs(s.velocity()).max())
        if v > vmax:
            vmax = v
        if t_seismic is None and v > 1e-3:
            t_seismic = rep["time"]
        if rep["status"] != 0 or rep["time"] >= span * (1 - 1e-12) or time.perf_counter() - t0 > wall_limit:
            break
    wall = time.perf_counter() - t0
    out = {"span_years": 100.0, "reached_years": rep["time"] / YEAR, "accepted_steps": int(rep["it_count"]),
           "wall_s": wall, "steps_per_s": rep["it_count"] / wall, "max_V_seen": vmax,
           "first_seismic_time_years": None if t_seismic is None else t_seismic / YEAR, "status": int(rep["status"])}
    s.close()
    return out


def run_case(argv):
    """Small, fixed workloads for profiling one kernel under ncu:

    python bench.py --case tc_kv [R]
        R realisations (default 64) of the 800-fault network sharing one
        kernel matrix: three K.V launches of the tensor-core GEMM (2.05 GB of
        BF16 hi + lo entries per launch).
    python bench.py --case tc_shapes [R ...]
        for each R (default 64), the same batch: the autotuner's timing of the
        three GEMM shapes (persistent, one unit per CTA with the deepest or a
        2-stage ring), three calls, one JSON line per R; checks that K.V is
        unchanged bit for bit across the calls.
    python bench.py --case tc_round [cg|tridiag]
        the same batch, six solve rounds launched one by one (launch list of
        a round: GEMM, pressure, friction, step control).
    python bench.py --case hmatrix_kv [n_faults box_m [tuned]]
        the 4000-fault network in 20 km x 20 km (N = 81 750; or n_faults in a
        box_m square) as an H-matrix (leaf 64, eta 2, ACA 1e-6, FP32
        factors): three K.V launches (several kernels each); "tuned" runs the
        autotuner first, "grids D W" sets the CTAs of the dense-row and
        small-leaf kernels (dfn_set_hmat_grids).
    python bench.py --case hmatrix_ensemble_kv [tuned]
        the 64 networks of the ensemble64 leg as H-matrices (leaf 64, eta 2,
        ACA 1e-7, FP32 factors) in one batch: three K.V launches of the
        batch; "tuned" runs the autotuner first (one JSON line).
    python bench.py --case s64_kv [R]
        R realisations (default 64) of the 800-fault network sharing one FP64
        kernel matrix: three K.V launches of the FP64 GEMM (4.1 GB per launch).
    python bench.py --case hmatrix_autotune
        the same network with CG pressure: the autotuner's timing of the
        stage pressure systems by one CTA each and by a cluster of CTAs each
        (one JSON line).
    python bench.py --case hmatrix_round
        the same network with shear loading (1e-9 m/s) and CG pressure: four
        solve steps launched one by one (launch list of a step: the H-matrix
        K.V kernels, the pressure solves, the stage kernel, step control).
    python bench.py --case ensemble_round
        eight 120-fault networks (FP32 storage, tridiagonal pressure), forty
        solve rounds launched one by one.

    Each case exits 0 after printing one line, so the same command can run once
    without ncu and then under it.
    """
    from demystification_dfn_b200 import networks
    from demystification_dfn_b200.ensemble import Ensemble

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
        from demystification_dfn_b200.simulation import Simulation

        nf = int(argv[1]) if len(argv) > 1 else 4000
        box = float(argv[2]) if len(argv) > 2 else 20000.0
        p = networks.fault_network(n_faults=nf, box=box, seed=0, kernel="hmatrix", tol=1e-6)
        e = Simulation(p, storage="fp32", hmat_leaf=64, hmat_eta=2.0, hmat_eps=1e-6)
        if len(argv) > 3 and argv[3] == "tuned":
            import json

            print(json.dumps(e.autotune()))
        elif len(argv) > 5 and argv[3] == "grids":
            e.set_hmat_grids(int(argv[4]), int(argv[5]))
        rng = np.random.default_rng(0)
        for _ in range(3):
            e.kernel(rng.normal(size=e.N))
    elif case == "hmatrix_ensemble_kv":
        import json

        members = networks.ensemble(64, kernel="hmatrix")
        e = Ensemble(members, storage="fp32", pressure="tridiag", hmat_leaf=64, hmat_eta=2.0, hmat_eps=1e-7)
        if len(argv) > 1 and argv[1] == "tuned":
            print(json.dumps({"kv_bytes": e.kernel_bytes, "tune": e.autotune()}))
        rng = np.random.default_rng(0)
        for _ in range(3):
            e.kernel([rng.normal(size=n) for n in e.n_elements])
    elif case == "s64_kv":
        # R realisations of the 800-fault network, FP64 shared kernel matrix:
        # three K.V launches of the FP64 GEMM (4.1 GB of K per launch)
        R = int(argv[1]) if len(argv) > 1 else 64
        base = networks.fault_network(n_faults=800, seed=0)
        e = Ensemble(networks.shared_geometry_ensemble(R, base=base, seed=0), storage="fp64_shared")
        rng = np.random.default_rng(0)
        N = e.n_elements[0]
        for _ in range(3):
            e.kernel([rng.normal(size=N) for _ in range(R)])
    elif case == "hmatrix_autotune":
        import json

        from demystification_dfn_b200.simulation import Simulation

        p = networks.fault_network(n_faults=4000, box=20000.0, seed=0, kernel="hmatrix", tol=1e-6)
        e = Simulation(p, storage="fp32", pressure="cg", hmat_leaf=64, hmat_eta=2.0, hmat_eps=1e-6)
        print(json.dumps(e.autotune()))
    elif case == "hmatrix_round":
        from demystification_dfn_b200.simulation import Simulation

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


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's own
    algorithm for the path (oracle/, the reference cannot be compiled here)
    on all host threads, on this arm's workload, metric and config."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    steps, dt, N = time_oracle_steps(make_problem(0), threads, args.warmup, args.steps, args.cpu_budget)
    v = steps / dt
    line = {
        "impl": "reference", "metric": "RK45 accepted steps/s", "value": v, "unit": "steps/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(N),
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} accepted steps of the workload after {args.warmup} warm-up steps "
                                   f"({dt:.1f} s), matrix-free directII as in the reference"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def _sig(x, n=4):
    return float(f"{x:.{n}g}") if isinstance(x, float) else x


def metric_summary(extras):
    """Small keys for the end of the line: the metric's comparison (batched
    mixed precision vs plain FP64 on the 64-network ensemble, steps/s and
    slip error), the shared-geometry tensor-core batch against its FP64
    shared-K counterpart, and the H-matrix K.V fraction of HBM."""
    out = {}
    ns = extras.get("ensemble64")
    if ns:
        keys = ("network_steps_per_s", "steps_per_s_vs_v_fp64", "time_to_t_end_vs_v_fp64", "slip_rel_err_vs_fp64",
                "kv_frac_of_measured_hbm")
        out["ensemble64"] = {name: {k: _sig(v[k], 3) for k in keys if k in v}
                             for name, v in ns.items() if isinstance(v, dict) and "network_steps_per_s" in v}
    tc = extras.get("tensor_core")
    if tc:
        out["shared_geometry64"] = {name: {k: _sig(v[k], 3) for k in ("network_steps_per_s", "kv_avg_ms",
                                                                      "slip_rel_err_vs_fp64_shared_k",
                                                                      "time_to_t_end")
                                           if k in v}
                                    for name, v in tc.items() if isinstance(v, dict) and
                                    ("network_steps_per_s" in v or "time_to_t_end" in v)}
    hm = extras.get("hmatrix")
    if hm:
        out["hmatrix_kv_frac_of_measured_hbm"] = _sig(hm.get("kv_frac_of_measured_hbm"), 3)
    return out


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "--case":
        return run_case(sys.argv[2:])
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--storage", default="fp64", choices=["fp64", "fp32", "bf16x2"])
    ap.add_argument("--pressure", default="cg", choices=["cg", "tridiag"])
    ap.add_argument("--gemv", default="tma", choices=["tma", "ldg"])
    ap.add_argument("--n-faults", type=int, default=None, help="smaller network (profiling only)")
    ap.add_argument("--no-extras", action="store_true", help="skip the mixed-precision and CPU legs")
    ap.add_argument("--ensemble", type=int, default=64, help="networks in the ensemble leg (0 = skip)")
    ap.add_argument("--ensemble-steps", type=int, default=10)
    ap.add_argument("--legs", default="precision,ensemble64,single_fault,hmatrix,tensor_core,span,learned,cpu",
                    help="comma list of the extra legs to run (ensemble, the 64 networks in three storages "
                         "sharded over the ranks; ensemble_span, the 64 networks over 1 simulated year; and "
                         "hmatrix_span, the H-matrix network toward 100 years, are available but not in the "
                         "default list)")
    ap.add_argument("--cpu-budget", "--ref-budget", dest="cpu_budget", type=float, default=60.0,
                    help="seconds of timed CPU-oracle steps (both arms)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)

    from demystification_dfn_b200.simulation import Simulation

    problem = make_problem(rank, args.n_faults)
    sim = Simulation(problem, storage=args.storage, pressure=args.pressure, device=local, gemv=args.gemv)
    stream = torch.cuda.current_stream()
    sim.set_stream(stream.cuda_stream)
    N = sim.N
    kv_bytes = sim.kernel_bytes

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up
    sim.solve_steps(args.warmup)
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    sim.profile_kv(True)
    l0 = sim.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    rep = sim.solve_steps(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    launches = sim.launches - l0
    kv_ms, kv_n = sim.profile_kv_read()
    sim.profile_kv(False)
    clk = clocks.stop()
    st_ref = sim.state()        # FP64 state after the timed steps, for the mixed-precision check
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1e3)

    # end-to-end through the C ABI with pinned host buffers every step
    st = sim.state()
    Yh = torch.from_numpy(st["Y"]).pin_memory().numpy()
    Ph = torch.from_numpy(st["P"]).pin_memory().numpy()
    outs = [torch.empty(N, dtype=torch.float64).pin_memory().numpy() for _ in range(5)]
    e2e_steps = max(10, args.steps // 2)
    tcur, ttry = st["time"], st["t_try"]
    v0_dc = np.asarray(sim.arrays.V0) / np.asarray(sim.arrays.Dc)
    psi = Yh[N:2 * N]
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        r = sim.step_host(Yh, Ph, tcur, ttry, outs)
        # next step's input is this step's result, read back on the host
        # (psi = ln(theta V0 / Dc), in place)
        Yh[:N] = outs[0]
        np.multiply(outs[1], v0_dc, out=psi)
        np.log(psi, out=psi)
        Yh[2 * N:] = outs[4]
        Ph[:] = outs[2]
        tcur, ttry = r.time, r.t_try
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * e2e_steps / float(te.item())

    extras = {}
    legs = set() if args.no_extras else set(args.legs.split(","))
    if rank == 0 and "precision" in legs:
        # mixed-precision storage of the same network (same steps, same start)
        for store in ("fp32", "bf16x2"):
            if store == args.storage:
                continue
            s2 = Simulation(problem, storage=store, pressure=args.pressure, device=local, gemv=args.gemv)
            s2.set_stream(stream.cuda_stream)
            s2.solve_steps(args.warmup)
            torch.cuda.synchronize()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            s2.solve_steps(args.steps)
            a1.record(stream)
            torch.cuda.synchronize()
            st2 = s2.state()
            Vr, V2 = st_ref["Y"][:N], st2["Y"][:N]
            pr, p2 = st_ref["Y"][N:2 * N], st2["Y"][N:2 * N]
            extras[store] = {"steps_per_s": args.steps / (a0.elapsed_time(a1) / 1e3),
                             "kv_bytes": s2.kernel_bytes,
                             "kv_ms": s2.time_kernel(10),
                             "rel_err_V_vs_fp64": float(np.abs(V2 - Vr).max() / np.abs(Vr).max()),
                             "rel_err_psi_vs_fp64": float(np.abs(p2 - pr).max() / np.abs(pr).max()),
                             "rel_err_time_vs_fp64": abs(st2["time"] - st_ref["time"]) / st_ref["time"],
                             "compared_after": f"{args.warmup}+{args.steps} accepted steps from the same start"}
            s2.close()

    if args.ensemble > 0 and "ensemble" in legs:
        # batched ensemble: many networks of uneven size in one handle, one
        # launch per kernel for the whole batch, per-network step control;
        # with several ranks each rank takes its share of the networks
        # (placed by K.V bytes) and the throughput is the job's
        from demystification_dfn_b200 import networks
        from demystification_dfn_b200.ensemble import Ensemble
        from demystification_dfn_b200.layout import build_arrays
        from demystification_dfn_b200.sharding import reduce_timing, shard_by_work

        allm = networks.ensemble(args.ensemble)
        sizes = [build_arrays(p).N for p in allm]
        members = [allm[i] for i in shard_by_work(sizes, world, rank)]
        hbm, _ = peaks()
        ens_out = {"networks": len(allm), "steps_per_network": args.ensemble_steps, "ranks": world,
                   "placement": "networks sharded over ranks by K.V bytes"}
        for store in ("fp64", "fp32", "bf16x2"):
            ens = Ensemble(members, storage=store, pressure=args.pressure, device=local, gemv=args.gemv)
            ens.set_stream(stream.cuda_stream)
            tune = ens.autotune()
            ens.solve(n_steps=3)
            torch.cuda.synchronize()
            ens.profile_kv(True)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            reps = ens.solve(n_steps=args.ensemble_steps, check=False)
            a1.record(stream)
            torch.cuda.synchronize()
            kms, kn = ens.profile_kv_read()
            ms_local = a0.elapsed_time(a1)
            ms_e, work = reduce_timing(ms_local, len(members) * args.ensemble_steps,
                                       dist=dist if world > 1 else None, device="cuda")
            done = sum(1 for r in reps if r["status"] == 0)
            kavg = kms / max(kn, 1)
            gbs = ens.kernel_bytes / (kavg / 1e3) / 1e9
            ens_out[store] = {"steps_per_s": work / (ms_e / 1e3),
                              "ms_per_round_avg": ms_e / max(kn // 6, 1), "networks_ok": done,
                              "elements_on_rank0": int(sum(ens.n_elements)), "kv_bytes_rank0": ens.kernel_bytes,
                              "kv_avg_ms": kavg, "kv_GBps": gbs, "kv_frac_of_measured_hbm": gbs / hbm,
                              "rejected": int(sum(r["rejected"] for r in reps)),
                              "probe_halvings": int(sum(r["probe_halvings"] for r in reps)),
                              "stage_cg_failures": int(sum(r["stage_cg_failures"] for r in reps)),
                              "autotune": tune,
                              "status_counts": {str(s): sum(1 for r in reps if r["status"] == s)
                                                for s in sorted({r["status"] for r in reps})}}
            if store == "fp64":
                ref_states = [ens.state(i) for i in range(len(members))]
            else:
                err = 0.0
                for i in range(len(members)):
                    s_i = ens.state(i)
                    n_i = len(s_i["P"])
                    v_ref = ref_states[i]["Y"][:n_i]
                    err = max(err, float(np.abs(s_i["Y"][:n_i] - v_ref).max() / np.abs(v_ref).max()))
                ens_out[store]["max_rel_err_V_vs_fp64"] = err
            ens.close()
        extras["ensemble"] = ens_out

    if rank == 0 and "single_fault" in legs:
        extras["single_fault"] = leg_single_fault(args, local, stream)
    if rank == 0 and "hmatrix" in legs:
        extras["hmatrix"] = leg_hmatrix(args, local, stream)
    if rank == 0 and "tensor_core" in legs:
        extras["tensor_core"] = leg_tensor_core(args, local, stream)
    if rank == 0 and "span" in legs:
        extras["span"] = leg_span(args, local, stream)
    if rank == 0 and "ensemble_span" in legs:
        extras["ensemble_span"] = leg_ensemble_span(args, local, stream)
    if rank == 0 and "hmatrix_span" in legs:
        extras["hmatrix_span"] = leg_hmatrix_span(args, local, stream)
    if rank == 0 and "learned" in legs:
        extras["learned_newton"] = leg_learned(args, local, stream)
    if rank == 0 and "ensemble64" in legs:
        extras["ensemble64"] = leg_ensemble64(args, local, stream)

    if rank == 0:
        hbm, src = peaks()
        kv_avg = kv_ms / max(kv_n, 1)
        achieved = kv_bytes / (kv_avg / 1e3) / 1e9
        cpu = None
        if "cpu" in legs and world == 1:
            # the reference arm's sample: the same warm-up, step count and
            # budget on all host threads
            threads = os.cpu_count() or 1
            steps_c, dt_c, _ = time_oracle_steps(make_problem(0, args.n_faults), threads, args.warmup, args.steps,
                                                 args.cpu_budget)
            cpu = {"value": steps_c / dt_c, "unit": "steps/s", "cores": threads, "kind": "port",
                   "sample": f"{steps_c} accepted steps of the workload after {args.warmup} warm-up steps "
                             f"({dt_c:.1f} s), matrix-free directII as in the reference"}
            # one core (the reference's own build is serial): right-hand
            # sides per second, measured (not an extrapolated step rate)
            t1 = cpu_rhs_seconds(make_problem(0, args.n_faults), 1)
            cpu["rhs_evals_per_s_1core"] = 1.0 / t1
            cpu["gpu_rhs_evals_per_accepted_step"] = rep["rhs_evals"] / max(rep["it_count"], 1)
        line = {
            "metric": "RK45 accepted steps/s", "value": value, "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": bench_config(N),
            "impl_options": {"kernel_storage": args.storage, "pressure_solver": args.pressure, "kv_impl": args.gemv},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic_per_launch(args.storage),
                         "peak_source": src, "kernel": "K.V stream (%s)" % args.gemv,
                         "algorithmic_bytes_per_launch": kv_bytes, "avg_launch_ms": kv_avg,
                         "launches_timed": kv_n},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 8 * 4 * N + 16,
                    "d2h_bytes_per_step": 8 * 5 * N},
            "gpu_launches": launches,
            "clocks": clk,
            "report": {k: rep[k] for k in ("attempts", "rejected", "rhs_evals", "cg_iterations", "probe_halvings",
                                           "time")},
        }
        if extras:
            line["extras"] = extras
        # the compact summary goes last: the tail of a long line is what a
        # truncated log keeps
        summary = metric_summary(extras)
        if summary:
            line["summary"] = summary
        print(json.dumps(line))
    sim.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
