"""The allocation-free pressure step against the handle-based one.

dfn_compute_P_noalloc exists for callers that must not allocate device
memory (a host program whose pool allocator owns all device memory, or a
time loop that cannot take the device-wide synchronisation of cudaMalloc /
cudaFree). It keeps its CG work vectors in a fixed array inside the library.
This test allocates the inputs and outputs itself (the entry point never
does), calls the entry point twice in a row through the C ABI and compares
each result with dfn_compute_P on the same problem, within the tolerance of
the other pressure tests (both stop CG at max|r| < tol_solver).

The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from demystification_dfn_b200 import networks
from demystification_dfn_b200._lib import load

pytestmark = pytest.mark.gpu

TOL = 1e-6
MAX = 65536   # DFN_NOALLOC_MAX_ELEMENTS


def _device_inputs(arrays, torch):
    N = arrays.N
    node = arrays.node
    dx, dy = node[1:, 0] - node[:-1, 0], node[1:, 1] - node[:-1, 1]
    ds = np.sqrt(dx * dx + dy * dy)
    p = arrays.permeability
    permx = np.zeros(N + 1)
    permx[1:N] = 2.0 * p[:-1] * p[1:] / (p[:-1] + p[1:])
    first = arrays.fault_first
    src_elem = np.array([first[f - 1] + i - 1 for f, i in zip(arrays.src_fault, arrays.src_index)], dtype=np.int64)

    def dev(a, dtype):
        return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")

    return {
        "P": dev(arrays.P, torch.float64), "permx": dev(permx, torch.float64), "ds": dev(ds, torch.float64),
        "src_fault": dev(arrays.src_fault, torch.int64), "src_elem": dev(src_elem, torch.int64),
        "Q": dev(arrays.src_Q, torch.float64), "tb": dev(arrays.src_t_beg, torch.float64),
        "te": dev(arrays.src_t_end, torch.float64),
    }


def _call(lib, arrays, d, dt, Pt, Pd, torch, N=None, tol=None):
    ier = ctypes.c_int32(-1)
    a = arrays
    st = lib.dfn_compute_P_noalloc(
        a.N if N is None else N, dt, a.time0, d["P"].data_ptr(), d["permx"].data_ptr(), d["ds"].data_ptr(),
        a.porosity, a.dyn_viscosity, a.fluid_comp, a.rock_comp, a.tol_solver if tol is None else tol,
        len(a.src_fault),
        d["src_fault"].data_ptr(), d["src_elem"].data_ptr(), d["Q"].data_ptr(), d["tb"].data_ptr(),
        d["te"].data_ptr(), Pt.data_ptr(), Pd.data_ptr(), ctypes.byref(ier),
        torch.cuda.current_stream().cuda_stream)
    return st, ier.value


def test_noalloc_pressure_matches_handle_entry_point():
    import torch
    from demystification_dfn_b200.simulation import Simulation

    lib = load()
    p = networks.single_fault(n_el=300, length=3000.0, mode="modeIII", tol=TOL)
    with Simulation(p, pressure="cg") as sim:
        a = sim.arrays
        d = _device_inputs(a, torch)
        Pt = torch.zeros(a.N, dtype=torch.float64, device="cuda")
        Pd = torch.zeros(a.N, dtype=torch.float64, device="cuda")
        # two calls in a row: the shared scratch keeps the previous call's
        # contents, the second call must not depend on them
        for dt in (100.0, 5000.0):
            st, ier = _call(lib, a, d, dt, Pt, Pd, torch)
            assert st == 0 and ier == 0
            ref_P, ref_Pd, ref_ier = sim.compute_P(dt)
            assert ref_ier == 0
            assert np.abs(Pt.cpu().numpy() - ref_P).max() < 1e3 * TOL
            assert np.abs(Pd.cpu().numpy() - ref_Pd).max() < 1e3 * TOL / dt


def test_noalloc_rejects_oversized_problem():
    import torch

    lib = load()
    p = networks.single_fault(n_el=64, length=640.0, mode="modeIII", tol=TOL)
    from demystification_dfn_b200 import build_arrays

    a = build_arrays(p)
    d = _device_inputs(a, torch)
    Pt = torch.zeros(a.N, dtype=torch.float64, device="cuda")
    Pd = torch.zeros(a.N, dtype=torch.float64, device="cuda")
    for n in (70000, MAX + 1):
        st, _ = _call(lib, a, d, 10.0, Pt, Pd, torch, N=n)
        assert st == 5
        assert b"DFN_NOALLOC_MAX_ELEMENTS" in lib.dfn_last_error()


def test_noalloc_iteration_cap_leaves_outputs_untouched():
    """A tolerance no CG iterate can meet: after 200 iterations the call
    reports ier = 1 and leaves both outputs as they were (the reference's
    compute_P returns before writing them), on two calls in a row."""
    import torch

    lib = load()
    p = networks.single_fault(n_el=300, length=3000.0, mode="modeIII", tol=TOL)
    from demystification_dfn_b200 import build_arrays

    a = build_arrays(p)
    d = _device_inputs(a, torch)
    for dt in (5000.0, 86400.0):
        Pt = torch.full((a.N,), 123.25, dtype=torch.float64, device="cuda")
        Pd = torch.full((a.N,), -7.5, dtype=torch.float64, device="cuda")
        st, ier = _call(lib, a, d, dt, Pt, Pd, torch, tol=1e-300)
        assert st == 0 and ier == 1
        assert bool((Pt == 123.25).all()) and bool((Pd == -7.5).all())


def test_noalloc_at_the_maximum_size_matches_oracle():
    """N = DFN_NOALLOC_MAX_ELEMENTS (one 655 km fault of 10 m elements with
    injection at its centre): every grid-stride loop of the one-CTA solver
    and the whole scratch area are used. Checked against the oracle's CG
    (a handle would assemble a 69 GB dense kernel at this size), then the
    same call again."""
    import torch
    from oracle import Oracle

    lib = load()
    p = networks.single_fault(n_el=MAX, length=10.0 * MAX, mode="modeIII", tol=TOL)
    from demystification_dfn_b200 import build_arrays

    a = build_arrays(p)
    assert a.N == MAX
    d = _device_inputs(a, torch)
    o = Oracle(a)
    dt = 100.0
    ref_P, ref_Pd, ref_ier = o.compute_P(dt)
    o.close()
    assert ref_ier == 0
    for _ in range(2):
        Pt = torch.zeros(a.N, dtype=torch.float64, device="cuda")
        Pd = torch.zeros(a.N, dtype=torch.float64, device="cuda")
        st, ier = _call(lib, a, d, dt, Pt, Pd, torch)
        assert st == 0 and ier == 0
        assert np.abs(Pt.cpu().numpy() - ref_P).max() < 1e3 * TOL
        assert np.abs(Pd.cpu().numpy() - ref_Pd).max() < 1e3 * TOL / dt
