"""CPU checks of the oracle's restatement of the reference H-matrix
(src/hmatrix/*): cluster tree, block partition, full-pivot ACA."""
import numpy as np

from oracle import Oracle
from demystification_dfn_b200 import networks


def test_cluster_order_is_a_permutation_and_leaves_tile_the_matrix():
    p = networks.fault_network(n_faults=30, box=1200.0, seed=4, kernel="hmatrix")
    o = Oracle(p)
    o.use_hmatrix(leaf=16, eta=2.0, eps=1e-6)
    perm = o.hmat_perm()
    assert sorted(perm.tolist()) == list(range(o.N))
    st = o.hmat_stats()
    assert st["clusters"] % 2 == 1          # binary tree: 1 + 2 * splits
    assert st["leaves"] > st["dense_leaves"] > 0


def test_hmatrix_kv_approximates_dense():
    p = networks.fault_network(n_faults=25, box=1000.0, seed=6, kernel="hmatrix")
    o = Oracle(p)
    v = np.random.default_rng(0).normal(size=o.N)
    o.use_dense()
    dT, dN = o.kernel(v)
    for eps in (1e-4, 1e-8):
        o.use_hmatrix(leaf=16, eta=2.0, eps=eps)
        hT, hN = o.kernel(v)
        assert np.abs(hT - dT).max() <= 20 * eps * np.abs(dT).max()
        assert np.abs(hN - dN).max() <= 20 * eps * np.abs(dN).max()


def test_mode3_single_fault_hmatrix():
    p = networks.single_fault(n_el=600, length=6000.0, mode="modeIII", kernel="hmatrix")
    o = Oracle(p)
    v = np.random.default_rng(1).normal(size=o.N)
    o.use_dense()
    dT, _ = o.kernel(v)
    assert o.use_hmatrix(leaf=32, eta=3.0, eps=1e-8)
    hT, _ = o.kernel(v)
    assert np.abs(hT - dT).max() <= 1e-6 * np.abs(dT).max()
