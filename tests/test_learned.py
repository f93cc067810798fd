"""The learned Newton guess: oracle gradients (CPU) and, on the GPU, the
training kernels, the Newton formulation, and what the guess saves."""
import numpy as np
import pytest

import mlp_oracle
from demystification_dfn_b200 import learned, networks


def _samples(n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, 7)).astype(np.float32)
    t = (np.sin(x[:, 0]) * 0.5 - 0.2 * x[:, 3] ** 2).astype(np.float32)
    return x, t


def test_mlp_oracle_gradient_matches_finite_differences():
    x, t = _samples(64)
    w = learned.init_weights(1).astype(np.float64)
    _, g = mlp_oracle.loss_grad(w, x, t)
    rng = np.random.default_rng(2)
    for p in rng.choice(len(w), 25, replace=False):
        e = np.zeros_like(w)
        e[p] = 1e-6
        fd = (mlp_oracle.loss_grad(w + e, x, t)[0] - mlp_oracle.loss_grad(w - e, x, t)[0]) / 2e-6
        assert abs(fd - g[p]) <= 1e-6 + 1e-5 * abs(g[p])


@pytest.mark.gpu
def test_gpu_mlp_loss_and_gradient_match_oracle():
    x, t = _samples(1000, 3)
    w = learned.init_weights(4)
    loss, g = learned.loss_grad(x, t, w)
    ol, og = mlp_oracle.loss_grad(w, x, t)
    assert abs(loss - ol) <= 1e-5 * abs(ol)
    assert np.abs(g - og).max() <= 1e-4 * np.abs(og).max()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 31, 1000])
def test_gpu_mlp_tensor_core_inference_matches_oracle(n):
    """The friction kernel's inference path (FP16 operands, FP32
    accumulation) against the FP64 forward pass; ragged row counts leave
    lanes of the last warp without a row."""
    x, _ = _samples(n, 7)
    w = learned.init_weights(8)
    y = learned.infer(x, w)
    ref = mlp_oracle.forward(w, x.astype(np.float64))[0]
    assert np.abs(y - ref).max() <= 1e-2 * np.abs(ref).max() + 1e-3


@pytest.mark.gpu
def test_gpu_mlp_training_reduces_loss():
    x, t = _samples(20000, 5)
    w, loss = learned.train(x, t, epochs=15, batch=2048, lr=3e-3, seed=1)
    assert loss[1] < 0.2 * loss[0]
    l2, _ = mlp_oracle.loss_grad(w, x, t)
    assert l2 < 0.2 * float(np.mean(t.astype(np.float64) ** 2))


def _net(seed=31, **kw):
    return networks.small_network(seed=seed, n_faults=4, tol=1e-8, **kw)


@pytest.mark.gpu
def test_newton_formulation_reproduces_initial_velocity():
    from demystification_dfn_b200.simulation import Simulation

    p = _net()
    with Simulation(p, formulation="newton", pressure="tridiag") as s:
        V = s.velocity()
        V0 = s.arrays.V
        real = ~s.arrays.fake_mask
        assert np.abs(V[real] - V0[real]).max() <= 1e-10 * np.abs(V0[real]).max()


@pytest.mark.gpu
def test_newton_formulation_matches_v_formulation():
    """Without pore-pressure forcing both formulations integrate the same ODE
    (the V formulation is the time derivative of the friction law); at the
    same final time (runs land on t_end) slip rate and log-state agree to
    1e-6. With a diffusing pressure they differ at O(h): the reference's
    V formulation uses the secant (P_temp - P)/dt for dP/dt and the pressure
    at t_try for its first stage, the Newton formulation uses P_temp itself."""
    from demystification_dfn_b200.simulation import Simulation

    p = _net(dP=0.0)
    t_end = 5000.0
    with Simulation(p, formulation="v", pressure="tridiag") as a, \
            Simulation(p, formulation="newton", pressure="tridiag") as b:
        a.solve_to(t_end)
        rb = b.solve_to(t_end)
        assert rb["status"] == 0 and rb["newton_fail"] == 0
        sa, sb = a.state(), b.state()
        assert abs(sa["time"] - sb["time"]) <= 1e-12 * t_end
        N = a.N
        Va, Vb = sa["Y"][:N], b.velocity()
        assert np.abs(Vb - Va).max() <= 1e-6 * np.abs(Va).max()
        pa, pb = sa["Y"][N:2 * N], sb["Y"][N:2 * N]
        assert np.abs(pb - pa).max() <= 1e-6 * np.abs(pa).max()


@pytest.mark.gpu
def test_learned_guess_saves_newton_iterations():
    """Record solves on states spanning slow and fast slip, train on the GPU,
    then evaluate new states from three starts: the quasi-static root w0
    (radiation damping neglected), the bounded analytic start min(w0, wr)
    and the learned correction on top of it. All roots agree to the Newton
    tolerance; the learned guess needs fewer iterations than the quasi-static
    start and no more than the bounded one (which already brings most solves
    to a single iteration, below what an FP32 guess can improve on)."""
    from demystification_dfn_b200.simulation import Simulation

    p = _net(seed=33)
    rng = np.random.default_rng(0)

    def states(s, n):
        N = s.N
        Y0 = s.state()["Y"]
        out = []
        for _ in range(n):
            Y = Y0.copy()
            # slip perturbations drive the stress (and V) over many decades,
            # up to fast slip (~1 m/s) where radiation damping matters
            Y[:N] = rng.normal(0.0, 10 ** rng.uniform(-5, -2.6), N)
            Y[:N][s.arrays.fake_mask] = 0.0
            Y[N:2 * N] += rng.normal(0.0, 0.5, N)
            out.append(Y)
        return out

    with Simulation(p, formulation="newton", pressure="tridiag") as s:
        s.record(200000)
        for Y in states(s, 1500):
            s.friction_law(1.0, Y)
        x, t = s.record_read(200000)
    assert len(t) > 10000
    w, loss = learned.train(x, t, epochs=40, batch=2048, lr=2e-3, seed=0)
    assert loss[1] < loss[0]
    test_states = None
    res = {}
    for guess in ("quasistatic", "analytic", "mlp"):
        with Simulation(p, formulation="newton", pressure="tridiag", guess=guess) as s:
            if guess == "mlp":
                s.set_mlp(w)
            if test_states is None:
                test_states = states(s, 50)
            before = s.report()
            outs = [s.friction_law(1.0, Y) for Y in test_states]
            after = s.report()
            res[guess] = (after["newton_iters"] - before["newton_iters"],
                          after["newton_solves"] - before["newton_solves"], outs)
            assert after["newton_fail"] == before["newton_fail"], guess
    iq, nq, oq = res["quasistatic"]
    ia, na, oa = res["analytic"]
    im, nm, om = res["mlp"]
    assert nq == na == nm
    assert im < iq and ia < iq
    assert im <= ia
    for yq, ya, ym in zip(oq, oa, om):
        N = len(ya) // 3
        assert np.abs(ym[:N] - ya[:N]).max() <= 1e-9 * np.abs(ya[:N]).max()
        assert np.abs(yq[:N] - ya[:N]).max() <= 1e-9 * np.abs(ya[:N]).max()
