"""The learned initial guess of the friction Newton solve.

A small FP32 MLP (7 -> 64 -> 64 -> 1, SiLU) predicts the correction from the
bounded analytic start wa (the friction-only root w0 = tau/(sigma_eff a) or
the radiation-only root, whichever is nearer zero) to the friction-law root
w = asinh(V C/(2 V0)). It is trained on solves that the
Newton formulation records while it runs, by the library's own GPU forward
and backward kernels (dfn_mlp_train); the Newton solve stays the judge: a
guess only sets the starting point, convergence is tested on the FP64
residual. See include/dfn_b200.h for the inputs and the weight layout.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

N_IN, N_H = 7, 64
N_PARAMS = N_IN * N_H + N_H + N_H * N_H + N_H + N_H + 1   # 4737


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def init_weights(seed=0):
    """Seeded Glorot-uniform weights, zero biases, flat DFN_MLP_PARAMS array."""
    rng = np.random.default_rng(seed)

    def glorot(fan_in, fan_out):
        lim = np.sqrt(6.0 / (fan_in + fan_out))
        return rng.uniform(-lim, lim, size=(fan_in, fan_out))

    w = np.concatenate([glorot(N_IN, N_H).ravel(), np.zeros(N_H), glorot(N_H, N_H).ravel(), np.zeros(N_H),
                        glorot(N_H, 1).ravel() * 0.1, np.zeros(1)])
    return w.astype(np.float32)


def train(x, t, weights=None, epochs=20, batch=4096, lr=2e-3, seed=0):
    """Train on (x [n,7], t [n]) with the GPU kernels; returns (weights, loss first/last epoch)."""
    lib = _lib.load()
    x = np.ascontiguousarray(x, dtype=np.float32)
    t = np.ascontiguousarray(t, dtype=np.float32)
    w = init_weights(seed) if weights is None else np.array(weights, dtype=np.float32, copy=True)
    loss = np.zeros(2, dtype=np.float32)
    _lib.check(lib.dfn_mlp_train(_fp(x), _fp(t), len(t), _fp(w), int(epochs), int(batch), float(lr),
                                 int(seed), _fp(loss)), lib)
    return w, loss


def loss_grad(x, t, weights):
    """Mean squared error and its gradient, computed by the GPU kernels."""
    lib = _lib.load()
    x = np.ascontiguousarray(x, dtype=np.float32)
    t = np.ascontiguousarray(t, dtype=np.float32)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    g = np.zeros(N_PARAMS, dtype=np.float32)
    _lib.check(lib.dfn_mlp_loss_grad(_fp(x), _fp(t), len(t), _fp(w), _fp(loss), _fp(g)), lib)
    return float(loss[0]), g


def infer(x, weights):
    """Network outputs for rows x [n, 7] by the friction kernel's inference
    path (FP16 tensor-core MMAs, FP32 accumulation)."""
    lib = _lib.load()
    x = np.ascontiguousarray(x, dtype=np.float32)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    y = np.zeros(len(x), dtype=np.float32)
    _lib.check(lib.dfn_mlp_infer(_fp(x), len(x), _fp(w), _fp(y)), lib)
    return y
