"""numpy FP64 oracle of the learned-guess MLP (test infrastructure only).

Forward pass and backward pass of the 7 -> 64 -> 64 -> 1 SiLU network with
the flat weight layout of include/dfn_b200.h, and the mean squared error.
The network has no counterpart in the reference; this oracle checks the
GPU training kernels' loss and gradients (and is itself checked against
finite differences in tests/test_oracle.py).
"""
import numpy as np

N_IN, N_H = 7, 64


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    W1 = w[o:o + N_IN * N_H].reshape(N_IN, N_H); o += N_IN * N_H
    b1 = w[o:o + N_H]; o += N_H
    W2 = w[o:o + N_H * N_H].reshape(N_H, N_H); o += N_H * N_H
    b2 = w[o:o + N_H]; o += N_H
    W3 = w[o:o + N_H]; o += N_H
    b3 = w[o]
    return W1, b1, W2, b2, W3, b3


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(w, x):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    z1 = x @ W1 + b1
    h1 = silu(z1)
    z2 = h1 @ W2 + b2
    h2 = silu(z2)
    return h2 @ W3 + b3, (x, z1, h1, z2, h2)


def loss_grad(w, x, t):
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(w)
    out, (x, z1, h1, z2, h2) = forward(w, x)
    n = len(t)
    d = out - t
    loss = float(np.mean(d * d))
    dout = 2.0 * d / n
    gW3 = h2.T @ dout
    gb3 = dout.sum()
    d2 = np.outer(dout, W3) * dsilu(z2)
    gW2 = h1.T @ d2
    gb2 = d2.sum(axis=0)
    d1 = (d2 @ W2.T) * dsilu(z1)
    gW1 = x.T @ d1
    gb1 = d1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g
