"""FP64 numpy restatement of the learned insertion proposal's network — TEST INFRASTRUCTURE ONLY.

Checks the device kernels' forward values and gradients. The network has no counterpart in RASPA3; it plugs into the
uniform first-bead sampling of CBMC::growMoleculeMultipleFirstBeadSwapInsertion (src/raspakit/cbmc/
multiple_first_bead.cpp:23-27).

Features: for each fractional coordinate s_a (a = x, y, z) and n = 1..16, sin(2 pi n s_a) and cos(2 pi n s_a), ordered
feature[32 a + 2 (n - 1) + 0] = sin, feature[32 a + 2 (n - 1) + 1] = cos (96 inputs).
Network: h1 = silu(W1 phi + b1) (64), h2 = silu(W2 h1 + b2) (64), f = w3 . h2 + b3 (the log-density, unnormalised).
Loss over a batch: L = (1 / B) sum_i weight_i (f(s_i) - target_i)^2.
Parameter vector order: W1 (64 x 96, row-major), b1 (64), W2 (64 x 64, row-major), b2 (64), w3 (64), b3 (1).
"""

from __future__ import annotations

import numpy as np

N_IN, N_H = 96, 64
N_PARAMS = N_H * N_IN + N_H + N_H * N_H + N_H + N_H + 1


def unpack(theta):
    theta = np.asarray(theta, dtype=np.float64)
    o = 0
    W1 = theta[o:o + N_H * N_IN].reshape(N_H, N_IN); o += N_H * N_IN
    b1 = theta[o:o + N_H]; o += N_H
    W2 = theta[o:o + N_H * N_H].reshape(N_H, N_H); o += N_H * N_H
    b2 = theta[o:o + N_H]; o += N_H
    w3 = theta[o:o + N_H]; o += N_H
    b3 = theta[o]
    return W1, b1, W2, b2, w3, b3


def features(s):
    s = np.asarray(s, dtype=np.float64).reshape(-1, 3)
    n = np.arange(1, 17, dtype=np.float64)
    out = np.empty((len(s), N_IN))
    for a in range(3):
        arg = 2.0 * np.pi * s[:, a:a + 1] * n[None, :]
        out[:, 32 * a + 0:32 * a + 32:2] = np.sin(arg)
        out[:, 32 * a + 1:32 * a + 32:2] = np.cos(arg)
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    sg = 1.0 / (1.0 + np.exp(-z))
    return sg * (1.0 + z * (1.0 - sg))


def forward(theta, s):
    W1, b1, W2, b2, w3, b3 = unpack(theta)
    phi = features(s)
    z1 = phi @ W1.T + b1
    h1 = silu(z1)
    z2 = h1 @ W2.T + b2
    h2 = silu(z2)
    return h2 @ w3 + b3


def loss_and_grad(theta, s, target, weight=None):
    W1, b1, W2, b2, w3, b3 = unpack(theta)
    phi = features(s)
    B = len(phi)
    w = np.ones(B) if weight is None else np.asarray(weight, dtype=np.float64)
    z1 = phi @ W1.T + b1
    h1 = silu(z1)
    z2 = h1 @ W2.T + b2
    h2 = silu(z2)
    f = h2 @ w3 + b3
    r = f - np.asarray(target, dtype=np.float64)
    loss = float(np.sum(w * r * r) / B)
    df = 2.0 * w * r / B
    g_w3 = h2.T @ df
    g_b3 = df.sum()
    dz2 = (df[:, None] * w3[None, :]) * dsilu(z2)
    g_W2 = dz2.T @ h1
    g_b2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * dsilu(z1)
    g_W1 = dz1.T @ phi
    g_b1 = dz1.sum(0)
    grad = np.concatenate([g_W1.ravel(), g_b1, g_W2.ravel(), g_b2, g_w3, [g_b3]])
    return loss, grad
