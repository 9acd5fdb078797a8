"""Test infrastructure: FP64 numpy restatement of the learned con2prim guess
(the checker for the CUDA training and inference kernels).

Network: x (3) -> 64 ReLU -> 64 ReLU -> 1, on the features of a conservative
state U = (D, S, E):  f = (log(Q/tau), log max(|S|/tau, 1e-30), log(tau/D)),
tau = E - D, Q = E - sqrt(|S|^2 + D^2), normalised as (f - mu) / sigma; the output y predicts
t = (log(p/tau) - mu_t) / sigma_t, and the guess is p0 = tau exp(y sigma_t + mu_t).
The reference has no learned part; the Newton solve it seeds is
rhllc::GetPhysValueStab (solvers/rhllc/src/rhllc_flux_stab.cpp:123-220).

Parameter vector layout (4481 floats): W1 [64][3], b1 [64], W2 [64][64] (row = output
neuron), b2 [64], W3 [64], b3 [1].
"""
from __future__ import annotations

import numpy as np

H = 64
N_PARAMS = H * 3 + H + H * H + H + H + 1


def unpack(theta):
    theta = np.asarray(theta, np.float64)
    o = 0
    W1 = theta[o:o + H * 3].reshape(H, 3); o += H * 3
    b1 = theta[o:o + H]; o += H
    W2 = theta[o:o + H * H].reshape(H, H); o += H * H
    b2 = theta[o:o + H]; o += H
    W3 = theta[o:o + H]; o += H
    b3 = theta[o]
    return W1, b1, W2, b2, W3, b3


def features(U):
    U = np.asarray(U, np.float64)
    D = U[:, 0]
    E = U[:, 4]
    tau = E - D
    m2 = (U[:, 1] * U[:, 1] + U[:, 2] * U[:, 2]) + U[:, 3] * U[:, 3]
    S = np.sqrt(m2)
    Q = E - np.sqrt(m2 + D * D)
    f = np.stack([np.log(Q / tau), np.log(np.maximum(S / tau, 1e-30)), np.log(tau / D)], 1)
    return f, tau


def forward(theta, x):
    W1, b1, W2, b2, W3, b3 = unpack(theta)
    a1 = x @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    y = h2 @ W3 + b3
    return y, (a1, h1, a2, h2)


def loss_and_grad(theta, x, t, n_total=None):
    """Mean squared error over the batch (divided by n_total if given) and its gradient."""
    W1, b1, W2, b2, W3, b3 = unpack(theta)
    y, (a1, h1, a2, h2) = forward(theta, x)
    n = n_total or len(x)
    r = y - t
    loss = (r ** 2).sum() / n
    dy = 2.0 * r / n
    dW3 = h2.T @ dy
    db3 = dy.sum()
    da2 = np.outer(dy, W3) * (a2 > 0)
    dW2 = da2.T @ h1
    db2 = da2.sum(0)
    dh1 = da2 @ W2
    da1 = dh1 * (a1 > 0)
    dW1 = da1.T @ x
    db1 = da1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3, [db3]])
    return loss, g
