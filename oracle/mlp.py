"""Test infrastructure: a float64 numpy statement of the exchange control-variate network and of
the multi-fidelity estimator, the comparison standard for safire_b200/csrc/mlp.cu.

Network (no reference counterpart): standardised features xn = (x - mean) * istd, then
z1 = xn W1^T + b1, a1 = gelu(z1), z2 = a1 W2^T + b2, a2 = gelu(z2), y = a2 . w3 + b3 in
standardised target units; prediction = y * y_std + y_mean.  Loss = mean Huber(y - tn) with
tn = (t - y_mean) / y_std and threshold HUBER (r^2 / 2 inside, HUBER (|r| - HUBER / 2) outside).
Parameters are one flat block [W1 | b1 | W2 | b2 | w3 | b3].

Estimator: with exact values e_s on a uniform random subset S (|S| = k, without replacement) of
the W walkers and predictions f_w on all of them, the weighted sum sum_w omega_w e_w is estimated
by sum_w omega_w f_w + (W / k) sum_{s in S} omega_s (e_s - f_s), unbiased over S for any f.
"""
from __future__ import annotations

import math

import numpy as np

HUBER = 2.0


def _huber(r):
    a = np.abs(r)
    loss = np.where(a <= HUBER, 0.5 * r * r, HUBER * (a - 0.5 * HUBER))
    return np.mean(loss), np.clip(r, -HUBER, HUBER) / r.size


def split_params(p, D, H):
    o = 0
    W1 = p[o:o + H * D].reshape(H, D); o += H * D
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o:o + 1]
    return W1, b1, W2, b2, w3, b3


def _erf(x):
    return np.vectorize(math.erf)(x)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


def forward(p, X, D, H, mean, istd):
    W1, b1, W2, b2, w3, b3 = split_params(np.asarray(p, np.float64), D, H)
    xn = (np.asarray(X, np.float64) - mean) * istd
    z1 = xn @ W1.T + b1
    a1 = gelu(z1)
    z2 = a1 @ W2.T + b2
    a2 = gelu(z2)
    y = a2 @ w3 + b3[0]
    return y, (xn, z1, a1, z2, a2)


def predict(p, X, D, H, mean, istd, y_mean, y_std):
    return forward(p, X, D, H, mean, istd)[0] * y_std + y_mean


def loss_and_grad(p, X, t, D, H, mean, istd, y_mean, y_std):
    """Loss mean((y - tn)^2) / 2 and its gradient with respect to the flat parameters."""
    W1, b1, W2, b2, w3, b3 = split_params(np.asarray(p, np.float64), D, H)
    y, (xn, z1, a1, z2, a2) = forward(p, X, D, H, mean, istd)
    B = y.size
    r = y - (np.asarray(t, np.float64) - y_mean) / y_std
    loss, dy = _huber(r)
    dw3 = a2.T @ dy
    db3 = np.array([dy.sum()])
    dz2 = np.outer(dy, w3) * gelu_grad(z2)
    dW2 = dz2.T @ a1
    db2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * gelu_grad(z1)
    dW1 = dz1.T @ xn
    db1 = dz1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dw3, db3])
    return loss, g


def multifidelity_sum(omega, f, exact_subset, subset):
    """sum_w omega_w f_w + (W / k) sum_{s in subset} omega_s (e_s - f_s)."""
    omega = np.asarray(omega)
    f = np.asarray(f)
    subset = np.asarray(subset)
    W, k = omega.size, subset.size
    return np.sum(omega * f) + (W / k) * np.sum(omega[subset] * (np.asarray(exact_subset) - f[subset]))


def bf16(x):
    """Round to bfloat16 (nearest, ties to even) and back to float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def loss_and_grad_bf16(p, X, t, D, H, mean, istd, y_mean, y_std):
    """The network with the GPU kernels' rounding points (standardised features, weight matrices,
    activations and backward signals rounded to bfloat16; sums in float64): prediction y in
    standardised units, loss and flat gradient."""
    W1, b1, W2, b2, w3, b3 = split_params(np.asarray(p, np.float32).astype(np.float64), D, H)
    xn = bf16((np.asarray(X, np.float32) - np.float32(mean)) * np.float32(istd)).astype(np.float64)
    W1b, W2b = bf16(W1).astype(np.float64), bf16(W2).astype(np.float64)
    z1 = xn @ W1b.T + b1
    a1 = bf16(gelu(z1)).astype(np.float64)
    z2 = a1 @ W2b.T + b2
    a2 = bf16(gelu(z2)).astype(np.float64)
    y = a2 @ w3 + b3[0]
    B = y.size
    r = y - (np.asarray(t, np.float64) - y_mean) / y_std
    loss, dy = _huber(r)
    dz2 = bf16(np.outer(dy, w3) * gelu_grad(z2)).astype(np.float64)
    dz1 = bf16((dz2 @ W2b) * gelu_grad(z1)).astype(np.float64)
    g = np.concatenate([(dz1.T @ xn).ravel(), dz1.sum(0), (dz2.T @ a1).ravel(), dz2.sum(0),
                        a2.T @ dy, [dy.sum()]])
    return y, loss, g


def multifidelity_sum_weighted(omega, f, exact, draws, prob):
    """The Horvitz-Thompson form for k draws with replacement at probabilities prob:
    sum_w omega_w f_w + sum_{draws j} omega_j (e_j - f_j) / (k prob_j); unbiased for any f."""
    omega, f, exact, prob = (np.asarray(x) for x in (omega, f, exact, prob))
    draws = np.asarray(draws)
    k = draws.size
    return np.sum(omega * f) + np.sum(omega[draws] * (exact[draws] - f[draws]) / (k * prob[draws]))
