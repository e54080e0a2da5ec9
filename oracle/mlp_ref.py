"""CPU oracle of the learned predictor -- TEST INFRASTRUCTURE ONLY.

A float64 numpy statement of the network in redzone_b200/csrc/rz_mlp.cu (12 -> 64 -> 64 -> 64,
ReLU hidden layers; softmax cross-entropy over outputs 0..62 with soft targets plus 0.5 x binary
cross-entropy of output 63; everything averaged over the batch), with the same flat parameter
layout, and a statement of the 12 features. Used to check the CUDA forward/backward kernels and
the feature kernel; the analytic gradient here is itself checked by finite differences in
tests/test_mlp_oracle.py.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H, N_OUT, N_CFG = 12, 64, 64, 63
BIT_WEIGHT = 0.5
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_IN * N_H
OFF_W2 = OFF_B1 + N_H
OFF_B2 = OFF_W2 + N_H * N_H
OFF_W3 = OFF_B2 + N_H
OFF_B3 = OFF_W3 + N_H * N_OUT
N_PARAMS = OFF_B3 + N_OUT


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(N_IN, N_H), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(N_H, N_H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(N_H, N_OUT), p[OFF_B3:N_PARAMS])


def forward(p, x):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    h1 = np.maximum(x @ w1 + b1, 0.0)
    h2 = np.maximum(h1 @ w2 + b2, 0.0)
    return h1, h2, h2 @ w3 + b3


def loss_and_grad(p, x, t):
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    nb = x.shape[0]
    w1, b1, w2, b2, w3, b3 = unpack(p)
    h1, h2, o = forward(p, x)
    z = o[:, :N_CFG]
    z = z - z.max(axis=1, keepdims=True)
    lse = np.log(np.exp(z).sum(axis=1, keepdims=True))
    logp = z - lse
    ce = -(t[:, :N_CFG] * logp).sum(axis=1)
    zb, tb = o[:, N_CFG], t[:, N_CFG]
    bce = np.maximum(zb, 0) - zb * tb + np.log1p(np.exp(-np.abs(zb)))
    loss = float(np.mean(ce + BIT_WEIGHT * bce))
    do = np.zeros_like(o)
    do[:, :N_CFG] = (np.exp(logp) - t[:, :N_CFG]) / nb
    do[:, N_CFG] = BIT_WEIGHT * (1.0 / (1.0 + np.exp(-zb)) - tb) / nb
    dh2 = (do @ w3.T) * (h2 > 0)
    dh1 = (dh2 @ w2.T) * (h1 > 0)
    g = np.concatenate([(x.T @ dh1).ravel(), dh1.sum(0), (h1.T @ dh2).ravel(), dh2.sum(0), (h2.T @ do).ravel(),
                        do.sum(0)])
    return loss, g


def features(idx, n, k, w, sample=4096):
    """The 12 features of rz_mlp_features for one instance (float64)."""
    idx = np.asarray(idx, np.uint64)
    s_n = min(k, sample)
    s = np.sort(idx[:s_n].astype(np.int64))
    scale = n / max(s_n, 1)
    gaps = np.log2(1.0 + np.diff(s) / scale) if s_n > 1 else np.zeros(0)
    m = gaps.sum() / (s_n - 1) if s_n > 1 else 0.0
    v = max((gaps ** 2).sum() / (s_n - 1) - m * m, 0.0) if s_n > 1 else 0.0
    tail = (s >= n - k).sum() / s_n if s_n else 0.0
    hist = np.zeros(5)
    if s_n:
        starts = np.flatnonzero(np.concatenate([[True], np.diff(s) != 1]))
        lens = np.diff(np.concatenate([starts, [s_n]]))
        for L in lens:
            hist[0 if L == 1 else 1 if L < 4 else 2 if L < 16 else 3 if L < 64 else 4] += 1
        hist /= max(len(lens), 1)
    return np.array([np.log2(max(n, 1)) / 32, np.log2(max(k, 1)) / 32, k / max(n, 1), w / 32, m / 8, v / 16, tail,
                     *hist])
