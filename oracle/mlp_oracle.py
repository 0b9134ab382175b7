"""FP64 oracle of the row-binning MLP.  TEST INFRASTRUCTURE ONLY.

Restates, in numpy float64, what the CUDA kernels of the learned path
compute: the 8 per-row features, the 8 -> 32 -> 32 -> 2 network, its loss
(squared error on output 0 plus BCE-with-logits on output 1, averaged over
the batch) and the analytic gradient.  The tests check the GPU gradient
against this one, and this one against central finite differences.

Parameter layout (1426 floats, as the library): W1[32][8], b1[32],
W2[32][32], b2[32], W3[2][32], b3[2], mean[8], inv_sd[8].
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 8, 32, 2
W1, B1 = 0, 256
W2, B2 = 288, 1312
W3, B3 = 1344, 1408
N_TRAINED = 1410
MU, INV_SD = 1410, 1418
N_PARAMS = 1426


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[W1:B1].reshape(N_HID, N_IN), p[B1:W2], p[W2:B2].reshape(N_HID, N_HID),
            p[B2:W3], p[W3:B3].reshape(N_OUT, N_HID), p[B3:N_TRAINED],
            p[MU:INV_SD], p[INV_SD:N_PARAMS])


def features(A, B):
    """Raw features (n x 8) of every row of A for the product A x B."""
    brp = np.asarray(B.row_ptr, np.int64)
    bci = np.asarray(B.col_idx, np.int64)
    blen = np.diff(brp)
    first = np.where(blen > 0, bci[np.minimum(brp[:-1], max(bci.size - 1, 0))], 0) \
        if bci.size else np.zeros(B.rows, np.int64)
    last = np.where(blen > 0, bci[np.maximum(brp[1:] - 1, 0)], 0) \
        if bci.size else np.zeros(B.rows, np.int64)
    arp = np.asarray(A.row_ptr, np.int64)
    k = np.asarray(A.col_idx, np.int64)
    nnz = np.diff(arp).astype(np.float64)
    rows = np.repeat(np.arange(A.rows), np.diff(arp))
    ln = blen[k]
    ops = np.zeros(A.rows)
    np.add.at(ops, rows, ln)
    maxlen = np.zeros(A.rows)
    np.maximum.at(maxlen, rows, ln)
    has = ln > 0
    lo = np.full(A.rows, np.inf)
    hi = np.full(A.rows, -np.inf)
    np.minimum.at(lo, rows[has], first[k[has]])
    np.maximum.at(hi, rows[has], last[k[has]])
    span = np.where(hi >= lo, hi - lo + 1, 0.0)
    mean_b = (brp[-1] / B.rows) if B.rows else 0.0
    raw = np.stack([nnz, ops, maxlen, np.where(nnz > 0, ops / np.maximum(nnz, 1), 0.0),
                    span, np.minimum(ops, span), np.full(A.rows, float(B.cols)),
                    np.full(A.rows, mean_b)], axis=1)
    return np.log2(1.0 + raw)


def forward(p, X):
    w1, b1, w2, b2, w3, b3, mu, isd = unpack(p)
    x = (np.asarray(X, np.float64) - mu) * isd
    a1 = x @ w1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ w2.T + b2
    h2 = np.maximum(a2, 0.0)
    y = h2 @ w3.T + b3
    return x, a1, h1, a2, h2, y


def loss(p, X, T):
    *_, y = forward(p, X)
    T = np.asarray(T, np.float64)
    e0 = y[:, 0] - T[:, 0]
    z = y[:, 1]
    bce = np.log1p(np.exp(-np.abs(z))) + np.maximum(z, 0.0) - z * T[:, 1]
    return float(np.mean(e0 * e0 + bce))


def gradient(p, X, T):
    """(loss, dL/dp over the 1410 trained parameters)."""
    x, a1, h1, a2, h2, y = forward(p, X)
    w1, b1, w2, b2, w3, b3, _, _ = unpack(p)
    T = np.asarray(T, np.float64)
    n = x.shape[0]
    dy = np.empty_like(y)
    dy[:, 0] = 2.0 * (y[:, 0] - T[:, 0]) / n
    dy[:, 1] = (1.0 / (1.0 + np.exp(-y[:, 1])) - T[:, 1]) / n
    g = np.zeros(N_TRAINED)
    g[W3:B3] = (dy.T @ h2).ravel()
    g[B3:N_TRAINED] = dy.sum(0)
    d2 = (dy @ w3) * (a2 > 0)
    g[W2:B2] = (d2.T @ h1).ravel()
    g[B2:W3] = d2.sum(0)
    d1 = (d2 @ w2) * (a1 > 0)
    g[W1:B1] = (d1.T @ x).ravel()
    g[B1:W2] = d1.sum(0)
    return loss(p, X, T), g


def finite_difference(p, X, T, idx, h=1e-6):
    p = np.asarray(p, np.float64).copy()
    out = []
    for i in idx:
        old = p[i]
        p[i] = old + h
        lp = loss(p, X, T)
        p[i] = old - h
        lm = loss(p, X, T)
        p[i] = old
        out.append((lp - lm) / (2 * h))
    return np.array(out)
