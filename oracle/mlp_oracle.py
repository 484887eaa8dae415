"""numpy restatement of the read-cost model (features, MLP forward, MSE gradient, Adam).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels in
haystackfm_b200/csrc/mlp.cu, imported by tests/ (never by the package).  The model has no
counterpart in the reference; this file states its definition once, in plain numpy, with
the same BF16 rounding points as the kernels:
  X (BF16) -> H1 = bf16(relu(X W1b^T + b1)) -> H2 = bf16(relu(H1 W2b^T + b2))
  -> Y = H2 W3b^T + b3 (FP32),   W*b = bf16(W*)
  loss = mean((Y - T)^2) over rows and the 3 outputs
  dY = 2 (Y - T) / (3 n); dH2 = bf16((dY W3b) * [H2 > 0]); dH1 = bf16((dH2 W2b) * [H1 > 0])
  dW3 = dY^T H2, dW2 = dH2^T H1, dW1 = dH1^T X, db* = column sums.
With rounding=False every rounding point is the identity (float64 throughout), which is
what the finite-difference check of the analytic gradient uses.
"""
from __future__ import annotations

import numpy as np

IN, INP, HID, OUT = 258, 272, 128, 3
P_W1 = 0
P_B1 = P_W1 + HID * INP
P_W2 = P_B1 + HID
P_B2 = P_W2 + HID * HID
P_W3 = P_B2 + HID
P_B3 = P_W3 + OUT * HID
NPARAM = P_B3 + OUT


def bf16(a) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def bf16_bits(a) -> np.ndarray:
    return (bf16(a).view(np.uint32) >> 16).astype(np.uint16)


def from_bits(bits) -> np.ndarray:
    return (np.asarray(bits, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def unpack(p):
    p = np.asarray(p)
    return (p[P_W1:P_B1].reshape(HID, INP), p[P_B1:P_W2], p[P_W2:P_B2].reshape(HID, HID), p[P_B2:P_W3],
            p[P_W3:P_B3].reshape(OUT, HID), p[P_B3:NPARAM])


def features(flat: np.ndarray, off: np.ndarray) -> np.ndarray:
    """Feature rows (float32, BF16-valued) of encoded reads (codes 1..4 = A, C, G, T)."""
    nq = len(off) - 1
    x = np.zeros((nq, INP), dtype=np.float32)
    for i in range(nq):
        r = flat[int(off[i]):int(off[i + 1])].astype(np.int64) - 1
        L = len(r)
        if L >= 4:
            w = np.lib.stride_tricks.sliding_window_view(r, 4)
            ok = ((w >= 0) & (w < 4)).all(axis=1)
            idx = (w[ok] * np.array([64, 16, 4, 1])).sum(axis=1)
            c = np.bincount(idx, minlength=256).astype(np.float32)
            v = int(ok.sum())
        else:
            c, v = np.zeros(256, np.float32), 0
        if v:
            x[i, :256] = np.float32(256) * c / np.float32(v) - np.float32(1)
        x[i, 256] = (np.log2(np.float32(L + 1)) - np.float32(10)) * np.float32(0.25)
        if L >= 4:
            x[i, 257] = np.float32(L - 3 - v) / np.float32(L - 3)
    return bf16(x)


def forward(p, X, rounding=True, cache=False):
    rd = bf16 if rounding else (lambda a: a)
    W1, b1, W2, b2, W3, b3 = unpack(p)
    f = np.float64
    W1b, W2b, W3b = (rd(W).astype(f) for W in (W1, W2, W3))
    X = np.asarray(X, dtype=f)
    H1 = rd(np.maximum(X @ W1b.T + b1, 0).astype(np.float32 if rounding else f)).astype(f)
    H2 = rd(np.maximum(H1 @ W2b.T + b2, 0).astype(np.float32 if rounding else f)).astype(f)
    Y = H2 @ W3b.T + b3
    if cache:
        return Y, (X, H1, H2, W1b, W2b, W3b)
    return Y


def loss_grad(p, X, T, rounding=True):
    """-> (loss, grad[NPARAM]) of the batch mean squared error."""
    rd = bf16 if rounding else (lambda a: a)
    Y, (X, H1, H2, W1b, W2b, W3b) = forward(p, X, rounding, cache=True)
    n = len(X)
    T = np.asarray(T, dtype=np.float64)
    D = Y - T
    loss = float((D * D).sum() / (n * OUT))
    dY = 2.0 * D / (n * OUT)
    g = np.zeros(NPARAM, dtype=np.float64)
    g[P_W3:P_B3] = (dY.T @ H2).reshape(-1)
    g[P_B3:NPARAM] = dY.sum(0)
    cast = (lambda a: a.astype(np.float32)) if rounding else (lambda a: a)
    dH2 = rd(cast((dY @ W3b) * (H2 > 0))).astype(np.float64)
    g[P_W2:P_B2] = (dH2.T @ H1).reshape(-1)
    g[P_B2:P_W3] = dH2.sum(0)
    dH1 = rd(cast((dH2 @ W2b) * (H1 > 0))).astype(np.float64)
    g[P_W1:P_B1] = (dH1.T @ X).reshape(-1)
    g[P_B1:P_W2] = dH1.sum(0)
    return loss, g


def adam(p, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba 2015) in float32; returns (p, m, v)."""
    f = np.float32
    m = f(b1) * m + f(1 - b1) * g
    v = f(b2) * v + f(1 - b2) * g * g
    c1, c2 = f(1 - b1 ** step), f(1 - b2 ** step)
    p = p - f(lr) * (m / c1) / (np.sqrt(v / c2) + f(eps))
    return p.astype(f), m.astype(f), v.astype(f)
