"""The cost model's numpy oracle, pinned on the CPU: its BF16 rounding against torch's,
its analytic gradient against finite differences, its features against a direct count."""
from __future__ import annotations

import numpy as np
import torch

from oracle import mlp_oracle as M


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    a = np.concatenate([rng.standard_normal(20000).astype(np.float32) * 10.0 ** rng.integers(-6, 6, 20000),
                        # exact ties between two BF16 values (both parities of the kept bit)
                        (np.arange(1, 2001, dtype=np.uint32) << 16 | 0x8000).view(np.float32),
                        np.array([0.0, -0.0, 1.0, -1.0, 3.4e38, 1e-40], dtype=np.float32)])
    want = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(M.bf16(a).view(np.uint32), want.view(np.uint32))
    assert np.array_equal(M.from_bits(M.bf16_bits(a)), want)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = rng.standard_normal(M.NPARAM) * 0.1
    W1 = p[M.P_W1:M.P_B1].reshape(M.HID, M.INP)
    W1[:, M.IN:] = 0.0
    X = np.zeros((6, M.INP))
    X[:, :M.IN] = rng.standard_normal((6, M.IN))
    T = rng.standard_normal((6, M.OUT))
    loss, g = M.loss_grad(p, X, T, rounding=False)
    assert np.isclose(loss, ((M.forward(p, X, rounding=False) - T) ** 2).mean())
    idx = np.concatenate([rng.integers(M.P_W1, M.P_B1, 40), rng.integers(M.P_B1, M.P_W2, 10),
                          rng.integers(M.P_W2, M.P_B2, 40), rng.integers(M.P_B2, M.P_W3, 10),
                          rng.integers(M.P_W3, M.P_B3, 20), np.arange(M.P_B3, M.NPARAM)])
    h = 1e-6
    for k in idx:
        q = p.copy(); q[k] += h
        lp = M.loss_grad(q, X, T, rounding=False)[0]
        q[k] -= 2 * h
        lm = M.loss_grad(q, X, T, rounding=False)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-4 * abs(fd), (k, fd, g[k])


def test_features_direct_count():
    rng = np.random.default_rng(2)
    reads = [rng.integers(1, 5, n).astype(np.uint8) for n in (0, 3, 4, 5, 150, 1000)]
    reads[4][[10, 70]] = 5            # N codes break the 4-mers that contain them
    reads.append(np.full(40, 5, np.uint8))
    flat = np.concatenate(reads)
    off = np.zeros(len(reads) + 1, np.uint64)
    off[1:] = np.cumsum([len(r) for r in reads])
    x = M.features(flat, off)
    for i, r in enumerate(reads):
        cnt = np.zeros(256)
        v = 0
        for p in range(len(r) - 3):
            w = r[p:p + 4]
            if all(1 <= c <= 4 for c in w):
                cnt[(w[0] - 1) * 64 + (w[1] - 1) * 16 + (w[2] - 1) * 4 + (w[3] - 1)] += 1
                v += 1
        want = np.zeros(M.INP, np.float32)
        if v:
            want[:256] = np.float32(256) * cnt.astype(np.float32) / np.float32(v) - np.float32(1)
        want[256] = (np.log2(np.float32(len(r) + 1)) - 10) * 0.25
        if len(r) >= 4:
            want[257] = np.float32(len(r) - 3 - v) / np.float32(len(r) - 3)
        assert np.array_equal(x[i], M.bf16(want))
    assert (x[:, M.IN:] == 0).all()


def test_adam_step():
    p = np.array([1.0, -2.0, 0.5], np.float32)
    g = np.array([0.1, -0.3, 0.0], np.float32)
    q, m, v = M.adam(p, np.zeros(3, np.float32), np.zeros(3, np.float32), g, 1, 1e-2)
    # first bias-corrected step moves each weight by lr * sign(g) (to within eps)
    assert np.allclose(q, p - 1e-2 * np.sign(g), atol=1e-6)
