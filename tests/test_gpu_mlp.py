"""The cost model's CUDA kernels against the numpy oracle (features exact, forward and
gradient within BF16/FP32 tolerance, Adam step), training convergence, the schedule, and
the learned SMEM path against the plain one (byte-identical)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from haystackfm_b200 import alphabet as al
from haystackfm_b200 import synth
from haystackfm_b200.cost_model import LearnedSmem, ReadCostModel, prediction_error, work_targets
from haystackfm_b200.fm_index import BidirFmIndex, FmIndexConfig, KIND_BIDIR, _build
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def _reads(n=700, seed=0):
    ref = synth.iupac_reference(total=400_000, n_contigs=8, seed=seed)
    flat, off, lens = synth.sample_mixed_reads(ref, n_reads=n, long_median=600, max_len=3000, seed=seed + 1)
    flat[:: 997] = 7                      # a few ambiguity codes inside reads
    return flat, off


def _dev(flat, off):
    return (torch.from_numpy(np.ascontiguousarray(flat)).to(DEV),
            torch.from_numpy(np.ascontiguousarray(off.astype(np.uint64)).view(np.int64)).to(DEV))


def _bits_to_f32(x):
    return M.from_bits(x.cpu().numpy().view(np.uint16))


def test_features_match_oracle():
    flat, off = _reads()
    q, o = _dev(flat, off)
    m = ReadCostModel(0, seed=1)
    got = _bits_to_f32(m.features(q, o, len(off) - 1))
    want = M.features(flat, off)
    assert np.array_equal(np.delete(got, 256, axis=1), np.delete(want, 256, axis=1))
    # length column: log2 on the device vs numpy, equal up to one BF16 step
    assert np.all(np.abs(got[:, 256] - want[:, 256]) <= np.abs(want[:, 256]) * 2 ** -7 + 1e-6)


def _problem(seed=3, n=700):
    flat, off = _reads(n, seed)
    q, o = _dev(flat, off)
    m = ReadCostModel(0, seed=seed)
    x = m.features(q, o, len(off) - 1)
    X = _bits_to_f32(x).astype(np.float64)
    rng = np.random.default_rng(seed)
    T = rng.standard_normal((len(X), 3)).astype(np.float32) + np.array([9.0, 3.0, 6.0], np.float32)
    return m, x, X, torch.from_numpy(T).to(DEV), T


def test_forward_matches_oracle():
    m, x, X, t, T = _problem()
    p = m.get_params()
    got = m.forward(x).cpu().numpy()
    want = M.forward(p, X)
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 1e-2 * scale + 1e-3


def test_gradient_matches_oracle():
    """Gradient check: the CUDA backward pass (mma.sync BF16, FP32 accumulation) against the
    numpy oracle with the same rounding points; relative L2 error per tensor <= 2e-2."""
    m, x, X, t, T = _problem(seed=4)
    p = m.get_params()
    g_gpu, loss_gpu = m.grad(x, t)
    loss_ref, g_ref = M.loss_grad(p, X, T)
    assert abs(loss_gpu - loss_ref) <= 1e-3 * abs(loss_ref)
    bounds = [(M.P_W1, M.P_B1), (M.P_B1, M.P_W2), (M.P_W2, M.P_B2), (M.P_B2, M.P_W3), (M.P_W3, M.P_B3),
              (M.P_B3, M.NPARAM)]
    for a, b in bounds:
        err = np.linalg.norm(g_gpu[a:b] - g_ref[a:b]) / (np.linalg.norm(g_ref[a:b]) + 1e-12)
        assert err <= 2e-2, (a, b, err)
    # padded W1 columns see zero inputs: zero gradient
    W1g = g_gpu[M.P_W1:M.P_B1].reshape(M.HID, M.INP)
    assert (W1g[:, M.IN:] == 0).all()


def test_adam_step_matches_oracle():
    m, x, X, t, T = _problem(seed=5, n=256)
    p0 = m.get_params()
    g, _ = m.grad(x, t)
    m.train(x, t, epochs=1, batch=len(T), lr=1e-3, seed=0)   # one full-batch step
    p1 = m.get_params()
    want, _, _ = M.adam(p0, np.zeros_like(p0), np.zeros_like(p0), g, 1, 1e-3)
    # same step up to the summation order of the batch (rows shuffled)
    assert np.abs(p1 - want).max() <= 2e-5


def test_training_reduces_loss():
    """Targets that are a fixed function of the features: the loss must fall well below
    the variance of the targets."""
    flat, off = _reads(4000, seed=6)
    q, o = _dev(flat, off)
    m = ReadCostModel(0, seed=6)
    x = m.features(q, o, len(off) - 1)
    X = torch.from_numpy(_bits_to_f32(x)).to(DEV)
    t = torch.stack([X[:, 256] * 4 + 9, X[:, :16].sum(1) * 0.5 + 3, torch.relu(X[:, 5]) + 6], 1).contiguous()
    m.init_output_bias(t)
    losses = m.train(x, t, epochs=60, batch=512, lr=2e-3, seed=1)
    var = float(t.var(0).mean())
    assert losses[-1] < 0.2 * var and losses[-1] < losses[0]
    err = prediction_error(m.forward(x), t)
    assert err.r2[0] > 0.9


def test_schedule_bins():
    rng = np.random.default_rng(7)
    n = 5000
    y = np.stack([rng.uniform(0, 20, n), rng.uniform(0, 6, n), rng.uniform(0, 8, n)], 1).astype(np.float32)
    m = ReadCostModel(0)
    order, nw = m.schedule(torch.from_numpy(y).to(DEV), warp_min_hits=100.0)
    order = order.cpu().numpy().astype(np.int64)
    assert np.array_equal(np.sort(order), np.arange(n))
    routed = y[:, 1] >= np.log1p(np.float32(100.0))
    assert nw == routed.sum() and routed[order[:nw]].all()
    key = np.floor(y[order[nw:], 0] * (4096 / 24)).astype(np.int64)
    assert (np.diff(key) <= 0).all()                              # costliest first
    o2, nw2 = m.schedule(torch.from_numpy(y).to(DEV), warp_min_hits=0.0)
    assert nw2 == 0


def test_learned_smem_bit_exact():
    ref = synth.iupac_reference(total=1_000_000, n_contigs=10, seed=8)
    flat, off, lens = synth.sample_mixed_reads(ref, n_reads=600, long_median=800, max_len=4000, seed=9)
    b = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=8), 0,
               KIND_BIDIR)
    idx = BidirFmIndex.from_bytes(b)
    h = idx.handle
    bounds = np.ascontiguousarray(idx.seq_boundaries(), dtype=np.uint32)
    q, o = _dev(flat, off)
    nq = len(off) - 1
    ls = LearnedSmem(h, 0, seed=1, warp_min_hits=200.0)
    losses, x, t = ls.fit(q, o, nq, 19, 0, bounds, 64, epochs=20, batch=128, lr=2e-3)
    assert losses[-1] < losses[0]
    want = h.mems_sched_packed(flat, off, 19, 0, bounds, 64)
    order, nw, y = ls.plan(q, o, nq)
    got = h.mems_sched_packed(flat, off, 19, 0, bounds, 64, order=order.cpu().numpy(), n_warp=nw)
    for g_, w_ in zip(got[:3], want[:3]):
        assert np.array_equal(g_, w_)
    err = prediction_error(y, t)
    assert err.spearman_touches > 0.4            # length and composition rank the work
