"""Host-side pieces of the mixed-length workload and the cost model (CPU only): the
repeat-rich genome, the mixed-length read generator, and the cost model's target and
error helpers."""
from __future__ import annotations

import numpy as np
import torch

from haystackfm_b200 import synth
from haystackfm_b200.cost_model import prediction_error, work_targets


def _dup_fraction(g: np.ndarray, k: int = 16) -> float:
    w = np.lib.stride_tricks.sliding_window_view(g.astype(np.uint64) - 1, k)[::7]
    keys = (w * (4 ** np.arange(k, dtype=np.uint64))).sum(axis=1)
    _, cnt = np.unique(keys, return_counts=True)
    return float((cnt > 1).sum() / len(cnt))


def test_repeat_reference_shape():
    ref = synth.repeat_reference(total=1_000_000, n_contigs=5, seed=3)
    assert len(ref.contigs) == 5 and sum(len(c) for c in ref.contigs) == 1_000_000
    g = np.concatenate(ref.contigs)
    assert g.min() >= 1 and g.max() <= 4                     # ACGT only: no N, no ambiguity codes
    uniform = np.random.default_rng(3).integers(1, 5, size=1_000_000, dtype=np.uint8)
    assert _dup_fraction(g) > 10 * max(_dup_fraction(uniform), 1e-4)   # repeat copies share 16-mers


def test_mixed_reads_lengths_and_errors():
    ref = synth.repeat_reference(total=2_000_000, n_contigs=4, seed=4)
    flat, off, lens = synth.sample_mixed_reads(ref, n_reads=2000, seed=5, n_rate=0.0)
    assert len(off) == 2001 and int(off[-1]) == len(flat) and np.array_equal(np.diff(off.astype(np.int64)), lens)
    assert flat.min() >= 1 and flat.max() <= 4
    short = lens == 150
    assert 0.75 < short.mean() < 0.85
    assert lens[~short].min() >= 100 and lens.max() <= 10_000
    assert 2000 < np.median(lens[~short]) < 4500
    again = synth.sample_mixed_reads(ref, n_reads=2000, seed=5, n_rate=0.0)
    assert np.array_equal(again[0], flat)                    # seeded


def test_mutate_rates():
    rng = np.random.default_rng(6)
    s = rng.integers(1, 5, size=20_000, dtype=np.uint8)
    assert np.array_equal(synth._mutate(s, 0.0, rng), s)
    m = synth._mutate(s, 0.3, rng)
    assert m.min() >= 1 and m.max() <= 4
    assert abs(len(m) - len(s)) < 0.02 * len(s)              # insertions and deletions balance


def test_avoid_masked_spans():
    ref = synth.iupac_reference(total=500_000, n_contigs=4, seed=7)
    flat, off, lens = synth.sample_mixed_reads(ref, n_reads=300, seed=8, avoid_masked=True, n_rate=0.0)
    assert len(lens) == 300 and flat.min() >= 1 and flat.max() <= 4


def test_work_targets_and_errors():
    log = np.array([[0, 0, 0, 1], [9, 1, 3, 0], [0xFFFFFFFF, 2, 5, 0]], dtype=np.uint32)
    t = work_targets(torch.from_numpy(log.view(np.int32)))
    assert t.dtype == torch.float32 and t.shape == (3, 3)
    assert np.allclose(t.numpy(), np.log1p(log[:, :3].astype(np.float64)), rtol=1e-6)
    y = torch.tensor([[1.0, 2.0, 3.0], [2.0, 1.0, 0.5], [3.0, 0.0, 1.0]])
    e = prediction_error(y, y)
    assert np.allclose(e.mae, 0) and np.allclose(e.r2, 1) and abs(e.spearman_touches - 1) < 1e-9
    e2 = prediction_error(-y, y)
    assert e2.spearman_touches < 0


def test_device_generators_shapes_and_seeding():
    """The genome-scale generators (run here on the CPU device): ACGT-only repeat genome
    with shared 16-mers, reads with the stated error model, seeded."""
    from haystackfm_b200 import synth_gpu as sg
    g, b = sg.repeat_genome(total=3_000_000, n_contigs=5, seed=3, device="cpu")
    assert g.shape[0] == 3_000_000 and int(b[-1]) == 3_000_000 and len(b) == 5
    assert int(g.min()) >= 1 and int(g.max()) <= 4
    uniform = np.random.default_rng(3).integers(1, 5, size=3_000_000, dtype=np.uint8)
    assert _dup_fraction(g.numpy()) > 10 * max(_dup_fraction(uniform), 1e-4)
    g2, _ = sg.repeat_genome(total=3_000_000, n_contigs=5, seed=3, device="cpu")
    assert torch.equal(g, g2)
    r = sg.sample_reads(g, b, 4000, seed=4)
    assert r.shape == (4000, 150) and 0.0003 < float((r == 5).float().mean()) < 0.003
    flat, off = sg.sample_mixed_reads(g, b, 3000, seed=5)
    lens = torch.diff(off).numpy()
    assert int(off[-1]) == flat.shape[0] and 0.75 < (lens == 150).mean() < 0.85
    assert lens.max() <= 10_000 and 2000 < np.median(lens[lens != 150]) < 4500
    f2, o2 = sg.sample_mixed_reads(g, b, 3000, seed=5)
    assert torch.equal(flat, f2) and torch.equal(off, o2)
