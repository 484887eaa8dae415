"""The scheduled SMEM entry point: any read order and any warp routing give the oracle's
bytes, and the per-read work log agrees with the results it describes."""
from __future__ import annotations

import numpy as np
import pytest

from haystackfm_b200 import _lib as L
from haystackfm_b200 import alphabet as al
from haystackfm_b200 import synth
from haystackfm_b200.errors import FmIndexError
from haystackfm_b200.fm_index import BidirFmIndex, FmIndexConfig, KIND_BIDIR, _build

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed_case(oracle):
    """2 Mbp IUPAC reference (N runs of mean 60 bp: a reference N matches every query base,
    and reads longer than the longest N run make the SMEM sweep quadratic in it); 240
    mixed-length reads (150 bp and 100 bp .. 10 kbp)."""
    ref = synth.iupac_reference(total=2_000_000, n_contigs=20, n_run_mean=60, seed=31)
    flat, off, lens = synth.sample_mixed_reads(ref, n_reads=240, seed=32)
    b = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=10), 0,
               KIND_BIDIR)
    idx = BidirFmIndex.from_bytes(b)
    bounds = idx.seq_boundaries()
    want = oracle.OracleIndex(b, KIND_BIDIR).mems_packed(flat, off, 19, 0, bounds, 64, threads=8)
    return idx, flat, off, lens, bounds, want


def _same(got, want):
    for g, w in zip(got[:3], want):
        assert np.array_equal(g, w)


def test_orders_and_routing_bit_exact(mixed_case):
    idx, flat, off, lens, bounds, want = mixed_case
    h = idx.handle
    nq = len(off) - 1
    rng = np.random.default_rng(0)
    _same(h.mems_sched_packed(flat, off, 19, 0, bounds, 64), want)
    _same(h.mems_sched_packed(flat, off, 19, 0, bounds, 64, order=np.arange(nq)[::-1]), want)
    perm = rng.permutation(nq)
    _same(h.mems_sched_packed(flat, off, 19, 0, bounds, 64, order=perm), want)
    _same(h.mems_sched_packed(flat, off, 19, 0, bounds, 64, order=perm, n_warp=17), want)
    _same(h.mems_sched_packed(flat, off, 19, 0, bounds, 64, order=np.argsort(-lens), n_warp=nq), want)


def test_work_log(mixed_case):
    idx, flat, off, lens, bounds, want = mixed_case
    h = idx.handle
    nq = len(off) - 1
    order = np.argsort(-lens, kind="stable")
    got = h.mems_sched_packed(flat, off, 19, 0, bounds, 64, order=order, n_warp=5, work_log=True)
    _same(got, want)
    hit_off, hits, _, log = got
    assert np.array_equal(log[:, 1], np.diff(hit_off.astype(np.int64)))
    npos = np.add.reduceat(np.r_[hits[:, 5].astype(np.int64), 0], hit_off[:-1].astype(np.int64))
    npos[np.diff(hit_off.astype(np.int64)) == 0] = 0
    assert np.array_equal(log[:, 2], npos)
    assert (log[:, 0] > 0).all()
    assert (log[order[:5], 3] & 1).all()             # routed reads ran on the warp kernel
    # longer reads do more extension work
    assert np.corrcoef(lens, log[:, 0].astype(np.float64))[0, 1] > 0.6
    # the log does not depend on the order for reads that stay on one kernel
    got2 = h.mems_sched_packed(flat, off, 19, 0, bounds, 64, work_log=True)
    same_path = ((got2[3][:, 3] & 1) == 0) & ((log[:, 3] & 1) == 0)
    assert np.array_equal(got2[3][same_path, 0], log[same_path, 0])


def test_bad_order_rejected(mixed_case):
    idx, flat, off, lens, bounds, want = mixed_case
    h = idx.handle
    nq = len(off) - 1
    bad = np.arange(nq)
    bad[3] = 4                                        # duplicate: not a permutation
    with pytest.raises(FmIndexError):
        h.mems_sched_packed(flat, off, 19, 0, bounds, 64, order=bad)
    big = np.arange(nq)
    big[0] = nq                                       # out of range
    with pytest.raises(FmIndexError):
        h.mems_sched_packed(flat, off, 19, 0, bounds, 64, order=big)
    with pytest.raises(FmIndexError):
        h.mems_sched_packed(flat, off, 19, 0, bounds, 64, order=None, n_warp=3)
    _same(h.mems_sched_packed(flat, off, 19, 0, bounds, 64), want)   # handle still usable


def test_long_reads_segmented_sweep_repeats(oracle):
    """Reads of 1-10 kbp on an ACGT genome with repeat families and tandem repeats take the
    segmented SMEM sweep (256-position segments merged along the true pivot chain): bytes
    equal the oracle's whole-read sweep, in both index alphabets' ACGT case."""
    ref = synth.repeat_reference(total=3_000_000, n_contigs=6, seed=41)
    flat, off, lens = synth.sample_mixed_reads(ref, n_reads=120, short_frac=0.3, long_median=2500, seed=42,
                                               n_rate=0.0)
    assert (lens > 1024).sum() >= 40
    for tag in (1, 0):
        b = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=8),
                   tag, KIND_BIDIR)
        idx = BidirFmIndex.from_bytes(b)
        bounds = idx.seq_boundaries()
        want = oracle.OracleIndex(b, KIND_BIDIR).mems_packed(flat, off, 19, 0, bounds, 256, threads=8)
        got = idx.handle.mems_packed(flat, off, 19, 0, bounds, 256)
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
        # and under a schedule that puts the long reads first
        _same(idx.handle.mems_sched_packed(flat, off, 19, 0, bounds, 256, order=np.argsort(-lens)), want)


def test_autotune_keeps_results(oracle):
    """The autotuner picks one of its candidate settings by measurement and results stay
    byte-identical under every setting."""
    import torch
    ref = synth.repeat_reference(total=2_000_000, n_contigs=4, seed=51)
    flat, off, lens = synth.sample_mixed_reads(ref, n_reads=80, short_frac=0.5, long_median=2000, seed=52,
                                               n_rate=0.0)
    b = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=8), 1,
               KIND_BIDIR)
    idx = BidirFmIndex.from_bytes(b)
    h = idx.handle
    bounds = idx.seq_boundaries()
    want = oracle.OracleIndex(b, KIND_BIDIR).mems_packed(flat, off, 19, 0, bounds, 128, threads=8)
    q = torch.from_numpy(flat).cuda()
    o = torch.from_numpy(off.view(np.int64)).cuda()
    res = h.autotune_mems(q, o, len(off) - 1, 19, 0, bounds, 128, reps=1)
    chosen = (res["mems_variant"], res["seg_len"], res["queue_chunk"], res["threads_per_read"], res["read_order"])
    assert chosen in L.TUNE_CANDIDATES
    assert h.tuning() == {"mems_variant": chosen[0], "seg_len": chosen[1], "queue_chunk": chosen[2],
                          "threads_per_read": chosen[3], "read_order": chosen[4]}
    assert len(res["candidates_ms"]) == len(L.TUNE_CANDIDATES) and all(v > 0 for v in res["candidates_ms"].values())
    for v, sl, ch, tp, od in [(3, 64, 1, 1, 0), (3, 4096, 1, 1, 0), (2, 512, 1, 1, 0), (4, 512, 1, 1, 0),
                              (3, 512, 7, 1, 0), (3, 256, 64, 1, 0), (3, 512, 1, 32, 0), (2, 512, 3, 32, 0),
                              (3, 512, 1, 4, 0), (3, 512, 1, 8, 0), (3, 512, 1, 16, 0), (2, 512, 3, 4, 0),
                              (3, 512, 1, 1, 1), (3, 64, 1, 1, 1), (2, 512, 5, 1, 1), (4, 512, 1, 1, 1),
                              (3, 512, 1, 8, 1)]:
        h.set_tuning(v, sl, ch, tp, od)
        _same(h.mems_packed(flat, off, 19, 0, bounds, 128), want)
        _same(h.mems_sched_packed(flat, off, 19, 0, bounds, 128), want)
    for bad in [(5, 512, 1, 1, 0), (3, 100, 1, 1, 0), (3, 512, 0, 1, 0), (3, 512, 65, 1, 0), (3, 512, 1, 2, 0),
                (3, 512, 1, 12, 0), (3, 512, 1, 1, 2)]:
        with pytest.raises(FmIndexError):
            h.set_tuning(*bad)


def test_plain_launch_bit_exact(mixed_case, oracle):
    """The plain launch (mems_variant 4: one thread per read, local sets, count pass +
    write pass) gives the oracle's bytes — long reads, set overflows into the warp kernel
    and pool sizing by the count pass included — in SMEM and MEM mode, with and without
    positions."""
    idx, flat, off, lens, bounds, want = mixed_case
    h = idx.handle
    saved = h.tuning()
    h.set_tuning(4, saved["seg_len"])
    try:
        _same(h.mems_packed(flat, off, 19, 0, bounds, 64), want)
        _same(h.mems_packed(flat, off, 19, 0, bounds, 64), want)          # warm pools
        o = oracle.OracleIndex(idx.to_bytes(), KIND_BIDIR)
        short = np.nonzero(lens <= 400)[0][:60]
        sub_flat = np.concatenate([flat[int(off[i]):int(off[i + 1])] for i in short])
        sub_off = np.concatenate([[0], np.cumsum(lens[short])]).astype(np.uint64)
        _same(h.mems_packed(sub_flat, sub_off, 15, 1, bounds, 8), o.mems_packed(sub_flat, sub_off, 15, 1, bounds, 8))
        _same(h.mems_packed(sub_flat, sub_off, 19, 0, [], 8), o.mems_packed(sub_flat, sub_off, 19, 0, [], 8))
    finally:
        h.set_tuning(saved["mems_variant"], saved["seg_len"])


@pytest.mark.parametrize("tpr", [4, 8, 16])
def test_sub_warp_groups_bit_exact(oracle, tpr):
    """Every read on a group of 4, 8 or 16 lanes (threads_per_read): the oracle's bytes on
    an IUPAC reference in SMEM and MEM mode, including reads whose interval sets outgrow the
    group's capacity (N stretches) and go on to the warp tier, and reads up to 3 kbp."""
    ref = synth.iupac_reference(total=1_000_000, n_contigs=12, n_run_mean=60, seed=61)
    flat, off, lens = synth.sample_mixed_reads(ref, n_reads=300, short_frac=0.8, long_median=1200, max_len=3000,
                                               seed=62, n_rate=0.002)
    nfl = np.concatenate([flat, np.full(6, 5, np.uint8), flat[:60]])      # a 6-N stretch: ~5k intervals
    noff = np.concatenate([off, [off[-1] + 66]]).astype(np.uint64)
    b = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=8), 0,
               KIND_BIDIR)
    idx = BidirFmIndex.from_bytes(b)
    h = idx.handle
    bounds = idx.seq_boundaries()
    o = oracle.OracleIndex(b, KIND_BIDIR)
    saved = h.tuning()
    h.set_tuning(3, 512, 1, tpr)
    try:
        _same(h.mems_packed(nfl, noff, 19, 0, bounds, 64), o.mems_packed(nfl, noff, 19, 0, bounds, 64, threads=8))
        short = np.nonzero(lens <= 300)[0][:80]
        sf = np.concatenate([flat[int(off[i]):int(off[i + 1])] for i in short])
        so = np.concatenate([[0], np.cumsum(lens[short])]).astype(np.uint64)
        _same(h.mems_packed(sf, so, 15, 1, bounds, 16), o.mems_packed(sf, so, 15, 1, bounds, 16, threads=8))
    finally:
        h.set_tuning(saved["mems_variant"], saved["seg_len"], saved["queue_chunk"], saved["threads_per_read"])


def test_prefix_read_order_bit_exact(oracle):
    """read_order = 1 (reads queued by their first 16 codes, a device radix sort) gives the
    bytes of the caller's order, on a batch large enough for the multi-pass sort, in SMEM
    and MEM mode; a subsample equals the oracle's."""
    ref = synth.iupac_reference(total=2_000_000, n_contigs=20, n_run_mean=60, seed=121)
    reads = synth.sample_reads(ref, n_reads=30_000, seed=122)
    flat, off = synth.pack_rows(reads)
    b = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=10), 0,
               KIND_BIDIR)
    idx = BidirFmIndex.from_bytes(b)
    h = idx.handle
    bounds = idx.seq_boundaries()
    saved = h.tuning()
    try:
        h.set_tuning(3, 512, 1, 1, 0)
        want = h.mems_packed(flat, off, 19, 0, bounds, 64)
        want_mem = h.mems_packed(flat[:150 * 3000], off[:3001], 17, 1, bounds, 8)
        h.set_tuning(3, 512, 1, 1, 1)
        assert h.tuning()["read_order"] == 1
        for _ in range(2):
            _same(h.mems_packed(flat, off, 19, 0, bounds, 64), want)
        _same(h.mems_packed(flat[:150 * 3000], off[:3001], 17, 1, bounds, 8), want_mem)
        sf, so = flat[:150 * 2000], off[:2001]
        _same(h.mems_packed(sf, so, 19, 0, bounds, 64),
              oracle.OracleIndex(b, KIND_BIDIR).mems_packed(sf, so, 19, 0, bounds, 64, threads=8))
    finally:
        h.set_tuning(saved["mems_variant"], saved["seg_len"], saved["queue_chunk"], saved["threads_per_read"],
                     saved["read_order"])
