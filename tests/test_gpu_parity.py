"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle, bit for bit.

Counts and locate hits compare in the reference CPU order; MEM hits compare in the
library's canonical order (MEMs by (query_start, query_end), hits of one MEM by fwd_lo),
which the oracle reproduces.
"""
from __future__ import annotations

import random

import numpy as np
import pytest

from haystackfm_b200 import alphabet as al
from haystackfm_b200 import synth
from haystackfm_b200.fm_index import BidirFmIndex, FmIndex, FmIndexConfig, KIND_BIDIR, KIND_FM, _Handle, _build
from haystackfm_b200._lib import pack_queries
from tests.golden import reference_vectors as gv
from tests.helpers import Lcg, concat, enc, seqs_codes

pytestmark = pytest.mark.gpu


def build(oracle, seqs, rate=1, lookup=0, tag=0, encoding=0, kind=KIND_FM):
    b = oracle.build_index_bytes(seqs_codes(seqs), rate=rate, lookup_depth=lookup, tag=tag, encoding=encoding,
                                 kind=kind)
    return oracle.OracleIndex(b, kind), _Handle(b, kind)


def check_count_locate(o, h, queries, caps=(0,)):
    flat, off = pack_queries(queries)
    want_c = o.count_packed(flat, off)
    got_c = h.count_packed(flat, off)
    assert np.array_equal(got_c, want_c)
    for cap in caps:
        wc, wo, wp = o.locate_packed(flat, off, cap)
        gc, go, gp = h.locate_packed(flat, off, cap)
        assert np.array_equal(gc, wc)
        assert np.array_equal(go, wo)
        assert np.array_equal(gp, wp)


def check_mems(o, h, queries, min_len, mode, bounds, cap):
    flat, off = pack_queries(queries)
    wo, wh, wp = o.mems_packed(flat, off, min_len, mode, bounds, cap)
    go, gh, gp = h.mems_packed(flat, off, min_len, mode, bounds, cap)
    assert np.array_equal(go, wo)
    assert np.array_equal(gh, wh)
    assert np.array_equal(gp, wp)


def test_golden_count_locate(oracle):
    for text, pat, want in gv.COUNT_VECTORS:
        o, h = build(oracle, [text])
        assert h.count_packed(*pack_queries([enc(pat)]))[0] == want
    for seqs, rate, pat, kind, want in gv.QUERY_CASES:
        o, h = build(oracle, seqs, rate=rate)
        check_count_locate(o, h, [enc(pat)])
    for seqs, pat in gv.LOCATE_IUPAC_CASES + gv.LOCATE_GPU_CASES:
        o, h = build(oracle, seqs, rate=1)
        check_count_locate(o, h, [enc(pat)])
    for rate in gv.MULTI_SEQ_RATES:
        o, h = build(oracle, gv.MULTI_SEQ_RATE_SEQS, rate=rate)
        check_count_locate(o, h, [enc(p) for p in gv.MULTI_SEQ_RATE_PATTERNS])


def test_lookup_and_quirk(oracle):
    for text, depth, pats in gv.LOOKUP_CASES:
        for tag in (0, 1):
            o, h = build(oracle, [text], lookup=depth, tag=tag)
            check_count_locate(o, h, [enc(p) for p in pats])
    o, h = build(oracle, ["TTCCNGGTT"], lookup=3)
    check_count_locate(o, h, [enc("CCAGG"), enc("CNGG")])
    assert h.count_packed(*pack_queries([enc("CCAGG")]))[0] == 0


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_random_iupac_count_locate(oracle, seed):
    rng = random.Random(seed)
    alphabet = ["ACGT", "ACGTN", "ACGTACGTNNRYSWKMBDHV"][seed % 3]
    seqs = ["".join(rng.choice(alphabet) for _ in range(rng.randint(50, 3000))) for _ in range(rng.randint(1, 6))]
    for rate, lookup, tag, encoding in [(32, 0, 0, 0), (7, 4, 0, 1), (1, 3, 1, 0), (32, 6, seed % 2, 0)]:
        o, h = build(oracle, seqs, rate=rate, lookup=lookup, tag=tag, encoding=encoding)
        qs = []
        for _ in range(300):
            if rng.random() < 0.6:
                s = rng.choice(seqs); a = rng.randrange(len(s))
                q = list(enc(s[a:a + rng.randint(1, 40)]))
                for k in range(len(q)):
                    if rng.random() < 0.05:
                        q[k] = rng.randint(1, 15)
                qs.append(np.array(q, np.uint8))
            else:
                qs.append(np.array([rng.randint(1, 15) for _ in range(rng.randint(0, 12))], np.uint8))
        qs.append(np.zeros(0, np.uint8))                       # empty pattern: whole text
        qs.append(np.array([0, 16, 1], np.uint8))              # sentinel / out-of-range codes: no match
        check_count_locate(o, h, qs, caps=(0, 1, 3))


def test_interval_set_overflow_fallback(oracle):
    """All-ambiguity queries on an ambiguity-rich reference grow interval sets far beyond the
    fast-path capacity; the fallback must give the same answer (no cap, as the CPU)."""
    rng = random.Random(42)
    seqs = ["".join(rng.choice("ACGTNRYSWKMBDHV") for _ in range(4000))]
    o, h = build(oracle, seqs, rate=8)
    qs = [enc("N" * k) for k in (1, 2, 3, 5, 8)] + [enc("NNRNNYNN"), enc("ACGTNNNNACGT")]
    check_count_locate(o, h, qs, caps=(0, 5))
    ob, hb = build(oracle, seqs, rate=8, kind=KIND_BIDIR)
    _, bounds = concat(seqs)
    check_mems(ob, hb, [enc("NNNNNNNN"), enc("ANNNNNNNNT"), enc("RYRYRYRYRY")], 1, 0, bounds, 16)
    check_mems(ob, hb, [enc("NNNNNN"), enc("NRNNYNN")], 2, 1, bounds, 16)


def test_golden_mems(oracle):
    for seqs, q, min_len, mode in gv.MEM_IUPAC_CASES:
        o, h = build(oracle, seqs, kind=KIND_BIDIR)
        _, bounds = concat(seqs)
        check_mems(o, h, [enc(q)], min_len, mode, bounds, 1024)
        check_mems(o, h, [enc(q)], min_len, mode, None, 1024)
    for seqs, qs, min_len, mode, cap in gv.MEM_POSITION_CASES:
        o, h = build(oracle, seqs, kind=KIND_BIDIR)
        _, bounds = concat(seqs)
        check_mems(o, h, [enc(x) for x in qs], min_len, mode, bounds, cap)
    for ref, q in gv.BRUTE_FORCE_CASES:
        o, h = build(oracle, [ref], kind=KIND_BIDIR)
        for mode in (0, 1):
            check_mems(o, h, [enc(q)], 1, mode, [len(ref) + 1], 1024)
    q = gv.SMEM_DROP_QUERY
    for (a, b), (c, d) in [((4, 30), (5, 176)), ((0, 171), (150, 176))]:
        o, h = build(oracle, [q[a:b], q[c:d]], rate=32, kind=KIND_BIDIR)
        _, bounds = concat([q[a:b], q[c:d]])
        check_mems(o, h, [enc(q)], 19, 0, bounds, 1024)


def test_smem_randomized_lcg(oracle):
    """The reference's randomized SMEM case set (src/fm_index/smem.rs:805-870) on the GPU."""
    rng = Lcg()
    for it in range(40):
        full = rng.dna(200)
        a, b = full[10:60], full[40:160]
        noise = rng.dna(80, "ACGTNRY") if it % 2 == 0 else rng.dna(80)
        seqs = [a, b, noise]
        o, h = build(oracle, seqs, rate=32, kind=KIND_BIDIR)
        _, bounds = concat(seqs)
        for mode in (0, 1):
            check_mems(o, h, [enc(full)], 15, mode, bounds, 1024)


def test_exact_dna_config(oracle):
    """1 Mbp uniform ACGT, ExactDna, rate 32, 10,000 32-mers (90% substrings): every query."""
    ref, q = synth.exact_dna_workload(ref_len=1_000_000, n_queries=10_000, seed=1)
    b = _build([al.DnaSequence(ref)], FmIndexConfig(sa_sample_rate=32, lookup_depth=0), 1, KIND_FM)
    o = oracle.OracleIndex(b, KIND_FM)
    h = _Handle(b, KIND_FM)
    flat, off = synth.pack_rows(q)
    assert np.array_equal(h.count_packed(flat, off), o.count_packed(flat, off, threads=8))
    wc, wo, wp = o.locate_packed(flat, off, 0, threads=8)
    gc, go, gp = h.locate_packed(flat, off, 0)
    assert np.array_equal(gc, wc) and np.array_equal(go, wo) and np.array_equal(gp, wp)
    assert int(wc.sum()) >= 9000


def test_iupac_config_subsample(oracle):
    """Scaled IUPAC workload (2 Mbp, 40 contigs, N runs, ambiguity codes; 150 bp reads with
    errors): locate of the first 32-mer (lookup depth 10, cap 1024) and SMEMs (min_len 19,
    max_hits 1024) on a read subsample, bit-exact."""
    ref = synth.iupac_reference(total=2_000_000, n_contigs=40, seed=7)
    reads = synth.sample_reads(ref, n_reads=600, seed=8)
    seqs = [al.DnaSequence(c) for c in ref.contigs]
    b = _build(seqs, FmIndexConfig(sa_sample_rate=32, lookup_depth=10), 0, KIND_BIDIR)
    o = oracle.OracleIndex(b, KIND_BIDIR)
    hb = BidirFmIndex.from_bytes(b)
    flat, off = synth.pack_rows(reads, 32)
    wc, wo, wp = o.locate_packed(flat, off, 1024, threads=8)
    gc, go, gp = hb.handle.locate_packed(flat, off, 1024)
    assert np.array_equal(gc, wc) and np.array_equal(go, wo) and np.array_equal(gp, wp)
    flat, off = synth.pack_rows(reads)
    bounds = hb.seq_boundaries()
    wo, wh, wp = o.mems_packed(flat, off, 19, 0, bounds, 1024, threads=8)
    go, gh, gp = hb.handle.mems_packed(flat, off, 19, 0, bounds, 1024)
    assert np.array_equal(go, wo) and np.array_equal(gh, wh) and np.array_equal(gp, wp)


def test_python_api_mirror(oracle):
    """The FmIndex / BidirFmIndex mirror returns the reference's result types."""
    idx = FmIndex.build_cpu([al.DnaSequence.from_str("ACGTACGT")], FmIndexConfig(sa_sample_rate=1))
    assert idx.count(enc("ACGT")) == 2
    assert sorted(idx.locate(enc("ACGT"))) == [("seq_0", 0), ("seq_0", 4)]
    assert idx.count(np.zeros(0, np.uint8)) == idx.text_len()
    bd = BidirFmIndex.build_cpu([al.DnaSequence.from_str("ACGTACGTACGTACGT")], FmIndexConfig(sa_sample_rate=1))
    hits = bd.find_mems_gpu([al.DnaSequence.from_str("ACGT")], 1, bd.seq_boundaries(), 1)
    assert hits[0][0].truncated and len(hits[0][0].positions) == 1
    hits = bd.find_mems_gpu([al.DnaSequence.from_str("ACGT")], 1, [], 1024)
    assert hits[0] and all(not m.positions for m in hits[0])
    assert bd.find_smems_gpu([], 1, bd.seq_boundaries(), 1024) == []
    again = BidirFmIndex.from_bytes(bd.to_bytes())
    assert again.find_smems_gpu([al.DnaSequence.from_str("CGTA")], 1, again.seq_boundaries()) == \
        bd.find_smems_gpu([al.DnaSequence.from_str("CGTA")], 1, bd.seq_boundaries())


def test_resolve_dedup_paths_identical(oracle):
    """Deduplicated and plain resolve give the same bytes (repeated intervals across reads)."""
    from haystackfm_b200._lib import HFM_FLAG_DEDUP_ALWAYS, HFM_FLAG_DEDUP_NEVER
    ref = synth.iupac_reference(total=400_000, n_contigs=10, seed=21)
    reads = synth.sample_reads(ref, n_reads=300, seed=22)
    b = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=16, lookup_depth=6), 0,
               KIND_BIDIR)
    o = oracle.OracleIndex(b, KIND_BIDIR)
    flat, off = synth.pack_rows(reads)
    flat32, off32 = synth.pack_rows(reads, 24)
    from haystackfm_b200.fm_index import _header_fields
    bounds = _header_fields(b, 4)[2]
    want_m = o.mems_packed(flat, off, 15, 0, bounds, 300)
    want_l = o.locate_packed(flat32, off32, 50)
    for flags in (HFM_FLAG_DEDUP_ALWAYS, HFM_FLAG_DEDUP_NEVER, 0):
        h = _Handle(b, KIND_BIDIR, 0, flags)
        for _ in range(2):       # repeated calls on one handle reuse its buffers
            got = h.mems_packed(flat, off, 15, 0, bounds, 300)
            for g, w in zip(got, want_m):
                assert np.array_equal(g, w)
            got = h.locate_packed(flat32, off32, 50)
            for g, w in zip(got, want_l):
                assert np.array_equal(g, w)
