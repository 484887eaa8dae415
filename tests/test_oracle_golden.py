"""Pins the CPU oracle against the reference's golden vectors and known answers.

Every expected value comes from a haystackfm test (see tests/golden/reference_vectors.py);
brute-force matchers add property checks on random inputs like the reference's proptests.
"""
from __future__ import annotations

import random
import struct

import numpy as np
import pytest

from haystackfm_b200 import alphabet as al
from tests.golden import reference_vectors as gv
from tests.helpers import Lcg, brute_force_mems, concat, enc, map_positions, naive_positions, seqs_codes


def fm(orc, seqs, rate=1, lookup=0, tag=0, encoding=0, kind=0, headers=None):
    b = orc.build_index_bytes(seqs_codes(seqs), rate=rate, lookup_depth=lookup, tag=tag,
                              encoding=encoding, kind=kind, headers=headers)
    return orc.OracleIndex(b, kind), b


def test_compat_table_golden():
    for code in range(16):
        syms = al.compatible_symbols(code)
        assert len(syms) == gv.COMPAT_LEN[code]
        assert list(syms) + [0] * (16 - len(syms)) == gv.COMPAT_ROWS[code]
        for b in syms:   # symmetry (src/alphabet.rs:519-530)
            assert code in al.compatible_symbols(b)


def test_encoding_roundtrip():
    for code, ch in enumerate("$ACGTNRYSWKMBDHV"):
        assert al.encode_char(ch) == code and al.decode_char(code) == ch
    assert al.encode_char("u") == al.T and al.encode_char("-") is None and al.encode_char("X") is None
    text, bounds = al.concatenate_sequences([al.DnaSequence.from_str(s) for s in gv.CONCAT_VECTOR[0]])
    assert list(text) == gv.CONCAT_VECTOR[1] and list(bounds) == gv.CONCAT_VECTOR[2]


@pytest.mark.parametrize("text,expected", gv.C_ARRAY_VECTORS)
def test_c_array_golden(oracle, text, expected):
    seq = np.asarray(text[:-1], dtype=np.uint8)   # builder appends the sentinel
    _, b = fm(oracle, [seq])
    assert list(struct.unpack("<16I", b[:64])) == expected


def test_count_vectors(oracle):
    for text, pat, want in gv.COUNT_VECTORS:
        idx, _ = fm(oracle, [text])
        assert idx.count(enc(pat)) == want, (text, pat)


def test_query_cases(oracle):
    for seqs, rate, pat, kind, want in gv.QUERY_CASES:
        idx, _ = fm(oracle, seqs, rate=rate)
        if kind == "count":
            assert idx.count(enc(pat)) == want, (seqs, pat)
        else:
            assert sorted(idx.locate(enc(pat))) == want, (seqs, pat)
    seqs, mp = gv.MAP_POSITION_CASE
    idx, _ = fm(oracle, seqs)
    text, bounds = concat(seqs)
    assert map_positions(bounds, list(mp)) == [mp[k] for k in mp]
    assert sorted(idx.locate(enc("A"))) == [(0, 0), (1, 3)]
    assert sorted(idx.locate(enc("T"))) == [(0, 3), (1, 0)]
    assert idx.count(np.zeros(0, np.uint8)) == idx.text_len   # tests/query_tests.rs:161-167
    seqs, counts = gv.MULTI_SEQ_QUERIES
    idx, _ = fm(oracle, seqs)
    for p, c in counts.items():
        assert idx.count(enc(p)) == c
    assert idx.num_sequences == 3


def test_multi_sequence_all_sample_rates(oracle):
    ref, _ = fm(oracle, gv.MULTI_SEQ_RATE_SEQS, rate=1)
    for rate in gv.MULTI_SEQ_RATES:
        idx, _ = fm(oracle, gv.MULTI_SEQ_RATE_SEQS, rate=rate)
        for p in gv.MULTI_SEQ_RATE_PATTERNS:
            assert sorted(idx.locate(enc(p))) == sorted(ref.locate(enc(p))), (rate, p)


def test_random_vs_bruteforce(oracle):
    """count == len(locate) == brute force across sample rates (tests/proptest_correctness.rs)."""
    rng = random.Random(0xDEADBEEFCAFEBABE)
    for it in range(120):
        nseq = rng.randint(1, 4)
        seqs = ["".join(rng.choice("ACGT") for _ in range(rng.randint(5, 150))) for _ in range(nseq)]
        rate = rng.randint(1, 32)
        idx, _ = fm(oracle, seqs, rate=rate)
        text, bounds = concat(seqs)
        for _ in range(4):
            if rng.random() < 0.5:
                s = rng.choice(seqs)
                a = rng.randrange(len(s))
                pat = s[a:a + rng.randint(1, 15)]
            else:
                pat = "".join(rng.choice("ACGT") for _ in range(rng.randint(1, 8)))
            p = enc(pat)
            want = sorted(map_positions(bounds, naive_positions(text, p)))
            got = sorted(idx.locate(p))
            assert got == want and idx.count(p) == len(want), (seqs, pat, rate)


def test_iupac_locate_bruteforce(oracle):
    """IUPAC query x IUPAC reference (tests/locate_iupac_parity.rs cases + random)."""
    for seqs, pat in gv.LOCATE_IUPAC_CASES + gv.LOCATE_GPU_CASES:
        idx, _ = fm(oracle, seqs)
        text, bounds = concat(seqs)
        p = enc(pat)
        if len(p) == 0:
            assert idx.count(p) == len(text)
            continue
        want = sorted(map_positions(bounds, naive_positions(text, p)))
        assert sorted(idx.locate(p)) == want, (seqs, pat)
    rng = random.Random(7)
    for _ in range(60):
        seqs = ["".join(rng.choice("ACGTACGTNRYSWKMBDHV") for _ in range(rng.randint(5, 80)))
                for _ in range(rng.randint(1, 3))]
        idx, _ = fm(oracle, seqs, rate=rng.choice([1, 4, 32]))
        text, bounds = concat(seqs)
        for _ in range(4):
            p = enc("".join(rng.choice("ACGTNRYSWKMBDHV") for _ in range(rng.randint(1, 6))))
            want = sorted(map_positions(bounds, naive_positions(text, p)))
            assert sorted(idx.locate(p)) == want


def test_lookup_consistency(oracle):
    for text, depth, pats in gv.LOOKUP_CASES:
        with_lut, _ = fm(oracle, [text], lookup=depth)
        without, _ = fm(oracle, [text])
        for p in pats:
            assert with_lut.count(enc(p)) == without.count(enc(p)), (text, p)
        ex_lut, _ = fm(oracle, [text], lookup=depth, tag=1)
        ex_no, _ = fm(oracle, [text], tag=1)
        for p in pats:
            assert ex_lut.count(enc(p)) == ex_no.count(enc(p)), (text, p)
    text, depth, pat, want = gv.LOOKUP_SHORT_PATTERN
    assert fm(oracle, [text], lookup=depth)[0].count(enc(pat)) == want
    text, depth, pat = gv.EXACT_N_ZERO
    assert fm(oracle, [text], lookup=depth, tag=1)[0].count(enc(pat)) == 0
    assert fm(oracle, [text], lookup=depth, tag=0)[0].count(enc(pat)) > 0


def test_lookup_seed_quirk(oracle):
    """Lookup seeding only sees exact ACGT intervals (src/fm_index/query.rs:225-242): a reference N
    inside the last `depth` pattern positions is missed with the table and found without it."""
    with_lut, _ = fm(oracle, ["TTCCNGGTT"], lookup=3)
    without, _ = fm(oracle, ["TTCCNGGTT"])
    p = enc("CCAGG")
    assert without.count(p) == 1 and with_lut.count(p) == 0
    q = enc("CNGG")   # pattern's own N: last 3 = NGG not all core -> full search, equal
    text, _ = concat(["TTCCNGGTT"])
    assert without.count(q) == with_lut.count(q) == len(naive_positions(text, q)) == 2


def test_sa_and_resolve(oracle):
    rng = random.Random(3)
    for _ in range(20):
        seqs = ["".join(rng.choice("ACGTN") for _ in range(rng.randint(1, 60))) for _ in range(rng.randint(1, 4))]
        text, _ = concat(seqs)
        sa = oracle.suffix_array(text)
        naive = sorted(range(len(text)), key=lambda i: bytes(text[i:]))
        assert list(sa) == naive
        full, _ = fm(oracle, seqs, rate=1)
        for rate in (2, 5, 32):
            idx, _ = fm(oracle, seqs, rate=rate)
            rows = np.arange(idx.text_len, dtype=np.uint32)
            # multi-sequence rows whose suffix starts at a sentinel are never walked (no query
            # reaches them); every other row must resolve identically at every rate
            assert list(idx.resolve_rows(rows)) == list(full.resolve_rows(rows))


def test_bincode_roundtrip_and_errors(oracle):
    for kind in (0, 1):
        for enc_ in (0, 1):
            idx, b = fm(oracle, ["ACGTNACGTRY", "TTGCA"], rate=4, lookup=2 if kind == 0 else 0,
                        encoding=enc_, kind=kind)
            assert idx.to_bytes() == b
    _, b = fm(oracle, ["ACGT"], rate=4)
    bad = b[:-1] + b"\xff"                       # serialize.rs:128-146
    with pytest.raises(ValueError):
        oracle.OracleIndex(bad, 0)
    with pytest.raises(ValueError):
        oracle.OracleIndex(b[:40], 0)
    _, bb = fm(oracle, ["ACGT"], kind=1)
    with pytest.raises(ValueError):
        oracle.OracleIndex(bb[:3], 1)
    with pytest.raises(ValueError):
        oracle.OracleIndex(bb[:100], 1)


def test_onehot_equals_bitplane(oracle):
    rng = random.Random(11)
    seqs = ["".join(rng.choice("ACGTNNRY") for _ in range(300)) for _ in range(3)]
    a, _ = fm(oracle, seqs, rate=8, encoding=0)
    b, _ = fm(oracle, seqs, rate=8, encoding=1)
    for c in range(16):
        for i in range(0, a.text_len + 1, 7):
            assert a.rank(c, i) == b.rank(c, i)
    for _ in range(30):
        p = enc("".join(rng.choice("ACGTN") for _ in range(rng.randint(1, 5))))
        assert a.locate(p) == b.locate(p)


def test_extend_counts(oracle):
    """extend_right/extend_left sizes equal unidirectional counts (tests/bidir_correctness.rs:83-123)."""
    for text in ["ACGTACGT", "AAACCCGGGTTT", "ACGT", "TTTTTTTT", "ACGTTAGCCAGTACGT"]:
        bd, _ = fm(oracle, [text], kind=1)
        uni, _ = fm(oracle, [text])
        for pat in ["A", "AC", "ACG", "ACGT", "TT", "GGG"]:
            p = enc(pat)
            iv = (0, bd.text_len, 0, bd.text_len)
            for c in p:
                iv = bd.extend(0, iv, int(c))
                if iv is None:
                    break
            got = 0 if iv is None else iv[1] - iv[0]
            assert got == uni.count(p)
            iv = (0, bd.text_len, 0, bd.text_len)
            for c in p[::-1]:
                iv = bd.extend(1, iv, int(c))
                if iv is None:
                    break
            assert (0 if iv is None else iv[1] - iv[0]) == uni.count(p)


def _mem_keys(mems):
    return [(qs, qe, cnt) for qs, qe, cnt, _ in mems]


def test_smem_known_answers(oracle):
    for ref, q, min_len, mode, want in gv.SMEM_CASES:
        bd, _ = fm(oracle, [ref], kind=1)
        got = bd.mems_native(enc(q), min_len, 0 if mode == "smem" else 1)
        assert [(a, b) for a, b, _, _ in got] == [(a, b) for a, b, _ in want], (ref, q)
        for (a, b, c, _), (_, _, wc) in zip(got, want):
            if wc is not None:
                assert c == wc
            else:
                assert c >= 1
    bd, _ = fm(oracle, ["ACGTACGT"], kind=1)
    (m,) = bd.find_smems(enc("ACGT"), 1, locate=True)
    assert sorted(m[3]) == [(0, 0), (0, 4)]
    (m,) = fm(oracle, ["ACGT"], kind=1)[0].find_smems(enc("N"), 1, locate=True)
    assert sorted(o for _, o in m[3]) == [0, 1, 2, 3]


def test_smem_mem_bruteforce(oracle):
    for ref, q in gv.BRUTE_FORCE_CASES:
        bd, _ = fm(oracle, [ref], kind=1)
        want = brute_force_mems(ref, q, 1)
        assert [(a, b) for a, b, _, _ in bd.find_smems(enc(q), 1)] == want, (ref, q)
    ref, q = "ACGTTAGCCAGTACGT", "CGTTAGC"
    bd, _ = fm(oracle, [ref], kind=1)
    assert [(a, b) for a, b, _, _ in bd.find_mems(enc(q), 1)] == brute_force_mems(ref, q, 1)
    for m in bd.find_mems(enc("CGTTAGCAGT"), 1):
        s, e = m[0], m[1]
        assert "CGTTAGCAGT"[s:e] in ref
    # smem_positions_are_valid (tests/bidir_correctness.rs:262-294)
    ref, q = "ACGTTAGCCAGTACGT", "AGTACGT"
    bd, _ = fm(oracle, [ref], kind=1)
    for s, e, cnt, pos in bd.find_smems(enc(q), 1, locate=True):
        assert cnt == len(pos)
        for _, p in pos:
            assert ref[p:p + e - s] == q[s:e]


def test_smem_drop_regression(oracle):
    q = gv.SMEM_DROP_QUERY
    for (a, b), (c, d) in [((4, 30), (5, 176)), ((0, 171), (150, 176))]:
        bd, _ = fm(oracle, [q[a:b], q[c:d]], kind=1)
        sm = bd.find_smems(enc(q), 19, locate=True)
        hit = {s for m in sm for s, _ in m[3]}
        assert hit == {0, 1}, (a, b, c, d, [(x[0], x[1]) for x in sm])


def test_smems_equal_containment_filtered_mems(oracle):
    """src/fm_index/smem.rs:805-870 with the same LCG and seed."""
    rng = Lcg()
    for it in range(80):
        full = rng.dna(200)
        a, b = full[10:60], full[40:160]
        noise = rng.dna(80, "ACGTNRY") if it % 2 == 0 else rng.dna(80)
        bd, _ = fm(oracle, [a, b, noise], kind=1)
        q = enc(full)
        sm = [(x[0], x[1]) for x in bd.find_smems(q, 15)]
        mems = [(x[0], x[1]) for x in bd.find_mems(q, 15)]
        expected = sorted(m for m in mems if not any(o != m and o[0] <= m[0] and m[1] <= o[1] for o in mems))
        assert sorted(sm) == expected, full


def test_mem_hit_contract(oracle):
    """GPU MemHit contract: per-(qs,qe) summed counts equal CPU Mems and position sets equal
    (tests/mem_iupac_parity.rs:54-64, tests/gpu_mem_positions_parity.rs:40-88)."""
    for seqs, q, min_len, mode in gv.MEM_IUPAC_CASES:
        bd, _ = fm(oracle, seqs, kind=1)
        text, bounds = concat(seqs)
        native = bd.mems_native(enc(q), min_len, mode, locate=True)
        off, hits, pos = bd.mems_batch([enc(q)], min_len, mode, bounds, 1024)
        merged = {}
        for h in hits:
            merged[(h[0], h[1])] = merged.get((h[0], h[1]), 0) + int(h[2])
        assert sorted((k[0], k[1], v) for k, v in merged.items()) == sorted(_mem_keys(native))
        pset = {}
        for h in hits:
            po = int(h[6]) | (int(h[7]) << 32)
            pset.setdefault((h[0], h[1]), set()).update(map(tuple, pos[po:po + h[5]].tolist()))
        for qs, qe, _, p in native:
            assert pset.get((qs, qe), set()) == set(p)
    for seqs, qs_, min_len, mode, cap in gv.MEM_POSITION_CASES:
        bd, _ = fm(oracle, seqs, kind=1)
        _, bounds = concat(seqs)
        off, hits, pos = bd.mems_batch([enc(x) for x in qs_], min_len, mode, bounds, cap)
        if cap == 1:
            assert hits[0][5] == 1 and hits[0][3] == 1
        if qs_ == ["A"]:
            assert len(hits) == 0
    bd, _ = fm(oracle, ["ACGTACGT"], kind=1)
    off, hits, pos = bd.mems_batch([enc("ACGT")], 1, 1, None, 1024)   # no boundaries: no resolve
    assert len(hits) > 0 and all(h[5] == 0 for h in hits) and len(pos) == 0
