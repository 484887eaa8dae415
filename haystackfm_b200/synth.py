"""Seeded synthetic references and reads for the benchmark workloads.

No public dataset is named for this path, so every input is generated here with the
shapes and value distributions of the two workloads:

* exact_dna_workload — one uniform ACGT reference (1 Mbp by default), ExactDna; 32-mer
  queries, 90% substrings at uniform positions and 10% uniform random ACGT.
* iupac_workload — contigs with lognormal lengths (mu=13, sigma=1) rescaled to the total
  (100 Mbp, 200 contigs by default); uniform ACGT, N runs covering 2% of the bases
  (geometric run lengths, mean 500) and 0.5% single ambiguity codes (R..V uniform).  Reads
  (150 bp) are drawn from either strand of the unmasked ACGT sequence — the N runs and
  ambiguity codes mask only the reference — with 1% substitutions and 0.1% N.
* repeat_reference — ACGT-only genome with interspersed repeat families (300 bp and 6 kbp
  consensus, 10-20% divergent copies, 40% of the bases) and tandem repeats (period 2-60,
  5%), the scaled shape of a mammalian assembly.
* sample_mixed_reads — mixed-length reads on either reference: 80% 150 bp (1%
  substitutions), 20% lognormal lengths (median 3 kbp, clipped to 100 bp .. 10 kbp) with 8%
  mixed substitutions / insertions / deletions.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

A, C, G, T, N = 1, 2, 3, 4, 5


@dataclass
class Reference:
    contigs: list           # list of np.uint8 code arrays (masked reference)
    truth: list             # unmasked ACGT arrays (reads come from these)
    seed: int


def exact_dna_workload(ref_len=1_000_000, n_queries=10_000, qlen=32, substr_frac=0.9, seed=1):
    rng = np.random.default_rng(seed)
    ref = rng.integers(1, 5, size=ref_len, dtype=np.uint8)
    n_sub = int(round(n_queries * substr_frac))
    starts = rng.integers(0, ref_len - qlen + 1, size=n_sub)
    subs = ref[starts[:, None] + np.arange(qlen)[None, :]]
    rand = rng.integers(1, 5, size=(n_queries - n_sub, qlen), dtype=np.uint8)
    q = np.concatenate([subs, rand]).astype(np.uint8)
    q = q[rng.permutation(n_queries)]
    return ref, q


def _lognormal_lengths(rng, n, total, mu=13.0, sigma=1.0, min_len=1000):
    raw = rng.lognormal(mu, sigma, size=n)
    lens = np.maximum(np.floor(raw / raw.sum() * total).astype(np.int64), min_len)
    diff = total - int(lens.sum())
    lens[int(np.argmax(lens))] += diff          # exact total
    return lens


def iupac_reference(total=100_000_000, n_contigs=200, n_frac=0.02, n_run_mean=500, iupac_frac=0.005,
                    seed=2) -> Reference:
    rng = np.random.default_rng(seed)
    lens = _lognormal_lengths(rng, n_contigs, total, min_len=max(1000, total // (n_contigs * 50)))
    truth_all = rng.integers(1, 5, size=total, dtype=np.uint8)
    masked = truth_all.copy()
    # N runs: geometric lengths with the given mean, uniform starts, until 2% is covered
    target = int(total * n_frac)
    n_runs = max(1, target // n_run_mean)
    run_len = rng.geometric(1.0 / n_run_mean, size=n_runs * 2)
    run_len = run_len[np.cumsum(run_len) <= target] if run_len.sum() > target else run_len
    starts = rng.integers(0, total, size=len(run_len))
    for s, l in zip(starts, run_len):
        masked[s:s + l] = N
    # single ambiguity codes R..V (6..15) at uniform positions outside the N runs
    k = int(total * iupac_frac)
    free = np.flatnonzero(masked != N)
    pos = free[rng.choice(len(free), size=min(k, len(free)), replace=False)] if k else free[:0]
    masked[pos] = rng.integers(6, 16, size=len(pos), dtype=np.uint8)
    bounds = np.concatenate([[0], np.cumsum(lens)])
    contigs = [masked[bounds[i]:bounds[i + 1]] for i in range(n_contigs)]
    truth = [truth_all[bounds[i]:bounds[i + 1]] for i in range(n_contigs)]
    return Reference(contigs, truth, seed)


def repeat_reference(total=100_000_000, n_contigs=24, interspersed_frac=0.40, tandem_frac=0.05,
                     n_short_families=10, n_long_families=10, short_len=300, long_len=6000,
                     divergence=(0.10, 0.20), seed=11) -> Reference:
    """ACGT-only genome with repeats, the scaled shape of a mammalian assembly: uniform
    background; interspersed copies of `n_short_families` 300 bp and `n_long_families`
    6 kbp consensus sequences (long-family copies 5'-truncated to a uniform length in
    [500, 6000]) at per-copy substitution divergence uniform in `divergence`, covering
    `interspersed_frac` of the bases; tandem repeats (period uniform in 2..60, array length
    uniform in 100..3000, 5% substitutions) covering `tandem_frac`.  Contig lengths are
    lognormal (mu=13, sigma=1) rescaled to `total`.  No N runs, no ambiguity codes."""
    rng = np.random.default_rng(seed)
    lens = _lognormal_lengths(rng, n_contigs, total)
    g = rng.integers(1, 5, size=int(lens.sum()), dtype=np.uint8)
    fams = [rng.integers(1, 5, size=short_len, dtype=np.uint8) for _ in range(n_short_families)] + \
           [rng.integers(1, 5, size=long_len, dtype=np.uint8) for _ in range(n_long_families)]
    placed = 0
    target = interspersed_frac * len(g)
    while placed < target:
        f = int(rng.integers(0, len(fams)))
        cons = fams[f]
        if f >= n_short_families:
            cons = cons[len(cons) - int(rng.integers(500, len(cons) + 1)):]
        d = rng.uniform(*divergence)
        cp = cons.copy()
        sub = rng.random(len(cp)) < d
        cp[sub] = ((cp[sub] - 1 + rng.integers(1, 4, size=int(sub.sum()), dtype=np.uint8)) % 4) + 1
        if rng.random() < 0.5:
            cp = (5 - cp)[::-1]
        at = int(rng.integers(0, len(g) - len(cp)))
        g[at:at + len(cp)] = cp
        placed += len(cp)
    placed = 0
    target = tandem_frac * len(g)
    while placed < target:
        per = int(rng.integers(2, 61))
        L = int(rng.integers(100, 3001))
        unit = rng.integers(1, 5, size=per, dtype=np.uint8)
        arr = np.tile(unit, L // per + 1)[:L]
        sub = rng.random(L) < 0.05
        arr[sub] = ((arr[sub] - 1 + rng.integers(1, 4, size=int(sub.sum()), dtype=np.uint8)) % 4) + 1
        at = int(rng.integers(0, len(g) - L))
        g[at:at + L] = arr
        placed += L
    contigs, o = [], 0
    for l in lens:
        contigs.append(g[o:o + int(l)].copy())
        o += int(l)
    return Reference(contigs=contigs, truth=contigs, seed=seed)


def sample_reads(ref: Reference, n_reads=1_000_000, read_len=150, sub_rate=0.01, n_rate=0.001, seed=3):
    """Reads from either strand of the unmasked sequence with substitutions and Ns."""
    rng = np.random.default_rng(seed)
    lens = np.array([len(t) for t in ref.truth])
    ok = np.nonzero(lens >= read_len)[0]
    w = (lens[ok] - read_len + 1).astype(np.float64)
    cid = ok[rng.choice(len(ok), size=n_reads, p=w / w.sum())]
    starts = (rng.random(n_reads) * (lens[cid] - read_len + 1)).astype(np.int64)
    reads = np.empty((n_reads, read_len), dtype=np.uint8)
    for c in np.unique(cid):
        sel = np.nonzero(cid == c)[0]
        reads[sel] = ref.truth[c][starts[sel, None] + np.arange(read_len)[None, :]]
    rc = rng.random(n_reads) < 0.5
    reads[rc] = (5 - reads[rc])[:, ::-1]
    sub = rng.random(reads.shape) < sub_rate
    shift = rng.integers(1, 4, size=reads.shape, dtype=np.uint8)
    reads = np.where(sub, ((reads - 1 + shift) % 4) + 1, reads).astype(np.uint8)
    reads[rng.random(reads.shape) < n_rate] = N
    return reads


def _mutate(seq: np.ndarray, rate: float, rng) -> np.ndarray:
    """Mixed errors at `rate` per base: substitutions, 1-base insertions and deletions in
    equal shares."""
    ev = rng.random(len(seq))
    kind = rng.integers(0, 3, size=len(seq))
    hit = ev < rate
    sub = hit & (kind == 0)
    ins = hit & (kind == 1)
    dele = hit & (kind == 2)
    out = seq.copy()
    shift = rng.integers(1, 4, size=len(seq), dtype=np.uint8)
    out[sub] = ((out[sub] - 1 + shift[sub]) % 4) + 1
    reps = np.ones(len(seq), dtype=np.int64)
    reps[dele] = 0
    reps[ins] = 2
    res = np.repeat(out, reps)
    # the second copy of an inserted base becomes a random base
    first = np.cumsum(reps) - reps
    pos = first[ins] + 1
    res[pos] = rng.integers(1, 5, size=len(pos), dtype=np.uint8)
    return res


def _mutate_many(cat: np.ndarray, seg: np.ndarray, rate: float, rng):
    """_mutate over many sequences at once (`cat`: their concatenation, `seg`: their
    lengths).  -> (concatenated results, result lengths)."""
    n = len(cat)
    ev = rng.random(n, dtype=np.float32)
    kind = rng.integers(0, 3, size=n, dtype=np.uint8)
    shift = rng.integers(1, 4, size=n, dtype=np.uint8)
    hit = ev < rate
    sub = hit & (kind == 0)
    ins = hit & (kind == 1)
    dele = hit & (kind == 2)
    out = cat.copy()
    out[sub] = ((out[sub] - 1 + shift[sub]) % 4) + 1
    reps = np.ones(n, dtype=np.int8)
    reps[dele] = 0
    reps[ins] = 2
    res = np.repeat(out, reps)
    ends = np.cumsum(reps, dtype=np.int64)
    pos = ends[ins] - 1                      # the second copy of each inserted base
    res[pos] = rng.integers(1, 5, size=len(pos), dtype=np.uint8)
    bounds = np.cumsum(seg)
    rl = np.diff(np.concatenate([[0], ends[bounds - 1]]))
    return res, rl


def sample_mixed_reads(ref: Reference, n_reads=200_000, short_frac=0.8, short_len=150, long_median=3000,
                       long_sigma=0.6, min_len=100, max_len=10_000, short_sub=0.01, long_err=0.08,
                       n_rate=0.001, seed=5, avoid_masked=False):
    """Mixed-length reads as a flat batch: `short_frac` of fixed `short_len` reads with
    substitutions, the rest lognormal (median `long_median`, clipped to [min_len, max_len])
    with mixed substitutions / insertions / deletions at `long_err`; either strand, Ns at
    `n_rate`.  avoid_masked: draw only source spans whose reference holds no N (reads from
    sequenced regions; spans across an N run make the SMEM search quadratic in the run
    length).  Returns (flat u8 codes, u64 offsets[n+1], lengths)."""
    rng = np.random.default_rng(seed)
    is_long = rng.random(n_reads) >= short_frac
    lens = np.full(n_reads, short_len, dtype=np.int64)
    ll = np.exp(np.log(long_median) + long_sigma * rng.standard_normal(int(is_long.sum())))
    lens[is_long] = np.clip(ll.astype(np.int64), min_len, max_len)
    src_len = np.where(is_long, (lens * 1.05).astype(np.int64) + 8, lens)   # room for deletions
    clen = np.array([len(t) for t in ref.truth])
    # contig by length-weighted draw among contigs that hold the longest source span
    w_all = (clen - src_len.max() + 1).clip(min=0).astype(np.float64)
    cid = rng.choice(len(clen), size=n_reads, p=w_all / w_all.sum())
    starts = (rng.random(n_reads) * (clen[cid] - src_len + 1)).astype(np.int64)
    if avoid_masked:
        base = np.concatenate([[0], np.cumsum(clen)])
        gsum = np.concatenate([[0], np.cumsum(np.concatenate(ref.contigs) == N)])
        for _ in range(1000):
            a = base[cid] + starts
            bad = gsum[a + src_len] - gsum[a] > 0
            if not bad.any():
                break
            k = int(bad.sum())
            cid[bad] = rng.choice(len(clen), size=k, p=w_all / w_all.sum())
            starts[bad] = (rng.random(k) * (clen[cid[bad]] - src_len[bad] + 1)).astype(np.int64)
    rc = rng.random(n_reads) < 0.5
    out = [None] * n_reads
    # short reads, vectorised per contig
    sh = np.nonzero(~is_long)[0]
    rows = np.empty((len(sh), short_len), dtype=np.uint8)
    for c in np.unique(cid[sh]):
        sel = np.nonzero(cid[sh] == c)[0]
        rows[sel] = ref.truth[c][starts[sh[sel], None] + np.arange(short_len)[None, :]]
    flip = rc[sh]
    rows[flip] = (5 - rows[flip])[:, ::-1]
    sub = rng.random(rows.shape) < short_sub
    shift = rng.integers(1, 4, size=rows.shape, dtype=np.uint8)
    rows = np.where(sub, ((rows - 1 + shift) % 4) + 1, rows).astype(np.uint8)
    for k, i in enumerate(sh):
        out[i] = rows[k]
    # long reads: source spans (reverse-complemented where drawn), then mixed errors, in
    # vectorised chunks of reads
    li = np.nonzero(is_long)[0]
    chunk = 4_000
    for a in range(0, len(li), chunk):
        idx = li[a:a + chunk]
        srcs = [ref.truth[cid[i]][starts[i]:starts[i] + src_len[i]] for i in idx]
        srcs = [x[::-1] if rc[i] else x for x, i in zip(srcs, idx)]
        cat = np.concatenate(srcs).astype(np.uint8)
        seg = src_len[idx].astype(np.int64)
        flip = np.repeat(rc[idx], seg)
        cat = np.where(flip, 5 - cat, cat).astype(np.uint8)
        res, rl = _mutate_many(cat, seg, long_err, rng)
        roff = np.concatenate([[0], np.cumsum(rl)])
        for k, i in enumerate(idx):
            out[i] = res[roff[k]:roff[k] + min(int(rl[k]), int(lens[i]))]
    lens = np.array([len(s) for s in out], dtype=np.int64)
    flat = np.concatenate(out).astype(np.uint8) if out else np.zeros(0, np.uint8)
    if n_rate > 0:
        flat[rng.random(len(flat)) < n_rate] = N
    off = np.zeros(n_reads + 1, dtype=np.uint64)
    np.cumsum(lens, out=off[1:])
    return flat, off, lens


def pack_rows(rows: np.ndarray, width=None):
    """Fixed-length reads (n, L) -> (flat codes, u64 offsets) of the first `width` codes."""
    if width is not None:
        rows = rows[:, :width]
    rows = np.ascontiguousarray(rows, dtype=np.uint8)
    n, l = rows.shape
    off = (np.arange(n + 1, dtype=np.uint64) * np.uint64(l))
    return rows.reshape(-1), off
