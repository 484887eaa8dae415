"""Seeded synthetic inputs of the genome-scale workloads, generated on the GPU.

The 3.1 Gbp repeat-rich genome and its millions of reads take minutes with the numpy
generators of `synth`; these produce the same distributions on the device in seconds:

* repeat_genome — ACGT-only genome: uniform background; interspersed copies of 10
  300 bp and 10 6 kbp consensus sequences (long-family copies 5'-truncated to a uniform
  length in [500, 6000]), each copy with substitution divergence uniform in 10-20% and a
  random strand, covering 40% of the bases; tandem repeats (period uniform in 2..60, array
  length uniform in 100..3000, 5% substitutions) covering 5%.  Copies and arrays are laid
  between background stretches without overlapping one another.  Contig lengths are
  lognormal (mu=13, sigma=1) rescaled to the total.
* sample_reads — reads from either strand with substitutions and Ns (as synth.sample_reads).
* sample_mixed_reads — 80% 150 bp reads (1% substitutions) and 20% lognormal lengths
  (median 3 kbp, clipped to 100..10,000) with 8% substitutions / insertions / deletions in
  equal shares (as synth.sample_mixed_reads).

Every function takes a seed and gives the same output for the same seed and sizes.
"""
from __future__ import annotations

import numpy as np
import torch

A, C, G, T, N = 1, 2, 3, 4, 5


def _gen(seed: int, device) -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def _contig_lengths(total: int, n_contigs: int, rng: np.random.Generator, min_len: int = 1000) -> np.ndarray:
    raw = rng.lognormal(13.0, 1.0, size=n_contigs)
    lens = np.maximum(np.floor(raw / raw.sum() * total).astype(np.int64), min_len)
    lens[int(np.argmax(lens))] += total - int(lens.sum())
    return lens


def _substitute(x: torch.Tensor, rate: float, g: torch.Generator) -> torch.Tensor:
    """ACGT codes with a fraction `rate` replaced by one of the three other bases."""
    hit = torch.rand(x.shape, generator=g, device=x.device) < rate
    shift = torch.randint(1, 4, x.shape, generator=g, device=x.device, dtype=torch.uint8)
    return torch.where(hit, ((x - 1 + shift) % 4) + 1, x)


def repeat_genome(total: int = 3_100_000_000, n_contigs: int = 24, seed: int = 11, device="cuda",
                  interspersed_frac: float = 0.40, tandem_frac: float = 0.05):
    """-> (genome u8 tensor on `device`, exclusive contig ends as numpy int64)."""
    rng = np.random.default_rng(seed)
    g = _gen(seed, device)
    lens = _contig_lengths(total, n_contigs, rng)
    # consensus sequences
    fams = [rng.integers(1, 5, size=300, dtype=np.uint8) for _ in range(10)] + \
           [rng.integers(1, 5, size=6000, dtype=np.uint8) for _ in range(10)]
    cons = torch.from_numpy(np.concatenate(fams)).to(device)
    fam_off = np.concatenate([[0], np.cumsum([len(f) for f in fams])])
    # interspersed copies: family, length, source offset, divergence, strand
    est = int(interspersed_frac * total / 1700) + 1000
    fam = rng.integers(0, 20, size=est)
    clen = np.where(fam < 10, 300, rng.integers(500, 6001, size=est))
    keep = np.cumsum(clen) <= interspersed_frac * total
    keep[np.argmin(keep) if not keep.all() else len(keep) - 1] = True       # reach the target
    fam, clen = fam[keep], clen[keep]
    csrc = fam_off[fam] + np.where(fam < 10, 0, 6000 - clen)                # 5'-truncated long copies
    cdiv = rng.uniform(0.10, 0.20, size=len(fam)).astype(np.float32)
    crc = rng.random(len(fam)) < 0.5
    # tandem arrays: period, length
    est_t = int(tandem_frac * total / 1550) + 100
    per = rng.integers(2, 61, size=est_t)
    tlen = rng.integers(100, 3001, size=est_t)
    keep = np.cumsum(tlen) <= tandem_frac * total
    keep[np.argmin(keep) if not keep.all() else len(keep) - 1] = True
    per, tlen = per[keep], tlen[keep]
    units = rng.integers(1, 5, size=int(per.sum()), dtype=np.uint8)
    unit_off = np.concatenate([[0], np.cumsum(per)[:-1]])
    # segments in random order, separated by background gaps
    nseg = len(clen) + len(tlen)
    slen = np.concatenate([clen, tlen]).astype(np.int64)
    free = total - int(slen.sum())
    if free < 0:
        raise ValueError("repeat fractions exceed the genome")
    order = rng.permutation(nseg)
    cuts = np.sort(rng.integers(0, free + 1, size=nseg))
    gaps = np.diff(np.concatenate([[0], cuts]))                             # background before each segment
    starts = np.empty(nseg, dtype=np.int64)
    starts[order] = np.cumsum(gaps) + np.concatenate([[0], np.cumsum(slen[order])[:-1]])
    out = torch.randint(1, 5, (total,), generator=g, device=device, dtype=torch.uint8)
    # segment kinds: copy k < len(clen), tandem array otherwise
    d_start = torch.from_numpy(starts).to(device)
    d_len = torch.from_numpy(slen).to(device)
    d_src = torch.from_numpy(np.concatenate([csrc, unit_off]).astype(np.int64)).to(device)
    d_per = torch.from_numpy(np.concatenate([np.zeros(len(clen), np.int64), per])).to(device)
    d_div = torch.from_numpy(np.concatenate([cdiv, np.full(len(tlen), 0.05, np.float32)])).to(device)
    d_rc = torch.from_numpy(np.concatenate([crc, np.zeros(len(tlen), bool)])).to(device)
    d_units = torch.from_numpy(units).to(device)
    ncopy = len(clen)
    chunk = 4096
    for a in range(0, nseg, chunk):
        b = min(nseg, a + chunk)
        L = d_len[a:b]
        seg = torch.repeat_interleave(torch.arange(a, b, device=device), L)
        first = torch.cumsum(L, 0) - L
        local = torch.arange(len(seg), device=device) - torch.repeat_interleave(first, L)
        is_copy = seg < ncopy
        rc = d_rc[seg]
        ll = torch.where(rc, d_len[seg] - 1 - local, local)
        src_copy = cons[(d_src[seg] + ll).clamp(max=len(cons) - 1)]
        src_copy = torch.where(rc, 5 - src_copy, src_copy)
        per_s = d_per[seg].clamp(min=1)
        src_tan = d_units[(d_src[seg] + local % per_s).clamp(max=len(d_units) - 1)]
        base = torch.where(is_copy, src_copy, src_tan)
        hit = torch.rand(len(seg), generator=g, device=device) < d_div[seg]
        shift = torch.randint(1, 4, (len(seg),), generator=g, device=device, dtype=torch.uint8)
        base = torch.where(hit, ((base - 1 + shift) % 4) + 1, base)
        out[d_start[seg] + local] = base
    return out, np.cumsum(lens)


def _pick_starts(bounds: np.ndarray, need: torch.Tensor, g: torch.Generator, device):
    """Uniform start positions of spans of length `need` inside contigs (length-weighted)."""
    ends = torch.from_numpy(np.asarray(bounds, dtype=np.int64)).to(device)
    begins = torch.cat([torch.zeros(1, dtype=torch.int64, device=device), ends[:-1]])
    clen = ends - begins
    w = (clen - int(need.max()) + 1).clamp(min=0).double()
    cid = torch.multinomial(w, len(need), replacement=True, generator=g)
    room = (clen[cid] - need + 1).clamp(min=1)
    off = (torch.rand(len(need), generator=g, device=device, dtype=torch.float64) * room.double()).long()
    return begins[cid] + off


def sample_reads(genome: torch.Tensor, bounds, n_reads: int, read_len: int = 150, sub_rate: float = 0.01,
                 n_rate: float = 0.001, seed: int = 3, chunk: int = 1_000_000) -> torch.Tensor:
    """Reads (n_reads, read_len) u8 on the genome's device, from either strand."""
    device = genome.device
    g = _gen(seed, device)
    out = torch.empty((n_reads, read_len), dtype=torch.uint8, device=device)
    ar = torch.arange(read_len, device=device)
    for a in range(0, n_reads, chunk):
        m = min(chunk, n_reads - a)
        st = _pick_starts(bounds, torch.full((m,), read_len, dtype=torch.int64, device=device), g, device)
        r = genome[st[:, None] + ar[None, :]]
        rc = torch.rand(m, generator=g, device=device) < 0.5
        r = torch.where(rc[:, None], (5 - r).flip(1), r)
        r = _substitute(r, sub_rate, g)
        if n_rate > 0:
            r = torch.where(torch.rand(r.shape, generator=g, device=device) < n_rate, torch.full_like(r, N), r)
        out[a:a + m] = r
    return out


def sample_mixed_reads(genome: torch.Tensor, bounds, n_reads: int, short_frac: float = 0.8, short_len: int = 150,
                       long_median: int = 3000, long_sigma: float = 0.6, min_len: int = 100, max_len: int = 10_000,
                       short_sub: float = 0.01, long_err: float = 0.08, seed: int = 5, chunk: int = 50_000):
    """-> (flat u8 codes, int64 offsets[n_reads + 1]) on the genome's device."""
    device = genome.device
    g = _gen(seed, device)
    is_long = torch.rand(n_reads, generator=g, device=device) >= short_frac
    ll = torch.exp(np.log(long_median) + long_sigma * torch.randn(n_reads, generator=g, device=device))
    lens = torch.where(is_long, ll.long().clamp(min_len, max_len), torch.full_like(ll, short_len).long())
    pieces = []
    for a in range(0, n_reads, chunk):
        b = min(n_reads, a + chunk)
        L = lens[a:b]
        lg = is_long[a:b]
        src = torch.where(lg, (L.double() * 1.05).long() + 8, L)            # room for deletions
        st = _pick_starts(bounds, src, g, device)
        seg = torch.repeat_interleave(torch.arange(b - a, device=device), src)
        first = torch.cumsum(src, 0) - src
        local = torch.arange(len(seg), device=device) - torch.repeat_interleave(first, src)
        rc = (torch.rand(b - a, generator=g, device=device) < 0.5)[seg]
        pos = st[seg] + torch.where(rc, src[seg] - 1 - local, local)
        x = genome[pos]
        x = torch.where(rc, 5 - x, x)
        longb = lg[seg]
        # short reads: substitutions; long reads: substitutions, insertions, deletions
        ev = torch.rand(len(seg), generator=g, device=device)
        kind = torch.randint(0, 3, (len(seg),), generator=g, device=device)
        shift = torch.randint(1, 4, (len(seg),), generator=g, device=device, dtype=torch.uint8)
        subh = torch.where(longb, (ev < long_err) & (kind == 0), ev < short_sub)
        ins = longb & (ev < long_err) & (kind == 1)
        dele = longb & (ev < long_err) & (kind == 2)
        x = torch.where(subh, ((x - 1 + shift) % 4) + 1, x)
        reps = torch.ones(len(seg), dtype=torch.int64, device=device)
        reps[dele] = 0
        reps[ins] = 2
        res = torch.repeat_interleave(x, reps)
        ends = torch.cumsum(reps, 0)
        ipos = ends[ins] - 1
        res[ipos] = torch.randint(1, 5, (len(ipos),), generator=g, device=device, dtype=torch.uint8)
        # per read: the first min(result length, target length) codes
        seg_end = torch.cumsum(src, 0)
        rl = torch.diff(torch.cat([torch.zeros(1, dtype=torch.int64, device=device), ends[seg_end - 1]]))
        keep_len = torch.minimum(rl, L)
        rseg = torch.repeat_interleave(torch.arange(b - a, device=device), rl)
        rfirst = torch.cumsum(rl, 0) - rl
        rlocal = torch.arange(len(res), device=device) - torch.repeat_interleave(rfirst, rl)
        pieces.append((res[rlocal < keep_len[rseg]], keep_len))
    flat = torch.cat([p[0] for p in pieces])
    lens_out = torch.cat([p[1] for p in pieces])
    off = torch.zeros(n_reads + 1, dtype=torch.int64, device=device)
    off[1:] = torch.cumsum(lens_out, 0)
    return flat, off
