"""Shared test helpers: index construction from strings and brute-force matchers."""
from __future__ import annotations

import numpy as np

from haystackfm_b200 import alphabet as al


def enc(s: str) -> np.ndarray:
    return al.encode(s)


def seqs_codes(seqs):
    return [al.encode(s) if isinstance(s, str) else np.asarray(s, dtype=np.uint8) for s in seqs]


def concat(seqs):
    text, bounds = al.concatenate_sequences([al.DnaSequence(c) for c in seqs_codes(seqs)])
    return text, bounds


def naive_positions(text_codes, pat_codes, tag=0):
    """Absolute text positions i where every pattern code is compatible with text[i+k]."""
    table = al.compat_table(tag)
    n, m = len(text_codes), len(pat_codes)
    out = []
    if m == 0:
        return list(range(n))
    for i in range(n - m + 1):
        if all(int(text_codes[i + k]) in table[int(pat_codes[k])] for k in range(m)):
            out.append(i)
    return out


def map_positions(bounds, positions):
    res = []
    for p in positions:
        idx = int(np.searchsorted(bounds, p, side="right"))
        start = 0 if idx == 0 else int(bounds[idx - 1])
        res.append((idx, p - start))
    return res


def brute_force_mems(reference: str, query: str, min_len: int):
    """Exact-string MEMs (src/fm_index/smem.rs:380-403)."""
    n = len(query)
    out = set()
    for s in range(n):
        for e in range(s + min_len, n + 1):
            sub = query[s:e]
            if sub not in reference:
                continue
            rmax = e == n or query[s:e + 1] not in reference
            lmax = s == 0 or query[s - 1:e] not in reference
            if rmax and lmax:
                out.add((s, e))
    return sorted(out)


class Lcg:
    """The reference's randomized-test LCG (src/fm_index/smem.rs:807-813)."""

    def __init__(self, state=0xDEADBEEFCAFEF00D):
        self.state = state

    def next(self) -> int:
        self.state = (self.state * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        return self.state >> 33

    def dna(self, n, alphabet="ACGT"):
        return "".join(alphabet[self.next() % len(alphabet)] for _ in range(n))
