"""Host-side ingest: FASTA / FASTQ parsing and read batching for the query entry points.

`parse_fasta` follows the reference's parser (src/wasm/js_api.rs:18-68): `>` lines are
headers, blank lines are skipped, sequence lines of a record are concatenated, and input
without any header is one sequence per non-blank line.  Reads are packed into the
(flat codes, u64 offsets) layout every `hfm_*_batch` call takes, encoded with the
alphabet's 256-entry table in one vectorised pass.
"""
from __future__ import annotations

from typing import Iterable, List, Tuple

import numpy as np

from .alphabet import ENCODE_LUT, SENTINEL, DnaSequence
from .errors import FmIndexError


def parse_fasta(text: str) -> List[DnaSequence]:
    """src/wasm/js_api.rs:18-68"""
    seqs: List[DnaSequence] = []
    cur, header = None, None
    for raw in text.splitlines():
        line = raw.strip()
        if not line:
            continue
        if line.startswith(">"):
            if cur is not None and cur:
                seqs.append(DnaSequence.from_str_with_header("".join(cur), header or ""))
            header = line[1:].strip()
            cur = []
        elif cur is not None:
            cur.append(line)
        else:
            seqs.append(DnaSequence.from_str(line))
    if cur is not None and cur:
        seqs.append(DnaSequence.from_str_with_header("".join(cur), header or ""))
    if not seqs:
        raise FmIndexError("InvalidCharacter", "no sequences found in input")
    return seqs


def parse_fastq(text: str) -> List[Tuple[str, str]]:
    """Four-line FASTQ records -> [(name, sequence)]."""
    lines = [l.rstrip("\r") for l in text.splitlines()]
    out = []
    i = 0
    while i < len(lines):
        if not lines[i].strip():
            i += 1
            continue
        if not lines[i].startswith("@") or i + 3 >= len(lines) or not lines[i + 2].startswith("+"):
            raise FmIndexError("InvalidCharacter", f"malformed FASTQ record at line {i + 1}")
        out.append((lines[i][1:].strip(), lines[i + 1].strip()))
        i += 4
    return out


def encode_reads(reads: Iterable[str]) -> Tuple[np.ndarray, np.ndarray]:
    """ASCII reads -> (flat u8 codes, u64 offsets[n+1]); invalid characters raise."""
    reads = list(reads)
    off = np.zeros(len(reads) + 1, dtype=np.uint64)
    if reads:
        np.cumsum([len(r) for r in reads], out=off[1:])
    raw = np.frombuffer("".join(reads).encode("ascii"), dtype=np.uint8)
    codes = ENCODE_LUT[raw]
    bad = np.nonzero((codes < 0) | (codes == SENTINEL))[0]
    if len(bad):
        k = int(bad[0])
        q = int(np.searchsorted(off, k, side="right")) - 1
        raise FmIndexError.invalid_character(chr(raw[k]), k - int(off[q]))
    flat = codes.astype(np.uint8) if len(codes) else np.zeros(1, dtype=np.uint8)
    return flat, off


def parse_reads(text, fmt: str = "auto", threads: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """hfm_parse_reads: FASTA / FASTQ / one-read-per-line text (str or bytes) -> the packed
    (flat u8 codes, u64 offsets[n+1]) batch, parsed and encoded natively on the host's
    threads.  Same reads as parse_fasta / parse_fastq + encode_reads; a character outside
    the alphabet raises FmIndexError("InvalidCharacter")."""
    import ctypes as C
    from . import _lib as L
    raw = text.encode("ascii") if isinstance(text, str) else bytes(text)
    f = {"auto": 0, "fasta": 1, "fastq": 2}[fmt]
    res = C.POINTER(L.HfmReads)()
    L.check(L.lib().hfm_parse_reads(raw, len(raw), f, threads, C.byref(res)))
    try:
        r = res.contents
        off = np.ctypeslib.as_array(r.offsets, shape=(r.n + 1,)).copy()
        flat = np.ctypeslib.as_array(r.codes, shape=(r.n_codes,)).copy() if r.n_codes else np.zeros(1, np.uint8)
    finally:
        L.lib().hfm_free(res)
    return flat, off


def batches(n: int, batch: int):
    """[start, end) ranges covering n reads in batches of at most `batch`."""
    for a in range(0, n, batch):
        yield a, min(n, a + batch)


def slice_packed(flat: np.ndarray, off: np.ndarray, a: int, b: int):
    """Reads a..b of a packed batch as their own packed batch (offsets rebased to 0)."""
    lo, hi = int(off[a]), int(off[b])
    sub = off[a:b + 1] - off[a]
    return flat[lo:hi] if hi > lo else np.zeros(1, dtype=np.uint8), sub
