"""ctypes binding of the CPU oracle (liboracle_hfm.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py; never by the haystackfm_b200 package.
The oracle restates the reference's Rust CPU query path (see hfm_oracle.cpp for
the file:line map).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_hfm.so")
_lib = None

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)


def build() -> str:
    """Compile liboracle_hfm.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_last_error.restype = C.c_char_p
        L.orc_load.restype = C.c_void_p
        L.orc_load.argtypes = [u8p, C.c_uint64, C.c_int]
        L.orc_index_free.argtypes = [C.c_void_p]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_text_len.restype = C.c_uint32
        L.orc_text_len.argtypes = [C.c_void_p]
        L.orc_num_sequences.restype = C.c_uint32
        L.orc_num_sequences.argtypes = [C.c_void_p]
        L.orc_build.argtypes = [u8p, u64p, C.c_uint32, C.POINTER(C.c_char_p), C.c_uint32, C.c_uint32,
                                C.c_uint8, C.c_uint32, C.c_int, C.POINTER(u8p), u64p]
        L.orc_to_bytes.argtypes = [C.c_void_p, C.POINTER(u8p), u64p]
        L.orc_rank.argtypes = [C.c_void_p, C.c_int, C.c_uint8, C.c_uint32, u32p]
        L.orc_resolve_rows.argtypes = [C.c_void_p, u32p, C.c_uint64, u32p]
        L.orc_count_batch.argtypes = [C.c_void_p, u8p, u64p, C.c_uint32, u32p, C.c_int]
        L.orc_locate_batch.argtypes = [C.c_void_p, u8p, u64p, C.c_uint32, C.c_uint32, C.c_int, u32p,
                                       C.POINTER(u64p), C.POINTER(u32p), u64p]
        L.orc_mems_batch.argtypes = [C.c_void_p, u8p, u64p, C.c_uint32, C.c_uint32, C.c_uint32, u32p,
                                     C.c_uint32, C.c_uint32, C.c_int, C.POINTER(u64p), C.POINTER(u32p),
                                     u64p, C.POINTER(u32p), u64p]
        L.orc_mems_native.argtypes = [C.c_void_p, u8p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_int,
                                      C.POINTER(u32p), u64p, C.POINTER(u32p), u64p]
        L.orc_extend.argtypes = [C.c_void_p, C.c_int, u32p, C.c_uint8, u32p]
        L.orc_smem_segment_check.argtypes = [C.c_void_p, u8p, u64p, C.c_uint32, C.c_uint32, C.c_uint32,
                                             u32p, u32p]
        L.orc_suffix_array.argtypes = [u8p, C.c_uint64, u32p]
        L.orc_suffix_array_doubling.argtypes = [u8p, C.c_uint64, u32p, C.c_int]
        L.orc_set_build_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def _take(ptr, n, dtype):
    """Copy n elements out of a malloc'd buffer and free it."""
    if n:
        arr = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)
    else:
        arr = np.zeros(0, dtype=dtype)
    lib().orc_free(ptr)
    return arr


def pack_queries(queries):
    """Encoded queries (sequences of codes 0..15) -> (flat u8, u64 offsets)."""
    lens = np.fromiter((len(q) for q in queries), dtype=np.uint64, count=len(queries))
    off = np.zeros(len(queries) + 1, dtype=np.uint64)
    np.cumsum(lens, out=off[1:])
    flat = np.zeros(max(int(off[-1]), 1), dtype=np.uint8)
    pos = 0
    for q in queries:
        b = np.asarray(q, dtype=np.uint8)
        flat[pos:pos + len(b)] = b
        pos += len(b)
    return flat, off


def build_index_bytes(seqs, *, rate=32, lookup_depth=0, tag=0, encoding=0, kind=0, headers=None) -> bytes:
    """Oracle construction (prefix-doubling suffix sort): FmIndex (kind 0) or BidirFmIndex (kind 1) bincode."""
    flat, off = pack_queries(seqs)
    hdr = None
    if headers is not None:
        hdr = (C.c_char_p * len(seqs))(*[h.encode() for h in headers])
    out = u8p()
    n = C.c_uint64()
    rc = lib().orc_build(_p(flat, u8p), _p(off, u64p), len(seqs), hdr, rate, lookup_depth, tag,
                         encoding, kind, C.byref(out), C.byref(n))
    if rc != 0:
        raise ValueError(lib().orc_last_error().decode())
    b = bytes(np.ctypeslib.as_array(out, shape=(n.value,))) if n.value else b""
    lib().orc_free(out)
    return b


def suffix_array(codes) -> np.ndarray:
    """Comparison sort of the suffixes (build_suffix_array_naive)."""
    t = np.ascontiguousarray(codes, dtype=np.uint8)
    out = np.zeros(len(t), dtype=np.uint32)
    lib().orc_suffix_array(_p(t, u8p), len(t), _p(out, u32p))
    return out


def suffix_array_doubling(codes, threads: int = 1) -> np.ndarray:
    """The prefix-doubling sorter that the oracle's index construction uses."""
    t = np.ascontiguousarray(codes, dtype=np.uint8)
    out = np.zeros(len(t), dtype=np.uint32)
    lib().orc_suffix_array_doubling(_p(t, u8p), len(t), _p(out, u32p), int(threads))
    return out


def set_build_threads(threads: int) -> None:
    """Host threads of the oracle's suffix sort during index construction."""
    lib().orc_set_build_threads(int(threads))


class OracleIndex:
    """A loaded FmIndex (kind 0) or BidirFmIndex (kind 1) on the CPU oracle."""

    def __init__(self, data: bytes, kind: int):
        self._buf = np.frombuffer(data, dtype=np.uint8).copy()
        self.kind = kind
        h = lib().orc_load(_p(self._buf, u8p), len(self._buf), kind)
        if not h:
            raise ValueError(lib().orc_last_error().decode())
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_index_free(self.h)
            self.h = None

    @property
    def text_len(self) -> int:
        return lib().orc_text_len(self.h)

    @property
    def num_sequences(self) -> int:
        return lib().orc_num_sequences(self.h)

    def to_bytes(self) -> bytes:
        out = u8p()
        n = C.c_uint64()
        lib().orc_to_bytes(self.h, C.byref(out), C.byref(n))
        b = bytes(np.ctypeslib.as_array(out, shape=(n.value,)))
        lib().orc_free(out)
        return b

    def rank(self, c: int, i: int, which: int = 0) -> int:
        r = C.c_uint32()
        lib().orc_rank(self.h, which, c, i, C.byref(r))
        return r.value

    def resolve_rows(self, rows) -> np.ndarray:
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        out = np.zeros(len(rows), dtype=np.uint32)
        lib().orc_resolve_rows(self.h, _p(rows, u32p), len(rows), _p(out, u32p))
        return out

    def count_batch(self, queries, threads: int = 1) -> np.ndarray:
        flat, off = pack_queries(queries)
        return self.count_packed(flat, off, threads)

    def count_packed(self, flat, off, threads: int = 1) -> np.ndarray:
        nq = len(off) - 1
        out = np.zeros(nq, dtype=np.uint32)
        lib().orc_count_batch(self.h, _p(flat, u8p), _p(off, u64p), nq, _p(out, u32p), threads)
        return out

    def count(self, pattern) -> int:
        return int(self.count_batch([pattern])[0])

    def locate_batch(self, queries, max_hits: int = 0, threads: int = 1):
        flat, off = pack_queries(queries)
        return self.locate_packed(flat, off, max_hits, threads)

    def locate_packed(self, flat, off, max_hits: int = 0, threads: int = 1):
        """-> (counts u32[nq], offsets u64[nq+1], pairs u32[total, 2] of (seq_idx, pos))."""
        nq = len(off) - 1
        counts = np.zeros(nq, dtype=np.uint32)
        o = u64p()
        pr = u32p()
        tot = C.c_uint64()
        lib().orc_locate_batch(self.h, _p(flat, u8p), _p(off, u64p), nq, max_hits, threads,
                               _p(counts, u32p), C.byref(o), C.byref(pr), C.byref(tot))
        offsets = _take(o, nq + 1, np.uint64)
        pairs = _take(pr, 2 * tot.value, np.uint32).reshape(-1, 2)
        return counts, offsets, pairs

    def locate(self, pattern):
        """FmIndex::locate with headers replaced by sequence indices, CPU order."""
        _, _, pairs = self.locate_batch([pattern])
        return [(int(s), int(p)) for s, p in pairs]

    def mems_batch(self, queries, min_len: int, mode: int = 0, ref_bounds=None, max_hits: int = 1024,
                   threads: int = 1):
        flat, off = pack_queries(queries)
        return self.mems_packed(flat, off, min_len, mode, ref_bounds, max_hits, threads)

    def mems_packed(self, flat, off, min_len: int, mode: int = 0, ref_bounds=None, max_hits: int = 1024,
                    threads: int = 1):
        """GPU-contract MemHits -> (hit_offsets u64[nq+1], hits u32[nh, 8], positions u32[np, 2])."""
        nq = len(off) - 1
        rb = np.ascontiguousarray(ref_bounds if ref_bounds is not None else [], dtype=np.uint32)
        rbp = _p(rb, u32p) if len(rb) else None
        ho = u64p()
        hits = u32p()
        nh = C.c_uint64()
        pos = u32p()
        npos = C.c_uint64()
        rc = lib().orc_mems_batch(self.h, _p(flat, u8p), _p(off, u64p), nq, min_len, mode, rbp, len(rb),
                                  max_hits, threads, C.byref(ho), C.byref(hits), C.byref(nh), C.byref(pos),
                                  C.byref(npos))
        if rc != 0:
            raise ValueError(lib().orc_last_error().decode())
        hit_off = _take(ho, nq + 1, np.uint64)
        h = _take(hits, 8 * nh.value, np.uint32).reshape(-1, 8)
        p = _take(pos, 2 * npos.value, np.uint32).reshape(-1, 2)
        return hit_off, h, p

    def mems_native(self, query, min_len: int, mode: int = 0, locate: bool = False):
        """CPU find_smems/find_mems -> list of (qs, qe, match_count, [(seq_idx, pos), ...])."""
        q = np.ascontiguousarray(query, dtype=np.uint8)
        if len(q) == 0:
            q = np.zeros(1, dtype=np.uint8)
            n = 0
        else:
            n = len(q)
        mems = u32p()
        nm = C.c_uint64()
        pos = u32p()
        npos = C.c_uint64()
        rc = lib().orc_mems_native(self.h, _p(q, u8p), n, min_len, mode, int(locate), C.byref(mems),
                                   C.byref(nm), C.byref(pos), C.byref(npos))
        if rc != 0:
            raise ValueError(lib().orc_last_error().decode())
        m = _take(mems, 4 * nm.value, np.uint32).reshape(-1, 4)
        p = _take(pos, 2 * npos.value, np.uint32).reshape(-1, 2)
        out, k = [], 0
        for qs, qe, cnt, npos_i in m:
            out.append((int(qs), int(qe), int(cnt), [(int(a), int(b)) for a, b in p[k:k + npos_i]]))
            k += int(npos_i)
        return out

    def find_smems(self, query, min_len: int, locate: bool = False):
        return self.mems_native(query, min_len, 0, locate)

    def find_mems(self, query, min_len: int, locate: bool = False):
        return self.mems_native(query, min_len, 1, locate)

    def smem_segment_check(self, flat: np.ndarray, off: np.ndarray, min_len: int, seg_len: int):
        """-> (reads whose segmented SMEM sweep differs from the whole-read one, reads checked)."""
        flat = np.ascontiguousarray(flat if len(flat) else np.zeros(1, np.uint8), dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.uint64)
        bad, n = np.zeros(1, np.uint32), np.zeros(1, np.uint32)
        rc = lib().orc_smem_segment_check(self.h, _p(flat, u8p), _p(off, u64p), len(off) - 1, min_len, seg_len,
                                          _p(bad, u32p), _p(n, u32p))
        if rc:
            raise RuntimeError(lib().orc_last_error().decode())
        return int(bad[0]), int(n[0])

    def extend(self, direction: int, iv, c: int):
        a = np.ascontiguousarray(iv, dtype=np.uint32)
        o = np.zeros(4, dtype=np.uint32)
        ok = lib().orc_extend(self.h, direction, _p(a, u32p), c, _p(o, u32p))
        return tuple(int(x) for x in o) if ok else None
