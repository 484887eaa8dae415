"""Host-side mirror of haystackfm's FmIndex / BidirFmIndex query API over the C ABI.

Names, argument meanings and error behaviour follow the reference
(src/fm_index/mod.rs, query.rs, bidir_index.rs, smem.rs, src/gpu/*.rs); every query runs
on the GPU through libhfm.so.  Index construction (`build_cpu`) runs the library's native
builder and produces the reference's bincode bytes, which `from_bytes` loads.
"""
from __future__ import annotations

import ctypes as C
import struct
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

from . import _lib as L
from .alphabet import DnaSequence, TAG_EXACT, TAG_IUPAC
from .errors import FmIndexError

KIND_FM = 0
KIND_BIDIR = 1
MODE_SMEM = 0
MODE_MEM = 1


class OccEncoding:
    """src/occ/mod.rs:93-97"""
    Bitplane = 0
    OneHot = 1


class IupacDna:
    tag = TAG_IUPAC


class ExactDna:
    tag = TAG_EXACT


@dataclass
class FmIndexConfig:
    """src/fm_index/mod.rs:23-54"""
    sa_sample_rate: int = 32
    use_gpu: bool = True
    lookup_depth: int = 0
    build_threads: int = 1
    occ_encoding: int = OccEncoding.Bitplane


@dataclass
class MemHit:
    """src/gpu/mem_hit.rs:6-19"""
    query_start: int
    query_end: int
    match_count: int
    positions: List[Tuple[int, int]] = field(default_factory=list)
    truncated: bool = False


def _header_fields(data: bytes, base: int = 0):
    """(text_len, num_sequences, seq_boundaries, headers, end offset) of FmIndex bincode."""
    o = base + 64 + 2 + 32
    (n,) = struct.unpack_from("<Q", data, o); o += 8 + 4 * n          # superblock checkpoints
    (n,) = struct.unpack_from("<Q", data, o); o += 8 + n              # block data
    o += 8 + 4 + 4                                                  # stride, encoding, text_len
    (n,) = struct.unpack_from("<Q", data, o); o += 8 + n              # SA marker words
    (n,) = struct.unpack_from("<Q", data, o); o += 8 + 4 * n          # sa values
    o += 8                                                          # sample rate, ssa text_len
    text_len, nseq = struct.unpack_from("<II", data, o); o += 8
    (n,) = struct.unpack_from("<Q", data, o); o += 8
    bounds = np.frombuffer(data, dtype="<u4", count=n, offset=o).copy(); o += 4 * n
    (nh,) = struct.unpack_from("<Q", data, o); o += 8
    headers = []
    for _ in range(nh):
        (k,) = struct.unpack_from("<Q", data, o); o += 8
        headers.append(data[o:o + k].decode("utf-8")); o += k
    return text_len, nseq, bounds, headers


def _take_bytes(ptr, n: int) -> bytes:
    """Copy n bytes from a library-allocated block (ctypes.string_at takes a C int size,
    too small for genome-scale indices)."""
    return np.ctypeslib.as_array(ptr, shape=(n,)).tobytes() if n else b""


def _build(sequences: Sequence[DnaSequence], config: FmIndexConfig, tag: int, kind: int) -> bytes:
    if not sequences:
        raise FmIndexError.empty_sequence()
    codes = [s.as_slice() for s in sequences]
    flat, off = L.pack_queries(codes)
    hdr = (C.c_char_p * len(sequences))(*[s.header().encode() for s in sequences])
    # build_threads 0 or 1 -> single-threaded, as FmIndexConfig::build_threads (src/fm_index/mod.rs:33-36)
    opts = L.HfmBuildOpts(config.sa_sample_rate, config.lookup_depth, tag, config.occ_encoding,
                          max(1, int(config.build_threads)))
    out = L.u8p()
    n = C.c_size_t()
    L.check(L.lib().hfm_build_index(L.ptr(flat, L.u8p), L.ptr(off, L.u64p), len(sequences), hdr, C.byref(opts),
                                    kind, C.byref(out), C.byref(n)))
    data = _take_bytes(out, n.value)
    L.lib().hfm_free(out)
    return data


def _build_gpu(sequences: Sequence[DnaSequence], config: FmIndexConfig, tag: int, kind: int, device: int = 0) -> bytes:
    """hfm_build_index_gpu: the same bytes as _build, constructed on the GPU."""
    if not sequences:
        raise FmIndexError.empty_sequence()
    codes = [s.as_slice() for s in sequences]
    flat, off = L.pack_queries(codes)
    hdr = (C.c_char_p * len(sequences))(*[s.header().encode() for s in sequences])
    opts = L.HfmBuildOpts(config.sa_sample_rate, config.lookup_depth, tag, config.occ_encoding, 1)
    out = L.u8p()
    n = C.c_size_t()
    L.check(L.lib().hfm_build_index_gpu(L.ptr(flat, L.u8p), L.ptr(off, L.u64p), len(sequences), hdr, C.byref(opts),
                                        kind, device, C.byref(out), C.byref(n)))
    try:
        data = _take_bytes(out, n.value)
    finally:
        L.lib().hfm_free(out)
    return data


class _Handle:
    """Owns one device-resident index (hfm_index*)."""

    def __init__(self, data: bytes, kind: int, device: int = 0, flags: int = 0):
        self._buf = np.frombuffer(data, dtype=np.uint8)
        h = C.c_void_p()
        opts = L.HfmOpts(device, flags)
        L.check(L.lib().hfm_index_load(L.ptr(self._buf, L.u8p), len(data), kind, C.byref(opts), C.byref(h)))
        self.h = h
        self.kind = kind
        self.device = device

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and L._lib is not None:
            L._lib.hfm_index_free(self.h)
            self.h = None
        self._src = None

    def device_bytes(self) -> dict:
        """hfm_index_device_bytes: {"index": bytes of the layout, "work": work areas and results}."""
        a, b = C.c_uint64(), C.c_uint64()
        L.check(L.lib().hfm_index_device_bytes(self.h, C.byref(a), C.byref(b)))
        return {"index": a.value, "work": b.value}

    def export_layout(self) -> bytes:
        """hfm_index_export_layout: the device records of this index as one blob."""
        out = L.u8p()
        n = C.c_uint64()
        L.check(L.lib().hfm_index_export_layout(self.h, C.byref(out), C.byref(n)))
        try:
            return _take_bytes(out, n.value)
        finally:
            L.lib().hfm_free(out)

    @classmethod
    def from_layout(cls, blob: bytes, device: int = 0, flags: int = 0) -> "_Handle":
        """hfm_index_load_layout: a handle from a blob of export_layout, without the host
        transform of the bincode records."""
        o = cls.__new__(cls)
        o._buf = np.frombuffer(blob, dtype=np.uint8)
        h = C.c_void_p()
        opts = L.HfmOpts(device, flags)
        L.check(L.lib().hfm_index_load_layout(L.ptr(o._buf, L.u8p), len(blob), C.byref(opts), C.byref(h)))
        o.h, o.device, o._src = h, device, None
        o.kind = int(np.frombuffer(blob[8:12], dtype="<u4")[0])
        return o

    def share(self) -> "_Handle":
        """hfm_index_share: another handle on this index (own stream and work buffers)."""
        o = _Handle.__new__(_Handle)
        h = C.c_void_p()
        L.check(L.lib().hfm_index_share(self.h, C.byref(h)))
        o.h, o.kind, o.device, o._buf, o._src = h, self.kind, self.device, self._buf, self
        return o

    def info(self) -> L.HfmIndexInfo:
        info = L.HfmIndexInfo()
        L.check(L.lib().hfm_index_info_get(self.h, C.byref(info)))
        return info

    def stats(self) -> L.HfmStats:
        s = L.HfmStats()
        L.check(L.lib().hfm_last_stats(self.h, C.byref(s)))
        return s

    def stream(self) -> int:
        return L.lib().hfm_index_stream(self.h) or 0

    def set_counters(self, on: bool):
        L.check(L.lib().hfm_set_counters(self.h, int(on)))

    # -- packed-array entry points (numpy in, numpy out) ------------------------------
    def count_packed(self, flat: np.ndarray, off: np.ndarray) -> np.ndarray:
        nq = len(off) - 1
        out = np.zeros(max(nq, 1), dtype=np.uint32)
        L.check(L.lib().hfm_count_batch(self.h, L.ptr(flat, L.u8p), L.ptr(off, L.u64p), nq, L.ptr(out, L.u32p)))
        return out[:nq]

    def locate_packed(self, flat: np.ndarray, off: np.ndarray, max_hits: int = 0):
        """-> (counts u32[nq], offsets u64[nq+1], pairs u32[total, 2] of (seq_idx, pos_in_seq))."""
        nq = len(off) - 1
        res = C.POINTER(L.HfmHits)()
        L.check(L.lib().hfm_locate_batch(self.h, L.ptr(flat, L.u8p), L.ptr(off, L.u64p), nq, max_hits, C.byref(res)))
        try:
            r = res.contents
            offsets = np.ctypeslib.as_array(r.offsets, shape=(nq + 1,)).copy()
            counts = np.ctypeslib.as_array(r.counts, shape=(nq,)).copy() if nq else np.zeros(0, np.uint32)
            pairs = (np.ctypeslib.as_array(r.pairs, shape=(2 * r.total,)).reshape(-1, 2).copy()
                     if r.total else np.zeros((0, 2), np.uint32))
        finally:
            L.lib().hfm_free(res)
        return counts, offsets, pairs

    def mems_packed(self, flat: np.ndarray, off: np.ndarray, min_len: int, mode: int, ref_bounds, max_hits: int):
        """-> (hit_offsets u64[nq+1], hits u32[n_hits, 8], positions u32[n_pos, 2]).

        hits columns: query_start, query_end, match_count, truncated, fwd_lo, n_pos, pos_off_lo, pos_off_hi."""
        nq = len(off) - 1
        rb = np.ascontiguousarray(ref_bounds if ref_bounds is not None else [], dtype=np.uint32)
        rbp = L.ptr(rb, L.u32p) if len(rb) else None
        res = C.POINTER(L.HfmMemOut)()
        L.check(L.lib().hfm_mems_batch(self.h, L.ptr(flat, L.u8p), L.ptr(off, L.u64p), nq, min_len, mode, rbp,
                                       len(rb), max_hits, C.byref(res)))
        try:
            r = res.contents
            hit_off = np.ctypeslib.as_array(r.hit_offsets, shape=(nq + 1,)).copy()
            hits = (np.ctypeslib.as_array(C.cast(r.hits, L.u32p), shape=(8 * r.n_hits,)).reshape(-1, 8).copy()
                    if r.n_hits else np.zeros((0, 8), np.uint32))
            pos = (np.ctypeslib.as_array(r.positions, shape=(2 * r.n_positions,)).reshape(-1, 2).copy()
                   if r.n_positions else np.zeros((0, 2), np.uint32))
        finally:
            L.lib().hfm_free(res)
        return hit_off, hits, pos


    def mems_sched_packed(self, flat: np.ndarray, off: np.ndarray, min_len: int, mode: int, ref_bounds,
                          max_hits: int, order=None, n_warp: int = 0, work_log: bool = False):
        """hfm_mems_batch_device_sched on a host batch staged through torch device tensors.

        order: permutation of 0..nq-1 (queue order) or None; n_warp: the first n_warp reads
        of `order` run on the warp-per-read kernel.  -> (hit_offsets, hits, positions, log)
        with log u32[nq, 4] (touches, MemHits, positions, flags) when work_log, else None."""
        import torch
        nq = len(off) - 1
        dev = torch.device("cuda", self.device)
        q_d = torch.from_numpy(np.ascontiguousarray(flat, dtype=np.uint8)).to(dev)
        off_d = torch.from_numpy(np.ascontiguousarray(off, dtype=np.uint64).view(np.int64)).to(dev)
        ord_d = (torch.from_numpy(np.ascontiguousarray(order, dtype=np.uint32).view(np.int32)).to(dev)
                 if order is not None else None)
        log_d = torch.zeros(max(4 * nq, 1), dtype=torch.int32, device=dev) if work_log else None
        rb = np.ascontiguousarray(ref_bounds if ref_bounds is not None else [], dtype=np.uint32)
        rbp = L.ptr(rb, L.u32p) if len(rb) else None
        sc = L.HfmSched(ord_d.data_ptr() if ord_d is not None else None, n_warp, 0,
                        log_d.data_ptr() if log_d is not None else None)
        dm = L.HfmDevMems()
        torch.cuda.synchronize(dev)
        L.check(L.lib().hfm_mems_batch_device_sched(self.h, q_d.data_ptr(), off_d.data_ptr(), nq, min_len, mode,
                                                    rbp, len(rb), max_hits, C.byref(sc), C.byref(dm)))
        hit_off = device_to_host(dm.d_hit_offsets, nq + 1, "<i8", dev).view(np.uint64)
        hits = device_to_host(dm.d_hits, 8 * dm.n_hits, "<i4", dev).view(np.uint32).reshape(-1, 8)
        pos = device_to_host(dm.d_positions, 2 * dm.n_positions, "<i4", dev).view(np.uint32).reshape(-1, 2)
        log = log_d[:4 * nq].cpu().numpy().view(np.uint32).reshape(nq, 4) if work_log else None
        return hit_off, hits, pos, log


    def tuning(self) -> dict:
        t = L.HfmTuning()
        L.check(L.lib().hfm_get_tuning(self.h, C.byref(t)))
        return {"mems_variant": t.mems_variant, "seg_len": t.seg_len, "queue_chunk": t.queue_chunk,
                "threads_per_read": t.threads_per_read, "read_order": t.read_order}

    def set_tuning(self, mems_variant: int, seg_len: int, queue_chunk: int = None, threads_per_read: int = None,
                   read_order: int = None):
        cur = self.tuning()
        t = L.HfmTuning(mems_variant, seg_len, cur["queue_chunk"] if queue_chunk is None else queue_chunk,
                        cur["threads_per_read"] if threads_per_read is None else threads_per_read,
                        cur["read_order"] if read_order is None else read_order)
        L.check(L.lib().hfm_set_tuning(self.h, C.byref(t)))

    def autotune_mems(self, q_d, off_d, nq: int, min_len: int, mode: int, ref_bounds, max_hits: int, reps: int = 2):
        """hfm_autotune_mems on a device batch (torch tensors) -> {chosen setting, candidates' ms}."""
        rb = np.ascontiguousarray(ref_bounds if ref_bounds is not None else [], dtype=np.uint32)
        best = L.HfmTuning()
        times = np.zeros(len(L.TUNE_CANDIDATES), dtype=np.float32)
        L.check(L.lib().hfm_autotune_mems(self.h, q_d.data_ptr(), off_d.data_ptr(), nq, min_len, mode,
                                          L.ptr(rb, L.u32p) if len(rb) else None, len(rb), max_hits, reps,
                                          C.byref(best), times.ctypes.data_as(C.POINTER(C.c_float))))
        return {"mems_variant": best.mems_variant, "seg_len": best.seg_len, "queue_chunk": best.queue_chunk,
                "threads_per_read": best.threads_per_read, "read_order": best.read_order,
                "candidates_ms": {f"v{v}/seg{sl}/chunk{ch}/tpr{tp}/order{od}": round(float(t), 3)
                                  for (v, sl, ch, tp, od), t in zip(L.TUNE_CANDIDATES, times)}}


class _DeviceArray:
    """A raw device pointer exposed through __cuda_array_interface__ (read by torch)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}


def device_to_host(ptr, n: int, typestr: str, device) -> np.ndarray:
    """Copy n elements at a library-owned device pointer to a new numpy array."""
    import torch
    dt = {"<i4": np.int32, "<i8": np.int64, "<f4": np.float32}[typestr]
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dt)
    with torch.cuda.device(device):
        return torch.as_tensor(_DeviceArray(int(ptr), int(n), typestr), device=device).cpu().numpy()


class FmIndex:
    """Device-resident FmIndex (src/fm_index/mod.rs:58-72)."""

    def __init__(self, data: bytes, device: int = 0, _kind: int = KIND_FM, _base: int = 0):
        self._bytes = data
        self._h = _Handle(data, _kind, device) if _kind == KIND_FM else None
        self._text_len, self._nseq, self._bounds, self._headers = _header_fields(data, _base)

    # -- construction / persistence ------------------------------------------------
    @classmethod
    def build_cpu(cls, sequences, config: FmIndexConfig = None, device: int = 0) -> "FmIndex":
        return cls.build_cpu_with(IupacDna, sequences, config, device)

    @classmethod
    def build_cpu_with(cls, alphabet, sequences, config: FmIndexConfig = None, device: int = 0) -> "FmIndex":
        return cls(_build(sequences, config or FmIndexConfig(), alphabet.tag, KIND_FM), device)

    @staticmethod
    def build_bytes(sequences, config: FmIndexConfig = None, alphabet=IupacDna) -> bytes:
        return _build(sequences, config or FmIndexConfig(), alphabet.tag, KIND_FM)

    @classmethod
    def from_bytes(cls, data: bytes, device: int = 0) -> "FmIndex":
        return cls(bytes(data), device)

    def to_bytes(self) -> bytes:
        return self._bytes

    # -- properties -----------------------------------------------------------------
    def text_len(self) -> int:
        return self._text_len

    def num_sequences(self) -> int:
        return self._nseq

    def seq_boundaries(self) -> np.ndarray:
        return self._bounds

    def headers(self) -> List[str]:
        return self._headers

    def map_position(self, text_pos: int):
        """src/fm_index/query.rs:342-357"""
        idx = int(np.searchsorted(self._bounds, text_pos, side="right"))
        if idx >= len(self._bounds):
            return None
        start = 0 if idx == 0 else int(self._bounds[idx - 1])
        return idx, text_pos - start

    @property
    def handle(self) -> _Handle:
        return self._h

    # -- queries (GPU) ----------------------------------------------------------------
    def count_batch(self, patterns) -> np.ndarray:
        flat, off = L.pack_queries(patterns)
        return self.handle.count_packed(flat, off)

    def count(self, pattern) -> int:
        """FmIndex::count (src/fm_index/query.rs:9-14), computed on the GPU."""
        return int(self.count_batch([pattern])[0])

    def locate_batch_gpu(self, queries, max_hits: int = 0) -> List[List[Tuple[int, int]]]:
        """locate_batch_gpu (src/gpu/locate.rs:52): per query [(seq_idx, pos_in_seq)], CPU order."""
        flat, off = L.pack_queries(queries)
        _, offsets, pairs = self.handle.locate_packed(flat, off, max_hits)
        return [[(int(s), int(p)) for s, p in pairs[offsets[i]:offsets[i + 1]]] for i in range(len(queries))]

    def locate_gpu(self, queries, max_hits: int = 0) -> List[List[Tuple[str, int]]]:
        """FmIndex::locate_gpu (src/fm_index/query.rs:367-384)."""
        return [[(self._headers[s], p) for s, p in hits] for hits in self.locate_batch_gpu(queries, max_hits)]

    def locate(self, pattern) -> List[Tuple[str, int]]:
        """FmIndex::locate (src/fm_index/query.rs:22-39), computed on the GPU."""
        return self.locate_gpu([pattern])[0]

    def locate_positions(self, pattern) -> List[int]:
        """Absolute text offsets (src/fm_index/query.rs:46-55)."""
        out = []
        for s, p in self.locate_batch_gpu([pattern])[0]:
            out.append(p + (0 if s == 0 else int(self._bounds[s - 1])))
        return out


class BidirFmIndex:
    """Forward + reverse index pair (src/fm_index/bidir_index.rs:29-34)."""

    def __init__(self, data: bytes, device: int = 0):
        self._bytes = data
        (fl,) = struct.unpack_from("<I", data, 0)
        self._h = _Handle(data, KIND_BIDIR, device)
        self.fwd = FmIndex(data, device, _kind=KIND_BIDIR, _base=4)
        self.fwd._h = self._h          # locate / count run on the forward half of the same handle

    @classmethod
    def build_cpu(cls, sequences, config: FmIndexConfig = None, device: int = 0) -> "BidirFmIndex":
        return cls.build_cpu_with(IupacDna, sequences, config, device)

    @classmethod
    def build_cpu_with(cls, alphabet, sequences, config: FmIndexConfig = None, device: int = 0) -> "BidirFmIndex":
        return cls(_build(sequences, config or FmIndexConfig(), alphabet.tag, KIND_BIDIR), device)

    @staticmethod
    def build_bytes(sequences, config: FmIndexConfig = None, alphabet=IupacDna) -> bytes:
        return _build(sequences, config or FmIndexConfig(), alphabet.tag, KIND_BIDIR)

    @classmethod
    def from_bytes(cls, data: bytes, device: int = 0) -> "BidirFmIndex":
        if len(data) < 4:
            raise FmIndexError("DeserializeError", "truncated bidirectional index")
        return cls(bytes(data), device)

    def to_bytes(self) -> bytes:
        return self._bytes

    @property
    def handle(self) -> _Handle:
        return self._h

    def text_len(self) -> int:
        return self.fwd.text_len()

    def num_sequences(self) -> int:
        return self.fwd.num_sequences()

    def seq_boundaries(self) -> np.ndarray:
        """src/fm_index/bidir_index.rs:85-87"""
        return self.fwd.seq_boundaries()

    def mems_arrays(self, queries, min_len: int, mode: int, ref_boundaries=None, max_hits_per_mem: int = 1024):
        flat, off = L.pack_queries(queries)
        return self._h.mems_packed(flat, off, min_len, mode, ref_boundaries, max_hits_per_mem)

    def _mem_hits(self, queries, min_len, mode, ref_boundaries, max_hits_per_mem) -> List[List[MemHit]]:
        hit_off, hits, pos = self.mems_arrays(queries, min_len, mode, ref_boundaries, max_hits_per_mem)
        out = []
        for i in range(len(queries)):
            row = []
            for h in hits[hit_off[i]:hit_off[i + 1]]:
                po = int(h[6]) | (int(h[7]) << 32)
                row.append(MemHit(int(h[0]), int(h[1]), int(h[2]),
                                  [(int(a), int(b)) for a, b in pos[po:po + int(h[5])]], bool(h[3])))
            out.append(row)
        return out

    def find_smems_gpu(self, queries, min_len: int, ref_boundaries=(), max_hits_per_mem: int = 1024):
        """src/fm_index/bidir_index.rs:225-245 with CPU find_smems semantics."""
        return self._mem_hits(queries, min_len, MODE_SMEM, ref_boundaries, max_hits_per_mem)

    def find_mems_gpu(self, queries, min_len: int, ref_boundaries=(), max_hits_per_mem: int = 1024):
        """src/fm_index/bidir_index.rs:256-276 with CPU find_mems semantics."""
        return self._mem_hits(queries, min_len, MODE_MEM, ref_boundaries, max_hits_per_mem)

    def locate_gpu(self, queries, max_hits: int = 0):
        return self.fwd.locate_gpu(queries, max_hits)

    def count(self, pattern) -> int:
        return self.fwd.count(pattern)
