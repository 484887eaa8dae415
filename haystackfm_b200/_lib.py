"""ctypes binding of libhfm.so (the C ABI declared in include/hfm.h).

The library is the product: every query runs through its CUDA kernels.  Loading fails
loudly when libhfm.so is missing or when a query is issued without a CUDA device; there
is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .errors import FmIndexError

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhfm.so")

HFM_FLAG_DEDUP_ALWAYS = 1
HFM_FLAG_DEDUP_NEVER = 2

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)


class HfmOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("flags", C.c_uint32)]


class HfmIndexInfo(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("text_len", C.c_uint32), ("num_sequences", C.c_uint32),
                ("sample_rate", C.c_uint32), ("lookup_depth", C.c_uint32), ("alphabet_tag", C.c_uint32),
                ("num_lanes", C.c_uint32), ("encoding", C.c_uint32), ("device_bytes", C.c_uint64)]


class HfmHits(C.Structure):
    _fields_ = [("nq", C.c_uint32), ("_pad", C.c_uint32), ("total", C.c_uint64), ("offsets", u64p),
                ("counts", u32p), ("pairs", u32p)]


class HfmReads(C.Structure):
    _fields_ = [("n", C.c_uint64), ("n_codes", C.c_uint64), ("offsets", u64p), ("codes", u8p)]


class HfmMemHit(C.Structure):
    _fields_ = [("query_start", C.c_uint32), ("query_end", C.c_uint32), ("match_count", C.c_uint32),
                ("truncated", C.c_uint32), ("fwd_lo", C.c_uint32), ("n_pos", C.c_uint32),
                ("pos_off", C.c_uint64)]


class HfmMemOut(C.Structure):
    _fields_ = [("nq", C.c_uint32), ("_pad", C.c_uint32), ("n_hits", C.c_uint64), ("n_positions", C.c_uint64),
                ("hit_offsets", u64p), ("hits", C.POINTER(HfmMemHit)), ("positions", u32p)]


class HfmDevHits(C.Structure):
    _fields_ = [("nq", C.c_uint32), ("_pad", C.c_uint32), ("total", C.c_uint64), ("d_offsets", C.c_void_p),
                ("d_counts", C.c_void_p), ("d_pairs", C.c_void_p)]


class HfmDevMems(C.Structure):
    _fields_ = [("nq", C.c_uint32), ("_pad", C.c_uint32), ("n_hits", C.c_uint64), ("n_positions", C.c_uint64),
                ("d_hit_offsets", C.c_void_p), ("d_hits", C.c_void_p), ("d_positions", C.c_void_p)]


class HfmSched(C.Structure):
    _fields_ = [("d_order", C.c_void_p), ("n_warp", C.c_uint32), ("_pad", C.c_uint32), ("d_work_log", C.c_void_p)]


class HfmTuning(C.Structure):
    _fields_ = [("mems_variant", C.c_uint32), ("seg_len", C.c_uint32), ("queue_chunk", C.c_uint32),
                ("threads_per_read", C.c_uint32), ("read_order", C.c_uint32)]


# hfm_autotune_mems candidates {variant, seg_len, queue_chunk, threads_per_read}, in order
TUNE_CANDIDATES = [(3, 512, 1, 1, 0), (3, 256, 1, 1, 0), (3, 1024, 1, 1, 0), (2, 512, 1, 1, 0), (3, 512, 4, 1, 0),
                   (3, 512, 16, 1, 0), (3, 512, 1, 4, 0), (3, 512, 1, 8, 0), (3, 512, 1, 32, 0), (3, 512, 1, 1, 1),
                   (3, 1024, 1, 1, 1)]


class HfmStats(C.Structure):
    _fields_ = [("ms_search", C.c_float), ("ms_resolve", C.c_float), ("ms_total", C.c_float),
                ("ms_search_kernel", C.c_float), ("ms_resolve_kernel", C.c_float),
                ("search_launches", C.c_uint32), ("resolve_launches", C.c_uint32),
                ("other_launches", C.c_uint32), ("fallback_reads", C.c_uint32),
                ("occ_touches", C.c_uint64), ("lf_calls", C.c_uint64), ("rows_resolved", C.c_uint64),
                ("hits_out", C.c_uint64), ("rows_unique", C.c_uint64)]


class HfmBuildOpts(C.Structure):
    _fields_ = [("sa_sample_rate", C.c_uint32), ("lookup_depth", C.c_uint32), ("alphabet_tag", C.c_uint32),
                ("occ_encoding", C.c_uint32), ("threads", C.c_uint32)]


# every symbol include/hfm.h declares, with its ctypes signature
SIGNATURES = {
    "hfm_build_index": (C.c_int, [u8p, u64p, C.c_uint32, C.POINTER(C.c_char_p), C.POINTER(HfmBuildOpts), C.c_int,
                                  C.POINTER(u8p), C.POINTER(C.c_size_t)]),
    "hfm_build_index_gpu": (C.c_int, [u8p, u64p, C.c_uint32, C.POINTER(C.c_char_p), C.POINTER(HfmBuildOpts),
                                      C.c_int, C.c_int, C.POINTER(u8p), C.POINTER(C.c_size_t)]),
    "hfm_index_load": (C.c_int, [u8p, C.c_size_t, C.c_int, C.POINTER(HfmOpts), C.POINTER(C.c_void_p)]),
    "hfm_parse_reads": (C.c_int, [C.c_char_p, C.c_uint64, C.c_uint32, C.c_uint32, C.POINTER(C.POINTER(HfmReads))]),
    "hfm_index_device_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "hfm_index_export_layout": (C.c_int, [C.c_void_p, C.POINTER(u8p), C.POINTER(C.c_uint64)]),
    "hfm_index_load_layout": (C.c_int, [u8p, C.c_uint64, C.POINTER(HfmOpts), C.POINTER(C.c_void_p)]),
    "hfm_index_free": (None, [C.c_void_p]),
    "hfm_index_share": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "hfm_index_info_get": (C.c_int, [C.c_void_p, C.POINTER(HfmIndexInfo)]),
    "hfm_count_batch": (C.c_int, [C.c_void_p, u8p, u64p, C.c_uint32, u32p]),
    "hfm_locate_batch": (C.c_int, [C.c_void_p, u8p, u64p, C.c_uint32, C.c_uint32, C.POINTER(C.POINTER(HfmHits))]),
    "hfm_mems_batch": (C.c_int, [C.c_void_p, u8p, u64p, C.c_uint32, C.c_uint32, C.c_uint32, u32p, C.c_uint32,
                                 C.c_uint32, C.POINTER(C.POINTER(HfmMemOut))]),
    "hfm_count_batch_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "hfm_count_batch_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "hfm_locate_batch_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                          C.POINTER(HfmDevHits)]),
    "hfm_mems_batch_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                        u32p, C.c_uint32, C.c_uint32, C.POINTER(HfmDevMems)]),
    "hfm_mems_batch_device_sched": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                              C.c_uint32, u32p, C.c_uint32, C.c_uint32, C.POINTER(HfmSched),
                                              C.POINTER(HfmDevMems)]),
    "hfm_mlp_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    "hfm_mlp_free": (None, [C.c_void_p]),
    "hfm_mlp_set_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "hfm_mlp_get_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "hfm_mlp_stream": (C.c_void_p, [C.c_void_p]),
    "hfm_mlp_features": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "hfm_mlp_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "hfm_mlp_predict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "hfm_mlp_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                               C.POINTER(C.c_float)]),
    "hfm_mlp_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "hfm_mlp_schedule": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_void_p,
                                   C.POINTER(C.c_uint32)]),
    "hfm_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(HfmTuning)]),
    "hfm_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(HfmTuning)]),
    "hfm_autotune_mems": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, u32p,
                                    C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(HfmTuning),
                                    C.POINTER(C.c_float)]),
    "hfm_free": (None, [C.c_void_p]),
    "hfm_last_error": (C.c_char_p, []),
    "hfm_index_stream": (C.c_void_p, [C.c_void_p]),
    "hfm_last_stats": (C.c_int, [C.c_void_p, C.POINTER(HfmStats)]),
    "hfm_set_counters": (C.c_int, [C.c_void_p, C.c_int]),
    "hfm_set_timeout": (C.c_int, [C.c_void_p, C.c_uint32]),
    "hfm_mems_graph_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint32,
                                        C.c_uint32, u32p, C.c_uint32, C.c_uint32, C.c_uint64,
                                        C.POINTER(C.c_void_p)]),
    "hfm_mems_graph_launch": (C.c_int, [C.c_void_p, C.POINTER(HfmDevMems), C.POINTER(C.c_uint32)]),
    "hfm_mems_graph_free": (None, [C.c_void_p]),
    "hfm_mems_graph_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_uint32)]),
    "hfm_mems_graph_add_locate": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64,
                                            C.c_uint64]),
    "hfm_mems_graph_locate_result": (C.c_int, [C.c_void_p, C.POINTER(HfmDevHits)]),
    "hfm_mems_reserve": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64]),
    "hfm_probe_gather": (C.c_int, [C.c_int, C.c_uint64, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
}

_lib = None


def lib():
    """Load libhfm.so (building it first if the tree has no build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        L.hfm_suffix_array.restype = C.c_int
        L.hfm_suffix_array.argtypes = [u8p, C.c_uint32, u32p]
        _lib = L
    return _lib


def check(status: int):
    if status != 0:
        raise FmIndexError.from_status(status, lib().hfm_last_error().decode(errors="replace"))


def ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def pack_queries(queries):
    """Encoded queries -> (flat u8 codes, u64 offsets[nq+1])."""
    arrs = [np.asarray(q.as_slice() if hasattr(q, "as_slice") else q, dtype=np.uint8) for q in queries]
    off = np.zeros(len(arrs) + 1, dtype=np.uint64)
    if arrs:
        np.cumsum([len(a) for a in arrs], out=off[1:])
    flat = np.concatenate(arrs) if arrs and off[-1] else np.zeros(1, dtype=np.uint8)
    return np.ascontiguousarray(flat, dtype=np.uint8), off
