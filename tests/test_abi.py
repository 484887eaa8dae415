"""CPU-side checks of the C ABI: the library loads, exports every declared symbol, the
native index builder reproduces the oracle's bytes, and malformed bincode is rejected
before any device work (so these run without a GPU)."""
from __future__ import annotations

import ctypes as C
import os
import random
import re

import numpy as np
import pytest

from haystackfm_b200 import _lib as L
from haystackfm_b200 import alphabet as al
from haystackfm_b200.errors import HFM_E_FORMAT, HFM_E_ARG
from haystackfm_b200.fm_index import FmIndexConfig, _build, KIND_FM, KIND_BIDIR
from tests.helpers import concat, seqs_codes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "hfm.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hfm_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) <= set(L.SIGNATURES), set(syms) - set(L.SIGNATURES)


def _seqs(rng, n, alphabet, lo, hi):
    return ["".join(rng.choice(alphabet) for _ in range(rng.randint(lo, hi))) for _ in range(n)]


def product_bytes(seqs, rate=32, lookup=0, tag=0, enc=0, kind=0):
    sq = [al.DnaSequence(c) for c in seqs_codes(seqs)]
    return _build(sq, FmIndexConfig(sa_sample_rate=rate, lookup_depth=lookup, occ_encoding=enc, build_threads=2),
                  tag, kind)


def test_builder_matches_oracle_bytes(oracle):
    rng = random.Random(5)
    cases = [(["ACGT"], 1, 0, 0, 0, 0), (["ACGTNACGT"], 4, 3, 1, 0, 0), (["ACGT", "TGCA"], 2, 0, 0, 1, 1)]
    for _ in range(40):
        seqs = _seqs(rng, rng.randint(1, 4), rng.choice(["ACGT", "ACGTN", "ACGTNRYSWKMBDHV"]), 1, 300)
        cases.append((seqs, rng.choice([1, 2, 7, 32]), rng.choice([0, 0, 2, 4]), rng.choice([0, 1]),
                      rng.choice([0, 1]), rng.choice([0, 1])))
    for seqs, rate, lookup, tag, enc, kind in cases:
        want = oracle.build_index_bytes(seqs_codes(seqs), rate=rate, lookup_depth=lookup if kind == 0 or True else 0,
                                        tag=tag, encoding=enc, kind=kind)
        got = product_bytes(seqs, rate, lookup, tag, enc, kind)
        assert got == want, (seqs, rate, lookup, tag, enc, kind)


def test_suffix_array_matches_naive(oracle):
    rng = random.Random(9)
    lib = L.lib()
    for _ in range(60):
        seqs = _seqs(rng, rng.randint(1, 5), rng.choice(["A", "AC", "ACGT", "ACGTN"]), 1, 400)
        text, _ = concat(seqs)
        want = oracle.suffix_array(text)
        got = np.zeros(len(text), dtype=np.uint32)
        t = np.ascontiguousarray(text, dtype=np.uint8)
        assert lib.hfm_suffix_array(L.ptr(t, L.u8p), len(t), L.ptr(got, L.u32p)) == 0
        assert np.array_equal(got, want)


def _load_status(data: bytes, kind: int):
    buf = np.frombuffer(data, dtype=np.uint8).copy() if data else np.zeros(1, np.uint8)
    h = C.c_void_p()
    return L.lib().hfm_index_load(L.ptr(buf, L.u8p), len(data), kind, None, C.byref(h))


def test_malformed_bincode_rejected_before_device_work():
    good = product_bytes(["ACGTACGT"], rate=4)
    assert _load_status(good[:-1] + b"\xff", KIND_FM) == HFM_E_FORMAT       # unknown alphabet tag
    assert _load_status(good[:50], KIND_FM) == HFM_E_FORMAT                 # truncated
    bad_c = bytearray(good); bad_c[4] ^= 1                                   # C array inconsistent
    assert _load_status(bytes(bad_c), KIND_FM) == HFM_E_FORMAT
    bidir = product_bytes(["ACGT", "TTGA"], kind=1)
    assert _load_status(bidir[:3], KIND_BIDIR) == HFM_E_FORMAT
    assert _load_status(bidir[:200], KIND_BIDIR) == HFM_E_FORMAT
    assert _load_status(good, 7) == HFM_E_ARG


def test_build_rejects_bad_input():
    with pytest.raises(Exception):
        _build([], FmIndexConfig(), 0, KIND_FM)
    with pytest.raises(Exception):
        _build([al.DnaSequence(np.array([1, 0, 2], np.uint8))], FmIndexConfig(), 0, KIND_FM)


def test_null_arguments_rejected_without_a_gpu():
    """The scheduling, tuning and cost-model entry points reject missing handles and
    outputs with HFM_E_ARG and a message, before touching a device."""
    import ctypes as C
    from haystackfm_b200 import _lib as L
    lib = L.lib()
    E_ARG = -4
    dm = L.HfmDevMems()
    sc = L.HfmSched(None, 0, 0, None)
    t = L.HfmTuning(3, 512, 1, 1)
    assert lib.hfm_mems_batch_device_sched(None, None, None, 0, 19, 0, None, 0, 64, C.byref(sc), C.byref(dm)) == E_ARG
    assert lib.hfm_get_tuning(None, C.byref(t)) == E_ARG
    assert lib.hfm_set_tuning(None, C.byref(t)) == E_ARG
    assert lib.hfm_autotune_mems(None, None, None, 0, 19, 0, None, 0, 64, 1, C.byref(t), None) == E_ARG
    assert lib.hfm_mlp_create(0, 1, None) == E_ARG
    assert lib.hfm_mlp_set_params(None, None) == E_ARG
    assert lib.hfm_mlp_get_params(None, None) == E_ARG
    assert lib.hfm_mlp_forward(None, None, 0, None) == E_ARG
    assert lib.hfm_mlp_train(None, None, None, 0, 1, 1, 1e-3, 0, None) == E_ARG
    nw = C.c_uint32()
    assert lib.hfm_mlp_schedule(None, None, 0, 0.0, None, C.byref(nw)) == E_ARG
    assert lib.hfm_last_error()                               # a message was set
    lib.hfm_mlp_free(None)                                    # no-ops
    assert lib.hfm_mlp_stream(None) in (None, 0)


def test_oracle_doubling_sort_equals_comparison_sort(oracle):
    """The oracle builds its indices with a prefix-doubling suffix sort (an algorithm
    independent of the product's SA-IS); it must give the comparison sort's order on texts
    with interior sentinels, long runs and periodic stretches."""
    rng = np.random.default_rng(13)
    for trial in range(120):
        n = int(rng.integers(1, 600))
        kind = trial % 4
        if kind == 0:
            t = rng.integers(0, 16, n).astype(np.uint8)
        elif kind == 1:
            t = rng.integers(0, 3, n).astype(np.uint8)
        elif kind == 2:
            t = np.full(n, int(rng.integers(0, 16)), np.uint8)
        else:
            t = np.tile(rng.integers(0, 5, int(rng.integers(1, 9))).astype(np.uint8), n)[:n]
        want = oracle.suffix_array(t)
        for threads in (1, 3):
            assert np.array_equal(oracle.suffix_array_doubling(t, threads), want), (trial, threads)


def test_null_handle_timeout_rejected():
    assert L.lib().hfm_set_timeout(None, 5) == HFM_E_ARG


def test_graph_and_probe_arguments_rejected_without_a_gpu():
    """The graph and probe entry points check their arguments before any device work: a
    missing graph or output, an unsupported probe span, a buffer below 64 MiB."""
    import ctypes as C
    lib = L.lib()
    g = C.c_void_p()
    assert lib.hfm_mems_graph_create(None, None, None, 0, 0, 19, 0, None, 0, 64, 0, C.byref(g)) == HFM_E_ARG
    assert lib.hfm_mems_graph_launch(None, None, None) == HFM_E_ARG
    assert lib.hfm_mems_graph_add_locate(None, None, None, 0, 0, 0, 0) == HFM_E_ARG
    assert lib.hfm_mems_graph_locate_result(None, None) == HFM_E_ARG
    assert lib.hfm_mems_graph_info(None, None, None, None) == HFM_E_ARG
    lib.hfm_mems_graph_free(None)                             # no-op
    gbs = C.c_float()
    assert lib.hfm_probe_gather(0, 1 << 30, 48, C.byref(gbs), None) == HFM_E_ARG
    assert b"span" in lib.hfm_last_error()
    assert lib.hfm_probe_gather(0, 1 << 20, 32, C.byref(gbs), None) == HFM_E_ARG
    assert lib.hfm_probe_gather(0, 1 << 30, 32, None, None) == HFM_E_ARG


def test_malformed_layout_blob_rejected_before_device_work():
    """hfm_index_load_layout checks magic, version, kind and every length against the blob
    before it touches a device: all of these fail with HFM_E_FORMAT on a machine without a
    GPU."""
    import ctypes as C
    from haystackfm_b200.errors import HFM_E_FORMAT
    lib = L.lib()
    h = C.c_void_p()

    def load(blob):
        buf = np.frombuffer(blob, dtype=np.uint8) if blob else np.zeros(1, np.uint8)
        return lib.hfm_index_load_layout(L.ptr(buf, L.u8p), len(blob), None, C.byref(h))
    hdr = np.array([0x444D4648, 1, 1, 2], dtype="<u4").tobytes()
    assert load(b"") == HFM_E_FORMAT
    assert load(b"HFMD") == HFM_E_FORMAT                                   # truncated header
    assert load(np.array([0x12345678, 1, 1, 2], dtype="<u4").tobytes()) == HFM_E_FORMAT   # magic
    assert load(np.array([0x444D4648, 9, 1, 2], dtype="<u4").tobytes()) == HFM_E_FORMAT   # version
    assert load(np.array([0x444D4648, 1, 1, 1], dtype="<u4").tobytes()) == HFM_E_FORMAT   # bidir needs 2
    assert load(hdr) == HFM_E_FORMAT                                       # no direction records
    assert load(hdr + bytes(200)) == HFM_E_FORMAT                          # truncated direction
    assert b"truncated" in lib.hfm_last_error()
    assert load(hdr + bytes(400)) == HFM_E_FORMAT                          # sizes inconsistent
    assert b"inconsistent" in lib.hfm_last_error()
