"""The CUDA-graph-captured SMEM/MEM chain: replays give the adaptive chain's bytes (and so
the oracle's), for new reads written into the captured input buffers, and a batch that
outgrows a captured capacity is rerun on the adaptive chain and re-captured."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from haystackfm_b200 import _lib as L
from haystackfm_b200 import alphabet as al
from haystackfm_b200 import synth
from haystackfm_b200.fm_index import BidirFmIndex, FmIndexConfig, KIND_BIDIR, _build, device_to_host

pytestmark = pytest.mark.gpu


def _host(dm, nq, dev):
    hoff = device_to_host(dm.d_hit_offsets, nq + 1, "<i8", dev).view(np.uint64)
    hits = device_to_host(dm.d_hits, 8 * dm.n_hits, "<i4", dev).view(np.uint32).reshape(-1, 8)
    pos = device_to_host(dm.d_positions, 2 * dm.n_positions, "<i4", dev).view(np.uint32).reshape(-1, 2)
    return hoff, hits, pos


def _same(a, b):
    for x, y in zip(a, b):
        assert x.shape == y.shape and np.array_equal(x, y)


def _case(ref, tag, seed, oracle):
    import torch
    data = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=10), tag,
                  KIND_BIDIR)
    idx = BidirFmIndex.from_bytes(data)
    h = idx.handle
    lib = L.lib()
    bounds = np.ascontiguousarray(idx.seq_boundaries(), dtype=np.uint32)
    bp = L.ptr(bounds, L.u32p)
    batches = []
    for k in range(3):
        flat, off, _ = synth.sample_mixed_reads(ref, n_reads=600, short_frac=0.9, long_median=1500, max_len=3000,
                                                seed=seed + k, n_rate=0.0)
        batches.append((flat, off))
    nq = 600
    cap_bases = max(int(b[1][-1]) for b in batches)
    q_d = torch.zeros(cap_bases + 16, dtype=torch.uint8, device="cuda")
    o_d = torch.zeros(nq + 1, dtype=torch.int64, device="cuda")

    def load(b):
        flat, off = b
        q_d[:len(flat)] = torch.from_numpy(flat).cuda()
        o_d.copy_(torch.from_numpy(off.view(np.int64)).cuda())
        torch.cuda.synchronize()

    def adaptive():
        dm = L.HfmDevMems()
        torch.cuda.synchronize()
        L.check(lib.hfm_mems_batch_device(h.h, q_d.data_ptr(), o_d.data_ptr(), nq, 19, 0, bp, len(bounds), 64,
                                          C.byref(dm)))
        return _host(dm, nq, 0)

    load(batches[0])
    want0 = adaptive()
    o = oracle.OracleIndex(data, KIND_BIDIR)
    _same(want0, o.mems_packed(*batches[0], 19, 0, bounds, 64, threads=8))
    return h, lib, bounds, bp, batches, nq, q_d, o_d, load, adaptive, want0, cap_bases


@pytest.mark.parametrize("kind", ["iupac", "exact"])
def test_graph_replays_and_falls_back(oracle, kind):
    if kind == "iupac":
        ref = synth.iupac_reference(total=2_000_000, n_contigs=20, n_run_mean=60, seed=71)
        tag = 0
    else:
        ref = synth.repeat_reference(total=2_000_000, n_contigs=4, seed=72)
        tag = 1
    h, lib, bounds, bp, batches, nq, q_d, o_d, load, adaptive, want0, cap_bases = _case(ref, tag, 73, oracle)
    npos0 = len(want0[2])
    g = C.c_void_p()
    L.check(lib.hfm_mems_graph_create(h.h, q_d.data_ptr(), o_d.data_ptr(), nq, cap_bases, 19, 0, bp, len(bounds), 64,
                                      2 * npos0 + 4096, C.byref(g)))
    try:
        rep = C.c_uint32()
        for b in (0, 1, 2, 0):
            load(batches[b])
            want = adaptive()
            dm = L.HfmDevMems()
            L.check(lib.hfm_mems_graph_launch(g, C.byref(dm), C.byref(rep)))
            _same(_host(dm, nq, 0), want)
            assert rep.value in (0, 1)
        dm = L.HfmDevMems()
        L.check(lib.hfm_mems_graph_launch(g, C.byref(dm), C.byref(rep)))
        n_rep, n_fb, why = C.c_uint32(), C.c_uint32(), C.c_uint32()
        L.check(lib.hfm_mems_graph_info(g, C.byref(n_rep), C.byref(n_fb), C.byref(why)))
        # captured capacities hold (re-captured after any fallback): the replay's outputs
        assert rep.value == 1 and why.value == 0, (n_rep.value, n_fb.value, why.value)
        _same(_host(dm, nq, 0), want)
    finally:
        lib.hfm_mems_graph_free(g)
    # a capacity too small for the batch: rerun on the adaptive chain, then captured again
    if npos0 > 8192:
        g = C.c_void_p()
        L.check(lib.hfm_mems_graph_create(h.h, q_d.data_ptr(), o_d.data_ptr(), nq, cap_bases, 19, 0, bp, len(bounds),
                                          64, 0, C.byref(g)))
        try:
            load(batches[0])
            rep = C.c_uint32()
            dm = L.HfmDevMems()
            L.check(lib.hfm_mems_graph_launch(g, C.byref(dm), C.byref(rep)))
            assert rep.value == 0
            _same(_host(dm, nq, 0), want0)
            dm = L.HfmDevMems()
            L.check(lib.hfm_mems_graph_launch(g, C.byref(dm), C.byref(rep)))
            assert rep.value == 1
            _same(_host(dm, nq, 0), want0)
        finally:
            lib.hfm_mems_graph_free(g)


def test_shared_handles_run_concurrently(oracle):
    """Handles sharing one device-resident index (hfm_index_share), driven from two host
    threads at once, give the parent's (and the oracle's) bytes; freeing the shares leaves
    the parent usable."""
    import threading
    ref = synth.iupac_reference(total=1_000_000, n_contigs=10, n_run_mean=60, seed=81)
    data = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=10), 0,
                  KIND_BIDIR)
    idx = BidirFmIndex.from_bytes(data)
    bounds = idx.seq_boundaries()
    reads = synth.sample_reads(ref, n_reads=3000, seed=82)
    flat, off = synth.pack_rows(reads)
    want = oracle.OracleIndex(data, KIND_BIDIR).mems_packed(flat, off, 19, 0, bounds, 64, threads=8)
    shares = [idx.handle.share() for _ in range(2)]
    got = [None, None]

    def run(k):
        got[k] = [shares[k].mems_packed(flat, off, 19, 0, bounds, 64) for _ in range(3)]
    ts = [threading.Thread(target=run, args=(k,)) for k in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for k in range(2):
        for r in got[k]:
            _same(r, want)
    del shares, got
    _same(idx.handle.mems_packed(flat, off, 19, 0, bounds, 64), want)


def _host_hits(h, dev):
    counts = device_to_host(h.d_counts, h.nq, "<i4", dev).view(np.uint32)
    offs = device_to_host(h.d_offsets, h.nq + 1, "<i8", dev).view(np.uint64)
    pairs = device_to_host(h.d_pairs, 2 * h.total, "<i4", dev).view(np.uint32).reshape(-1, 2)
    return counts, offs, pairs


def test_graph_with_locate_chain(oracle):
    """The locate chain captured ahead of the SMEM chain: one replay gives the locate CSR of
    hfm_locate_batch_device and of the oracle, and the SMEM outputs as before; a batch of
    patterns whose positions outgrow the locate capacity (all-N runs over an IUPAC reference)
    reruns both chains adaptively, with the same bytes, and then replays."""
    import torch
    ref = synth.iupac_reference(total=2_000_000, n_contigs=20, n_run_mean=60, seed=91)
    h, lib, bounds, bp, batches, nq, q_d, o_d, load, adaptive, want0, cap_bases = _case(ref, 0, 93, oracle)
    data = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=10), 0,
                  KIND_BIDIR)
    orc = oracle.OracleIndex(data, KIND_BIDIR)
    rng = np.random.default_rng(94)
    reads = synth.sample_reads(ref, n_reads=2000, seed=95)
    kmers = [r[:32] for r in reads]
    plain = kmers[:1500] + [r[40:52] for r in reads[:500]]          # few positions each
    heavy = kmers[:1460] + [np.full(int(k), 5, np.uint8) for k in rng.integers(2, 5, 40)] + \
        [r[40:52] for r in reads[:500]]                               # all-N: many positions
    lq = len(plain)
    assert len(heavy) == lq
    packed = [L.pack_queries(q) for q in (plain, heavy)]
    lcap = max(int(p[1][-1]) for p in packed)
    lq_d = torch.zeros(lcap + 16, dtype=torch.uint8, device="cuda")
    lo_d = torch.zeros(lq + 1, dtype=torch.int64, device="cuda")

    def lload(k):
        flat, off = packed[k]
        lq_d[:len(flat)] = torch.from_numpy(flat).cuda()
        lo_d.copy_(torch.from_numpy(off.astype(np.int64)).cuda())
        torch.cuda.synchronize()

    def ladaptive():
        r = L.HfmDevHits()
        torch.cuda.synchronize()
        L.check(lib.hfm_locate_batch_device(h.h, lq_d.data_ptr(), lo_d.data_ptr(), lq, 256, C.byref(r)))
        return _host_hits(r, 0)

    lload(0)
    lwant = ladaptive()
    _same(lwant, orc.locate_packed(*packed[0], 256, threads=8))
    g = C.c_void_p()
    L.check(lib.hfm_mems_graph_create(h.h, q_d.data_ptr(), o_d.data_ptr(), nq, cap_bases, 19, 0, bp, len(bounds), 64,
                                      2 * len(want0[2]) + 4096, C.byref(g)))
    try:
        L.check(lib.hfm_mems_graph_add_locate(g, lq_d.data_ptr(), lo_d.data_ptr(), lq, 256, 0,
                                              2 * len(lwant[2]) + 1024))
        rep = C.c_uint32()
        why = C.c_uint32()
        load(batches[0])
        for k in (0, 1, 1, 0):
            lload(k)
            lw = ladaptive()
            if k == 1:
                _same(lw, orc.locate_packed(*packed[1], 256, threads=8))
                assert len(lw[2]) > 2 * len(lwant[2]) + 1024
            dm = L.HfmDevMems()
            L.check(lib.hfm_mems_graph_launch(g, C.byref(dm), C.byref(rep)))
            L.check(lib.hfm_mems_graph_info(g, None, None, C.byref(why)))
            lr = L.HfmDevHits()
            L.check(lib.hfm_mems_graph_locate_result(g, C.byref(lr)))
            _same(_host_hits(lr, 0), lw)
            _same(_host(dm, nq, 0), want0)
            if k == 1 and rep.value == 0:
                assert why.value & 64       # HFM_GRAPH_LOCATE
        assert rep.value == 1 and why.value == 0
        assert lib.hfm_mems_graph_add_locate(g, lq_d.data_ptr(), lo_d.data_ptr(), lq, 256, 0, 0) != 0
    finally:
        lib.hfm_mems_graph_free(g)


def test_graph_with_prefix_order(oracle):
    """A handle tuned to the prefix queue order (read_order 1): the captured chain sorts the
    reads inside the graph and its replays give the adaptive chain's bytes."""
    ref = synth.iupac_reference(total=2_000_000, n_contigs=20, n_run_mean=60, seed=131)
    h, lib, bounds, bp, batches, nq, q_d, o_d, load, adaptive, want0, cap_bases = _case(ref, 0, 133, oracle)
    h.set_tuning(3, 512, 1, 1, 1)
    g = C.c_void_p()
    L.check(lib.hfm_mems_graph_create(h.h, q_d.data_ptr(), o_d.data_ptr(), nq, cap_bases, 19, 0, bp, len(bounds), 64,
                                      2 * len(want0[2]) + 4096, C.byref(g)))
    try:
        rep = C.c_uint32()
        for b in (0, 1, 2, 1):
            load(batches[b])
            want = adaptive()
            dm = L.HfmDevMems()
            L.check(lib.hfm_mems_graph_launch(g, C.byref(dm), C.byref(rep)))
            _same(_host(dm, nq, 0), want)
        assert rep.value == 1
    finally:
        lib.hfm_mems_graph_free(g)
        h.set_tuning(3, 512, 1, 1, 0)
