"""The allocation-free count entry point against the regular one and the oracle.

hfm_count_batch_noalloc exists for callers that cannot let a library allocate GPU memory
(a framework owning the device memory through its own pool, a latency-bound serving loop).
It must give exactly the counts of hfm_count_batch_device (and so of the oracle), call
after call, while keeping its scratch in the library's static device array.  Past its
static limits it must fail with a clear status instead of giving a wrong count.  This
file sorts last so that a failure here comes after every other test has run.

Device calls run on the handle's own non-blocking stream: every device buffer torch
writes is synchronised before the call that reads or overwrites it.
"""
from __future__ import annotations

import numpy as np
import pytest

from haystackfm_b200 import _lib as L
from haystackfm_b200 import alphabet as al
from haystackfm_b200 import synth
from haystackfm_b200.errors import HFM_E_ARG, HFM_E_OVERFLOW
from haystackfm_b200.fm_index import FmIndexConfig, KIND_FM, _Handle, _build

pytestmark = pytest.mark.gpu


def _device_queries(torch, qs):
    flat, off = L.pack_queries(qs)
    dq = torch.from_numpy(flat).cuda()
    doff = torch.from_numpy(off.astype(np.int64)).cuda()
    return flat, off, dq, doff


def _count_device(torch, lib, h, dq, doff, nq):
    out = torch.zeros(nq, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    L.check(lib.hfm_count_batch_device(h.h, dq.data_ptr(), doff.data_ptr(), nq, out.data_ptr()))
    return out.cpu().numpy().view(np.uint32).copy()


def _count_noalloc(torch, lib, h, dq, doff, nq):
    out = torch.full((nq,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.hfm_count_batch_noalloc(h.h, dq.data_ptr(), doff.data_ptr(), nq, out.data_ptr())
    return rc, out.cpu().numpy().view(np.uint32).copy()


def test_noalloc_count_matches_regular_count_twice(oracle):
    import torch
    ref = synth.iupac_reference(total=400_000, n_contigs=8, seed=31)
    reads = synth.sample_reads(ref, n_reads=3000, seed=32)
    data = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=8), 0,
                  KIND_FM)
    h = _Handle(data, KIND_FM)
    lib = L.lib()
    # 32-mers (mostly lookup-seeded) plus all-N and unseeded patterns whose interval sets
    # outgrow the fast pass and go through the long-tail pass
    qs = [r[:32] for r in reads] + [np.full(k, 5, np.uint8) for k in (3, 8, 20)] + \
         [np.concatenate([r[:20], np.full(6, 5, np.uint8)]) for r in reads[:200]]
    flat, off, dq, doff = _device_queries(torch, qs)
    nq = len(qs)
    want = _count_device(torch, lib, h, dq, doff, nq)
    assert np.array_equal(want, oracle.OracleIndex(data, KIND_FM).count_packed(flat, off))
    for _ in range(2):       # the shared scratch keeps the previous call's contents
        rc, got = _count_noalloc(torch, lib, h, dq, doff, nq)
        L.check(rc)
        assert np.array_equal(got, want)
    assert int(want[-1]) > 0
    # more queries than the static work area allows: a clear error, nothing launched
    rc, _ = _count_noalloc(torch, lib, h, dq, doff, 16)
    L.check(rc)
    torch.cuda.synchronize()
    rc = lib.hfm_count_batch_noalloc(h.h, dq.data_ptr(), doff.data_ptr(), (1 << 20) + 1, dq.data_ptr())
    assert rc == HFM_E_ARG and b"exceed" in lib.hfm_last_error()


def test_noalloc_count_reports_set_overflow(oracle):
    """A query whose interval set outgrows the static long-tail area (2,048 intervals):
    all-N patterns over 3,000 short contigs, where every `x..$` suffix breaks the matching
    rows into another interval (4,869 intervals at 8 Ns).  The allocation-free call must
    return HFM_E_OVERFLOW; the regular call (growing work area) still counts exactly."""
    import torch
    rng = np.random.default_rng(41)
    contigs = [rng.integers(1, 5, 200).astype(np.uint8) for _ in range(3000)]
    data = _build([al.DnaSequence(c) for c in contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=0), 0,
                  KIND_FM)
    h = _Handle(data, KIND_FM)
    lib = L.lib()
    qs = [np.full(k, 5, np.uint8) for k in (8, 10)]
    flat, off, dq, doff = _device_queries(torch, qs)
    want = _count_device(torch, lib, h, dq, doff, len(qs))
    assert np.array_equal(want, oracle.OracleIndex(data, KIND_FM).count_packed(flat, off))
    assert int(want[0]) == 3000 * (200 - 8 + 1)
    rc, _ = _count_noalloc(torch, lib, h, dq, doff, len(qs))
    assert rc == HFM_E_OVERFLOW and b"2048" in lib.hfm_last_error()
    # the next call starts from cleared counters and is exact again
    small = [c[:16] for c in contigs[:64]]
    flat2, off2, dq2, doff2 = _device_queries(torch, small)
    rc, got = _count_noalloc(torch, lib, h, dq2, doff2, len(small))
    L.check(rc)
    assert np.array_equal(got, _count_device(torch, lib, h, dq2, doff2, len(small)))
