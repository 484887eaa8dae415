"""The allocation-free count entry point against the regular one.

hfm_count_batch_noalloc exists for callers that cannot let a library allocate GPU memory
(a framework owning the device memory through its own pool, a latency-bound serving loop).
It must give exactly the counts of hfm_count_batch_device, call after call, while keeping
its scratch in the library's static device array.  This file sorts last so that a failure
here comes after every other test has run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from haystackfm_b200 import _lib as L
from haystackfm_b200 import alphabet as al
from haystackfm_b200 import synth
from haystackfm_b200.errors import HFM_E_ARG
from haystackfm_b200.fm_index import FmIndexConfig, KIND_FM, _Handle, _build

pytestmark = pytest.mark.gpu


def test_noalloc_count_matches_regular_count_twice():
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
    flat, off = L.pack_queries(qs)
    nq = len(qs)
    dq = torch.from_numpy(flat).cuda()
    doff = torch.from_numpy(off.astype(np.int64)).cuda()
    want = torch.zeros(nq, dtype=torch.int32, device="cuda")
    L.check(lib.hfm_count_batch_device(h.h, dq.data_ptr(), doff.data_ptr(), nq, want.data_ptr()))
    want_np = want.cpu().numpy().view(np.uint32)
    for _ in range(2):       # the shared scratch keeps the previous call's contents
        got = torch.full((nq,), -1, dtype=torch.int32, device="cuda")
        L.check(lib.hfm_count_batch_noalloc(h.h, dq.data_ptr(), doff.data_ptr(), nq, got.data_ptr()))
        assert np.array_equal(got.cpu().numpy().view(np.uint32), want_np)
    assert int(want_np[-1]) > 0
    # more queries than the static work area allows: a clear error, nothing launched
    rc = lib.hfm_count_batch_noalloc(h.h, dq.data_ptr(), doff.data_ptr(), (1 << 20) + 1, got.data_ptr())
    assert rc == HFM_E_ARG and b"exceed" in lib.hfm_last_error()
