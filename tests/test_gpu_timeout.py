"""Host-side deadline of a handle: a wait that runs out returns HFM_E_TIMEOUT, the device
work it abandoned finishes on its own (nothing spins on the device), and the next call on
the same handle gives the exact results again."""
from __future__ import annotations

import numpy as np
import pytest

from haystackfm_b200 import _lib as L
from haystackfm_b200 import alphabet as al
from haystackfm_b200 import synth
from haystackfm_b200.errors import FmIndexError, HFM_E_TIMEOUT
from haystackfm_b200.fm_index import BidirFmIndex, FmIndexConfig, KIND_BIDIR, _build

pytestmark = pytest.mark.gpu


def test_deadline_returns_timeout_and_handle_recovers():
    ref = synth.iupac_reference(total=2_000_000, n_contigs=20, seed=51)
    reads = synth.sample_reads(ref, n_reads=100_000, seed=52)
    data = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=32, lookup_depth=10),
                  0, KIND_BIDIR)
    idx = BidirFmIndex.from_bytes(data)
    h = idx.handle
    bounds = idx.seq_boundaries()
    flat, off = synth.pack_rows(reads)
    want = h.mems_packed(flat, off, 19, 0, bounds, 1024)
    lib = L.lib()
    L.check(lib.hfm_set_timeout(h.h, 1))       # 1 ms: far below the search kernel's time
    with pytest.raises(FmIndexError) as e:
        h.mems_packed(flat, off, 19, 0, bounds, 1024)
    assert e.value.status == HFM_E_TIMEOUT
    L.check(lib.hfm_set_timeout(h.h, 0))
    got = h.mems_packed(flat, off, 19, 0, bounds, 1024)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    L.check(lib.hfm_set_timeout(h.h, 60_000))  # a generous deadline changes nothing
    got = h.mems_packed(flat, off, 19, 0, bounds, 1024)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
