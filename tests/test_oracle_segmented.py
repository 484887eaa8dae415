"""The segmented SMEM sweep the library runs on long reads (segment chains, fix-up sweeps
from the previous segment's exit, merge along the true pivot chain) yields the same SMEMs
as the whole-read sweep: checked on the CPU with the oracle's own pivot step, with short
segments so that every read crosses many segment boundaries."""
from __future__ import annotations

import pytest

from haystackfm_b200 import alphabet as al
from haystackfm_b200 import synth
from haystackfm_b200.fm_index import FmIndexConfig, KIND_BIDIR, _build


@pytest.mark.parametrize("genome", ["iupac", "repeats"])
def test_segmented_sweep_equals_whole_read(oracle, genome):
    if genome == "iupac":
        ref = synth.iupac_reference(total=300_000, n_contigs=6, n_run_mean=40, seed=61)
        tag, n_rate = 0, 0.002
    else:
        ref = synth.repeat_reference(total=300_000, n_contigs=3, seed=62)
        tag, n_rate = 1, 0.0
    flat, off, lens = synth.sample_mixed_reads(ref, n_reads=40, short_frac=0.2, long_median=500, max_len=1200,
                                               seed=63, n_rate=n_rate)
    b = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=16, lookup_depth=6), tag,
               KIND_BIDIR)
    o = oracle.OracleIndex(b, KIND_BIDIR)
    for seg_len, min_len in ((32, 12), (64, 19), (160, 19)):
        bad, checked = o.smem_segment_check(flat, off, min_len, seg_len)
        assert checked >= 25 and bad == 0, (seg_len, min_len, bad, checked)
