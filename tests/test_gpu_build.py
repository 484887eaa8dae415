"""GPU index construction (hfm_build_index_gpu) against the CPU builder: the bincode bytes
must be identical — suffix order, BWT, compacted Occ records, sampled SA with forced
sequence starts, lookup table — for both alphabets, both Occ encodings and both index
kinds, on texts with many sequences, long runs and periodic stretches."""
from __future__ import annotations

import random

import numpy as np
import pytest

from haystackfm_b200 import alphabet as al
from haystackfm_b200 import synth
from haystackfm_b200.fm_index import FmIndexConfig, KIND_BIDIR, KIND_FM, _build, _build_gpu

pytestmark = pytest.mark.gpu


def _both(contigs, rate, lookup, tag, enc, kind):
    seqs = [al.DnaSequence(np.asarray(c, dtype=np.uint8)) for c in contigs]
    cfg = FmIndexConfig(sa_sample_rate=rate, lookup_depth=lookup, occ_encoding=enc, build_threads=2)
    return _build(seqs, cfg, tag, kind), _build_gpu(seqs, cfg, tag, kind)


def test_gpu_builder_bytes_equal_cpu_builder_small():
    rng = random.Random(7)
    for trial in range(40):
        alphabet = rng.choice([[1, 2, 3, 4], [1, 2, 3, 4, 5], list(range(1, 16)), [1], [1, 2]])
        tag = 1 if max(alphabet) <= 4 and rng.random() < 0.5 else 0
        contigs = []
        for _ in range(rng.randint(1, 6)):
            n = rng.randint(1, 700)
            kind = rng.random()
            if kind < 0.2:
                c = [rng.choice(alphabet)] * n                            # a run
            elif kind < 0.4:
                unit = [rng.choice(alphabet) for _ in range(rng.randint(1, 9))]
                c = (unit * (n // len(unit) + 1))[:n]                     # periodic
            else:
                c = [rng.choice(alphabet) for _ in range(n)]
            contigs.append(c)
        rate = rng.choice([1, 2, 7, 32])
        lookup = rng.choice([0, 0, 2, 5])
        enc = rng.choice([0, 1])
        kind = rng.choice([KIND_FM, KIND_BIDIR])
        cpu, gpu = _both(contigs, rate, lookup, tag, enc, kind)
        assert gpu == cpu, (trial, rate, lookup, tag, enc, kind)


def test_gpu_builder_bytes_equal_cpu_builder_genomes():
    ref = synth.iupac_reference(total=3_000_000, n_contigs=30, seed=61)
    cpu, gpu = _both(ref.contigs, 32, 10, 0, 0, KIND_BIDIR)
    assert gpu == cpu
    rep = synth.repeat_reference(total=3_000_000, n_contigs=6, seed=62)
    cpu, gpu = _both(rep.contigs, 32, 10, 1, 0, KIND_BIDIR)
    assert gpu == cpu


def test_random_gather_probe_rates():
    """The random-gather probe: every record span gives a finite positive rate, and the
    wider spans move more bytes per second than the 32-byte one (more sectors per miss)."""
    import ctypes as C
    from haystackfm_b200 import _lib as L
    lib = L.lib()
    rates = {}
    for span in (32, 64, 96):
        gbs, ms = C.c_float(), C.c_float()
        L.check(lib.hfm_probe_gather(0, 1 << 30, span, C.byref(gbs), C.byref(ms)))
        assert 0 < gbs.value < 1e5 and ms.value > 0
        rates[span] = gbs.value
    assert rates[64] > rates[32] * 0.8 and rates[96] > rates[32] * 0.8


def test_layout_blob_round_trip(oracle):
    """The device-layout blob: a handle loaded from it answers exactly as the one loaded
    from the bincode (and as the oracle), for both record formats, and exporting it again
    gives the same blob."""
    from haystackfm_b200.fm_index import BidirFmIndex, _Handle
    for tag, ref in ((0, synth.iupac_reference(total=300_000, n_contigs=6, seed=101)),
                     (1, synth.repeat_reference(total=300_000, n_contigs=3, seed=102))):
        data = _build([al.DnaSequence(c) for c in ref.contigs], FmIndexConfig(sa_sample_rate=16, lookup_depth=8), tag,
                      KIND_BIDIR)
        idx = BidirFmIndex.from_bytes(data)
        blob = idx.handle.export_layout()
        h2 = _Handle.from_layout(blob)
        assert h2.export_layout() == blob
        reads = synth.sample_reads(ref, n_reads=500, seed=103)
        flat, off = synth.pack_rows(reads)
        bounds = idx.seq_boundaries()
        want = oracle.OracleIndex(data, KIND_BIDIR).mems_packed(flat, off, 19, 0, bounds, 64, threads=8)
        for hh in (idx.handle, h2):
            got = hh.mems_packed(flat, off, 19, 0, bounds, 64)
            for g, w in zip(got, want):
                assert np.array_equal(g, w)
        k32, o32 = synth.pack_rows(reads, 32)
        a = idx.handle.locate_packed(k32, o32, 100)
        b = h2.locate_packed(k32, o32, 100)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
