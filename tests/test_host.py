"""Host-side logic on CPU: FASTA/FASTQ ingest, batching, and the multi-rank sharding path
(world_size 2 over gloo) with the CPU oracle standing in for the per-rank query."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from haystackfm_b200 import _lib as L
from haystackfm_b200 import alphabet as al
from haystackfm_b200 import io as hio
from haystackfm_b200.errors import FmIndexError
from haystackfm_b200.shard import shard_range


def test_parse_fasta_semantics():
    seqs = hio.parse_fasta(">chr1 desc\nACGT\nAC\n\n>chr2\nNNRY\n")
    assert [s.header() for s in seqs] == ["chr1 desc", "chr2"]
    assert list(seqs[0].as_slice()) == list(al.encode("ACGTAC"))
    plain = hio.parse_fasta("ACGT\n\nTTGA\n")
    assert len(plain) == 2 and plain[0].header() == ""
    with pytest.raises(FmIndexError):
        hio.parse_fasta("\n\n")
    with pytest.raises(FmIndexError):
        hio.parse_fasta(">x\nACXT\n")


def test_fastq_and_encoding():
    recs = hio.parse_fastq("@r1\nACGTN\n+\nIIIII\n@r2\nGGRY\n+\nIIII\n")
    assert recs == [("r1", "ACGTN"), ("r2", "GGRY")]
    flat, off = hio.encode_reads([r for _, r in recs])
    assert list(off) == [0, 5, 9]
    assert list(flat[:5]) == list(al.encode("ACGTN"))
    with pytest.raises(FmIndexError):
        hio.encode_reads(["AC-T"])
    sub_f, sub_o = hio.slice_packed(flat, off, 1, 2)
    assert list(sub_o) == [0, 4] and list(sub_f) == list(al.encode("GGRY"))
    assert list(hio.batches(10, 4)) == [(0, 4), (4, 8), (8, 10)]


def test_shard_ranges_cover_exactly():
    for n in (0, 1, 7, 100):
        for w in (1, 2, 3, 8):
            ranges = [shard_range(n, r, w) for r in range(w)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(ranges[i][1] == ranges[i + 1][0] for i in range(w - 1))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, data, queries, out_dir):
    import torch.distributed as dist
    from oracle import oracle as orc
    from haystackfm_b200.shard import max_over_ranks, run_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    idx = orc.OracleIndex(data, 0)       # every rank holds its own index replica

    def query(a, b):
        return [int(c) for c in idx.count_batch(queries[a:b])]

    res = run_sharded(len(queries), query, dist)
    t = max_over_ranks(float(rank + 1), dist)
    if rank == 0:
        np.save(os.path.join(out_dir, "res.npy"), np.array(res, dtype=np.int64))
        np.save(os.path.join(out_dir, "t.npy"), np.array([t]))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_run_gloo_world2(oracle, tmp_path):
    rng = np.random.default_rng(0)
    ref = "".join(rng.choice(list("ACGTN"), 3000))
    data = oracle.build_index_bytes([al.encode(ref)], rate=8)
    queries = [al.encode(ref[i:i + rng.integers(3, 12)]) for i in rng.integers(0, 2900, 37)]
    want = [int(c) for c in oracle.OracleIndex(data, 0).count_batch(queries)]
    mp.spawn(_worker, args=(2, _free_port(), data, queries, str(tmp_path)), nprocs=2, join=True)
    assert list(np.load(tmp_path / "res.npy")) == want
    assert float(np.load(tmp_path / "t.npy")[0]) == 2.0


def _py_packed_fasta(text):
    seqs = hio.parse_fasta(text)
    flat, off = L.pack_queries([s.as_slice() for s in seqs])
    return flat, off


def test_native_read_parser_matches_python_readers():
    """hfm_parse_reads gives the packed batch of parse_fasta / parse_fastq + encode_reads:
    multi-line and header-less FASTA, blank lines, CRLF, lower case and U, FASTQ with blank
    lines between records, and automatic format detection."""
    fasta = ">r1 x\r\nACGT\r\nac\r\n\r\n>empty\n>r2\n  NNRYu  \n"
    for fmt in ("auto", "fasta"):
        f, o = hio.parse_reads(fasta, fmt)
        pf, po = _py_packed_fasta(fasta)
        assert np.array_equal(o, po) and np.array_equal(f[:int(o[-1])], pf[:int(po[-1])])
    plain = "ACGT\n\nTTGA\nn\n"
    f, o = hio.parse_reads(plain)
    pf, po = _py_packed_fasta(plain)
    assert np.array_equal(o, po) and np.array_equal(f[:int(o[-1])], pf[:int(po[-1])])
    fastq = "@r1\nACGTN\n+\nIIIII\n\n@r2 d\nggry\n+r2\nIIII\n@r3\n\n+\n\n"
    for fmt in ("auto", "fastq"):
        f, o = hio.parse_reads(fastq, fmt)
        pf, po = hio.encode_reads([r for _, r in hio.parse_fastq(fastq)])
        assert np.array_equal(o, po) and np.array_equal(f[:int(o[-1])], pf[:int(po[-1])])
    f, o = hio.parse_reads("", "fastq")
    assert list(o) == [0]


def test_native_read_parser_large_batch_and_errors():
    """A FASTQ batch large enough for the threaded encoding equals the Python encoding;
    bad characters, '$', malformed records and empty FASTA input fail with the reference's
    error kinds and the read and position in the message."""
    rng = np.random.default_rng(5)
    reads = ["".join(rng.choice(list("ACGTNRYacgtu"), int(rng.integers(50, 300)))) for _ in range(60_000)]
    text = "".join(f"@q{i}\n{r}\n+\n{'I' * len(r)}\n" for i, r in enumerate(reads))
    f, o = hio.parse_reads(text, "auto", threads=4)
    pf, po = hio.encode_reads(reads)
    assert np.array_equal(o, po) and np.array_equal(f, pf)
    f, o = hio.parse_reads(text.replace("\n", "\r\n"), "fastq", threads=3)    # stretches cut inside CRLF text
    assert np.array_equal(o, po) and np.array_equal(f, pf)
    bad = text[:-1] + "\n@bad\nACGXT\n+\nIIIII\n"
    with pytest.raises(FmIndexError) as e:
        hio.parse_reads(bad, threads=4)
    assert e.value.kind == "InvalidCharacter" and "'X' at position 3 of read 60000" in str(e.value)
    with pytest.raises(FmIndexError) as e:
        hio.parse_reads(">a\nAC$T\n")
    assert e.value.kind == "InvalidCharacter" and "'$' at position 2 of read 0" in str(e.value)
    with pytest.raises(FmIndexError) as e:
        hio.parse_reads("@r1\nACGT\nIIII\n", "fastq")
    assert e.value.kind == "DeserializeError" and "line 1" in str(e.value)
    with pytest.raises(FmIndexError) as e:
        hio.parse_reads("\n \n>only-header\n")
    assert e.value.kind == "InvalidCharacter"
