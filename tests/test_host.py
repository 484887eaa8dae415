"""Host-side logic on CPU: FASTA/FASTQ ingest, batching, and the multi-rank sharding path
(world_size 2 over gloo) with the CPU oracle standing in for the per-rank query."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

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
