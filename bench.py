#!/usr/bin/env python
"""SMEM+locate reads/s on one B200 — the IUPAC batch locate + SMEM workload.

Workload (one step): 1,000,000 reads of 150 bp against a 100 Mbp synthetic reference of
200 contigs (lognormal lengths mu=13 sigma=1; uniform ACGT, N runs over 2% with geometric
lengths of mean 500, 0.5% single ambiguity codes); reads from either strand with 1%
substitutions and 0.1% N; IupacDna, sa_sample_rate 32, lookup_depth 10.  Per read: locate
of its first 32-mer (max 1024 positions per merged interval) and find_smems with
min_len 19 and max_hits_per_mem 1024, positions mapped to the reference boundaries.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--reads R]

`value` is device-resident throughput (reads in HBM before the timed region, results left
in HBM); `e2e` goes through the C ABI with host buffers (H2D of the reads from pinned
memory and D2H of every result inside the timed region).  After timing, the outputs of the
timed calls for the first PARITY_READS reads are compared byte for byte with the CPU
oracle (`parity` in the line; a mismatch exits non-zero).  --impl reference times the CPU
restatement of the reference path on the host cores (the Rust reference cannot be built
here) on an index the oracle builds itself, without loading libhfm.so.  Both arms time the
same CPU_SAMPLE reads.  Multi-GPU: one process per GPU, each with its own index replica and
its own 1M reads (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SMEM+locate reads/s on 1 B200, learned-binned vs plain (bit-exact); p99 latency"
PARITY_READS = 65_536      # timed outputs of these reads are byte-compared with the oracle
CPU_SAMPLE = 8_192         # reads both CPU legs time (the reference arm: one pass per step)
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--reads", type=int, default=1_000_000)
    ap.add_argument("--ref-len", type=int, default=100_000_000)
    ap.add_argument("--contigs", type=int, default=200)
    ap.add_argument("--e2e-chunk", type=int, default=125_000)
    ap.add_argument("--e2e-streams", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="time the plain order only")
    ap.add_argument("--train-reads", type=int, default=1_000_000,
                    help="reads (a separate seeded sample) whose logged work trains the cost model")
    ap.add_argument("--train-epochs", type=int, default=4)
    ap.add_argument("--no-genome", action="store_true", help="skip the 3.1 Gbp genome workloads")
    ap.add_argument("--no-plain-launch", action="store_true", help="skip timing the plain launch baseline")
    ap.add_argument("--no-graph", action="store_true", help="skip the CUDA-graph chain measurement")
    ap.add_argument("--genome-len", type=int, default=3_100_000_000)
    ap.add_argument("--genome-reads", type=int, default=2_000_000, help="mixed-length reads (uneven, training)")
    ap.add_argument("--eval-reads", type=int, default=10_000_000, help="held-out 150 bp reads")
    ap.add_argument("--eval-mixed", type=int, default=1_000_000, help="held-out mixed-length reads")
    ap.add_argument("--genome-steps", type=int, default=2)
    ap.add_argument("--genome-parity", type=int, default=2048, help="reads per set checked against the oracle")
    ap.add_argument("--no-serving", action="store_true", help="skip the batch-latency measurement")
    ap.add_argument("--serving-batches", type=int, default=1000)
    ap.add_argument("--serving-workers", type=int, default=3)
    ap.add_argument("--read-order", type=int, default=1,
                    help="read_order of the profile modes (1: the autotuner's choice on the IUPAC workload)")
    ap.add_argument("--profile-step", action="store_true",
                    help="only the W + K headline steps (the launch-list command)")
    ap.add_argument("--profile-smem", action="store_true",
                    help="one SMEM search launch (no position resolve) for ncu, then its work counters")
    return ap.parse_args()


def bench_config(args, world):
    """The workload's config dict: identical, key for key, in both arms."""
    return {"workload": "iupac_batch_locate_smem", "reads_per_step_per_gpu": args.reads, "read_len": 150,
            "ref_len": args.ref_len, "contigs": args.contigs, "alphabet": "IupacDna", "sa_sample_rate": 32,
            "lookup_depth": 10, "min_len": 19, "max_hits_per_mem": 1024, "locate_kmer": 32,
            "seeds": {"reference": 2, "reads": 3}, "parallelism": f"replicas{world}" if world > 1 else "single",
            "l2": "no flush: index (0.7 GB device layout) + reads (150 MB) + outputs exceed the 126 MB L2"}


def iupac_inputs(args, rank=0):
    """Seeded reference and reads of the workload (numpy only: loads no native library)."""
    from haystackfm_b200 import synth
    ref = synth.iupac_reference(total=args.ref_len, n_contigs=args.contigs, seed=2)
    reads = synth.sample_reads(ref, n_reads=args.reads, seed=3 + rank)
    return ref, reads


def workload(args, rank=0):
    from haystackfm_b200 import alphabet as al
    from haystackfm_b200.fm_index import FmIndexConfig, KIND_BIDIR, _build
    key = hashlib.sha1(f"iupac-v1-{args.ref_len}-{args.contigs}-2-rate32-lut10".encode()).hexdigest()[:16]
    cache_dir = os.path.join(tempfile.gettempdir(), "hfm_bench_cache")
    os.makedirs(cache_dir, exist_ok=True)
    path = os.path.join(cache_dir, key + ".bin")
    ref, reads = iupac_inputs(args, rank)
    t0 = time.time()
    if os.path.exists(path):
        data = open(path, "rb").read()
        built = False
    else:
        data = _build([al.DnaSequence(c) for c in ref.contigs],
                      FmIndexConfig(sa_sample_rate=32, lookup_depth=10, build_threads=os.cpu_count() or 1), 0,
                      KIND_BIDIR)
        tmp = path + f".{os.getpid()}"
        with open(tmp, "wb") as f:
            f.write(data)
        os.replace(tmp, path)
        built = True
    build_s = time.time() - t0
    return ref, data, reads, build_s, built


def native_libs_loaded():
    """Shared objects of this repository mapped into the process (from /proc/self/maps)."""
    try:
        maps = open("/proc/self/maps").read()
    except OSError:
        return None
    return sorted({ln.split()[-1] for ln in maps.splitlines() if ln.endswith(".so") and ROOT in ln})


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def cpu_time(o, reads, bounds, threads):
    """Oracle (C++ restatement of the reference CPU path) over `reads`: locate of the first
    32-mer (cap 1024) + find_smems (min_len 19, max_hits 1024).  -> (seconds, outputs)."""
    from haystackfm_b200 import synth
    t0 = time.perf_counter()
    f32, o32 = synth.pack_rows(reads, 32)
    loc = o.locate_packed(f32, o32, 1024, threads)
    fr, orr = synth.pack_rows(reads)
    mems = o.mems_packed(fr, orr, 19, 0, bounds, 1024, threads)
    return time.perf_counter() - t0, loc, mems


def run_reference(args):
    """The reference arm: the oracle builds its own index (prefix-doubling suffix sort, no
    code of libhfm.so) and times CPU_SAMPLE reads per step on every host core."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle import oracle as orc
    orc.build()
    threads = os.cpu_count() or 1
    ref, reads = iupac_inputs(args)
    t0 = time.time()
    orc.set_build_threads(threads)
    data = orc.build_index_bytes(ref.contigs, rate=32, lookup_depth=10, tag=0, kind=1)
    build_s = time.time() - t0
    o = orc.OracleIndex(data, 1)
    bounds = _bounds_of(data)
    sample = reads[:CPU_SAMPLE]
    for _ in range(args.warmup):
        cpu_time(o, sample[:max(256, CPU_SAMPLE // 8)], bounds, threads)
    tot_t = 0.0
    for _ in range(args.steps):
        dt, _, _ = cpu_time(o, sample, bounds, threads)
        tot_t += dt
    value = len(sample) * args.steps / tot_t
    libs = native_libs_loaded()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "reads/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded generators, haystackfm_b200/synth.py)",
        "config": bench_config(args, world),
        "cpu_baseline": {"value": value, "unit": "reads/s", "cores": threads, "kind": "port",
                         "sample": f"the first {len(sample)} reads of the workload each step (locate of the 32-mer "
                                   f"+ find_smems), oracle/hfm_oracle.cpp (the Rust reference cannot be built "
                                   f"here), {threads} threads"},
        "e2e": {"value": value, "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "index": {"builder": "oracle (prefix-doubling suffix sort)", "build_s": round(build_s, 1),
                  "sha256": hashlib.sha256(data).hexdigest()},
        "native_libs": libs,
    }
    if libs and any("libhfm" in x for x in libs):
        raise SystemExit("reference arm loaded libhfm.so")
    print(json.dumps(line), flush=True)


def _bounds_of(data):
    """seq_boundaries of the forward index inside BidirFmIndex bincode (struct only)."""
    import struct
    o = 4 + 64 + 2 + 32
    (n,) = struct.unpack_from("<Q", data, o); o += 8 + 4 * n
    (n,) = struct.unpack_from("<Q", data, o); o += 8 + n
    o += 16
    (n,) = struct.unpack_from("<Q", data, o); o += 8 + n
    (n,) = struct.unpack_from("<Q", data, o); o += 8 + 4 * n
    o += 16
    (n,) = struct.unpack_from("<Q", data, o); o += 8
    return np.frombuffer(data, dtype="<u4", count=n, offset=o).copy()


def gpu_prefix_outputs(h, lib, L, dev, k32_d, off32_d, reads_d, off_d, n, bounds, npre):
    """Runs the timed step's two calls once more and copies the outputs of the first `npre`
    reads (a prefix of each CSR) to the host, in the oracle's array format."""
    from haystackfm_b200.fm_index import device_to_host as d2h
    nb = len(bounds)
    dh = L.HfmDevHits()
    L.check(lib.hfm_locate_batch_device(h.h, k32_d.data_ptr(), off32_d.data_ptr(), n, 1024, C.byref(dh)))
    offs = d2h(dh.d_offsets, npre + 1, "<i8", dev).view(np.uint64)
    counts = d2h(dh.d_counts, npre, "<i4", dev).view(np.uint32)
    pairs = d2h(dh.d_pairs, 2 * int(offs[-1]), "<i4", dev).view(np.uint32).reshape(-1, 2)
    dm = L.HfmDevMems()
    L.check(lib.hfm_mems_batch_device(h.h, reads_d.data_ptr(), off_d.data_ptr(), n, 19, 0, L.ptr(bounds, L.u32p),
                                      nb, 1024, C.byref(dm)))
    hoff = d2h(dm.d_hit_offsets, npre + 1, "<i8", dev).view(np.uint64)
    hits = d2h(dm.d_hits, 8 * int(hoff[-1]), "<i4", dev).view(np.uint32).reshape(-1, 8)
    npos = 0
    if len(hits):
        last = hits[-1]
        npos = (int(last[6]) | (int(last[7]) << 32)) + int(last[5])
    pos = d2h(dm.d_positions, 2 * npos, "<i4", dev).view(np.uint32).reshape(-1, 2)
    return (counts, offs, pairs), (hoff, hits, pos)


def device_mems_tensors(torch, dev, dm, n, clone):
    """hfm_dev_mems outputs as torch views (or copies) of the library's device arrays."""
    from haystackfm_b200.fm_index import _DeviceArray

    def view(ptr, k, ts):
        if k == 0:
            return torch.zeros(0, dtype=torch.int32, device=dev)
        t = torch.as_tensor(_DeviceArray(int(ptr), int(k), ts), device=dev)
        return t.clone() if clone else t
    return (view(dm.d_hit_offsets, n + 1, "<i8"), view(dm.d_hits, 8 * dm.n_hits, "<i4"),
            view(dm.d_positions, 2 * dm.n_positions, "<i4"))


def device_hits_tensors(torch, dev, dh):
    """Views of a locate result's device arrays (counts, offsets, pairs) as torch tensors."""
    from haystackfm_b200.fm_index import _DeviceArray
    n = dh.nq

    def view(ptr, k, ts):
        if k == 0:
            return torch.zeros(0, dtype=torch.int32, device=dev)
        return torch.as_tensor(_DeviceArray(int(ptr), int(k), ts), device=dev)
    return (view(dh.d_counts, n, "<i4"), view(dh.d_offsets, n + 1, "<i8"), view(dh.d_pairs, 2 * dh.total, "<i4"))


def compare_outputs(got, want):
    """Byte comparison of (locate, mems) output tuples; -> list of differing arrays."""
    names = [("locate", ("counts", "offsets", "pairs")), ("mems", ("hit_offsets", "hits", "positions"))]
    bad = []
    for (grp, fields), g, w in zip(names, got, want):
        for f, a, b in zip(fields, g, w):
            if a.shape != b.shape or not np.array_equal(a, b):
                bad.append(f"{grp}.{f}")
    return bad


def profile_smem(args):
    """One SMEM search pass without position resolve (the launch ncu captures), then the
    same pass with work counters to report its Occ touches."""
    import torch
    from haystackfm_b200 import _lib as L
    from haystackfm_b200.fm_index import BidirFmIndex
    _, data, reads, _, _ = workload(args)
    idx = BidirFmIndex.from_bytes(data)
    h, lib, n = idx.handle, L.lib(), args.reads
    h.set_tuning(3, 512, 1, 1, args.read_order)
    rd = torch.from_numpy(reads.reshape(-1)).cuda()
    off = torch.arange(0, (n + 1) * 150, 150, dtype=torch.int64, device="cuda")
    dm = L.HfmDevMems()
    L.check(lib.hfm_mems_batch_device(h.h, rd.data_ptr(), off.data_ptr(), n, 19, 0, None, 0, 1024, C.byref(dm)))
    s = h.stats()
    h.set_counters(True)
    L.check(lib.hfm_mems_batch_device(h.h, rd.data_ptr(), off.data_ptr(), n, 19, 0, None, 0, 1024, C.byref(dm)))
    print(json.dumps({"profile": "smem_search", "reads": n, "k_mems_ms": s.ms_search_kernel,
                      "fallback_reads": s.fallback_reads, "mem_hits": dm.n_hits,
                      "occ_touches": h.stats().occ_touches}), flush=True)


def profile_step(args):
    """W untimed and K timed headline steps (locate of the 32-mer + find_smems over the
    batch, plain order, default tuning) and nothing else: the command the launch list
    (one ncu metric, every launch) is taken from."""
    import torch
    from haystackfm_b200 import _lib as L
    from haystackfm_b200.fm_index import BidirFmIndex
    _, data, reads, _, _ = workload(args)
    idx = BidirFmIndex.from_bytes(data)
    h, lib, n = idx.handle, L.lib(), args.reads
    h.set_tuning(3, 512, 1, 1, args.read_order)
    bounds = np.ascontiguousarray(idx.seq_boundaries(), dtype=np.uint32)
    rd = torch.from_numpy(reads.reshape(-1)).cuda()
    off = torch.arange(0, (n + 1) * 150, 150, dtype=torch.int64, device="cuda")
    k32 = torch.from_numpy(np.ascontiguousarray(reads[:, :32]).reshape(-1)).cuda()
    off32 = torch.arange(0, (n + 1) * 32, 32, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    launches = []
    for k in range(args.warmup + args.steps):
        dh, dm = L.HfmDevHits(), L.HfmDevMems()
        L.check(lib.hfm_locate_batch_device(h.h, k32.data_ptr(), off32.data_ptr(), n, 1024, C.byref(dh)))
        s1 = h.stats()
        L.check(lib.hfm_mems_batch_device(h.h, rd.data_ptr(), off.data_ptr(), n, 19, 0, L.ptr(bounds, L.u32p),
                                          len(bounds), 1024, C.byref(dm)))
        s2 = h.stats()
        launches.append(sum(s.search_launches + s.resolve_launches + s.other_launches for s in (s1, s2)))
    torch.cuda.synchronize()
    print(json.dumps({"profile": "headline_step", "reads": n, "warmup": args.warmup, "steps": args.steps,
                      "launches_per_step": launches, "mem_hits": dm.n_hits, "mem_positions": dm.n_positions,
                      "locate_positions": dh.total}), flush=True)


def ingest_bench(reads):
    """The workload's reads as FASTQ text (307 bytes a record), parsed and encoded by
    hfm_parse_reads on every host core, best of three: -> rate and a byte comparison of
    the packed batch with the reads."""
    from haystackfm_b200 import io as hio
    n, m = reads.shape
    sym = np.frombuffer(b"$ACGTNRYSWKMBDHV", dtype=np.uint8)
    rec = np.empty((n, m * 2 + 7), dtype=np.uint8)
    rec[:, 0:3] = np.frombuffer(b"@r\n", dtype=np.uint8)
    rec[:, 3:3 + m] = sym[reads]
    rec[:, 3 + m:6 + m] = np.frombuffer(b"\n+\n", dtype=np.uint8)
    rec[:, 6 + m:6 + 2 * m] = ord("I")
    rec[:, 6 + 2 * m] = ord("\n")
    text = rec.tobytes()
    best = None
    for _ in range(3):
        t0 = time.perf_counter()
        flat, off = hio.parse_reads(text, "fastq")
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    equal = len(off) == n + 1 and bool(np.array_equal(flat, reads.reshape(-1)))
    return {"format": "FASTQ", "bytes": len(text), "reads": n, "s": round(best, 3),
            "reads_per_s": round(n / best), "gb_per_s": round(len(text) / best / 1e9, 2),
            "threads": os.cpu_count(), "equal": equal,
            "path": "hfm_parse_reads (text -> packed codes + offsets), the input of hfm_locate_batch / hfm_mems_batch"}


def serving_latency(h, lib, L, kp, rp, bounds, n, n_batches, seed=17):
    """Batch latency through the host-buffer C ABI: batches of log-uniform size 1..100,000
    reads (mean ~8.7k) taken from the workload's reads, each a locate of the first 32-mer
    plus find_smems with every result copied back, issued back to back on one handle.
    -> p50 / p99 / max latency per batch and the sustained reads/s."""
    rng = np.random.default_rng(seed)
    sizes = np.minimum(np.exp(rng.uniform(0, np.log(100_000), n_batches)).astype(np.int64), n)
    starts = rng.integers(0, n - sizes + 1)
    nb = len(bounds)
    lat = []
    t_all = time.perf_counter()
    for a, m in zip(starts, sizes):
        a, m = int(a), int(m)
        off150 = np.arange(0, (m + 1) * 150, 150, dtype=np.uint64)
        off32 = np.arange(0, (m + 1) * 32, 32, dtype=np.uint64)
        t0 = time.perf_counter()
        res = C.POINTER(L.HfmHits)()
        L.check(lib.hfm_locate_batch(h.h, L.ptr(kp[a * 32:], L.u8p), L.ptr(off32, L.u64p), m, 1024, C.byref(res)))
        mo = C.POINTER(L.HfmMemOut)()
        L.check(lib.hfm_mems_batch(h.h, L.ptr(rp[a * 150:], L.u8p), L.ptr(off150, L.u64p), m, 19, 0,
                                   L.ptr(bounds, L.u32p), nb, 1024, C.byref(mo)))
        lat.append((time.perf_counter() - t0) * 1e3)
        lib.hfm_free(res)
        lib.hfm_free(mo)
    total_s = time.perf_counter() - t_all
    lat = np.array(lat)
    return {"batches": int(n_batches), "batch_reads": "log-uniform 1..100000", "mean_batch": float(sizes.mean()),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat.max()), "reads_per_s": float(sizes.sum() / total_s),
            "path": "hfm_locate_batch + hfm_mems_batch, host buffers, one handle, back to back"}


def serving_loop(h, lib, L, torch, dev, q, off, pool, bounds, n_batches, model, workers, rate=2000.0, seed=17):
    """The serving loop: batches arrive as a Poisson stream (mean `rate` per second) with sizes
    log-uniform in 1..100,000 reads, taken from a pool of mixed-length reads (80% 150 bp, 20%
    long) held in HBM.  A batch is admitted once the predicted output bytes of the batches in
    flight plus its own fit the HBM budget (the free device memory at the start, less a
    margin); admitted batches run on `workers` handles that share the index (their own
    streams and buffers), each as locate of every read's first 32-mer (cap 1024) then
    find_smems (min_len 19, max_hits 1024).  Latency = completion - arrival, on the host
    clock."""
    import queue
    import threading
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_batches))
    sizes = np.minimum(np.exp(rng.uniform(0, np.log(100_000), n_batches)).astype(np.int64), pool)
    sizes = np.maximum(sizes, 1)
    starts = rng.integers(0, pool - sizes + 1)
    nb = len(bounds)
    bp = L.ptr(bounds, L.u32p)
    # first 32 codes of every read of the pool, and their offsets
    lens = (off[1:] - off[:-1])
    idx32 = off[:-1, None] + torch.arange(32, device=dev)[None, :]
    k32 = q[idx32.clamp(max=q.shape[0] - 1)].reshape(-1).contiguous()
    o32 = torch.arange(0, (pool + 1) * 32, 32, dtype=torch.int64, device=dev)
    assert int(lens.min()) >= 32
    # predicted output bytes per read (positions x 8 + MemHits x 32), from the cost model
    y = model.model.predict(q, off, pool)
    per = (torch.expm1(y[:, 2].double().clamp(max=40)) * 8 + torch.expm1(y[:, 1].double().clamp(max=40)) * 32 + 64)
    cum = torch.cat([torch.zeros(1, dtype=torch.float64, device=dev), torch.cumsum(per, 0)]).cpu().numpy()
    free_b, _ = torch.cuda.mem_get_info(dev)
    budget = max(1.0, 0.5 * free_b)
    handles = [h.share() for _ in range(workers)]
    cond = threading.Condition()
    state = {"inflight": 0.0, "max_inflight": 0.0, "waited": 0}
    lat = np.zeros(n_batches)
    svc = np.zeros(n_batches)
    done_t = np.zeros(n_batches)
    work = queue.Queue()
    errors = []

    def worker(hh):
        try:
            while True:
                item = work.get()
                if item is None:
                    return
                i, a, m, est = item
                with cond:
                    if state["inflight"] + est > budget and state["inflight"] > 0:
                        state["waited"] += 1
                    while state["inflight"] + est > budget and state["inflight"] > 0:
                        cond.wait()
                    state["inflight"] += est
                    state["max_inflight"] = max(state["max_inflight"], state["inflight"])
                svc0 = time.perf_counter()
                dh = L.HfmDevHits()
                L.check(lib.hfm_locate_batch_device(hh.h, k32.data_ptr(), o32[a:].data_ptr(), m, 1024, C.byref(dh)))
                dm = L.HfmDevMems()
                L.check(lib.hfm_mems_batch_device(hh.h, q.data_ptr(), off[a:].data_ptr(), m, 19, 0, bp, nb, 1024,
                                                  C.byref(dm)))
                t = time.perf_counter()
                done_t[i] = t
                lat[i] = t - (t0 + arrivals[i])
                svc[i] = t - svc0
                with cond:
                    state["inflight"] -= est
                    cond.notify_all()
        except Exception as e:              # reported after the loop
            errors.append(repr(e))
            with cond:
                cond.notify_all()

    torch.cuda.synchronize()
    ths = [threading.Thread(target=worker, args=(hh,)) for hh in handles]
    for t_ in ths:
        t_.start()
    t0 = time.perf_counter()
    for i in range(n_batches):
        now = time.perf_counter() - t0
        if arrivals[i] > now:
            time.sleep(arrivals[i] - now)
        a, m = int(starts[i]), int(sizes[i])
        work.put((i, a, m, float(cum[a + m] - cum[a])))
    for _ in ths:
        work.put(None)
    for t_ in ths:
        t_.join()
    del handles
    if errors:
        raise RuntimeError("serving worker failed: " + errors[0])
    span = float(done_t.max() - t0)
    return {"batches": int(n_batches), "arrivals": f"Poisson, mean {rate:.1f} batches/s",
            "batch_reads": "log-uniform 1..100000", "mean_batch": float(sizes.mean()),
            "offered_reads_per_s": float(sizes.sum() / arrivals[-1]),
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "max_ms": float(lat.max() * 1e3), "service_p50_ms": float(np.percentile(svc, 50) * 1e3),
            "service_p99_ms": float(np.percentile(svc, 99) * 1e3), "reads_per_s": float(sizes.sum() / span),
            "workers": workers,
            "hbm_budget_gb": round(budget / 1e9, 1), "max_inflight_predicted_gb": round(state["max_inflight"] / 1e9, 2),
            "batches_held_by_admission": int(state["waited"]),
            "path": "hfm_locate_batch_device + hfm_mems_batch_device on handles sharing one device-resident index"}


def genome_workloads(args, device, torch):
    """The uneven-read and learned-predictor workloads on a 3.1 Gbp repeat-rich ACGT genome (ExactDna
    bidirectional index, sa_sample_rate 32, lookup_depth 10, built on the GPU):

    * uneven: 2M mixed-length reads, find_smems (min_len 19, max_hits 1024, positions
      mapped): the persistent work-queue path (autotuned) against the plain
      one-thread-per-read launch with its count pass;
    * learned: the read-cost model trained on the work the exact kernel logs for those
      2M reads, evaluated on 10M held-out 150 bp reads and 1M held-out mixed-length reads:
      prediction error, and the learned path (outputs pre-sized from the predicted totals,
      binned order when it is faster) against the plain launch, outputs compared byte for
      byte;
    * parity: outputs for a read subsample against the CPU oracle on the same index bytes."""
    from haystackfm_b200 import alphabet as al
    from haystackfm_b200 import synth_gpu as sg
    from haystackfm_b200 import _lib as L
    from haystackfm_b200.cost_model import LearnedSmem, prediction_error, work_targets
    from haystackfm_b200.fm_index import BidirFmIndex, FmIndexConfig, KIND_BIDIR, _build_gpu
    from haystackfm_b200.fm_index import device_to_host as d2h
    dev = torch.device("cuda", device)
    out = {"genome": f"{args.genome_len / 1e9:.2f} Gbp ACGT, 24 contigs, 40% interspersed repeats (20 families, "
                     f"300 bp / 6 kbp consensus, 10-20% divergent copies), 5% tandem repeats (period 2-60)",
           "alphabet": "ExactDna", "sa_sample_rate": 32, "lookup_depth": 10, "min_len": 19, "max_hits_per_mem": 1024,
           "data": "synthetic, generated on the GPU (haystackfm_b200/synth_gpu.py, seeds 11/21/22/23)"}
    t0 = time.time()
    genome, gb = sg.repeat_genome(total=args.genome_len, n_contigs=24, seed=11, device=dev)
    r3_q, r3_o = sg.sample_mixed_reads(genome, gb, args.genome_reads, seed=21)
    e150 = sg.sample_reads(genome, gb, args.eval_reads, n_rate=0.0, seed=22)
    em_q, em_o = sg.sample_mixed_reads(genome, gb, args.eval_mixed, seed=23)
    host = genome.cpu().numpy()
    del genome
    torch.cuda.synchronize()
    out["synth_s"] = round(time.time() - t0, 1)
    begins = np.concatenate([[0], gb[:-1]])
    seqs = [al.DnaSequence(host[a:b]) for a, b in zip(begins, gb)]
    torch.cuda.empty_cache()
    t0 = time.time()
    data = _build_gpu(seqs, FmIndexConfig(sa_sample_rate=32, lookup_depth=10), 1, KIND_BIDIR, device=device)
    out["index_build_s"] = round(time.time() - t0, 1)
    out["index_bytes"] = len(data)
    out["index_sha256"] = hashlib.sha256(data).hexdigest()
    del seqs, host
    t0 = time.time()
    idx = BidirFmIndex.from_bytes(data, device=device)
    out["index_load_s"] = round(time.time() - t0, 1)
    h = idx.handle
    # the device-layout blob: export once, then a load without the host record transform
    from haystackfm_b200.fm_index import _Handle
    t0 = time.time()
    blob = h.export_layout()
    out["layout_bytes"] = len(blob)
    out["layout_export_s"] = round(time.time() - t0, 2)
    t0 = time.time()
    h_layout = _Handle.from_layout(blob, device=device)
    out["layout_load_s"] = round(time.time() - t0, 2)
    del h_layout, blob
    lib = L.lib()
    bounds = np.ascontiguousarray(idx.seq_boundaries(), dtype=np.uint32)
    nb = len(bounds)
    bp = L.ptr(bounds, L.u32p)
    stream = torch.cuda.ExternalStream(h.stream(), device=dev)

    def timed(fn, steps, warmup=1):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def mems(q, o, n):
        dm = L.HfmDevMems()
        L.check(lib.hfm_mems_batch_device(h.h, q.data_ptr(), o.data_ptr(), n, 19, 0, bp, nb, 1024, C.byref(dm)))
        return dm

    def with_tuning(variant, fn):
        saved = h.tuning()
        h.set_tuning(variant, saved["seg_len"], saved["queue_chunk"], saved["threads_per_read"])
        try:
            return fn()
        finally:
            h.set_tuning(saved["mems_variant"], saved["seg_len"], saved["queue_chunk"], saved["threads_per_read"])

    n3 = args.genome_reads
    steps = args.genome_steps
    tuning = h.autotune_mems(r3_q, r3_o, n3, 19, 0, bounds, 1024, reps=1)
    ms_persist = timed(lambda: mems(r3_q, r3_o, n3), steps)
    ms_plain = with_tuning(4, lambda: timed(lambda: mems(r3_q, r3_o, n3), steps))
    # the same search as one CUDA-graph replay of the fixed-capacity chain
    dm0 = mems(r3_q, r3_o, n3)
    npos3 = int(dm0.n_positions)
    g = C.c_void_p()
    nbases3 = int(r3_o[-1].item())
    L.check(lib.hfm_mems_graph_create(h.h, r3_q.data_ptr(), r3_o.data_ptr(), n3, nbases3, 19, 0, bp, nb, 1024,
                                      int(npos3 * 1.25) + 4096, C.byref(g)))
    rep = C.c_uint32()
    dmg = L.HfmDevMems()

    def glaunch():
        L.check(lib.hfm_mems_graph_launch(g, C.byref(dmg), C.byref(rep)))

    def host_ms(fn, k, warm=1):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3 / k
    ms_graph = host_ms(glaunch, steps, warm=2)     # a first batch past a capacity re-captures
    g_replayed = int(rep.value)
    snap = device_mems_tensors(torch, dev, dmg, n3, clone=True)
    now = device_mems_tensors(torch, dev, mems(r3_q, r3_o, n3), n3, clone=False)
    g_eq = all(a.shape == b.shape and bool(torch.equal(a, b)) for a, b in zip(snap, now))
    del snap, now
    lib.hfm_mems_graph_free(g)
    ms_adapt_host = host_ms(lambda: mems(r3_q, r3_o, n3), steps)
    out["uneven"] = {"reads": n3, "read_bases": int(r3_o[-1].item()),
                     "graph_ms_host": round(ms_graph, 2), "adaptive_ms_host": round(ms_adapt_host, 2),
                     "graph_last_launch_replayed": g_replayed, "graph_outputs_equal": g_eq,
                     "graph_speedup_vs_plain_launch": round(ms_plain / ms_graph, 3),
                     "mix": "80% 150 bp (1% substitutions), 20% lognormal median 3 kbp up to 10 kbp (8% subs/indels)",
                     "persistent_ms": round(ms_persist, 2), "persistent_reads_per_s": n3 / (ms_persist / 1e3),
                     "plain_launch_ms": round(ms_plain, 2), "plain_launch_reads_per_s": n3 / (ms_plain / 1e3),
                     "speedup_vs_plain_launch": round(ms_plain / ms_persist, 3), "autotuned": tuning}
    # learned: train on the logged work of the 2M reads, evaluate on held-out reads
    ls = LearnedSmem(h, device, seed=1)
    t0 = time.time()
    losses, _, _ = ls.fit(r3_q, r3_o, n3, 19, 0, bounds, 1024, epochs=args.train_epochs, batch=8192, lr=1e-3,
                          calibrate_all=True)
    learned = {"train_reads": n3, "epochs": args.train_epochs, "fit_s": round(time.time() - t0, 1),
               "train_mse": [round(float(v), 4) for v in losses],
               "holdout_error": ls.holdout_error.as_dict() if ls.holdout_error else None,
               "order_enabled": bool(ls.enabled), "calibration": ls.calibration, "presize": True}
    o150 = torch.arange(0, (args.eval_reads + 1) * 150, 150, dtype=torch.int64, device=dev)
    q150 = e150.reshape(-1)
    for name, (q, o, n) in (("eval_150bp", (q150, o150, args.eval_reads)),
                            ("eval_mixed", (em_q, em_o, args.eval_mixed))):
        log = ls.log_work(q, o, n, 19, 0, bounds, 1024)
        _, _, y = ls.plan(q, o, n)
        err = prediction_error(y, work_targets(log)).as_dict()
        del log
        ms_l = timed(lambda: ls.run(q, o, n, 19, 0, bp, nb, 1024), steps)
        dm = ls.run(q, o, n, 19, 0, bp, nb, 1024)
        got = device_mems_tensors(torch, dev, dm, n, clone=True)
        ms_pl = with_tuning(4, lambda: timed(lambda: mems(q, o, n), steps))
        dm = with_tuning(4, lambda: mems(q, o, n))
        ref = device_mems_tensors(torch, dev, dm, n, clone=False)
        eq = all(a.shape == b.shape and bool(torch.equal(a, b)) for a, b in zip(got, ref))
        ms_p = timed(lambda: mems(q, o, n), steps)
        learned[name] = {"reads": n, "prediction_error": err, "learned_ms": round(ms_l, 2),
                         "learned_reads_per_s": n / (ms_l / 1e3), "plain_launch_ms": round(ms_pl, 2),
                         "persistent_unlearned_ms": round(ms_p, 2),
                         "speedup_vs_plain_launch": round(ms_pl / ms_l, 3),
                         "speedup_vs_persistent_unlearned": round(ms_p / ms_l, 3),
                         "outputs_equal_to_plain_launch": eq, "mem_hits": int(dm.n_hits),
                         "mem_positions": int(dm.n_positions)}
        del got, ref
    out["learned"] = learned
    # serving loop on the same device-resident index
    if not args.no_serving and args.serving_batches > 0:
        sv = serving_loop(h, lib, L, torch, dev, em_q, em_o, args.eval_mixed, bounds, args.serving_batches,
                          ls, args.serving_workers)
        # the same stream below capacity: 70% of the throughput the loop sustained above,
        # so that latency is service time plus ordinary queueing, not an unbounded backlog
        sub_rate = 0.7 * sv["reads_per_s"] / max(1.0, sv["mean_batch"])
        sv["below_capacity"] = serving_loop(h, lib, L, torch, dev, em_q, em_o, args.eval_mixed, bounds,
                                            max(50, args.serving_batches // 4), ls, args.serving_workers,
                                            rate=sub_rate, seed=18)
        out["serving"] = sv
    # parity subsample against the oracle (CPU) on the same index bytes
    if not args.no_cpu_baseline and args.genome_parity > 0:
        from oracle import oracle as orc
        orc.build()
        t0 = time.time()
        o = orc.OracleIndex(data, 1)
        threads = os.cpu_count() or 1
        k = args.genome_parity
        par = {}
        for name, (q, off) in (("uneven", (r3_q, r3_o)), ("eval_150bp", (q150, o150))):
            offs = off[:k + 1].cpu().numpy().astype(np.uint64)
            flat = q[:int(offs[-1])].cpu().numpy()
            dm = mems(q, off, int(len(off) - 1))
            hoff = d2h(dm.d_hit_offsets, k + 1, "<i8", dev).view(np.uint64)
            hits = d2h(dm.d_hits, 8 * int(hoff[-1]), "<i4", dev).view(np.uint32).reshape(-1, 8)
            npos = 0
            if len(hits):
                npos = (int(hits[-1][6]) | (int(hits[-1][7]) << 32)) + int(hits[-1][5])
            pos = d2h(dm.d_positions, 2 * npos, "<i4", dev).view(np.uint32).reshape(-1, 2)
            want = o.mems_packed(flat, offs, 19, 0, bounds, 1024, threads)
            bad = [f for f, a, b in zip(("hit_offsets", "hits", "positions"), (hoff, hits, pos), want)
                   if a.shape != b.shape or not np.array_equal(a, b)]
            par[name] = {"reads_checked": k, "equal": not bad, "mismatched": bad, "mem_hits": int(len(want[1]))}
        par["oracle_s"] = round(time.time() - t0, 1)
        par["what"] = "timed path's outputs (MemHit CSR, positions) for the first reads of each set vs oracle/hfm_oracle.cpp"
        out["parity"] = par
        del o
    del ls, idx, h
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_smem:
        return profile_smem(args)
    if args.profile_step:
        return profile_step(args)
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(minutes=20),
                                device_id=torch.device("cuda", local))
    from haystackfm_b200 import synth
    from haystackfm_b200.fm_index import BidirFmIndex

    if dist and rank != 0:
        dist.barrier()          # rank 0 builds (or finds) the cached index first
    ref, data, reads, build_s, built = workload(args, rank)
    if dist and rank == 0:
        dist.barrier()
    idx = BidirFmIndex.from_bytes(data, device=local)
    h = idx.handle
    lib = __import__("haystackfm_b200._lib", fromlist=["lib"]).lib()
    from haystackfm_b200 import _lib as L
    bounds = np.ascontiguousarray(idx.seq_boundaries(), dtype=np.uint32)
    nb = len(bounds)
    n = args.reads

    # device-resident inputs
    dev = torch.device("cuda", local)
    reads_d = torch.from_numpy(reads.reshape(-1)).to(dev)
    off_d = torch.arange(0, (n + 1) * 150, 150, dtype=torch.int64, device=dev)
    k32_d = torch.from_numpy(np.ascontiguousarray(reads[:, :32]).reshape(-1)).to(dev)
    off32_d = torch.arange(0, (n + 1) * 32, 32, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(h.stream(), device=dev)
    memory = []

    def mem_mark(label):
        """Device memory after a phase: free, held by this handle, reserved by torch (GB)."""
        free_b, _ = torch.cuda.mem_get_info(dev)
        db = h.device_bytes()
        memory.append({"after": label, "free_gb": round(free_b / 1e9, 1), "handle_work_gb": round(db["work"] / 1e9, 1),
                       "handle_index_gb": round(db["index"] / 1e9, 2),
                       "torch_reserved_gb": round(torch.cuda.memory_reserved(dev) / 1e9, 1)})
        print("[bench] memory", json.dumps(memory[-1]), file=sys.stderr, flush=True)
    mem_mark("index load")

    # learned cost model: trained on the logged work of a separate seeded read sample
    learned, learned_info, tuning_main = None, None, None
    if not args.no_learned:
        from haystackfm_b200.cost_model import LearnedSmem, prediction_error, work_targets
        tr = synth.sample_reads(ref, n_reads=args.train_reads, seed=1000 + rank)
        tr_d = torch.from_numpy(tr.reshape(-1)).to(dev)
        tr_off = torch.arange(0, (args.train_reads + 1) * 150, 150, dtype=torch.int64, device=dev)
        tuning_main = h.autotune_mems(tr_d, tr_off, args.train_reads, 19, 0, bounds, 1024, reps=1)
        learned = LearnedSmem(h, local, seed=1)
        t0 = time.perf_counter()
        losses, _, _ = learned.fit(tr_d, tr_off, args.train_reads, 19, 0, bounds, 1024, epochs=args.train_epochs,
                                   batch=8192, lr=1e-3, calibrate_all=True)
        torch.cuda.synchronize()
        fit_s = time.perf_counter() - t0
        del tr_d, tr_off
        ev_log = learned.log_work(reads_d, off_d, n, 19, 0, bounds, 1024)
        _, _, y_ev = learned.plan(reads_d, off_d, n)
        learned_info = {"train_reads": args.train_reads, "epochs": args.train_epochs, "fit_s": round(fit_s, 2),
                        "train_mse": [round(float(v), 5) for v in losses],
                        "holdout_error": learned.holdout_error.as_dict() if learned.holdout_error else None,
                        "eval_error": prediction_error(y_ev, work_targets(ev_log)).as_dict(),
                        "calibration": learned.calibration, "enabled": bool(learned.enabled)}
        del ev_log

    def step(stats_out=None, plain=False):
        dh = L.HfmDevHits()
        L.check(lib.hfm_locate_batch_device(h.h, k32_d.data_ptr(), off32_d.data_ptr(), n, 1024, C.byref(dh)))
        s1 = h.stats()
        if learned is not None and not plain:
            dm = learned.run(reads_d, off_d, n, 19, 0, L.ptr(bounds, L.u32p), nb, 1024)
            extra = 5 if learned.enabled else 0          # features, MLP forward, 3 binning kernels
        else:
            dm = L.HfmDevMems()
            L.check(lib.hfm_mems_batch_device(h.h, reads_d.data_ptr(), off_d.data_ptr(), n, 19, 0,
                                              L.ptr(bounds, L.u32p), nb, 1024, C.byref(dm)))
            extra = 0
        s2 = h.stats()
        if stats_out is not None:
            stats_out.append((s1, s2, dh.total, dm.n_hits, dm.n_positions, extra))

    mem_mark("autotune + learned fit")
    # work counters (one untimed pass): algorithmic bytes per launch
    h.set_counters(True)
    cnt = []
    step(cnt)
    h.set_counters(False)
    c_loc, c_mem, loc_total, n_hits, n_pos, _ = cnt[0]

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    per = []
    ev0.record(stream)
    for _ in range(args.steps):
        step(per)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n * args.steps / (ms / 1000.0)
    launches = sum(s1.search_launches + s1.resolve_launches + s1.other_launches + s2.search_launches +
                   s2.resolve_launches + s2.other_launches + p[5] for p in per for s1, s2 in [p[:2]])

    mem_mark("timed steps")
    # the plain order, same loop (the learned path's fallback and its yardstick)
    plain_info = None
    if learned is not None:
        for _ in range(args.warmup):
            step(plain=True)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step(plain=True)
        ev1.record(stream)
        torch.cuda.synchronize()
        pms = ev0.elapsed_time(ev1)
        if dist:
            t = torch.tensor([pms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            pms = float(t.item())
        plain_info = {"value": world * n * args.steps / (pms / 1000.0), "ms_per_step": pms / args.steps}
        learned_info["speedup_vs_plain"] = round(plain_info["ms_per_step"] / (ms / args.steps), 4)
    # the plain one-thread-per-read launch with its count pass (the reference GPU path's
    # structure), same loop: the baseline of the persistent path
    plain_launch = None
    if not args.no_plain_launch:
        saved = h.tuning()
        h.set_tuning(4, saved["seg_len"], 1, 1)
        for _ in range(max(1, args.warmup // 2)):
            step(plain=True)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step(plain=True)
        ev1.record(stream)
        torch.cuda.synchronize()
        lms = ev0.elapsed_time(ev1)
        h.set_tuning(saved["mems_variant"], saved["seg_len"], saved["queue_chunk"], saved["threads_per_read"])
        if dist:
            t = torch.tensor([lms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            lms = float(t.item())
        plain_launch = {"value": world * n * args.steps / (lms / 1000.0), "ms_per_step": lms / args.steps,
                        "value_speedup": round(lms / ms, 4),
                        "what": "locate + find_smems with the SMEM search as one thread per read over a grid of the "
                                "batch, local-memory sets, count pass + host-read totals + write pass"}
    mem_mark("plain launch")
    # learned order vs plain order on the whole batch: every output array byte for byte
    learned_parity = None
    if learned is not None:
        dm_p = L.HfmDevMems()
        L.check(lib.hfm_mems_batch_device(h.h, reads_d.data_ptr(), off_d.data_ptr(), n, 19, 0, L.ptr(bounds, L.u32p),
                                          nb, 1024, C.byref(dm_p)))
        snap = device_mems_tensors(torch, dev, dm_p, n, clone=True)
        dm_l = learned.run(reads_d, off_d, n, 19, 0, L.ptr(bounds, L.u32p), nb, 1024)
        now = device_mems_tensors(torch, dev, dm_l, n, clone=False)
        eq = all(a.shape == b.shape and bool(torch.equal(a, b)) for a, b in zip(snap, now))
        learned_parity = {"reads_checked": n, "equal": eq, "mem_hits": int(dm_l.n_hits),
                          "mem_positions": int(dm_l.n_positions)}
        del snap, now
        torch.cuda.empty_cache()      # the 24 GB snapshot back to the device, for the library's pools
    mem_mark("learned vs plain comparison")
    # the CUDA-graph-captured SMEM chain against the adaptive chain on the same batch
    # (host clock around each call: both include their waits for the device)
    graph_info = None
    if not args.no_graph:
        g = C.c_void_p()
        L.check(lib.hfm_mems_graph_create(h.h, reads_d.data_ptr(), off_d.data_ptr(), n, n * 150, 19, 0,
                                          L.ptr(bounds, L.u32p), nb, 1024, int(n_pos * 1.25) + 4096, C.byref(g)))
        # the locate of the 32-mers ahead of it in the same graph: one replay = one step
        L.check(lib.hfm_mems_graph_add_locate(g, k32_d.data_ptr(), off32_d.data_ptr(), n, 1024, 0,
                                              int(loc_total * 1.25) + 4096))
        rep = C.c_uint32()
        dmg = L.HfmDevMems()

        def host_ms(fn, k):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(k):
                fn()
            torch.cuda.synchronize()
            return (time.perf_counter() - t0) * 1e3 / k

        def glaunch():
            L.check(lib.hfm_mems_graph_launch(g, C.byref(dmg), C.byref(rep)))

        def adapt():
            dh = L.HfmDevHits()
            L.check(lib.hfm_locate_batch_device(h.h, k32_d.data_ptr(), off32_d.data_ptr(), n, 1024, C.byref(dh)))
            dm = L.HfmDevMems()
            L.check(lib.hfm_mems_batch_device(h.h, reads_d.data_ptr(), off_d.data_ptr(), n, 19, 0,
                                              L.ptr(bounds, L.u32p), nb, 1024, C.byref(dm)))
        for _ in range(2):
            glaunch()
        g_ms = host_ms(glaunch, args.steps)
        replayed = int(rep.value)
        a_ms = host_ms(adapt, args.steps)
        glaunch()
        replayed = replayed and int(rep.value)
        snap = device_mems_tensors(torch, dev, dmg, n, clone=True)
        lr = L.HfmDevHits()
        L.check(lib.hfm_mems_graph_locate_result(g, C.byref(lr)))
        lsnap = [x.clone() for x in device_hits_tensors(torch, dev, lr)]
        dh_a = L.HfmDevHits()
        L.check(lib.hfm_locate_batch_device(h.h, k32_d.data_ptr(), off32_d.data_ptr(), n, 1024, C.byref(dh_a)))
        lnow = device_hits_tensors(torch, dev, dh_a)
        leq = all(a.shape == b.shape and bool(torch.equal(a, b)) for a, b in zip(lsnap, lnow))
        dm_a = L.HfmDevMems()
        L.check(lib.hfm_mems_batch_device(h.h, reads_d.data_ptr(), off_d.data_ptr(), n, 19, 0, L.ptr(bounds, L.u32p),
                                          nb, 1024, C.byref(dm_a)))
        now = device_mems_tensors(torch, dev, dm_a, n, clone=False)
        geq = leq and all(a.shape == b.shape and bool(torch.equal(a, b)) for a, b in zip(snap, now))
        del snap, now, lsnap, lnow
        lib.hfm_mems_graph_free(g)
        torch.cuda.empty_cache()
        graph_info = {"graph_ms": round(g_ms, 3), "adaptive_ms": round(a_ms, 3), "speedup": round(a_ms / g_ms, 4),
                      "last_launch_replayed": replayed, "outputs_equal": geq,
                      "what": "the headline step (locate of the 32-mers + find_smems of the batch): one CUDA graph "
                              "replay of the fixed-capacity chains (hfm_mems_graph_add_locate + "
                              "hfm_mems_graph_launch) vs hfm_locate_batch_device + hfm_mems_batch_device; host clock "
                              "per call; every output array compared"}
    mem_mark("graph")
    # kernel times (CUDA events around each launch, recorded by the library on its stream)
    k_mems_ms = statistics.mean(s2.ms_search_kernel for _, s2, *_ in per)
    k_res_mem_ms = statistics.mean(s2.ms_resolve_kernel for _, s2, *_ in per)
    k_bs_ms = statistics.mean(s1.ms_search_kernel for s1, *_ in per)
    k_res_loc_ms = statistics.mean(s1.ms_resolve_kernel for s1, *_ in per)
    # algorithmic bytes (32 B per random Occ / SA-marker / sa_vals / lookup touch, read bytes,
    # 8 B per output position, 16 B per MEM hit header).  The resolve kernel walks each
    # distinct SA row once (rows_unique after deduplication); copying the positions to every
    # hit is a separate streaming kernel.
    def rows_walked(c):
        return c.rows_unique if c.rows_unique else c.rows_resolved
    b_mems = 32 * c_mem.occ_touches + 150 * n + 16 * c_mem.hits_out
    b_res_mem = 32 * (2 * c_mem.lf_calls + rows_walked(c_mem)) + 8 * rows_walked(c_mem)
    b_bs = 32 * c_loc.occ_touches + 32 * n
    b_res_loc = 32 * (2 * c_loc.lf_calls + rows_walked(c_loc)) + 8 * rows_walked(c_loc)
    kern = {"k_mems": (k_mems_ms, b_mems, c_mem.occ_touches, "Occ touches"),
            "k_resolve(smem)": (k_res_mem_ms, b_res_mem, c_mem.lf_calls, "LF steps"),
            "k_bsearch": (k_bs_ms, b_bs, c_loc.occ_touches, "Occ touches"),
            "k_resolve(locate)": (k_res_loc_ms, b_res_loc, c_loc.lf_calls, "LF steps")}
    for k, v in kern.items():
        print(f"[bench] {k}: {v[0]:.3f} ms/launch, alg {v[1] / 1e9:.3f} GB, {v[2]} {v[3]}", file=sys.stderr)
    s1, s2 = per[-1][0], per[-1][1]
    print(f"[bench] locate phases {s1.ms_search:.2f}+{s1.ms_resolve:.2f} ms, mems phases {s2.ms_search:.2f}+"
          f"{s2.ms_resolve:.2f} ms, fallback reads {s1.fallback_reads}/{s2.fallback_reads}, step {ms / args.steps:.1f} ms",
          file=sys.stderr)
    dom = max(kern, key=lambda k: kern[k][0])
    kms, kbytes, units, unit_name = kern[dom]
    try:
        peaks = json.load(open(MEASURED_PEAKS))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = FALLBACK_HBM_GBS, "fallback"
    achieved = kbytes / (kms / 1000.0) / 1e9 if kms > 0 else 0.0
    traffic, sectors = None, {}
    tpath = os.path.join(ROOT, "profiles", "traffic_per_unit.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
        if dom in tj:
            traffic = tj[dom]["dram_bytes_per_unit"] * units
            if "l1_global_sectors_per_unit" in tj[dom]:
                # from the same ncu capture: algorithmic bytes over the 32 B sectors the
                # kernel's global loads and stores moved, and the L2 / L1 sector hit rates
                sectors = {"sector_efficiency": round((kbytes / units) / (32 * tj[dom]["l1_global_sectors_per_unit"]), 3),
                           "l2_hit_rate": tj[dom]["l2_sector_hit_rate"], "l1_hit_rate": tj[dom]["l1_sector_hit_rate"],
                           "source": tj[dom]["source"]}
    # the random-access ceiling: independent 32 B / 64 B / 96 B loads over 8 GB on every SM
    # (the access pattern of Occ records, which a streaming copy does not have)
    gather = {}
    for span in (32, 64, 96):
        gbs, gms = C.c_float(), C.c_float()
        L.check(lib.hfm_probe_gather(local, 8 << 30, span, C.byref(gbs), C.byref(gms)))
        gather[f"random_{span}B_gbs"] = round(gbs.value, 1)
    rec_span = 32 if h.info().num_lanes <= 5 else 96      # narrow / wide Occ record
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                "random_gather_ceiling": gather, "record_bytes": rec_span, "sectors": sectors,
                # touches/s of the kernel (32 algorithmic bytes each) over record fetches/s of the probe
                "frac_of_random_gather": (achieved / 32) / (gather[f"random_{rec_span}B_gbs"] / rec_span),
                "kernel_ms": kms, "alg_bytes": kbytes, "units": units, "unit_name": unit_name,
                "kernels_ms": {k: v[0] for k, v in kern.items()},
                "kernels_gbs": {k: (v[1] / (v[0] / 1000) / 1e9 if v[0] > 0 else None) for k, v in kern.items()}}

    mem_mark("roofline")
    # end to end through the host-buffer C ABI (pinned reads in, every result out)
    reads_pin = torch.empty(n * 150, dtype=torch.uint8, pin_memory=True)
    reads_pin.numpy()[:] = reads.reshape(-1)
    k32_pin = torch.empty(n * 32, dtype=torch.uint8, pin_memory=True)
    k32_pin.numpy()[:] = np.ascontiguousarray(reads[:, :32]).reshape(-1)
    rp, kp = reads_pin.numpy(), k32_pin.numpy()
    ch = min(args.e2e_chunk, n)

    # Two handles sharing the device-resident index (own streams and buffers) driven by two
    # host threads: one handle's kernels overlap the other's result copies.
    handles = [h] + [h.share() for _ in range(args.e2e_streams - 1)]

    def run_chunks(hh, chunks, acc):
        h2d = d2h = 0
        for a in chunks:
            b = min(n, a + ch)
            m = b - a
            off150 = np.arange(0, (m + 1) * 150, 150, dtype=np.uint64)
            off32 = np.arange(0, (m + 1) * 32, 32, dtype=np.uint64)
            res = C.POINTER(L.HfmHits)()
            L.check(lib.hfm_locate_batch(hh.h, L.ptr(kp[a * 32:], L.u8p), L.ptr(off32, L.u64p), m, 1024, C.byref(res)))
            d2h += (m + 1) * 8 + m * 4 + res.contents.total * 8
            lib.hfm_free(res)
            mo = C.POINTER(L.HfmMemOut)()
            L.check(lib.hfm_mems_batch(hh.h, L.ptr(rp[a * 150:], L.u8p), L.ptr(off150, L.u64p), m, 19, 0,
                                       L.ptr(bounds, L.u32p), nb, 1024, C.byref(mo)))
            d2h += (m + 1) * 8 + mo.contents.n_hits * 32 + mo.contents.n_positions * 8
            lib.hfm_free(mo)
            h2d += m * 32 + (m + 1) * 8 + m * 150 + (m + 1) * 8 + nb * 4
        acc.append((h2d, d2h))

    def e2e_step():
        import threading
        starts = list(range(0, n, ch))
        acc, threads = [], []
        for k, hh in enumerate(handles):
            t = threading.Thread(target=run_chunks, args=(hh, starts[k::len(handles)], acc))
            t.start()
            threads.append(t)
        for t in threads:
            t.join()
        if len(acc) != len(handles):
            raise RuntimeError("an end-to-end worker failed")
        return sum(a for a, _ in acc), sum(b for _, b in acc)

    e2e_s, h2d, d2h = 0.0, 0, 0
    if not args.no_e2e:
        e2e_step()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            h2d, d2h = e2e_step()
        e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": world * n * args.steps / e2e_s if e2e_s else None, "unit": "reads/s", "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "chunk_reads": ch, "handles": args.e2e_streams}
    if not args.no_e2e:
        # the copy ceiling: one 2 GiB device-to-pinned-host copy on this box
        src = torch.empty(2 << 30, dtype=torch.uint8, device=dev)
        dst = torch.empty(2 << 30, dtype=torch.uint8, pin_memory=True)
        dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record()
        dst.copy_(src, non_blocking=True)
        c1.record()
        torch.cuda.synchronize()
        d2h_gbs = (2 << 30) / (c0.elapsed_time(c1) / 1e3) / 1e9
        e2e["d2h_copy_gbs"] = round(d2h_gbs, 1)
        e2e["copy_bound_reads_per_s"] = round(n / (d2h / (d2h_gbs * 1e9)), 0) if d2h else None
        del src, dst

    serving = None
    if not args.no_serving and rank == 0 and world == 1:      # single-GPU measurements
        serving = serving_latency(h, lib, L, kp, rp, bounds, n, 300)

    # CPU baseline (the same CPU_SAMPLE reads the reference arm times) and parity: the timed
    # calls' outputs for the first PARITY_READS reads, byte for byte against the oracle
    cpu, parity = None, None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        orc.build()
        o = orc.OracleIndex(data, 1)
        threads = os.cpu_count() or 1
        dt, _, _ = cpu_time(o, reads[:CPU_SAMPLE], bounds, threads)
        dt1, _, _ = cpu_time(o, reads[:1024], bounds, 1)
        cpu = {"value": CPU_SAMPLE / dt, "unit": "reads/s", "cores": threads, "kind": "port",
               "sample": f"the first {CPU_SAMPLE} reads of the workload ({dt:.1f} s): locate of the 32-mer + "
                         f"find_smems, oracle/hfm_oracle.cpp, {threads} threads (the reference arm times the same "
                         f"reads)",
               "single_core": {"value": 1024 / dt1, "sample": f"the first 1024 reads ({dt1:.1f} s), 1 thread"}}
        npre = min(PARITY_READS, n)
        t0 = time.perf_counter()
        got = gpu_prefix_outputs(h, lib, L, dev, k32_d, off32_d, reads_d, off_d, n, bounds, npre)
        _, wloc, wmem = cpu_time(o, reads[:npre], bounds, threads)
        bad = compare_outputs(got, (wloc, wmem))
        parity = {"reads_checked": npre, "equal": not bad, "mismatched": bad,
                  "locate_positions": int(len(wloc[2])), "mem_hits": int(len(wmem[1])),
                  "mem_positions": int(len(wmem[2])), "oracle_s": round(time.perf_counter() - t0, 1),
                  "what": "outputs of the timed device calls (locate CSR, MemHit CSR, positions) for the first "
                          f"{npre} reads vs oracle/hfm_oracle.cpp on the same index bytes"}
        del o
    if learned is not None and learned_parity is not None:
        if parity is None:
            parity = {}
        parity["learned_vs_plain"] = learned_parity
    run_path = ("learned-binned" if learned is not None and learned.enabled else
                "plain order (learned order not faster on held-out reads)"
                if learned is not None and learned.calibration is not None else
                "plain order (cost model not predictive on held-out reads)" if learned is not None else "plain")
    genome = None
    if not args.no_genome and rank == 0 and world == 1:
        del handles, idx, h, learned
        import gc
        gc.collect()
        torch.cuda.empty_cache()
        genome = genome_workloads(args, local, torch)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "reads/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generators, haystackfm_b200/synth.py)",
            "config": bench_config(args, world),
            "run": {"path": run_path,
                    "index_build_s": round(build_s, 1), "index_cached": not built,
                    "index_sha256": hashlib.sha256(data).hexdigest(),
                    "locate_positions": int(loc_total), "mem_hits": int(n_hits), "mem_positions": int(n_pos),
                    "distinct_rows_walked": int(rows_walked(c_mem) + rows_walked(c_loc)),
                    "autotuned": tuning_main},
            "parity": parity,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "memory": memory,
            "ingest": ingest_bench(reads) if rank == 0 else None,
            "plain": plain_info, "plain_launch": plain_launch, "graph": graph_info, "learned": learned_info,
            "serving": serving,
            "genome": genome,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if parity and (not parity.get("equal", True) or
                   (parity.get("learned_vs_plain") and not parity["learned_vs_plain"]["equal"])):
        raise SystemExit("parity mismatch: " + json.dumps(parity))


if __name__ == "__main__":
    main()
