// api.cu — the C ABI (include/hfm.h): device-resident index, query pipelines,
// per-handle memory arenas and streams.
//
// A handle owns one CUDA stream and grow-only device buffers; calls on one handle are
// serialised by its mutex, separate handles (e.g. one per GPU) run concurrently.  This
// replaces the reference's process-wide wgpu context and its per-call index uploads
// (src/gpu/context_cache.rs:11-19, src/gpu/locate.rs:69-111,
// src/fm_index/bidir_index.rs:410-411).

#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <string>
#include <thread>
#include <vector>

#include "dev_index.cuh"
#include "hfm_internal.h"
#include "resolve.cuh"
#include "search.cuh"

namespace hfm {

static thread_local std::string g_err;

int set_error(int status, const std::string& msg) {
  g_err = msg;
  return status;
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t _e = (call);                                                                      \
    if (_e != cudaSuccess)                                                                        \
      return set_error(_e == cudaErrorMemoryAllocation ? HFM_E_OOM : HFM_E_CUDA,                  \
                       std::string(#call) + ": " + cudaGetErrorString(_e));                       \
  } while (0)

#define RET(x) do { int _r = (x); if (_r != HFM_OK) return _r; } while (0)

// Runs the statement block with FM bound to the index's Occ record format as a
// compile-time constant (the SMEM kernels are specialised per format).
#define WITH_FMT(fmt, ...)                                                                        \
  do {                                                                                            \
    if ((fmt) == OCC_NARROW) { constexpr uint32_t FM = OCC_NARROW; __VA_ARGS__ }                   \
    else { constexpr uint32_t FM = OCC_WIDE; __VA_ARGS__ }                                        \
  } while (0)

// compatible_symbols / ExactDna::compatible (src/alphabet.rs:174-193,286-294) as bit masks
static void compat_masks(uint32_t tag, uint16_t out[16]) {
  static const uint8_t iupac[16][15] = {
      {0}, {1, 5, 6, 9, 11, 13, 14, 15}, {2, 5, 7, 8, 11, 12, 14, 15}, {3, 5, 6, 8, 10, 12, 13, 15},
      {4, 5, 7, 9, 10, 12, 13, 14}, {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15},
      {1, 3, 5, 6, 8, 9, 10, 11, 12, 13, 14, 15}, {2, 4, 5, 7, 8, 9, 10, 11, 12, 13, 14, 15},
      {2, 3, 5, 6, 7, 8, 10, 11, 12, 13, 14, 15}, {1, 4, 5, 6, 7, 9, 10, 11, 12, 13, 14, 15},
      {3, 4, 5, 6, 7, 8, 9, 10, 12, 13, 14, 15}, {1, 2, 5, 6, 7, 8, 9, 11, 12, 13, 14, 15},
      {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {1, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15},
      {1, 2, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {1, 2, 3, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}};
  for (int c = 0; c < 16; c++) {
    uint16_t m = 0;
    if (tag == 1) { if (c >= 1 && c <= 4) m = (uint16_t)(1u << c); }
    else for (int k = 0; k < 15; k++) if (iupac[c][k]) m |= (uint16_t)(1u << iupac[c][k]);
    out[c] = m;
  }
}

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return HFM_OK;
    if (p) cudaFree(p);
    p = nullptr; cap = 0;
    size_t want = std::max<size_t>(bytes + std::min<size_t>(bytes / 4, 256ull << 20), 256);   // growth slack
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      e = cudaMalloc(&p, bytes);
      if (e != cudaSuccess) { cudaGetLastError(); p = nullptr; return set_error(HFM_E_OOM, "cudaMalloc failed: " + std::to_string(bytes) + " bytes"); }
      want = bytes;
    }
    cap = want;
    return HFM_OK;
  }
  template <class T> T* as() const { return (T*)p; }
  void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};

struct Counters {                    // device-side counters, one block per handle
  unsigned long long iv_used, hit_used, touches, steps, seg_used;
  uint32_t n_ovf, still_ovf, walk_err, queue, queue2, n_mid, n_wrp, queue3, seg_queue, merge_queue, fix_queue, _pad;
};

struct FmDev {
  DevFm d{};
  DevBuf occ, sb, ssa, sa_vals, lut, bounds, compat;
  size_t nbytes[7] = {0, 0, 0, 0, 0, 0, 0};   // bytes in use of the seven buffers above, in that order
  uint32_t text_len = 0, num_seqs = 0, lookup_depth = 0, tag = 0, num_lanes = 0, encoding = 0, rate = 0, fmt = 0;
  std::vector<uint32_t> seq_boundaries;
  size_t bytes() const { return occ.cap + sb.cap + ssa.cap + sa_vals.cap + lut.cap + bounds.cap + compat.cap; }
};

}  // namespace hfm

using namespace hfm;

struct hfm_index {
  int device = 0, kind = 0;
  FmDev fwd, rev;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  bool count_work = false;
  // per-call work buffers (grow-only)
  DevBuf q, qoff, counts, nhits, niv, ivoff, status, ovf, ivpool, hitpool, seg_row, seg_off, pos_base, seg_base,
      scan_tmp, out_pairs, ref_bounds, hit_start, hit_count, hit_base, hits, npos_scan, work, cwork, ctr,
      mivpool, bswork, memwork, hkeys, hslot, hflags, huid, urow, ulen, uoff, uout, blockmap, blockmap2, ovf2, ovf3,
      lflag, lpos, sids, lids, ucount, ubase, uread, uk, ubits, uexit, ust, ucoff, ucnt, segpool, fxe, fxc, fxx,
      fxo, fxn, npos, loc_pairs, okeys, oids, otemp;
  uint32_t flags = 0;
  uint32_t seg_len = 512;  // SMEM reads longer than 2 * seg_len take the segmented sweep
  uint32_t queue_chunk = 1;       // reads a per-thread kernel takes from its queue per atomic
  uint32_t threads_per_read = 1;  // 32: every read on the warp-per-read kernel
  uint32_t read_order = 0;        // 1: SMEM queue in the order of the reads' first 16 codes
  DevBuf iota;                    // 0..nq-1 (the order of a batch sent whole to the warp kernel)
  int mems_variant = 3;   // SMEM fast-kernel variant (see mems_device): 2 local 32-entry
                          // candidate lists; 3 global 1024-entry lists
  int num_sms = 0;
  uint64_t iv_cap = 0, miv_cap = 0, hit_cap = 0;   // pool capacities in elements (uint2 / BIv / hit)
  uint64_t seg_cap = 0;                            // segment candidate pool capacity (Cand)
  Counters* h_ctr = nullptr;        // pinned
  uint32_t timeout_ms = 0;          // host-side deadline of every wait on the stream (0: none)
  std::vector<void*> orphans;       // result blocks of calls that timed out (freed once the stream drains)
  bool shared_index = false;        // fwd / rev device buffers belong to another handle
  cudaEvent_t ev_wait = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t evk[4] = {nullptr, nullptr, nullptr, nullptr};   // main search kernel, resolve kernel
  bool k_search_rec = false, k_resolve_rec = false;
  hfm_stats stats{};
};

namespace hfm {

// ---------------------------------------------------------------------------
// Device layout construction (host transform of the bincode records)
// ---------------------------------------------------------------------------
static int upload(DevBuf& b, const void* src, size_t bytes, cudaStream_t s) {
  RET(b.ensure(std::max<size_t>(bytes, 16)));
  if (bytes) CK(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, s));
  return HFM_OK;
}

static int build_device_fm(const HostFm& h, FmDev& f, cudaStream_t s) {
  const uint32_t n = h.text_len, L = h.num_lanes;
  const uint64_t nblk = ((uint64_t)n + 63) / 64;
  const uint64_t nsb = (nblk + (1u << SB_BLOCK_SHIFT) - 1) >> SB_BLOCK_SHIFT;
  // symbols absent from the lane map are absent from the text
  uint16_t sym_mask = 0;
  for (int sy = 0; sy < 16; sy++) if (h.s2l[sy] != 0xFF) sym_mask |= (uint16_t)(1u << sy);
  const bool narrow = (sym_mask & ~0x1Fu) == 0;       // codes 0..4 only
  const uint32_t fmt = narrow ? OCC_NARROW : OCC_WIDE;
  const uint64_t rec_u32 = narrow ? OCC_NARROW_U4 * 4 : OCC_WIDE_U4 * 4;
  std::vector<uint32_t> occ(nblk * rec_u32, 0);
  std::vector<uint32_t> sb(nsb * 16, 0);
  std::vector<uint32_t> ssa(nblk * 4, 0);
  const uint64_t width = h.encoding == 0 ? h.num_planes : L;
  // Decode the reference records (compacted lanes, u32 superblock count + u16 delta per
  // lane) into whole per-symbol counts and 4 symbol-code bitplanes, then re-encode them as
  // the device records: whole counts (wide) or counts from the start of the device
  // superblock of 1024 records, which fit a u16 (narrow).
  auto decode = [&](uint64_t b, uint32_t cnt[16], uint64_t planes[4]) {
    const uint8_t* r = h.block_data + b * h.block_stride;
    uint64_t words[16] = {0};
    for (uint64_t w = 0; w < width; w++) std::memcpy(&words[w], r + L * 6 + w * 8, 8);
    for (int c = 0; c < 16; c++) cnt[c] = 0;
    for (int p = 0; p < 4; p++) planes[p] = 0;
    for (uint32_t l = 0; l < L; l++) {
      uint32_t sbv; uint16_t dv;
      std::memcpy(&sbv, r + l * 4, 4); std::memcpy(&dv, r + L * 4 + l * 2, 2);
      uint32_t sym = h.l2s[l];
      cnt[sym] = sbv + dv;
      uint64_t m;
      if (h.encoding == 1) m = words[l];
      else if (h.num_planes == 0) m = ~0ull;
      else { m = ~0ull; for (uint32_t p = 0; p < h.num_planes; p++) m &= ((l >> p) & 1) ? words[p] : ~words[p]; }
      if (b == nblk - 1 && (n & 63)) m &= (1ull << (n & 63)) - 1;   // rows past the text
      for (int p = 0; p < 4; p++) if ((sym >> p) & 1) planes[p] |= m;
    }
  };
  auto fill = [&](uint64_t b0, uint64_t b1) {
    uint32_t cnt[16], base[16];
    uint64_t planes[4];
    for (uint64_t b = b0; b < b1; b++) {
      decode(b, cnt, planes);
      const uint64_t sbi = b >> SB_BLOCK_SHIFT;
      if ((b & ((1u << SB_BLOCK_SHIFT) - 1)) == 0 || b == b0) {
        if ((b & ((1u << SB_BLOCK_SHIFT) - 1)) == 0) {
          std::memcpy(base, cnt, 64);
          std::memcpy(&sb[sbi * 16], cnt, 64);
        } else {                                        // a thread's range starts inside a superblock
          uint32_t c0[16]; uint64_t p0[4];
          decode(sbi << SB_BLOCK_SHIFT, c0, p0);
          std::memcpy(base, c0, 64);
        }
      }
      uint32_t* rec = &occ[b * rec_u32];
      uint32_t d[16];
      for (int c = 0; c < 16; c++) d[c] = cnt[c] - base[c];
      if (narrow) {
        rec[0] = d[1] | (d[2] << 16); rec[1] = d[3] | (d[4] << 16);
        std::memcpy(rec + 2, &planes[0], 8); std::memcpy(rec + 4, &planes[1], 8); std::memcpy(rec + 6, &planes[2], 8);
      } else {
        std::memcpy(rec, cnt, 64);           // whole counts before the record
        std::memcpy(rec + 16, planes, 32);
      }
      // sampled-SA record: bits + rank before (validated equal to the stored sb + delta)
      uint64_t word; uint32_t sbs; uint16_t dd;
      std::memcpy(&word, h.ssa_words + b * 14, 8); std::memcpy(&sbs, h.ssa_words + b * 14 + 8, 4);
      std::memcpy(&dd, h.ssa_words + b * 14 + 12, 2);
      if (b == nblk - 1 && (n & 63)) word &= (1ull << (n & 63)) - 1;
      ssa[b * 4 + 0] = (uint32_t)word; ssa[b * 4 + 1] = (uint32_t)(word >> 32); ssa[b * 4 + 2] = sbs + dd;
    }
  };
  {
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (nblk < (1u << 16)) nt = 1;
    std::vector<std::thread> th;
    const uint64_t per = (nblk + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
      uint64_t b0 = t * per, b1 = std::min<uint64_t>(nblk, b0 + per);
      if (b0 < b1) th.emplace_back(fill, b0, b1);
    }
    for (auto& x : th) x.join();
  }
  uint16_t cm[16];
  compat_masks(h.tag, cm);
  const void* srcs[7] = {occ.data(), sb.data(), ssa.data(), h.sa_vals, h.has_lookup ? h.lookup_intervals : nullptr,
                         h.seq_boundaries.data(), cm};
  const size_t sizes[7] = {occ.size() * 4, sb.size() * 4, ssa.size() * 4, (size_t)h.n_sa_vals * 4,
                           h.has_lookup ? (size_t)h.n_lookup * 8 : 0, h.seq_boundaries.size() * 4, sizeof(cm)};
  DevBuf* bufs[7] = {&f.occ, &f.sb, &f.ssa, &f.sa_vals, &f.lut, &f.bounds, &f.compat};
  for (int k = 0; k < 7; k++) {
    if (k == 4 && !h.has_lookup) continue;
    RET(upload(*bufs[k], srcs[k], sizes[k], s));
    f.nbytes[k] = sizes[k];
  }
  CK(cudaStreamSynchronize(s));      // host vectors die at return
  DevFm& d = f.d;
  d.occ = f.occ.as<uint4>(); d.sb = f.sb.as<uint32_t>(); d.ssa = f.ssa.as<uint4>();
  d.sa_vals = f.sa_vals.as<uint32_t>(); d.seq_bounds = f.bounds.as<uint32_t>();
  d.lut = h.has_lookup ? f.lut.as<uint2>() : nullptr;
  d.text_len = n; d.num_seqs = (uint32_t)h.seq_boundaries.size(); d.sample_rate = h.sample_rate;
  d.lut_depth = h.has_lookup ? h.lookup_depth : 0; d.tag = h.tag;
  d.lut_radix = (uint32_t)h.lookup_core.size(); d.num_blocks = (uint32_t)nblk; d.fmt = fmt;
  std::memcpy(d.C, h.C, 64); std::memcpy(d.s2l, h.s2l, 16); std::memcpy(d.l2s, h.l2s, 16);
  std::memset(d.lut_digit, 0xFF, 16);
  for (size_t k = h.lookup_core.size(); k-- > 0;) if (h.lookup_core[k] < 16) d.lut_digit[h.lookup_core[k]] = (uint8_t)k;
  d.sym_mask = sym_mask;
  f.text_len = n; f.num_seqs = h.num_sequences; f.lookup_depth = d.lut_depth; f.tag = h.tag;
  f.num_lanes = L; f.encoding = h.encoding; f.rate = h.sample_rate; f.seq_boundaries = h.seq_boundaries;
  f.fmt = fmt;
  return HFM_OK;
}

// ---------------------------------------------------------------------------
// Scan helper: out[0..n] = exclusive scan of in (stride in elements), out[n] = total.
// ---------------------------------------------------------------------------
template <class T>
static int scan(hfm_index* x, const T* in, uint32_t stride, uint64_t n, uint64_t* out, uint32_t& launches) {
  if (n == 0) { CK(cudaMemsetAsync(out, 0, 8, x->stream)); return HFM_OK; }
  uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  RET(x->scan_tmp.ensure((tiles + 1) * 8));
  uint64_t* sums = x->scan_tmp.as<uint64_t>();
  k_scan_tiles<T><<<(unsigned)tiles, SCAN_T, 0, x->stream>>>(in, stride, n, out, sums);
  k_scan_sums<<<1, 1024, 0, x->stream>>>(sums, (uint32_t)tiles);
  k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, x->stream>>>(out, n, sums, (uint32_t)tiles);
  launches += 3;
  CK(cudaGetLastError());
  return HFM_OK;
}

// Waits until `ev` has completed.  Without a deadline this is cudaEventSynchronize; with
// one (hfm_set_timeout) the host polls the event and gives up with HFM_E_TIMEOUT once the
// deadline has passed.  The abandoned work stays queued on the handle's stream: the next
// call on the handle runs after it, so the handle remains usable.
static int wait_event(hfm_index* x, cudaEvent_t ev) {
  if (!x->timeout_ms) { CK(cudaEventSynchronize(ev)); return HFM_OK; }
  const auto t0 = std::chrono::steady_clock::now();
  const auto limit = std::chrono::milliseconds(x->timeout_ms);
  for (;;) {
    cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return HFM_OK;
    if (e != cudaErrorNotReady) CK(e);
    if (std::chrono::steady_clock::now() - t0 >= limit)
      return set_error(HFM_E_TIMEOUT, "device work did not finish within " + std::to_string(x->timeout_ms) + " ms");
    std::this_thread::yield();
  }
}

static int wait_stream(hfm_index* x) {
  CK(cudaEventRecord(x->ev_wait, x->stream));
  return wait_event(x, x->ev_wait);
}

static int read_ctr(hfm_index* x) {
  CK(cudaMemcpyAsync(x->h_ctr, x->ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, x->stream));
  return wait_stream(x);
}

static Counters* dctr(hfm_index* x) { return x->ctr.as<Counters>(); }

static int read_u64(hfm_index* x, const uint64_t* dsrc, uint64_t& v) {
  CK(cudaMemcpyAsync(&x->h_ctr->steps, dsrc, 8, cudaMemcpyDeviceToHost, x->stream));
  RET(wait_stream(x));
  v = x->h_ctr->steps;
  return HFM_OK;
}

static constexpr uint32_t BS_SET_CAP = 64;     // fast-path interval-set capacity (backward search)
static constexpr uint32_t BS_WARP_SET_CAP = 8192;   // long-tail pass, per warp
static constexpr uint32_t MEM_SET_CAP = FAST_SET_CAP;   // fast-path interval-set capacity (SMEM / MEM)
static constexpr uint32_t MEM_WARP_SET_CAP = 8192;  // long-tail pass, per warp
static constexpr int MEM_KC = 32;              // fast-path candidate capacity (thread-local)
static constexpr uint32_t MID_CAND_CAP = 1024;  // candidate list of the per-thread rerun (global memory)
static constexpr uint32_t MID_THREADS_PER_SM = 256;
static constexpr uint32_t FAST_CAND_CAP = 1024;  // global candidate list of fast-pass variant 3
static constexpr int MEMS_PLAIN = 4;             // mems_variant of the plain one-thread-per-read launch

// Backward search for a batch.  with_ivs = false: counts only.
static int run_bsearch(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq, uint32_t cap,
                       bool with_ivs, uint32_t* d_counts, uint32_t& launches) {
  const FmDev& F = x->fwd;
  RET(x->nhits.ensure((size_t)nq * 8 + 8)); RET(x->niv.ensure((size_t)nq * 4 + 4));
  RET(x->ivoff.ensure((size_t)nq * 8 + 8)); RET(x->status.ensure((size_t)nq * 4 + 4));
  RET(x->ovf.ensure((size_t)nq * 4 + 4));
  if (with_ivs) {
    if (x->iv_cap < (uint64_t)nq * 2 + 1024) x->iv_cap = (uint64_t)nq * 2 + 1024;
    RET(x->ivpool.ensure(x->iv_cap * 8));
    x->iv_cap = x->ivpool.cap / 8;
  }
  // persistent fast pass: one wave of resident threads, BS_SET_CAP intervals per set
  int bpsm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k_bsearch<false, 32>, 256, 0));
  uint64_t threads = (uint64_t)std::max(1, bpsm) * x->num_sms * 256;
  threads = std::min<uint64_t>(threads, ((uint64_t)nq + 255) / 256 * 256);
  RET(x->bswork.ensure(std::max<uint64_t>(threads, 32) * 2 * BS_SET_CAP * 8));
  for (int attempt = 0; attempt < 8; attempt++) {
    CK(cudaMemsetAsync(x->ctr.p, 0, sizeof(Counters), x->stream));
    Pool pool{x->ivpool.p, &dctr(x)->iv_used, x->iv_cap};
    BsOut o{d_counts, with_ivs ? x->nhits.as<uint64_t>() : nullptr, x->niv.as<uint32_t>(), x->ivoff.as<uint64_t>(),
            x->status.as<uint32_t>(), x->ovf.as<uint32_t>(), &dctr(x)->n_ovf, &dctr(x)->touches};
    if (nq) {
      unsigned grid = (unsigned)(threads / 256);
      if (x->bswork.cap < (size_t)grid * 256 * 2 * BS_SET_CAP * 8) return set_error(HFM_E_ARG, "internal: work area too small");
      cudaEventRecord(x->evk[0], x->stream);
      if (x->count_work)
        k_bsearch<true, 32><<<grid, 256, 0, x->stream>>>(F.d, F.compat.as<uint16_t>(), d_q, d_qoff, nullptr, nq, cap,
                                                        x->bswork.as<uint2>(), BS_SET_CAP, &dctr(x)->queue, pool, o,
                                                        &dctr(x)->still_ovf);
      else
        k_bsearch<false, 32><<<grid, 256, 0, x->stream>>>(F.d, F.compat.as<uint16_t>(), d_q, d_qoff, nullptr, nq, cap,
                                                         x->bswork.as<uint2>(), BS_SET_CAP, &dctr(x)->queue, pool, o,
                                                         &dctr(x)->still_ovf);
      cudaEventRecord(x->evk[1], x->stream);
      x->k_search_rec = true;
      launches++;
      CK(cudaGetLastError());
    }
    RET(read_ctr(x));
    uint32_t n_ovf = x->h_ctr->n_ovf;
    if (n_ovf) {
      // long tail: one warp per overflowed query, sets in per-warp global regions, growing
      // 4x until every query fits
      uint32_t set_cap = BS_WARP_SET_CAP;
      while (true) {
        uint64_t per_warp = (uint64_t)set_cap * 2 * 8;
        uint64_t warps = std::min<uint64_t>({(uint64_t)n_ovf, (uint64_t)x->num_sms * 16,
                                             std::max<uint64_t>(4, (2ull << 30) / per_warp)});
        unsigned grid = (unsigned)((warps + 3) / 4);
        RET(x->work.ensure((size_t)grid * 4 * per_warp));
        CK(cudaMemsetAsync(&dctr(x)->still_ovf, 0, 4, x->stream));
        CK(cudaMemsetAsync(&dctr(x)->queue2, 0, 4, x->stream));
        if (x->count_work)
          k_bsearch_warp<true><<<grid, 128, 0, x->stream>>>(F.d, F.compat.as<uint16_t>(), d_q, d_qoff, x->ovf.as<uint32_t>(),
                                                           n_ovf, cap, x->work.as<uint2>(), set_cap, &dctr(x)->queue2, pool,
                                                           o, &dctr(x)->still_ovf);
        else
          k_bsearch_warp<false><<<grid, 128, 0, x->stream>>>(F.d, F.compat.as<uint16_t>(), d_q, d_qoff, x->ovf.as<uint32_t>(),
                                                            n_ovf, cap, x->work.as<uint2>(), set_cap, &dctr(x)->queue2, pool,
                                                            o, &dctr(x)->still_ovf);
        launches++;
        CK(cudaGetLastError());
        RET(read_ctr(x));
        if (x->h_ctr->still_ovf == 0) break;
        if (set_cap >= (1u << 24)) return set_error(HFM_E_OVERFLOW, "interval set exceeds 2^24 intervals");
        set_cap *= 4;
      }
    }
    if (!with_ivs || x->h_ctr->iv_used <= x->iv_cap) {
      x->stats.occ_touches += x->h_ctr->touches;
      return HFM_OK;
    }
    x->iv_cap = x->h_ctr->iv_used + x->h_ctr->iv_used / 2 + 1024;   // pool exhausted: grow, re-run
    RET(x->ivpool.ensure(x->iv_cap * 8));
    x->iv_cap = x->ivpool.cap / 8;
  }
  return set_error(HFM_E_OVERFLOW, "interval pool did not converge");
}

static int resolve(hfm_index* x, const FmDev& F, const uint32_t* seg_row, uint32_t stride, const uint64_t* seg_off,
                   uint64_t nseg, uint64_t total, const uint32_t* d_bounds, uint32_t nb, uint32_t* out,
                   uint32_t& launches, uint32_t& other) {
  if (total == 0) return HFM_OK;
  if (nseg >= 0xFFFFFFFFull) return set_error(HFM_E_ARG, "too many intervals in one call");
  uint64_t blocks = (total + RES_T - 1) / RES_T;
  RET(x->blockmap.ensure(blocks * 4 + 4));
  k_block_first<<<(unsigned)((nseg + 255) / 256), 256, 0, x->stream>>>(seg_off, (uint32_t)nseg, RES_T,
                                                                     x->blockmap.as<uint32_t>());
  other++;
  ResolveArgs A{seg_row, stride, seg_off, (uint32_t)nseg, total, d_bounds, nb,
                F.rate ? F.rate : F.text_len, out, &dctr(x)->walk_err, &dctr(x)->steps, x->blockmap.as<uint32_t>()};
  // grid.x limit 2^31-1 blocks covers 5e11 positions
  cudaEventRecord(x->evk[2], x->stream);
  if (x->count_work) k_resolve<true><<<(unsigned)blocks, RES_T, 0, x->stream>>>(F.d, A);
  else k_resolve<false><<<(unsigned)blocks, RES_T, 0, x->stream>>>(F.d, A);
  cudaEventRecord(x->evk[3], x->stream);
  x->k_resolve_rec = true;
  launches++;
  CK(cudaGetLastError());
  return HFM_OK;
}

// Resolve with deduplication of identical segments (see k_dedup_*): each distinct
// (first row, length) is walked once and copied to every hit that has it.
static int resolve_segments(hfm_index* x, const FmDev& F, const uint32_t* seg_row, uint32_t stride,
                            const uint64_t* seg_off, uint64_t nseg, uint64_t total, const uint32_t* d_bounds,
                            uint32_t nb, uint32_t* out, uint32_t& launches, uint32_t& other) {
  if (total == 0) return HFM_OK;
  bool dedup = (x->flags & HFM_FLAG_DEDUP_ALWAYS) || (!(x->flags & HFM_FLAG_DEDUP_NEVER) && total >= 4 * nseg);
  if (!dedup || nseg < 2) return resolve(x, F, seg_row, stride, seg_off, nseg, total, d_bounds, nb, out, launches, other);
  uint64_t size = 1024;
  while (size < 2 * nseg) size <<= 1;
  RET(x->hkeys.ensure(size * 8)); RET(x->hslot.ensure(nseg * 4 + 4));
  RET(x->hflags.ensure(size * 4)); RET(x->huid.ensure((size + 1) * 8));
  CK(cudaMemsetAsync(x->hkeys.p, 0xFF, size * 8, x->stream));
  k_dedup_insert<<<(unsigned)((nseg + 255) / 256), 256, 0, x->stream>>>(seg_row, stride, seg_off, (uint32_t)nseg,
                                                                      x->hkeys.as<unsigned long long>(), size - 1,
                                                                      x->hslot.as<uint32_t>());
  k_dedup_flags<<<(unsigned)((size + 255) / 256), 256, 0, x->stream>>>(x->hkeys.as<unsigned long long>(), size,
                                                                     x->hflags.as<uint32_t>());
  other += 2;
  CK(cudaGetLastError());
  RET(scan(x, x->hflags.as<uint32_t>(), 1, size, x->huid.as<uint64_t>(), other));
  uint64_t nuniq = 0;
  RET(read_u64(x, x->huid.as<uint64_t>() + size, nuniq));
  RET(x->urow.ensure(nuniq * 4 + 4)); RET(x->ulen.ensure(nuniq * 4 + 4)); RET(x->uoff.ensure((nuniq + 1) * 8));
  k_dedup_compact<<<(unsigned)((size + 255) / 256), 256, 0, x->stream>>>(x->hkeys.as<unsigned long long>(), size,
                                                                       x->huid.as<uint64_t>(), x->urow.as<uint32_t>(),
                                                                       x->ulen.as<uint32_t>());
  other++;
  CK(cudaGetLastError());
  RET(scan(x, x->ulen.as<uint32_t>(), 1, nuniq, x->uoff.as<uint64_t>(), other));
  uint64_t utotal = 0;
  RET(read_u64(x, x->uoff.as<uint64_t>() + nuniq, utotal));
  RET(x->uout.ensure(utotal * 8 + 8));
  RET(resolve(x, F, x->urow.as<uint32_t>(), 1, x->uoff.as<uint64_t>(), nuniq, utotal, d_bounds, nb,
              x->uout.as<uint32_t>(), launches, other));
  RET(x->blockmap2.ensure(((total + EXP_BLK - 1) / EXP_BLK) * 4 + 4));
  k_block_first<<<(unsigned)((nseg + 255) / 256), 256, 0, x->stream>>>(seg_off, (uint32_t)nseg, EXP_BLK,
                                                                     x->blockmap2.as<uint32_t>());
  k_dedup_expand<<<(unsigned)((total + EXP_BLK - 1) / EXP_BLK), EXP_T, 0, x->stream>>>(
      seg_off, (uint32_t)nseg, total, x->hslot.as<uint32_t>(), x->huid.as<uint64_t>(), x->uoff.as<uint64_t>(),
      x->uout.as<uint2>(), reinterpret_cast<uint2*>(out), x->blockmap2.as<uint32_t>());
  other += 2;
  CK(cudaGetLastError());
  x->stats.rows_unique += utotal;
  return HFM_OK;
}

static void begin_stats(hfm_index* x) {
  x->stats = hfm_stats{};
  x->k_search_rec = x->k_resolve_rec = false;
  cudaEventRecord(x->ev[0], x->stream);
}
static int end_stats(hfm_index* x) {
  cudaEventRecord(x->ev[2], x->stream);
  RET(wait_event(x, x->ev[2]));
  float a = 0, b = 0;
  cudaEventElapsedTime(&a, x->ev[0], x->ev[1]);
  cudaEventElapsedTime(&b, x->ev[1], x->ev[2]);
  x->stats.ms_search = a; x->stats.ms_resolve = b; x->stats.ms_total = a + b;
  float ks = 0, kr = 0;
  if (x->k_search_rec) cudaEventElapsedTime(&ks, x->evk[0], x->evk[1]);
  if (x->k_resolve_rec) cudaEventElapsedTime(&kr, x->evk[2], x->evk[3]);
  x->stats.ms_search_kernel = ks; x->stats.ms_resolve_kernel = kr;
  return HFM_OK;
}

// ---------------------------------------------------------------------------
// Pipelines (device buffers in, device buffers out)
// ---------------------------------------------------------------------------
static int count_device(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq, uint32_t* d_counts) {
  begin_stats(x);
  uint32_t launches = 0;
  RET(run_bsearch(x, d_q, d_qoff, nq, 0, false, d_counts, launches));
  cudaEventRecord(x->ev[1], x->stream);
  RET(end_stats(x));
  x->stats.search_launches = launches;
  return HFM_OK;
}

static int locate_device(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq, uint32_t cap,
                         hfm_dev_hits* out) {
  begin_stats(x);
  uint32_t launches = 0, other = 0;
  RET(x->counts.ensure((size_t)nq * 4 + 4));
  RET(run_bsearch(x, d_q, d_qoff, nq, cap, true, x->counts.as<uint32_t>(), launches));
  RET(x->seg_base.ensure(((size_t)nq + 1) * 8));
  RET(x->pos_base.ensure(((size_t)nq + 1) * 8));
  RET(scan(x, x->niv.as<uint32_t>(), 1, nq, x->seg_base.as<uint64_t>(), other));
  RET(scan(x, x->nhits.as<uint64_t>(), 1, nq, x->pos_base.as<uint64_t>(), other));
  uint64_t nseg = 0, total = 0;
  RET(read_u64(x, x->seg_base.as<uint64_t>() + nq, nseg));
  RET(read_u64(x, x->pos_base.as<uint64_t>() + nq, total));
  RET(x->seg_row.ensure(nseg * 4 + 4));
  RET(x->seg_off.ensure((nseg + 1) * 8));
  RET(x->out_pairs.ensure(total * 8 + 8));
  if (nq) {
    k_gather_locate<<<(nq + 255) / 256, 256, 0, x->stream>>>(x->ivpool.as<uint2>(), x->ivoff.as<uint64_t>(),
                                                            x->niv.as<uint32_t>(), x->seg_base.as<uint64_t>(),
                                                            x->pos_base.as<uint64_t>(), nq, cap,
                                                            x->seg_row.as<uint32_t>(), x->seg_off.as<uint64_t>());
    other++;
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(x->seg_off.as<uint64_t>() + nseg, &total, 8, cudaMemcpyHostToDevice, x->stream));
  cudaEventRecord(x->ev[1], x->stream);
  uint32_t rl = 0;
  RET(resolve_segments(x, x->fwd, x->seg_row.as<uint32_t>(), 1, x->seg_off.as<uint64_t>(), nseg, total,
              x->fwd.bounds.as<uint32_t>(), (uint32_t)x->fwd.seq_boundaries.size(), x->out_pairs.as<uint32_t>(), rl, other));
  RET(read_ctr(x));
  RET(end_stats(x));
  x->stats.search_launches = launches; x->stats.resolve_launches = rl; x->stats.other_launches = other;
  x->stats.rows_resolved = total; x->stats.lf_calls = x->h_ctr->steps;
  if (x->h_ctr->walk_err) return set_error(HFM_E_WALK, "LF walk exceeded sample_rate steps: index inconsistent");
  out->nq = nq; out->total = total;
  out->d_offsets = x->pos_base.as<uint64_t>(); out->d_counts = x->counts.as<uint32_t>();
  out->d_pairs = x->out_pairs.as<uint32_t>();
  return HFM_OK;
}

// Sort key of a read for the prefix queue order: its first 16 codes, 4 bits each, the first
// code in the top bits; a shorter read is padded with code 0, which no read holds.
__global__ void k_prefix_keys(const uint8_t* __restrict__ q, const uint64_t* __restrict__ qoff, uint32_t n,
                              unsigned long long* __restrict__ keys, uint32_t* __restrict__ ids) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t o = qoff[i], len = qoff[i + 1] - o;
  unsigned long long k = 0;
#pragma unroll
  for (uint32_t j = 0; j < 16; j++) k = (k << 4) | (j < len ? (unsigned long long)(q[o + j] & 15u) : 0ull);
  keys[i] = k;
  ids[i] = i;
}

// The queue order of read_order = 1: reads sorted by their first 16 codes (radix sort of
// key / index pairs on the handle's stream).  Reads that share a prefix then sit in one
// warp and carry the same reference windows (on an IUPAC text, the N-run windows that a
// read's first bases select), so their interval sets have alike sizes and their Occ
// records are fetched once for the warp.  Any order gives the same results.
static int prefix_order(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq, const uint32_t*& order,
                        uint32_t& launches, bool launch = true) {
  RET(x->okeys.ensure((size_t)nq * 16 + 16));
  RET(x->oids.ensure((size_t)nq * 8 + 8));
  unsigned long long* k_in = x->okeys.as<unsigned long long>();
  unsigned long long* k_out = k_in + nq;
  uint32_t* i_in = x->oids.as<uint32_t>();
  uint32_t* i_out = i_in + nq;
  size_t temp = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, temp, k_in, k_out, i_in, i_out, (int)nq, 0, 64, x->stream));
  RET(x->otemp.ensure(temp + 16));
  order = i_out;
  if (!launch) return HFM_OK;                  // sizing pass of a graph capture
  k_prefix_keys<<<(nq + 255) / 256, 256, 0, x->stream>>>(d_q, d_qoff, nq, k_in, i_in);
  CK(cudaGetLastError());
  CK(cub::DeviceRadixSort::SortPairs(x->otemp.p, temp, k_in, k_out, i_in, i_out, (int)nq, 0, 64, x->stream));
  launches += nq > 8192 ? 11 : 2;     // keys, then a histogram, a scan and 8 one-sweep passes (one tile when small)
  order = i_out;
  return HFM_OK;
}

static int mems_device(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq, uint32_t min_len,
                       uint32_t mode, const uint32_t* h_bounds, uint32_t nb, uint32_t cap, hfm_dev_mems* out,
                       const hfm_sched* sc = nullptr) {
  if (x->kind != HFM_KIND_BIDIR) return set_error(HFM_E_ARG, "MEM/SMEM search needs a bidirectional index");
  if (mode > 1) return set_error(HFM_E_ARG, "mode must be 0 (SMEM) or 1 (MEM)");
  const uint32_t* order = sc ? sc->d_order : nullptr;
  uint32_t n_warp = sc ? sc->n_warp : 0;
  bool own_order = false;                      // an order made here: a permutation by construction
  if (!sc && x->threads_per_read > 1 && x->mems_variant != MEMS_PLAIN && nq) {
    // every read on the lane-group kernels (a warp or 4, 8, 16 lanes per read): the
    // identity order, all of it routed
    RET(x->iota.ensure((size_t)nq * 4));
    k_iota<<<(nq + 255) / 256, 256, 0, x->stream>>>(x->iota.as<uint32_t>(), nq);
    CK(cudaGetLastError());
    order = x->iota.as<uint32_t>();
    n_warp = nq;
  }
  uint32_t* wlog = sc ? sc->d_work_log : nullptr;
  if (n_warp > nq) return set_error(HFM_E_ARG, "sched.n_warp exceeds nq");
  if (n_warp && !order) return set_error(HFM_E_ARG, "sched.n_warp needs sched.d_order");
  begin_stats(x);
  uint32_t launches = 0, other = 0;
  if (!order && x->read_order == 1 && x->threads_per_read == 1 && x->mems_variant != MEMS_PLAIN && nq > 1) {
    RET(prefix_order(x, d_q, d_qoff, nq, order, other));
    own_order = true;
  }
  if (order && nq && !own_order) {
    // the order must be a permutation of 0..nq-1: every read is processed exactly once
    RET(x->hflags.ensure((size_t)nq * 4));
    CK(cudaMemsetAsync(x->hflags.p, 0, (size_t)nq * 4, x->stream));
    CK(cudaMemsetAsync(&dctr(x)->walk_err, 0, 4, x->stream));
    k_check_perm<<<(nq + 255) / 256, 256, 0, x->stream>>>(order, nq, x->hflags.as<uint32_t>(), &dctr(x)->walk_err);
    other++;
    CK(cudaGetLastError());
    RET(read_ctr(x));
    if (x->h_ctr->walk_err) return set_error(HFM_E_ARG, "sched.d_order is not a permutation of 0..nq-1");
  }
  bool counting = x->count_work || wlog;
  RET(x->ref_bounds.ensure((size_t)nb * 4 + 4));
  if (nb) CK(cudaMemcpyAsync(x->ref_bounds.p, h_bounds, (size_t)nb * 4, cudaMemcpyHostToDevice, x->stream));
  RET(x->hit_start.ensure((size_t)nq * 8 + 8)); RET(x->hit_count.ensure((size_t)nq * 4 + 4));
  RET(x->status.ensure((size_t)nq * 4 + 4)); RET(x->ovf.ensure((size_t)nq * 4 + 4));
  if (x->miv_cap < (uint64_t)nq * 24 + 4096) x->miv_cap = (uint64_t)nq * 24 + 4096;     // BIv = 16 B
  if (x->hit_cap < (uint64_t)nq * 24 + 4096) x->hit_cap = (uint64_t)nq * 24 + 4096;   // hit = 32 B
  MemsParams P{min_len, mode, cap, nb ? 1u : 0u};
  const FmDev& Fw = x->fwd; const FmDev& Rv = x->rev;
  // persistent fast pass: one wave of resident threads, MEM_SET_CAP intervals per set.
  // Variant 2: 8 resident blocks of 128 threads per SM with a 32-entry candidate list in
  // local memory; variant 3 (default): 8 blocks per SM with a 1024-entry list per thread
  // in global memory, so reads up to ~10 kbp finish in this pass.  The kernels are
  // specialised for the index's Occ record format (narrow or wide).
  int variant = x->mems_variant;
  int bpsm = 0;
  const uint32_t fmt = Fw.fmt;
  WITH_FMT(fmt, {
    if (variant == 3) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k_mems<false, 32, 0, 8, FM>, 128, 0));
    else CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k_mems<false, 32, MEM_KC, 8, FM>, 128, 0));
  });
  const uint64_t full_threads = (uint64_t)std::max(1, bpsm) * x->num_sms * 128;
  uint64_t threads = std::min<uint64_t>(full_threads, ((uint64_t)nq + 127) / 128 * 128);
  // Long reads (SMEM mode with global candidate lists) take the segmented sweep: the
  // fast pass gets the other reads, in the same relative order.
  const uint32_t* fast_ids = order ? order + n_warp : nullptr;
  uint32_t n_fast = nq - n_warp, n_long = 0;
  uint64_t n_units = 0;
  if (mode == 0 && variant == 3 && n_fast > 0 && min_len > 0) {
    RET(x->lflag.ensure((size_t)n_fast * 4 + 4));
    RET(x->lpos.ensure(((size_t)n_fast + 1) * 8));
    k_long_flags<<<(n_fast + 255) / 256, 256, 0, x->stream>>>(fast_ids, n_fast, d_qoff, 2 * x->seg_len,
                                                              x->lflag.as<uint32_t>());
    other++;
    CK(cudaGetLastError());
    RET(scan(x, x->lflag.as<uint32_t>(), 1, n_fast, x->lpos.as<uint64_t>(), other));
    uint64_t nl = 0;
    RET(read_u64(x, x->lpos.as<uint64_t>() + n_fast, nl));
    n_long = (uint32_t)nl;
    if (n_long) {
      RET(x->sids.ensure((size_t)n_fast * 4 + 4));
      RET(x->lids.ensure((size_t)n_long * 4 + 4));
      RET(x->ucount.ensure((size_t)n_long * 4 + 4));
      k_split_ids<<<(n_fast + 255) / 256, 256, 0, x->stream>>>(fast_ids, n_fast, x->lflag.as<uint32_t>(),
                                                               x->lpos.as<uint64_t>(), x->sids.as<uint32_t>(),
                                                               x->lids.as<uint32_t>(), x->ucount.as<uint32_t>(), d_qoff,
                                                               x->seg_len);
      other++;
      CK(cudaGetLastError());
      RET(x->ubase.ensure(((size_t)n_long + 1) * 8));
      RET(scan(x, x->ucount.as<uint32_t>(), 1, n_long, x->ubase.as<uint64_t>(), other));
      RET(read_u64(x, x->ubase.as<uint64_t>() + n_long, n_units));
      RET(x->uread.ensure(n_units * 4)); RET(x->uk.ensure(n_units * 4));
      RET(x->ubits.ensure(n_units * (x->seg_len / 32) * 4)); RET(x->uexit.ensure(n_units * 4));
      RET(x->ust.ensure(n_units * 4)); RET(x->ucoff.ensure(n_units * 8)); RET(x->ucnt.ensure(n_units * 4));
      RET(x->fxe.ensure(n_units * 4)); RET(x->fxc.ensure(n_units * 4)); RET(x->fxx.ensure(n_units * 4));
      RET(x->fxo.ensure(n_units * 8)); RET(x->fxn.ensure(n_units * 4));
      k_unit_fill<<<(n_long + 255) / 256, 256, 0, x->stream>>>(x->lids.as<uint32_t>(), n_long, x->ubase.as<uint64_t>(),
                                                               x->uread.as<uint32_t>(), x->uk.as<uint32_t>());
      other++;
      CK(cudaGetLastError());
      fast_ids = x->sids.as<uint32_t>();
      n_fast -= n_long;
      x->seg_cap = std::max<uint64_t>(x->seg_cap, n_units * 24 + 65536);
      threads = std::max<uint64_t>(threads, std::min<uint64_t>(full_threads, (n_units + 127) / 128 * 128));
    }
  }
  const bool plain = variant == MEMS_PLAIN;
  if (plain && (order || n_warp)) return set_error(HFM_E_ARG, "the plain launch takes no schedule");
  if (!plain) {
    RET(x->memwork.ensure(std::max<uint64_t>(threads, 32) * 4 * MEM_SET_CAP * 16));
    // variant 3: candidate lists in global memory (FAST_CAND_CAP per thread), so long reads
    // stay on the fast pass instead of overflowing a 32-entry local list
    if (variant == 3) RET(x->cwork.ensure((size_t)std::max<uint64_t>(threads, 128) * FAST_CAND_CAP * sizeof(Cand)));
  } else if (nq) {
    // plain launch, count pass: every read's MemHits and positions counted by a full
    // search, read back and prefix-summed to size the outputs before the write pass
    RET(x->npos.ensure((size_t)nq * 4 + 4));
    CK(cudaMemsetAsync(x->ctr.p, 0, sizeof(Counters), x->stream));
    MemsOut oc{x->hit_start.as<uint64_t>(), x->hit_count.as<uint32_t>(), x->status.as<uint32_t>(),
               x->ovf.as<uint32_t>(), &dctr(x)->n_ovf, &dctr(x)->touches};
    Pool none{nullptr, &dctr(x)->iv_used, 0};
    cudaEventRecord(x->evk[0], x->stream);
    WITH_FMT(fmt, {
      if (counting)
        k_mems_plain<true, 0, FM><<<(nq + 127) / 128, 128, 0, x->stream>>>(
            Fw.d, Rv.d, Fw.compat.as<uint16_t>(), Rv.compat.as<uint16_t>(), d_q, d_qoff, P, nq, none, none, oc,
            x->npos.as<uint32_t>(), &dctr(x)->seg_used);
      else
        k_mems_plain<false, 0, FM><<<(nq + 127) / 128, 128, 0, x->stream>>>(
            Fw.d, Rv.d, Fw.compat.as<uint16_t>(), Rv.compat.as<uint16_t>(), d_q, d_qoff, P, nq, none, none, oc,
            x->npos.as<uint32_t>(), &dctr(x)->seg_used);
    });
    launches++;
    CK(cudaGetLastError());
    RET(read_ctr(x));
    const uint64_t ivs_need = x->h_ctr->seg_used;
    x->stats.occ_touches += x->h_ctr->touches;
    RET(x->hit_base.ensure(((size_t)nq + 1) * 8));
    RET(scan(x, x->hit_count.as<uint32_t>(), 1, nq, x->hit_base.as<uint64_t>(), other));
    uint64_t counted = 0;
    RET(read_u64(x, x->hit_base.as<uint64_t>() + nq, counted));
    x->hit_cap = counted + 4096;             // exact for the reads the write pass completes
    x->miv_cap = ivs_need + 4096;
  }
  bool done = false;
  for (int attempt = 0; attempt < 8 && !done; attempt++) {
    RET(x->mivpool.ensure(x->miv_cap * 16)); x->miv_cap = x->mivpool.cap / 16;
    if (n_long) { RET(x->segpool.ensure(x->seg_cap * sizeof(Cand))); x->seg_cap = x->segpool.cap / sizeof(Cand); }
    RET(x->hitpool.ensure(x->hit_cap * 32)); x->hit_cap = x->hitpool.cap / 32;
    CK(cudaMemsetAsync(x->ctr.p, 0, sizeof(Counters), x->stream));
    if (wlog && nq) CK(cudaMemsetAsync(wlog, 0, (size_t)nq * 16, x->stream));
    Pool ivp{x->mivpool.p, &dctr(x)->iv_used, x->miv_cap}, hp{x->hitpool.p, &dctr(x)->hit_used, x->hit_cap};
    MemsOut o{x->hit_start.as<uint64_t>(), x->hit_count.as<uint32_t>(), x->status.as<uint32_t>(),
              x->ovf.as<uint32_t>(), &dctr(x)->n_ovf, &dctr(x)->touches};
    if (n_warp) {   // reads the schedule sends straight to the warp-per-read kernel head the long-tail list
      CK(cudaMemcpyAsync(x->ovf.p, order, (size_t)n_warp * 4, cudaMemcpyDeviceToDevice, x->stream));
      CK(cudaMemcpyAsync(&dctr(x)->n_ovf, &n_warp, 4, cudaMemcpyHostToDevice, x->stream));
    }
    if (plain && nq) {
      // plain launch, write pass: the same search again, writing into the counted pools
      WITH_FMT(fmt, {
        if (counting)
          k_mems_plain<true, 1, FM><<<(nq + 127) / 128, 128, 0, x->stream>>>(
              Fw.d, Rv.d, Fw.compat.as<uint16_t>(), Rv.compat.as<uint16_t>(), d_q, d_qoff, P, nq, ivp, hp, o,
              x->npos.as<uint32_t>(), &dctr(x)->seg_used);
        else
          k_mems_plain<false, 1, FM><<<(nq + 127) / 128, 128, 0, x->stream>>>(
              Fw.d, Rv.d, Fw.compat.as<uint16_t>(), Rv.compat.as<uint16_t>(), d_q, d_qoff, P, nq, ivp, hp, o,
              x->npos.as<uint32_t>(), &dctr(x)->seg_used);
      });
      launches++;
      CK(cudaGetLastError());
      cudaEventRecord(x->evk[1], x->stream);
      x->k_search_rec = true;
    }
    if (!plain && (n_fast > 0 || n_long > 0)) cudaEventRecord(x->evk[0], x->stream);
    if (!plain && n_fast > 0 && n_long == 0) {     // with long reads, k_mems_seg runs the short reads too
      MemsWork W{x->memwork.as<BIv>(), MEM_SET_CAP, variant == 3 ? x->cwork.as<Cand>() : nullptr,
                 variant == 3 ? FAST_CAND_CAP : 0u, &dctr(x)->queue, fast_ids, n_fast, &dctr(x)->still_ovf, 0u, wlog};
      W.chunk = x->queue_chunk;
      unsigned grid = (unsigned)(threads / 128);
      if (x->memwork.cap < (size_t)grid * 128 * 4 * MEM_SET_CAP * 16) return set_error(HFM_E_ARG, "internal: work area too small");
      if (variant == 3 && x->cwork.cap < (size_t)grid * 128 * FAST_CAND_CAP * sizeof(Cand))
        return set_error(HFM_E_ARG, "internal: candidate area too small");
      WITH_FMT(fmt, {
        if (counting && variant == 3)
          k_mems<true, 32, 0, 5, FM><<<grid, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                  Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, hp, o, W);
        else if (counting)
          k_mems<true, 32, MEM_KC, 5, FM><<<grid, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                       Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, hp,
                                                                       o, W);
        else if (variant == 3)
          k_mems<false, 32, 0, 8, FM><<<grid, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                   Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, hp, o, W);
        else
          k_mems<false, 32, MEM_KC, 8, FM><<<grid, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                        Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, hp,
                                                                        o, W);
      });
      launches++;
      CK(cudaGetLastError());
    }
    if (n_long > 0) {
      // segmented sweep of the long reads, then the merge along each read's true chain
      SegWork G{x->seg_len, x->seg_len / 32, x->uread.as<uint32_t>(), x->uk.as<uint32_t>(), (uint32_t)n_units, x->ubits.as<uint32_t>(),
                x->uexit.as<uint32_t>(), x->ust.as<uint32_t>(), x->ucoff.as<uint64_t>(), x->ucnt.as<uint32_t>(),
                x->segpool.as<Cand>(), &dctr(x)->seg_used, x->seg_cap, fast_ids, n_fast, x->lids.as<uint32_t>(),
                x->ubase.as<uint64_t>(), n_long, &dctr(x)->merge_queue, &dctr(x)->touches, x->fxe.as<uint32_t>(),
                x->fxc.as<uint32_t>(), x->fxx.as<uint32_t>(), x->fxo.as<uint64_t>(), x->fxn.as<uint32_t>()};
      MemsWork W{x->memwork.as<BIv>(), MEM_SET_CAP, x->cwork.as<Cand>(), FAST_CAND_CAP, &dctr(x)->seg_queue, nullptr,
                 0u, &dctr(x)->still_ovf, 0u, wlog};
      W.chunk = x->queue_chunk;
      MemsWork Wf = W;
      Wf.queue = &dctr(x)->fix_queue;
      uint64_t ts = std::min<uint64_t>(threads / 128 * 128, (n_units + n_fast + 127) / 128 * 128);
      uint64_t tmg = std::min<uint64_t>(threads / 128 * 128, ((uint64_t)n_long + 127) / 128 * 128);
      unsigned gs = (unsigned)std::max<uint64_t>(1, ts / 128), gm = (unsigned)std::max<uint64_t>(1, tmg / 128);
      if (x->memwork.cap < (size_t)gs * 128 * 4 * MEM_SET_CAP * 16 || x->cwork.cap < (size_t)gs * 128 * FAST_CAND_CAP * sizeof(Cand))
        return set_error(HFM_E_ARG, "internal: work area too small");
      WITH_FMT(fmt, {
        if (counting) {
          k_mems_seg<true, 32, 5, FM><<<gs, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                 Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, hp, o, W, G);
          k_mems_fix<true, 32, 5, FM><<<gs, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                 Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, Wf, G);
          k_mems_merge<true, 32, 5, FM><<<gm, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                   Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, hp, o,
                                                                   W, G);
        } else {
          k_mems_seg<false, 32, 8, FM><<<gs, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                  Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, hp, o, W,
                                                                  G);
          k_mems_fix<false, 32, 8, FM><<<gs, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                  Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, Wf, G);
          k_mems_merge<false, 32, 8, FM><<<gm, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                    Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, hp, o,
                                                                    W, G);
        }
      });
      launches += 3;
      CK(cudaGetLastError());
    }
    if (!plain && (n_fast > 0 || n_long > 0)) {
      cudaEventRecord(x->evk[1], x->stream);
      x->k_search_rec = true;
    }
    RET(read_ctr(x));
    uint32_t n_ovf = x->h_ctr->n_ovf;
    const uint32_t* wlist = x->ovf.as<uint32_t>();
    if (n_ovf) {
      x->stats.fallback_reads += n_ovf;
      // Reads that outgrew only the 32-entry candidate list (long reads) rerun on the
      // per-thread kernel with a MID_CAND_CAP-entry list in global memory; set overflows,
      // reads the schedule routed, and middle-tier overflows go to the warp-per-read kernel.
      RET(x->ovf2.ensure((size_t)nq * 4 + 4));
      RET(x->ovf3.ensure((size_t)nq * 4 + 4));
      CK(cudaMemsetAsync(&dctr(x)->n_mid, 0, 12, x->stream));
      k_split_ovf<<<(n_ovf + 255) / 256, 256, 0, x->stream>>>(x->ovf.as<uint32_t>(), n_ovf, n_warp,
                                                              x->status.as<uint32_t>(), x->ovf3.as<uint32_t>(),
                                                              &dctr(x)->n_mid, x->ovf2.as<uint32_t>(), &dctr(x)->n_wrp);
      other++;
      CK(cudaGetLastError());
      RET(read_ctr(x));
      uint32_t n_mid = x->h_ctr->n_mid;
      if (n_mid) {
        uint64_t tm = std::min<uint64_t>({((uint64_t)n_mid + 127) / 128 * 128, (uint64_t)x->num_sms * MID_THREADS_PER_SM,
                                          threads / 128 * 128});
        tm = std::max<uint64_t>(tm, 128);
        unsigned grid = (unsigned)(tm / 128);
        if (x->memwork.cap < (size_t)grid * 128 * 4 * MEM_SET_CAP * 16) return set_error(HFM_E_ARG, "internal: work area too small");
        RET(x->cwork.ensure((size_t)grid * 128 * MID_CAND_CAP * sizeof(Cand)));
        MemsWork W{x->memwork.as<BIv>(), MEM_SET_CAP, x->cwork.as<Cand>(), MID_CAND_CAP, &dctr(x)->queue3,
                   x->ovf3.as<uint32_t>(), n_mid, &dctr(x)->still_ovf, 0u, wlog};
        MemsOut o2 = o;
        o2.ovf_list = x->ovf2.as<uint32_t>();
        o2.n_ovf = &dctr(x)->n_wrp;
        WITH_FMT(fmt, {
          if (counting)
            k_mems<true, 32, 0, 5, FM><<<grid, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                    Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, hp, o2,
                                                                    W);
          else
            k_mems<false, 32, 0, 8, FM><<<grid, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(),
                                                                     Rv.compat.as<uint16_t>(), d_q, d_qoff, P, ivp, hp, o2,
                                                                     W);
        });
        launches++;
        CK(cudaGetLastError());
        RET(read_ctr(x));
      }
      n_ovf = x->h_ctr->n_wrp;
      wlist = x->ovf2.as<uint32_t>();
    }
    const uint32_t G = (!sc && n_warp == nq && x->threads_per_read > 1) ? x->threads_per_read : 32u;
    if (n_ovf && G < 32) {
      // sub-warp pass over every read (threads_per_read 4, 8 or 16): one read per group of
      // G lanes with the fast pass's set and candidate capacities; reads that outgrow them
      // go on to the warp tier below
      const uint64_t per_group = (uint64_t)MEM_SET_CAP * 4 * 16 + (uint64_t)FAST_CAND_CAP * sizeof(Cand);
      const uint64_t groups = std::min<uint64_t>({(uint64_t)n_ovf, (uint64_t)x->num_sms * (2048 / G),
                                                  std::max<uint64_t>(128 / G, (8ull << 30) / per_group)});
      const unsigned grid = (unsigned)((groups * G + 127) / 128);
      RET(x->work.ensure((size_t)grid * (128 / G) * MEM_SET_CAP * 4 * 16));
      RET(x->cwork.ensure((size_t)grid * (128 / G) * FAST_CAND_CAP * sizeof(Cand)));
      RET(x->ovf3.ensure((size_t)nq * 4 + 4));
      CK(cudaMemsetAsync(&dctr(x)->n_mid, 0, 4, x->stream));
      CK(cudaMemsetAsync(&dctr(x)->queue2, 0, 4, x->stream));
      MemsWork W{x->work.as<BIv>(), MEM_SET_CAP, x->cwork.as<Cand>(), FAST_CAND_CAP, &dctr(x)->queue2, wlist,
                 n_ovf, &dctr(x)->still_ovf, 0u, wlog};
      MemsOut o3 = o;
      o3.ovf_list = x->ovf3.as<uint32_t>();
      o3.n_ovf = &dctr(x)->n_mid;
      auto sub = [&](auto kern) {
        kern<<<grid, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(), Rv.compat.as<uint16_t>(), d_q, d_qoff,
                                          P, ivp, hp, o3, W);
      };
      if (G == 4) { if (counting) sub(k_mems_warp<true, 4>); else sub(k_mems_warp<false, 4>); }
      else if (G == 8) { if (counting) sub(k_mems_warp<true, 8>); else sub(k_mems_warp<false, 8>); }
      else { if (counting) sub(k_mems_warp<true, 16>); else sub(k_mems_warp<false, 16>); }
      launches++;
      CK(cudaGetLastError());
      RET(read_ctr(x));
      n_ovf = x->h_ctr->n_mid;
      wlist = x->ovf3.as<uint32_t>();
    }
    if (n_ovf) {
      // long tail: one warp per overflowed read, 4 sets and a candidate list per warp,
      // growing 4x until every read fits
      uint32_t set_cap = MEM_WARP_SET_CAP, cand_cap = 1024;
      while (true) {
        uint64_t per_warp = (uint64_t)set_cap * 4 * 16 + (uint64_t)cand_cap * sizeof(Cand);
        uint64_t warps = std::min<uint64_t>({(uint64_t)n_ovf, (uint64_t)x->num_sms * 16,
                                             std::max<uint64_t>(4, (2ull << 30) / per_warp)});
        unsigned grid = (unsigned)((warps + 3) / 4);
        RET(x->work.ensure((size_t)grid * 4 * set_cap * 4 * 16));
        RET(x->cwork.ensure((size_t)grid * 4 * cand_cap * sizeof(Cand)));
        CK(cudaMemsetAsync(&dctr(x)->still_ovf, 0, 4, x->stream));
        CK(cudaMemsetAsync(&dctr(x)->queue2, 0, 4, x->stream));
        MemsWork W{x->work.as<BIv>(), set_cap, x->cwork.as<Cand>(), cand_cap, &dctr(x)->queue2, wlist,
                   n_ovf, &dctr(x)->still_ovf, 1u, wlog};
        if (counting)
          k_mems_warp<true><<<grid, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(), Rv.compat.as<uint16_t>(),
                                                        d_q, d_qoff, P, ivp, hp, o, W);
        else
          k_mems_warp<false><<<grid, 128, 0, x->stream>>>(Fw.d, Rv.d, Fw.compat.as<uint16_t>(), Rv.compat.as<uint16_t>(),
                                                         d_q, d_qoff, P, ivp, hp, o, W);
        launches++;
        CK(cudaGetLastError());
        RET(read_ctr(x));
        if (x->h_ctr->still_ovf == 0) break;
        if (set_cap >= (1u << 22)) return set_error(HFM_E_OVERFLOW, "MEM interval set exceeds 2^22 intervals");
        set_cap *= 4; cand_cap *= 4;
      }
    }
    if (x->h_ctr->iv_used <= x->miv_cap && x->h_ctr->hit_used <= x->hit_cap &&
        (n_long == 0 || x->h_ctr->seg_used <= x->seg_cap)) { done = true; break; }
    x->miv_cap = std::max(x->miv_cap, (uint64_t)(x->h_ctr->iv_used * 3 / 2 + 4096));
    x->hit_cap = std::max(x->hit_cap, (uint64_t)(x->h_ctr->hit_used * 3 / 2 + 4096));
    if (n_long) x->seg_cap = std::max(x->seg_cap, (uint64_t)(x->h_ctr->seg_used * 3 / 2 + 65536));
  }
  if (!done) return set_error(HFM_E_OVERFLOW, "MEM pools did not converge");
  x->stats.occ_touches += x->h_ctr->touches;
  // CSR of hits, then positions
  RET(x->hit_base.ensure(((size_t)nq + 1) * 8));
  RET(scan(x, x->hit_count.as<uint32_t>(), 1, nq, x->hit_base.as<uint64_t>(), other));
  uint64_t nh = 0;
  RET(read_u64(x, x->hit_base.as<uint64_t>() + nq, nh));
  RET(x->hits.ensure(nh * 32 + 32));
  if (nq) {
    k_gather_hits<<<(nq + 255) / 256, 256, 0, x->stream>>>(x->hitpool.as<uint4>(), x->hit_start.as<uint64_t>(),
                                                          x->hit_count.as<uint32_t>(), x->hit_base.as<uint64_t>(), nq,
                                                          x->hits.as<uint4>());
    other++;
    CK(cudaGetLastError());
  }
  RET(x->npos_scan.ensure((nh + 1) * 8));
  RET(scan(x, x->hits.as<uint32_t>() + 5, 8, nh, x->npos_scan.as<uint64_t>(), other));
  uint64_t npos = 0;
  RET(read_u64(x, x->npos_scan.as<uint64_t>() + nh, npos));
  if (nh) {
    k_set_pos_off<<<(unsigned)((nh + 255) / 256), 256, 0, x->stream>>>(x->hits.as<uint32_t>(), x->npos_scan.as<uint64_t>(), nh);
    other++;
    CK(cudaGetLastError());
  }
  if (wlog && nq) {
    k_work_log<<<(nq + 255) / 256, 256, 0, x->stream>>>(x->hit_base.as<uint64_t>(), x->npos_scan.as<uint64_t>(), nq, wlog);
    other++;
    CK(cudaGetLastError());
  }
  RET(x->out_pairs.ensure(npos * 8 + 8));
  cudaEventRecord(x->ev[1], x->stream);
  uint32_t rl = 0;
  RET(resolve_segments(x, Fw, x->hits.as<uint32_t>() + 4, 8, x->npos_scan.as<uint64_t>(), nh, npos,
              x->ref_bounds.as<uint32_t>(), nb, x->out_pairs.as<uint32_t>(), rl, other));
  RET(read_ctr(x));
  RET(end_stats(x));
  x->stats.search_launches = launches; x->stats.resolve_launches = rl; x->stats.other_launches = other;
  x->stats.rows_resolved = npos; x->stats.lf_calls = x->h_ctr->steps; x->stats.hits_out = nh;
  if (x->h_ctr->walk_err) return set_error(HFM_E_WALK, "LF walk exceeded sample_rate steps: index inconsistent");
  out->nq = nq; out->n_hits = nh; out->n_positions = npos;
  out->d_hit_offsets = x->hit_base.as<uint64_t>(); out->d_hits = x->hits.as<hfm_mem_hit>();
  out->d_positions = x->out_pairs.as<uint32_t>();
  return HFM_OK;
}

// ---------------------------------------------------------------------------
// The SMEM/MEM pass chain with fixed capacities, for CUDA-graph capture.
//
// mems_device decides on the host between passes (the overflow tiers it runs, how many
// long-read segments there are, how large the outputs are) and so reads counters back
// after every pass.  This chain makes every such decision on the device: each pass runs
// over capacities fixed beforehand (the handle's reserved pools, `pos_cap` positions) and
// reads its counts from device memory, so the whole chain is one stream of asynchronous
// work that a CUDA graph can capture and replay.  Whatever outgrows a capacity is only
// flagged (pool counters, still_ovf, the totals' overflow bit): the host checks the flags
// after the replay and reruns the batch on mems_device, which gives the same results.
//
// fixed_chain(launch = false) makes every allocation the chain needs; fixed_chain(launch =
// true) issues the same sequence of kernels and copies, allocating nothing.
// ---------------------------------------------------------------------------
struct GraphTotals { uint64_t nh, npos, upos; uint32_t ovf, _pad; };

// Totals of the chain: MemHits, and the position counts the resolve passes cover, both 0
// (with ovf set) when a count exceeds the position capacity.
__global__ void k_graph_totals(const uint64_t* __restrict__ hit_base, uint32_t nq, const uint64_t* __restrict__ pos_total,
                               const uint64_t* __restrict__ u_total, uint64_t pos_cap, uint64_t upos_cap,
                               GraphTotals* __restrict__ t) {
  if (blockIdx.x || threadIdx.x) return;
  const uint64_t np = *pos_total, nu = u_total ? *u_total : 0;
  const bool over = np > pos_cap || nu > upos_cap;
  t->nh = hit_base[nq];
  t->npos = over ? 0 : np;
  t->upos = over ? 0 : nu;
  t->ovf = over ? 1u : 0u;
}

struct FixedChain {
  const uint8_t* d_q; const uint64_t* d_qoff; uint32_t nq;
  uint64_t max_bases;          // reads of at most this many codes in total
  MemsParams P; uint32_t nb;   // ref bounds already in x->ref_bounds
  bool dedup;
  uint64_t pos_cap;
  uint64_t upos_cap;           // distinct positions (rows walked once by the deduplicated resolve)
  GraphTotals* d_tot; GraphTotals* h_tot;     // device / pinned host
  uint64_t threads;            // resident threads of the persistent kernels
  uint32_t warp_cap = MEM_WARP_SET_CAP, warp_cands = 1024;   // warp tier: intervals per set, candidates
};

static int fixed_chain(hfm_index* x, FixedChain& c, bool launch) {
  const uint32_t nq = c.nq;
  const FmDev& Fw = x->fwd; const FmDev& Rv = x->rev;
  const uint32_t fmt = Fw.fmt;
  uint32_t dummy = 0;
  auto SCAN = [&](auto* in, uint32_t stride, uint64_t n, uint64_t* out) -> int {
    if (!launch) {
      uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
      return x->scan_tmp.ensure((tiles + 1) * 8);
    }
    return scan(x, in, stride, n, out, dummy);
  };
  const uint64_t hcap = x->hit_cap, pcap = c.pos_cap, upcap = std::min(c.upos_cap, c.pos_cap);
  if (hcap >= 0xFFFFFFFFull) return set_error(HFM_E_ARG, "MemHit capacity above 2^32");
  // work buffers
  RET(x->hit_start.ensure((size_t)nq * 8 + 8)); RET(x->hit_count.ensure((size_t)nq * 4 + 4));
  RET(x->status.ensure((size_t)nq * 4 + 4)); RET(x->ovf.ensure((size_t)nq * 4 + 4));
  RET(x->ovf2.ensure((size_t)nq * 4 + 4)); RET(x->ovf3.ensure((size_t)nq * 4 + 4));
  RET(x->mivpool.ensure(x->miv_cap * 16)); RET(x->hitpool.ensure(hcap * 32));
  if (!launch) {                     // occupancy queried outside the capture
    int bpsm = 0;
    WITH_FMT(fmt, { CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k_mems<false, 32, 0, 8, FM>, 128, 0)); });
    c.threads = (uint64_t)std::max(1, bpsm) * x->num_sms * 128;
  }
  const uint64_t threads = c.threads;
  RET(x->memwork.ensure(threads * 4 * MEM_SET_CAP * 16));
  RET(x->cwork.ensure((size_t)threads * FAST_CAND_CAP * sizeof(Cand)));
  const bool seg = c.P.mode == 0 && c.P.min_len > 0;
  const uint64_t ucap = c.max_bases / x->seg_len + nq + 1;    // segments of the long reads
  if (seg) {
    RET(x->lflag.ensure((size_t)nq * 4 + 4)); RET(x->lpos.ensure(((size_t)nq + 1) * 8));
    RET(x->sids.ensure((size_t)nq * 4 + 4)); RET(x->lids.ensure((size_t)nq * 4 + 4));
    RET(x->ucount.ensure((size_t)nq * 4 + 4)); RET(x->ubase.ensure(((size_t)nq + 1) * 8));
    RET(x->uread.ensure(ucap * 4)); RET(x->uk.ensure(ucap * 4));
    RET(x->ubits.ensure(ucap * (x->seg_len / 32) * 4)); RET(x->uexit.ensure(ucap * 4));
    RET(x->ust.ensure(ucap * 4)); RET(x->ucoff.ensure(ucap * 8)); RET(x->ucnt.ensure(ucap * 4));
    RET(x->fxe.ensure(ucap * 4)); RET(x->fxc.ensure(ucap * 4)); RET(x->fxx.ensure(ucap * 4));
    RET(x->fxo.ensure(ucap * 8)); RET(x->fxn.ensure(ucap * 4));
    x->seg_cap = std::max<uint64_t>(x->seg_cap, ucap * 24 + 65536);
    RET(x->segpool.ensure(x->seg_cap * sizeof(Cand)));
  }
  // warp tier: up to 16 warps per SM, at most 2 GB of sets
  const uint64_t per_warp = (uint64_t)c.warp_cap * 4 * 16;
  const uint64_t wwarps = std::max<uint64_t>(4, std::min<uint64_t>((uint64_t)x->num_sms * 8, (2ull << 30) / per_warp));
  const uint32_t wgrid = (uint32_t)((wwarps + 3) / 4);
  RET(x->work.ensure((size_t)wgrid * 4 * per_warp));
  RET(x->cwork.ensure(std::max<size_t>((size_t)threads * FAST_CAND_CAP, (size_t)wgrid * 4 * c.warp_cands) * sizeof(Cand)));
  RET(x->hit_base.ensure(((size_t)nq + 1) * 8));
  RET(x->hits.ensure((hcap + 1) * 32));
  RET(x->npos_scan.ensure((hcap + 1) * 8));
  RET(x->out_pairs.ensure(pcap * 8 + 8));
  const uint64_t rblocks = (pcap + RES_T - 1) / RES_T, eblocks = (pcap + EXP_BLK - 1) / EXP_BLK;
  RET(x->blockmap.ensure(rblocks * 4 + 4));
  uint64_t hsize = 1024;
  while (hsize < 2 * hcap) hsize <<= 1;
  if (c.dedup) {
    RET(x->hkeys.ensure(hsize * 8)); RET(x->hslot.ensure(hcap * 4 + 4));
    RET(x->hflags.ensure(hsize * 4)); RET(x->huid.ensure((hsize + 1) * 8));
    RET(x->urow.ensure(hcap * 4 + 4)); RET(x->ulen.ensure(hcap * 4 + 4)); RET(x->uoff.ensure((hcap + 1) * 8));
    RET(x->uout.ensure(upcap * 8 + 8));
    RET(x->blockmap2.ensure(eblocks * 4 + 4));
  }
  const MemsParams& P = c.P;
  Counters* dc = dctr(x);
  Pool ivp{x->mivpool.p, &dc->iv_used, x->miv_cap}, hp{x->hitpool.p, &dc->hit_used, hcap};
  MemsOut o{x->hit_start.as<uint64_t>(), x->hit_count.as<uint32_t>(), x->status.as<uint32_t>(),
            x->ovf.as<uint32_t>(), &dc->n_ovf, &dc->touches};
  const uint16_t* cfw = Fw.compat.as<uint16_t>();
  const uint16_t* crv = Rv.compat.as<uint16_t>();
  if (launch) CK(cudaMemsetAsync(x->ctr.p, 0, sizeof(Counters), x->stream));
  // the prefix queue order (read_order 1), inside the captured work like the rest
  const uint32_t* ord = nullptr;
  if (x->read_order == 1 && x->threads_per_read == 1 && nq > 1) RET(prefix_order(x, c.d_q, c.d_qoff, nq, ord, dummy, launch));
  // search: long reads cut into segments, every read through the segment queue
  if (seg) {
    if (launch) {
      k_long_flags<<<(nq + 255) / 256, 256, 0, x->stream>>>(ord, nq, c.d_qoff, 2 * x->seg_len, x->lflag.as<uint32_t>());
      CK(cudaGetLastError());
    }
    RET(SCAN(x->lflag.as<uint32_t>(), 1, nq, x->lpos.as<uint64_t>()));
    if (launch) {
      CK(cudaMemsetAsync(x->ucount.p, 0, (size_t)nq * 4, x->stream));
      k_split_ids<<<(nq + 255) / 256, 256, 0, x->stream>>>(ord, nq, x->lflag.as<uint32_t>(), x->lpos.as<uint64_t>(),
                                                           x->sids.as<uint32_t>(), x->lids.as<uint32_t>(),
                                                           x->ucount.as<uint32_t>(), c.d_qoff, x->seg_len);
      CK(cudaGetLastError());
    }
    RET(SCAN(x->ucount.as<uint32_t>(), 1, nq, x->ubase.as<uint64_t>()));   // ubase[nq] = segments
    const uint64_t* n_long_dev = x->lpos.as<uint64_t>() + nq;
    const uint64_t* n_units_dev = x->ubase.as<uint64_t>() + nq;
    if (launch) {
      k_unit_fill<<<(nq + 255) / 256, 256, 0, x->stream>>>(x->lids.as<uint32_t>(), nq, x->ubase.as<uint64_t>(),
                                                           x->uread.as<uint32_t>(), x->uk.as<uint32_t>(), n_long_dev);
      CK(cudaGetLastError());
      SegWork G{x->seg_len, x->seg_len / 32, x->uread.as<uint32_t>(), x->uk.as<uint32_t>(), 0u, x->ubits.as<uint32_t>(),
                x->uexit.as<uint32_t>(), x->ust.as<uint32_t>(), x->ucoff.as<uint64_t>(), x->ucnt.as<uint32_t>(),
                x->segpool.as<Cand>(), &dc->seg_used, x->seg_cap, x->sids.as<uint32_t>(), 0u, x->lids.as<uint32_t>(),
                x->ubase.as<uint64_t>(), 0u, &dc->merge_queue, &dc->touches, x->fxe.as<uint32_t>(),
                x->fxc.as<uint32_t>(), x->fxx.as<uint32_t>(), x->fxo.as<uint64_t>(), x->fxn.as<uint32_t>(),
                n_units_dev, n_long_dev, nq};
      MemsWork W{x->memwork.as<BIv>(), MEM_SET_CAP, x->cwork.as<Cand>(), FAST_CAND_CAP, &dc->seg_queue, nullptr,
                 0u, &dc->still_ovf, 0u, nullptr, nullptr};
      W.chunk = x->queue_chunk;
      MemsWork Wf = W;
      Wf.queue = &dc->fix_queue;
      const unsigned g = (unsigned)(threads / 128);
      WITH_FMT(fmt, {
        k_mems_seg<false, 32, 8, FM><<<g, 128, 0, x->stream>>>(Fw.d, Rv.d, cfw, crv, c.d_q, c.d_qoff, P, ivp, hp, o, W, G);
        k_mems_fix<false, 32, 8, FM><<<g, 128, 0, x->stream>>>(Fw.d, Rv.d, cfw, crv, c.d_q, c.d_qoff, P, ivp, Wf, G);
        k_mems_merge<false, 32, 8, FM><<<g, 128, 0, x->stream>>>(Fw.d, Rv.d, cfw, crv, c.d_q, c.d_qoff, P, ivp, hp, o, W,
                                                                 G);
      });
      CK(cudaGetLastError());
    }
  } else if (launch) {
    MemsWork W{x->memwork.as<BIv>(), MEM_SET_CAP, x->cwork.as<Cand>(), FAST_CAND_CAP, &dc->queue, ord, nq,
               &dc->still_ovf, 0u, nullptr, nullptr};
    W.chunk = x->queue_chunk;
    WITH_FMT(fmt, {
      k_mems<false, 32, 0, 8, FM><<<(unsigned)(threads / 128), 128, 0, x->stream>>>(Fw.d, Rv.d, cfw, crv, c.d_q,
                                                                                    c.d_qoff, P, ivp, hp, o, W);
    });
    CK(cudaGetLastError());
  }
  // overflow tiers, over the device lists: a per-thread rerun with a 1024-entry candidate
  // list, then one warp per read with sets of MEM_WARP_SET_CAP intervals
  if (launch) {
    k_split_ovf<<<(nq + 255) / 256, 256, 0, x->stream>>>(x->ovf.as<uint32_t>(), nq, 0u, x->status.as<uint32_t>(),
                                                         x->ovf3.as<uint32_t>(), &dc->n_mid, x->ovf2.as<uint32_t>(),
                                                         &dc->n_wrp, &dc->n_ovf);
    CK(cudaGetLastError());
    const uint64_t tm = std::max<uint64_t>(128, std::min<uint64_t>((uint64_t)x->num_sms * MID_THREADS_PER_SM, threads));
    MemsWork Wm{x->memwork.as<BIv>(), MEM_SET_CAP, x->cwork.as<Cand>(), MID_CAND_CAP, &dc->queue3, x->ovf3.as<uint32_t>(),
                0u, &dc->still_ovf, 0u, nullptr, &dc->n_mid};
    MemsOut o2 = o;
    o2.ovf_list = x->ovf2.as<uint32_t>();
    o2.n_ovf = &dc->n_wrp;
    WITH_FMT(fmt, {
      k_mems<false, 32, 0, 8, FM><<<(unsigned)(tm / 128), 128, 0, x->stream>>>(Fw.d, Rv.d, cfw, crv, c.d_q, c.d_qoff, P,
                                                                                ivp, hp, o2, Wm);
    });
    MemsWork Ww{x->work.as<BIv>(), c.warp_cap, x->cwork.as<Cand>(), c.warp_cands, &dc->queue2, x->ovf2.as<uint32_t>(), 0u,
                &dc->still_ovf, 1u, nullptr, &dc->n_wrp};
    k_mems_warp<false><<<wgrid, 128, 0, x->stream>>>(Fw.d, Rv.d, cfw, crv, c.d_q, c.d_qoff, P, ivp, hp, o, Ww);
    CK(cudaGetLastError());
  }
  // CSR of MemHits (hits past the count stay zero, so their position counts add nothing)
  RET(SCAN(x->hit_count.as<uint32_t>(), 1, nq, x->hit_base.as<uint64_t>()));
  if (launch) {
    CK(cudaMemsetAsync(x->hits.p, 0, (hcap + 1) * 32, x->stream));
    k_gather_hits<<<(nq + 255) / 256, 256, 0, x->stream>>>(x->hitpool.as<uint4>(), x->hit_start.as<uint64_t>(),
                                                          x->hit_count.as<uint32_t>(), x->hit_base.as<uint64_t>(), nq,
                                                          x->hits.as<uint4>());
    CK(cudaGetLastError());
  }
  RET(SCAN(x->hits.as<uint32_t>() + 5, 8, hcap, x->npos_scan.as<uint64_t>()));
  if (launch) {
    k_set_pos_off<<<(unsigned)((hcap + 255) / 256), 256, 0, x->stream>>>(x->hits.as<uint32_t>(), x->npos_scan.as<uint64_t>(),
                                                                        hcap);
    CK(cudaGetLastError());
  }
  const uint32_t* seg_row = x->hits.as<uint32_t>() + 4;
  const uint64_t* seg_off = x->npos_scan.as<uint64_t>();
  const uint32_t* d_bounds = x->ref_bounds.as<uint32_t>();
  const uint32_t guard = Fw.rate ? Fw.rate : Fw.text_len;
  if (c.dedup) {
    if (launch) {
      CK(cudaMemsetAsync(x->hkeys.p, 0xFF, hsize * 8, x->stream));
      k_dedup_insert<<<(unsigned)((hcap + 255) / 256), 256, 0, x->stream>>>(seg_row, 8, seg_off, (uint32_t)hcap,
                                                                           x->hkeys.as<unsigned long long>(), hsize - 1,
                                                                           x->hslot.as<uint32_t>());
      k_dedup_flags<<<(unsigned)((hsize + 255) / 256), 256, 0, x->stream>>>(x->hkeys.as<unsigned long long>(), hsize,
                                                                           x->hflags.as<uint32_t>());
      CK(cudaGetLastError());
    }
    RET(SCAN(x->hflags.as<uint32_t>(), 1, hsize, x->huid.as<uint64_t>()));
    if (launch) {
      CK(cudaMemsetAsync(x->ulen.p, 0, hcap * 4 + 4, x->stream));
      k_dedup_compact<<<(unsigned)((hsize + 255) / 256), 256, 0, x->stream>>>(x->hkeys.as<unsigned long long>(), hsize,
                                                                             x->huid.as<uint64_t>(), x->urow.as<uint32_t>(),
                                                                             x->ulen.as<uint32_t>());
      CK(cudaGetLastError());
    }
    RET(SCAN(x->ulen.as<uint32_t>(), 1, hcap, x->uoff.as<uint64_t>()));     // uoff[hcap] = distinct positions
    if (launch) {
      k_graph_totals<<<1, 32, 0, x->stream>>>(x->hit_base.as<uint64_t>(), nq, seg_off + hcap,
                                              x->uoff.as<uint64_t>() + hcap, pcap, upcap, c.d_tot);
      k_block_first<<<(unsigned)((hcap + 255) / 256), 256, 0, x->stream>>>(x->uoff.as<uint64_t>(), (uint32_t)hcap, RES_T,
                                                                          x->blockmap.as<uint32_t>(),
                                                                          (upcap + RES_T - 1) / RES_T);
      ResolveArgs A{x->urow.as<uint32_t>(), 1, x->uoff.as<uint64_t>(), (uint32_t)hcap, upcap, d_bounds, c.nb, guard,
                    x->uout.as<uint32_t>(), &dc->walk_err, &dc->steps, x->blockmap.as<uint32_t>(), &c.d_tot->upos};
      k_resolve<false><<<(unsigned)((upcap + RES_T - 1) / RES_T), RES_T, 0, x->stream>>>(Fw.d, A);
      k_block_first<<<(unsigned)((hcap + 255) / 256), 256, 0, x->stream>>>(seg_off, (uint32_t)hcap, EXP_BLK,
                                                                          x->blockmap2.as<uint32_t>(), eblocks);
      k_dedup_expand<<<(unsigned)((pcap + EXP_BLK - 1) / EXP_BLK), EXP_T, 0, x->stream>>>(
          seg_off, (uint32_t)hcap, pcap, x->hslot.as<uint32_t>(), x->huid.as<uint64_t>(), x->uoff.as<uint64_t>(),
          x->uout.as<uint2>(), reinterpret_cast<uint2*>(x->out_pairs.p), x->blockmap2.as<uint32_t>(), &c.d_tot->npos);
      CK(cudaGetLastError());
    }
  } else if (launch) {
    k_graph_totals<<<1, 32, 0, x->stream>>>(x->hit_base.as<uint64_t>(), nq, seg_off + hcap, nullptr, pcap, pcap,
                                            c.d_tot);
    k_block_first<<<(unsigned)((hcap + 255) / 256), 256, 0, x->stream>>>(seg_off, (uint32_t)hcap, RES_T,
                                                                        x->blockmap.as<uint32_t>(), rblocks);
    ResolveArgs A{seg_row, 8, seg_off, (uint32_t)hcap, pcap, d_bounds, c.nb, guard, x->out_pairs.as<uint32_t>(),
                  &dc->walk_err, &dc->steps, x->blockmap.as<uint32_t>(), &c.d_tot->npos};
    k_resolve<false><<<(unsigned)((pcap + RES_T - 1) / RES_T), RES_T, 0, x->stream>>>(Fw.d, A);
    CK(cudaGetLastError());
  }
  if (launch) {
    CK(cudaMemcpyAsync(c.h_tot, c.d_tot, sizeof(GraphTotals), cudaMemcpyDeviceToHost, x->stream));
    CK(cudaMemcpyAsync(x->h_ctr, x->ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, x->stream));
  }
  return HFM_OK;
}

// The locate chain (backward search, CSR of merged intervals, resolve) with fixed
// capacities, the same way: `iv_cap` merged intervals over the batch, `pos_cap` positions,
// its own counters block and result array so that it can precede the SMEM chain in one
// captured graph.
struct FixedLocate {
  const uint8_t* d_q; const uint64_t* d_qoff; uint32_t nq; uint32_t max_hits;
  uint64_t iv_cap, pos_cap, upos_cap;
  uint32_t warp_cap = BS_WARP_SET_CAP;
  bool dedup;
  uint64_t threads;
  Counters* ctr;                // device counters of this chain
  GraphTotals* d_tot; GraphTotals* h_tot;
  Counters* h_ctr;              // pinned copy of ctr after the chain
};

static int fixed_locate(hfm_index* x, FixedLocate& c, bool launch) {
  const FmDev& F = x->fwd;
  const uint32_t nq = c.nq;
  uint32_t dummy = 0;
  auto SCAN = [&](auto* in, uint32_t stride, uint64_t n, uint64_t* out) -> int {
    if (!launch) {
      uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
      return x->scan_tmp.ensure((tiles + 1) * 8);
    }
    return scan(x, in, stride, n, out, dummy);
  };
  const uint64_t icap = c.iv_cap, pcap = c.pos_cap, upcap = std::min(c.upos_cap, c.pos_cap);
  if (icap >= 0xFFFFFFFFull) return set_error(HFM_E_ARG, "interval capacity above 2^32");
  RET(x->counts.ensure((size_t)nq * 4 + 4)); RET(x->nhits.ensure((size_t)nq * 8 + 8));
  RET(x->niv.ensure((size_t)nq * 4 + 4)); RET(x->ivoff.ensure((size_t)nq * 8 + 8));
  RET(x->status.ensure((size_t)nq * 4 + 4)); RET(x->ovf.ensure((size_t)nq * 4 + 4));
  RET(x->ivpool.ensure(icap * 8));
  if (!launch) {
    int bpsm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k_bsearch<false, 32>, 256, 0));
    c.threads = std::min<uint64_t>((uint64_t)std::max(1, bpsm) * x->num_sms * 256, ((uint64_t)nq + 255) / 256 * 256);
  }
  RET(x->bswork.ensure(std::max<uint64_t>(c.threads, 32) * 2 * BS_SET_CAP * 8));
  const uint64_t per_warp = (uint64_t)c.warp_cap * 2 * 8;
  const uint64_t wwarps = std::max<uint64_t>(4, std::min<uint64_t>((uint64_t)x->num_sms * 8, (2ull << 30) / per_warp));
  const uint32_t wgrid = (uint32_t)((wwarps + 3) / 4);
  RET(x->work.ensure((size_t)wgrid * 4 * per_warp));
  RET(x->seg_base.ensure(((size_t)nq + 1) * 8)); RET(x->pos_base.ensure(((size_t)nq + 1) * 8));
  RET(x->seg_row.ensure(icap * 4 + 4)); RET(x->seg_off.ensure((icap + 1) * 8));
  RET(x->loc_pairs.ensure(pcap * 8 + 8));
  const uint64_t rblocks = (pcap + RES_T - 1) / RES_T, eblocks = (pcap + EXP_BLK - 1) / EXP_BLK;
  RET(x->blockmap.ensure(rblocks * 4 + 4));
  uint64_t hsize = 1024;
  while (hsize < 2 * icap) hsize <<= 1;
  if (c.dedup) {
    RET(x->hkeys.ensure(hsize * 8)); RET(x->hslot.ensure(icap * 4 + 4));
    RET(x->hflags.ensure(hsize * 4)); RET(x->huid.ensure((hsize + 1) * 8));
    RET(x->urow.ensure(icap * 4 + 4)); RET(x->ulen.ensure(icap * 4 + 4)); RET(x->uoff.ensure((icap + 1) * 8));
    RET(x->uout.ensure(upcap * 8 + 8));
    RET(x->blockmap2.ensure(eblocks * 4 + 4));
  }
  Counters* dc = c.ctr;
  Pool pool{x->ivpool.p, &dc->iv_used, icap};
  BsOut o{x->counts.as<uint32_t>(), x->nhits.as<uint64_t>(), x->niv.as<uint32_t>(), x->ivoff.as<uint64_t>(),
          x->status.as<uint32_t>(), x->ovf.as<uint32_t>(), &dc->n_ovf, &dc->touches};
  const uint16_t* cm = F.compat.as<uint16_t>();
  if (launch) {
    CK(cudaMemsetAsync(dc, 0, sizeof(Counters), x->stream));
    k_bsearch<false, 32><<<(unsigned)(c.threads / 256), 256, 0, x->stream>>>(F.d, cm, c.d_q, c.d_qoff, nullptr, nq,
                                                                            c.max_hits, x->bswork.as<uint2>(), BS_SET_CAP,
                                                                            &dc->queue, pool, o, &dc->still_ovf);
    k_bsearch_warp<false><<<wgrid, 128, 0, x->stream>>>(F.d, cm, c.d_q, c.d_qoff, x->ovf.as<uint32_t>(), 0u, c.max_hits,
                                                       x->work.as<uint2>(), c.warp_cap, &dc->queue2, pool, o,
                                                       &dc->still_ovf, &dc->n_ovf);
    k_zero_failed<<<(nq + 255) / 256, 256, 0, x->stream>>>(x->status.as<uint32_t>(), nq, x->niv.as<uint32_t>(),
                                                           x->nhits.as<uint64_t>());
    CK(cudaGetLastError());
  }
  RET(SCAN(x->niv.as<uint32_t>(), 1, nq, x->seg_base.as<uint64_t>()));      // seg_base[nq] = intervals
  RET(SCAN(x->nhits.as<uint64_t>(), 1, nq, x->pos_base.as<uint64_t>()));    // pos_base[nq] = positions
  const uint64_t* seg_off = x->seg_off.as<uint64_t>();
  const uint32_t* seg_row = x->seg_row.as<uint32_t>();
  const uint32_t guard = F.rate ? F.rate : F.text_len;
  const uint32_t nb = (uint32_t)F.seq_boundaries.size();
  const uint32_t* d_bounds = F.bounds.as<uint32_t>();
  if (launch) {
    k_gather_locate<<<(nq + 255) / 256, 256, 0, x->stream>>>(x->ivpool.as<uint2>(), x->ivoff.as<uint64_t>(),
                                                            x->niv.as<uint32_t>(), x->seg_base.as<uint64_t>(),
                                                            x->pos_base.as<uint64_t>(), nq, c.max_hits,
                                                            x->seg_row.as<uint32_t>(), x->seg_off.as<uint64_t>());
    k_seal_segments<<<(unsigned)std::min<uint64_t>((icap + 256) / 256, 65535), 256, 0, x->stream>>>(
        x->seg_off.as<uint64_t>(), x->seg_base.as<uint64_t>() + nq, x->pos_base.as<uint64_t>() + nq, icap);
    CK(cudaGetLastError());
  }
  if (c.dedup) {
    if (launch) {
      CK(cudaMemsetAsync(x->hkeys.p, 0xFF, hsize * 8, x->stream));
      k_dedup_insert<<<(unsigned)((icap + 255) / 256), 256, 0, x->stream>>>(seg_row, 1, seg_off, (uint32_t)icap,
                                                                           x->hkeys.as<unsigned long long>(), hsize - 1,
                                                                           x->hslot.as<uint32_t>());
      k_dedup_flags<<<(unsigned)((hsize + 255) / 256), 256, 0, x->stream>>>(x->hkeys.as<unsigned long long>(), hsize,
                                                                           x->hflags.as<uint32_t>());
      CK(cudaGetLastError());
    }
    RET(SCAN(x->hflags.as<uint32_t>(), 1, hsize, x->huid.as<uint64_t>()));
    if (launch) {
      CK(cudaMemsetAsync(x->ulen.p, 0, icap * 4 + 4, x->stream));
      k_dedup_compact<<<(unsigned)((hsize + 255) / 256), 256, 0, x->stream>>>(x->hkeys.as<unsigned long long>(), hsize,
                                                                             x->huid.as<uint64_t>(), x->urow.as<uint32_t>(),
                                                                             x->ulen.as<uint32_t>());
      CK(cudaGetLastError());
    }
    RET(SCAN(x->ulen.as<uint32_t>(), 1, icap, x->uoff.as<uint64_t>()));
    if (launch) {
      k_graph_totals<<<1, 32, 0, x->stream>>>(x->seg_base.as<uint64_t>(), nq, x->pos_base.as<uint64_t>() + nq,
                                              x->uoff.as<uint64_t>() + icap, pcap, upcap, c.d_tot);
      k_block_first<<<(unsigned)((icap + 255) / 256), 256, 0, x->stream>>>(x->uoff.as<uint64_t>(), (uint32_t)icap, RES_T,
                                                                          x->blockmap.as<uint32_t>(),
                                                                          (upcap + RES_T - 1) / RES_T);
      ResolveArgs A{x->urow.as<uint32_t>(), 1, x->uoff.as<uint64_t>(), (uint32_t)icap, upcap, d_bounds, nb, guard,
                    x->uout.as<uint32_t>(), &dc->walk_err, &dc->steps, x->blockmap.as<uint32_t>(), &c.d_tot->upos};
      k_resolve<false><<<(unsigned)((upcap + RES_T - 1) / RES_T), RES_T, 0, x->stream>>>(F.d, A);
      k_block_first<<<(unsigned)((icap + 255) / 256), 256, 0, x->stream>>>(seg_off, (uint32_t)icap, EXP_BLK,
                                                                          x->blockmap2.as<uint32_t>(), eblocks);
      k_dedup_expand<<<(unsigned)((pcap + EXP_BLK - 1) / EXP_BLK), EXP_T, 0, x->stream>>>(
          seg_off, (uint32_t)icap, pcap, x->hslot.as<uint32_t>(), x->huid.as<uint64_t>(), x->uoff.as<uint64_t>(),
          x->uout.as<uint2>(), reinterpret_cast<uint2*>(x->loc_pairs.p), x->blockmap2.as<uint32_t>(), &c.d_tot->npos);
      CK(cudaGetLastError());
    }
  } else if (launch) {
    k_graph_totals<<<1, 32, 0, x->stream>>>(x->seg_base.as<uint64_t>(), nq, x->pos_base.as<uint64_t>() + nq, nullptr,
                                            pcap, pcap, c.d_tot);
    k_block_first<<<(unsigned)((icap + 255) / 256), 256, 0, x->stream>>>(seg_off, (uint32_t)icap, RES_T,
                                                                        x->blockmap.as<uint32_t>(), rblocks);
    ResolveArgs A{seg_row, 1, seg_off, (uint32_t)icap, pcap, d_bounds, nb, guard, x->loc_pairs.as<uint32_t>(),
                  &dc->walk_err, &dc->steps, x->blockmap.as<uint32_t>(), &c.d_tot->npos};
    k_resolve<false><<<(unsigned)((pcap + RES_T - 1) / RES_T), RES_T, 0, x->stream>>>(F.d, A);
    CK(cudaGetLastError());
  }
  if (launch) {
    CK(cudaMemcpyAsync(c.h_tot, c.d_tot, sizeof(GraphTotals), cudaMemcpyDeviceToHost, x->stream));
    CK(cudaMemcpyAsync(c.h_ctr, dc, sizeof(Counters), cudaMemcpyDeviceToHost, x->stream));
  }
  return HFM_OK;
}

// H2D of a host query batch into the handle's buffers.
static int stage_queries(hfm_index* x, const uint8_t* q, const uint64_t* q_off, uint32_t nq) {
  if (nq && (!q_off)) return set_error(HFM_E_ARG, "q_off is NULL");
  uint64_t bytes = nq ? q_off[nq] : 0;
  for (uint32_t i = 0; i < nq; i++) if (q_off[i + 1] < q_off[i]) return set_error(HFM_E_ARG, "q_off not ascending");
  if (bytes && !q) return set_error(HFM_E_ARG, "q is NULL");
  RET(x->q.ensure(bytes + 16));
  RET(x->qoff.ensure(((size_t)nq + 1) * 8));
  if (bytes) CK(cudaMemcpyAsync(x->q.p, q, bytes, cudaMemcpyHostToDevice, x->stream));
  if (nq) CK(cudaMemcpyAsync(x->qoff.p, q_off, ((size_t)nq + 1) * 8, cudaMemcpyHostToDevice, x->stream));
  return HFM_OK;
}

// Result blocks of the host-buffer entry points come from a process-wide cache of
// pinned host memory: the device-to-host copy of a result runs at link speed and a
// block released by hfm_free is reused by the next call instead of being re-pinned.
struct PinnedCache {
  std::mutex mu;
  std::multimap<size_t, void*> free_blocks;
  std::unordered_map<void*, size_t> owned;
  size_t cached_bytes = 0;
};
static PinnedCache& pinned_cache() { static PinnedCache* c = new PinnedCache(); return *c; }
static constexpr size_t PINNED_CACHE_MAX = 48ull << 30;

static void* host_result_alloc(size_t bytes) {
  PinnedCache& P = pinned_cache();
  std::lock_guard<std::mutex> lk(P.mu);
  auto it = P.free_blocks.lower_bound(bytes);
  if (it != P.free_blocks.end() && it->first <= 2 * bytes + (64ull << 20)) {
    void* p = it->second;
    P.cached_bytes -= it->first;
    P.free_blocks.erase(it);
    return p;
  }
  size_t sz = (bytes + (2ull << 20) - 1) & ~((2ull << 20) - 1);
  void* p = nullptr;
  if (cudaHostAlloc(&p, sz, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return std::malloc(bytes);          // pageable fallback, released by std::free
  }
  P.owned[p] = sz;
  return p;
}

static void host_result_free(void* p) {
  PinnedCache& P = pinned_cache();
  std::lock_guard<std::mutex> lk(P.mu);
  auto it = P.owned.find(p);
  if (it == P.owned.end()) { std::free(p); return; }
  if (P.cached_bytes + it->second > PINNED_CACHE_MAX) { cudaFreeHost(p); P.owned.erase(it); return; }
  P.free_blocks.insert({it->second, p});
  P.cached_bytes += it->second;
}

struct Guard {
  hfm_index* x;
  std::unique_lock<std::mutex> lk;
  explicit Guard(hfm_index* i) : x(i), lk(i->mu) {
    cudaSetDevice(i->device);
    if (!i->orphans.empty()) {           // a timed-out call left copies in flight: let them land
      cudaStreamSynchronize(i->stream);
      for (void* p : i->orphans) host_result_free(p);
      i->orphans.clear();
    }
  }
};

// A handle on the same device-resident index with its own stream and work buffers (the
// index's buffers are not copied and stay owned by `x`).
static int make_shadow(hfm_index* x, hfm_index** out) {
  std::unique_ptr<hfm_index> sh(new hfm_index());
  sh->device = x->device; sh->kind = x->kind; sh->flags = x->flags; sh->num_sms = x->num_sms;
  sh->seg_len = x->seg_len; sh->mems_variant = x->mems_variant; sh->count_work = x->count_work;
  sh->queue_chunk = x->queue_chunk; sh->threads_per_read = x->threads_per_read; sh->read_order = x->read_order;
  sh->timeout_ms = x->timeout_ms;
  sh->shared_index = true;
  for (int k = 0; k < 2; k++) {
    const FmDev& src = k ? x->rev : x->fwd;
    FmDev& dst = k ? sh->rev : sh->fwd;
    dst.d = src.d; dst.occ = src.occ; dst.sb = src.sb; dst.ssa = src.ssa; dst.sa_vals = src.sa_vals; dst.lut = src.lut;
    dst.bounds = src.bounds; dst.compat = src.compat; dst.text_len = src.text_len; dst.num_seqs = src.num_seqs;
    dst.lookup_depth = src.lookup_depth; dst.tag = src.tag; dst.num_lanes = src.num_lanes; dst.encoding = src.encoding;
    dst.rate = src.rate; dst.fmt = src.fmt; dst.seq_boundaries = src.seq_boundaries;
    std::memcpy(dst.nbytes, src.nbytes, sizeof(dst.nbytes));
  }
  CK(cudaSetDevice(x->device));
  CK(cudaStreamCreateWithFlags(&sh->stream, cudaStreamNonBlocking));
  for (auto& e : sh->ev) CK(cudaEventCreate(&e));
  for (auto& e : sh->evk) CK(cudaEventCreate(&e));
  CK(cudaEventCreateWithFlags(&sh->ev_wait, cudaEventDisableTiming));
  CK(cudaMallocHost((void**)&sh->h_ctr, sizeof(Counters)));
  RET(sh->ctr.ensure(sizeof(Counters)));
  *out = sh.release();
  return HFM_OK;
}

}  // namespace hfm

// ===========================================================================
// extern "C"
// ===========================================================================
extern "C" {

const char* hfm_last_error(void) { return hfm::g_err.c_str(); }

void hfm_free(void* p) {
  if (p) host_result_free(p);
}

int hfm_index_load(const uint8_t* bytes, size_t len, int kind, const hfm_opts* opts, hfm_index** out) {
  if (!bytes || !out) return set_error(HFM_E_ARG, "NULL argument");
  if (kind != HFM_KIND_FM && kind != HFM_KIND_BIDIR) return set_error(HFM_E_ARG, "kind must be 0 or 1");
  *out = nullptr;
  HostFm hf, hr;
  if (kind == HFM_KIND_FM) RET(parse_fm(bytes, len, hf));
  else {
    // BidirFmIndex::from_bytes (src/fm_index/bidir_index.rs:195-210)
    if (len < 4) return set_error(HFM_E_FORMAT, "truncated bidirectional index");
    uint32_t fl; std::memcpy(&fl, bytes, 4);
    if (len < 4ull + fl) return set_error(HFM_E_FORMAT, "truncated forward index");
    RET(parse_fm(bytes + 4, fl, hf));
    RET(parse_fm(bytes + 4 + fl, len - 4 - fl, hr));
    if (hr.text_len != hf.text_len) return set_error(HFM_E_FORMAT, "forward and reverse text lengths differ");
  }
  int dev = opts ? opts->device : 0;
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (dev < 0 || dev >= ndev) return set_error(HFM_E_ARG, "device ordinal out of range");
  CK(cudaSetDevice(dev));
  std::unique_ptr<hfm_index> x(new hfm_index());
  x->device = dev; x->kind = kind; x->flags = opts ? opts->flags : 0;
  CK(cudaDeviceGetAttribute(&x->num_sms, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking));
  for (auto& e : x->ev) CK(cudaEventCreate(&e));
  for (auto& e : x->evk) CK(cudaEventCreate(&e));
  CK(cudaEventCreateWithFlags(&x->ev_wait, cudaEventDisableTiming));
  CK(cudaMallocHost((void**)&x->h_ctr, sizeof(Counters)));
  RET(x->ctr.ensure(sizeof(Counters)));
  RET(build_device_fm(hf, x->fwd, x->stream));
  if (kind == HFM_KIND_BIDIR) RET(build_device_fm(hr, x->rev, x->stream));
  *out = x.release();
  return HFM_OK;
}

// ---------------------------------------------------------------------------
// Device-layout blob: the handle's device records (after the transform from the bincode
// records that hfm_index_load makes on the host), so that a later load is a read and an
// upload.  No counterpart in the reference.  Layout, all little-endian:
//   "HFMD" | u32 version 1 | u32 kind | u32 directions
//   per direction: DevFm (pointers zero) | 8 x u32 FmDev scalars | u32 nbounds | nbounds x u32
//                  | 7 x u64 buffer bytes | the 7 buffers' bytes
// ---------------------------------------------------------------------------
static constexpr uint32_t LAYOUT_VERSION = 1;

int hfm_index_export_layout(hfm_index* x, uint8_t** bytes_out, uint64_t* len_out) {
  if (!x || !bytes_out || !len_out) return set_error(HFM_E_ARG, "NULL argument");
  *bytes_out = nullptr; *len_out = 0;
  Guard g(x);
  const int nd = x->kind == HFM_KIND_BIDIR ? 2 : 1;
  const FmDev* dirs[2] = {&x->fwd, &x->rev};
  uint64_t total = 16;
  for (int k = 0; k < nd; k++) {
    total += sizeof(DevFm) + 8 * 4 + 4 + dirs[k]->seq_boundaries.size() * 4 + 7 * 8;
    for (size_t b : dirs[k]->nbytes) total += b;
  }
  uint8_t* out = (uint8_t*)std::malloc(total);
  if (!out) return set_error(HFM_E_OOM, "host allocation failed");
  uint8_t* w = out;
  auto put = [&](const void* src, size_t n) { std::memcpy(w, src, n); w += n; };
  const uint32_t hdr[4] = {0x444D4648u, LAYOUT_VERSION, (uint32_t)x->kind, (uint32_t)nd};
  put(hdr, 16);
  for (int k = 0; k < nd; k++) {
    const FmDev& f = *dirs[k];
    DevFm d = f.d;
    d.occ = nullptr; d.sb = nullptr; d.ssa = nullptr; d.sa_vals = nullptr; d.lut = nullptr; d.seq_bounds = nullptr;
    put(&d, sizeof(d));
    const uint32_t sc[8] = {f.text_len, f.num_seqs, f.lookup_depth, f.tag, f.num_lanes, f.encoding, f.rate, f.fmt};
    put(sc, 32);
    const uint32_t nbnd = (uint32_t)f.seq_boundaries.size();
    put(&nbnd, 4);
    put(f.seq_boundaries.data(), (size_t)nbnd * 4);
    put(f.nbytes, 7 * 8);
    const DevBuf* bufs[7] = {&f.occ, &f.sb, &f.ssa, &f.sa_vals, &f.lut, &f.bounds, &f.compat};
    for (int b = 0; b < 7; b++) {
      if (f.nbytes[b]) {
        cudaError_t e = cudaMemcpy(w, bufs[b]->p, f.nbytes[b], cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { std::free(out); cudaGetLastError(); return set_error(HFM_E_CUDA, "layout copy failed"); }
      }
      w += f.nbytes[b];
    }
  }
  *bytes_out = out; *len_out = total;
  return HFM_OK;
}

int hfm_index_load_layout(const uint8_t* bytes, uint64_t len, const hfm_opts* opts, hfm_index** out) {
  if (!bytes || !out) return set_error(HFM_E_ARG, "NULL argument");
  *out = nullptr;
  // validate every length against the blob before any device work
  uint64_t r = 0;
  auto need = [&](uint64_t n) { return n <= len && r <= len - n; };
  if (!need(16)) return set_error(HFM_E_FORMAT, "truncated layout header");
  uint32_t hdr[4];
  std::memcpy(hdr, bytes, 16); r = 16;
  if (hdr[0] != 0x444D4648u) return set_error(HFM_E_FORMAT, "not a device-layout blob (magic)");
  if (hdr[1] != LAYOUT_VERSION) return set_error(HFM_E_FORMAT, "unsupported device-layout version");
  const int kind = (int)hdr[2];
  if ((kind != HFM_KIND_FM && kind != HFM_KIND_BIDIR) || hdr[3] != (kind == HFM_KIND_BIDIR ? 2u : 1u))
    return set_error(HFM_E_FORMAT, "bad kind or direction count");
  struct Dir { DevFm d; uint32_t sc[8]; std::vector<uint32_t> bnd; uint64_t nb[7]; uint64_t at[7]; };
  Dir dirs[2];
  for (uint32_t k = 0; k < hdr[3]; k++) {
    Dir& D = dirs[k];
    if (!need(sizeof(DevFm) + 36)) return set_error(HFM_E_FORMAT, "truncated direction header");
    std::memcpy(&D.d, bytes + r, sizeof(DevFm)); r += sizeof(DevFm);
    std::memcpy(D.sc, bytes + r, 32); r += 32;
    uint32_t nbnd; std::memcpy(&nbnd, bytes + r, 4); r += 4;
    if (!need((uint64_t)nbnd * 4 + 56)) return set_error(HFM_E_FORMAT, "truncated sequence bounds");
    D.bnd.resize(nbnd);
    std::memcpy(D.bnd.data(), bytes + r, (size_t)nbnd * 4); r += (uint64_t)nbnd * 4;
    std::memcpy(D.nb, bytes + r, 56); r += 56;
    const uint64_t nblk = ((uint64_t)D.d.text_len + 63) / 64;
    const uint64_t rec = D.d.fmt == OCC_NARROW ? OCC_NARROW_U4 * 16 : OCC_WIDE_U4 * 16;
    if (D.d.fmt > OCC_NARROW || D.nb[0] != nblk * rec || D.nb[2] != nblk * 16 || D.d.num_blocks != nblk ||
        D.nb[5] != (uint64_t)nbnd * 4 || D.nb[6] != 32 || D.sc[0] != D.d.text_len || D.sc[7] != D.d.fmt ||
        D.nb[1] != ((nblk + (1u << SB_BLOCK_SHIFT) - 1) >> SB_BLOCK_SHIFT) * 64 ||
        (D.nb[4] != 0) != (D.d.lut_depth != 0) || D.nb[3] % 4 || D.nb[4] % 8)
      return set_error(HFM_E_FORMAT, "device-layout sizes inconsistent with the text length");
    for (int b = 0; b < 7; b++) {
      if (!need(D.nb[b])) return set_error(HFM_E_FORMAT, "truncated device buffer");
      D.at[b] = r; r += D.nb[b];
    }
  }
  if (r != len) return set_error(HFM_E_FORMAT, "trailing bytes after the device layout");
  if (kind == HFM_KIND_BIDIR && dirs[0].d.text_len != dirs[1].d.text_len)
    return set_error(HFM_E_FORMAT, "forward and reverse text lengths differ");
  int dev = opts ? opts->device : 0;
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (dev < 0 || dev >= ndev) return set_error(HFM_E_ARG, "device ordinal out of range");
  CK(cudaSetDevice(dev));
  std::unique_ptr<hfm_index> x(new hfm_index());
  x->device = dev; x->kind = kind; x->flags = opts ? opts->flags : 0;
  CK(cudaDeviceGetAttribute(&x->num_sms, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking));
  for (auto& e : x->ev) CK(cudaEventCreate(&e));
  for (auto& e : x->evk) CK(cudaEventCreate(&e));
  CK(cudaEventCreateWithFlags(&x->ev_wait, cudaEventDisableTiming));
  CK(cudaMallocHost((void**)&x->h_ctr, sizeof(Counters)));
  RET(x->ctr.ensure(sizeof(Counters)));
  FmDev* fs[2] = {&x->fwd, &x->rev};
  for (uint32_t k = 0; k < hdr[3]; k++) {
    Dir& D = dirs[k];
    FmDev& f = *fs[k];
    DevBuf* bufs[7] = {&f.occ, &f.sb, &f.ssa, &f.sa_vals, &f.lut, &f.bounds, &f.compat};
    for (int b = 0; b < 7; b++) {
      if (!D.nb[b]) continue;
      RET(upload(*bufs[b], bytes + D.at[b], D.nb[b], x->stream));
      f.nbytes[b] = D.nb[b];
    }
    f.d = D.d;
    f.d.occ = f.occ.as<uint4>(); f.d.sb = f.sb.as<uint32_t>(); f.d.ssa = f.ssa.as<uint4>();
    f.d.sa_vals = f.sa_vals.as<uint32_t>(); f.d.seq_bounds = f.bounds.as<uint32_t>();
    f.d.lut = D.nb[4] ? f.lut.as<uint2>() : nullptr;
    f.text_len = D.sc[0]; f.num_seqs = D.sc[1]; f.lookup_depth = D.sc[2]; f.tag = D.sc[3];
    f.num_lanes = D.sc[4]; f.encoding = D.sc[5]; f.rate = D.sc[6]; f.fmt = D.sc[7];
    f.seq_boundaries = D.bnd;
  }
  CK(cudaStreamSynchronize(x->stream));
  *out = x.release();
  return HFM_OK;
}

int hfm_index_device_bytes(const hfm_index* x, uint64_t* index_bytes, uint64_t* work_bytes) {
  if (!x) return set_error(HFM_E_ARG, "NULL argument");
  const DevBuf* idx_bufs[] = {&x->fwd.occ, &x->fwd.sb, &x->fwd.ssa, &x->fwd.sa_vals, &x->fwd.lut, &x->fwd.bounds,
                              &x->fwd.compat, &x->rev.occ, &x->rev.sb, &x->rev.ssa, &x->rev.sa_vals, &x->rev.lut,
                              &x->rev.bounds, &x->rev.compat};
  const DevBuf* work_bufs[] = {
      &x->q, &x->qoff, &x->counts, &x->nhits, &x->niv, &x->ivoff, &x->status, &x->ovf, &x->ivpool, &x->hitpool,
      &x->seg_row, &x->seg_off, &x->pos_base, &x->seg_base, &x->scan_tmp, &x->out_pairs, &x->ref_bounds,
      &x->hit_start, &x->hit_count, &x->hit_base, &x->hits, &x->npos_scan, &x->work, &x->cwork, &x->ctr,
      &x->mivpool, &x->bswork, &x->memwork, &x->hkeys, &x->hslot, &x->hflags, &x->huid, &x->urow, &x->ulen,
      &x->uoff, &x->uout, &x->blockmap, &x->blockmap2, &x->ovf2, &x->ovf3, &x->lflag, &x->lpos, &x->sids,
      &x->lids, &x->ucount, &x->ubase, &x->uread, &x->uk, &x->ubits, &x->uexit, &x->ust, &x->ucoff, &x->ucnt,
      &x->segpool, &x->fxe, &x->fxc, &x->fxx, &x->fxo, &x->fxn, &x->npos, &x->iota, &x->loc_pairs,
      &x->okeys, &x->oids, &x->otemp};
  uint64_t a = 0, b = 0;
  if (!x->shared_index) for (const DevBuf* d : idx_bufs) a += d->cap;
  for (const DevBuf* d : work_bufs) b += d->cap;
  if (index_bytes) *index_bytes = a;
  if (work_bytes) *work_bytes = b;
  return HFM_OK;
}

void hfm_index_free(hfm_index* x) {
  if (!x) return;
  cudaSetDevice(x->device);
  if (x->stream) cudaStreamSynchronize(x->stream);
  for (void* p : x->orphans) host_result_free(p);
  if (x->shared_index)                // the index layout belongs to the handle this one shares
    for (FmDev* f : {&x->fwd, &x->rev})
      for (DevBuf* b : {&f->occ, &f->sb, &f->ssa, &f->sa_vals, &f->lut, &f->bounds, &f->compat}) { b->p = nullptr; b->cap = 0; }
  for (DevBuf* b : {&x->fwd.occ, &x->fwd.sb, &x->rev.sb, &x->fwd.ssa, &x->fwd.sa_vals, &x->fwd.lut, &x->fwd.bounds,
                    &x->fwd.compat, &x->rev.occ, &x->rev.ssa, &x->rev.sa_vals, &x->rev.lut,
                    &x->rev.bounds, &x->rev.compat, &x->q, &x->qoff, &x->counts, &x->nhits, &x->niv, &x->ivoff,
                    &x->status, &x->ovf, &x->ivpool, &x->hitpool, &x->seg_row, &x->seg_off, &x->pos_base,
                    &x->seg_base, &x->scan_tmp, &x->out_pairs, &x->ref_bounds, &x->hit_start, &x->hit_count,
                    &x->hit_base, &x->hits, &x->npos_scan, &x->work, &x->cwork, &x->ctr, &x->mivpool, &x->bswork, &x->memwork,
                    &x->hkeys, &x->hslot, &x->hflags, &x->huid, &x->urow, &x->ulen, &x->uoff, &x->uout,
                    &x->blockmap, &x->blockmap2, &x->ovf2, &x->ovf3, &x->lflag, &x->lpos, &x->sids, &x->lids,
                    &x->ucount, &x->ubase, &x->uread, &x->uk, &x->ubits, &x->uexit, &x->ust, &x->ucoff, &x->ucnt,
                    &x->segpool, &x->fxe, &x->fxc, &x->fxx, &x->fxo, &x->fxn, &x->npos, &x->iota, &x->loc_pairs,
                    &x->okeys, &x->oids, &x->otemp})
    b->release();
  for (auto& e : x->ev) if (e) cudaEventDestroy(e);
  for (auto& e : x->evk) if (e) cudaEventDestroy(e);
  if (x->ev_wait) cudaEventDestroy(x->ev_wait);
  if (x->h_ctr) cudaFreeHost(x->h_ctr);
  if (x->stream) cudaStreamDestroy(x->stream);
  delete x;
}

int hfm_index_info_get(const hfm_index* x, hfm_index_info* o) {
  if (!x || !o) return set_error(HFM_E_ARG, "NULL argument");
  o->kind = x->kind; o->text_len = x->fwd.text_len; o->num_sequences = x->fwd.num_seqs;
  o->sample_rate = x->fwd.rate; o->lookup_depth = x->fwd.lookup_depth; o->alphabet_tag = x->fwd.tag;
  o->num_lanes = x->fwd.num_lanes; o->encoding = x->fwd.encoding;
  o->device_bytes = x->fwd.bytes() + x->rev.bytes();
  return HFM_OK;
}

void* hfm_index_stream(hfm_index* x) { return x ? (void*)x->stream : nullptr; }

int hfm_last_stats(const hfm_index* x, hfm_stats* o) {
  if (!x || !o) return set_error(HFM_E_ARG, "NULL argument");
  *o = x->stats;
  return HFM_OK;
}

int hfm_get_tuning(const hfm_index* x, hfm_tuning* t) {
  if (!x || !t) return set_error(HFM_E_ARG, "NULL argument");
  t->mems_variant = (uint32_t)x->mems_variant;
  t->seg_len = x->seg_len;
  t->queue_chunk = x->queue_chunk;
  t->threads_per_read = x->threads_per_read;
  t->read_order = x->read_order;
  return HFM_OK;
}

int hfm_set_tuning(hfm_index* x, const hfm_tuning* t) {
  if (!x || !t) return set_error(HFM_E_ARG, "NULL argument");
  if (t->mems_variant < 2 || t->mems_variant > 4) return set_error(HFM_E_ARG, "mems_variant must be 2, 3 or 4");
  if (t->seg_len < 64 || t->seg_len > SEG_MAX || t->seg_len % 32) return set_error(HFM_E_ARG, "seg_len must be a multiple of 32 in 64..4096");
  if (t->queue_chunk < 1 || t->queue_chunk > 64) return set_error(HFM_E_ARG, "queue_chunk must be in 1..64");
  if (t->threads_per_read != 1 && t->threads_per_read != 4 && t->threads_per_read != 8 && t->threads_per_read != 16 &&
      t->threads_per_read != 32)
    return set_error(HFM_E_ARG, "threads_per_read must be 1, 4, 8, 16 or 32");
  if (t->read_order > 1) return set_error(HFM_E_ARG, "read_order must be 0 or 1");
  std::lock_guard<std::mutex> lk(x->mu);
  x->mems_variant = (int)t->mems_variant;
  x->seg_len = t->seg_len;
  x->queue_chunk = t->queue_chunk;
  x->threads_per_read = t->threads_per_read;
  x->read_order = t->read_order;
  return HFM_OK;
}

int hfm_autotune_mems(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq, uint32_t min_len,
                      uint32_t mode, const uint32_t* ref_bounds, uint32_t nb, uint32_t cap, uint32_t reps,
                      hfm_tuning* best, float* times_ms) {
  if (!x || !best || (nq && !d_qoff) || (nb && !ref_bounds)) return set_error(HFM_E_ARG, "NULL argument");
  if (x->kind != HFM_KIND_BIDIR) return set_error(HFM_E_ARG, "MEM/SMEM search needs a bidirectional index");
  reps = std::max(1u, reps);
  Guard g(x);
  // HFM_TUNE_CANDIDATES settings, in the order include/hfm.h lists them
  const hfm_tuning cands[HFM_TUNE_CANDIDATES] = {
      {3, 512, 1, 1, 0}, {3, 256, 1, 1, 0},  {3, 1024, 1, 1, 0}, {2, 512, 1, 1, 0},  {3, 512, 4, 1, 0}, {3, 512, 16, 1, 0},
      {3, 512, 1, 4, 0}, {3, 512, 1, 8, 0},  {3, 512, 1, 32, 0}, {3, 512, 1, 1, 1}, {3, 1024, 1, 1, 1}};
  const hfm_tuning saved{(uint32_t)x->mems_variant, x->seg_len, x->queue_chunk, x->threads_per_read, x->read_order};
  auto apply = [&](const hfm_tuning& t) {
    x->mems_variant = (int)t.mems_variant; x->seg_len = t.seg_len;
    x->queue_chunk = t.queue_chunk; x->threads_per_read = t.threads_per_read; x->read_order = t.read_order;
  };
  float best_ms = 0.f;
  int best_k = -1;
  for (int k = 0; k < HFM_TUNE_CANDIDATES; k++) {
    apply(cands[k]);
    float t = 0.f;
    for (uint32_t r = 0; r <= reps; r++) {       // first run warms the pools
      hfm_dev_mems out;
      int rc = mems_device(x, d_q, d_qoff, nq, min_len, mode, ref_bounds, nb, cap, &out);
      if (rc) { apply(saved); return rc; }
      if (r > 0) t = r == 1 ? x->stats.ms_total : std::min(t, x->stats.ms_total);
    }
    if (times_ms) times_ms[k] = t;
    if (best_k < 0 || t < best_ms) { best_ms = t; best_k = k; }
  }
  apply(cands[best_k]);
  *best = cands[best_k];
  return HFM_OK;
}

int hfm_mems_reserve(hfm_index* x, uint32_t nq, uint64_t intervals, uint64_t hits, uint64_t positions) {
  if (!x) return set_error(HFM_E_ARG, "NULL argument");
  Guard g(x);
  // the search pools (intervals of every candidate, MemHits) and the result arrays
  x->miv_cap = std::max<uint64_t>(x->miv_cap, intervals + 4096);
  x->hit_cap = std::max<uint64_t>(x->hit_cap, hits + 4096);
  RET(x->mivpool.ensure(x->miv_cap * 16)); x->miv_cap = x->mivpool.cap / 16;
  RET(x->hitpool.ensure(x->hit_cap * 32)); x->hit_cap = x->hitpool.cap / 32;
  RET(x->hits.ensure(hits * 32 + 32));
  RET(x->npos_scan.ensure((hits + 1) * 8));
  RET(x->out_pairs.ensure(positions * 8 + 8));
  RET(x->hit_start.ensure((size_t)nq * 8 + 8)); RET(x->hit_count.ensure((size_t)nq * 4 + 4));
  RET(x->hit_base.ensure(((size_t)nq + 1) * 8));
  RET(x->status.ensure((size_t)nq * 4 + 4)); RET(x->ovf.ensure((size_t)nq * 4 + 4));
  return HFM_OK;
}

int hfm_set_timeout(hfm_index* x, uint32_t ms) {
  if (!x) return set_error(HFM_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(x->mu);
  x->timeout_ms = ms;
  return HFM_OK;
}

int hfm_set_counters(hfm_index* x, int enable) {
  if (!x) return set_error(HFM_E_ARG, "NULL argument");
  x->count_work = enable != 0;
  return HFM_OK;
}

int hfm_count_batch_device(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq, uint32_t* d_counts) {
  if (!x || (nq && (!d_qoff || !d_counts))) return set_error(HFM_E_ARG, "NULL argument");
  Guard g(x);
  return count_device(x, d_q, d_qoff, nq, d_counts);
}

int hfm_locate_batch_device(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq, uint32_t cap,
                            hfm_dev_hits* out) {
  if (!x || !out || (nq && !d_qoff)) return set_error(HFM_E_ARG, "NULL argument");
  Guard g(x);
  return locate_device(x, d_q, d_qoff, nq, cap, out);
}

int hfm_mems_batch_device(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq, uint32_t min_len,
                          uint32_t mode, const uint32_t* ref_bounds, uint32_t nb, uint32_t cap, hfm_dev_mems* out) {
  if (!x || !out || (nq && !d_qoff) || (nb && !ref_bounds)) return set_error(HFM_E_ARG, "NULL argument");
  Guard g(x);
  return mems_device(x, d_q, d_qoff, nq, min_len, mode, ref_bounds, nb, cap, out);
}

int hfm_mems_batch_device_sched(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq,
                                uint32_t min_len, uint32_t mode, const uint32_t* ref_bounds, uint32_t nb, uint32_t cap,
                                const hfm_sched* sched, hfm_dev_mems* out) {
  if (!x || !out || (nq && !d_qoff) || (nb && !ref_bounds)) return set_error(HFM_E_ARG, "NULL argument");
  Guard g(x);
  return mems_device(x, d_q, d_qoff, nq, min_len, mode, ref_bounds, nb, cap, out, sched);
}

int hfm_count_batch(hfm_index* x, const uint8_t* q, const uint64_t* q_off, uint32_t nq, uint32_t* counts_out) {
  if (!x || (nq && !counts_out)) return set_error(HFM_E_ARG, "NULL argument");
  Guard g(x);
  RET(stage_queries(x, q, q_off, nq));
  RET(x->counts.ensure((size_t)nq * 4 + 4));
  RET(count_device(x, x->q.as<uint8_t>(), x->qoff.as<uint64_t>(), nq, x->counts.as<uint32_t>()));
  if (nq) CK(cudaMemcpyAsync(counts_out, x->counts.p, (size_t)nq * 4, cudaMemcpyDeviceToHost, x->stream));
  return wait_stream(x);
}

int hfm_locate_batch(hfm_index* x, const uint8_t* q, const uint64_t* q_off, uint32_t nq, uint32_t cap, hfm_hits** out) {
  if (!x || !out) return set_error(HFM_E_ARG, "NULL argument");
  *out = nullptr;
  Guard g(x);
  RET(stage_queries(x, q, q_off, nq));
  hfm_dev_hits d{};
  RET(locate_device(x, x->q.as<uint8_t>(), x->qoff.as<uint64_t>(), nq, cap, &d));
  // one malloc block: struct | offsets | counts | pairs
  size_t bytes = sizeof(hfm_hits) + ((size_t)nq + 1) * 8 + (size_t)nq * 4 + 4 + (size_t)d.total * 8;
  uint8_t* blk = (uint8_t*)host_result_alloc(bytes);
  if (!blk) return set_error(HFM_E_OOM, "host allocation failed");
  hfm_hits* h = (hfm_hits*)blk;
  h->nq = nq; h->_pad = 0; h->total = d.total;
  h->offsets = (uint64_t*)(blk + sizeof(hfm_hits));
  h->pairs = (uint32_t*)(h->offsets + nq + 1);
  h->counts = h->pairs + d.total * 2;
  CK(cudaMemcpyAsync(h->offsets, d.d_offsets, ((size_t)nq + 1) * 8, cudaMemcpyDeviceToHost, x->stream));
  if (d.total) CK(cudaMemcpyAsync(h->pairs, d.d_pairs, (size_t)d.total * 8, cudaMemcpyDeviceToHost, x->stream));
  if (nq) CK(cudaMemcpyAsync(h->counts, d.d_counts, (size_t)nq * 4, cudaMemcpyDeviceToHost, x->stream));
  int rc = wait_stream(x);
  if (rc != HFM_OK) {
    if (rc == HFM_E_TIMEOUT) x->orphans.push_back(blk);   // copies may still land in blk
    else host_result_free(blk);
    return rc;
  }
  *out = h;
  return HFM_OK;
}

int hfm_mems_batch(hfm_index* x, const uint8_t* q, const uint64_t* q_off, uint32_t nq, uint32_t min_len, uint32_t mode,
                   const uint32_t* ref_bounds, uint32_t nb, uint32_t cap, hfm_mem_out** out) {
  if (!x || !out || (nb && !ref_bounds)) return set_error(HFM_E_ARG, "NULL argument");
  *out = nullptr;
  Guard g(x);
  RET(stage_queries(x, q, q_off, nq));
  hfm_dev_mems d{};
  RET(mems_device(x, x->q.as<uint8_t>(), x->qoff.as<uint64_t>(), nq, min_len, mode, ref_bounds, nb, cap, &d));
  size_t bytes = sizeof(hfm_mem_out) + ((size_t)nq + 1) * 8 + (size_t)d.n_hits * sizeof(hfm_mem_hit) +
                 (size_t)d.n_positions * 8 + 8;
  uint8_t* blk = (uint8_t*)host_result_alloc(bytes);
  if (!blk) return set_error(HFM_E_OOM, "host allocation failed");
  hfm_mem_out* m = (hfm_mem_out*)blk;
  m->nq = nq; m->_pad = 0; m->n_hits = d.n_hits; m->n_positions = d.n_positions;
  m->hit_offsets = (uint64_t*)(blk + sizeof(hfm_mem_out));
  m->hits = (hfm_mem_hit*)(m->hit_offsets + nq + 1);
  m->positions = (uint32_t*)(m->hits + d.n_hits);
  CK(cudaMemcpyAsync(m->hit_offsets, d.d_hit_offsets, ((size_t)nq + 1) * 8, cudaMemcpyDeviceToHost, x->stream));
  if (d.n_hits) CK(cudaMemcpyAsync(m->hits, d.d_hits, (size_t)d.n_hits * sizeof(hfm_mem_hit), cudaMemcpyDeviceToHost, x->stream));
  if (d.n_positions) CK(cudaMemcpyAsync(m->positions, d.d_positions, (size_t)d.n_positions * 8, cudaMemcpyDeviceToHost, x->stream));
  int rc = wait_stream(x);
  if (rc != HFM_OK) {
    if (rc == HFM_E_TIMEOUT) x->orphans.push_back(blk);   // copies may still land in blk
    else host_result_free(blk);
    return rc;
  }
  *out = m;
  return HFM_OK;
}

// ---------------------------------------------------------------------------
// CUDA-graph-captured SMEM/MEM pass chain
// ---------------------------------------------------------------------------
struct hfm_graph {
  hfm_index* sh = nullptr;           // shadow handle: the index's device layout, own buffers and stream
  cudaGraphExec_t exec = nullptr;
  FixedChain c{};
  bool stale = true;                 // capture (again) before the next replay
  uint64_t* h_bases = nullptr;       // pinned: the batch's total codes, then both chains' totals and counters
  uint32_t replays = 0, fallbacks = 0, last_reason = 0;
  DevBuf tot;                        // GraphTotals of the SMEM chain, then of the locate chain
  std::vector<uint32_t> bounds;      // host copy of the reference bounds (for the adaptive rerun)
  bool has_loc = false;              // a locate chain precedes the SMEM chain in the graph
  FixedLocate lc{};
  DevBuf lctr;                       // the locate chain's counters
  hfm_dev_hits loc_out{};            // the locate result of the last launch
};

namespace hfm {

static void free_graph(hfm_graph* g) {
  if (!g) return;
  if (g->sh) {
    cudaSetDevice(g->sh->device);
    if (g->sh->stream) cudaStreamSynchronize(g->sh->stream);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    g->tot.release();
    g->lctr.release();
    hfm_index_free(g->sh);             // a shadow: the index buffers stay with their handle
  }
  if (g->h_bases) cudaFreeHost(g->h_bases);
  delete g;
}

static int capture(hfm_graph* g) {
  hfm_index* x = g->sh;
  if (g->exec) { cudaGraphExecDestroy(g->exec); g->exec = nullptr; }
  if (g->has_loc) RET(fixed_locate(x, g->lc, false));   // every allocation, outside the capture
  RET(fixed_chain(x, g->c, false));
  CK(cudaStreamSynchronize(x->stream));
  CK(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
  int rc = g->has_loc ? fixed_locate(x, g->lc, true) : HFM_OK;
  if (rc == HFM_OK) rc = fixed_chain(x, g->c, true);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(x->stream, &graph);
  if (rc != HFM_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
  if (e != cudaSuccess) return set_error(HFM_E_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&g->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) { g->exec = nullptr; return set_error(HFM_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)); }
  g->stale = false;
  return HFM_OK;
}

}  // namespace hfm

extern "C" int hfm_mems_graph_create(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq,
                                     uint64_t max_bases, uint32_t min_len, uint32_t mode, const uint32_t* ref_bounds,
                                     uint32_t nb, uint32_t max_hits, uint64_t max_positions, hfm_graph** out) {
  if (!x || !out || !d_qoff || !nq || (nb && !ref_bounds)) return set_error(HFM_E_ARG, "NULL argument or empty batch");
  if (x->kind != HFM_KIND_BIDIR) return set_error(HFM_E_ARG, "MEM/SMEM search needs a bidirectional index");
  if (mode > 1) return set_error(HFM_E_ARG, "mode must be 0 (SMEM) or 1 (MEM)");
  *out = nullptr;
  std::unique_lock<std::mutex> lk(x->mu);
  CK(cudaSetDevice(x->device));
  std::unique_ptr<hfm_graph, void (*)(hfm_graph*)> g(new hfm_graph(), free_graph);
  RET(make_shadow(x, &g->sh));
  hfm_index* sh = g->sh;
  if (sh->mems_variant == MEMS_PLAIN) sh->mems_variant = 3;
  sh->miv_cap = std::max<uint64_t>(x->miv_cap, (uint64_t)nq * 24 + 4096);
  sh->hit_cap = std::max<uint64_t>(x->hit_cap, (uint64_t)nq * 24 + 4096);
  sh->seg_cap = x->seg_cap;
  CK(cudaMallocHost((void**)&g->h_bases, 512));
  RET(g->tot.ensure(2 * sizeof(GraphTotals)));
  RET(sh->ref_bounds.ensure((size_t)nb * 4 + 4));
  if (nb) CK(cudaMemcpy(sh->ref_bounds.p, ref_bounds, (size_t)nb * 4, cudaMemcpyHostToDevice));
  g->bounds.assign(ref_bounds, ref_bounds + nb);
  FixedChain& c = g->c;
  c.d_q = d_q; c.d_qoff = d_qoff; c.nq = nq; c.max_bases = max_bases;
  c.P = MemsParams{min_len, mode, max_hits, nb ? 1u : 0u};
  c.nb = nb;
  c.dedup = !(x->flags & HFM_FLAG_DEDUP_NEVER);
  c.pos_cap = std::max<uint64_t>(max_positions, 4096);
  c.upos_cap = c.pos_cap / 16 + 4096;        // distinct positions: grown on a fallback
  c.d_tot = g->tot.as<GraphTotals>();
  c.h_tot = reinterpret_cast<GraphTotals*>(g->h_bases + 1);
  lk.unlock();
  {
    std::lock_guard<std::mutex> lg(sh->mu);
    RET(capture(g.get()));
  }
  *out = g.release();
  return HFM_OK;
}

extern "C" int hfm_mems_graph_launch(hfm_graph* g, hfm_dev_mems* out, uint32_t* replayed) {
  if (!g || !out) return set_error(HFM_E_ARG, "NULL argument");
  hfm_index* x = g->sh;
  std::lock_guard<std::mutex> lk(x->mu);
  CK(cudaSetDevice(x->device));
  FixedChain& c = g->c;
  // the one read before the replay: the batch must fit the captured segment capacity
  CK(cudaMemcpyAsync(g->h_bases, c.d_qoff + c.nq, 8, cudaMemcpyDeviceToHost, x->stream));
  RET(wait_stream(x));
  uint32_t reason = g->h_bases[0] <= c.max_bases ? 0u : HFM_GRAPH_BASES;
  if (!reason) {
    if (g->stale) RET(capture(g));
    CK(cudaGraphLaunch(g->exec, x->stream));
    RET(wait_stream(x));
    const Counters& k = *x->h_ctr;
    const GraphTotals& t = *c.h_tot;
    if (k.walk_err) return set_error(HFM_E_WALK, "LF walk exceeded sample_rate steps: index inconsistent");
    reason = (k.iv_used > x->miv_cap ? HFM_GRAPH_INTERVALS : 0u) | (k.hit_used > x->hit_cap ? HFM_GRAPH_HITS : 0u) |
             (k.seg_used > x->seg_cap ? HFM_GRAPH_SEGMENTS : 0u) | (k.still_ovf ? HFM_GRAPH_WARP_SETS : 0u) |
             (t.ovf ? HFM_GRAPH_POSITIONS : 0u);
    if (reason & HFM_GRAPH_WARP_SETS) {       // the next capture gets larger warp-tier sets
      c.warp_cap = std::min<uint32_t>(c.warp_cap * 4, 1u << 22);
      c.warp_cands = std::min<uint32_t>(c.warp_cands * 4, 1u << 20);
    }
    if (g->has_loc) {
      const Counters& lk = *g->lc.h_ctr;
      const GraphTotals& lt = *g->lc.h_tot;
      if (lk.walk_err) return set_error(HFM_E_WALK, "LF walk exceeded sample_rate steps: index inconsistent");
      if (lk.iv_used > g->lc.iv_cap || lk.still_ovf || lt.ovf) reason |= HFM_GRAPH_LOCATE;
      if (lk.still_ovf) g->lc.warp_cap = std::min<uint32_t>(g->lc.warp_cap * 4, 1u << 22);
      if (lk.iv_used > g->lc.iv_cap) g->lc.iv_cap = lk.iv_used + lk.iv_used / 4 + 4096;
      if (!(reason & HFM_GRAPH_LOCATE)) {
        FixedLocate& l = g->lc;
        g->loc_out = hfm_dev_hits{l.nq, 0, lt.npos, x->pos_base.as<uint64_t>(), x->counts.as<uint32_t>(),
                                  x->loc_pairs.as<uint32_t>()};
      }
    }
    g->last_reason = reason;
    if (!reason) {
      g->replays++;
      out->nq = c.nq; out->n_hits = t.nh; out->n_positions = t.npos;
      out->d_hit_offsets = x->hit_base.as<uint64_t>(); out->d_hits = x->hits.as<hfm_mem_hit>();
      out->d_positions = x->out_pairs.as<uint32_t>();
      if (replayed) *replayed = 1;
      return HFM_OK;
    }
  }
  // a capacity was outgrown: the adaptive chains (same results), then capture again with
  // the capacities they grew to.  The adaptive locate leaves its positions where the SMEM
  // chain puts its own, so it runs first and its positions move to the locate buffer.
  g->last_reason = reason;
  g->fallbacks++;
  g->stale = true;
  if (g->has_loc && (reason & (HFM_GRAPH_LOCATE | HFM_GRAPH_BASES))) {
    FixedLocate& l = g->lc;
    hfm_dev_hits h{};
    RET(locate_device(x, l.d_q, l.d_qoff, l.nq, l.max_hits, &h));
    RET(x->loc_pairs.ensure(h.total * 8 + 8));
    if (h.total) CK(cudaMemcpyAsync(x->loc_pairs.p, h.d_pairs, h.total * 8, cudaMemcpyDeviceToDevice, x->stream));
    h.d_pairs = x->loc_pairs.as<uint32_t>();
    g->loc_out = h;
    l.pos_cap = std::max<uint64_t>(l.pos_cap, h.total + h.total / 4 + 4096);
    // distinct positions: what the adaptive run walked (all its positions when it did not
    // deduplicate: never fewer distinct than that), at least twice the old capacity
    const uint64_t ru = x->stats.rows_unique ? x->stats.rows_unique : h.total;
    l.upos_cap = std::max<uint64_t>(2 * l.upos_cap, ru + ru / 4 + 4096);
  }
  c.max_bases = std::max<uint64_t>(c.max_bases, g->h_bases[0] + g->h_bases[0] / 4);
  RET(mems_device(x, c.d_q, c.d_qoff, c.nq, c.P.min_len, c.P.mode, g->bounds.empty() ? nullptr : g->bounds.data(),
                  c.nb, c.P.max_hits, out));
  c.pos_cap = std::max<uint64_t>(c.pos_cap, out->n_positions + out->n_positions / 4 + 4096);
  if (reason & HFM_GRAPH_POSITIONS) {
    const uint64_t ru = x->stats.rows_unique ? x->stats.rows_unique : out->n_positions;
    c.upos_cap = std::max<uint64_t>(2 * c.upos_cap, ru + ru / 4 + 4096);
  }
  if (replayed) *replayed = 0;
  return HFM_OK;
}

extern "C" int hfm_mems_graph_add_locate(hfm_graph* g, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq,
                                         uint32_t max_hits, uint64_t max_intervals, uint64_t max_positions) {
  if (!g || !d_qoff || !nq) return set_error(HFM_E_ARG, "NULL argument or empty batch");
  if (g->has_loc) return set_error(HFM_E_ARG, "the graph already has a locate chain");
  hfm_index* x = g->sh;
  std::lock_guard<std::mutex> lk(x->mu);
  CK(cudaSetDevice(x->device));
  RET(g->lctr.ensure(sizeof(Counters)));
  FixedLocate& l = g->lc;
  l.d_q = d_q; l.d_qoff = d_qoff; l.nq = nq; l.max_hits = max_hits;
  l.iv_cap = std::max<uint64_t>(max_intervals, (uint64_t)nq * 2 + 4096);
  l.pos_cap = std::max<uint64_t>(max_positions, 4096);
  l.upos_cap = l.pos_cap / 16 + 4096;
  l.dedup = !(x->flags & HFM_FLAG_DEDUP_NEVER);
  l.ctr = g->lctr.as<Counters>();
  l.d_tot = g->tot.as<GraphTotals>() + 1;
  l.h_tot = reinterpret_cast<GraphTotals*>(g->h_bases + 8);
  l.h_ctr = reinterpret_cast<Counters*>(g->h_bases + 16);
  g->has_loc = true;
  int rc = capture(g);
  if (rc != HFM_OK) g->has_loc = false;
  return rc;
}

extern "C" int hfm_mems_graph_locate_result(const hfm_graph* g, hfm_dev_hits* out) {
  if (!g || !out) return set_error(HFM_E_ARG, "NULL argument");
  if (!g->has_loc) return set_error(HFM_E_ARG, "the graph has no locate chain");
  *out = g->loc_out;
  return HFM_OK;
}

extern "C" void hfm_mems_graph_free(hfm_graph* g) { free_graph(g); }

extern "C" int hfm_mems_graph_info(const hfm_graph* g, uint32_t* replays, uint32_t* fallbacks, uint32_t* last_reason) {
  if (!g) return set_error(HFM_E_ARG, "NULL argument");
  if (replays) *replays = g->replays;
  if (fallbacks) *fallbacks = g->fallbacks;
  if (last_reason) *last_reason = g->last_reason;
  return HFM_OK;
}

extern "C" int hfm_index_share(hfm_index* x, hfm_index** out) {
  if (!x || !out) return set_error(HFM_E_ARG, "NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(x->mu);
  return make_shadow(x, out);
}

}  // extern "C"

// ===========================================================================
// Allocation-free count entry point.
//
// Some callers cannot let a library call cudaMalloc: a host framework that owns all of
// the GPU's memory through its own pool allocator (and would be pushed out of memory or
// bypassed by foreign allocations), or a latency-bound serving loop where cudaMalloc's
// implicit device synchronisation and multi-millisecond cost are not acceptable.
// hfm_count_batch_noalloc serves them: it runs the same backward-search kernels as
// hfm_count_batch_device, but its work area (interval sets, queue counters, per-query
// status and overflow list) is the file-scope device array below instead of buffers the
// handle allocates.  The caller passes device inputs and the device output.
//
// Costs and limits:
//  * the array (NOALLOC_SCRATCH_BYTES, 17 MiB) exists on every GPU that loads this
//    library, for the life of the process;
//  * at most NOALLOC_MAX_QUERIES queries per call, and an interval set of at most
//    NOALLOC_WARP_SET_CAP intervals per query (larger sets return HFM_E_OVERFLOW);
//  * every call shares the one array, so calls that overlap on the GPU (two streams, two
//    handles, two host threads) race and must be serialised by the caller;
//  * the first call on a device resolves the array's device address with
//    cudaGetSymbolAddress (with that device current); make that first call before any
//    stream capture is started.
// ===========================================================================
namespace hfm {

constexpr uint32_t NOALLOC_MAX_QUERIES = 1u << 20;
constexpr uint32_t NOALLOC_THREADS = 16384;        // fast pass: 64 blocks x 256 threads
constexpr uint32_t NOALLOC_SET_CAP = 32;           // fast pass: intervals per set
constexpr uint32_t NOALLOC_WARPS = 32;             // long-tail pass: 8 blocks x 4 warps
constexpr uint32_t NOALLOC_WARP_SET_CAP = 2048;    // long-tail pass: intervals per set
constexpr size_t NOALLOC_CTR_BYTES = 256;
constexpr size_t NOALLOC_FAST_BYTES = (size_t)NOALLOC_THREADS * 2 * NOALLOC_SET_CAP * sizeof(uint2);
constexpr size_t NOALLOC_TAIL_BYTES = (size_t)NOALLOC_WARPS * 2 * NOALLOC_WARP_SET_CAP * sizeof(uint2);
constexpr size_t NOALLOC_LIST_BYTES = (size_t)NOALLOC_MAX_QUERIES * sizeof(uint32_t);
constexpr size_t NOALLOC_SCRATCH_BYTES =
    NOALLOC_CTR_BYTES + NOALLOC_FAST_BYTES + NOALLOC_TAIL_BYTES + 2 * NOALLOC_LIST_BYTES;   // 17 MiB + 256 B

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

struct NoallocCtr { unsigned int queue, queue2; uint32_t n_ovf, still_ovf; unsigned long long used, touches; };

// Device address of g_noalloc_scratch per device ordinal (host code cannot use the
// symbol itself: on the host it names a stand-in, not device memory).
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[256] = {nullptr};

static int noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= 256) return set_error(HFM_E_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);   // the calling device is current
    if (e != cudaSuccess || !p)
      return set_error(HFM_E_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
    g_noalloc_addr[device] = p;
  }
  *out = (unsigned char*)g_noalloc_addr[device];
  return HFM_OK;
}

}  // namespace hfm

extern "C" int hfm_count_batch_noalloc(hfm_index* x, const uint8_t* d_q, const uint64_t* d_qoff, uint32_t nq,
                                       uint32_t* d_counts) {
  if (!x || (nq && (!d_qoff || !d_counts))) return set_error(HFM_E_ARG, "NULL argument");
  if (nq > NOALLOC_MAX_QUERIES)
    return set_error(HFM_E_ARG, "hfm_count_batch_noalloc: " + std::to_string(nq) + " queries exceed the limit of " +
                                    std::to_string(NOALLOC_MAX_QUERIES) + " per call");
  Guard g(x);
  unsigned char* base = nullptr;
  RET(noalloc_scratch(x->device, &base));
  if (nq == 0) return HFM_OK;
  NoallocCtr* ctr = (NoallocCtr*)base;
  uint2* fast = (uint2*)(base + NOALLOC_CTR_BYTES);
  uint2* tail = (uint2*)(base + NOALLOC_CTR_BYTES + NOALLOC_FAST_BYTES);
  uint32_t* status = (uint32_t*)(base + NOALLOC_CTR_BYTES + NOALLOC_FAST_BYTES + NOALLOC_TAIL_BYTES);
  uint32_t* ovf = status + NOALLOC_MAX_QUERIES;
  const FmDev& F = x->fwd;
  // the previous call's counters are still in the array: clear them
  CK(cudaMemsetAsync(ctr, 0, sizeof(NoallocCtr), x->stream));
  Pool pool{nullptr, &ctr->used, 0};
  BsOut o{d_counts, nullptr, nullptr, nullptr, status, ovf, &ctr->n_ovf, &ctr->touches};
  k_bsearch<false, 32><<<NOALLOC_THREADS / 256, 256, 0, x->stream>>>(F.d, F.compat.as<uint16_t>(), d_q, d_qoff, nullptr,
                                                                     nq, 0, fast, NOALLOC_SET_CAP, &ctr->queue, pool,
                                                                     o, &ctr->still_ovf);
  CK(cudaGetLastError());
  uint32_t n_ovf = 0;
  CK(cudaMemcpyAsync(&n_ovf, &ctr->n_ovf, sizeof(uint32_t), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  if (n_ovf) {
    k_bsearch_warp<false><<<NOALLOC_WARPS / 4, 128, 0, x->stream>>>(F.d, F.compat.as<uint16_t>(), d_q, d_qoff, ovf, n_ovf,
                                                                   0, tail, NOALLOC_WARP_SET_CAP, &ctr->queue2, pool,
                                                                   o, &ctr->still_ovf);
    CK(cudaGetLastError());
    uint32_t still = 0;
    CK(cudaMemcpyAsync(&still, &ctr->still_ovf, sizeof(uint32_t), cudaMemcpyDeviceToHost, x->stream));
    CK(cudaStreamSynchronize(x->stream));
    if (still)
      return set_error(HFM_E_OVERFLOW, "hfm_count_batch_noalloc: an interval set exceeds " +
                                           std::to_string(NOALLOC_WARP_SET_CAP) + " intervals (use hfm_count_batch)");
  }
  CK(cudaStreamSynchronize(x->stream));
  return HFM_OK;
}
