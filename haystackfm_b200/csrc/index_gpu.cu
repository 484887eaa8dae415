// index_gpu.cu — FM-index construction on the GPU, emitting the same bincode bytes as the
// CPU builder (index_build.cpp).
//
// Replaces FmIndex::build / BidirFmIndex::build (src/fm_index/mod.rs:209-284,
// src/fm_index/bidir_index.rs:91-116), whose wgpu pipelines sort suffixes by prefix
// doubling (src/suffix_array/gpu.rs:86) and build a 16-lane Occ table
// (src/occ/gpu.rs:34).  This builder keeps the CPU builder's contract instead — compacted
// lanes, either alphabet, the depth-k lookup table (src/fm_index/mod.rs:117-195) — so its
// bytes equal FmIndex::build_cpu_with's for the same input, at genome scale.
//
// Suffix sorting is prefix doubling (Manber & Myers) over CUB radix sort, refining only the
// suffixes whose group is still tied (as Larsson & Sadakane do): round 0 sorts every suffix
// by its first 21 (ACGT texts) or 12 (IUPAC texts) codes packed into 64 bits; each later
// round h sorts the tied suffixes by (rank[i], rank[i + h]) and splits their groups.
// Ranks are 1 + the first SA slot of the suffix's group; 0 stands for "past the end", so a
// proper prefix sorts first, as build_suffix_array_naive (src/suffix_array/cpu.rs:20-25).
// Device memory: about 39 bytes per text position during the sort.

#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "hfm_internal.h"

namespace hfm {

#define GCK(call)                                                                                 \
  do {                                                                                            \
    cudaError_t _e = (call);                                                                      \
    if (_e != cudaSuccess)                                                                        \
      return set_error(_e == cudaErrorMemoryAllocation ? HFM_E_OOM : HFM_E_CUDA,                  \
                       std::string(#call) + ": " + cudaGetErrorString(_e));                       \
  } while (0)
#define GRET(x) do { int _r = (x); if (_r != HFM_OK) return _r; } while (0)

// Device allocation released at scope exit.
struct DMem {
  void* p = nullptr;
  ~DMem() { if (p) cudaFree(p); }
  int alloc(size_t bytes) {
    if (p) { cudaFree(p); p = nullptr; }
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return set_error(HFM_E_OOM, "cudaMalloc failed during GPU index construction: " + std::to_string(bytes) + " bytes");
    }
    return HFM_OK;
  }
  void release() { if (p) cudaFree(p); p = nullptr; }
  template <class T> T* as() const { return (T*)p; }
};

static unsigned grid_for(uint64_t n, unsigned t = 256) {
  uint64_t g = (n + t - 1) / t;
  return (unsigned)std::min<uint64_t>(g, 1u << 30);
}

// ---- suffix sorting ------------------------------------------------------------------

// key[i] = the first k codes of suffix i, each as code + 1 in `bits` bits (0 past the end).
__global__ void k_sa_keys0(const uint8_t* __restrict__ t, uint64_t n, int bits, int k, uint64_t* __restrict__ key,
                           uint32_t* __restrict__ val) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t v = 0;
    for (int j = 0; j < k; j++) v = (v << bits) | (i + j < n ? (uint64_t)t[i + j] + 1 : 0ull);
    key[i] = v;
    val[i] = (uint32_t)i;
  }
}

// head[j] = 1 where sorted key j starts a new group.
__global__ void k_heads(const uint64_t* __restrict__ key, uint64_t m, uint8_t* __restrict__ head) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x)
    head[j] = (j == 0 || key[j] != key[j - 1]) ? 1 : 0;
}

// g_in[j] = slot of j when it heads a group (slots: `slot` or j itself), else 0.
__global__ void k_head_slots(const uint8_t* __restrict__ head, const uint32_t* __restrict__ slot, uint64_t m,
                             uint32_t* __restrict__ g_in) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x)
    g_in[j] = head[j] ? (slot ? slot[j] : (uint32_t)j) : 0u;
}

// rank[suffix] = 1 + first slot of its group; tied[j] = its group has more than one member.
__global__ void k_set_ranks(const uint32_t* __restrict__ suf, const uint32_t* __restrict__ g, const uint8_t* __restrict__ head,
                            uint64_t m, uint32_t* __restrict__ rank, uint8_t* __restrict__ tied) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
    rank[suf[j]] = g[j] + 1;
    bool single = head[j] && (j + 1 == m || head[j + 1]);
    tied[j] = single ? 0 : 1;
  }
}

// Round h: the tied suffixes (slots U) keyed by (rank[i], rank[i + h]).
__global__ void k_sa_keys(const uint32_t* __restrict__ U, uint64_t m, const uint32_t* __restrict__ sa,
                          const uint32_t* __restrict__ rank, uint64_t n, uint64_t h, uint64_t* __restrict__ key,
                          uint32_t* __restrict__ val) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < m; t += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t i = sa[U[t]];
    uint64_t r2 = (uint64_t)i + h < n ? rank[i + h] : 0u;
    key[t] = ((uint64_t)rank[i] << 32) | r2;
    val[t] = i;
  }
}

__global__ void k_scatter_sa(const uint32_t* __restrict__ U, const uint32_t* __restrict__ val, uint64_t m,
                             uint32_t* __restrict__ sa) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < m; t += (uint64_t)gridDim.x * blockDim.x)
    sa[U[t]] = val[t];
}

struct SaBufs {
  DMem k0, k1, v0, v1, U, rank, head, tied, tmp;
  size_t tmp_bytes = 0;
};

static int cub_tmp(SaBufs& B, size_t need) {
  if (need <= B.tmp_bytes && B.tmp.p) return HFM_OK;
  GRET(B.tmp.alloc(need));
  B.tmp_bytes = need;
  return HFM_OK;
}

// Suffix array of d_text[0..n) into d_sa (device, n u32).
static int gpu_suffix_array(const uint8_t* d_text, uint64_t n, uint32_t* d_sa, uint8_t max_code, cudaStream_t s) {
  if (n == 0) return HFM_OK;
  SaBufs B;
  GRET(B.k0.alloc(n * 8)); GRET(B.k1.alloc(n * 8));
  GRET(B.v0.alloc(n * 4)); GRET(B.v1.alloc(n * 4));
  GRET(B.rank.alloc(n * 4)); GRET(B.head.alloc(n)); GRET(B.tied.alloc(n)); GRET(B.U.alloc(n * 4));
  const int bits = max_code + 1 <= 7 ? 3 : 5;
  const int k = 64 / bits;
  k_sa_keys0<<<grid_for(n), 256, 0, s>>>(d_text, n, bits, k, B.k0.as<uint64_t>(), B.v0.as<uint32_t>());
  GCK(cudaGetLastError());
  uint64_t* kc; uint32_t* vc;
  {
    cub::DoubleBuffer<uint64_t> dk(B.k0.as<uint64_t>(), B.k1.as<uint64_t>());
    cub::DoubleBuffer<uint32_t> dv(B.v0.as<uint32_t>(), B.v1.as<uint32_t>());
    size_t need = 0;
    GCK(cub::DeviceRadixSort::SortPairs(nullptr, need, dk, dv, n, 0, bits * k, s));
    GRET(cub_tmp(B, need));
    GCK(cub::DeviceRadixSort::SortPairs(B.tmp.p, need, dk, dv, n, 0, bits * k, s));
    kc = dk.Current(); vc = dv.Current();
  }
  // vc = SA by the first k codes; copy it to d_sa
  GCK(cudaMemcpyAsync(d_sa, vc, n * 4, cudaMemcpyDeviceToDevice, s));
  uint64_t* kalt = kc == B.k0.as<uint64_t>() ? B.k1.as<uint64_t>() : B.k0.as<uint64_t>();
  uint32_t* g_in = reinterpret_cast<uint32_t*>(kalt);          // 2n u32 of free room
  uint32_t* g = g_in + n;
  k_heads<<<grid_for(n), 256, 0, s>>>(kc, n, B.head.as<uint8_t>());
  k_head_slots<<<grid_for(n), 256, 0, s>>>(B.head.as<uint8_t>(), nullptr, n, g_in);
  GCK(cudaGetLastError());
  {
    size_t need = 0;
    GCK(cub::DeviceScan::InclusiveScan(nullptr, need, g_in, g, cub::Max(), n, s));
    GRET(cub_tmp(B, need));
    GCK(cub::DeviceScan::InclusiveScan(B.tmp.p, need, g_in, g, cub::Max(), n, s));
  }
  k_set_ranks<<<grid_for(n), 256, 0, s>>>(d_sa, g, B.head.as<uint8_t>(), n, B.rank.as<uint32_t>(), B.tied.as<uint8_t>());
  GCK(cudaGetLastError());
  // U = slots of tied suffixes (ascending)
  DMem nsel;
  GRET(nsel.alloc(8));
  uint64_t m = 0;
  auto select_tied = [&](const uint32_t* slots_in, uint64_t cnt, uint32_t* slots_out) -> int {
    size_t need = 0;
    if (slots_in) {
      GCK(cub::DeviceSelect::Flagged(nullptr, need, slots_in, B.tied.as<uint8_t>(), slots_out, nsel.as<uint64_t>(),
                                     (int64_t)cnt, s));
      GRET(cub_tmp(B, need));
      GCK(cub::DeviceSelect::Flagged(B.tmp.p, need, slots_in, B.tied.as<uint8_t>(), slots_out, nsel.as<uint64_t>(),
                                     (int64_t)cnt, s));
    } else {
      thrust::counting_iterator<uint32_t> it(0);
      GCK(cub::DeviceSelect::Flagged(nullptr, need, it, B.tied.as<uint8_t>(), slots_out, nsel.as<uint64_t>(),
                                     (int64_t)cnt, s));
      GRET(cub_tmp(B, need));
      GCK(cub::DeviceSelect::Flagged(B.tmp.p, need, it, B.tied.as<uint8_t>(), slots_out, nsel.as<uint64_t>(),
                                     (int64_t)cnt, s));
    }
    GCK(cudaMemcpyAsync(&m, nsel.p, 8, cudaMemcpyDeviceToHost, s));
    GCK(cudaStreamSynchronize(s));
    return HFM_OK;
  };
  GRET(select_tied(nullptr, n, B.U.as<uint32_t>()));
  for (uint64_t h = (uint64_t)k; m > 0; h *= 2) {
    if (h >= 2 * n) return set_error(HFM_E_CUDA, "suffix sort did not converge");
    // keys of the tied suffixes, sorted; their slots keep the group order
    k_sa_keys<<<grid_for(m), 256, 0, s>>>(B.U.as<uint32_t>(), m, d_sa, B.rank.as<uint32_t>(), n, h, B.k0.as<uint64_t>(),
                                          B.v0.as<uint32_t>());
    GCK(cudaGetLastError());
    cub::DoubleBuffer<uint64_t> dk(B.k0.as<uint64_t>(), B.k1.as<uint64_t>());
    cub::DoubleBuffer<uint32_t> dv(B.v0.as<uint32_t>(), B.v1.as<uint32_t>());
    {
      size_t need = 0;
      GCK(cub::DeviceRadixSort::SortPairs(nullptr, need, dk, dv, m, 0, 64, s));
      GRET(cub_tmp(B, need));
      GCK(cub::DeviceRadixSort::SortPairs(B.tmp.p, need, dk, dv, m, 0, 64, s));
    }
    uint64_t* kk = dk.Current();
    uint32_t* vv = dv.Current();
    uint64_t* ka = kk == B.k0.as<uint64_t>() ? B.k1.as<uint64_t>() : B.k0.as<uint64_t>();
    uint32_t* gi = reinterpret_cast<uint32_t*>(ka);
    uint32_t* gg = gi + m;
    k_scatter_sa<<<grid_for(m), 256, 0, s>>>(B.U.as<uint32_t>(), vv, m, d_sa);
    k_heads<<<grid_for(m), 256, 0, s>>>(kk, m, B.head.as<uint8_t>());
    k_head_slots<<<grid_for(m), 256, 0, s>>>(B.head.as<uint8_t>(), B.U.as<uint32_t>(), m, gi);
    GCK(cudaGetLastError());
    {
      size_t need = 0;
      GCK(cub::DeviceScan::InclusiveScan(nullptr, need, gi, gg, cub::Max(), m, s));
      GRET(cub_tmp(B, need));
      GCK(cub::DeviceScan::InclusiveScan(B.tmp.p, need, gi, gg, cub::Max(), m, s));
    }
    k_set_ranks<<<grid_for(m), 256, 0, s>>>(vv, gg, B.head.as<uint8_t>(), m, B.rank.as<uint32_t>(), B.tied.as<uint8_t>());
    GCK(cudaGetLastError());
    // the next round's tied slots go to the value buffer the sort left free, which then
    // becomes U (the old U buffer takes its place in the value double buffer)
    DMem& vfree = vv == B.v0.as<uint32_t>() ? B.v1 : B.v0;
    GRET(select_tied(B.U.as<uint32_t>(), m, vfree.as<uint32_t>()));
    std::swap(B.U.p, vfree.p);
  }
  GCK(cudaStreamSynchronize(s));
  return HFM_OK;
}

// ---- BWT, Occ records, sampled SA, lookup table ---------------------------------------

__global__ void k_bwt(const uint8_t* __restrict__ t, const uint32_t* __restrict__ sa, uint64_t n, uint8_t* __restrict__ bwt) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t v = sa[j];
    bwt[j] = t[v == 0 ? n - 1 : v - 1];
  }
}

struct LaneMap { uint8_t s2l[16]; uint32_t L, width, enc; uint64_t stride; };

// cnt[l * nblk + b] = rows of lane l in block b.
__global__ void k_block_counts(const uint8_t* __restrict__ bwt, uint64_t n, uint64_t nblk, LaneMap M,
                               uint32_t* __restrict__ cnt) {
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nblk; b += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t c[16];
    for (int l = 0; l < 16; l++) c[l] = 0;
    uint64_t end = min(n, (b + 1) * 64);
    for (uint64_t i = b * 64; i < end; i++) c[M.s2l[bwt[i] & 15]]++;
    for (uint32_t l = 0; l < M.L; l++) cnt[l * nblk + b] = c[l];
  }
}

__device__ __forceinline__ void put_bytes(uint8_t* dst, const void* src, int k) {
  const uint8_t* s = (const uint8_t*)src;
  for (int i = 0; i < k; i++) dst[i] = s[i];
}

// Records [sb u32 x L][delta u16 x L][words u64 x width] (src/occ/mod.rs:114-183) and the
// superblock checkpoints (every 8 blocks, src/occ/cpu.rs:23-119); cum = exclusive scans.
__global__ void k_occ_records(const uint8_t* __restrict__ bwt, uint64_t n, uint64_t nblk, LaneMap M,
                              const uint32_t* __restrict__ cum, uint8_t* __restrict__ rec, uint32_t* __restrict__ sbout) {
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nblk; b += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t words[16];
    for (int w = 0; w < 16; w++) words[w] = 0;
    uint64_t end = min(n, (b + 1) * 64);
    for (uint64_t i = b * 64; i < end; i++) {
      uint32_t lane = M.s2l[bwt[i] & 15];
      uint64_t bit = 1ull << (i & 63);
      if (M.enc == 0) { for (uint32_t p = 0; p < M.width; p++) if ((lane >> p) & 1) words[p] |= bit; }
      else words[lane] |= bit;
    }
    uint8_t* r = rec + b * M.stride;
    uint64_t b0 = b & ~7ull;
    for (uint32_t l = 0; l < M.L; l++) {
      uint32_t sbv = cum[l * nblk + b0];
      uint16_t dv = (uint16_t)(cum[l * nblk + b] - sbv);
      put_bytes(r + l * 4, &sbv, 4);
      put_bytes(r + M.L * 4 + l * 2, &dv, 2);
      if (b == b0) sbout[(b / 8) * M.L + l] = sbv;
    }
    for (uint32_t w = 0; w < M.width; w++) put_bytes(r + M.L * 6 + w * 8, &words[w], 8);
  }
}

// Sampled-SA words: bit j of word w = row 64w+j is sampled (SA value a multiple of the
// rate, or a sequence start; src/suffix_array/mod.rs:71-118).
__global__ void k_ssa_words(const uint32_t* __restrict__ sa, uint64_t n, uint32_t rate, const uint64_t* __restrict__ forced,
                            uint64_t nw, uint64_t* __restrict__ words, uint32_t* __restrict__ wcnt) {
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t word = 0;
    uint64_t end = min(n, (w + 1) * 64);
    for (uint64_t i = w * 64; i < end; i++) {
      uint32_t v = sa[i];
      bool mult = rate == 0 ? v == 0 : v % rate == 0;
      if (mult || ((forced[v >> 6] >> (v & 63)) & 1)) word |= 1ull << (i & 63);
    }
    words[w] = word;
    wcnt[w] = (uint32_t)__popcll(word);
  }
}

__global__ void k_ssa_records(const uint32_t* __restrict__ sa, uint64_t n, const uint64_t* __restrict__ words,
                              const uint32_t* __restrict__ wcum, uint64_t nw, uint8_t* __restrict__ rec,
                              uint32_t* __restrict__ vals) {
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t word = words[w];
    uint32_t sbb = wcum[w & ~7ull];
    uint16_t delta = (uint16_t)(wcum[w] - sbb);
    uint8_t* r = rec + w * 14;
    put_bytes(r, &word, 8); put_bytes(r + 8, &sbb, 4); put_bytes(r + 12, &delta, 2);
    uint32_t k = wcum[w];
    for (uint64_t m = word; m; m &= m - 1) vals[k++] = sa[w * 64 + __ffsll((long long)m) - 1];
  }
}

// OccTable::rank over the records just built (src/occ/mod.rs:330-363).
__device__ uint32_t ref_rank(const uint8_t* rec, LaneMap M, uint8_t c, uint32_t i) {
  if (i == 0) return 0;
  uint32_t lane = M.s2l[c];
  if (lane == 0xFF) return 0;
  uint32_t pos = i - 1, off = pos & 63;
  const uint8_t* r = rec + (uint64_t)(pos >> 6) * M.stride;
  uint32_t sbv = 0; uint16_t dv = 0;
  uint8_t* ps = (uint8_t*)&sbv; for (int k = 0; k < 4; k++) ps[k] = r[lane * 4 + k];
  uint8_t* pd = (uint8_t*)&dv; for (int k = 0; k < 2; k++) pd[k] = r[M.L * 4 + lane * 2 + k];
  uint64_t m = ~0ull;
  auto word = [&](uint32_t w) { uint64_t v = 0; uint8_t* pv = (uint8_t*)&v; for (int k = 0; k < 8; k++) pv[k] = r[M.L * 6 + w * 8 + k]; return v; };
  if (M.enc == 1) m = word(lane);
  else for (uint32_t p = 0; p < M.width; p++) { uint64_t v = word(p); m &= ((lane >> p) & 1) ? v : ~v; }
  uint64_t mask = off == 63 ? ~0ull : ((1ull << (off + 1)) - 1);
  return sbv + dv + (uint32_t)__popcll(m & mask);
}

// LookupTable::build (src/fm_index/lookup.rs:37-91), one entry per thread: the BFS visits
// entry idx only through non-empty ancestors, and a symbol absent from the text leaves its
// subtree at (0, 0).  Digits: the first extension (the pattern's last code) is the most
// significant.
__global__ void k_lookup(const uint8_t* __restrict__ rec, LaneMap M, const uint32_t* __restrict__ C, uint32_t n,
                         uint32_t depth, uint64_t size, uint2* __restrict__ out) {
  for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < size; idx += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = n;
    uint2 res = make_uint2(0, 0);
    uint64_t div = size / 4;
    for (uint32_t level = 1; level <= depth; level++, div /= 4) {
      uint32_t d = (uint32_t)((idx / (div ? div : 1ull)) % 4);
      uint8_t sym = (uint8_t)(d + 1);
      uint32_t upper = sym + 1 < 16 ? C[sym + 1] : n;
      if (upper - C[sym] == 0) break;                               // absent symbol: (0, 0)
      uint32_t nlo = C[sym] + ref_rank(rec, M, sym, lo), nhi = C[sym] + ref_rank(rec, M, sym, hi);
      if (level == depth) { res = make_uint2(nlo, nhi); break; }
      if (nlo >= nhi) break;                                        // empty ancestor: (0, 0)
      lo = nlo; hi = nhi;
    }
    out[idx] = res;
  }
}

// One FmIndex of text[0..n) (host copy `text`, device copy d_text) into f.
static int build_fm_gpu(const std::vector<uint8_t>& text, const uint8_t* d_text, const std::vector<uint32_t>& bounds,
                        const std::vector<std::string>& headers, const hfm_build_opts& o, uint32_t lookup_depth,
                        BuiltFm& f, cudaStream_t s) {
  const uint64_t n = text.size();
  f.tag = (uint8_t)o.alphabet_tag; f.encoding = o.occ_encoding; f.text_len = (uint32_t)n; f.rate = o.sa_sample_rate;
  f.num_sequences = (uint32_t)bounds.size(); f.bounds = bounds; f.headers = headers; f.lookup_depth = lookup_depth;
  // C array from the text (src/c_array.rs:14-31)
  uint64_t freq[16] = {0};
  for (uint64_t i = 0; i < n; i++) freq[text[i] & 15]++;
  uint32_t acc = 0;
  for (int c = 0; c < 16; c++) { f.C[c] = acc; acc += (uint32_t)freq[c]; }
  uint8_t max_code = 0;
  for (int c = 0; c < 16; c++) if (freq[c]) max_code = (uint8_t)c;
  DMem sa;
  GRET(sa.alloc(n * 4));
  GRET(gpu_suffix_array(d_text, n, sa.as<uint32_t>(), max_code, s));
  DMem bwt;
  GRET(bwt.alloc(n));
  k_bwt<<<grid_for(n), 256, 0, s>>>(d_text, sa.as<uint32_t>(), n, bwt.as<uint8_t>());
  GCK(cudaGetLastError());
  // lanes: symbols present, in code order (src/occ/cpu.rs:23-60)
  std::memset(f.s2l, 0xFF, 16); std::memset(f.l2s, 0, 16);
  uint8_t L = 0;
  for (int c = 0; c < 16; c++) if (freq[c]) { f.s2l[c] = L; f.l2s[L] = (uint8_t)c; L++; }
  uint8_t P = 0;
  if (L > 1) { uint32_t v = L - 1; while (v) { P++; v >>= 1; } }
  f.num_lanes = L; f.num_planes = P;
  LaneMap M;
  std::memcpy(M.s2l, f.s2l, 16);
  for (int c = 0; c < 16; c++) if (M.s2l[c] == 0xFF) M.s2l[c] = 0;   // absent codes never occur
  M.L = L; M.width = f.encoding == 0 ? P : L; M.enc = f.encoding;
  M.stride = (uint64_t)L * 6 + (uint64_t)M.width * 8;
  f.block_stride = M.stride;
  const uint64_t nblk = (n + 63) / 64;
  DMem cnt, cum, rec, sbout;
  GRET(cnt.alloc(nblk * L * 4)); GRET(cum.alloc(nblk * L * 4));
  GRET(rec.alloc(nblk * M.stride)); GRET(sbout.alloc(((nblk + 7) / 8) * L * 4));
  k_block_counts<<<grid_for(nblk), 256, 0, s>>>(bwt.as<uint8_t>(), n, nblk, M, cnt.as<uint32_t>());
  GCK(cudaGetLastError());
  {
    DMem tmp;
    size_t need = 0;
    GCK(cub::DeviceScan::ExclusiveSum(nullptr, need, cnt.as<uint32_t>(), cum.as<uint32_t>(), nblk, s));
    GRET(tmp.alloc(need));
    for (uint32_t l = 0; l < L; l++)
      GCK(cub::DeviceScan::ExclusiveSum(tmp.p, need, cnt.as<uint32_t>() + l * nblk, cum.as<uint32_t>() + l * nblk, nblk, s));
  }
  k_occ_records<<<grid_for(nblk), 256, 0, s>>>(bwt.as<uint8_t>(), n, nblk, M, cum.as<uint32_t>(), rec.as<uint8_t>(),
                                               sbout.as<uint32_t>());
  GCK(cudaGetLastError());
  cnt.release(); cum.release(); bwt.release();
  // sampled SA with every sequence start forced (src/fm_index/mod.rs:154-162)
  std::vector<uint64_t> forced((n + 63) / 64 + 1, 0);
  forced[0] |= 1;
  for (size_t k = 0; k + 1 < bounds.size(); k++) forced[bounds[k] >> 6] |= 1ull << (bounds[k] & 63);
  const uint64_t nw = (n + 63) / 64;
  DMem dforced, dwords, dwcnt, dwcum, dssa;
  GRET(dforced.alloc(forced.size() * 8)); GRET(dwords.alloc(nw * 8)); GRET(dwcnt.alloc(nw * 4 + 4));
  GRET(dwcum.alloc(nw * 4 + 4)); GRET(dssa.alloc(nw * 14));
  GCK(cudaMemcpyAsync(dforced.p, forced.data(), forced.size() * 8, cudaMemcpyHostToDevice, s));
  k_ssa_words<<<grid_for(nw), 256, 0, s>>>(sa.as<uint32_t>(), n, o.sa_sample_rate, dforced.as<uint64_t>(), nw,
                                           dwords.as<uint64_t>(), dwcnt.as<uint32_t>());
  GCK(cudaGetLastError());
  GCK(cudaMemsetAsync(dwcnt.as<uint32_t>() + nw, 0, 4, s));
  {
    DMem tmp;
    size_t need = 0;
    GCK(cub::DeviceScan::ExclusiveSum(nullptr, need, dwcnt.as<uint32_t>(), dwcum.as<uint32_t>(), nw + 1, s));
    GRET(tmp.alloc(need));
    GCK(cub::DeviceScan::ExclusiveSum(tmp.p, need, dwcnt.as<uint32_t>(), dwcum.as<uint32_t>(), nw + 1, s));
  }
  uint32_t nsamp = 0;
  GCK(cudaMemcpyAsync(&nsamp, dwcum.as<uint32_t>() + nw, 4, cudaMemcpyDeviceToHost, s));
  GCK(cudaStreamSynchronize(s));
  DMem dvals;
  GRET(dvals.alloc((uint64_t)nsamp * 4 + 4));
  k_ssa_records<<<grid_for(nw), 256, 0, s>>>(sa.as<uint32_t>(), n, dwords.as<uint64_t>(), dwcum.as<uint32_t>(), nw,
                                             dssa.as<uint8_t>(), dvals.as<uint32_t>());
  GCK(cudaGetLastError());
  sa.release();
  // lookup table over ACGT (src/fm_index/lookup.rs:37-91)
  DMem dlut, dC;
  uint64_t lsize = 0;
  if (lookup_depth > 0) {
    lsize = 1;
    for (uint32_t i = 0; i < lookup_depth; i++) lsize *= 4;
    GRET(dlut.alloc(lsize * 8)); GRET(dC.alloc(64));
    GCK(cudaMemcpyAsync(dC.p, f.C, 64, cudaMemcpyHostToDevice, s));
    k_lookup<<<grid_for(lsize), 256, 0, s>>>(rec.as<uint8_t>(), M, dC.as<uint32_t>(), (uint32_t)n, lookup_depth, lsize,
                                             dlut.as<uint2>());
    GCK(cudaGetLastError());
  }
  // results to the host
  try {
    f.block_data.resize(nblk * M.stride);
    f.sb.resize(((nblk + 7) / 8) * L);
    f.ssa_words.resize(nw * 14);
    f.sa_vals.resize(nsamp);
    f.lut.resize(lsize);
  } catch (const std::bad_alloc&) {
    return set_error(HFM_E_OOM, "host allocation failed during index construction");
  }
  GCK(cudaMemcpyAsync(f.block_data.data(), rec.p, f.block_data.size(), cudaMemcpyDeviceToHost, s));
  GCK(cudaMemcpyAsync(f.sb.data(), sbout.p, f.sb.size() * 4, cudaMemcpyDeviceToHost, s));
  GCK(cudaMemcpyAsync(f.ssa_words.data(), dssa.p, f.ssa_words.size(), cudaMemcpyDeviceToHost, s));
  if (nsamp) GCK(cudaMemcpyAsync(f.sa_vals.data(), dvals.p, (size_t)nsamp * 4, cudaMemcpyDeviceToHost, s));
  if (lsize) GCK(cudaMemcpyAsync(f.lut.data(), dlut.p, lsize * 8, cudaMemcpyDeviceToHost, s));
  GCK(cudaStreamSynchronize(s));
  return HFM_OK;
}

}  // namespace hfm

using namespace hfm;

extern "C" int hfm_build_index_gpu(const uint8_t* codes, const uint64_t* seq_off, uint32_t nseq,
                                   const char* const* headers, const hfm_build_opts* opts, int kind, int device,
                                   uint8_t** bytes_out, size_t* len_out) {
  if (!codes && nseq) return set_error(HFM_E_ARG, "codes is NULL");
  if (nseq == 0) return set_error(HFM_E_ARG, "empty sequence list");
  if (!opts || !bytes_out || !len_out || !seq_off) return set_error(HFM_E_ARG, "NULL argument");
  if (kind != HFM_KIND_FM && kind != HFM_KIND_BIDIR) return set_error(HFM_E_ARG, "kind must be 0 or 1");
  if (opts->alphabet_tag > 1 || opts->occ_encoding > 1) return set_error(HFM_E_ARG, "bad alphabet tag or encoding");
  if (opts->lookup_depth > 13) return set_error(HFM_E_ARG, "lookup_depth above 13 (4^13 entries)");
  std::vector<uint8_t> text;
  std::vector<uint32_t> bounds;
  std::vector<std::string> hs;
  GRET(concat_text(codes, seq_off, nseq, headers, text, bounds, hs));
  int ndev = 0;
  GCK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return set_error(HFM_E_ARG, "device ordinal out of range");
  GCK(cudaSetDevice(device));
  cudaStream_t s = nullptr;
  GCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); } } sg{s};
  BuiltFm fwd, rev;
  const uint64_t n = text.size();
  {
    DMem dt;
    GRET(dt.alloc(n));
    GCK(cudaMemcpyAsync(dt.p, text.data(), n, cudaMemcpyHostToDevice, s));
    GRET(build_fm_gpu(text, dt.as<uint8_t>(), bounds, hs, *opts, opts->lookup_depth, fwd, s));
  }
  if (kind == HFM_KIND_BIDIR) {
    // reverse_as_sequence (src/fm_index/bidir_index.rs:523-532): drop the final sentinel,
    // reverse, then concatenate as one sequence (which appends a new sentinel).
    std::vector<uint8_t> rtext(text.rbegin() + 1, text.rend());
    rtext.push_back(0);
    std::vector<uint8_t>().swap(text);
    DMem dt;
    GRET(dt.alloc(n));
    GCK(cudaMemcpyAsync(dt.p, rtext.data(), n, cudaMemcpyHostToDevice, s));
    GRET(build_fm_gpu(rtext, dt.as<uint8_t>(), {(uint32_t)n}, {"seq_0"}, *opts, 0, rev, s));
  }
  return emit_bytes(fwd, rev, kind, bytes_out, len_out);
}
