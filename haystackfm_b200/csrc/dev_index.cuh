// dev_index.cuh — device-resident FM-index layout and the rank / LF / extension
// primitives every kernel uses.
//
// Device layout (built once by hfm_index_load from the reference's bincode records):
//   occ   : one 96-byte record per 64 BWT rows: 16 x u32 counts of every symbol code before
//           the block, then 4 x u64 bitplanes of each row's 4-bit symbol code.  The reference
//           compacts symbols to lanes and splits counts into superblock + u16 delta; on the
//           device the lane IS the symbol code and the count is whole, so a rank is one
//           record read (3 DRAM sectors) and no table lookup.
//   ssa   : one 16-byte record per 64 rows: u64 "row is sampled" bits + u32 count of
//           sampled rows before the word (SampledSuffixArray, src/suffix_array/mod.rs:54-63).
//   sa_vals, seq_boundaries, lookup intervals: as in the reference.
// rank(c, i) = occ[(i-1)/64].count[c] + popc(rows of code c <= (i-1)%64),
// identical to OccTable::rank (src/occ/mod.rs:330-363).
#pragma once
#include <cstdint>

namespace hfm {

struct DevFm {
  const uint4* occ;          // 6 x uint4 per block
  const uint4* ssa;          // 1 x uint4 per block
  const uint32_t* sa_vals;
  const uint2* lut;          // nullptr when the index has no lookup table
  const uint32_t* seq_bounds;
  uint32_t text_len, num_seqs, sample_rate, lut_depth;
  uint32_t tag, lut_radix, num_blocks, _pad;
  uint32_t C[16];
  uint8_t s2l[16], l2s[16], lut_digit[16];
  uint16_t sym_mask;         // symbols present in the text
  uint16_t _pad2;
};

struct BIv { uint32_t flo, fhi, rlo, rhi; };

// Per-kernel shared copies of the small tables (divergent indexing from registers or
// the parameter bank would serialise).
struct SmemFm {
  uint32_t C[16];
  uint8_t s2l[16], l2s[16], dig[16];
  uint16_t compat_mask[16];   // compatible-symbol set of each query code as a bit mask
};

__device__ __forceinline__ void smem_fm_init(SmemFm& s, const DevFm& F, const uint16_t* compat_masks) {
  int t = threadIdx.x;
  if (t < 16) {
    s.C[t] = F.C[t]; s.s2l[t] = F.s2l[t]; s.l2s[t] = F.l2s[t]; s.dig[t] = F.lut_digit[t];
    s.compat_mask[t] = compat_masks[t];
  }
}

__device__ __forceinline__ uint64_t u2to64(uint32_t lo, uint32_t hi) { return ((uint64_t)hi << 32) | lo; }

__device__ __forceinline__ uint32_t sel4(uint4 x, uint32_t i) {
  return (i & 2) ? ((i & 1) ? x.w : x.z) : ((i & 1) ? x.y : x.x);
}
__device__ __forceinline__ uint32_t sel16(uint4 a, uint4 b, uint4 c, uint4 d, uint32_t i) {
  uint4 x = (i & 8) ? ((i & 4) ? d : c) : ((i & 4) ? b : a);
  return sel4(x, i & 3);
}

struct OccRec { uint4 c0, c1, c2, c3, p0, p1; };

__device__ __forceinline__ OccRec load_occ(const DevFm& F, uint32_t blk) {
  const uint4* r = F.occ + (size_t)blk * 6;
  OccRec o;
  o.c0 = __ldg(r); o.c1 = __ldg(r + 1); o.c2 = __ldg(r + 2); o.c3 = __ldg(r + 3);
  o.p0 = __ldg(r + 4); o.p1 = __ldg(r + 5);
  return o;
}

// Rank of every symbol code at position i (counts of code s in bwt[0..i)), absent codes 0.
__device__ __forceinline__ void sym_ranks(const DevFm& F, const SmemFm& S, uint32_t i, uint32_t r[16]) {
  if (i == 0) {
#pragma unroll
    for (int s = 0; s < 16; s++) r[s] = 0;
    return;
  }
  uint32_t pos = i - 1, off = pos & 63;
  OccRec o = load_occ(F, pos >> 6);
  uint64_t low = (2ull << off) - 1ull;          // bits 0..off (off = 63 -> all ones)
  uint64_t pl[4] = {u2to64(o.p0.x, o.p0.y), u2to64(o.p0.z, o.p0.w), u2to64(o.p1.x, o.p1.y), u2to64(o.p1.z, o.p1.w)};
  // symbol masks by successive splits on planes 3,2,1,0: m[s] = rows of code s among bits <= off
  uint64_t m[16];
  m[0] = low;
#pragma unroll
  for (int p = 3; p >= 0; --p) {
    const int cnt = 1 << (3 - p);
#pragma unroll
    for (int k = cnt - 1; k >= 0; --k) { uint64_t v = m[k]; m[2 * k + 1] = v & pl[p]; m[2 * k] = v & ~pl[p]; }
  }
  uint32_t cw[16] = {o.c0.x, o.c0.y, o.c0.z, o.c0.w, o.c1.x, o.c1.y, o.c1.z, o.c1.w,
                     o.c2.x, o.c2.y, o.c2.z, o.c2.w, o.c3.x, o.c3.y, o.c3.z, o.c3.w};
#pragma unroll
  for (int s = 0; s < 16; s++) r[s] = cw[s] + (uint32_t)__popcll(m[s]);
}

// One LF step with the sampled-SA test (FmIndex::resolve_sa loop body,
// src/fm_index/query.rs:282-291; lf_step src/occ/mod.rs:456-480).  Returns true with
// *val = SA value when row `pos` is sampled; otherwise advances pos = LF(pos).
__device__ __forceinline__ bool lf_or_sample(const DevFm& F, const SmemFm& S, uint32_t& pos, uint32_t& val) {
  uint32_t blk = pos >> 6, off = pos & 63;
  uint4 w = __ldg(F.ssa + blk);
  OccRec o = load_occ(F, blk);            // issued before the sampled test: overlaps its latency
  uint64_t word = u2to64(w.x, w.y);
  uint64_t below = (1ull << off) - 1ull;
  if ((word >> off) & 1ull) {
    val = __ldg(F.sa_vals + w.z + (uint32_t)__popcll(word & below));
    return true;
  }
  uint64_t p0 = u2to64(o.p0.x, o.p0.y), p1 = u2to64(o.p0.z, o.p0.w);
  uint64_t p2 = u2to64(o.p1.x, o.p1.y), p3 = u2to64(o.p1.z, o.p1.w);
  uint32_t lane = (uint32_t)((p0 >> off) & 1) | ((uint32_t)((p1 >> off) & 1) << 1) |
                  ((uint32_t)((p2 >> off) & 1) << 2) | ((uint32_t)((p3 >> off) & 1) << 3);
  uint64_t m = below & ((lane & 1) ? p0 : ~p0) & ((lane & 2) ? p1 : ~p1) & ((lane & 4) ? p2 : ~p2) &
               ((lane & 8) ? p3 : ~p3);
  uint32_t rank = sel16(o.c0, o.c1, o.c2, o.c3, lane) + (uint32_t)__popcll(m);
  pos = S.C[lane] + rank;
  return false;
}

// partition_point(bounds, b <= p): first index with bounds[idx] > p.
__device__ __forceinline__ uint32_t upper_bound_u32(const uint32_t* b, uint32_t n, uint32_t p) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) { uint32_t mid = (lo + hi) >> 1; if (b[mid] <= p) lo = mid + 1; else hi = mid; }
  return lo;
}

}  // namespace hfm
