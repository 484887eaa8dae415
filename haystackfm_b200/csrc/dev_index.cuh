// dev_index.cuh — device-resident FM-index layout and the rank / LF / extension
// primitives every kernel uses.
//
// Device layout (built once by hfm_index_load from the reference's bincode records):
//   occ   : one record per 64 BWT rows, two formats:
//             wide   (96 B, any text): 16 x u32 counts of every code before the record, then
//                    4 x u64 planes of the rows' 4-bit codes (three 32-byte sectors);
//             narrow (32 B, texts of codes 0..4 only — ExactDna and ACGT-only IUPAC texts):
//                    4 x u16 counts of codes 1..4 from the start of the record's superblock
//                    (1,024 records = 65,536 rows) to the record, then 3 x u64 planes (one
//                    sector); the count of code 0 is the rows before the border minus the
//                    other four.
//   sb    : (narrow) 16 x u32 per superblock: count of every code before the superblock
//           (a few MB at 3.1 Gbp; it stays in L2).
//   ssa   : one 16-byte record per 64 rows: u64 "row is sampled" bits + u32 count of
//           sampled rows before the word (SampledSuffixArray, src/suffix_array/mod.rs:54-63).
//   sa_vals, seq_boundaries, lookup intervals: as in the reference.
// rank(c, i) = count[(i-1)/64][c] (+ sb[(i-1)/65536][c], narrow) + popc(rows of code c <=
// (i-1)%64), identical to OccTable::rank (src/occ/mod.rs:330-363), whose records instead
// hold compacted lanes with a u32 superblock count and a u16 delta per lane
// (src/occ/mod.rs:144).  Wide records keep whole counts: on IUPAC texts an extension emits
// many intervals, and each would otherwise need one more dependent load for its superblock
// count (measured: 173 ms against 199 ms for the SMEM search of 1M reads).
#pragma once
#include <cstdint>

namespace hfm {

enum : uint32_t { OCC_WIDE = 0, OCC_NARROW = 1 };
constexpr uint32_t SB_BLOCK_SHIFT = 10;           // records per superblock: 1024 (65,536 rows)
constexpr uint32_t OCC_WIDE_U4 = 6;               // uint4 per wide record
constexpr uint32_t OCC_NARROW_U4 = 2;             // uint4 per narrow record

struct DevFm {
  const uint4* occ;          // OCC_WIDE_U4 or OCC_NARROW_U4 uint4 per record
  const uint32_t* sb;        // 16 x u32 per superblock (narrow records)
  const uint4* ssa;          // 1 x uint4 per block
  const uint32_t* sa_vals;
  const uint2* lut;          // nullptr when the index has no lookup table
  const uint32_t* seq_bounds;
  uint32_t text_len, num_seqs, sample_rate, lut_depth;
  uint32_t tag, lut_radix, num_blocks, fmt;
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

// One record with the rows of a border selected.  A border i (0 <= i <= text_len) is the
// position between BWT rows i-1 and i: the record of row i-1, rows 0..(i-1)%64 selected
// (border 0: record 0 with no row selected; its counts and superblock entry are 0).
template <uint32_t FMT>
struct Border {
  uint4 a, b, c, d, e, f;  // wide: a..d = counts, e, f = planes; narrow: a = counts + p0, b = p1, p2
  uint64_t low;            // selected rows
  uint32_t sbi, i;         // superblock (narrow), the border itself

  __device__ __forceinline__ uint64_t plane(int k) const {
    if (FMT == OCC_WIDE) return k == 0 ? u2to64(e.x, e.y) : k == 1 ? u2to64(e.z, e.w) : k == 2 ? u2to64(f.x, f.y)
                                                                                                  : u2to64(f.z, f.w);
    return k == 0 ? u2to64(a.z, a.w) : k == 1 ? u2to64(b.x, b.y) : k == 2 ? u2to64(b.z, b.w) : 0ull;
  }
  // rows of code s among the selected ones (s a compile-time constant after unrolling)
  __device__ __forceinline__ uint64_t eq(int s) const {
    uint64_t m = low & ((s & 1) ? plane(0) : ~plane(0)) & ((s & 2) ? plane(1) : ~plane(1)) &
                 ((s & 4) ? plane(2) : ~plane(2));
    if (FMT == OCC_WIDE) m &= (s & 8) ? plane(3) : ~plane(3);
    return m;
  }
  // wide: count of code s before the record; narrow (s in 1..4): from the superblock start
  __device__ __forceinline__ uint32_t delta(int s) const {
    if (FMT == OCC_WIDE) {
      const uint4 w = s < 4 ? a : s < 8 ? b : s < 12 ? c : d;
      return sel4(w, (uint32_t)s & 3);
    }
    const uint32_t w = s <= 2 ? a.x : a.y;
    return ((s - 1) & 1) ? (w >> 16) : (w & 0xFFFFu);
  }
  // wide: rank of code s at the border; narrow: rank within the superblock
  __device__ __forceinline__ uint32_t local(int s) const { return delta(s) + (uint32_t)__popcll(eq(s)); }
};

template <uint32_t FMT>
__device__ __forceinline__ Border<FMT> load_border(const DevFm& F, uint32_t i) {
  Border<FMT> r;
  uint32_t pos = i ? i - 1 : 0u, blk = pos >> 6;
  r.low = i ? (2ull << (pos & 63)) - 1ull : 0ull;        // rows 0..pos%64 (pos%64 = 63: all)
  r.sbi = blk >> SB_BLOCK_SHIFT;
  r.i = i;
  if (FMT == OCC_WIDE) {
    const uint4* p = F.occ + (size_t)blk * OCC_WIDE_U4;
    r.a = __ldg(p); r.b = __ldg(p + 1); r.c = __ldg(p + 2); r.d = __ldg(p + 3); r.e = __ldg(p + 4); r.f = __ldg(p + 5);
  } else {
    const uint4* p = F.occ + (size_t)blk * OCC_NARROW_U4;
    r.a = __ldg(p); r.b = __ldg(p + 1); r.c = make_uint4(0, 0, 0, 0); r.d = r.c; r.e = r.c; r.f = r.c;
  }
  return r;
}

__device__ __forceinline__ uint32_t sb_count(const DevFm& F, uint32_t sbi, uint32_t s) {
  return __ldg(F.sb + (size_t)sbi * 16 + s);
}

// Absolute rank of code s at a border (occ(s, i)).
template <uint32_t FMT>
__device__ __forceinline__ uint32_t border_rank(const DevFm& F, const Border<FMT>& B, int s) {
  if constexpr (FMT == OCC_NARROW) {
    if (s == 0) {
      uint32_t t = 0;
#pragma unroll
      for (int c = 1; c <= 4; c++) t += sb_count(F, B.sbi, c) + B.local(c);
      return B.i - t;
    }
    return sb_count(F, B.sbi, s) + B.local(s);
  } else {
    const uint64_t sel0 = (s & 1) ? 0ull : ~0ull, sel1 = (s & 2) ? 0ull : ~0ull;
    const uint64_t sel2 = (s & 4) ? 0ull : ~0ull, sel3 = (s & 8) ? 0ull : ~0ull;
    const uint64_t m = B.low & (B.plane(0) ^ sel0) & (B.plane(1) ^ sel1) & (B.plane(2) ^ sel2) & (B.plane(3) ^ sel3);
    const uint4 w = s < 4 ? B.a : s < 8 ? B.b : s < 12 ? B.c : B.d;
    return sel4(w, (uint32_t)s & 3) + (uint32_t)__popcll(m);
  }
}

// The interval [lo, hi) of the BWT split by symbol: calls f(s, d, r, sbi) for every code s
// in ascending order (0..4 narrow, 0..15 wide), d = occ(s, hi) - occ(s, lo), and the lo
// border's count r: occ(s, lo) = r (wide) or sb_count(F, sbi, s) + r (narrow; one
// L2-resident load, made only for the codes the caller keeps).  `last` = the highest code
// the caller needs.
template <uint32_t FMT, class Fn>
__device__ __forceinline__ void split_by_symbol(const DevFm& F, uint32_t lo, uint32_t hi, uint32_t last, Fn&& f) {
  if constexpr (FMT == OCC_NARROW) {
    const Border<FMT> L = load_border<FMT>(F, lo), H = load_border<FMT>(F, hi);
    const bool same_sb = L.sbi == H.sbi;
    uint32_t d[5], r[5];
    uint32_t sum = 0, rsum = 0;
#pragma unroll
    for (int s = 1; s <= 4; s++) {
      const uint32_t a = L.local(s);
      uint32_t v = H.local(s) - a;
      if (!same_sb) v += sb_count(F, H.sbi, s) - sb_count(F, L.sbi, s);
      d[s] = v; sum += v; r[s] = a; rsum += a;
    }
    d[0] = (hi - lo) - sum;
    r[0] = (lo - (L.sbi << (SB_BLOCK_SHIFT + 6))) - rsum;   // rows of the superblock before lo, minus codes 1..4
#pragma unroll
    for (int s = 0; s <= 4; s++) f(s, d[s], r[s], L.sbi);
  } else {
    // Wide records: the 16 masks of each border by a split tree over its planes, then the
    // counts; groups of codes past `last` are not formed.
    const Border<FMT> L = load_border<FMT>(F, lo), H = load_border<FMT>(F, hi);
    uint32_t rl[16], rh[16];
    {
      uint64_t m[16];
      m[0] = L.low;
#pragma unroll
      for (int p = 3; p >= 0; --p) {
        const int cnt = 1 << (3 - p);
        const uint64_t pv = L.plane(p);
#pragma unroll
        for (int k = cnt - 1; k >= 0; --k) { uint64_t v = m[k]; m[2 * k + 1] = v & pv; m[2 * k] = v & ~pv; }
      }
#pragma unroll
      for (int t = 0; t < 16; t++) rl[t] = L.delta(t) + (uint32_t)__popcll(m[t]);
      m[0] = H.low;
#pragma unroll
      for (int p = 3; p >= 0; --p) {
        const int cnt = 1 << (3 - p);
        const uint64_t pv = H.plane(p);
#pragma unroll
        for (int k = cnt - 1; k >= 0; --k) { uint64_t v = m[k]; m[2 * k + 1] = v & pv; m[2 * k] = v & ~pv; }
      }
#pragma unroll
      for (int t = 0; t < 16; t++) rh[t] = H.delta(t) + (uint32_t)__popcll(m[t]);
    }
#pragma unroll
    for (int t = 0; t < 16; t++) {
      if ((uint32_t)t > last) break;
      f(t, rh[t] - rl[t], rl[t], 0u);
    }
  }
}

// The code of BWT row `row` and its rank at that row (LF step of a one-row interval,
// lane_and_mask_bitplane + rank_at_lane, src/occ/mod.rs:434-480).
template <uint32_t FMT>
__device__ __forceinline__ void row_code_rank(const DevFm& F, uint32_t row, uint32_t& code, uint32_t& rank) {
  Border<FMT> B = load_border<FMT>(F, row + 1);     // the record of `row`, rows 0..row%64
  const uint32_t off = row & 63;
  uint32_t c = (uint32_t)((B.plane(0) >> off) & 1) | ((uint32_t)((B.plane(1) >> off) & 1) << 1) |
               ((uint32_t)((B.plane(2) >> off) & 1) << 2);
  if (FMT == OCC_WIDE) c |= (uint32_t)((B.plane(3) >> off) & 1) << 3;
  B.low >>= 1;                                         // rows before `row` only
  B.i = row;
  code = c;
  uint32_t r;
  if (FMT == OCC_WIDE) {
    uint64_t m = B.low & ((c & 1) ? B.plane(0) : ~B.plane(0)) & ((c & 2) ? B.plane(1) : ~B.plane(1)) &
                 ((c & 4) ? B.plane(2) : ~B.plane(2)) & ((c & 8) ? B.plane(3) : ~B.plane(3));
    const uint4 w = c < 4 ? B.a : c < 8 ? B.b : c < 12 ? B.c : B.d;
    r = sel4(w, c & 3) + (uint32_t)__popcll(m);
  } else if (c == 0) {
    r = border_rank<FMT>(F, B, 0);
  } else {
    uint64_t m = B.low & ((c & 1) ? B.plane(0) : ~B.plane(0)) & ((c & 2) ? B.plane(1) : ~B.plane(1)) &
                 ((c & 4) ? B.plane(2) : ~B.plane(2));
    uint32_t w = c <= 2 ? B.a.x : B.a.y;
    r = sb_count(F, B.sbi, c) + (((c - 1) & 1) ? (w >> 16) : (w & 0xFFFFu)) + (uint32_t)__popcll(m);
  }
  rank = r;
}

// Rank of every symbol code at border i (counts of code s in bwt[0..i)), absent codes 0.
// Used by the backward search and the warp-per-read kernels.
template <uint32_t FMT>
__device__ __forceinline__ void sym_ranks_t(const DevFm& F, uint32_t i, uint32_t r[16]) {
  const Border<FMT> B = load_border<FMT>(F, i);
  if (FMT == OCC_NARROW) {
    uint32_t t = 0;
#pragma unroll
    for (int s = 1; s <= 4; s++) { r[s] = sb_count(F, B.sbi, s) + B.local(s); t += r[s]; }
    r[0] = i - t;
#pragma unroll
    for (int s = 5; s < 16; s++) r[s] = 0;
  } else {
#pragma unroll
    for (int s = 0; s < 16; s++) r[s] = B.local(s);
  }
}

__device__ __forceinline__ void sym_ranks(const DevFm& F, const SmemFm& S, uint32_t i, uint32_t r[16]) {
  (void)S;
  if (F.fmt == OCC_NARROW) sym_ranks_t<OCC_NARROW>(F, i, r);
  else sym_ranks_t<OCC_WIDE>(F, i, r);
}

// One LF step with the sampled-SA test (FmIndex::resolve_sa loop body,
// src/fm_index/query.rs:282-291; lf_step src/occ/mod.rs:456-480).  Returns true with
// *val = SA value when row `pos` is sampled; otherwise advances pos = LF(pos).
template <uint32_t FMT>
__device__ __forceinline__ bool lf_or_sample_t(const DevFm& F, const SmemFm& S, uint32_t& pos, uint32_t& val) {
  const uint32_t blk = pos >> 6, off = pos & 63;
  uint4 w = __ldg(F.ssa + blk);
  uint32_t code, rank;
  row_code_rank<FMT>(F, pos, code, rank);            // issued before the sampled test: overlaps its latency
  uint64_t word = u2to64(w.x, w.y);
  if ((word >> off) & 1ull) {
    val = __ldg(F.sa_vals + w.z + (uint32_t)__popcll(word & ((1ull << off) - 1ull)));
    return true;
  }
  pos = S.C[code] + rank;
  return false;
}

__device__ __forceinline__ bool lf_or_sample(const DevFm& F, const SmemFm& S, uint32_t& pos, uint32_t& val) {
  if (F.fmt == OCC_NARROW) return lf_or_sample_t<OCC_NARROW>(F, S, pos, val);
  return lf_or_sample_t<OCC_WIDE>(F, S, pos, val);
}

// partition_point(bounds, b <= p): first index with bounds[idx] > p.
__device__ __forceinline__ uint32_t upper_bound_u32(const uint32_t* b, uint32_t n, uint32_t p) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) { uint32_t mid = (lo + hi) >> 1; if (b[mid] <= p) lo = mid + 1; else hi = mid; }
  return lo;
}

}  // namespace hfm
