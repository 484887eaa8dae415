// search.cuh — per-read search kernels: IUPAC backward search (count / locate
// intervals) and the bidirectional SMEM / MEM candidate search.
//
// Execution model: persistent grids (one wave of resident threads) pull reads from a
// device work queue; one thread owns one read at a time.  A read's path is a chain of
// ~|read| dependent rank steps, so throughput comes from keeping ~10^5 reads in flight,
// not from spreading one read over a warp.  Interval sets live in per-thread slices of a
// global work area, interleaved across the 32 lanes of a warp (element i of every lane is
// one contiguous run: 128 B per u32 plane of the SMEM sets, 256 B per uint2 of the backward
// search sets) with a fixed capacity; a read whose set, candidate list or output outgrows
// it is queued for a fallback pass with much larger slices (a per-thread rerun for long
// candidate lists, then one warp per read).  There is therefore no cap on interval-set
// size, as in the reference CPU (src/fm_index/query.rs:248-274,
// src/fm_index/smem.rs:332-357).  SMEM reads longer than 2 * seg_len are swept in
// segments whose pivot chains are merged (below), so no single read is a long serial chain.
#pragma once
#include <type_traits>
#include "dev_index.cuh"

namespace hfm {

// Interval-set capacity of the per-thread SMEM kernels (warp-interleaved sets, STRIDE 32).
constexpr uint32_t FAST_SET_CAP = 768;

// Results are bump-allocated in pools; per-read (offset, count) record where they went.
struct Pool {
  void* base;
  unsigned long long* used;   // device counter (elements)
  uint64_t cap;               // elements
};

__device__ __forceinline__ uint64_t thread_reserve(Pool& p, uint32_t n) {
  if (n == 0) return 0;
  unsigned long long off = atomicAdd(p.used, (unsigned long long)n);
  return (off + n <= p.cap) ? off : ~0ull;
}

// Status bits per read.
enum : uint32_t { ST_OK = 0, ST_SET_OVF = 1, ST_CAND_OVF = 2, ST_POOL_OVF = 4 };

// A thread's interval set: element i at p[i * STRIDE].
template <class T, int STRIDE>
struct SetRef {
  T* p;
  __device__ __forceinline__ T& operator[](uint32_t i) const { return p[(size_t)i * STRIDE]; }
};

// Interval sets of the SMEM path store a bidirectional interval as three u32 planes
// (flo, rlo, size): fhi - flo == rhi - rlo always holds, so 12 bytes carry the 16 of a BIv
// and the sets' traffic (most DRAM writes of the search) drops by a quarter.  Single-row
// intervals (the front list of a TwoList) store only (flo, rlo): their size is 1.
template <int STRIDE>
struct SetRef<BIv, STRIDE> {
  uint32_t* p;          // this thread's slot: field f of element i at p[(f * cap + i) * STRIDE]
  uint32_t plane_;      // cap * STRIDE (warp-interleaved sets: always FAST_SET_CAP * 32)
  __device__ __forceinline__ uint32_t pl() const { return STRIDE == 32 ? FAST_SET_CAP * 32 : plane_; }
  struct Ref {
    uint32_t* a; uint32_t plane;
    __device__ __forceinline__ operator BIv() const {
      uint32_t f = a[0], r = a[plane], z = a[2 * plane];
      return BIv{f, f + z, r, r + z};
    }
    __device__ __forceinline__ Ref& operator=(const BIv& v) {
      a[0] = v.flo; a[plane] = v.rlo; a[2 * plane] = v.fhi - v.flo;
      return *this;
    }
  };
  __device__ __forceinline__ Ref operator[](uint32_t i) const { return Ref{p + (size_t)i * STRIDE, pl()}; }
  __device__ __forceinline__ BIv single(uint32_t i) const {
    const uint32_t* a = p + (size_t)i * STRIDE;
    uint32_t f = a[0], r = a[pl()];
    return BIv{f, f + 1, r, r + 1};
  }
  __device__ __forceinline__ void set_single(uint32_t i, uint32_t flo, uint32_t rlo) const {
    uint32_t* a = p + (size_t)i * STRIDE;
    a[0] = flo; a[pl()] = rlo;
  }
};

// Set s (of NS) of the calling thread inside `work`, `cap` elements each.
// STRIDE 32: warp-interleaved slices (fast path); STRIDE 1: contiguous per-thread slices.
template <class T, int STRIDE>
__device__ __forceinline__ SetRef<T, STRIDE> thread_set(T* work, uint32_t cap, int NS, int s) {
  uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (std::is_same<T, BIv>::value) {
    uint32_t* w = reinterpret_cast<uint32_t*>(work);           // 3 planes of cap u32 per set
    if (STRIDE == 32) {
      uint64_t warp = tid >> 5, lane = tid & 31;
      return SetRef<T, STRIDE>{w + ((warp * NS + s) * cap * 3) * 32 + lane, cap * STRIDE};
    }
    return SetRef<T, STRIDE>{w + (tid * NS + s) * cap * 3, cap * STRIDE};
  } else {
    if (STRIDE == 32) {
      uint64_t warp = tid >> 5, lane = tid & 31;
      return SetRef<T, STRIDE>{work + ((warp * NS + s) * cap) * 32 + lane};
    }
    return SetRef<T, STRIDE>{work + (tid * NS + s) * cap};
  }
}

// Next read from the device queue: reads are ids[k] (or k itself when ids is null).
__device__ __forceinline__ bool next_read(unsigned int* ctr, uint32_t n, const uint32_t* ids, uint32_t& i) {
  uint32_t k = atomicAdd(ctr, 1u);
  if (k >= n) return false;
  i = ids ? ids[k] : k;
  return true;
}

// The same queue taken `chunk` consecutive entries per atomic: the thread works through its
// chunk before it takes the next one (a tunable; 1 = one entry per atomic).
struct QueueCursor { uint32_t next = 0, end = 0; };
__device__ __forceinline__ bool next_read_chunked(unsigned int* ctr, uint32_t n, const uint32_t* ids, uint32_t chunk,
                                                  QueueCursor& c, uint32_t& i) {
  if (c.next >= c.end) {
    const uint32_t k = atomicAdd(ctr, chunk);
    if (k >= n) return false;
    c.next = k;
    c.end = min(n, k + chunk);
  }
  const uint32_t k = c.next++;
  i = ids ? ids[k] : k;
  return true;
}

// =====================================================================================
// Backward search (FmIndex::backward_search, src/fm_index/query.rs:219-277)
// =====================================================================================

// Insert a non-empty interval into a sorted, coalesced set (the effect of
// merge_intervals_inplace, src/fm_index/query.rs:390-407, applied incrementally).
template <class SR>
__device__ __forceinline__ bool iv_insert(const SR& a, uint32_t& n, uint32_t cap, uint32_t lo, uint32_t hi) {
  uint32_t j = n;
  while (j > 0 && a[j - 1].x > lo) j--;
  if (j > 0 && a[j - 1].y >= lo) { j--; lo = a[j].x; hi = max(hi, a[j].y); }
  uint32_t e = j;
  while (e < n && a[e].x <= hi) { hi = max(hi, a[e].y); e++; }
  uint32_t removed = e - j;
  if (removed == 0) {
    if (n >= cap) return false;
    for (uint32_t k = n; k > j; k--) a[k] = a[k - 1];
    n++;
  } else if (removed > 1) {
    for (uint32_t k = e; k < n; k++) a[k - removed + 1] = a[k];
    n -= removed - 1;
  }
  a[j] = make_uint2(lo, hi);
  return true;
}

struct BsOut {
  uint32_t* counts;      // exact count per query
  uint64_t* nhits;       // sum of min(size, cap) per query (nullptr: count only)
  uint32_t* niv;         // intervals per query
  uint64_t* ivoff;       // pool offset of the intervals
  uint32_t* status;      // per-query status bits
  uint32_t* ovf_list;    // queries to re-run with large sets
  uint32_t* n_ovf;
  unsigned long long* touches;  // Occ record touches (counted only with COUNT_TOUCH)
};

// Returns the final number of intervals in cur (0 = no match), or ~0u on set overflow.
template <bool COUNT_TOUCH, class SR>
__device__ __forceinline__ uint32_t backward_search_one(const DevFm& F, const SmemFm& S, const uint8_t* p,
                                                        uint32_t m, SR& cur, SR& nxt, uint32_t cap,
                                                        uint64_t& touches) {
  cur[0] = make_uint2(0, F.text_len);
  if (m == 0) return 1;
  uint32_t n = 1, start = m;
  if (F.lut && m >= F.lut_depth) {
    // LookupTable::get (src/fm_index/lookup.rs:101-111): rightmost code is the most
    // significant digit of the base-radix index.
    uint64_t idx = 0; bool ok = true;
    for (int k = (int)F.lut_depth - 1; k >= 0; --k) {
      uint8_t c = p[m - F.lut_depth + k];
      uint32_t d = c < 16 ? S.dig[c] : 0xFF;
      if (d == 0xFF) { ok = false; break; }
      idx = idx * F.lut_radix + d;
    }
    if (ok) {
      uint2 iv = __ldg(F.lut + idx);
      if (COUNT_TOUCH) touches++;
      if (iv.x >= iv.y) return 0;
      cur[0] = iv; start = m - F.lut_depth;
    }
  }
  for (uint32_t k = start; k-- > 0;) {
    uint8_t c = p[k];
    uint32_t mask = c < 16 ? S.compat_mask[c] : 0;
    mask &= F.sym_mask;                   // symbol_count(r) == 0 -> skipped
    if (!mask) return 0;
    uint32_t nn = 0;
    if (n == 1) {
      // one source interval: symbol order is already ascending row order
      uint2 iv = cur[0];
      uint32_t rl[16], rh[16];
      sym_ranks(F, S, iv.x, rl);
      sym_ranks(F, S, iv.y, rh);
      if (COUNT_TOUCH) touches += (iv.x != 0) + (iv.y != 0);
#pragma unroll
      for (int r = 0; r < 16; r++) {
        if (!((mask >> r) & 1)) continue;
        uint32_t nl = S.C[r] + rl[r], nh = S.C[r] + rh[r];
        if (nl < nh && !iv_insert(nxt, nn, cap, nl, nh)) return ~0u;
      }
    } else {
      // Outputs for symbol r lie in [C[r], C[r+1]) in source order, so a stable counting
      // sort by symbol yields ascending rows: count per symbol, then place.
      uint32_t cnt[16];
#pragma unroll
      for (int r = 0; r < 16; r++) cnt[r] = 0;
      for (uint32_t i = 0; i < n; i++) {
        uint2 iv = cur[i];
        uint32_t rl[16], rh[16];
        sym_ranks(F, S, iv.x, rl);
        sym_ranks(F, S, iv.y, rh);
        if (COUNT_TOUCH) touches += (iv.x != 0) + (iv.y != 0);
#pragma unroll
        for (int r = 0; r < 16; r++) cnt[r] += (((mask >> r) & 1) && rh[r] > rl[r]) ? 1u : 0u;
      }
      uint32_t total = 0;
#pragma unroll
      for (int r = 0; r < 16; r++) { uint32_t t = cnt[r]; cnt[r] = total; total += t; }
      if (total > cap) return ~0u;
      for (uint32_t i = 0; i < n; i++) {
        uint2 iv = cur[i];
        uint32_t rl[16], rh[16];
        sym_ranks(F, S, iv.x, rl);
        sym_ranks(F, S, iv.y, rh);
#pragma unroll
        for (int r = 0; r < 16; r++)
          if (((mask >> r) & 1) && rh[r] > rl[r]) nxt[cnt[r]++] = make_uint2(S.C[r] + rl[r], S.C[r] + rh[r]);
      }
      // coalesce touching neighbours (merge_intervals_inplace, query.rs:390-407)
      for (uint32_t e = 0; e < total; e++) {
        uint2 v = nxt[e];
        if (nn > 0) {
          uint2 last = nxt[nn - 1];
          if (v.x <= last.y) { nxt[nn - 1] = make_uint2(last.x, max(last.y, v.y)); continue; }
        }
        nxt[nn++] = v;
      }
    }
    if (nn == 0) return 0;
    SR t = cur; cur = nxt; nxt = t; n = nn;
  }
  return n;
}

// Persistent backward search.  ids == nullptr: every query 0..n-1; otherwise the listed
// queries (fallback pass; reads that overflow there bump *still_ovf).
template <bool COUNT_TOUCH, int STRIDE>
__global__ void __launch_bounds__(256) k_bsearch(DevFm F, const uint16_t* __restrict__ compat_masks,
                                                const uint8_t* __restrict__ q, const uint64_t* __restrict__ qoff,
                                                const uint32_t* __restrict__ ids, uint32_t n, uint32_t hit_cap,
                                                uint2* work, uint32_t set_cap, unsigned int* queue, Pool pool,
                                                BsOut out, uint32_t* still_ovf) {
  __shared__ SmemFm S;
  smem_fm_init(S, F, compat_masks);
  __syncthreads();
  SetRef<uint2, STRIDE> A = thread_set<uint2, STRIDE>(work, set_cap, 2, 0);
  SetRef<uint2, STRIDE> B = thread_set<uint2, STRIDE>(work, set_cap, 2, 1);
  uint64_t touches = 0;
  uint32_t i;
  while (next_read(queue, n, ids, i)) {
    SetRef<uint2, STRIDE> cur = A, nxt = B;
    uint64_t o = qoff[i];
    uint32_t niv = backward_search_one<COUNT_TOUCH>(F, S, q + o, (uint32_t)(qoff[i + 1] - o), cur, nxt, set_cap,
                                                    touches);
    uint32_t st = ST_OK;
    if (niv == ~0u) { st = ST_SET_OVF; niv = 0; }
    uint32_t cnt = 0; uint64_t hits = 0;
    for (uint32_t k = 0; k < niv; k++) {
      uint2 v = cur[k];
      uint32_t sz = v.y - v.x;
      cnt += sz; hits += (hit_cap && sz > hit_cap) ? hit_cap : sz;
    }
    uint64_t off = 0;
    if (out.nhits && niv) {
      off = thread_reserve(pool, niv);
      if (off == ~0ull) st |= ST_POOL_OVF;
      else { uint2* dst = (uint2*)pool.base + off; for (uint32_t k = 0; k < niv; k++) dst[k] = cur[k]; }
    }
    out.counts[i] = cnt;
    if (out.nhits) { out.nhits[i] = hits; out.niv[i] = niv; out.ivoff[i] = off; }
    out.status[i] = st;
    if (st & ST_SET_OVF) {
      if (ids) atomicAdd(still_ovf, 1u);
      else out.ovf_list[atomicAdd(out.n_ovf, 1u)] = i;
    }
  }
  if (COUNT_TOUCH && touches) atomicAdd(out.touches, (unsigned long long)touches);
}

// =====================================================================================
// Bidirectional extension (BidirInterval::extend_right / extend_left,
// src/fm_index/bidir.rs:80-143) over a whole interval set (extend_multi_right/left,
// src/fm_index/smem.rs:332-357).  The set is emitted interval-major (the reference emits
// base-major); set order never changes which strings are found, and MEM hits are
// emitted in ascending fwd_lo order at the end.
// =====================================================================================

// A thread's interval set is kept as two lists in one slice of `cap` entries: intervals
// of one row from the front ([0, n1)) and larger ones from the back ([cap-nb, cap)).  A
// one-row interval extends only by the symbol of its row — one LF step on one record —
// so every lane runs a cheap uniform loop over its singles, then the full 16-symbol rank
// loop over the rest, instead of branching per interval (which diverges within a warp).
template <class SR>
struct TwoList {
  SR s; uint32_t n1, nb;
  __device__ __forceinline__ uint32_t size() const { return n1 + nb; }
};

// DIR 0 = right (ranks on the reverse index), 1 = left (ranks on the forward index).
template <int DIR, bool COUNT_TOUCH, uint32_t FMT, class SR>
__device__ __forceinline__ void extend_set(const DevFm& X, const SmemFm& S, uint32_t mask, const TwoList<SR>& in,
                                           TwoList<SR>& out, uint32_t cap, uint32_t& cov, bool& ovf,
                                           uint64_t& touches) {
  out.n1 = 0; out.nb = 0; cov = 0;
  const uint32_t top = mask ? 31u - __clz(mask) : 0u;     // highest code that can extend
  for (uint32_t i = 0; i < in.n1; i++) {
    BIv iv = in.s.single(i);
    uint32_t a = DIR == 0 ? iv.rlo : iv.flo, base = DIR == 0 ? iv.flo : iv.rlo;
    uint32_t s0, rk;
    row_code_rank<FMT>(X, a, s0, rk);
    if (COUNT_TOUCH) touches += 1;
    if ((mask >> s0) & 1) {
      if (out.n1 + out.nb >= cap) { ovf = true; return; }
      if (DIR == 0) out.s.set_single(out.n1++, base, S.C[s0] + rk);
      else out.s.set_single(out.n1++, S.C[s0] + rk, base);
      cov += 1;
    }
  }
  for (uint32_t k = 0; k < in.nb; k++) {
    BIv iv = in.s[cap - 1 - k];
    uint32_t a = DIR == 0 ? iv.rlo : iv.flo, b = DIR == 0 ? iv.rhi : iv.fhi;
    uint32_t base = DIR == 0 ? iv.flo : iv.rlo;
    if (COUNT_TOUCH) touches += (a != 0) + (b != 0);
    uint32_t run = 0;
    // count_smaller_than (src/fm_index/bidir.rs:125-143): the new interval of symbol s on
    // the other strand starts after every code below s, $ included
    split_by_symbol<FMT>(X, a, b, top, [&](int s, uint32_t d, uint32_t r, uint32_t sbi) {
      if (!ovf && ((mask >> s) & 1) && d) {
        if (out.n1 + out.nb >= cap) { ovf = true; return; }
        const uint32_t lo = S.C[s] + (FMT == OCC_WIDE ? r : sb_count(X, sbi, s) + r);
        if (d == 1) {
          if (DIR == 0) out.s.set_single(out.n1++, base + run, lo);
          else out.s.set_single(out.n1++, lo, base + run);
        } else {
          BIv e;
          if (DIR == 0) { e.flo = base + run; e.fhi = base + run + d; e.rlo = lo; e.rhi = lo + d; }
          else { e.flo = lo; e.fhi = lo + d; e.rlo = base + run; e.rhi = base + run + d; }
          out.s[cap - 1 - out.nb++] = e;
        }
        cov += d;
      }
      run += d;
    });
    if (ovf) return;
  }
}

// Does any interval of the set extend by a compatible symbol?
template <int DIR, bool COUNT_TOUCH, uint32_t FMT, class SR>
__device__ __forceinline__ bool any_extend(const DevFm& X, const SmemFm& S, uint32_t mask, const TwoList<SR>& in,
                                           uint32_t cap, uint64_t& touches) {
  bool any = false;
  const uint32_t top = mask ? 31u - __clz(mask) : 0u;
  for (uint32_t i = 0; i < in.n1; i++) {
    BIv iv = in.s.single(i);
    uint32_t s0, rk;
    row_code_rank<FMT>(X, DIR == 0 ? iv.rlo : iv.flo, s0, rk);
    if (COUNT_TOUCH) touches += 1;
    any |= (mask >> s0) & 1;
  }
  if (any) return true;
  for (uint32_t k = 0; k < in.nb; k++) {
    BIv iv = in.s[cap - 1 - k];
    uint32_t a = DIR == 0 ? iv.rlo : iv.flo, b = DIR == 0 ? iv.rhi : iv.fhi;
    if (COUNT_TOUCH) touches += (a != 0) + (b != 0);
    split_by_symbol<FMT>(X, a, b, top, [&](int s, uint32_t d, uint32_t, uint32_t) { any |= ((mask >> s) & 1) && d; });
    if (any) return true;
  }
  return false;
}

struct Cand { uint32_t qs, qe, count, nivs; uint64_t ivoff; uint32_t pivot, _pad; };

struct MemsOut {
  uint64_t* hit_start;      // per read: offset of its hits in the hit pool
  uint32_t* hit_count;      // per read: number of hits
  uint32_t* status;
  uint32_t* ovf_list;
  uint32_t* n_ovf;
  unsigned long long* touches;
};

struct MemsParams {
  uint32_t min_len, mode, max_hits, resolve;   // resolve = ref bounds given
};

// Shell sort of a set by fwd_lo (hits of one MEM in ascending fwd_lo order).
__device__ __forceinline__ void sort_by_flo(BIv* a, uint32_t n) {
  for (uint32_t gap = n / 2; gap > 0; gap /= 2)
    for (uint32_t i = gap; i < n; i++) {
      BIv t = a[i]; uint32_t j = i;
      while (j >= gap && a[j - gap].flo > t.flo) { a[j] = a[j - gap]; j -= gap; }
      a[j] = t;
    }
}

// The full interval (the empty pattern) as a one-element two-list set.
template <class SR>
__device__ __forceinline__ void start_full(TwoList<SR>& t, const BIv& full, uint32_t set_cap) {
  if (full.fhi - full.flo == 1) { t.s.set_single(0, full.flo, full.rlo); t.n1 = 1; t.nb = 0; }
  else { t.s[set_cap - 1] = full; t.n1 = 0; t.nb = 1; }
}

__device__ __forceinline__ uint32_t qmask(const SmemFm& S, uint8_t c) { return c < 16 ? S.compat_mask[c] : 0u; }

// One pivot of the SMEM sweep (collect_smem_candidates loop body,
// src/fm_index/smem.rs:154-222): forward extension from `pivot`, every right-maximal prefix
// extended left maximally (extend_left_maximally, smem.rs:227-243), candidates passed to
// emit(qs, qe, count, set, pivot).  Returns the next pivot, max(reach, pivot + 1), or ~0u
// on overflow (flags in st).  The sweep is a chain pivot -> next(pivot) that depends only
// on the read, which is what lets a long read be cut into independently swept segments.
template <bool COUNT_TOUCH, uint32_t FMT, class SR, class Emit>
__device__ __forceinline__ uint32_t smem_pivot(const DevFm& Fw, const DevFm& Rv, const SmemFm& Sf, const SmemFm& Sr,
                                               const uint8_t* q, uint32_t n, uint32_t pivot, const MemsParams& P,
                                               const SR& curr, const SR& nxt, const SR& wa, const SR& wb,
                                               uint32_t set_cap, uint32_t& st, uint64_t& touches, Emit& emit) {
  using TL = TwoList<SR>;
  const BIv full = {0, Fw.text_len, 0, Fw.text_len};
  bool ovf = false;
  TL c{curr, 0, 0}, x{nxt, 0, 0};
  start_full(x, full, set_cap);
  uint32_t cov;
  extend_set<0, COUNT_TOUCH, FMT>(Rv, Sr, qmask(Sr, q[pivot]), x, c, set_cap, cov, ovf, touches);
  if (ovf) { st |= ST_SET_OVF; return ~0u; }
  if (c.size() == 0) return pivot + 1;
  uint32_t j = pivot + 1, reach = pivot + 1;
  for (;;) {
    uint32_t end, ncov = 0;
    bool next_empty, record;
    x.n1 = x.nb = 0;
    if (j == n) { end = n; next_empty = true; record = true; }
    else {
      extend_set<0, COUNT_TOUCH, FMT>(Rv, Sr, qmask(Sr, q[j]), c, x, set_cap, ncov, ovf, touches);
      if (ovf) { st |= ST_SET_OVF; return ~0u; }
      end = j; next_empty = x.size() == 0; record = ncov != cov;
    }
    if (record) {
      // right-maximal prefix [pivot, end): extend_left_maximally (smem.rs:227-243)
      reach = end;
      TL b = c;
      uint32_t start = pivot, bcov = cov;
      TL bufs[2] = {TL{wa, 0, 0}, TL{wb, 0, 0}};
      int t = 0;
      while (start > 0) {
        uint32_t lcov;
        extend_set<1, COUNT_TOUCH, FMT>(Fw, Sf, qmask(Sf, q[start - 1]), b, bufs[t], set_cap, lcov, ovf, touches);
        if (ovf) { st |= ST_SET_OVF; return ~0u; }
        if (bufs[t].size() == 0) break;
        b = bufs[t]; bcov = lcov; t ^= 1; start--;
      }
      if (end - start >= P.min_len) {
        // right-maximality (smem.rs:202-207); with no left extension it is next_empty
        bool rmax = end == n ||
                    (start == pivot ? next_empty : !any_extend<0, COUNT_TOUCH, FMT>(Rv, Sr, qmask(Sr, q[end]), b, set_cap, touches));
        if (rmax && !emit(start, end, bcov, b, pivot)) return ~0u;
      }
    }
    if (j == n || x.size() == 0) break;
    TL tt = c; c = x; x = tt; cov = ncov; j++;
  }
  return max(reach, pivot + 1);
}

// Appends candidates (with their interval sets copied to the interval pool) to a list.
template <class SR>
struct CandSink {
  Cand* cands; uint32_t nc, cap; Pool* ivpool; uint32_t* st; uint32_t set_cap;
  __device__ __forceinline__ bool operator()(uint32_t qs, uint32_t qe, uint32_t count, const TwoList<SR>& ivs,
                                             uint32_t pivot) {
    if (nc >= cap) { *st |= ST_CAND_OVF; return false; }
    uint32_t niv = ivs.size();
    uint64_t off = thread_reserve(*ivpool, niv);
    if (off == ~0ull) { *st |= ST_POOL_OVF; return false; }
    BIv* dst = (BIv*)ivpool->base + off;
    for (uint32_t k = 0; k < ivs.n1; k++) dst[k] = ivs.s.single(k);
    for (uint32_t k = 0; k < ivs.nb; k++) dst[ivs.n1 + k] = ivs.s[set_cap - 1 - k];
    cands[nc++] = Cand{qs, qe, count, niv, off, pivot, 0u};
    return true;
  }
};

// Candidate search for one read into `sink` (find_mems or find_smems candidates).  Returns
// the number of candidates, or ~0u on overflow of a set, the candidate list or the
// interval pool (flags in st).
template <bool COUNT_TOUCH, uint32_t FMT, class SR, class Sink>
__device__ uint32_t mems_sweep(const DevFm& Fw, const DevFm& Rv, const SmemFm& Sf, const SmemFm& Sr,
                               const uint8_t* q, uint32_t n, const MemsParams& P, const SR& curr, const SR& nxt,
                               const SR& wa, const SR& wb, uint32_t set_cap, Sink& sink, uint32_t& st,
                               uint64_t& touches) {
  using TL = TwoList<SR>;
  if (n == 0 || P.min_len == 0) return 0;
  const BIv full = {0, Fw.text_len, 0, Fw.text_len};
  bool ovf = false;
  if (P.mode == 1) {
    // find_mems: raw_mem_from(i) for every start (src/fm_index/smem.rs:250-295)
    for (uint32_t i = 0; i < n; i++) {
      TL c{curr, 0, 0}, x{nxt, 0, 0};
      start_full(c, full, set_cap);
      uint32_t cov = 0, j = i;
      bool matched = false;
      while (j < n) {
        uint32_t ncov;
        extend_set<0, COUNT_TOUCH, FMT>(Rv, Sr, qmask(Sr, q[j]), c, x, set_cap, ncov, ovf, touches);
        if (ovf) { st |= ST_SET_OVF; return ~0u; }
        if (x.size() == 0) break;
        TL t = c; c = x; x = t; cov = ncov; j++; matched = true;
      }
      if (!matched || j - i < P.min_len) continue;
      bool lmax = i == 0 || !any_extend<1, COUNT_TOUCH, FMT>(Fw, Sf, qmask(Sf, q[i - 1]), c, set_cap, touches);
      if (!lmax) continue;
      if (!sink(i, j, cov, c, i)) return ~0u;
    }
    return sink.nc;
  }
  // find_smems: collect_smem_candidates (src/fm_index/smem.rs:154-222)
  uint32_t pivot = 0;
  while (pivot < n) {
    pivot = smem_pivot<COUNT_TOUCH, FMT>(Fw, Rv, Sf, Sr, q, n, pivot, P, curr, nxt, wa, wb, set_cap, st, touches, sink);
    if (pivot == ~0u) return ~0u;
  }
  return sink.nc;
}

template <bool COUNT_TOUCH, uint32_t FMT, class SR>
__device__ uint32_t mems_one(const DevFm& Fw, const DevFm& Rv, const SmemFm& Sf, const SmemFm& Sr,
                             const uint8_t* q, uint32_t n, const MemsParams& P, const SR& curr, const SR& nxt,
                             const SR& wa, const SR& wb, uint32_t set_cap, Cand* cands, uint32_t cand_cap,
                             Pool& ivpool, uint32_t& st, uint64_t& touches) {
  CandSink<SR> sink{cands, 0, cand_cap, &ivpool, &st, set_cap};
  return mems_sweep<COUNT_TOUCH, FMT>(Fw, Rv, Sf, Sr, q, n, P, curr, nxt, wa, wb, set_cap, sink, st, touches);
}

// Sort candidates by (qs, qe) (stable), drop duplicates, keep the containment-maximal ones
// (find_smems, src/fm_index/smem.rs:84-103).  Returns the survivors compacted in place.
template <bool LONG_LISTS = false>
__device__ __forceinline__ uint32_t finalize_smems(Cand* c, uint32_t n) {
  if (LONG_LISTS && n > 128) {
    // Shell sort (Ciura's gaps) for the long lists of long reads.  Candidates with equal
    // (qs, qe) name the same pattern, so the same count and interval set: which of them
    // the dedup below keeps does not matter, and the sort need not be stable.
    const uint32_t gaps[8] = {701, 301, 132, 57, 23, 10, 4, 1};
    for (int gi = 0; gi < 8; gi++) {
      uint32_t g = gaps[gi];
      if (g >= n) continue;
      for (uint32_t i = g; i < n; i++) {
        Cand t = c[i];
        uint64_t k = ((uint64_t)t.qs << 32) | t.qe;
        uint32_t j = i;
        while (j >= g && ((((uint64_t)c[j - g].qs) << 32) | c[j - g].qe) > k) { c[j] = c[j - g]; j -= g; }
        c[j] = t;
      }
    }
  } else {
    for (uint32_t i = 1; i < n; i++) {         // insertion sort
      Cand t = c[i]; uint32_t j = i;
      while (j > 0 && (c[j - 1].qs > t.qs || (c[j - 1].qs == t.qs && c[j - 1].qe > t.qe))) { c[j] = c[j - 1]; j--; }
      c[j] = t;
    }
  }
  uint32_t w = 0;
  for (uint32_t i = 0; i < n; i++)
    if (w == 0 || c[w - 1].qs != c[i].qs || c[w - 1].qe != c[i].qe) c[w++] = c[i];
  n = w; w = 0;
  // Sorted by (qs, qe) and distinct, c[i] lies inside another candidate exactly when the
  // next one shares its start (and so ends later) or an earlier one (qs <= c[i].qs) ends
  // at or after c[i].qe: a running maximum of qe replaces the all-pairs test.
  uint32_t max_qe = 0;
  bool any = false;
  for (uint32_t i = 0; i < n; i++) {
    bool contained = (i + 1 < n && c[i + 1].qs == c[i].qs) || (any && max_qe >= c[i].qe);
    uint32_t qe = c[i].qe;
    if (!any || qe > max_qe) max_qe = qe;
    any = true;
    if (!contained) c[w++] = c[i];
  }
  return w;
}

// Writes the hits of one read (one per SA interval of each surviving MEM) into the hit
// pool; returns false on pool exhaustion.
__device__ __forceinline__ bool write_hits(Cand* c, uint32_t n, const MemsParams& P, Pool& ivpool,
                                           Pool& hitpool, uint64_t& start, uint32_t& count) {
  uint32_t total = 0;
  for (uint32_t k = 0; k < n; k++) total += c[k].nivs;
  count = total;
  if (total == 0) { start = 0; return true; }
  uint64_t off = thread_reserve(hitpool, total);
  if (off == ~0ull) return false;
  start = off;
  uint32_t* h = (uint32_t*)hitpool.base + off * 8;
  for (uint32_t k = 0; k < n; k++) {
    BIv* ivs = (BIv*)ivpool.base + c[k].ivoff;
    sort_by_flo(ivs, c[k].nivs);
    for (uint32_t t = 0; t < c[k].nivs; t++) {
      uint32_t sz = ivs[t].fhi - ivs[t].flo;
      uint32_t eff = P.resolve ? min(sz, P.max_hits) : 0u;
      uint4 a = make_uint4(c[k].qs, c[k].qe, sz, sz > P.max_hits ? 1u : 0u);
      uint4 b = make_uint4(ivs[t].flo, eff, 0u, 0u);
      reinterpret_cast<uint4*>(h)[0] = a; reinterpret_cast<uint4*>(h)[1] = b;
      h += 8;
    }
  }
  return true;
}

struct MemsWork {
  BIv* sets; uint32_t set_cap;        // 4 sets per thread
  Cand* cands; uint32_t cand_cap;     // contiguous per thread (fallback pass); nullptr: local
  unsigned int* queue;
  const uint32_t* ids; uint32_t n;    // reads to process, in queue order (ids == nullptr: 0..n-1)
  uint32_t* still_ovf;
  uint32_t rerun;                     // 1: a rerun of overflowed reads (counted in still_ovf)
  uint32_t* work_log;                 // COUNT_TOUCH only: 4 u32 per read, [0] += Occ touches, [3] |= 1 on overflow
                                      // (the warp-per-read kernel also sets bit 1)
  const uint32_t* n_dev;              // when set, the number of reads is read here (graph-captured chains)
  uint32_t chunk;                     // queue entries taken per atomic (0 or 1: one)
  __device__ __forceinline__ uint32_t count() const { return n_dev ? *n_dev : n; }
  __device__ __forceinline__ uint32_t step() const { return chunk > 1 ? chunk : 1u; }
};

// Splits the fast pass's overflow list: the first `first_warp` entries (reads a schedule
// routed) and reads whose interval sets overflowed go to the warp-per-read list; reads that
// outgrew only the candidate list go to the per-thread rerun with a larger global list.
__global__ void k_split_ovf(const uint32_t* __restrict__ list, uint32_t n, uint32_t first_warp,
                            const uint32_t* __restrict__ status, uint32_t* __restrict__ mid,
                            uint32_t* __restrict__ n_mid, uint32_t* __restrict__ wrp, uint32_t* __restrict__ n_wrp,
                            const uint32_t* __restrict__ n_dev = nullptr) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (n_dev ? *n_dev : n)) return;
  uint32_t i = list[k];
  if (k < first_warp || (status[i] & ST_SET_OVF)) wrp[atomicAdd(n_wrp, 1u)] = i;
  else mid[atomicAdd(n_mid, 1u)] = i;
}

template <bool COUNT_TOUCH, int STRIDE, int KC, int MINB, uint32_t FMT>
__global__ void __launch_bounds__(128, MINB) k_mems(DevFm Fw, DevFm Rv, const uint16_t* __restrict__ compat_fw,
                                             const uint16_t* __restrict__ compat_rv, const uint8_t* __restrict__ q,
                                             const uint64_t* __restrict__ qoff, MemsParams P, Pool ivpool,
                                             Pool hitpool, MemsOut out, MemsWork W) {
  __shared__ SmemFm Sf, Sr;
  smem_fm_init(Sf, Fw, compat_fw);
  smem_fm_init(Sr, Rv, compat_rv);
  __syncthreads();
  const uint32_t SCAP = STRIDE == 32 ? FAST_SET_CAP : W.set_cap;
  using SR = SetRef<BIv, STRIDE>;
  SR s0 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 0), s1 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 1);
  SR s2 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 2), s3 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 3);
  Cand local_c[KC > 0 ? KC : 1];
  Cand* cands = local_c;
  uint32_t cand_cap = KC;
  if (KC == 0) {
    uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    cands = W.cands + tid * W.cand_cap;
    cand_cap = W.cand_cap;
  }
  uint64_t touches = 0;
  uint32_t i;
  const uint32_t nreads = W.count(), chunk = W.step();
  QueueCursor qc;
  while (next_read_chunked(W.queue, nreads, W.ids, chunk, qc, i)) {
    uint32_t st = ST_OK;
    uint64_t o = qoff[i];
    uint64_t t0 = touches;
    uint32_t nc = mems_one<COUNT_TOUCH, FMT>(Fw, Rv, Sf, Sr, q + o, (uint32_t)(qoff[i + 1] - o), P, s0, s1, s2, s3,
                                        SCAP, cands, cand_cap, ivpool, st, touches);
    uint64_t hs = 0; uint32_t hc = 0;
    if (nc != ~0u) {
      if (P.mode == 0) nc = finalize_smems(cands, nc);
      if (!write_hits(cands, nc, P, ivpool, hitpool, hs, hc)) st |= ST_POOL_OVF;
    }
    if (st) { hs = 0; hc = 0; }
    out.hit_start[i] = hs; out.hit_count[i] = hc; out.status[i] = st;
    bool ovf = st & (ST_SET_OVF | ST_CAND_OVF);
    if (COUNT_TOUCH && W.work_log) {
      W.work_log[4 * (size_t)i] += (uint32_t)(touches - t0);
      if (ovf) W.work_log[4 * (size_t)i + 3] |= 1u;
    }
    if (ovf) {
      if (W.rerun) atomicAdd(W.still_ovf, 1u);
      else out.ovf_list[atomicAdd(out.n_ovf, 1u)] = i;
    }
  }
  if (COUNT_TOUCH && touches) atomicAdd(out.touches, (unsigned long long)touches);
}


// =====================================================================================
// The plain launch: one thread per read over a grid the size of the batch, interval sets
// and candidate list in the thread's local memory, and a count pass before the write pass
// whose totals the host reads back to size the outputs — the structure of the reference's
// GPU search (one invocation per query, count-then-write, host prefix sum;
// shaders/mem_find.wgsl:179-372, src/gpu/mem_find.rs:213-244) restated with the CPU
// semantics.  It is the baseline the persistent path is measured against.  Reads whose
// sets or candidates outgrow the local capacity go to the warp-per-read kernel, so the
// results are those of every other path.
// =====================================================================================
constexpr uint32_t PLAIN_SET_CAP = 64;
constexpr int PLAIN_KC = 32;

// Count-pass sink: candidates with their MemHit count (nivs) and position count (in
// ivoff), no interval copies.
template <class SR>
struct CountSink {
  Cand* cands; uint32_t nc, cap; uint32_t* st; uint32_t set_cap; uint32_t max_hits, resolve;
  unsigned long long ivs_all;       // intervals of every candidate (the write pass's pool need)
  __device__ __forceinline__ bool operator()(uint32_t qs, uint32_t qe, uint32_t count, const TwoList<SR>& ivs,
                                             uint32_t pivot) {
    if (nc >= cap) { *st |= ST_CAND_OVF; return false; }
    uint64_t npos = 0;
    if (resolve) {
      npos = max_hits ? ivs.n1 : 0u;
      for (uint32_t k = 0; k < ivs.nb; k++) {
        BIv iv = ivs.s[set_cap - 1 - k];
        npos += min(iv.fhi - iv.flo, max_hits);
      }
    }
    ivs_all += ivs.size();
    cands[nc++] = Cand{qs, qe, count, ivs.size(), npos, pivot, 0u};
    return true;
  }
};

template <bool COUNT_TOUCH, int PASS, uint32_t FMT>
__global__ void __launch_bounds__(128) k_mems_plain(DevFm Fw, DevFm Rv, const uint16_t* __restrict__ compat_fw,
                                                   const uint16_t* __restrict__ compat_rv, const uint8_t* __restrict__ q,
                                                   const uint64_t* __restrict__ qoff, MemsParams P, uint32_t n,
                                                   Pool ivpool, Pool hitpool, MemsOut out, uint32_t* pos_count,
                                                   unsigned long long* ivs_need) {
  __shared__ SmemFm Sf, Sr;
  smem_fm_init(Sf, Fw, compat_fw);
  smem_fm_init(Sr, Rv, compat_rv);
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  using SR = SetRef<BIv, 1>;
  uint32_t lset[4][3 * PLAIN_SET_CAP];
  SR s0{lset[0], PLAIN_SET_CAP}, s1{lset[1], PLAIN_SET_CAP}, s2{lset[2], PLAIN_SET_CAP}, s3{lset[3], PLAIN_SET_CAP};
  Cand cands[PLAIN_KC];
  uint64_t touches = 0;
  const uint64_t o = qoff[i];
  const uint32_t len = (uint32_t)(qoff[i + 1] - o);
  if (PASS == 0) {
    uint32_t st = ST_OK;
    CountSink<SR> sink{cands, 0, (uint32_t)PLAIN_KC, &st, PLAIN_SET_CAP, P.max_hits, P.resolve, 0ull};
    uint32_t nc = mems_sweep<COUNT_TOUCH, FMT>(Fw, Rv, Sf, Sr, q + o, len, P, s0, s1, s2, s3, PLAIN_SET_CAP, sink, st,
                                               touches);
    uint32_t hits = 0, pos = 0;
    if (nc != ~0u) {
      if (P.mode == 0) nc = finalize_smems(cands, nc);
      for (uint32_t k = 0; k < nc; k++) { hits += cands[k].nivs; pos += (uint32_t)cands[k].ivoff; }
      atomicAdd(ivs_need, sink.ivs_all);
    }
    if (st) { hits = 0; pos = 0; }
    out.hit_count[i] = hits; pos_count[i] = pos; out.status[i] = st;
  } else {
    // reads the count pass found too large for local memory keep their flags; a pool
    // overflow of an earlier attempt is cleared (the host regrew the pools)
    uint32_t st = out.status[i] & (ST_SET_OVF | ST_CAND_OVF);
    uint64_t hs = 0; uint32_t hc = 0;
    if (st == ST_OK) {
      CandSink<SR> sink{cands, 0, (uint32_t)PLAIN_KC, &ivpool, &st, PLAIN_SET_CAP};
      uint32_t nc = mems_sweep<COUNT_TOUCH, FMT>(Fw, Rv, Sf, Sr, q + o, len, P, s0, s1, s2, s3, PLAIN_SET_CAP, sink,
                                                 st, touches);
      if (nc != ~0u) {
        if (P.mode == 0) nc = finalize_smems(cands, nc);
        if (!write_hits(cands, nc, P, ivpool, hitpool, hs, hc)) st |= ST_POOL_OVF;
      }
      if (st) { hs = 0; hc = 0; }
    }
    out.status[i] = st;
    out.hit_start[i] = hs; out.hit_count[i] = hc;
    if (st & (ST_SET_OVF | ST_CAND_OVF)) out.ovf_list[atomicAdd(out.n_ovf, 1u)] = i;
  }
  if (COUNT_TOUCH && touches) atomicAdd(out.touches, (unsigned long long)touches);
}

// =====================================================================================
// Long reads: the SMEM sweep of a read cut into segments.
//
// The sweep visits a chain of pivots, next = max(reach(pivot), pivot + 1), and the next
// pivot depends only on the read and the current pivot.  k_mems_seg gives one thread to
// each seg_len-position segment of a long read and sweeps the chain as if a pivot started
// at the segment's first position, recording the pivots it visits, the first pivot past
// the segment, and its candidates tagged with their pivots.  k_mems_merge follows the
// read's true chain across the segments: where it lands on a pivot the segment visited,
// both chains agree from there to the segment's end, so the segment's candidates from that
// pivot on are exactly the true chain's; elsewhere the merge sweeps the true chain itself
// until it meets the segment's chain or leaves the segment.  The candidate set, and so
// every result, is the one the unsegmented sweep produces; the critical path of a 10 kbp
// read becomes one segment plus the merge instead of the whole read.
// =====================================================================================
constexpr uint32_t SEG_MAX = 4096;   // longest segment (pivot bitmap of SEG_MAX / 32 words)

struct SegWork {
  uint32_t seg_len, seg_words;    // positions per segment (multiple of 32, <= SEG_MAX)
  const uint32_t* unit_read;      // read of each unit (segment)
  const uint32_t* unit_k;         // segment index within its read
  uint32_t n_units;
  uint32_t* bits;                 // seg_words per unit: pivots the segment's chain visited
  uint32_t* exit_pivot;           // per unit: first pivot past the segment, ~0u on failure
  uint32_t* unit_st;              // per unit: status bits of a failed sweep
  uint64_t* cand_off;             // per unit: first candidate in the unit pool
  uint32_t* cand_cnt;             // per unit
  Cand* pool; unsigned long long* pool_used; uint64_t pool_cap;
  const uint32_t* short_ids;      // k_mems_seg also runs these whole reads after the segments
  uint32_t n_short;
  const uint32_t* long_ids;       // merge: long reads, in queue order
  const uint64_t* unit_base;      // merge: first unit of each long read (n_long + 1)
  uint32_t n_long;
  unsigned int* merge_queue;
  unsigned long long* touches;
  // fix-up pass: segment j swept again from the previous segment's exit pivot (the true
  // chain's entry whenever the previous segment's chain met the true one)
  uint32_t* fx_entry;             // entry pivot used, ~0u when not computed
  uint32_t* fx_conv;              // pivot where it met the segment's chain, ~0u if it did not
  uint32_t* fx_exit;              // first pivot past the segment when it did not meet it
  uint64_t* fx_off;               // its own candidates (pivots before fx_conv) in the pool
  uint32_t* fx_cnt;
  // when set (graph-captured chains), the counts are read here: units = *n_units_dev,
  // long reads = *n_long_dev, short reads = n_fast - *n_long_dev
  const uint64_t* n_units_dev;
  const uint64_t* n_long_dev;
  uint32_t n_fast;
  __device__ __forceinline__ uint32_t units() const { return n_units_dev ? (uint32_t)*n_units_dev : n_units; }
  __device__ __forceinline__ uint32_t longs() const { return n_long_dev ? (uint32_t)*n_long_dev : n_long; }
  __device__ __forceinline__ uint32_t shorts() const { return n_long_dev ? n_fast - (uint32_t)*n_long_dev : n_short; }
};

// flags[k] = 1 when read ids[k] (k itself without ids) is longer than min_len.
__global__ void k_long_flags(const uint32_t* __restrict__ ids, uint32_t n, const uint64_t* __restrict__ qoff,
                             uint32_t min_len, uint32_t* __restrict__ flags) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t i = ids ? ids[k] : k;
  flags[k] = (qoff[i + 1] - qoff[i]) > min_len ? 1u : 0u;
}

// Stable split of ids by flag (lpos = exclusive scan of flags).
__global__ void k_split_ids(const uint32_t* __restrict__ ids, uint32_t n, const uint32_t* __restrict__ flags,
                            const uint64_t* __restrict__ lpos, uint32_t* __restrict__ short_ids,
                            uint32_t* __restrict__ long_ids, uint32_t* __restrict__ seg_count,
                            const uint64_t* __restrict__ qoff, uint32_t seg_len) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t i = ids ? ids[k] : k;
  uint32_t l = (uint32_t)lpos[k];
  if (flags[k]) {
    long_ids[l] = i;
    uint32_t len = (uint32_t)(qoff[i + 1] - qoff[i]);
    seg_count[l] = (len + seg_len - 1) / seg_len;
  } else {
    short_ids[k - l] = i;
  }
}

__global__ void k_unit_fill(const uint32_t* __restrict__ long_ids, uint32_t n_long,
                            const uint64_t* __restrict__ unit_base, uint32_t* __restrict__ unit_read,
                            uint32_t* __restrict__ unit_k, const uint64_t* __restrict__ n_long_dev = nullptr) {
  uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= (n_long_dev ? (uint32_t)*n_long_dev : n_long)) return;
  uint64_t b = unit_base[r], e = unit_base[r + 1];
  for (uint64_t u = b; u < e; u++) { unit_read[u] = long_ids[r]; unit_k[u] = (uint32_t)(u - b); }
}

// One persistent queue over the segments of the long reads followed by the whole short
// reads of the batch (the longest jobs first; the short reads fill the tail).
template <bool COUNT_TOUCH, int STRIDE, int MINB, uint32_t FMT>
__global__ void __launch_bounds__(128, MINB) k_mems_seg(DevFm Fw, DevFm Rv, const uint16_t* __restrict__ compat_fw,
                                                 const uint16_t* __restrict__ compat_rv, const uint8_t* __restrict__ q,
                                                 const uint64_t* __restrict__ qoff, MemsParams P, Pool ivpool,
                                                 Pool hitpool, MemsOut out, MemsWork W, SegWork G) {
  __shared__ SmemFm Sf, Sr;
  smem_fm_init(Sf, Fw, compat_fw);
  smem_fm_init(Sr, Rv, compat_rv);
  __syncthreads();
  const uint32_t SCAP = STRIDE == 32 ? FAST_SET_CAP : W.set_cap;
  using SR = SetRef<BIv, STRIDE>;
  SR s0 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 0), s1 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 1);
  SR s2 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 2), s3 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 3);
  uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  Cand* cands = W.cands + tid * W.cand_cap;
  uint64_t touches = 0;
  const uint32_t n_units = G.units();
  const uint32_t njobs = n_units + G.shorts();
  uint32_t u;
  const uint32_t chunk = W.step();
  QueueCursor qc;
  while (next_read_chunked(W.queue, njobs, nullptr, chunk, qc, u)) {
    const bool unit = u < n_units;
    uint32_t i, s, e;
    uint32_t* bits = nullptr;
    if (unit) i = G.unit_read[u];
    else i = G.short_ids[u - n_units];
    uint64_t o = qoff[i];
    uint32_t n = (uint32_t)(qoff[i + 1] - o);
    if (unit) {
      s = G.unit_k[u] * G.seg_len;
      e = min(n, s + G.seg_len);
      bits = G.bits + (size_t)u * G.seg_words;
      for (uint32_t w = 0; w < G.seg_words; w++) bits[w] = 0;
    } else {
      s = 0;
      e = n;
    }
    uint32_t st = ST_OK;
    uint64_t t0 = touches;
    CandSink<SR> sink{cands, 0, W.cand_cap, &ivpool, &st, SCAP};
    uint32_t p = s;
    while (p < e) {
      if (unit) { uint32_t d = p - s; bits[d >> 5] |= 1u << (d & 31); }
      p = smem_pivot<COUNT_TOUCH, FMT>(Fw, Rv, Sf, Sr, q + o, n, p, P, s0, s1, s2, s3, SCAP, st, touches, sink);
      if (p == ~0u) break;
    }
    uint32_t nc = sink.nc;
    if (unit) {
      if (p != ~0u && nc) {
        unsigned long long off = atomicAdd(G.pool_used, (unsigned long long)nc);
        if (off + nc > G.pool_cap) { st |= ST_POOL_OVF; p = ~0u; }
        else {
          for (uint32_t c = 0; c < nc; c++) G.pool[off + c] = cands[c];
          G.cand_off[u] = off;
        }
      }
      if (p == ~0u || nc == 0) G.cand_off[u] = 0;
      G.cand_cnt[u] = p == ~0u ? 0u : nc;
      G.exit_pivot[u] = p;
      G.unit_st[u] = st;
      if (COUNT_TOUCH && W.work_log) atomicAdd(W.work_log + 4 * (size_t)i, (uint32_t)(touches - t0));
    } else {
      // a whole short read: the same sweep as the fast pass, then its hits
      uint64_t hs = 0; uint32_t hc = 0;
      if (p != ~0u) {
        nc = finalize_smems(cands, nc);
        if (!write_hits(cands, nc, P, ivpool, hitpool, hs, hc)) st |= ST_POOL_OVF;
      }
      if (st) { hs = 0; hc = 0; }
      out.hit_start[i] = hs; out.hit_count[i] = hc; out.status[i] = st;
      bool ovf = st & (ST_SET_OVF | ST_CAND_OVF);
      if (COUNT_TOUCH && W.work_log) {
        W.work_log[4 * (size_t)i] += (uint32_t)(touches - t0);
        if (ovf) W.work_log[4 * (size_t)i + 3] |= 1u;
      }
      if (ovf) out.ovf_list[atomicAdd(out.n_ovf, 1u)] = i;
    }
  }
  if (COUNT_TOUCH && touches) atomicAdd(G.touches, (unsigned long long)touches);
}

// Fix-up pass, one thread per segment after the first: sweeps from the previous segment's
// exit pivot until the chain meets this segment's chain (usually within a few pivots), so
// the merge below only has to check that the entry it assumed is the true one.
template <bool COUNT_TOUCH, int STRIDE, int MINB, uint32_t FMT>
__global__ void __launch_bounds__(128, MINB) k_mems_fix(DevFm Fw, DevFm Rv, const uint16_t* __restrict__ compat_fw,
                                                 const uint16_t* __restrict__ compat_rv, const uint8_t* __restrict__ q,
                                                 const uint64_t* __restrict__ qoff, MemsParams P, Pool ivpool,
                                                 MemsWork W, SegWork G) {
  __shared__ SmemFm Sf, Sr;
  smem_fm_init(Sf, Fw, compat_fw);
  smem_fm_init(Sr, Rv, compat_rv);
  __syncthreads();
  const uint32_t SCAP = STRIDE == 32 ? FAST_SET_CAP : W.set_cap;
  using SR = SetRef<BIv, STRIDE>;
  SR s0 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 0), s1 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 1);
  SR s2 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 2), s3 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 3);
  uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  Cand* cands = W.cands + tid * W.cand_cap;
  uint64_t touches = 0;
  uint32_t u;
  const uint32_t n_units = G.units();
  while (next_read(W.queue, n_units, nullptr, u)) {
    uint32_t i = G.unit_read[u], k = G.unit_k[u];
    G.fx_entry[u] = ~0u; G.fx_conv[u] = ~0u; G.fx_exit[u] = ~0u; G.fx_off[u] = 0; G.fx_cnt[u] = 0;
    if (k == 0 || G.exit_pivot[u - 1] == ~0u || G.exit_pivot[u] == ~0u) continue;
    uint64_t o = qoff[i];
    uint32_t n = (uint32_t)(qoff[i + 1] - o);
    uint32_t s = k * G.seg_len, e = min(n, s + G.seg_len);
    uint32_t entry = G.exit_pivot[u - 1];
    if (entry >= e) { G.fx_entry[u] = entry; G.fx_exit[u] = entry; continue; }
    const uint32_t* bits = G.bits + (size_t)u * G.seg_words;
    uint32_t st = ST_OK;
    uint64_t t0 = touches;
    CandSink<SR> sink{cands, 0, W.cand_cap, &ivpool, &st, SCAP};
    uint32_t p = entry;
    while (p < e && !((bits[(p - s) >> 5] >> ((p - s) & 31)) & 1u)) {
      p = smem_pivot<COUNT_TOUCH, FMT>(Fw, Rv, Sf, Sr, q + o, n, p, P, s0, s1, s2, s3, SCAP, st, touches, sink);
      if (p == ~0u) break;
    }
    if (COUNT_TOUCH && W.work_log) atomicAdd(W.work_log + 4 * (size_t)i, (uint32_t)(touches - t0));
    if (p == ~0u) continue;                       // the merge sweeps this segment itself
    uint32_t nc = sink.nc;
    if (nc) {
      unsigned long long off = atomicAdd(G.pool_used, (unsigned long long)nc);
      if (off + nc > G.pool_cap) continue;        // pool exhausted: counted, regrown by the host
      for (uint32_t c = 0; c < nc; c++) G.pool[off + c] = cands[c];
      G.fx_off[u] = off;
      G.fx_cnt[u] = nc;
    }
    if (p < e) { G.fx_conv[u] = p; G.fx_exit[u] = G.exit_pivot[u]; }
    else G.fx_exit[u] = p;
    G.fx_entry[u] = entry;
  }
  if (COUNT_TOUCH && touches) atomicAdd(G.touches, (unsigned long long)touches);
}

template <bool COUNT_TOUCH, int STRIDE, int MINB, uint32_t FMT>
__global__ void __launch_bounds__(128, MINB) k_mems_merge(DevFm Fw, DevFm Rv, const uint16_t* __restrict__ compat_fw,
                                                   const uint16_t* __restrict__ compat_rv,
                                                   const uint8_t* __restrict__ q, const uint64_t* __restrict__ qoff,
                                                   MemsParams P, Pool ivpool, Pool hitpool, MemsOut out, MemsWork W,
                                                   SegWork G) {
  __shared__ SmemFm Sf, Sr;
  smem_fm_init(Sf, Fw, compat_fw);
  smem_fm_init(Sr, Rv, compat_rv);
  __syncthreads();
  const uint32_t SCAP = STRIDE == 32 ? FAST_SET_CAP : W.set_cap;
  using SR = SetRef<BIv, STRIDE>;
  SR s0 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 0), s1 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 1);
  SR s2 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 2), s3 = thread_set<BIv, STRIDE>(W.sets, SCAP, 4, 3);
  uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  Cand* cands = W.cands + tid * W.cand_cap;
  uint64_t touches = 0;
  uint32_t r;
  const uint32_t n_long = G.longs();
  while (next_read(G.merge_queue, n_long, nullptr, r)) {
    uint32_t i = G.long_ids[r];
    uint64_t o = qoff[i];
    uint32_t n = (uint32_t)(qoff[i + 1] - o);
    uint64_t u0 = G.unit_base[r], u1 = G.unit_base[r + 1];
    uint32_t st = ST_OK;
    uint64_t t0 = touches;
    CandSink<SR> sink{cands, 0, W.cand_cap, &ivpool, &st, SCAP};
    bool fail = false;
    uint32_t t = 0;                                   // the true chain's next pivot
    for (uint64_t u = u0; u < u1 && !fail; u++) {
      uint32_t s = (uint32_t)(u - u0) * G.seg_len, e = min(n, s + G.seg_len);
      if (t >= e) continue;                           // the chain jumps over this segment
      if (G.exit_pivot[u] == ~0u) { st |= G.unit_st[u]; fail = true; break; }
      if (u > u0 && G.fx_entry[u] == t) {             // the fix-up pass started where the chain enters
        const Cand* fx = G.pool + G.fx_off[u];
        uint32_t fcnt = G.fx_cnt[u];
        for (uint32_t c = 0; c < fcnt && !fail; c++) {
          if (sink.nc >= sink.cap) { st |= ST_CAND_OVF; fail = true; break; }
          cands[sink.nc++] = fx[c];
        }
        if (fail) break;
        uint32_t cv = G.fx_conv[u];
        if (cv != ~0u) {
          const Cand* src = G.pool + G.cand_off[u];
          uint32_t cnt = G.cand_cnt[u];
          for (uint32_t c = 0; c < cnt; c++) {
            Cand cd = src[c];
            if (cd.pivot < cv) continue;
            if (sink.nc >= sink.cap) { st |= ST_CAND_OVF; fail = true; break; }
            cands[sink.nc++] = cd;
          }
          t = G.exit_pivot[u];
        } else {
          t = G.fx_exit[u];
        }
        continue;
      }
      uint32_t p = t;
      const uint32_t* bits = G.bits + u * G.seg_words;
      while (p < e && !((bits[(p - s) >> 5] >> ((p - s) & 31)) & 1u)) {
        p = smem_pivot<COUNT_TOUCH, FMT>(Fw, Rv, Sf, Sr, q + o, n, p, P, s0, s1, s2, s3, SCAP, st, touches, sink);
        if (p == ~0u) { fail = true; break; }
      }
      if (fail) break;
      if (p < e) {                                    // met the segment's chain at p
        const Cand* src = G.pool + G.cand_off[u];
        uint32_t cnt = G.cand_cnt[u];
        for (uint32_t c = 0; c < cnt; c++) {
          Cand cd = src[c];
          if (cd.pivot < p) continue;
          if (sink.nc >= sink.cap) { st |= ST_CAND_OVF; fail = true; break; }
          cands[sink.nc++] = cd;
        }
        t = G.exit_pivot[u];
      } else {
        t = p;
      }
    }
    uint64_t hs = 0; uint32_t hc = 0;
    if (!fail) {
      uint32_t nc = P.mode == 0 ? finalize_smems<true>(cands, sink.nc) : sink.nc;
      if (!write_hits(cands, nc, P, ivpool, hitpool, hs, hc)) st |= ST_POOL_OVF;
    }
    if (st) { hs = 0; hc = 0; }
    out.hit_start[i] = hs; out.hit_count[i] = hc; out.status[i] = st;
    bool ovf = st & (ST_SET_OVF | ST_CAND_OVF);
    if (COUNT_TOUCH && W.work_log) {
      atomicAdd(W.work_log + 4 * (size_t)i, (uint32_t)(touches - t0));
      if (ovf) atomicOr(W.work_log + 4 * (size_t)i + 3, 1u);
    }
    if (ovf) out.ovf_list[atomicAdd(out.n_ovf, 1u)] = i;
  }
  if (COUNT_TOUCH && touches) atomicAdd(out.touches, (unsigned long long)touches);
}
}  // namespace hfm

// =====================================================================================
// Warp-cooperative long-tail pass: one warp per read, the 32 lanes share the interval set
// of every step (reads whose sets outgrow the per-thread fast path: ambiguity codes near
// the start of a read, unseeded patterns inside N runs).  Same results as the per-thread
// code; sets live in a per-warp global region.
// =====================================================================================
namespace hfm {

__device__ __forceinline__ uint32_t lane_lt_mask() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ uint32_t warp_sum(uint32_t v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, d);
  return v;
}
__device__ __forceinline__ uint32_t warp_excl_scan(uint32_t v, uint32_t& total) {
  const int lane = threadIdx.x & 31;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) { uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d); if (lane >= d) x += y; }
  total = __shfl_sync(0xFFFFFFFFu, x, 31);
  return x - v;
}

// Lane groups of G = 4, 8, 16 or 32 lanes (one read per group in the sub-warp and
// warp-per-read SMEM kernels): the group's member mask, sum and exclusive scan.
template <int G>
__device__ __forceinline__ uint32_t grp_mask() {
  if (G == 32) return 0xFFFFFFFFu;
  return ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(uint32_t)(G - 1));
}
template <int G>
__device__ __forceinline__ uint32_t grp_sum(uint32_t v) {
  const uint32_t m = grp_mask<G>();
#pragma unroll
  for (int d = G / 2; d > 0; d >>= 1) v += __shfl_xor_sync(m, v, d, G);
  return v;
}
template <int G>
__device__ __forceinline__ uint32_t grp_excl_scan(uint32_t v, uint32_t& total) {
  const uint32_t m = grp_mask<G>();
  const int gl = threadIdx.x & (G - 1);
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < G; d <<= 1) { uint32_t y = __shfl_up_sync(m, x, d, G); if (gl >= d) x += y; }
  total = __shfl_sync(m, x, G - 1, G);
  return x - v;
}

// Backward-search step set (sorted, coalesced) with the warp: counting sort by symbol
// (pass 1 counts with ballots, pass 2 places), then lane 0 coalesces touching neighbours.
template <bool COUNT_TOUCH>
__device__ uint32_t warp_backward_search(const DevFm& F, const SmemFm& S, const uint8_t* p, uint32_t m,
                                         uint2*& cur, uint2*& nxt, uint32_t cap, uint64_t& touches) {
  const int lane = threadIdx.x & 31;
  cur[0] = make_uint2(0, F.text_len);
  if (m == 0) return 1;
  uint32_t n = 1, start = m;
  if (F.lut && m >= F.lut_depth) {
    uint64_t idx = 0; bool ok = true;
    for (int k = (int)F.lut_depth - 1; k >= 0; --k) {
      uint8_t c = p[m - F.lut_depth + k];
      uint32_t d = c < 16 ? S.dig[c] : 0xFF;
      if (d == 0xFF) { ok = false; break; }
      idx = idx * F.lut_radix + d;
    }
    if (ok) {
      uint2 iv = __ldg(F.lut + idx);
      if (COUNT_TOUCH && lane == 0) touches++;
      if (iv.x >= iv.y) return 0;
      if (lane == 0) cur[0] = iv;
      start = m - F.lut_depth;
    }
  }
  __syncwarp();
  for (uint32_t k = start; k-- > 0;) {
    uint8_t c = p[k];
    uint32_t mask = (c < 16 ? S.compat_mask[c] : 0) & F.sym_mask;
    if (!mask) return 0;
    uint32_t cnt[16];
#pragma unroll
    for (int r = 0; r < 16; r++) cnt[r] = 0;
    for (uint32_t b = 0; b < n; b += 32) {
      uint32_t i = b + lane;
      uint32_t rl[16], rh[16];
      uint2 iv = i < n ? cur[i] : make_uint2(0, 0);
      sym_ranks(F, S, iv.x, rl);
      sym_ranks(F, S, iv.y, rh);
      if (COUNT_TOUCH && i < n) touches += (iv.x != 0) + (iv.y != 0);
#pragma unroll
      for (int r = 0; r < 16; r++) cnt[r] += __popc(__ballot_sync(0xFFFFFFFFu, i < n && ((mask >> r) & 1) && rh[r] > rl[r]));
    }
    uint32_t total = 0;
#pragma unroll
    for (int r = 0; r < 16; r++) { uint32_t t = cnt[r]; cnt[r] = total; total += t; }
    if (total > cap) return ~0u;
    if (total == 0) return 0;
    for (uint32_t b = 0; b < n; b += 32) {
      uint32_t i = b + lane;
      uint32_t rl[16], rh[16];
      uint2 iv = i < n ? cur[i] : make_uint2(0, 0);
      sym_ranks(F, S, iv.x, rl);
      sym_ranks(F, S, iv.y, rh);
#pragma unroll
      for (int r = 0; r < 16; r++) {
        bool e = i < n && ((mask >> r) & 1) && rh[r] > rl[r];
        uint32_t bal = __ballot_sync(0xFFFFFFFFu, e);
        if (e) nxt[cnt[r] + __popc(bal & lane_lt_mask())] = make_uint2(S.C[r] + rl[r], S.C[r] + rh[r]);
        cnt[r] += __popc(bal);
      }
    }
    __syncwarp();
    uint32_t nn = 0;
    if (lane == 0) {   // coalesce touching neighbours (merge_intervals_inplace, query.rs:390-407)
      for (uint32_t e = 0; e < total; e++) {
        uint2 v = nxt[e];
        if (nn > 0) { uint2 last = nxt[nn - 1]; if (v.x <= last.y) { nxt[nn - 1] = make_uint2(last.x, max(last.y, v.y)); continue; } }
        nxt[nn++] = v;
      }
    }
    nn = __shfl_sync(0xFFFFFFFFu, nn, 0);
    __syncwarp();
    uint2* t = cur; cur = nxt; nxt = t; n = nn;
  }
  return n;
}

template <bool COUNT_TOUCH>
__global__ void __launch_bounds__(128) k_bsearch_warp(DevFm F, const uint16_t* __restrict__ compat_masks,
                                                     const uint8_t* __restrict__ q, const uint64_t* __restrict__ qoff,
                                                     const uint32_t* __restrict__ ids, uint32_t n, uint32_t hit_cap,
                                                     uint2* work, uint32_t set_cap, unsigned int* queue, Pool pool,
                                                     BsOut out, uint32_t* still_ovf,
                                                     const uint32_t* __restrict__ n_dev = nullptr) {
  __shared__ SmemFm S;
  smem_fm_init(S, F, compat_masks);
  __syncthreads();
  if (n_dev) n = *n_dev;                   // graph-captured chains: the count is on the device
  const int lane = threadIdx.x & 31;
  uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint2* A = work + warp * 2 * set_cap;
  uint2* B = A + set_cap;
  uint64_t touches = 0;
  for (;;) {
    uint32_t k = 0;
    if (lane == 0) k = atomicAdd(queue, 1u);
    k = __shfl_sync(0xFFFFFFFFu, k, 0);
    if (k >= n) break;
    uint32_t i = ids[k];
    uint2* cur = A; uint2* nxt = B;
    uint64_t o = qoff[i];
    uint32_t niv = warp_backward_search<COUNT_TOUCH>(F, S, q + o, (uint32_t)(qoff[i + 1] - o), cur, nxt, set_cap, touches);
    if (niv == ~0u) {
      if (lane == 0) { atomicAdd(still_ovf, 1u); out.status[i] = ST_SET_OVF; }
      continue;
    }
    uint32_t cnt = 0; uint64_t hits = 0;
    for (uint32_t b = lane; b < niv; b += 32) {
      uint2 v = cur[b]; uint32_t sz = v.y - v.x;
      cnt += sz; hits += (hit_cap && sz > hit_cap) ? hit_cap : sz;
    }
    cnt = warp_sum(cnt);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) hits += __shfl_xor_sync(0xFFFFFFFFu, hits, d);
    uint64_t off = 0; uint32_t st = ST_OK;
    if (out.nhits && niv) {
      if (lane == 0) off = thread_reserve(pool, niv);
      off = __shfl_sync(0xFFFFFFFFu, off, 0);
      if (off == ~0ull) st = ST_POOL_OVF;
      else { uint2* dst = (uint2*)pool.base + off; for (uint32_t b = lane; b < niv; b += 32) dst[b] = cur[b]; }
    }
    if (lane == 0) {
      out.counts[i] = cnt;
      if (out.nhits) { out.nhits[i] = hits; out.niv[i] = niv; out.ivoff[i] = off; }
      out.status[i] = st;
    }
    __syncwarp();
  }
  if (COUNT_TOUCH && touches) atomicAdd(out.touches, (unsigned long long)touches);
}

// One extension of the whole set by a group of G lanes (outputs in lane-chunk order).
template <int DIR, bool COUNT_TOUCH, int G = 32>
__device__ uint32_t warp_extend_set(const DevFm& X, const SmemFm& S, uint32_t mask, const BIv* in, uint32_t nin,
                                    BIv* out, uint32_t cap, uint32_t& cov, bool& ovf, uint64_t& touches) {
  const int lane = threadIdx.x & (G - 1);
  uint32_t nout = 0, covl = 0;
  for (uint32_t b = 0; b < nin; b += G) {
    uint32_t i = b + lane;
    BIv iv = i < nin ? in[i] : BIv{0, 0, 0, 0};
    uint32_t a = DIR == 0 ? iv.rlo : iv.flo, e = DIR == 0 ? iv.rhi : iv.fhi;
    uint32_t base = DIR == 0 ? iv.flo : iv.rlo;
    uint32_t rl[16], rh[16];
    sym_ranks(X, S, a, rl);
    sym_ranks(X, S, e, rh);
    if (COUNT_TOUCH && i < nin) touches += (a != 0) + (e != 0);
    uint32_t k = 0;
#pragma unroll
    for (int s = 0; s < 16; s++) k += (i < nin && ((mask >> s) & 1) && rh[s] > rl[s]) ? 1u : 0u;
    uint32_t total;
    uint32_t pos = nout + grp_excl_scan<G>(k, total);
    if (nout + total > cap) { ovf = true; return nout; }
    uint32_t run = 0;
#pragma unroll
    for (int s = 0; s < 16; s++) {
      uint32_t d = rh[s] - rl[s];
      if (i < nin && ((mask >> s) & 1) && d) {
        BIv o;
        if (DIR == 0) { o.flo = base + run; o.fhi = base + run + d; o.rlo = S.C[s] + rl[s]; o.rhi = S.C[s] + rh[s]; }
        else { o.flo = S.C[s] + rl[s]; o.fhi = S.C[s] + rh[s]; o.rlo = base + run; o.rhi = base + run + d; }
        out[pos++] = o;
        covl += d;
      }
      run += d;
    }
    nout += total;
  }
  cov = grp_sum<G>(covl);
  __syncwarp(grp_mask<G>());
  return nout;
}

template <int DIR, bool COUNT_TOUCH, int G = 32>
__device__ bool warp_any_extend(const DevFm& X, const SmemFm& S, uint32_t mask, const BIv* in, uint32_t nin,
                                uint64_t& touches) {
  const int lane = threadIdx.x & (G - 1);
  bool any = false;
  for (uint32_t b = 0; b < nin && !any; b += G) {
    uint32_t i = b + lane;
    BIv iv = i < nin ? in[i] : BIv{0, 0, 0, 0};
    uint32_t a = DIR == 0 ? iv.rlo : iv.flo, e = DIR == 0 ? iv.rhi : iv.fhi;
    uint32_t rl[16], rh[16];
    sym_ranks(X, S, a, rl);
    sym_ranks(X, S, e, rh);
    if (COUNT_TOUCH && i < nin) touches += (a != 0) + (e != 0);
    bool mine = false;
#pragma unroll
    for (int s = 0; s < 16; s++) mine |= i < nin && ((mask >> s) & 1) && rh[s] != rl[s];
    any = __any_sync(grp_mask<G>(), mine);
  }
  return any;
}

// Candidate search of one read by a group of G lanes; control flow is group-uniform.
template <bool COUNT_TOUCH, int G = 32>
__device__ uint32_t warp_mems_one(const DevFm& Fw, const DevFm& Rv, const SmemFm& Sf, const SmemFm& Sr,
                                  const uint8_t* q, uint32_t n, const MemsParams& P, BIv* curr, BIv* nxt, BIv* wa,
                                  BIv* wb, uint32_t set_cap, Cand* cands, uint32_t cand_cap, Pool& ivpool,
                                  uint32_t& st, uint64_t& touches) {
  const int lane = threadIdx.x & (G - 1);
  const uint32_t gm = grp_mask<G>();
  uint32_t nc = 0;
  if (n == 0 || P.min_len == 0) return 0;
  const BIv full = {0, Fw.text_len, 0, Fw.text_len};
  bool ovf = false;
  auto qmask = [&](const SmemFm& S, uint8_t c) -> uint32_t { return c < 16 ? S.compat_mask[c] : 0u; };
  auto emit = [&](uint32_t qs, uint32_t qe, uint32_t count, const BIv* ivs, uint32_t niv) -> bool {
    if (nc >= cand_cap) { st |= ST_CAND_OVF; return false; }
    uint64_t off = 0;
    if (lane == 0) off = thread_reserve(ivpool, niv);
    off = __shfl_sync(gm, off, 0, G);
    if (off == ~0ull) { st |= ST_POOL_OVF; return false; }
    BIv* dst = (BIv*)ivpool.base + off;
    for (uint32_t k = lane; k < niv; k += G) dst[k] = ivs[k];
    if (lane == 0) cands[nc] = Cand{qs, qe, count, niv, off};
    nc++;
    __syncwarp(gm);
    return true;
  };
  if (P.mode == 1) {
    for (uint32_t i = 0; i < n; i++) {
      BIv* c = curr; BIv* x = nxt;
      if (lane == 0) c[0] = full;
      __syncwarp(gm);
      uint32_t ncur = 1, cov = 0, j = i;
      bool matched = false;
      while (j < n) {
        uint32_t ncov;
        uint32_t nn = warp_extend_set<0, COUNT_TOUCH, G>(Rv, Sr, qmask(Sr, q[j]), c, ncur, x, set_cap, ncov, ovf, touches);
        if (ovf) { st |= ST_SET_OVF; return ~0u; }
        if (nn == 0) break;
        BIv* t = c; c = x; x = t; ncur = nn; cov = ncov; j++; matched = true;
      }
      if (!matched || j - i < P.min_len) continue;
      bool lmax = i == 0 || !warp_any_extend<1, COUNT_TOUCH, G>(Fw, Sf, qmask(Sf, q[i - 1]), c, ncur, touches);
      if (!lmax) continue;
      if (!emit(i, j, cov, c, ncur)) return ~0u;
    }
    return nc;
  }
  uint32_t pivot = 0;
  while (pivot < n) {
    BIv* c = curr; BIv* x = nxt;
    if (lane == 0) x[0] = full;
    __syncwarp(gm);
    uint32_t cov;
    uint32_t ncur = warp_extend_set<0, COUNT_TOUCH, G>(Rv, Sr, qmask(Sr, q[pivot]), x, 1, c, set_cap, cov, ovf, touches);
    if (ovf) { st |= ST_SET_OVF; return ~0u; }
    if (ncur == 0) { pivot++; continue; }
    uint32_t j = pivot + 1, reach = pivot + 1;
    for (;;) {
      uint32_t end, nn = 0, ncov = 0;
      bool next_empty, record;
      if (j == n) { end = n; next_empty = true; record = true; }
      else {
        nn = warp_extend_set<0, COUNT_TOUCH, G>(Rv, Sr, qmask(Sr, q[j]), c, ncur, x, set_cap, ncov, ovf, touches);
        if (ovf) { st |= ST_SET_OVF; return ~0u; }
        end = j; next_empty = nn == 0; record = ncov != cov;
      }
      if (record) {
        reach = end;
        const BIv* b = c;
        uint32_t nb = ncur, start = pivot, bcov = cov;
        BIv* bufs[2] = {wa, wb};
        int t = 0;
        while (start > 0) {
          uint32_t lcov;
          uint32_t nl = warp_extend_set<1, COUNT_TOUCH, G>(Fw, Sf, qmask(Sf, q[start - 1]), b, nb, bufs[t], set_cap, lcov, ovf, touches);
          if (ovf) { st |= ST_SET_OVF; return ~0u; }
          if (nl == 0) break;
          b = bufs[t]; nb = nl; bcov = lcov; t ^= 1; start--;
        }
        if (end - start >= P.min_len) {
          bool rmax = end == n ||
                      (start == pivot ? next_empty : !warp_any_extend<0, COUNT_TOUCH, G>(Rv, Sr, qmask(Sr, q[end]), b, nb, touches));
          if (rmax && !emit(start, end, bcov, b, nb)) return ~0u;
        }
      }
      if (j == n || nn == 0) break;
      BIv* tt = c; c = x; x = tt; ncur = nn; cov = ncov; j++;
    }
    pivot = max(reach, pivot + 1);
  }
  return nc;
}

// Persistent SMEM / MEM search with one read per group of G lanes (G = 32: the warp tier
// of reads whose sets outgrew the per-thread kernels; G = 4, 8, 16: the sub-warp
// candidates of the autotuner).  Group g of the grid owns sets and a candidate list at
// g * 4 * set_cap / g * cand_cap.
template <bool COUNT_TOUCH, int G = 32>
__global__ void __launch_bounds__(128) k_mems_warp(DevFm Fw, DevFm Rv, const uint16_t* __restrict__ compat_fw,
                                                  const uint16_t* __restrict__ compat_rv, const uint8_t* __restrict__ q,
                                                  const uint64_t* __restrict__ qoff, MemsParams P, Pool ivpool,
                                                  Pool hitpool, MemsOut out, MemsWork W) {
  __shared__ SmemFm Sf, Sr;
  smem_fm_init(Sf, Fw, compat_fw);
  smem_fm_init(Sr, Rv, compat_rv);
  __syncthreads();
  const int lane = threadIdx.x & (G - 1);
  const uint32_t gm = grp_mask<G>();
  uint64_t grp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  BIv* base = W.sets + grp * 4 * W.set_cap;
  Cand* cands = W.cands + grp * W.cand_cap;
  uint64_t touches = 0;
  for (;;) {
    uint32_t k = 0;
    if (lane == 0) k = atomicAdd(W.queue, 1u);
    k = __shfl_sync(gm, k, 0, G);
    if (k >= W.count()) break;
    uint32_t i = W.ids[k];
    uint32_t st = ST_OK;
    uint64_t o = qoff[i];
    uint64_t t0 = touches;
    uint32_t nc = warp_mems_one<COUNT_TOUCH, G>(Fw, Rv, Sf, Sr, q + o, (uint32_t)(qoff[i + 1] - o), P, base,
                                                base + W.set_cap, base + 2 * W.set_cap, base + 3 * W.set_cap,
                                                W.set_cap, cands, W.cand_cap, ivpool, st, touches);
    __syncwarp(gm);
    if (COUNT_TOUCH && W.work_log) {
      uint32_t d = grp_sum<G>((uint32_t)(touches - t0));
      if (lane == 0) { W.work_log[4 * (size_t)i] += d; W.work_log[4 * (size_t)i + 3] |= 3u; }
    }
    if (lane == 0) {
      uint64_t hs = 0; uint32_t hc = 0;
      if (nc != ~0u) {
        if (P.mode == 0) nc = finalize_smems<true>(cands, nc);
        if (!write_hits(cands, nc, P, ivpool, hitpool, hs, hc)) st |= ST_POOL_OVF;
      }
      if (st) { hs = 0; hc = 0; }
      out.hit_start[i] = hs; out.hit_count[i] = hc; out.status[i] = st;
      if (st & (ST_SET_OVF | ST_CAND_OVF)) {
        if (W.rerun) atomicAdd(W.still_ovf, 1u);
        else out.ovf_list[atomicAdd(out.n_ovf, 1u)] = i;      // on to the warp tier
      }
    }
    __syncwarp(gm);
  }
  if (COUNT_TOUCH && touches) atomicAdd(out.touches, (unsigned long long)touches);
}

}  // namespace hfm
