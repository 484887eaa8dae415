// resolve.cuh — SA-position resolve (LF walk to a sampled row) fused with the reference
// boundary map, plus the scan / gather kernels that lay results out per read.
//
// One thread per output position.  Positions are grouped in segments (one per SA
// interval, rows lo .. lo+n); a block finds its segments once and every thread locates
// its own segment in shared memory.  Replaces locate_resolve.wgsl:98-176,
// mem_resolve.wgsl:101-136 and ref_map.wgsl:32-59 of the reference, with the CPU
// resolve_sa / map_position semantics (src/fm_index/query.rs:282-357).
#pragma once
#include "dev_index.cuh"

namespace hfm {

struct ResolveArgs {
  const uint32_t* seg_row;      // row of the segment's first position
  uint32_t row_stride;          // in u32 units
  const uint64_t* seg_off;      // nseg + 1 ascending position offsets
  uint32_t nseg;
  uint64_t total;
  const uint32_t* bounds;       // map position -> (index, offset): partition_point(bounds <= p)
  uint32_t nb;
  uint32_t guard;               // max LF steps before the walk is declared broken
  uint32_t* out;                // 2 * total u32
  uint32_t* walk_err;
  unsigned long long* steps;    // LF steps (nullptr: not counted)
  const uint32_t* block_first;  // segment containing the first position of each block
  const uint64_t* total_dev;    // when set (graph-captured chains), the position count is read here
};

// block_first[b] = segment holding position b * blk (positions are CSR over segments).
// Blocks at or past max_blocks (the map's size) are skipped: a chain with fixed capacities
// runs this before it knows whether the positions fit.
__global__ void k_block_first(const uint64_t* __restrict__ seg_off, uint32_t nseg, uint32_t blk,
                              uint32_t* __restrict__ block_first, uint64_t max_blocks = ~0ull) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  uint64_t a = seg_off[s], e = seg_off[s + 1];
  if (a == e) return;
  const uint64_t last = min((e - 1) / blk, max_blocks - 1);
  for (uint64_t b = (a + blk - 1) / blk; b <= last; b++) block_first[b] = s;
}

// Segments [first, first + cnt) cover positions [b * blk, (b + 1) * blk) of block b.
__device__ __forceinline__ void block_segments(const uint32_t* block_first, uint64_t nblocks, uint32_t nseg,
                                               uint32_t& first, uint32_t& cnt) {
  uint64_t b = blockIdx.x;
  first = block_first[b];
  uint32_t last = b + 1 < nblocks ? block_first[b + 1] : nseg - 1;
  cnt = last - first + 1;
}

constexpr int RES_T = 256;
constexpr int RES_BOUNDS_SMEM = 2048;

template <bool COUNT>
__global__ void __launch_bounds__(RES_T) k_resolve(DevFm F, ResolveArgs A) {
  __shared__ SmemFm S;
  __shared__ uint64_t s_off[RES_T + 1];
  __shared__ uint32_t s_row[RES_T];
  __shared__ uint32_t s_b[RES_BOUNDS_SMEM];
  __shared__ uint32_t s_first, s_cnt;
  if (threadIdx.x < 16) { S.C[threadIdx.x] = F.C[threadIdx.x]; }
  const uint64_t total = A.total_dev ? *A.total_dev : A.total;
  uint64_t p0 = (uint64_t)blockIdx.x * RES_T;
  if (p0 >= total) return;                 // a grid sized for a capacity: blocks past the positions
  uint64_t p1 = min(p0 + RES_T, total);
  if (threadIdx.x == 0) {
    uint32_t f, c;
    block_segments(A.block_first, (total + RES_T - 1) / RES_T, A.nseg, f, c);
    s_first = f; s_cnt = c;
  }
  bool smem_b = A.nb <= RES_BOUNDS_SMEM;
  if (smem_b) for (uint32_t k = threadIdx.x; k < A.nb; k += RES_T) s_b[k] = A.bounds[k];
  __syncthreads();
  uint32_t first = s_first, cnt = s_cnt;
  bool local = cnt <= RES_T;
  if (local) {
    for (uint32_t k = threadIdx.x; k <= cnt; k += RES_T) s_off[k] = A.seg_off[first + k];
    for (uint32_t k = threadIdx.x; k < cnt; k += RES_T) s_row[k] = A.seg_row[(size_t)(first + k) * A.row_stride];
  }
  __syncthreads();
  uint64_t p = p0 + threadIdx.x;
  if (p >= p1) return;
  uint32_t seg, row;
  if (local) {
    uint32_t lo = 0, hi = cnt - 1;
    while (lo < hi) { uint32_t mid = (lo + hi + 1) >> 1; if (s_off[mid] <= p) lo = mid; else hi = mid - 1; }
    seg = lo; row = s_row[lo] + (uint32_t)(p - s_off[lo]);
  } else {
    uint32_t lo = first, hi = A.nseg - 1;
    while (lo < hi) { uint32_t mid = (lo + hi + 1) >> 1; if (A.seg_off[mid] <= p) lo = mid; else hi = mid - 1; }
    seg = lo; row = A.seg_row[(size_t)lo * A.row_stride] + (uint32_t)(p - A.seg_off[lo]);
  }
  (void)seg;
  // LF walk (resolve_sa, src/fm_index/query.rs:282-291)
  uint32_t pos = row, steps = 0, val = 0, text;
  bool ok = true;
  for (;;) {
    if (lf_or_sample(F, S, pos, val)) break;
    if (++steps > A.guard) { ok = false; break; }
  }
  uint32_t r0, r1;
  if (ok) {
    text = val + steps;
    uint32_t idx = smem_b ? upper_bound_u32(s_b, A.nb, text) : upper_bound_u32(A.bounds, A.nb, text);
    uint32_t start = idx == 0 ? 0 : (smem_b ? s_b[idx - 1] : A.bounds[idx - 1]);
    r0 = idx; r1 = text - start;
  } else {
    atomicAdd(A.walk_err, 1u);
    r0 = 0xFFFFFFFFu; r1 = 0xFFFFFFFFu;
  }
  reinterpret_cast<uint2*>(A.out)[p] = make_uint2(r0, r1);
  if (COUNT) atomicAdd(A.steps, (unsigned long long)(steps + 1));
}

// ---- resolve deduplication ----------------------------------------------------------
// Segments with the same (first row, length) resolve to the same positions: across a
// batch, hits on repeated strings (N runs, repeat copies) share their SA interval.  The
// segments are hashed, each distinct one is resolved once, and every hit copies its
// positions from it.  Output is identical to resolving every row.

constexpr unsigned long long HASH_EMPTY = ~0ull;

__device__ __forceinline__ uint64_t mix64(uint64_t k) {      // splitmix64 finaliser
  k ^= k >> 30; k *= 0xbf58476d1ce4e5b9ull; k ^= k >> 27; k *= 0x94d049bb133111ebull; k ^= k >> 31;
  return k;
}

__global__ void k_dedup_insert(const uint32_t* __restrict__ seg_row, uint32_t stride, const uint64_t* __restrict__ seg_off,
                               uint32_t nseg, unsigned long long* __restrict__ keys, uint64_t mask,
                               uint32_t* __restrict__ seg_slot) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  uint64_t n = seg_off[s + 1] - seg_off[s];
  if (n == 0) { seg_slot[s] = 0xFFFFFFFFu; return; }
  unsigned long long key = ((unsigned long long)seg_row[(size_t)s * stride] << 32) | (uint32_t)n;
  uint64_t h = mix64(key) & mask;
  // the table has at least twice as many slots as segments: an empty slot is always found
  for (uint64_t probe = 0; probe <= mask; probe++) {
    unsigned long long prev = atomicCAS(keys + h, HASH_EMPTY, key);
    if (prev == HASH_EMPTY || prev == key) { seg_slot[s] = (uint32_t)h; return; }
    h = (h + 1) & mask;
  }
  seg_slot[s] = 0xFFFFFFFFu;    // unreachable with a half-empty table
}

__global__ void k_dedup_flags(const unsigned long long* __restrict__ keys, uint64_t size, uint32_t* __restrict__ flags) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < size) flags[i] = keys[i] != HASH_EMPTY;
}

__global__ void k_dedup_compact(const unsigned long long* __restrict__ keys, uint64_t size,
                                const uint64_t* __restrict__ uid, uint32_t* __restrict__ urow,
                                uint32_t* __restrict__ ulen) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= size) return;
  unsigned long long k = keys[i];
  if (k == HASH_EMPTY) return;
  uint64_t u = uid[i];
  urow[u] = (uint32_t)(k >> 32); ulen[u] = (uint32_t)k;
}

// out[p] = resolved position of its segment's distinct copy.  A block copies EXP_BLK
// consecutive positions (EXP_PER per thread, strided for coalescing); its segments are
// staged in shared memory once.
constexpr int EXP_T = 256, EXP_PER = 8, EXP_BLK = EXP_T * EXP_PER;
__global__ void __launch_bounds__(EXP_T) k_dedup_expand(const uint64_t* __restrict__ seg_off, uint32_t nseg, uint64_t total,
                                                        const uint32_t* __restrict__ seg_slot,
                                                        const uint64_t* __restrict__ uid,
                                                        const uint64_t* __restrict__ uoff,
                                                        const uint2* __restrict__ uout, uint2* __restrict__ out,
                                                        const uint32_t* __restrict__ block_first,
                                                        const uint64_t* __restrict__ total_dev = nullptr) {
  __shared__ uint64_t s_off[EXP_BLK + 1];
  __shared__ uint64_t s_src[EXP_BLK];
  __shared__ uint32_t s_first, s_cnt;
  if (total_dev) total = *total_dev;
  uint64_t p0 = (uint64_t)blockIdx.x * EXP_BLK;
  if (p0 >= total) return;                 // a grid sized for a capacity: blocks past the positions
  uint64_t p1 = min(p0 + EXP_BLK, total);
  if (threadIdx.x == 0) {
    uint32_t f, c;
    block_segments(block_first, (total + EXP_BLK - 1) / EXP_BLK, nseg, f, c);
    s_first = f; s_cnt = c;
  }
  __syncthreads();
  uint32_t first = s_first, cnt = s_cnt;
  bool local = cnt <= EXP_BLK;
  if (local) {
    for (uint32_t k = threadIdx.x; k <= cnt; k += EXP_T) s_off[k] = seg_off[first + k];
    for (uint32_t k = threadIdx.x; k < cnt; k += EXP_T) {
      uint32_t slot = seg_slot[first + k];
      s_src[k] = slot == 0xFFFFFFFFu ? 0 : uoff[uid[slot]];
    }
  }
  __syncthreads();
  uint32_t lo = 0;                       // positions ascend per thread: resume the search
  for (int k = 0; k < EXP_PER; k++) {
    uint64_t p = p0 + threadIdx.x + (uint64_t)k * EXP_T;
    if (p >= p1) return;
    uint64_t src;
    if (local) {
      // still in the previous position's segment (the usual case for segments of more than
      // EXP_T positions), else a binary search over the rest
      if (lo + 1 < cnt && s_off[lo + 1] <= p) {
        uint32_t hi = cnt - 1;
        lo++;
        while (lo < hi) { uint32_t mid = (lo + hi + 1) >> 1; if (s_off[mid] <= p) lo = mid; else hi = mid - 1; }
      }
      src = s_src[lo] + (p - s_off[lo]);
    } else {
      uint32_t l = first, hi = nseg - 1;
      while (l < hi) { uint32_t mid = (l + hi + 1) >> 1; if (seg_off[mid] <= p) l = mid; else hi = mid - 1; }
      src = uoff[uid[seg_slot[l]]] + (p - seg_off[l]);
    }
    out[p] = uout[src];
  }
}

// ---- exclusive scan (u32 or u64 input) -> u64 output with out[n] = total ----------
constexpr int SCAN_T = 256, SCAN_ITEMS = 8, SCAN_TILE = SCAN_T * SCAN_ITEMS;

template <class T>
__global__ void __launch_bounds__(SCAN_T) k_scan_tiles(const T* __restrict__ in, uint32_t in_stride, uint64_t n,
                                                      uint64_t* __restrict__ out, uint64_t* __restrict__ tile_sums) {
  __shared__ uint64_t s[SCAN_T];
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint64_t v[SCAN_ITEMS], sum = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    uint64_t i = base + k;
    v[k] = i < n ? (uint64_t)in[i * in_stride] : 0;
    sum += v[k];
  }
  s[threadIdx.x] = sum;
  __syncthreads();
  for (int d = 1; d < SCAN_T; d <<= 1) {
    uint64_t t = threadIdx.x >= d ? s[threadIdx.x - d] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  uint64_t run = s[threadIdx.x] - sum;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    uint64_t i = base + k;
    if (i < n) out[i] = run;
    run += v[k];
  }
  if (threadIdx.x == SCAN_T - 1) tile_sums[blockIdx.x] = s[SCAN_T - 1];
}

// Scans tile sums in place (single block, sequential chunks).
__global__ void __launch_bounds__(1024) k_scan_sums(uint64_t* sums, uint32_t ntiles) {
  __shared__ uint64_t s[1024];
  __shared__ uint64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < ntiles; base += 1024) {
    uint32_t i = base + threadIdx.x;
    uint64_t v = i < ntiles ? sums[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
      uint64_t t = threadIdx.x >= d ? s[threadIdx.x - d] : 0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < ntiles) sums[i] = carry + s[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += s[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[ntiles] = carry;
}

__global__ void k_scan_add(uint64_t* out, uint64_t n, const uint64_t* __restrict__ sums, uint32_t ntiles) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += sums[i / SCAN_TILE];
  if (i == 0) out[n] = sums[ntiles];
}

// ---- gathers ------------------------------------------------------------------
// Locate: query intervals (pool) -> resolve segments in query order.
__global__ void k_gather_locate(const uint2* __restrict__ ivpool, const uint64_t* __restrict__ ivoff,
                                const uint32_t* __restrict__ niv, const uint64_t* __restrict__ seg_base,
                                const uint64_t* __restrict__ pos_base, uint32_t nq, uint32_t cap,
                                uint32_t* __restrict__ seg_row, uint64_t* __restrict__ seg_off) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  uint64_t sb = seg_base[i], run = pos_base[i];
  const uint2* iv = ivpool + ivoff[i];
  for (uint32_t k = 0; k < niv[i]; k++) {
    uint2 v = iv[k];
    uint32_t sz = v.y - v.x;
    seg_row[sb + k] = v.x; seg_off[sb + k] = run;
    run += (cap && sz > cap) ? cap : sz;
  }
}

// Mems: per-read hits (pool) -> CSR hit array.
__global__ void k_gather_hits(const uint4* __restrict__ hitpool, const uint64_t* __restrict__ hit_start,
                              const uint32_t* __restrict__ hit_count, const uint64_t* __restrict__ hit_base,
                              uint32_t nq, uint4* __restrict__ hits) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  const uint4* src = hitpool + hit_start[i] * 2;
  uint4* dst = hits + hit_base[i] * 2;
  for (uint32_t k = 0; k < hit_count[i] * 2; k++) dst[k] = src[k];
}

__global__ void k_set_pos_off(uint32_t* __restrict__ hits, const uint64_t* __restrict__ pos_off, uint64_t nh) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nh) return;
  uint64_t o = pos_off[i];
  hits[i * 8 + 6] = (uint32_t)o; hits[i * 8 + 7] = (uint32_t)(o >> 32);
}

// Per-read work record, words 1 and 2: MemHits and positions reported for read i.
__global__ void k_work_log(const uint64_t* __restrict__ hit_base, const uint64_t* __restrict__ npos_scan, uint32_t nq,
                           uint32_t* __restrict__ log) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  uint64_t h0 = hit_base[i], h1 = hit_base[i + 1];
  log[4 * (size_t)i + 1] = (uint32_t)(h1 - h0);
  uint64_t np = npos_scan[h1] - npos_scan[h0];
  log[4 * (size_t)i + 2] = np > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)np;
}

// Graph-captured locate chain: queries whose intervals did not fit the pool report none
// (they are flagged; the batch is rerun), so the CSR never reaches past the pool.
__global__ void k_zero_failed(const uint32_t* __restrict__ status, uint32_t n, uint32_t* __restrict__ niv,
                              uint64_t* __restrict__ nhits) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n && status[k] != 0) { niv[k] = 0; nhits[k] = 0; }
}

// seg_off[k] = total for k in [nseg, cap]: segments past the count are empty.
__global__ void k_seal_segments(uint64_t* __restrict__ seg_off, const uint64_t* __restrict__ nseg_p,
                                const uint64_t* __restrict__ total_p, uint64_t cap) {
  const uint64_t nseg = *nseg_p, total = *total_p;
  for (uint64_t k = nseg + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k <= cap; k += (uint64_t)gridDim.x * blockDim.x)
    seg_off[k] = total;
}

__global__ void k_iota(uint32_t* __restrict__ ids, uint32_t n) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) ids[k] = k;
}

// seen[] zeroed by the caller; *bad set when ids is not a permutation of 0..n-1.
__global__ void k_check_perm(const uint32_t* __restrict__ ids, uint32_t n, uint32_t* __restrict__ seen,
                             uint32_t* __restrict__ bad) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t i = ids[k];
  if (i >= n || atomicExch(seen + i, 1u) != 0) atomicExch(bad, 1u);
}

}  // namespace hfm
