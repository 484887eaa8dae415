// hfm_oracle.cpp — CPU restatement of haystackfm's query path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle (and the timed CPU
// baseline) for the CUDA path in haystackfm_b200/.  Only tests/, the smoke()
// entry point and bench.py's cpu_baseline / reference legs may load it; the
// product never links or calls it.
//
// Every function restates the reference's Rust CPU code (sriram98v/haystackfm,
// Rust edition 2021) and cites the file:line it follows.  The reference cannot be
// compiled here (no rustc/cargo, crates not vendored), so the restatement is pinned
// against the reference's own golden vectors and known-answer tests
// (tests/golden/*.json, tests/test_oracle_golden.py).
//
// What is restated:
//   * alphabet: IUPAC compatibility table and ExactDna          src/alphabet.rs:174-193,240-305,375-393
//   * CArray                                                   src/c_array.rs:14-67
//   * OccTable (compacted lanes, interleaved 64-pos records)   src/occ/mod.rs:99-480, src/occ/cpu.rs:23-140
//   * SampledSuffixArray (14-byte marker records)              src/suffix_array/mod.rs:71-201
//   * LookupTable (depth-k BFS)                                src/fm_index/lookup.rs:37-111
//   * FmIndex build (naive suffix sort), count/locate          src/fm_index/mod.rs:117-195,288-291,
//                                                              src/fm_index/query.rs:9-357,390-407
//   * BidirInterval and SMEM/MEM search                        src/fm_index/bidir.rs:51-143,
//                                                              src/fm_index/smem.rs:71-357,
//                                                              src/fm_index/bidir_index.rs:53-80,157-168,183-210,523-532
//   * bincode-1 layout of FmIndex / BidirFmIndex               src/fm_index/serialize.rs:13-80
//   * GPU MemHit contract (one hit per SA interval, capped)    src/fm_index/bidir_index.rs:307-514
//
// The suffix array here is a plain comparison sort (true lexicographic order of the
// encoded text, as `build_suffix_array_naive`, src/suffix_array/cpu.rs:20-25); the
// reference uses the psacak crate, whose tie order through interior sentinels is not
// reproducible here (documented as unpinned).

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// Alphabet (src/alphabet.rs:18-52, 174-193, 286-294)
// ---------------------------------------------------------------------------
enum : uint8_t { SENT = 0, A = 1, C = 2, G = 3, T = 4, N = 5, R = 6, Y = 7, S = 8, W = 9,
                 K = 10, M = 11, B = 12, D = 13, H = 14, V = 15 };

struct Compat { uint8_t len; uint8_t sym[16]; };

// compatible_symbols (src/alphabet.rs:174-193), same order as the Rust slices.
static const Compat IUPAC_COMPAT[16] = {
    {0, {}},
    {8, {A, N, R, W, M, D, H, V}},
    {8, {C, N, Y, S, M, B, H, V}},
    {8, {G, N, R, S, K, B, D, V}},
    {8, {T, N, Y, W, K, B, D, H}},
    {15, {A, C, G, T, N, R, Y, S, W, K, M, B, D, H, V}},
    {12, {A, G, N, R, S, W, K, M, B, D, H, V}},
    {12, {C, T, N, Y, S, W, K, M, B, D, H, V}},
    {12, {C, G, N, R, Y, S, K, M, B, D, H, V}},
    {12, {A, T, N, R, Y, W, K, M, B, D, H, V}},
    {12, {G, T, N, R, Y, S, W, K, B, D, H, V}},
    {12, {A, C, N, R, Y, S, W, M, B, D, H, V}},
    {14, {C, G, T, N, R, Y, S, W, K, M, B, D, H, V}},
    {14, {A, G, T, N, R, Y, S, W, K, M, B, D, H, V}},
    {14, {A, C, T, N, R, Y, S, W, K, M, B, D, H, V}},
    {14, {A, C, G, N, R, Y, S, W, K, M, B, D, H, V}},
};
// ExactDna::compatible (src/alphabet.rs:286-294).
static const Compat EXACT_COMPAT[16] = {
    {0, {}}, {1, {A}}, {1, {C}}, {1, {G}}, {1, {T}},
    {0, {}}, {0, {}}, {0, {}}, {0, {}}, {0, {}}, {0, {}}, {0, {}}, {0, {}}, {0, {}}, {0, {}}, {0, {}},
};
static const Compat EMPTY_COMPAT = {0, {}};

static const uint8_t CORE_SYMBOLS[4] = {A, C, G, T};  // alphabet_fns_from_tag (src/alphabet.rs:240-254)

static thread_local std::string g_err;

// ---------------------------------------------------------------------------
// Unaligned little-endian readers (the reference reads native-endian = LE)
// ---------------------------------------------------------------------------
static inline uint16_t ld16(const uint8_t* p) { uint16_t v; std::memcpy(&v, p, 2); return v; }
static inline uint32_t ld32(const uint8_t* p) { uint32_t v; std::memcpy(&v, p, 4); return v; }
static inline uint64_t ld64(const uint8_t* p) { uint64_t v; std::memcpy(&v, p, 8); return v; }

// ---------------------------------------------------------------------------
// CArray (src/c_array.rs:14-67)
// ---------------------------------------------------------------------------
struct CArray {
  uint32_t data[16] = {0};
  static CArray from_text(const std::vector<uint8_t>& text) {
    uint32_t freq[16] = {0};
    for (uint8_t ch : text) if (ch < 16) freq[ch]++;
    CArray c; uint32_t sum = 0;
    for (int i = 0; i < 16; i++) { c.data[i] = sum; sum += freq[i]; }
    return c;
  }
  uint32_t get(uint8_t c) const { return data[c]; }
  // symbol_count (src/c_array.rs:59-67)
  uint32_t symbol_count(uint8_t c, uint32_t text_len) const {
    uint32_t upper = (c + 1 < 16) ? data[c + 1] : text_len;
    return upper - data[c];
  }
};

// ---------------------------------------------------------------------------
// OccTable (src/occ/mod.rs:45-480)
// ---------------------------------------------------------------------------
static const uint8_t NO_LANE = 0xFF;

struct OccTable {
  uint8_t num_lanes = 0, num_planes = 0;
  uint8_t s2l[16], l2s[16];
  std::vector<uint32_t> sb;       // superblock_checkpoints
  std::vector<uint8_t> block_data;
  uint64_t block_stride = 0;
  uint32_t encoding = 0;          // 0 Bitplane, 1 OneHot
  uint32_t text_len = 0;

  const uint8_t* rec(uint64_t block) const { return block_data.data() + block * block_stride; }
  uint32_t sb_count_at(const uint8_t* r, int lane) const { return ld32(r + lane * 4); }
  uint32_t delta_at(const uint8_t* r, int lane) const { return ld16(r + num_lanes * 4 + lane * 2); }
  uint64_t word_at(const uint8_t* r, int w) const { return ld64(r + num_lanes * 6 + w * 8); }

  // lane_mask (src/occ/mod.rs:276-298)
  uint64_t lane_mask(const uint8_t* r, int lane) const {
    if (encoding == 1) { if (num_lanes == 0) return 0; return word_at(r, lane); }
    if (num_planes == 0) return ~0ull;
    uint64_t m = ~0ull;
    for (int p = 0; p < num_planes; p++) { uint64_t pv = word_at(r, p); m &= ((lane >> p) & 1) ? pv : ~pv; }
    return m;
  }
  // lane_at (src/occ/mod.rs:305-325)
  int lane_at(const uint8_t* r, uint32_t off) const {
    if (encoding == 1) {
      for (int l = 0; l < num_lanes; l++) if ((word_at(r, l) >> off) & 1) return l;
      return 0;
    }
    if (num_planes == 0) return 0;
    int lane = 0;
    for (int p = 0; p < num_planes; p++) lane |= (int)((word_at(r, p) >> off) & 1) << p;
    return lane;
  }
  // rank_at_lane (src/occ/mod.rs:346-363)
  uint32_t rank_at_lane(int lane, uint32_t i) const {
    uint32_t pos = i - 1; uint64_t block = pos / 64; uint32_t off = pos % 64;
    const uint8_t* r = rec(block);
    uint64_t bits = lane_mask(r, lane);
    uint64_t mask = (off == 63) ? ~0ull : ((1ull << (off + 1)) - 1);
    return sb_count_at(r, lane) + delta_at(r, lane) + (uint32_t)__builtin_popcountll(bits & mask);
  }
  // rank (src/occ/mod.rs:330-339)
  uint32_t rank(uint8_t c, uint32_t i) const {
    if (i == 0) return 0;
    uint8_t lane = s2l[c];
    if (lane == NO_LANE) return 0;
    return rank_at_lane(lane, i);
  }
  void prefetch_block(uint32_t pos) const {
    uint64_t base = (uint64_t)(pos / 64) * block_stride;
    if (base < block_data.size()) __builtin_prefetch(block_data.data() + base);
  }
  // rank_pair (src/occ/mod.rs:370-393)
  void rank_pair(uint8_t c, uint32_t lo, uint32_t hi, uint32_t& rlo, uint32_t& rhi) const {
    uint8_t lane = s2l[c];
    if (lane == NO_LANE) { rlo = rhi = 0; return; }
    if (lo) prefetch_block(lo - 1);
    if (hi) prefetch_block(hi - 1);
    rlo = lo == 0 ? 0 : rank_at_lane(lane, lo);
    rhi = hi == 0 ? 0 : rank_at_lane(lane, hi);
  }
  // lf_step (src/occ/mod.rs:456-480) with lane_and_mask_bitplane (:434-448)
  void lf_step(uint32_t pos, uint8_t& sym, uint32_t& rank_out) const {
    uint64_t block = pos / 64; uint32_t off = pos % 64;
    const uint8_t* r = rec(block);
    int lane; uint64_t bits;
    if (encoding == 0) {
      if (num_planes == 0) { lane = 0; bits = ~0ull; }
      else {
        lane = 0; bits = ~0ull;
        for (int p = 0; p < num_planes; p++) {
          uint64_t pv = word_at(r, p); uint64_t bit = (pv >> off) & 1;
          lane |= (int)bit << p; bits &= bit ? pv : ~pv;
        }
      }
    } else { lane = lane_at(r, off); bits = lane_mask(r, lane); }
    sym = l2s[lane];
    uint64_t mask = (1ull << off) - 1;
    rank_out = sb_count_at(r, lane) + delta_at(r, lane) + (uint32_t)__builtin_popcountll(bits & mask);
  }
};

// build_occ_table (src/occ/cpu.rs:23-119) followed by OccTable::from_parts (src/occ/mod.rs:114-183)
static OccTable build_occ(const std::vector<uint8_t>& bwt, uint32_t encoding) {
  uint32_t n = (uint32_t)bwt.size();
  uint64_t nblocks = (n + 63) / 64;
  std::vector<uint64_t> bits(nblocks * 16, 0);
  std::vector<uint32_t> cnts(nblocks * 16, 0);
  for (uint32_t pos = 0; pos < n; pos++) {
    uint8_t ch = bwt[pos];
    if (ch < 16) { bits[(pos / 64) * 16 + ch] |= 1ull << (pos % 64); cnts[(pos / 64) * 16 + ch]++; }
  }
  uint32_t totals[16] = {0};
  for (uint64_t b = 0; b < nblocks; b++) for (int c = 0; c < 16; c++) totals[c] += cnts[b * 16 + c];
  OccTable o;
  std::memset(o.s2l, NO_LANE, 16);
  uint8_t L = 0;
  for (int c = 0; c < 16; c++) if (totals[c] > 0) o.s2l[c] = L++;
  o.num_lanes = L;
  // num_planes_for (src/occ/mod.rs:100-106): u8::BITS - (L-1).leading_zeros(), 0 for L <= 1
  o.num_planes = 0;
  if (L > 1) { uint8_t v = L - 1; int lz = 0; for (int b = 7; b >= 0 && !((v >> b) & 1); b--) lz++; o.num_planes = (uint8_t)(8 - lz); }
  uint32_t width = (encoding == 0) ? o.num_planes : L;
  std::memset(o.l2s, 0, 16);
  for (int c = 0; c < 16; c++) if (o.s2l[c] != NO_LANE) o.l2s[o.s2l[c]] = (uint8_t)c;
  std::vector<uint16_t> deltas; deltas.reserve(nblocks * L);
  std::vector<uint64_t> lane_data; lane_data.reserve(nblocks * width);
  std::vector<uint32_t> cumulative(L, 0), sb_base(L, 0);
  for (uint64_t b = 0; b < nblocks; b++) {
    if (b % 8 == 0) { for (int l = 0; l < L; l++) o.sb.push_back(cumulative[l]); sb_base = cumulative; }
    std::vector<uint64_t> bl(width, 0);
    for (int c = 0; c < 16; c++) {
      uint8_t lane = o.s2l[c];
      if (lane == NO_LANE) continue;
      deltas.push_back((uint16_t)(cumulative[lane] - sb_base[lane]));
      if (encoding == 0) { for (uint32_t p = 0; p < width; p++) if ((lane >> p) & 1) bl[p] |= bits[b * 16 + c]; }
      else bl[lane] = bits[b * 16 + c];
      cumulative[lane] += cnts[b * 16 + c];
    }
    lane_data.insert(lane_data.end(), bl.begin(), bl.end());
  }
  // from_parts: interleave [sb u32 x L][delta u16 x L][words u64 x width]
  o.block_stride = (uint64_t)L * 4 + (uint64_t)L * 2 + (uint64_t)width * 8;
  uint64_t num_blocks = L ? deltas.size() / L : 0;
  o.block_data.assign(num_blocks * o.block_stride, 0);
  for (uint64_t b = 0; b < num_blocks; b++) {
    uint8_t* r = o.block_data.data() + b * o.block_stride;
    uint64_t sbi = b / 8;
    for (int l = 0; l < L; l++) { uint32_t v = o.sb[sbi * L + l]; std::memcpy(r + l * 4, &v, 4); }
    for (int l = 0; l < L; l++) { uint16_t v = deltas[b * L + l]; std::memcpy(r + L * 4 + l * 2, &v, 2); }
    for (uint32_t w = 0; w < width; w++) { uint64_t v = lane_data[b * width + w]; std::memcpy(r + L * 6 + w * 8, &v, 8); }
  }
  o.encoding = encoding;
  o.text_len = n;
  return o;
}

// ---------------------------------------------------------------------------
// SampledSuffixArray (src/suffix_array/mod.rs:54-201)
// ---------------------------------------------------------------------------
struct SSA {
  std::vector<uint8_t> word_data;   // 14-byte records: [u64 word][u32 sb][u16 delta]
  std::vector<uint32_t> sa_vals;
  uint32_t sample_rate = 0, text_len = 0;

  // get (src/suffix_array/mod.rs:185-201)
  bool get(uint32_t i, uint32_t& out) const {
    uint64_t w = i / 64; uint32_t bit = i % 64;
    const uint8_t* r = word_data.data() + w * 14;
    uint64_t word = ld64(r);
    if (!((word >> bit) & 1)) return false;
    uint64_t mask = bit == 0 ? 0 : ((1ull << bit) - 1);
    uint32_t rank = ld32(r + 8) + ld16(r + 12) + (uint32_t)__builtin_popcountll(word & mask);
    out = sa_vals[rank];
    return true;
  }
  void prefetch(uint32_t i) const {
    uint64_t off = (uint64_t)(i / 64) * 14;
    if (off < word_data.size()) __builtin_prefetch(word_data.data() + off);
  }
};

// SampledSuffixArray::from_full (src/suffix_array/mod.rs:71-118)
static SSA build_ssa(const std::vector<uint32_t>& sa, uint32_t rate, const std::vector<uint32_t>& forced_v) {
  SSA s;
  uint64_t n = sa.size(), nw = (n + 63) / 64;
  std::unordered_set<uint32_t> forced(forced_v.begin(), forced_v.end());
  std::vector<uint64_t> bv(nw, 0);
  for (uint64_t i = 0; i < n; i++) {
    uint32_t v = sa[i];
    bool mult = rate == 0 ? (v == 0) : (v % rate == 0);   // u32::is_multiple_of
    if (mult || forced.count(v)) { bv[i / 64] |= 1ull << (i % 64); s.sa_vals.push_back(v); }
  }
  s.word_data.assign(nw * 14, 0);
  uint32_t cum = 0, sbb = 0;
  for (uint64_t w = 0; w < nw; w++) {
    if (w % 8 == 0) sbb = cum;
    uint16_t delta = (uint16_t)(cum - sbb);
    uint8_t* r = s.word_data.data() + w * 14;
    std::memcpy(r, &bv[w], 8); std::memcpy(r + 8, &sbb, 4); std::memcpy(r + 12, &delta, 2);
    cum += (uint32_t)__builtin_popcountll(bv[w]);
  }
  s.sample_rate = rate; s.text_len = (uint32_t)n;
  return s;
}

// ---------------------------------------------------------------------------
// LookupTable (src/fm_index/lookup.rs:19-111)
// ---------------------------------------------------------------------------
struct Lookup {
  uint32_t depth = 0;
  std::vector<uint8_t> core;
  std::vector<std::pair<uint32_t, uint32_t>> intervals;
  // get (src/fm_index/lookup.rs:101-111)
  bool get(const uint8_t* codes, std::pair<uint32_t, uint32_t>& out) const {
    uint64_t radix = core.size(), idx = 0;
    for (int64_t k = (int64_t)depth - 1; k >= 0; k--) {
      int d = -1;
      for (size_t j = 0; j < core.size(); j++) if (core[j] == codes[k]) { d = (int)j; break; }
      if (d < 0) return false;
      idx = idx * radix + (uint64_t)d;
    }
    out = intervals[idx];
    return true;
  }
};

// LookupTable::build (src/fm_index/lookup.rs:37-91)
static Lookup build_lookup(uint32_t depth, uint32_t text_len, const CArray& c, const OccTable& occ,
                           const uint8_t* core, size_t ncore) {
  Lookup L; L.depth = depth; L.core.assign(core, core + ncore);
  uint64_t radix = ncore, size = 1;
  for (uint32_t i = 0; i < depth; i++) size *= radix;
  L.intervals.assign(size, {0, 0});
  struct E { uint64_t idx; uint32_t lo, hi; };
  std::vector<E> cur{{0, 0, text_len}}, next;
  for (uint32_t level = 1; level <= depth; level++) {
    next.clear();
    bool last = level == depth;
    for (const E& e : cur) {
      for (uint64_t d = 0; d < radix; d++) {
        uint64_t child = e.idx * radix + d;
        uint8_t sym = core[d];
        if (c.symbol_count(sym, text_len) == 0) continue;
        uint32_t cv = c.get(sym);
        uint32_t nlo = cv + occ.rank(sym, e.lo), nhi = cv + occ.rank(sym, e.hi);
        if (last) L.intervals[child] = {nlo, nhi};
        else if (nlo < nhi) next.push_back({child, nlo, nhi});
      }
    }
    if (!last) cur.swap(next);
  }
  return L;
}

// ---------------------------------------------------------------------------
// FmIndex (src/fm_index/mod.rs:58-72; query.rs)
// ---------------------------------------------------------------------------
struct Iv { uint32_t lo, hi; };

struct FmIndex {
  CArray c;
  OccTable occ;
  SSA ssa;
  uint32_t text_len = 0, num_sequences = 0;
  std::vector<uint32_t> seq_boundaries;
  std::vector<std::string> headers;
  bool has_lookup = false;
  Lookup lut;
  uint8_t tag = 0;

  const Compat& compat(uint8_t code) const {
    if (code >= 16) return EMPTY_COMPAT;
    return tag == 1 ? EXACT_COMPAT[code] : IUPAC_COMPAT[code];
  }

  // merge_intervals_inplace (src/fm_index/query.rs:390-407)
  static void merge(std::vector<Iv>& ivs) {
    std::sort(ivs.begin(), ivs.end(), [](const Iv& a, const Iv& b) { return a.lo < b.lo; });
    size_t w = 0; Iv cur = ivs[0];
    for (size_t r = 1; r < ivs.size(); r++) {
      if (ivs[r].lo <= cur.hi) cur.hi = std::max(cur.hi, ivs[r].hi);
      else { ivs[w++] = cur; cur = ivs[r]; }
    }
    ivs[w++] = cur; ivs.resize(w);
  }

  // backward_search (src/fm_index/query.rs:219-277)
  std::vector<Iv> backward_search(const uint8_t* p, size_t m) const {
    if (m == 0) return {{0, text_len}};
    std::vector<Iv> ivs; size_t start;
    if (has_lookup && m >= lut.depth) {
      std::pair<uint32_t, uint32_t> iv;
      if (lut.get(p + (m - lut.depth), iv)) {
        if (iv.first >= iv.second) return {};
        ivs.push_back({iv.first, iv.second}); start = m - lut.depth;
      } else { ivs.push_back({0, text_len}); start = m; }
    } else { ivs.push_back({0, text_len}); start = m; }
    std::vector<Iv> next; next.reserve(16);
    for (size_t k = start; k-- > 0;) {
      const Compat& cp = compat(p[k]);
      next.clear();
      for (const Iv& iv : ivs) {
        for (int j = 0; j < cp.len; j++) {
          uint8_t r = cp.sym[j];
          if (c.symbol_count(r, text_len) == 0) continue;
          uint32_t cv = c.get(r), rl, rh;
          occ.rank_pair(r, iv.lo, iv.hi, rl, rh);
          uint32_t nl = cv + rl, nh = cv + rh;
          if (nl < nh) next.push_back({nl, nh});
        }
      }
      if (next.size() > 1) merge(next);
      if (next.empty()) return {};
      ivs.swap(next);
    }
    return ivs;
  }

  // count (src/fm_index/query.rs:9-14)
  uint32_t count(const uint8_t* p, size_t m) const {
    uint32_t s = 0;
    for (const Iv& iv : backward_search(p, m)) s += iv.hi - iv.lo;
    return s;
  }

  // lf_mapping (src/fm_index/mod.rs:288-291)
  uint32_t lf(uint32_t i) const { uint8_t sym; uint32_t r; occ.lf_step(i, sym, r); return c.get(sym) + r; }

  // resolve_sa (src/fm_index/query.rs:282-291)
  uint32_t resolve_sa(uint32_t i) const {
    uint32_t steps = 0, v;
    for (;;) {
      if (ssa.get(i, v)) return v + steps;
      i = lf(i); steps++;
    }
  }

  // resolve_sa_batch (src/fm_index/query.rs:305-339): lockstep LF-walks with prefetch.
  void resolve_sa_batch(const std::vector<uint32_t>& rows, std::vector<uint32_t>& out) const {
    out.assign(rows.size(), 0);
    std::vector<uint32_t> cur(rows), steps(rows.size(), 0), active(rows.size()), nxt;
    for (uint32_t i = 0; i < rows.size(); i++) active[i] = i;
    nxt.reserve(rows.size());
    while (!active.empty()) {
      for (uint32_t l : active) { ssa.prefetch(cur[l]); occ.prefetch_block(cur[l]); }
      nxt.clear();
      for (uint32_t l : active) {
        uint32_t v;
        if (ssa.get(cur[l], v)) out[l] = v + steps[l];
        else { cur[l] = lf(cur[l]); steps[l]++; nxt.push_back(l); }
      }
      active.swap(nxt);
    }
  }

  // map_position (src/fm_index/query.rs:342-357)
  bool map_position(uint32_t p, uint32_t& seq, uint32_t& off) const {
    size_t idx = std::upper_bound(seq_boundaries.begin(), seq_boundaries.end(), p) - seq_boundaries.begin();
    if (idx >= seq_boundaries.size()) return false;
    uint32_t start = idx == 0 ? 0 : seq_boundaries[idx - 1];
    seq = (uint32_t)idx; off = p - start;
    return true;
  }
};

// BidirInterval (src/fm_index/bidir.rs:36-143)
struct BIv { uint32_t fwd_lo, fwd_hi, rev_lo, rev_hi; uint32_t size() const { return fwd_hi > fwd_lo ? fwd_hi - fwd_lo : 0; } };

// count_smaller_than (src/fm_index/bidir.rs:136-143)
static uint32_t count_smaller_than(uint8_t c, uint32_t lo, uint32_t hi, const FmIndex& idx) {
  uint32_t s = 0;
  for (int b = 0; b < std::min<int>(c, 16); b++) s += idx.occ.rank((uint8_t)b, hi) - idx.occ.rank((uint8_t)b, lo);
  return s;
}
// extend_right (src/fm_index/bidir.rs:80-100)
static bool extend_right(const BIv& iv, uint8_t c, const FmIndex& rev, BIv& out) {
  uint32_t cv = rev.c.get(c);
  uint32_t nl = cv + rev.occ.rank(c, iv.rev_lo), nh = cv + rev.occ.rank(c, iv.rev_hi);
  if (nl >= nh) return false;
  uint32_t off = count_smaller_than(c, iv.rev_lo, iv.rev_hi, rev);
  uint32_t sz = nh - nl;
  out = {iv.fwd_lo + off, iv.fwd_lo + off + sz, nl, nh};
  return true;
}
// extend_left (src/fm_index/bidir.rs:112-130)
static bool extend_left(const BIv& iv, uint8_t c, const FmIndex& fwd, BIv& out) {
  uint32_t cv = fwd.c.get(c);
  uint32_t nl = cv + fwd.occ.rank(c, iv.fwd_lo), nh = cv + fwd.occ.rank(c, iv.fwd_hi);
  if (nl >= nh) return false;
  uint32_t off = count_smaller_than(c, iv.fwd_lo, iv.fwd_hi, fwd);
  uint32_t sz = nh - nl;
  out = {nl, nh, iv.rev_lo + off, iv.rev_lo + off + sz};
  return true;
}

struct RawMem { uint32_t qs, qe, count; std::vector<BIv> ivs; };

struct Bidir {
  FmIndex fwd, rev;
  BIv full() const { return {0, fwd.text_len, 0, fwd.text_len}; }

  // extend_multi_right / extend_multi_left (src/fm_index/smem.rs:332-357)
  std::vector<BIv> multi_right(const std::vector<BIv>& ivs, uint8_t c) const {
    std::vector<BIv> out; const Compat& cp = rev.compat(c);
    for (int j = 0; j < cp.len; j++) for (const BIv& iv : ivs) { BIv e; if (extend_right(iv, cp.sym[j], rev, e)) out.push_back(e); }
    return out;
  }
  std::vector<BIv> multi_left(const std::vector<BIv>& ivs, uint8_t c) const {
    std::vector<BIv> out; const Compat& cp = fwd.compat(c);
    for (int j = 0; j < cp.len; j++) for (const BIv& iv : ivs) { BIv e; if (extend_left(iv, cp.sym[j], fwd, e)) out.push_back(e); }
    return out;
  }
  static uint32_t coverage(const std::vector<BIv>& ivs) { uint32_t s = 0; for (auto& i : ivs) s += i.size(); return s; }

  // extend_left_maximally (src/fm_index/smem.rs:227-243)
  std::vector<BIv> left_max(std::vector<BIv> ivs, const uint8_t* q, size_t from, size_t& start) const {
    start = from;
    while (start > 0) {
      std::vector<BIv> nx = multi_left(ivs, q[start - 1]);
      if (nx.empty()) break;
      ivs.swap(nx); start--;
    }
    return ivs;
  }

  // collect_smem_candidates (src/fm_index/smem.rs:154-222), one pivot of its loop:
  // appends the pivot's candidates (and, when piv is given, the pivot of each) and returns
  // the next pivot.
  size_t pivot_step(const uint8_t* q, size_t n, size_t min_len, size_t pivot, std::vector<RawMem>& out,
                    std::vector<size_t>* piv) const {
    std::vector<BIv> curr = multi_right({full()}, q[pivot]);
    if (curr.empty()) return pivot + 1;
    uint32_t cov = coverage(curr);
    std::vector<std::pair<std::vector<BIv>, size_t>> prefixes;
    size_t j = pivot + 1;
    for (;;) {
      if (j == n) { prefixes.push_back({curr, n}); break; }
      std::vector<BIv> nx = multi_right(curr, q[j]);
      uint32_t ncov = coverage(nx);
      if (ncov != cov) prefixes.push_back({curr, j});
      if (nx.empty()) break;
      curr.swap(nx); cov = ncov; j++;
    }
    size_t reach = prefixes.empty() ? pivot + 1 : prefixes.back().second;
    for (auto& pr : prefixes) {
      size_t start;
      std::vector<BIv> b = left_max(pr.first, q, pivot, start);
      size_t end = pr.second;
      if (end - start < min_len) continue;
      bool rmax = end == n || multi_right(b, q[end]).empty();
      if (!rmax) continue;
      out.push_back({(uint32_t)start, (uint32_t)end, coverage(b), std::move(b)});
      if (piv) piv->push_back(pivot);
    }
    return std::max(reach, pivot + 1);
  }

  std::vector<RawMem> smem_candidates(const uint8_t* q, size_t n, size_t min_len) const {
    std::vector<RawMem> out;
    size_t pivot = 0;
    while (pivot < n) pivot = pivot_step(q, n, min_len, pivot, out, nullptr);
    return out;
  }

  // raw_mem_from (src/fm_index/smem.rs:250-295)
  bool raw_mem_from(const uint8_t* q, size_t n, size_t i, size_t min_len, RawMem& out) const {
    std::vector<BIv> ivs{full()};
    size_t j = i; bool matched = false;
    while (j < n) {
      std::vector<BIv> nx = multi_right(ivs, q[j]);
      if (nx.empty()) break;
      ivs.swap(nx); j++; matched = true;
    }
    if (!matched) return false;
    if (j - i < min_len) return false;
    bool lmax = i == 0 || multi_left(ivs, q[i - 1]).empty();
    if (!lmax) return false;
    out = {(uint32_t)i, (uint32_t)j, coverage(ivs), std::move(ivs)};
    return true;
  }

  static void sort_dedup(std::vector<RawMem>& raws) {
    std::stable_sort(raws.begin(), raws.end(), [](const RawMem& a, const RawMem& b) {
      return a.qs != b.qs ? a.qs < b.qs : a.qe < b.qe; });
    std::vector<RawMem> d;
    for (auto& r : raws) if (d.empty() || d.back().qs != r.qs || d.back().qe != r.qe) d.push_back(std::move(r));
    raws.swap(d);
  }

  // find_smems without positions (src/fm_index/smem.rs:71-104)
  std::vector<RawMem> find_smems(const uint8_t* q, size_t n, size_t min_len) const {
    if (n == 0 || min_len == 0) return {};
    return filter_smems(smem_candidates(q, n, min_len));
  }
  static std::vector<RawMem> filter_smems(std::vector<RawMem> raws) {
    sort_dedup(raws);
    std::vector<RawMem> out;
    for (size_t i = 0; i < raws.size(); i++) {
      bool contained = false;
      for (size_t j = 0; j < raws.size() && !contained; j++)
        if (j != i && raws[j].qs <= raws[i].qs && raws[i].qe <= raws[j].qe &&
            !(raws[j].qs == raws[i].qs && raws[j].qe == raws[i].qe)) contained = true;
      if (!contained) out.push_back(raws[i]);
    }
    return out;
  }
  // find_mems without positions (src/fm_index/smem.rs:113-124)
  std::vector<RawMem> find_mems(const uint8_t* q, size_t n, size_t min_len) const {
    if (n == 0 || min_len == 0) return {};
    std::vector<RawMem> raws;
    for (size_t i = 0; i < n; i++) { RawMem r; if (raw_mem_from(q, n, i, min_len, r)) raws.push_back(std::move(r)); }
    sort_dedup(raws);
    return raws;
  }
};

// ---------------------------------------------------------------------------
// bincode 1 (fixint, little endian) reader / writer for FmIndex
// (src/fm_index/serialize.rs:55-80; field layouts src/occ/mod.rs:45-78,
//  src/suffix_array/mod.rs:54-63, src/fm_index/lookup.rs:19-27)
// ---------------------------------------------------------------------------
struct Rd {
  const uint8_t* p; uint64_t n, i = 0; bool bad = false;
  bool need(uint64_t k) { if (bad || n - i < k) { bad = true; return false; } return true; }
  uint8_t u8() { if (!need(1)) return 0; return p[i++]; }
  uint32_t u32() { if (!need(4)) return 0; uint32_t v = ld32(p + i); i += 4; return v; }
  uint64_t u64() { if (!need(8)) return 0; uint64_t v = ld64(p + i); i += 8; return v; }
  void raw(uint8_t* d, uint64_t k) { if (!need(k)) return; std::memcpy(d, p + i, k); i += k; }
  template <class T> void vec(std::vector<T>& v) {
    uint64_t len = u64(); if (bad) return;
    if (len > (n - i) / sizeof(T)) { bad = true; return; }
    v.resize(len); if (len) std::memcpy(v.data(), p + i, len * sizeof(T)); i += len * sizeof(T);
  }
};

static bool parse_fm(const uint8_t* p, uint64_t n, FmIndex& f) {
  Rd r{p, n};
  for (int k = 0; k < 16; k++) f.c.data[k] = r.u32();
  OccTable& o = f.occ;
  o.num_lanes = r.u8(); o.num_planes = r.u8();
  r.raw(o.s2l, 16); r.raw(o.l2s, 16);
  r.vec(o.sb); r.vec(o.block_data);
  o.block_stride = r.u64();
  o.encoding = r.u32(); if (o.encoding > 1) { g_err = "invalid OccEncoding variant"; return false; }
  o.text_len = r.u32();
  r.vec(f.ssa.word_data); r.vec(f.ssa.sa_vals);
  f.ssa.sample_rate = r.u32(); f.ssa.text_len = r.u32();
  f.text_len = r.u32(); f.num_sequences = r.u32();
  r.vec(f.seq_boundaries);
  uint64_t nh = r.u64();
  if (r.bad) { g_err = "truncated"; return false; }
  f.headers.clear();
  for (uint64_t k = 0; k < nh && !r.bad; k++) {
    uint64_t len = r.u64(); if (!r.need(len)) break;
    f.headers.emplace_back((const char*)p + r.i, (size_t)len); r.i += len;
  }
  uint8_t opt = r.u8();
  if (opt == 1) {
    f.has_lookup = true; f.lut.depth = r.u32(); r.vec(f.lut.core);
    uint64_t len = r.u64();
    if (!r.bad && len <= (r.n - r.i) / 8) {
      f.lut.intervals.resize(len);
      for (uint64_t k = 0; k < len; k++) { f.lut.intervals[k].first = r.u32(); f.lut.intervals[k].second = r.u32(); }
    } else r.bad = true;
  } else if (opt != 0) { g_err = "invalid Option tag"; return false; }
  f.tag = r.u8();
  if (r.bad) { g_err = "truncated"; return false; }
  if (f.tag > 1) { g_err = "unknown alphabet tag"; return false; }   // alphabet_fns_from_tag
  return true;
}

struct Wr {
  std::vector<uint8_t> b;
  void u8(uint8_t v) { b.push_back(v); }
  void u32(uint32_t v) { uint8_t t[4]; std::memcpy(t, &v, 4); b.insert(b.end(), t, t + 4); }
  void u64(uint64_t v) { uint8_t t[8]; std::memcpy(t, &v, 8); b.insert(b.end(), t, t + 8); }
  void raw(const void* d, uint64_t k) { const uint8_t* s = (const uint8_t*)d; b.insert(b.end(), s, s + k); }
  template <class T> void vec(const std::vector<T>& v) { u64(v.size()); raw(v.data(), v.size() * sizeof(T)); }
};

static void write_fm(const FmIndex& f, Wr& w) {
  for (int k = 0; k < 16; k++) w.u32(f.c.data[k]);
  const OccTable& o = f.occ;
  w.u8(o.num_lanes); w.u8(o.num_planes); w.raw(o.s2l, 16); w.raw(o.l2s, 16);
  w.vec(o.sb); w.vec(o.block_data); w.u64(o.block_stride); w.u32(o.encoding); w.u32(o.text_len);
  w.vec(f.ssa.word_data); w.vec(f.ssa.sa_vals); w.u32(f.ssa.sample_rate); w.u32(f.ssa.text_len);
  w.u32(f.text_len); w.u32(f.num_sequences); w.vec(f.seq_boundaries);
  w.u64(f.headers.size());
  for (auto& h : f.headers) { w.u64(h.size()); w.raw(h.data(), h.size()); }
  if (f.has_lookup) {
    w.u8(1); w.u32(f.lut.depth); w.vec(f.lut.core); w.u64(f.lut.intervals.size());
    for (auto& iv : f.lut.intervals) { w.u32(iv.first); w.u32(iv.second); }
  } else w.u8(0);
  w.u8(f.tag);
}

// ---------------------------------------------------------------------------
// Construction (oracle tooling; src/fm_index/mod.rs:117-195, src/bwt/cpu.rs:14-35)
// ---------------------------------------------------------------------------
static std::vector<uint32_t> naive_sa(const std::vector<uint8_t>& t) {
  // build_suffix_array_naive (src/suffix_array/cpu.rs:20-25): Rust slice ordering.
  std::vector<uint32_t> sa(t.size());
  for (uint32_t i = 0; i < sa.size(); i++) sa[i] = i;
  const uint8_t* d = t.data(); size_t n = t.size();
  std::sort(sa.begin(), sa.end(), [d, n](uint32_t a, uint32_t b) {
    size_t la = n - a, lb = n - b, l = std::min(la, lb);
    int c = std::memcmp(d + a, d + b, l);
    if (c != 0) return c < 0;
    return la < lb;
  });
  return sa;
}

// Parallel LSD radix sort of (key, value) pairs on the low `bits` bits of the keys; passes
// whose digit is the same for every key are skipped.
static void radix_sort_pairs(std::vector<uint64_t>& key, std::vector<uint32_t>& val, int bits, int threads) {
  const uint64_t n = key.size();
  std::vector<uint64_t> k2(n);
  std::vector<uint32_t> v2(n);
  threads = std::max(1, std::min<int>(threads, (int)std::max<uint64_t>(1, n >> 16)));
  const uint64_t per = (n + threads - 1) / threads;
  std::vector<uint64_t> hist((size_t)threads * 256);
  for (int shift = 0; shift < bits; shift += 8) {
    std::fill(hist.begin(), hist.end(), 0);
    std::vector<std::thread> th;
    for (int t = 0; t < threads; t++)
      th.emplace_back([&, t] {
        uint64_t a = t * per, b = std::min(n, a + per);
        uint64_t* h = &hist[(size_t)t * 256];
        for (uint64_t i = a; i < b; i++) h[(key[i] >> shift) & 255]++;
      });
    for (auto& x : th) x.join();
    th.clear();
    int nonzero = 0;
    for (int d = 0; d < 256; d++) {
      uint64_t s = 0;
      for (int t = 0; t < threads; t++) s += hist[(size_t)t * 256 + d];
      nonzero += s != 0;
    }
    if (nonzero <= 1) continue;                  // every key has this digit
    uint64_t run = 0;                            // digit-major, thread-minor offsets: stable
    for (int d = 0; d < 256; d++)
      for (int t = 0; t < threads; t++) { uint64_t c = hist[(size_t)t * 256 + d]; hist[(size_t)t * 256 + d] = run; run += c; }
    for (int t = 0; t < threads; t++)
      th.emplace_back([&, t] {
        uint64_t a = t * per, b = std::min(n, a + per);
        uint64_t* h = &hist[(size_t)t * 256];
        for (uint64_t i = a; i < b; i++) {
          uint64_t o = h[(key[i] >> shift) & 255]++;
          k2[o] = key[i]; v2[o] = val[i];
        }
      });
    for (auto& x : th) x.join();
    key.swap(k2); val.swap(v2);
  }
}

// Suffix array by prefix doubling (Manber & Myers 1993, refining only the groups that are
// still tied, as Larsson & Sadakane 2007 do).  It is an algorithm independent of the
// product's SA-IS builder, so an index built here checks that builder at scale.  The
// order is true lexicographic order of the code slices with a proper prefix first — the
// order of build_suffix_array_naive (src/suffix_array/cpu.rs:20-25), which `naive_sa`
// above computes by comparison; the two are compared in the oracle's own tests.
static std::vector<uint32_t> doubling_sa(const std::vector<uint8_t>& t, int threads) {
  const uint64_t n = t.size();
  std::vector<uint32_t> sa(n);
  if (n == 0) return sa;
  threads = std::max(1, threads);
  constexpr int K = 12;                          // 12 symbols of 5 bits: code + 1, 0 past the end
  std::vector<uint64_t> key(n);
  auto par = [&](uint64_t m, auto f) {
    int nt = (int)std::min<uint64_t>((uint64_t)threads, std::max<uint64_t>(1, m >> 14));
    uint64_t per = (m + nt - 1) / nt;
    std::vector<std::thread> th;
    for (int q = 0; q < nt; q++) th.emplace_back([&, q] { f(q * per, std::min(m, q * per + per)); });
    for (auto& x : th) x.join();
  };
  par(n, [&](uint64_t a, uint64_t b) {
    for (uint64_t i = a; i < b; i++) {
      uint64_t k = 0;
      for (int j = 0; j < K; j++) k = (k << 5) | (i + j < n ? (uint64_t)t[i + j] + 1 : 0);
      key[i] = k; sa[i] = (uint32_t)i;
    }
  });
  radix_sort_pairs(key, sa, 5 * K, threads);
  // rank = 1 + index of the last member of the suffix's group (0 is "past the end")
  std::vector<uint32_t> rank(n);
  std::vector<std::pair<uint32_t, uint32_t>> groups;   // [a, b) still tied
  {
    uint64_t a = 0;
    for (uint64_t j = 1; j <= n; j++)
      if (j == n || key[j] != key[a]) {
        for (uint64_t q = a; q < j; q++) rank[sa[q]] = (uint32_t)j;
        if (j - a > 1) groups.push_back({(uint32_t)a, (uint32_t)j});
        a = j;
      }
  }
  std::vector<uint64_t>().swap(key);
  std::vector<uint32_t> next_rank;
  for (uint64_t h = K; !groups.empty(); h *= 2) {
    next_rank = rank;                            // reads use this round's ranks only
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> out(threads);
    std::atomic<size_t> gi{0};
    std::vector<std::thread> th;
    for (int q = 0; q < threads; q++)
      th.emplace_back([&, q] {
        std::vector<std::pair<uint32_t, uint32_t>> tmp;
        for (size_t g; (g = gi.fetch_add(1)) < groups.size();) {
          uint32_t a = groups[g].first, b = groups[g].second;
          tmp.clear();
          for (uint32_t j = a; j < b; j++) {
            uint64_t i = sa[j];
            tmp.push_back({i + h < n ? rank[i + h] : 0u, (uint32_t)i});
          }
          std::sort(tmp.begin(), tmp.end());
          uint32_t s = 0;
          for (uint32_t j = 1; j <= b - a; j++)
            if (j == b - a || tmp[j].first != tmp[s].first) {
              for (uint32_t u = s; u < j; u++) { sa[a + u] = tmp[u].second; next_rank[tmp[u].second] = a + j; }
              if (j - s > 1) out[q].push_back({a + s, a + j});
              s = j;
            }
        }
      });
    for (auto& x : th) x.join();
    rank.swap(next_rank);
    groups.clear();
    for (auto& o : out) groups.insert(groups.end(), o.begin(), o.end());
  }
  return sa;
}

static int g_build_threads = 1;   // threads of the oracle's index construction

static FmIndex build_fm(const std::vector<uint8_t>& text, const std::vector<uint32_t>& bounds,
                        const std::vector<std::string>& headers, uint32_t rate, uint32_t lookup_depth,
                        uint8_t tag, uint32_t encoding) {
  FmIndex f;
  f.tag = tag;
  f.text_len = (uint32_t)text.size();
  f.num_sequences = (uint32_t)bounds.size();
  f.seq_boundaries = bounds;
  f.headers = headers;
  f.c = CArray::from_text(text);
  std::vector<uint32_t> sa = doubling_sa(text, g_build_threads);
  uint64_t n = text.size();
  std::vector<uint8_t> bwt(n);
  for (uint64_t i = 0; i < n; i++) bwt[i] = text[sa[i] == 0 ? n - 1 : sa[i] - 1];
  std::vector<uint32_t> starts{0};
  for (size_t k = 0; k + 1 < bounds.size(); k++) starts.push_back(bounds[k]);
  f.ssa = build_ssa(sa, rate, starts);
  f.occ = build_occ(bwt, encoding);
  if (lookup_depth > 0) { f.has_lookup = true; f.lut = build_lookup(lookup_depth, f.text_len, f.c, f.occ, CORE_SYMBOLS, 4); }
  return f;
}

struct Handle { int kind; FmIndex fm; Bidir bd; const FmIndex& fwd() const { return kind ? bd.fwd : fm; } };

}  // namespace orc

using namespace orc;

// ---------------------------------------------------------------------------
// C API used by tests (ctypes).  All outputs are malloc'd; free with orc_free.
// ---------------------------------------------------------------------------
template <class T> static T* dup_out(const std::vector<T>& v) {
  T* p = (T*)std::malloc(std::max<size_t>(1, v.size() * sizeof(T)));
  if (!v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}

template <class F> static void par_for(uint32_t nq, int threads, F f) {
  if (threads <= 1 || nq < 2) { f(0u, nq, 0); return; }
  std::vector<std::thread> th; uint32_t per = (nq + threads - 1) / threads;
  for (int t = 0; t < threads; t++) {
    uint32_t a = t * per, b = std::min(nq, a + per);
    if (a >= b) break;
    th.emplace_back(f, a, b, t);
  }
  for (auto& x : th) x.join();
}

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }
void orc_free(void* p) { std::free(p); }


// Build FmIndex (kind 0) or BidirFmIndex (kind 1) bincode bytes from encoded sequences.
// codes: concatenated sequence codes; seq_off[nseq+1]; headers: nseq C strings or NULL.
int orc_build(const uint8_t* codes, const uint64_t* seq_off, uint32_t nseq, const char* const* headers,
              uint32_t rate, uint32_t lookup_depth, uint8_t tag, uint32_t encoding, int kind,
              uint8_t** out, uint64_t* out_len) {
  if (nseq == 0) { g_err = "empty sequence list"; return -4; }
  // concatenate_sequences (src/alphabet.rs:375-393)
  std::vector<uint8_t> text; std::vector<uint32_t> bounds; std::vector<std::string> hs;
  for (uint32_t s = 0; s < nseq; s++) {
    text.insert(text.end(), codes + seq_off[s], codes + seq_off[s + 1]);
    text.push_back(0);
    bounds.push_back((uint32_t)text.size());
    std::string h = headers && headers[s] ? headers[s] : "";
    hs.push_back(h.empty() ? "seq_" + std::to_string(s) : h);
  }
  Wr w;
  FmIndex fwd = build_fm(text, bounds, hs, rate, lookup_depth, tag, encoding);
  if (kind == 0) write_fm(fwd, w);
  else {
    // BidirFmIndex::build_cpu_with (src/fm_index/bidir_index.rs:53-80) + reverse_as_sequence (:523-532)
    std::vector<uint8_t> rt(text.begin(), text.end() - 1);
    std::reverse(rt.begin(), rt.end());
    rt.push_back(0);
    FmIndex rev = build_fm(rt, {(uint32_t)rt.size()}, {"seq_0"}, rate, 0, tag, encoding);
    Wr wf, wr; write_fm(fwd, wf); write_fm(rev, wr);
    // to_bytes (src/fm_index/bidir_index.rs:183-192): [u32 LE fwd_len][fwd][rev]
    w.u32((uint32_t)wf.b.size()); w.raw(wf.b.data(), wf.b.size()); w.raw(wr.b.data(), wr.b.size());
  }
  *out = dup_out(w.b); *out_len = w.b.size();
  return 0;
}

void* orc_load(const uint8_t* bytes, uint64_t len, int kind) {
  Handle* h = new Handle(); h->kind = kind;
  bool ok;
  if (kind == 0) ok = parse_fm(bytes, len, h->fm);
  else {
    // from_bytes (src/fm_index/bidir_index.rs:195-210)
    if (len < 4) { g_err = "truncated bidirectional index"; delete h; return nullptr; }
    uint32_t fl = ld32(bytes);
    if (len < 4ull + fl) { g_err = "truncated forward index"; delete h; return nullptr; }
    ok = parse_fm(bytes + 4, fl, h->bd.fwd) && parse_fm(bytes + 4 + fl, len - 4 - fl, h->bd.rev);
  }
  if (!ok) { delete h; return nullptr; }
  return h;
}
void orc_index_free(void* h) { delete (Handle*)h; }
uint32_t orc_text_len(void* h) { return ((Handle*)h)->fwd().text_len; }
uint32_t orc_num_sequences(void* h) { return ((Handle*)h)->fwd().num_sequences; }

// Re-serialise (round trip check of the reader/writer pair).
int orc_to_bytes(void* hv, uint8_t** out, uint64_t* out_len) {
  Handle* h = (Handle*)hv; Wr w;
  if (h->kind == 0) write_fm(h->fm, w);
  else { Wr wf, wr; write_fm(h->bd.fwd, wf); write_fm(h->bd.rev, wr);
         w.u32((uint32_t)wf.b.size()); w.raw(wf.b.data(), wf.b.size()); w.raw(wr.b.data(), wr.b.size()); }
  *out = dup_out(w.b); *out_len = w.b.size();
  return 0;
}

// Raw structure access for white-box tests.
int orc_rank(void* hv, int which, uint8_t c, uint32_t i, uint32_t* out) {
  Handle* h = (Handle*)hv; const FmIndex& f = which == 1 ? h->bd.rev : h->fwd();
  *out = f.occ.rank(c, i); return 0;
}
int orc_resolve_rows(void* hv, const uint32_t* rows, uint64_t n, uint32_t* out) {
  Handle* h = (Handle*)hv;
  for (uint64_t k = 0; k < n; k++) out[k] = h->fwd().resolve_sa(rows[k]);
  return 0;
}


// count for a batch (FmIndex::count, src/fm_index/query.rs:9-14)
int orc_count_batch(void* hv, const uint8_t* q, const uint64_t* qo, uint32_t nq, uint32_t* out, int threads) {
  Handle* h = (Handle*)hv; const FmIndex& f = h->fwd();
  par_for(nq, threads, [&](uint32_t a, uint32_t b, int) {
    for (uint32_t i = a; i < b; i++) out[i] = f.count(q + qo[i], qo[i + 1] - qo[i]);
  });
  return 0;
}

// locate for a batch (FmIndex::locate, src/fm_index/query.rs:22-39): CPU order (merged
// intervals ascending, rows ascending), each hit as (seq_idx, pos_in_seq).  max_hits > 0
// keeps the first max_hits rows of every merged interval (the declared cap extension);
// 0 = every row.  counts_out gets the exact count.
int orc_locate_batch(void* hv, const uint8_t* q, const uint64_t* qo, uint32_t nq, uint32_t max_hits,
                     int threads, uint32_t* counts_out, uint64_t** offsets_out, uint32_t** pairs_out,
                     uint64_t* total_out) {
  Handle* h = (Handle*)hv; const FmIndex& f = h->fwd();
  int T = std::max(1, threads);
  std::vector<std::vector<uint32_t>> part(T);
  std::vector<uint64_t> nhit(nq);
  par_for(nq, T, [&](uint32_t a, uint32_t b, int t) {
    std::vector<uint32_t> rows, res;
    for (uint32_t i = a; i < b; i++) {
      std::vector<Iv> ivs = f.backward_search(q + qo[i], qo[i + 1] - qo[i]);
      rows.clear(); uint32_t cnt = 0;
      for (const Iv& iv : ivs) {
        cnt += iv.hi - iv.lo;
        uint32_t take = iv.hi - iv.lo;
        if (max_hits && take > max_hits) take = max_hits;
        for (uint32_t r = iv.lo; r < iv.lo + take; r++) rows.push_back(r);
      }
      counts_out[i] = cnt;
      f.resolve_sa_batch(rows, res);
      nhit[i] = res.size();
      for (uint32_t p : res) {
        uint32_t s, o;
        if (!f.map_position(p, s, o)) { s = 0xFFFFFFFFu; o = 0xFFFFFFFFu; }
        part[t].push_back(s); part[t].push_back(o);
      }
    }
  });
  std::vector<uint64_t> off(nq + 1, 0);
  for (uint32_t i = 0; i < nq; i++) off[i + 1] = off[i] + nhit[i];
  std::vector<uint32_t> pairs; pairs.reserve(off[nq] * 2);
  for (auto& p : part) pairs.insert(pairs.end(), p.begin(), p.end());
  *offsets_out = dup_out(off); *pairs_out = dup_out(pairs); *total_out = off[nq];
  return 0;
}

// find_smems / find_mems (mode 0 / 1) with the reference's GPU MemHit contract
// (src/fm_index/bidir_index.rs:391-514): one hit per SA interval of each CPU MEM,
// hits of one MEM in ascending fwd_lo order, positions = rows fwd_lo ..
// fwd_lo+min(size,max_hits) resolved by resolve_sa and mapped to (ref_id, offset)
// against ref_bounds (ref_map.wgsl:32-59); no positions when n_bounds == 0.
// hits: 8 u32 per hit = [qs, qe, match_count, truncated, fwd_lo, n_pos, pos_off_lo, pos_off_hi].
int orc_mems_batch(void* hv, const uint8_t* q, const uint64_t* qo, uint32_t nq, uint32_t min_len,
                   uint32_t mode, const uint32_t* rb, uint32_t nb, uint32_t max_hits, int threads,
                   uint64_t** hit_off_out, uint32_t** hits_out, uint64_t* nhits_out,
                   uint32_t** pos_out, uint64_t* npos_out) {
  Handle* h = (Handle*)hv;
  if (h->kind != 1) { g_err = "mems need a bidirectional index"; return -4; }
  const Bidir& bd = h->bd;
  int T = std::max(1, threads);
  struct Part { std::vector<uint32_t> hits; std::vector<uint32_t> pos; };
  std::vector<Part> part(T);
  std::vector<uint64_t> nh(nq);
  par_for(nq, T, [&](uint32_t a, uint32_t b, int t) {
    std::vector<uint32_t> rows, res;
    for (uint32_t i = a; i < b; i++) {
      const uint8_t* qq = q + qo[i]; size_t n = qo[i + 1] - qo[i];
      std::vector<RawMem> ms = mode == 0 ? bd.find_smems(qq, n, min_len) : bd.find_mems(qq, n, min_len);
      uint64_t cnt = 0;
      for (RawMem& m : ms) {
        std::vector<BIv> ivs = m.ivs;
        std::stable_sort(ivs.begin(), ivs.end(), [](const BIv& x, const BIv& y) { return x.fwd_lo < y.fwd_lo; });
        for (const BIv& iv : ivs) {
          uint32_t raw = iv.size();
          uint32_t eff = nb ? std::min(raw, max_hits) : 0;
          part[t].hits.insert(part[t].hits.end(), {m.qs, m.qe, raw, (uint32_t)(raw > max_hits), iv.fwd_lo, eff, 0u, 0u});
          rows.clear();
          for (uint32_t r = 0; r < eff; r++) rows.push_back(iv.fwd_lo + r);
          bd.fwd.resolve_sa_batch(rows, res);
          for (uint32_t p : res) {
            size_t rid = std::upper_bound(rb, rb + nb, p) - rb;
            uint32_t start = rid == 0 ? 0 : rb[rid - 1];
            part[t].pos.push_back((uint32_t)rid); part[t].pos.push_back(p - start);
          }
          cnt++;
        }
      }
      nh[i] = cnt;
    }
  });
  std::vector<uint64_t> off(nq + 1, 0);
  for (uint32_t i = 0; i < nq; i++) off[i + 1] = off[i] + nh[i];
  std::vector<uint32_t> hits, pos;
  for (auto& p : part) { hits.insert(hits.end(), p.hits.begin(), p.hits.end()); pos.insert(pos.end(), p.pos.begin(), p.pos.end()); }
  uint64_t po = 0;
  for (uint64_t k = 0; k < off[nq]; k++) {
    hits[k * 8 + 6] = (uint32_t)po; hits[k * 8 + 7] = (uint32_t)(po >> 32);
    po += hits[k * 8 + 5];
  }
  *hit_off_out = dup_out(off); *hits_out = dup_out(hits); *nhits_out = off[nq];
  *pos_out = dup_out(pos); *npos_out = pos.size() / 2;
  return 0;
}

// find_smems / find_mems with the CPU Mem semantics (src/fm_index/smem.rs:18-28,71-124,
// 299-315): one Mem per (qs,qe) with every position (seq_idx, pos) in extension order
// when locate != 0.  mems: 4 u32 per Mem = [qs, qe, match_count, n_positions].
int orc_mems_native(void* hv, const uint8_t* q, uint64_t n, uint32_t min_len, uint32_t mode, int locate,
                    uint32_t** mems_out, uint64_t* nmems_out, uint32_t** pos_out, uint64_t* npos_out) {
  Handle* h = (Handle*)hv;
  if (h->kind != 1) { g_err = "mems need a bidirectional index"; return -4; }
  const Bidir& bd = h->bd;
  std::vector<RawMem> ms = mode == 0 ? bd.find_smems(q, n, min_len) : bd.find_mems(q, n, min_len);
  std::vector<uint32_t> mem, pos;
  for (RawMem& m : ms) {
    uint32_t np = 0;
    if (locate) {
      // locate_raw -> locate_interval (src/fm_index/bidir_index.rs:157-168)
      for (const BIv& iv : m.ivs) for (uint32_t r = iv.fwd_lo; r < iv.fwd_hi; r++) {
        uint32_t p = bd.fwd.resolve_sa(r), s, o;
        if (!bd.fwd.map_position(p, s, o)) { s = o = 0xFFFFFFFFu; }
        pos.push_back(s); pos.push_back(o); np++;
      }
    }
    mem.insert(mem.end(), {m.qs, m.qe, m.count, np});
  }
  *mems_out = dup_out(mem); *nmems_out = ms.size(); *pos_out = dup_out(pos); *npos_out = pos.size() / 2;
  return 0;
}

// ---- check of the library's segmented SMEM sweep (no counterpart in the reference) ----
// The library cuts reads longer than 2 * seg_len into seg_len-position segments, sweeps
// the pivot chain of each segment from its first position, sweeps each segment again from
// the previous segment's exit pivot until that chain meets the segment's own, and merges
// along the true chain (haystackfm_b200/csrc/search.cuh, k_mems_seg / k_mems_fix /
// k_mems_merge).  This restates those three steps on the oracle's own pivot step so that
// the CPU suite can show the candidate set equals the whole-read sweep's.
static std::vector<RawMem> segmented_candidates(const Bidir& bd, const uint8_t* q, size_t n, size_t min_len,
                                                size_t seg) {
  const size_t NONE = ~(size_t)0;
  size_t U = (n + seg - 1) / seg;
  struct Unit {
    std::vector<char> seen; size_t exit = 0;
    std::vector<RawMem> c; std::vector<size_t> piv;
    size_t fx_entry = NONE, fx_conv = NONE, fx_exit = NONE; std::vector<RawMem> fc;
  };
  std::vector<Unit> u(U);
  for (size_t k = 0; k < U; k++) {                 // segment sweeps
    size_t s = k * seg, e = std::min(n, s + seg);
    u[k].seen.assign(e - s, 0);
    size_t p = s;
    while (p < e) { u[k].seen[p - s] = 1; p = bd.pivot_step(q, n, min_len, p, u[k].c, &u[k].piv); }
    u[k].exit = p;
  }
  for (size_t k = 1; k < U; k++) {                 // fix-up sweeps from the previous exit
    size_t s = k * seg, e = std::min(n, s + seg), entry = u[k - 1].exit;
    u[k].fx_entry = entry;
    if (entry >= e) { u[k].fx_exit = entry; continue; }
    size_t p = entry;
    while (p < e && !u[k].seen[p - s]) p = bd.pivot_step(q, n, min_len, p, u[k].fc, nullptr);
    if (p < e) { u[k].fx_conv = p; u[k].fx_exit = u[k].exit; } else u[k].fx_exit = p;
  }
  std::vector<RawMem> out;                          // merge along the true chain
  size_t t = 0;
  auto take = [&](const Unit& x, size_t from) {
    for (size_t i = 0; i < x.c.size(); i++) if (x.piv[i] >= from) out.push_back(x.c[i]);
  };
  for (size_t k = 0; k < U; k++) {
    size_t s = k * seg, e = std::min(n, s + seg);
    if (t >= e) continue;
    if (k > 0 && u[k].fx_entry == t) {
      out.insert(out.end(), u[k].fc.begin(), u[k].fc.end());
      if (u[k].fx_conv != NONE) { take(u[k], u[k].fx_conv); t = u[k].exit; } else t = u[k].fx_exit;
      continue;
    }
    size_t p = t;
    while (p < e && !u[k].seen[p - s]) p = bd.pivot_step(q, n, min_len, p, out, nullptr);
    if (p < e) { take(u[k], p); t = u[k].exit; } else t = p;
  }
  return out;
}

static bool same_mems(std::vector<RawMem> a, std::vector<RawMem> b) {
  if (a.size() != b.size()) return false;
  auto by_lo = [](const BIv& x, const BIv& y) { return x.fwd_lo < y.fwd_lo; };
  for (size_t i = 0; i < a.size(); i++) {
    if (a[i].qs != b[i].qs || a[i].qe != b[i].qe || a[i].count != b[i].count || a[i].ivs.size() != b[i].ivs.size())
      return false;
    std::sort(a[i].ivs.begin(), a[i].ivs.end(), by_lo);
    std::sort(b[i].ivs.begin(), b[i].ivs.end(), by_lo);
    for (size_t j = 0; j < a[i].ivs.size(); j++)
      if (a[i].ivs[j].fwd_lo != b[i].ivs[j].fwd_lo || a[i].ivs[j].fwd_hi != b[i].ivs[j].fwd_hi ||
          a[i].ivs[j].rev_lo != b[i].ivs[j].rev_lo || a[i].ivs[j].rev_hi != b[i].ivs[j].rev_hi)
        return false;
  }
  return true;
}

// For each read longer than seg_len: find_smems through the segmented sweep equals the
// whole-read sweep.  *mismatch = reads that differ, *checked = reads compared.
int orc_smem_segment_check(void* hv, const uint8_t* q, const uint64_t* off, uint32_t nq, uint32_t min_len,
                           uint32_t seg_len, uint32_t* mismatch, uint32_t* checked) {
  Handle* h = (Handle*)hv;
  if (h->kind != 1) { g_err = "mems need a bidirectional index"; return -4; }
  if (seg_len == 0 || min_len == 0) { g_err = "seg_len and min_len must be > 0"; return -4; }
  const Bidir& bd = h->bd;
  uint32_t bad = 0, n_checked = 0;
  for (uint32_t r = 0; r < nq; r++) {
    const uint8_t* qq = q + off[r];
    size_t n = off[r + 1] - off[r];
    if (n <= seg_len) continue;
    n_checked++;
    auto whole = bd.find_smems(qq, n, min_len);
    auto segd = Bidir::filter_smems(segmented_candidates(bd, qq, n, min_len, seg_len));
    if (!same_mems(whole, segd)) bad++;
  }
  *mismatch = bad;
  *checked = n_checked;
  return 0;
}

// Single bidirectional extension (BidirFmIndex::extend_right / extend_left,
// src/fm_index/bidir_index.rs:133-144).  dir 0 = right, 1 = left.  Returns 1 if non-empty.
int orc_extend(void* hv, int dir, const uint32_t* iv_in, uint8_t c, uint32_t* iv_out) {
  Handle* h = (Handle*)hv;
  BIv iv{iv_in[0], iv_in[1], iv_in[2], iv_in[3]}, o{};
  bool ok = dir == 0 ? extend_right(iv, c, h->bd.rev, o) : extend_left(iv, c, h->bd.fwd, o);
  iv_out[0] = o.fwd_lo; iv_out[1] = o.fwd_hi; iv_out[2] = o.rev_lo; iv_out[3] = o.rev_hi;
  return ok ? 1 : 0;
}

// Naive suffix array of a raw code string (oracle for the product's suffix sorter).
int orc_suffix_array(const uint8_t* t, uint64_t n, uint32_t* out) {
  std::vector<uint8_t> v(t, t + n);
  std::vector<uint32_t> sa = naive_sa(v);
  std::memcpy(out, sa.data(), n * 4);
  return 0;
}

// The prefix-doubling sorter that orc_build uses (checked against orc_suffix_array).
int orc_suffix_array_doubling(const uint8_t* t, uint64_t n, uint32_t* out, int threads) {
  std::vector<uint8_t> v(t, t + n);
  std::vector<uint32_t> sa = doubling_sa(v, threads);
  if (n) std::memcpy(out, sa.data(), n * 4);
  return 0;
}

// Host threads of orc_build's suffix sort (default 1).
void orc_set_build_threads(int threads) { g_build_threads = std::max(1, threads); }

}  // extern "C"
