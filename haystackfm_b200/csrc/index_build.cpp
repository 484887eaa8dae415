// index_build.cpp — FM-index construction emitting the reference's bincode layout.
//
// Replaces FmIndex::build_cpu_with + to_bytes (src/fm_index/mod.rs:95-195,
// src/fm_index/serialize.rs:13-26) and BidirFmIndex::build_cpu_with + to_bytes
// (src/fm_index/bidir_index.rs:53-80,183-192).  The suffix array comes from an own
// SA-IS implementation (induced sorting, Nong-Zhang-Chan 2009) instead of the psacak
// crate; it sorts in true lexicographic order of the encoded text.  Everything after the
// suffix array (BWT, C array, compacted Occ records, sampled SA markers, depth-k lookup
// table) reproduces the reference's byte layout, so the bytes load into the reference
// and into hfm_index_load alike.

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "hfm_internal.h"

namespace hfm {

static const uint32_t EMPTY = 0xFFFFFFFFu;

#define RET_STATUS(x) do { int _r = (x); if (_r != HFM_OK) return _r; } while (0)

// ---------------------------------------------------------------------------
// SA-IS.  T[n-1] must be the unique smallest symbol; symbols are < K.
// ---------------------------------------------------------------------------
template <class Ch>
static void sais(const Ch* T, uint32_t* SA, uint32_t n, uint32_t K) {
  if (n == 1) { SA[0] = 0; return; }
  std::vector<uint8_t> t(n);   // 1 = S-type, 0 = L-type
  t[n - 1] = 1;
  for (int64_t i = (int64_t)n - 2; i >= 0; i--)
    t[i] = (T[i] < T[i + 1] || (T[i] == T[i + 1] && t[i + 1])) ? 1 : 0;
  auto lms = [&](uint32_t i) { return i > 0 && t[i] && !t[i - 1]; };
  std::vector<uint32_t> cnt(K, 0), bkt(K);
  for (uint32_t i = 0; i < n; i++) cnt[T[i]]++;
  auto heads = [&]() { uint32_t s = 0; for (uint32_t c = 0; c < K; c++) { bkt[c] = s; s += cnt[c]; } };
  auto tails = [&]() { uint32_t s = 0; for (uint32_t c = 0; c < K; c++) { s += cnt[c]; bkt[c] = s; } };
  auto induce = [&]() {
    heads();
    for (uint32_t i = 0; i < n; i++) {
      uint32_t j = SA[i];
      if (j != EMPTY && j > 0 && !t[j - 1]) SA[bkt[T[j - 1]]++] = j - 1;
    }
    tails();
    for (uint32_t i = n; i-- > 0;) {
      uint32_t j = SA[i];
      if (j != EMPTY && j > 0 && t[j - 1]) SA[--bkt[T[j - 1]]] = j - 1;
    }
  };
  // 1. sort LMS substrings by induction
  std::fill(SA, SA + n, EMPTY);
  tails();
  for (uint32_t i = 1; i < n; i++) if (lms(i)) SA[--bkt[T[i]]] = i;
  induce();
  // 2. compact the sorted LMS positions and name the LMS substrings
  uint32_t n1 = 0;
  for (uint32_t i = 0; i < n; i++) if (SA[i] != EMPTY && lms(SA[i])) SA[n1++] = SA[i];
  std::fill(SA + n1, SA + n, EMPTY);
  uint32_t name = 0, prev = EMPTY;
  for (uint32_t i = 0; i < n1; i++) {
    uint32_t pos = SA[i];
    bool diff = false;
    for (uint32_t d = 0;; d++) {
      if (prev == EMPTY || T[pos + d] != T[prev + d] || t[pos + d] != t[prev + d]) { diff = true; break; }
      if (d > 0 && (lms(pos + d) || lms(prev + d))) break;
    }
    if (diff) { name++; prev = pos; }
    SA[n1 + pos / 2] = name - 1;
  }
  for (uint32_t i = n, j = n; i-- > n1;) if (SA[i] != EMPTY) SA[--j] = SA[i];
  uint32_t* s1 = SA + n - n1;
  uint32_t* sa1 = SA;
  // 3. sort the reduced string (recursively if names repeat)
  if (name < n1) sais<uint32_t>(s1, sa1, n1, name);
  else for (uint32_t i = 0; i < n1; i++) sa1[s1[i]] = i;
  // 4. induce the full order from the sorted LMS suffixes
  for (uint32_t i = 1, j = 0; i < n; i++) if (lms(i)) s1[j++] = i;
  for (uint32_t i = 0; i < n1; i++) sa1[i] = s1[sa1[i]];
  std::fill(SA + n1, SA + n, EMPTY);
  tails();
  for (uint32_t i = n1; i-- > 0;) { uint32_t j = SA[i]; SA[i] = EMPTY; SA[--bkt[T[j]]] = j; }
  induce();
}

// Suffix array of an encoded text (codes 0..15) in Rust-slice lexicographic order.  Every
// code is shifted up by one and the final sentinel becomes the unique 0, which keeps the
// order: the final "$" suffix is a prefix of every other "$..." suffix and sorts first.
void suffix_array(const uint8_t* text, uint32_t n, uint32_t* sa) {
  if (n == 0) return;
  std::vector<uint8_t> t(n);
  for (uint32_t i = 0; i + 1 < n; i++) t[i] = (uint8_t)(text[i] + 1);
  t[n - 1] = 0;
  sais<uint8_t>(t.data(), sa, n, 17);
}

// ---------------------------------------------------------------------------
// bincode-1 writer (fixint, little endian; src/fm_index/serialize.rs:55-67)
// ---------------------------------------------------------------------------
struct BinWriter {
  std::vector<uint8_t>& b;
  void put(const void* p, size_t k) { const uint8_t* s = (const uint8_t*)p; b.insert(b.end(), s, s + k); }
  void u8(uint8_t v) { b.push_back(v); }
  void u32(uint32_t v) { put(&v, 4); }
  void u64(uint64_t v) { put(&v, 8); }
};

void write_fm(const BuiltFm& f, std::vector<uint8_t>& out) {
  BinWriter w{out};
  for (int c = 0; c < 16; c++) w.u32(f.C[c]);
  // OccTable field order (src/occ/mod.rs:45-78)
  w.u8(f.num_lanes); w.u8(f.num_planes); w.put(f.s2l, 16); w.put(f.l2s, 16);
  w.u64(f.sb.size()); w.put(f.sb.data(), f.sb.size() * 4);
  w.u64(f.block_data.size()); w.put(f.block_data.data(), f.block_data.size());
  w.u64(f.block_stride); w.u32(f.encoding); w.u32(f.text_len);
  // SampledSuffixArray (src/suffix_array/mod.rs:54-63)
  w.u64(f.ssa_words.size()); w.put(f.ssa_words.data(), f.ssa_words.size());
  w.u64(f.sa_vals.size()); w.put(f.sa_vals.data(), f.sa_vals.size() * 4);
  w.u32(f.rate); w.u32(f.text_len);
  w.u32(f.text_len); w.u32(f.num_sequences);
  w.u64(f.bounds.size()); w.put(f.bounds.data(), f.bounds.size() * 4);
  w.u64(f.headers.size());
  for (auto& h : f.headers) { w.u64(h.size()); w.put(h.data(), h.size()); }
  if (f.lookup_depth > 0) {   // Option<LookupTable> (src/fm_index/lookup.rs:19-27)
    w.u8(1); w.u32(f.lookup_depth);
    static const uint8_t core[4] = {1, 2, 3, 4};
    w.u64(4); w.put(core, 4);
    w.u64(f.lut.size());
    for (auto& iv : f.lut) { w.u32(iv.first); w.u32(iv.second); }
  } else w.u8(0);
  w.u8(f.tag);
}

// Rank over the Occ records just built (same arithmetic as OccTable::rank, src/occ/mod.rs:330-363).
static uint32_t built_rank(const BuiltFm& f, uint8_t c, uint32_t i) {
  if (i == 0) return 0;
  uint8_t lane = f.s2l[c];
  if (lane == 0xFF) return 0;
  uint32_t pos = i - 1, off = pos & 63;
  const uint8_t* r = f.block_data.data() + (uint64_t)(pos >> 6) * f.block_stride;
  uint32_t L = f.num_lanes, sbv, bits_lo;
  uint16_t dv;
  std::memcpy(&sbv, r + lane * 4, 4);
  std::memcpy(&dv, r + L * 4 + lane * 2, 2);
  uint64_t m = ~0ull;
  if (f.encoding == 1) std::memcpy(&m, r + L * 6 + lane * 8, 8);
  else for (int p = 0; p < f.num_planes; p++) {
    uint64_t pv; std::memcpy(&pv, r + L * 6 + p * 8, 8);
    m &= ((lane >> p) & 1) ? pv : ~pv;
  }
  (void)bits_lo;
  uint64_t mask = (off == 63) ? ~0ull : ((1ull << (off + 1)) - 1);
  return sbv + dv + (uint32_t)__builtin_popcountll(m & mask);
}

static void build_fm(const uint8_t* text, uint32_t n, const std::vector<uint32_t>& bounds,
                     const std::vector<std::string>& headers, const hfm_build_opts& o,
                     uint32_t lookup_depth, BuiltFm& f) {
  f.tag = (uint8_t)o.alphabet_tag; f.encoding = o.occ_encoding; f.text_len = n; f.rate = o.sa_sample_rate;
  f.num_sequences = (uint32_t)bounds.size(); f.bounds = bounds; f.headers = headers;
  f.lookup_depth = lookup_depth;
  // C array from text (src/c_array.rs:14-31)
  uint64_t freq[16] = {0};
  for (uint32_t i = 0; i < n; i++) freq[text[i] & 15]++;
  uint32_t s = 0;
  for (int c = 0; c < 16; c++) { f.C[c] = s; s += (uint32_t)freq[c]; }
  // suffix array and BWT (src/bwt/cpu.rs:14-35)
  std::vector<uint32_t> sa(n);
  suffix_array(text, n, sa.data());
  std::vector<uint8_t> bwt(n);
  for (uint32_t i = 0; i < n; i++) bwt[i] = text[sa[i] == 0 ? n - 1 : sa[i] - 1];
  // sampled SA with every sequence start forced (src/fm_index/mod.rs:154-162,
  // src/suffix_array/mod.rs:71-118)
  std::vector<uint64_t> forced((n + 63) / 64 + 1, 0);
  forced[0] |= 1;
  for (size_t k = 0; k + 1 < bounds.size(); k++) forced[bounds[k] >> 6] |= 1ull << (bounds[k] & 63);
  uint64_t nw = (n + 63) / 64;
  f.ssa_words.assign(nw * 14, 0);
  f.sa_vals.clear(); f.sa_vals.reserve(n / std::max(1u, o.sa_sample_rate) + bounds.size() + 1);
  uint32_t cum = 0, sbb = 0;
  for (uint64_t w = 0; w < nw; w++) {
    uint64_t word = 0;
    for (uint32_t b = 0; b < 64; b++) {
      uint64_t i = w * 64 + b;
      if (i >= n) break;
      uint32_t v = sa[i];
      bool mult = o.sa_sample_rate == 0 ? v == 0 : v % o.sa_sample_rate == 0;
      if (mult || ((forced[v >> 6] >> (v & 63)) & 1)) { word |= 1ull << b; f.sa_vals.push_back(v); }
    }
    if (w % 8 == 0) sbb = cum;
    uint16_t delta = (uint16_t)(cum - sbb);
    uint8_t* r = f.ssa_words.data() + w * 14;
    std::memcpy(r, &word, 8); std::memcpy(r + 8, &sbb, 4); std::memcpy(r + 12, &delta, 2);
    cum += (uint32_t)__builtin_popcountll(word);
  }
  std::vector<uint32_t>().swap(sa);
  // Occ table: compacted lanes, interleaved records (src/occ/cpu.rs:23-119, src/occ/mod.rs:114-183)
  uint64_t totals[16] = {0};
  for (uint32_t i = 0; i < n; i++) totals[bwt[i] & 15]++;
  std::memset(f.s2l, 0xFF, 16); std::memset(f.l2s, 0, 16);
  uint8_t L = 0;
  for (int c = 0; c < 16; c++) if (totals[c]) { f.s2l[c] = L; f.l2s[L] = (uint8_t)c; L++; }
  uint8_t P = 0;
  if (L > 1) { uint32_t v = L - 1; while (v) { P++; v >>= 1; } }
  f.num_lanes = L; f.num_planes = P;
  uint32_t width = f.encoding == 0 ? P : L;
  f.block_stride = (uint64_t)L * 6 + (uint64_t)width * 8;
  uint64_t nb = (n + 63) / 64;
  f.block_data.assign(nb * f.block_stride, 0);
  f.sb.clear(); f.sb.reserve(((n + 511) / 512) * L);
  std::vector<uint32_t> cumu(L, 0), sbase(L, 0);
  for (uint64_t b = 0; b < nb; b++) {
    if (b % 8 == 0) { for (int l = 0; l < L; l++) f.sb.push_back(cumu[l]); sbase = cumu; }
    uint64_t bits[16] = {0}; uint32_t cnt[16] = {0};
    uint32_t end = (uint32_t)std::min<uint64_t>((b + 1) * 64, n);
    for (uint32_t i = (uint32_t)(b * 64); i < end; i++) { bits[bwt[i]] |= 1ull << (i & 63); cnt[bwt[i]]++; }
    uint8_t* r = f.block_data.data() + b * f.block_stride;
    uint64_t words[16] = {0};
    for (int c = 0; c < 16; c++) {
      uint8_t lane = f.s2l[c];
      if (lane == 0xFF) continue;
      uint32_t sbv = f.sb[(b / 8) * L + lane];
      uint16_t dv = (uint16_t)(cumu[lane] - sbase[lane]);
      std::memcpy(r + lane * 4, &sbv, 4);
      std::memcpy(r + L * 4 + lane * 2, &dv, 2);
      if (f.encoding == 0) { for (uint32_t p = 0; p < width; p++) if ((lane >> p) & 1) words[p] |= bits[c]; }
      else words[lane] = bits[c];
      cumu[lane] += cnt[c];
    }
    for (uint32_t k = 0; k < width; k++) std::memcpy(r + L * 6 + k * 8, &words[k], 8);
  }
  // depth-k lookup table, BFS over ACGT (src/fm_index/lookup.rs:37-91)
  if (lookup_depth > 0) {
    uint64_t size = 1;
    for (uint32_t i = 0; i < lookup_depth; i++) size *= 4;
    f.lut.assign(size, {0, 0});
    struct E { uint64_t idx; uint32_t lo, hi; };
    std::vector<E> cur{{0, 0, n}}, nxt;
    for (uint32_t level = 1; level <= lookup_depth; level++) {
      nxt.clear();
      bool last = level == lookup_depth;
      for (const E& e : cur) for (uint32_t d = 0; d < 4; d++) {
        uint8_t sym = (uint8_t)(d + 1);
        uint32_t upper = sym + 1 < 16 ? f.C[sym + 1] : n;
        if (upper - f.C[sym] == 0) continue;
        uint32_t nlo = f.C[sym] + built_rank(f, sym, e.lo), nhi = f.C[sym] + built_rank(f, sym, e.hi);
        if (last) f.lut[e.idx * 4 + d] = {nlo, nhi};
        else if (nlo < nhi) nxt.push_back({e.idx * 4 + d, nlo, nhi});
      }
      if (!last) cur.swap(nxt);
    }
  }
}


// concatenate_sequences (src/alphabet.rs:375-393): codes 1..15 per sequence, a 0 sentinel
// after each; bounds = exclusive ends; headers default to "seq_{i}".
int concat_text(const uint8_t* codes, const uint64_t* seq_off, uint32_t nseq, const char* const* headers,
                std::vector<uint8_t>& text, std::vector<uint32_t>& bounds, std::vector<std::string>& hs) {
  uint64_t total = 0;
  for (uint32_t s = 0; s < nseq; s++) total += seq_off[s + 1] - seq_off[s] + 1;
  if (total > 0xFFFFFFFFull) return set_error(HFM_E_ARG, "text too large: exceeds u32::MAX");
  const uint32_t n = (uint32_t)total;
  try {
    text.assign(n, 0); bounds.assign(nseq, 0); hs.assign(nseq, std::string());
  } catch (const std::bad_alloc&) {
    return set_error(HFM_E_OOM, "host allocation failed");
  }
  uint64_t pos = 0;
  for (uint32_t s = 0; s < nseq; s++) {
    uint64_t len = seq_off[s + 1] - seq_off[s];
    for (uint64_t k = 0; k < len; k++) {
      uint8_t c = codes[seq_off[s] + k];
      if (c == 0 || c > 15) return set_error(HFM_E_ARG, "invalid code in sequence");
      text[pos + k] = c;
    }
    pos += len; text[pos++] = 0; bounds[s] = (uint32_t)pos;
    std::string h = headers && headers[s] ? headers[s] : "";
    hs[s] = h.empty() ? "seq_" + std::to_string(s) : h;
  }
  return HFM_OK;
}

// FmIndex bytes (kind 0) or BidirFmIndex bytes, [u32 fwd_len][fwd][rev] (kind 1,
// src/fm_index/bidir_index.rs:183-192), in one malloc block.
int emit_bytes(const BuiltFm& fwd, const BuiltFm& rev, int kind, uint8_t** bytes_out, size_t* len_out) {
  std::vector<uint8_t> out;
  try {
    if (kind == HFM_KIND_FM) write_fm(fwd, out);
    else {
      std::vector<uint8_t> fb, rb;
      write_fm(fwd, fb); write_fm(rev, rb);
      uint32_t fl = (uint32_t)fb.size();
      out.resize(4); std::memcpy(out.data(), &fl, 4);
      out.insert(out.end(), fb.begin(), fb.end());
      out.insert(out.end(), rb.begin(), rb.end());
    }
  } catch (const std::bad_alloc&) {
    return set_error(HFM_E_OOM, "host allocation failed");
  }
  uint8_t* p = (uint8_t*)std::malloc(out.size());
  if (!p) return set_error(HFM_E_OOM, "host allocation failed");
  std::memcpy(p, out.data(), out.size());
  *bytes_out = p; *len_out = out.size();
  return HFM_OK;
}

}  // namespace hfm

using namespace hfm;

extern "C" int hfm_build_index(const uint8_t* codes, const uint64_t* seq_off, uint32_t nseq,
                               const char* const* headers, const hfm_build_opts* opts, int kind,
                               uint8_t** bytes_out, size_t* len_out) {
  if (!codes && nseq) return set_error(HFM_E_ARG, "codes is NULL");
  if (nseq == 0) return set_error(HFM_E_ARG, "empty sequence list");
  if (!opts || !bytes_out || !len_out) return set_error(HFM_E_ARG, "NULL argument");
  if (kind != HFM_KIND_FM && kind != HFM_KIND_BIDIR) return set_error(HFM_E_ARG, "kind must be 0 or 1");
  if (opts->alphabet_tag > 1 || opts->occ_encoding > 1) return set_error(HFM_E_ARG, "bad alphabet tag or encoding");
  std::vector<uint8_t> text;
  std::vector<uint32_t> bounds;
  std::vector<std::string> hs;
  RET_STATUS(concat_text(codes, seq_off, nseq, headers, text, bounds, hs));
  const uint32_t n = (uint32_t)text.size();
  BuiltFm fwd, rev;
  std::vector<uint8_t> rtext;
  bool par = (opts->threads == 0 || opts->threads > 1) && kind == HFM_KIND_BIDIR;
  if (kind == HFM_KIND_BIDIR) {
    // reverse_as_sequence (src/fm_index/bidir_index.rs:523-532): drop the final sentinel,
    // reverse, then concatenate as one sequence (which appends a new sentinel).
    rtext.assign(text.rbegin() + 1, text.rend());
    rtext.push_back(0);
  }
  try {
    if (par) {
      std::thread t([&] { build_fm(rtext.data(), n, {n}, {"seq_0"}, *opts, 0, rev); });
      build_fm(text.data(), n, bounds, hs, *opts, opts->lookup_depth, fwd);
      t.join();
    } else {
      build_fm(text.data(), n, bounds, hs, *opts, opts->lookup_depth, fwd);
      if (kind == HFM_KIND_BIDIR) build_fm(rtext.data(), n, {n}, {"seq_0"}, *opts, 0, rev);
    }
  } catch (const std::bad_alloc&) {
    return set_error(HFM_E_OOM, "host allocation failed during index construction");
  }
  return emit_bytes(fwd, rev, kind, bytes_out, len_out);
}

extern "C" int hfm_suffix_array(const uint8_t* text, uint32_t n, uint32_t* sa_out) {
  if (!text || !sa_out) return set_error(HFM_E_ARG, "NULL argument");
  suffix_array(text, n, sa_out);
  return HFM_OK;
}
