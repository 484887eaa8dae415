// bincode.cpp — reader for the reference's serialized FmIndex (bincode 1: fixint,
// little endian, u64 length prefixes, Option = u8 tag, unit enum = u32 index).
// Field order: src/fm_index/serialize.rs:55-67, src/occ/mod.rs:45-78,
// src/suffix_array/mod.rs:54-63, src/fm_index/lookup.rs:19-27.

#include <cstring>
#include <string>

#include "hfm_internal.h"

namespace hfm {

namespace {
struct Cursor {
  const uint8_t* p; uint64_t n, i = 0; bool bad = false; const char* what = "";
  bool need(uint64_t k, const char* w) { if (bad) return false; if (n - i < k) { bad = true; what = w; return false; } return true; }
  uint8_t u8(const char* w) { if (!need(1, w)) return 0; return p[i++]; }
  uint32_t u32(const char* w) { if (!need(4, w)) return 0; uint32_t v; std::memcpy(&v, p + i, 4); i += 4; return v; }
  uint64_t u64(const char* w) { if (!need(8, w)) return 0; uint64_t v; std::memcpy(&v, p + i, 8); i += 8; return v; }
  // Vec<T>: returns a pointer into the stream and the element count.
  const uint8_t* vec(uint64_t elem, uint64_t& count, const char* w) {
    count = u64(w);
    if (bad) return nullptr;
    if (count > (n - i) / elem) { bad = true; what = w; return nullptr; }
    const uint8_t* r = p + i; i += count * elem; return r;
  }
};

bool valid_utf8(const uint8_t* s, uint64_t n) {
  uint64_t i = 0;
  while (i < n) {
    uint8_t c = s[i];
    int k;
    if (c < 0x80) k = 0;
    else if ((c & 0xE0) == 0xC0) k = 1;
    else if ((c & 0xF0) == 0xE0) k = 2;
    else if ((c & 0xF8) == 0xF0) k = 3;
    else return false;
    if (i + k >= n) return false;
    for (int j = 1; j <= k; j++) if ((s[i + j] & 0xC0) != 0x80) return false;
    i += k + 1;
  }
  return true;
}

uint8_t planes_for(uint32_t L) { uint8_t P = 0; if (L > 1) { uint32_t v = L - 1; while (v) { P++; v >>= 1; } } return P; }
}  // namespace

int parse_fm(const uint8_t* p, uint64_t n, HostFm& f) {
  Cursor c{p, n};
  for (int k = 0; k < 16; k++) f.C[k] = c.u32("c_array");
  f.num_lanes = c.u8("occ.num_lanes"); f.num_planes = c.u8("occ.num_planes");
  if (c.need(32, "occ.lane maps")) { std::memcpy(f.s2l, p + c.i, 16); std::memcpy(f.l2s, p + c.i + 16, 16); c.i += 32; }
  uint64_t n_sb; c.vec(4, n_sb, "occ.superblock_checkpoints");
  f.block_data = c.vec(1, f.block_bytes, "occ.block_data");
  f.block_stride = c.u64("occ.block_stride");
  f.encoding = c.u32("occ.encoding");
  f.occ_text_len = c.u32("occ.text_len");
  f.ssa_words = c.vec(1, f.ssa_bytes, "sa_samples.word_data");
  const uint8_t* sv = c.vec(4, f.n_sa_vals, "sa_samples.sa_vals");
  f.sample_rate = c.u32("sa_samples.sample_rate");
  f.ssa_text_len = c.u32("sa_samples.text_len");
  f.text_len = c.u32("text_len");
  f.num_sequences = c.u32("num_sequences");
  uint64_t nb; const uint8_t* bp = c.vec(4, nb, "seq_boundaries");
  uint64_t nh = c.u64("seq_headers");
  if (c.bad) return set_error(HFM_E_FORMAT, std::string("truncated bincode at ") + c.what);
  f.seq_boundaries.resize(nb);
  if (nb) std::memcpy(f.seq_boundaries.data(), bp, nb * 4);
  f.headers.clear();
  for (uint64_t k = 0; k < nh; k++) {
    uint64_t len; const uint8_t* s = c.vec(1, len, "seq_headers[]");
    if (c.bad) return set_error(HFM_E_FORMAT, "truncated bincode at seq_headers");
    if (!valid_utf8(s, len)) return set_error(HFM_E_FORMAT, "invalid UTF-8 in sequence header");
    f.headers.emplace_back((const char*)s, (size_t)len);
  }
  uint8_t opt = c.u8("lookup");
  f.has_lookup = false; f.lookup_depth = 0; f.n_lookup = 0; f.lookup_intervals = nullptr;
  if (opt == 1) {
    f.has_lookup = true;
    f.lookup_depth = c.u32("lookup.depth");
    uint64_t nc; const uint8_t* cp = c.vec(1, nc, "lookup.core_symbols");
    if (!c.bad) f.lookup_core.assign(cp, cp + nc);
    f.lookup_intervals = c.vec(8, f.n_lookup, "lookup.intervals");
  } else if (opt != 0 && !c.bad) {
    return set_error(HFM_E_FORMAT, "invalid Option tag for lookup");
  }
  f.tag = c.u8("alphabet_tag");
  if (c.bad) return set_error(HFM_E_FORMAT, std::string("truncated bincode at ") + c.what);
  if (f.encoding > 1) return set_error(HFM_E_FORMAT, "invalid OccEncoding variant");
  if (f.tag > 1) return set_error(HFM_E_FORMAT, "unknown alphabet tag " + std::to_string(f.tag) + " in serialized FM-index");

  // ---- consistency checks: every device access must stay inside its buffer ----
  const uint32_t n_text = f.text_len;
  uint32_t L = f.num_lanes;
  if (L == 0 || L > 16) return set_error(HFM_E_FORMAT, "occ.num_lanes out of range");
  if (f.occ_text_len != n_text || f.ssa_text_len != n_text) return set_error(HFM_E_FORMAT, "text_len mismatch between parts");
  if (f.encoding == 0 && f.num_planes != planes_for(L)) return set_error(HFM_E_FORMAT, "occ.num_planes does not match num_lanes");
  uint64_t width = f.encoding == 0 ? f.num_planes : L;
  if (f.block_stride != (uint64_t)L * 6 + width * 8) return set_error(HFM_E_FORMAT, "occ.block_stride inconsistent");
  uint64_t need_blocks = ((uint64_t)n_text + 63) / 64;
  if (f.block_stride == 0 || f.block_bytes != need_blocks * f.block_stride) return set_error(HFM_E_FORMAT, "occ.block_data size inconsistent");
  for (int s = 0; s < 16; s++) if (f.s2l[s] != 0xFF && f.s2l[s] >= L) return set_error(HFM_E_FORMAT, "occ.symbol_to_lane out of range");
  for (uint32_t l = 0; l < L; l++) if (f.l2s[l] > 15) return set_error(HFM_E_FORMAT, "occ.lane_to_symbol out of range");
  if (f.ssa_bytes != need_blocks * 14) return set_error(HFM_E_FORMAT, "sa_samples.word_data size inconsistent");
  // sampled-SA marker ranks must agree with the bit counts and stay inside sa_vals
  uint64_t cum = 0;
  for (uint64_t w = 0; w < need_blocks; w++) {
    uint64_t word; uint32_t sb; uint16_t d;
    std::memcpy(&word, f.ssa_words + w * 14, 8); std::memcpy(&sb, f.ssa_words + w * 14 + 8, 4);
    std::memcpy(&d, f.ssa_words + w * 14 + 12, 2);
    if ((uint64_t)sb + d != cum) return set_error(HFM_E_FORMAT, "sa_samples marker ranks inconsistent");
    if (w == need_blocks - 1 && (n_text & 63)) word &= (1ull << (n_text & 63)) - 1;
    cum += (uint64_t)__builtin_popcountll(word);
  }
  if (cum > f.n_sa_vals) return set_error(HFM_E_FORMAT, "sa_samples has fewer values than marked rows");
  f.sa_vals_copy.resize(f.n_sa_vals);
  if (f.n_sa_vals) std::memcpy(f.sa_vals_copy.data(), sv, f.n_sa_vals * 4);
  f.sa_vals = f.sa_vals_copy.data();
  for (uint64_t k = 0; k < f.n_sa_vals; k++) if (f.sa_vals[k] >= n_text && n_text) return set_error(HFM_E_FORMAT, "sa value out of range");
  // C array must equal the prefix sums of the Occ totals: keeps every LF step in range
  {
    uint64_t b = need_blocks - 1;
    const uint8_t* r = f.block_data + b * f.block_stride;
    uint32_t off = (n_text - 1) & 63;
    uint64_t lt[16] = {0};
    for (uint32_t l = 0; l < L; l++) {
      uint32_t sb; uint16_t d;
      std::memcpy(&sb, r + l * 4, 4); std::memcpy(&d, r + L * 4 + l * 2, 2);
      uint64_t m = ~0ull;
      if (f.encoding == 1) std::memcpy(&m, r + L * 6 + l * 8, 8);
      else for (uint32_t q = 0; q < f.num_planes; q++) { uint64_t pv; std::memcpy(&pv, r + L * 6 + q * 8, 8); m &= ((l >> q) & 1) ? pv : ~pv; }
      uint64_t mask = off == 63 ? ~0ull : ((1ull << (off + 1)) - 1);
      lt[l] = (uint64_t)sb + d + (uint64_t)__builtin_popcountll(m & mask);
    }
    uint64_t sum = 0;
    for (int s = 0; s < 16; s++) {
      if (f.C[s] != sum) return set_error(HFM_E_FORMAT, "c_array inconsistent with the Occ table");
      if (f.s2l[s] != 0xFF) sum += lt[f.s2l[s]];
    }
    if (sum != n_text) return set_error(HFM_E_FORMAT, "Occ totals do not add up to text_len");
  }
  if (f.has_lookup) {
    uint64_t radix = f.lookup_core.size(), size = 1;
    if (radix == 0 || f.lookup_depth == 0 || f.lookup_depth > 16) return set_error(HFM_E_FORMAT, "lookup depth/core out of range");
    for (uint32_t k = 0; k < f.lookup_depth; k++) { size *= radix; if (size > (1ull << 34)) return set_error(HFM_E_FORMAT, "lookup table too large"); }
    if (f.n_lookup != size) return set_error(HFM_E_FORMAT, "lookup.intervals size != radix^depth");
    for (uint64_t k = 0; k < f.n_lookup; k++) {
      uint32_t lo, hi; std::memcpy(&lo, f.lookup_intervals + k * 8, 4); std::memcpy(&hi, f.lookup_intervals + k * 8 + 4, 4);
      if (lo > n_text || hi > n_text) return set_error(HFM_E_FORMAT, "lookup interval out of range");
    }
  }
  return HFM_OK;
}

}  // namespace hfm
