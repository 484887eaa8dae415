// hfm_internal.h — host-side declarations shared by the library's translation units.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/hfm.h"

namespace hfm {

// Thread-local last-error message; returns `status` for `return set_error(...)`.
int set_error(int status, const std::string& msg);

// One FmIndex parsed from bincode (views into the caller's bytes are copied into vectors
// only where the device layout needs a transform).
struct HostFm {
  uint32_t C[16];
  uint8_t num_lanes, num_planes, s2l[16], l2s[16];
  const uint8_t* block_data; uint64_t block_bytes, block_stride;
  uint32_t encoding, occ_text_len;
  const uint8_t* ssa_words; uint64_t ssa_bytes;
  const uint32_t* sa_vals; uint64_t n_sa_vals;     // may be unaligned in the byte stream: copied
  uint32_t sample_rate, ssa_text_len;
  uint32_t text_len, num_sequences;
  std::vector<uint32_t> seq_boundaries;
  std::vector<std::string> headers;
  bool has_lookup; uint32_t lookup_depth;
  std::vector<uint8_t> lookup_core;
  const uint8_t* lookup_intervals; uint64_t n_lookup;
  uint8_t tag;
  std::vector<uint32_t> sa_vals_copy;
};

// Parses and validates FmIndex bincode bytes (src/fm_index/serialize.rs:32-52).  Beyond
// what bincode itself checks, the layout is cross-checked so that no device access can
// leave its buffer.  Returns HFM_OK or HFM_E_FORMAT (message set).
int parse_fm(const uint8_t* p, uint64_t n, HostFm& f);

void suffix_array(const uint8_t* text, uint32_t n, uint32_t* sa);

// One FmIndex in the reference's record layout, ready for the bincode writer.
struct BuiltFm {
  uint32_t C[16];
  uint8_t num_lanes, num_planes, s2l[16], l2s[16];
  std::vector<uint32_t> sb;
  std::vector<uint8_t> block_data;
  uint64_t block_stride;
  uint32_t encoding, text_len;
  std::vector<uint8_t> ssa_words;
  std::vector<uint32_t> sa_vals;
  uint32_t rate;
  uint32_t num_sequences;
  std::vector<uint32_t> bounds;
  std::vector<std::string> headers;
  uint32_t lookup_depth;
  std::vector<std::pair<uint32_t, uint32_t>> lut;
  uint8_t tag;
};

// bincode-1 bytes of one FmIndex (src/fm_index/serialize.rs:55-67).
void write_fm(const BuiltFm& f, std::vector<uint8_t>& out);
int concat_text(const uint8_t* codes, const uint64_t* seq_off, uint32_t nseq, const char* const* headers,
                std::vector<uint8_t>& text, std::vector<uint32_t>& bounds, std::vector<std::string>& hs);
int emit_bytes(const BuiltFm& fwd, const BuiltFm& rev, int kind, uint8_t** bytes_out, size_t* len_out);

}  // namespace hfm

extern "C" int hfm_suffix_array(const uint8_t* text, uint32_t n, uint32_t* sa_out);
