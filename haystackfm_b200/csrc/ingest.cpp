// ingest.cpp — FASTA / FASTQ / plain-line text of reads to the packed batch layout
// (u8 codes, u64 offsets) that every query entry point takes, on the host's cores.
//
// The reference reads queries as Rust strings and encodes each with
// DnaSequence::from_str (src/alphabet.rs:54-94, src/alphabet.rs:226-245); its text parser
// for sequences is the FASTA reader of src/wasm/js_api.rs:18-68 (`>` headers, blank lines
// skipped, the lines of a record concatenated, input without any header read as one
// sequence per non-blank line).  FASTQ (four-line records) has no counterpart there; it
// follows the usual record layout.  The host threads find the lines (each over a stretch
// of the text), one pass over the lines finds the reads, and the threads then encode
// blocks of reads.

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "hfm_internal.h"

namespace hfm {
namespace {

// ASCII -> code (src/alphabet.rs:54-94): "$ACGTNRYSWKMBDHV" in either case, U/u as T;
// 0xFF = not an alphabet character.  The sentinel `$` is not allowed inside a read.
struct EncodeTable {
  uint8_t t[256];
  EncodeTable() {
    std::memset(t, 0xFF, sizeof(t));
    const char* sym = "$ACGTNRYSWKMBDHV";
    for (int c = 1; c < 16; c++) {
      t[(uint8_t)sym[c]] = (uint8_t)c;
      t[(uint8_t)(sym[c] | 0x20)] = (uint8_t)c;
    }
    t[(uint8_t)'U'] = 4; t[(uint8_t)'u'] = 4;
  }
};
const EncodeTable kEnc;

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

struct Line { uint64_t a, b; };          // [a, b): a line as written, its end of line dropped
struct Seg { uint64_t at; uint32_t len; };

inline Line trim(const char* s, Line l) {
  while (l.a < l.b && is_space(s[l.a])) l.a++;
  while (l.b > l.a && is_space(s[l.b - 1])) l.b--;
  return l;
}

// Lines of s[i, n), which starts a line; lines end at \n, \r\n or a lone \r.
void split_lines(const char* s, uint64_t i, uint64_t n, std::vector<Line>& raw) {
  while (i < n) {
    // the next \n by memchr, then a \r before it (a \r\n pair or a lone \r line end)
    const char* nl = (const char*)std::memchr(s + i, '\n', n - i);
    uint64_t j = nl ? (uint64_t)(nl - s) : n;
    const char* cr = (const char*)std::memchr(s + i, '\r', j - i);
    uint64_t next = j + 1;
    if (cr) {
      const uint64_t k = (uint64_t)(cr - s);
      next = (k + 1 == j) ? j + 1 : k + 1;       // \r\n: past both; a lone \r ends the line
      j = k;
    }
    raw.push_back({i, j});
    i = next;
  }
}

// The same lines, found by `nt` threads over stretches that start after a \n (every \n
// ends a line, so each stretch starts one), concatenated in order.
void split_lines_parallel(const char* s, uint64_t n, unsigned nt, std::vector<Line>& raw) {
  if (nt <= 1) { split_lines(s, 0, n, raw); return; }
  std::vector<uint64_t> cut(nt + 1, n);
  cut[0] = 0;
  for (unsigned t = 1; t < nt; t++) {
    const uint64_t p = std::max(cut[t - 1], n * t / nt);
    const char* nl = p < n ? (const char*)std::memchr(s + p, '\n', n - p) : nullptr;
    cut[t] = nl ? (uint64_t)(nl - s) + 1 : n;
  }
  std::vector<std::vector<Line>> part(nt);
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; t++)
    th.emplace_back([&, t]() { part[t].reserve((cut[t + 1] - cut[t]) / 64 + 16); split_lines(s, cut[t], cut[t + 1], part[t]); });
  for (auto& x : th) x.join();
  size_t total = 0;
  for (auto& v : part) total += v.size();
  raw.resize(total);
  size_t at = 0;
  for (auto& v : part) { std::copy(v.begin(), v.end(), raw.begin() + at); at += v.size(); }
}

}  // namespace
}  // namespace hfm

using namespace hfm;

extern "C" int hfm_parse_reads(const char* text, uint64_t len, uint32_t format, uint32_t threads, hfm_reads** out) {
  if (!out || (len && !text)) return set_error(HFM_E_ARG, "NULL argument");
  if (format > HFM_READS_FASTQ) return set_error(HFM_E_ARG, "format must be 0 (auto), 1 (FASTA) or 2 (FASTQ)");
  *out = nullptr;
  unsigned nt = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
  if (len < (8u << 20)) nt = 1;
  std::vector<Line> rl;
  split_lines_parallel(text, len, nt, rl);
  for (const Line& r : rl)
    if (r.b - r.a > 0xFFFFFFFFull) return set_error(HFM_E_ARG, "a line longer than 4 GiB");
  if (format == HFM_READS_AUTO) {                 // the first non-blank character decides
    format = HFM_READS_FASTA;
    for (const Line& r : rl) {
      const Line l = trim(text, r);
      if (l.b > l.a) { if (text[l.a] == '@') format = HFM_READS_FASTQ; break; }
    }
  }
  // reads as lists of segments (a FASTA record's lines), in input order
  std::vector<Seg> segs;
  std::vector<uint64_t> first;                    // first segment of each read; one past the last at the end
  segs.reserve(rl.size() / 4 + 16);
  first.reserve(rl.size() / 4 + 16);
  if (format == HFM_READS_FASTA) {
    // src/wasm/js_api.rs:18-68: headers, blank lines, concatenated record lines, header-less lines
    bool in_record = false;
    uint64_t rec_first = 0;
    auto close_record = [&]() { if (in_record && segs.size() > rec_first) first.push_back(rec_first); };
    for (const Line& r : rl) {
      const Line l = trim(text, r);
      if (l.b == l.a) continue;
      if (text[l.a] == '>') {
        close_record();
        in_record = true;
        rec_first = segs.size();
      } else if (in_record) {
        segs.push_back({l.a, (uint32_t)(l.b - l.a)});
      } else {
        first.push_back(segs.size());
        segs.push_back({l.a, (uint32_t)(l.b - l.a)});
      }
    }
    close_record();
    if (first.empty()) return set_error(HFM_E_CHAR, "no sequences found in input");
  } else {
    // @name / sequence / +[name] / quality; blank lines between records are skipped
    for (size_t i = 0; i < rl.size();) {
      if (trim(text, rl[i]).b == trim(text, rl[i]).a) { i++; continue; }
      if (text[rl[i].a] != '@' || i + 3 >= rl.size() || rl[i + 2].b == rl[i + 2].a ||
          text[rl[i + 2].a] != '+')
        return set_error(HFM_E_FORMAT, "malformed FASTQ record at line " + std::to_string(i + 1));
      first.push_back(segs.size());
      const Line sq = trim(text, rl[i + 1]);
      segs.push_back({sq.a, (uint32_t)(sq.b - sq.a)});
      i += 4;
    }
  }
  const uint64_t nr = first.size();
  first.push_back(segs.size());
  std::vector<uint64_t> off(nr + 1, 0);
  for (uint64_t r = 0; r < nr; r++) {
    uint64_t L = 0;
    for (uint64_t k = first[r]; k < first[r + 1]; k++) L += segs[k].len;
    off[r + 1] = off[r] + L;
  }
  const uint64_t ncodes = off[nr];
  const size_t head = (sizeof(hfm_reads) + 15) & ~(size_t)15;
  uint8_t* blk = (uint8_t*)std::malloc(head + (nr + 1) * 8 + ncodes + 16);
  if (!blk) return set_error(HFM_E_OOM, "host allocation failed");
  hfm_reads* res = (hfm_reads*)blk;
  res->n = nr; res->n_codes = ncodes;
  res->offsets = (uint64_t*)(blk + head);
  res->codes = (uint8_t*)(res->offsets + nr + 1);
  std::memcpy(res->offsets, off.data(), (nr + 1) * 8);
  // encode blocks of reads on the host threads; each keeps its first invalid character
  if (ncodes < (8u << 20)) nt = 1;
  nt = (unsigned)std::min<uint64_t>(nt, std::max<uint64_t>(nr, 1));
  std::vector<uint64_t> bad(nt, ~0ull);          // first invalid code index per thread
  auto enc = [&](unsigned t) {
    const uint64_t r0 = nr * t / nt, r1 = nr * (t + 1) / nt;
    for (uint64_t r = r0; r < r1; r++) {
      uint8_t* dst = res->codes + off[r];
      for (uint64_t k = first[r]; k < first[r + 1]; k++) {
        const uint8_t* src = (const uint8_t*)text + segs[k].at;
        uint8_t acc = 0;
        for (uint32_t i = 0; i < segs[k].len; i++) { uint8_t c = kEnc.t[src[i]]; dst[i] = c; acc |= c; }
        if (acc & 0xF0) {
          for (uint32_t i = 0; i < segs[k].len; i++)
            if (dst[i] == 0xFF) { bad[t] = (uint64_t)(dst - res->codes) + i; return; }
        }
        dst += segs[k].len;
      }
    }
  };
  if (nt == 1) enc(0);
  else {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++) th.emplace_back(enc, t);
    for (auto& x : th) x.join();
  }
  const uint64_t b = *std::min_element(bad.begin(), bad.end());
  if (b != ~0ull) {
    const uint64_t r = (uint64_t)(std::upper_bound(off.begin(), off.end(), b) - off.begin()) - 1;
    // the character as written: walk the read's segments to the code's source byte
    uint64_t rem = b - off[r], at = 0;
    for (uint64_t k = first[r]; k < first[r + 1]; k++) {
      if (rem < segs[k].len) { at = segs[k].at + rem; break; }
      rem -= segs[k].len;
    }
    std::free(blk);
    return set_error(HFM_E_CHAR, std::string("invalid DNA character '") + text[at] + "' at position " +
                                     std::to_string(b - off[r]) + " of read " + std::to_string(r));
  }
  *out = res;
  return HFM_OK;
}
