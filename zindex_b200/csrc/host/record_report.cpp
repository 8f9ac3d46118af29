#include "record_report.h"

#include <cinttypes>
#include <cstdio>
#include <cstring>

namespace zx {

namespace {

// write_field (src/power_merge/record_output.rs:64-80): standard CSV quoting.
void append_field(std::string& out, const std::string& v) {
  if (v.find_first_of("\t\r\n\"") == std::string::npos) {
    out += v;
    return;
  }
  out += '"';
  size_t from = 0;
  for (size_t q; (q = v.find('"', from)) != std::string::npos; from = q + 1) {
    out.append(v, from, q + 1 - from);
    out += '"';
  }
  out.append(v, from, std::string::npos);
  out += '"';
}

inline void append_u64(std::string& out, uint64_t v) {
  char buf[20];
  int n = 0;
  do {
    buf[n++] = (char)('0' + v % 10);
    v /= 10;
  } while (v);
  while (n) out += buf[--n];
}

// `{:.8}` of a non-negative double (Rust's fixed-point formatting, like a
// correctly rounding printf's "%.8f"): the exact binary value times 10^8,
// rounded to the nearest integer with ties to even, in fixed point. A
// normal double is m * 2^(E - 1075) with a 53-bit m; m * 10^8 fits in 81 bits.
void append_fixed8(std::string& out, double r) {
  uint64_t bits;
  memcpy(&bits, &r, 8);
  const int biased = (int)((bits >> 52) & 0x7FF);
  if (r == 0.0 || biased == 0) {  // zero (ratios are never subnormal)
    out += "0.00000000";
    return;
  }
  const int sh = 1075 - biased;  // r = m / 2^sh
  if (sh <= 0 || biased == 0x7FF) {  // huge or not finite: never a ratio
    char buf[400];
    int n = snprintf(buf, sizeof buf, "%.8f", r);
    out.append(buf, (size_t)n);
    return;
  }
  const uint64_t m = (bits & ((1ull << 52) - 1)) | (1ull << 52);
  const unsigned __int128 num = (unsigned __int128)m * 100000000u;
  uint64_t q = 0;
  if (sh < 128) {
    const unsigned __int128 whole = num >> sh;
    const unsigned __int128 rem = num - (whole << sh);
    const unsigned __int128 half = (unsigned __int128)1 << (sh - 1);
    q = (uint64_t)whole;
    if (rem > half || (rem == half && (q & 1))) ++q;
  }
  append_u64(out, q / 100000000u);
  out += '.';
  char frac[8];
  uint64_t f = q % 100000000u;
  for (int i = 7; i >= 0; --i, f /= 10) frac[i] = (char)('0' + f % 10);
  out.append(frac, 8);
}

}  // namespace

const char* record_header(RecordFormat format) {
  return format == RecordFormat::kCompact
             ? "query_id\tvalid_kmers\thits"
             : "query_id\tdataset_id\tdataset_name\tmatches\tqueried_seeds\tratio";
}

void append_record_hits(std::string& out, RecordFormat format, const std::string& name,
                        uint64_t total, const uint32_t* hit_colors, const uint64_t* hit_counts,
                        size_t hits, const std::vector<ColorMeta>& colors) {
  if (format == RecordFormat::kCompact) {
    out += name;
    out += '\t';
    append_u64(out, total);
    out += '\t';
    for (size_t i = 0; i < hits; ++i) {
      if (i) out += ',';
      append_u64(out, hit_colors[i]);
      out += ':';
      append_u64(out, hit_counts[i]);
    }
    out += '\n';
    return;
  }
  for (size_t i = 0; i < hits; ++i) {
    const uint32_t c = hit_colors[i];
    append_field(out, name);
    out += '\t';
    append_u64(out, c);
    out += '\t';
    append_field(out, colors[c].name);
    const double ratio = total == 0 ? 0.0 : (double)hit_counts[i] / (double)total;
    out += '\t';
    append_u64(out, hit_counts[i]);
    out += '\t';
    append_u64(out, total);
    out += '\t';
    append_fixed8(out, ratio);
    out += '\n';
  }
  if (!hits) {
    append_field(out, name);
    out += "\t.\t.\t0\t";
    append_u64(out, total);
    out += "\t0.00000000\n";
  }
}

void append_record(std::string& out, RecordFormat format, const std::string& name, uint64_t total,
                   const uint64_t* counts, const std::vector<ColorMeta>& colors, double min_ratio) {
  // Colour c is reported when min_ratio is 0, or when it was touched (count
  // > 0), total > 0 and count / total >= min_ratio.
  thread_local std::vector<uint32_t> hc;
  thread_local std::vector<uint64_t> hn;
  hc.clear();
  hn.clear();
  for (size_t c = 0; c < colors.size(); ++c) {
    if (min_ratio != 0.0 &&
        (total == 0 || counts[c] == 0 || !((double)counts[c] / (double)total >= min_ratio)))
      continue;
    hc.push_back((uint32_t)c);
    hn.push_back(counts[c]);
  }
  append_record_hits(out, format, name, total, hc.data(), hn.data(), hc.size(), colors);
}

}  // namespace zx
