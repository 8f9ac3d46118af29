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
  char buf[24];
  int n = snprintf(buf, sizeof buf, "%" PRIu64, v);
  out.append(buf, (size_t)n);
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
  char buf[96];
  if (format == RecordFormat::kCompact) {
    out += name;
    out += '\t';
    append_u64(out, total);
    out += '\t';
    for (size_t i = 0; i < hits; ++i) {
      int len = snprintf(buf, sizeof buf, i ? ",%u:%" PRIu64 : "%u:%" PRIu64, hit_colors[i],
                         hit_counts[i]);
      out.append(buf, (size_t)len);
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
    int len = snprintf(buf, sizeof buf, "\t%" PRIu64 "\t%" PRIu64 "\t%.8f\n", hit_counts[i], total,
                       ratio);
    out.append(buf, (size_t)len);
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
