// Per-record query report (`zorindex query --records`): the two output
// formats of the reference's record query (src/power_merge/record_output.rs)
// and its colour selection (RecordScores::write_record,
// src/power_merge/storage.rs:3109-3146).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "manifest.h"

namespace zx {

enum class RecordFormat {
  kTsv,      // query_id, dataset_id, dataset_name, matches, queried_seeds, ratio
  kCompact,  // query_id, valid_kmers, hits (comma-separated dataset_id:count)
};

// Header line (without '\n') of a format.
const char* record_header(RecordFormat format);

// Appends the lines of one record. counts holds one entry per colour. With
// min_ratio 0 every colour is reported; otherwise the colours with a non-zero
// count whose ratio count / total reaches min_ratio, in colour order. TSV
// writes one row per reported colour, or one "no hit" row; compact writes one
// row. TSV names are CSV-quoted when they hold a tab, CR, LF or quote.
void append_record(std::string& out, RecordFormat format, const std::string& name, uint64_t total,
                   const uint64_t* counts, const std::vector<ColorMeta>& colors, double min_ratio);

// Appends the lines of one record whose reported colours are already chosen:
// hit_colors[i] (ascending) with count hit_counts[i], i < hits.
void append_record_hits(std::string& out, RecordFormat format, const std::string& name,
                        uint64_t total, const uint32_t* hit_colors, const uint64_t* hit_counts,
                        size_t hits, const std::vector<ColorMeta>& colors);

}  // namespace zx
