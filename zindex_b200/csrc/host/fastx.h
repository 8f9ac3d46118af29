// FASTA/FASTQ reader producing one contiguous byte buffer of record
// sequences. It follows the parser configuration of the reference query
// (src/lib.rs:27-33: headers and qualities ignored, multi-line FASTA joined,
// LF or CRLF line ends). Non-ACGT bytes stay in place; the device seed
// kernels split runs at them, as split_non_actg does on the host in the
// reference. gzip and zstd inputs are decoded (src/lib.rs:283-321, 540-552).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace zx {

struct RecordBatch {
  std::vector<uint8_t> bases;      // concatenated sequences
  std::vector<uint64_t> offsets;   // records + 1 entries
  std::vector<std::string> names;  // first whitespace token of each header (optional)
  size_t records() const { return offsets.empty() ? 0 : offsets.size() - 1; }
};

// Parses a whole FASTA/FASTQ file. Throws zx::Error (kEFormat, kEIo).
RecordBatch read_fastx(const std::string& path, bool keep_names);
// Parses FASTA/FASTQ bytes already in memory.
void parse_fastx(const uint8_t* data, size_t len, RecordBatch& out, bool keep_names);

// Named records for per-record reports, under the stricter rules of the
// reference's record reader (src/power_merge/records.rs:150-290): trailing
// ASCII whitespace of a line is dropped and empty lines are skipped; the
// first line decides FASTQ ('@') or FASTA; the identifier is the header up to
// the first whitespace and must be non-empty UTF-8; sequence lines may not
// hold whitespace; FASTQ sequences run until the '+' line and qualities are
// consumed by length; at least one record is required. Throws zx::Error
// (kEFormat, kEIo) with the reference's messages.
RecordBatch read_named_records(const std::string& path);
void parse_named_records(const uint8_t* data, size_t len, RecordBatch& out);

}  // namespace zx
