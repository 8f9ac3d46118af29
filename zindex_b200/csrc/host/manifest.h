// Index directory model: manifest.json (src/power_merge/storage.rs:57-214)
// with the validation rules of Index::load_mode (storage.rs:2273-2570).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "json.h"

namespace zx {

enum IndexMode : int { kKmers = 0, kMinimizers = 1, kModimizers = 2, kFindere = 3 };
const char* index_mode_label(int mode);

struct GroupMeta {
  std::vector<uint32_t> members;
  uint64_t width = 0, offset = 0;
  uint64_t union_cardinality = 0, fallback_keys = 0;
  bool has_abandoned = false;
  uint64_t abandoned_keys = 0;
};

struct BankMeta {
  uint64_t component = 0;
  std::string file;
  uint64_t slots = 0, row_bits = 0;
  std::vector<GroupMeta> groups;
  bool fingerprint_first = false;
  bool routed = false;
  uint64_t source_slots = 0, partition = 0, partitions = 1;
  uint64_t row_bytes() const { return (row_bits + 7) / 8; }
  // Bytes of the fingerprint plane read per row (storage.rs:2798-2802).
  uint64_t lookup_bytes(int bits) const {
    return fingerprint_first ? (groups.size() * (uint64_t)bits + 7) / 8 : row_bytes();
  }
  std::string expected_filename() const;
};

struct ColorMeta {
  std::string name, path;
  uint64_t occurrences = 0, unique_kmers = 0;
};

struct Manifest {
  uint32_t version = 0;
  bool abandoned_recovery = true;
  bool has_abandoned_file = false;
  uint64_t abandoned_hashes = 0, abandoned_origins = 0;
  uint64_t k = 0;
  int hashes = 0;
  bool has_segment_length = false;
  uint64_t segment_length = 0;
  uint64_t seed = 0;
  int fingerprint_bits = 0;
  int index_mode = 0;
  uint64_t minimizer_size = 0;
  int minimizer_scheme = 0;  // 0 simd, 1 open-closed-mod
  bool homopolymer_compression = false;
  bool has_seed_pattern = false, has_randstrobemers = false;
  std::string seed_pattern;  // '#'/'_' spaced-seed pattern when has_seed_pattern
  uint64_t strobe_min = 0, strobe_max = 0;  // randstrobemer distances when has_randstrobemers
  std::string randstrobe_scheme;
  uint64_t modimizer_sampling = 16;
  uint64_t findere_z = 10;
  std::vector<ColorMeta> colors;
  std::vector<BankMeta> banks;
  // Source classes: consecutive banks sharing (component, source_slots); each
  // entry lists its bank ids in partition order.
  std::vector<std::vector<size_t>> classes;

  // Segment length used for a bank of `slots` cells.
  uint64_t segment_for(uint64_t slots) const;
};

// Parses and validates <dir>/manifest.json. Throws zx::Error.
Manifest load_manifest(const std::string& dir);
// Validation alone, for manifests built in memory.
void validate_manifest(Manifest& m);

}  // namespace zx
