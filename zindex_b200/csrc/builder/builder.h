// Index construction (the `zorindex build` side), restated on the host so
// indexes in the reference's directory format can be produced here: the
// reference builder is Rust and cannot be compiled on these machines.
// Construction is outside the GPU query path; its output format is what the
// query reads (manifest.json, bank-*.zorbank.zst, abandoned.zormap.zst).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "features_cpu.h"

namespace zx {

struct BuildOptions {
  std::string fof;     // one "name<TAB>path" (or "name path", or "path") per line
  std::string output;  // new index directory
  int hashes = 4;
  int fingerprint_bits = 8;
  FeatureParams features;
  double slot_scale = 1.0;
  uint64_t segment_length = 64;
  uint64_t min_subindex_documents = 128;
  int64_t max_subindexes = -1;  // -1: unlimited
  uint64_t max_subindex_size = 8ull << 30;
  bool drop_abandoned = false;
  int threads = 0;  // 0: hardware concurrency
  // Explicit dataset groups, e.g. "0,1,2;5,6": listed datasets share one
  // multi-member filter; every other dataset is a singleton group.
  std::string groups;
  // When set, genomes come from the seeded generator of synth.h instead of
  // the file of files ("kind:colors:min_len:max_len:seed").
  std::string synth;
  int zstd_level = 1;
  bool quiet = false;
  // Write banks in the legacy interleaved layout ("ZORPOW1", group fields
  // fingerprint then membership at each group's offset) instead of
  // fingerprint-first ("ZORPOW3").
  bool legacy_layout = false;
  // Construct on the GPU (build_index_device): distinct keys extracted,
  // sorted and deduplicated on the device and every filter peeled by one
  // device thread. Singleton groups of k-mer, minimizer and modimizer
  // indexes; the same directory format.
  bool device = false;
  int gpu = 0;  // CUDA device of the device builder
};

// Builds the index; throws zx::Error.
void build_index(const BuildOptions& options);

// Builder twin of layout::promotion_targets (src/power_merge/layout.rs:7-115):
// buckets are (slots, documents, width) sorted by slots; returns the target
// slots of each bucket.
std::vector<uint64_t> promotion_targets(const std::vector<uint64_t>& slots,
                                        const std::vector<uint64_t>& docs,
                                        const std::vector<uint64_t>& widths, uint64_t minimum,
                                        int64_t maximum);

}  // namespace zx
