// Shared phases of index construction, used by the host builder
// (builder.cpp) and the device builder (device_builder.cu): option checks
// and inputs, the bank layout (BuildConfig::slots, src/power_merge/mod.rs:
// 319-337; promotion, layout.rs:7-115; columns by width, storage.rs:
// 1644-1660; hash partitioning, storage.rs:1524-1642) and the index writer
// (bank files, the ZORABN2 recovery file, manifest.json, staging rename).
#pragma once
#include <atomic>
#include <chrono>
#include <exception>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../host/zstd_io.h"
#include "builder.h"
#include "synth.h"

namespace zx {
namespace build {

struct Input {
  std::string name, path;
};

struct Group {
  std::vector<uint32_t> members;  // sorted dataset ids; bit i <-> members[i]
  uint64_t width = 0;
  uint64_t cardinality = 0;
  uint64_t slots = 0;  // after promotion
  std::vector<uint64_t> keys, masks;
  // Filled during construction.
  uint64_t abandoned = 0;
  size_t cls = 0, column = 0;
  uint64_t offset = 0;
};

struct ClassLayout {
  uint64_t source_slots = 0, local_slots = 0, partitions = 1;
  std::vector<size_t> groups;  // in column order
  uint64_t row_bits = 0;
  // Host builder: per partition, slots * row_bytes bytes as u64 words (the
  // device builder keeps its rows in device memory).
  std::vector<std::vector<uint64_t>> rows;
};

struct Abandoned {
  uint32_t hash;
  uint32_t group;
  uint64_t mask;
};

template <class F>
void parallel_for(size_t n, int threads, F&& body) {
  std::atomic<size_t> next{0};
  std::vector<std::thread> pool;
  std::mutex mu;
  std::exception_ptr error;
  auto worker = [&] {
    for (size_t i; (i = next.fetch_add(1)) < n;) {
      try {
        body(i);
      } catch (...) {
        std::lock_guard<std::mutex> lock(mu);
        if (!error) error = std::current_exception();
        next = n;
      }
    }
  };
  int t = std::max(1, std::min<int>(threads, (int)n));
  for (int i = 1; i < t; ++i) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  if (error) std::rethrow_exception(error);
}

// Everything the phases share.
struct Context {
  BuildOptions opt;
  FeatureParams fp;
  int H = 0, b = 0, threads = 0;
  std::chrono::steady_clock::time_point t0;
  std::vector<Input> inputs;
  synth::GenomeSpec spec;  // when opt.synth is set
  std::vector<uint64_t> occurrences;  // features per dataset, repeats included
  std::vector<Group> groups;
  std::vector<ClassLayout> classes;
  std::vector<size_t> class_order;  // banks in increasing source-slot order
  bool partitioned = false;
  size_t promoted = 0;
  std::vector<Abandoned> abandoned;  // recovery records (empty with drop_abandoned)
};

double seconds_since(std::chrono::steady_clock::time_point t);
uint64_t next_pow2(uint64_t v);
// Option checks and the datasets (file of files or synthetic genomes).
void prepare(const BuildOptions& options, Context& bc);
// BuildConfig::slots (mod.rs:319-337) of a group of `cardinality` keys.
uint64_t config_slots(const BuildOptions& opt, int H, uint64_t cardinality);
// Promotion, classes, columns and partitions from the groups' slots and
// widths; host_rows allocates the host row buffers.
void plan_layout(Context& bc, bool host_rows);
// Writes the index: the payload of (class, partition) is produced by
// `payload` into the bank's framed writer (after its 40-byte header), one
// bank at a time when payload_threads is 1.
using PayloadFn = std::function<void(size_t cls, uint64_t partition, FramedWriter& w)>;
void write_index(Context& bc, const PayloadFn& payload, int payload_threads);

}  // namespace build

// The device builder (device_builder.cu; singleton groups of k-mer,
// minimizer or modimizer indexes).
void build_index_device(const BuildOptions& options);

}  // namespace zx
