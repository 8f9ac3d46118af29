// Seeded synthetic genomes for the benchmark workloads (no datasets are
// available offline). Every base is a pure function of (seed, genome,
// position), so reads can be sampled without materialising a genome.
//
// uniform: genome i = dna(len, seed + i) with dna(n, s)[j] =
//   "ACGT"[splitmix64(j ^ s) & 3] (the reference tests' generator).
// pool: lengths log-uniform in [min_len, max_len]; each 100 kbp block is,
//   with probability 0.3, a copy of one of 50 seeded 100 kbp core segments
//   (shared across genomes), otherwise i.i.d. uniform bases.
#pragma once
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../zx_hash.h"

namespace zx {
namespace synth {

constexpr uint64_t kBlock = 100000;
constexpr int kCoreSegments = 50;

struct GenomeSpec {
  std::string kind = "uniform";
  uint64_t colors = 10, min_len = 2000000, max_len = 2000000, seed = 1;
};

inline double unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

inline uint64_t genome_length(const GenomeSpec& s, uint64_t g) {
  if (s.kind == "uniform" || s.min_len == s.max_len) return s.min_len;
  double lo = std::log((double)s.min_len), hi = std::log((double)s.max_len);
  double u = unit(splitmix64(s.seed ^ splitmix64(0x6c656e67746800ull + g)));
  return (uint64_t)std::floor(std::exp(lo + u * (hi - lo)));
}

// Base `pos` of genome g (host and device: the device builder generates the
// same genomes in place).
ZX_HD char synth_base(bool pool, uint64_t seed, uint64_t g, uint64_t pos) {
  if (!pool) return "ACGT"[splitmix64(pos ^ (seed + g)) & 3];
  uint64_t block = pos / kBlock, off = pos % kBlock;
  uint64_t r = splitmix64(splitmix64(seed ^ 0x626c6f636bull) ^ (g << 24) ^ block);
  if (r % 1000 < 300) {
    uint64_t core = (r >> 32) % kCoreSegments;
    return "ACGT"[splitmix64(off ^ splitmix64(seed ^ 0x636f7265ull ^ (core << 40))) & 3];
  }
  return "ACGT"[splitmix64(pos ^ splitmix64(seed ^ 0x67656e6f6dull ^ (g << 20))) & 3];
}

inline char genome_base(const GenomeSpec& s, uint64_t g, uint64_t pos) {
  return synth_base(s.kind != "uniform", s.seed, g, pos);
}

inline void genome(const GenomeSpec& s, uint64_t g, std::vector<uint8_t>& out) {
  uint64_t n = genome_length(s, g);
  out.resize(n);
  for (uint64_t p = 0; p < n; ++p) out[p] = (uint8_t)genome_base(s, g, p);
}

// "kind:colors:min_len:max_len:seed", e.g. "pool:256:1000000:10000000:1".
inline bool parse_spec(const std::string& text, GenomeSpec& s) {
  std::vector<std::string> f;
  size_t a = 0;
  while (true) {
    size_t b = text.find(':', a);
    f.push_back(text.substr(a, b == std::string::npos ? std::string::npos : b - a));
    if (b == std::string::npos) break;
    a = b + 1;
  }
  if (f.size() != 5) return false;
  s.kind = f[0];
  s.colors = std::stoull(f[1]);
  s.min_len = std::stoull(f[2]);
  s.max_len = std::stoull(f[3]);
  s.seed = std::stoull(f[4]);
  return (s.kind == "uniform" || s.kind == "pool") && s.colors > 0 && s.min_len > 0 &&
         s.max_len >= s.min_len;
}

}  // namespace synth
}  // namespace zx
