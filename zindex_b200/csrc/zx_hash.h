// Integer mixing and seed arithmetic shared by the host runtime and the sm_100a
// kernels. Every function here is exact 64-bit wrapping arithmetic, so host and
// device produce identical bits.
//
// Reference formulas (Malfoy/Zindex):
//   splitmix64 / mixsplit ........ utils/ocm-minimizers/src/lib.rs:42-53
//   encode_base .................. utils/ocm-minimizers/src/lib.rs:7-15
//   canonical_encoded ............ utils/ocm-minimizers/src/lib.rs:31-40
//   fingerprint .................. src/power_merge/storage.rs:3214-3216
//   partition_id ................. src/power_merge/storage.rs:99-101
//   abandoned::hash .............. src/power_merge/abandoned.rs:5-10
//   PositionHash ................. src/power_merge/storage.rs:3452-3481
//   long k-mer polynomial hash ... src/lib.rs:683-731
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define ZX_HD __host__ __device__ __forceinline__
#else
#define ZX_HD static inline
#endif

namespace zx {

constexpr uint64_t kFingerprintSeed = 0x8E2D4F6A9B13C5D7ull;
constexpr uint64_t kPartitionSeed = 0x34B61D8F29A7C053ull;
constexpr uint64_t kRecoverySeed = 0xD6E8FEB86659FD93ull;
constexpr uint64_t kInnerHashSeed = 0xC6BC279692B5CC83ull;
constexpr uint64_t kLongKmerBase = 0x9e3779b185ebca87ull;
constexpr uint64_t kLongKmerDomain = 0x6b6d65722d763031ull;
constexpr int kMaxHashes = 32;

ZX_HD uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

ZX_HD uint64_t mixsplit(uint64_t key, uint64_t seed) { return splitmix64(key + seed); }

// A/a=0, C/c=1, G/g=2, T/t=3, anything else 4 (invalid).
ZX_HD uint32_t encode_base(uint8_t b) {
  switch (b) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return 4;
  }
}

ZX_HD uint64_t canonical_encoded(uint64_t encoded, int k) {
  uint64_t v = encoded, rc = 0;
  for (int i = 0; i < k; ++i) {
    rc = (rc << 2) | ((v & 3) ^ 3);
    v >>= 2;
  }
  return encoded < rc ? encoded : rc;
}

// Spaced seed (src/anchors.rs:10-90): a symmetric '#'/'_' pattern of width
// w <= 31 laid over a canonical k-mer (or minimizer m-mer) key, its first
// base in the key's top 2-bit field. The projection keeps the '#' bases in
// order (the reference's pext of the key with the 2-bit pattern mask); the
// seed's key is canonical_encoded(projection, weight). The '#' runs are
// precomputed so the projection is one shift-and-mask per run.
struct SpacedSeed {
  int width = 0, weight = 0, runs = 0;
  uint8_t shift[16] = {};  // per run, most significant first: source bit offset of its last base
  uint8_t len[16] = {};    // per run: bases
};

// Parses a pattern; returns false when it is invalid (the reference's rules:
// width 1..31, only '#' and '_', at least one '#', symmetric under reversal).
static inline bool parse_spaced_seed(const char* pattern, SpacedSeed* out) {
  int w = 0;
  while (pattern[w]) ++w;
  if (w < 1 || w > 31) return false;
  bool any = false;
  for (int i = 0; i < w; ++i) {
    if (pattern[i] != '#' && pattern[i] != '_') return false;
    if (pattern[i] != pattern[w - 1 - i]) return false;
    any |= pattern[i] == '#';
  }
  if (!any) return false;
  SpacedSeed p;
  p.width = w;
  for (int i = 0; i < w;) {
    if (pattern[i] != '#') {
      ++i;
      continue;
    }
    int j = i;
    while (j < w && pattern[j] == '#') ++j;
    // Bases i..j-1 sit at 2-bit fields w-1-i .. w-j (from the bottom).
    p.shift[p.runs] = (uint8_t)(2 * (w - j));
    p.len[p.runs] = (uint8_t)(j - i);
    ++p.runs;
    p.weight += j - i;
    i = j;
  }
  *out = p;
  return true;
}

ZX_HD uint64_t spaced_project(const SpacedSeed& p, uint64_t key) {
  uint64_t r = 0;
  for (int i = 0; i < p.runs; ++i) {
    const int bits = 2 * p.len[i];
    r = (r << bits) | ((key >> p.shift[i]) & ((1ull << bits) - 1));
  }
  return r;
}

// Reverse complement of a k-base 2-bit value (k <= 32).
ZX_HD uint64_t revcomp_encoded(uint64_t v, int k) {
#if defined(__CUDA_ARCH__)
  uint64_t y = __brevll(~v);
  y = ((y >> 1) & 0x5555555555555555ull) | ((y & 0x5555555555555555ull) << 1);
  return k == 32 ? y : y >> (64 - 2 * k);
#else
  uint64_t rc = 0;
  for (int i = 0; i < k; ++i) {
    rc = (rc << 2) | ((v & 3) ^ 3);
    v >>= 2;
  }
  return rc;
#endif
}

ZX_HD uint64_t spaced_canonical(const SpacedSeed& p, uint64_t key) {
  const uint64_t f = spaced_project(p, key), r = revcomp_encoded(f, p.weight);
  return f < r ? f : r;
}

// The strobe hash of a seed key (src/anchors.rs:136-151): XXH64 of the key's
// eight little-endian bytes with seed 0 (the published short-input rounds and
// avalanche).
ZX_HD uint64_t strobe_hash(uint64_t key) {
  const uint64_t P1 = 0x9E3779B185EBCA87ull, P2 = 0xC2B2AE3D27D4EB4Full,
                 P3 = 0x165667B19E3779F9ull, P4 = 0x85EBCA77C2B2AE63ull,
                 P5 = 0x27D4EB2F165667C5ull;
  uint64_t lane = key * P2;
  lane = ((lane << 31) | (lane >> 33)) * P1;
  uint64_t h = (P5 + 8) ^ lane;
  h = ((h << 27) | (h >> 37)) * P1 + P4;
  h = (h ^ (h >> 33)) * P2;
  h = (h ^ (h >> 29)) * P3;
  return h ^ (h >> 32);
}

ZX_HD uint64_t fingerprint(uint64_t key, uint64_t seed, int bits) {
  uint64_t mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
  return splitmix64(key ^ seed ^ kFingerprintSeed) & mask;
}

ZX_HD uint32_t partition_id(uint64_t key, uint64_t seed, uint32_t partitions) {
  return (uint32_t)(splitmix64(key ^ seed ^ kPartitionSeed) & (uint64_t)(partitions - 1));
}

ZX_HD uint32_t recovery_hash(uint64_t key, uint64_t seed) {
  return (uint32_t)(splitmix64(key ^ seed ^ kRecoverySeed) >> 32);
}

ZX_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// H cell positions of one key inside a bank of `cells` slots with segment
// length `seg` (a power of two).  Position i lives in segment base/seg + i.
ZX_HD void positions(uint64_t key, uint64_t seed, uint64_t cells, int hashes, uint64_t seg,
                     uint64_t* out) {
  uint64_t first = mixsplit(key, seed);
  uint64_t step = splitmix64(first);
  uint64_t count = cells / seg - (uint64_t)hashes + 1;
  uint64_t base = mulhi64(first, count) * seg;
  uint64_t h = first;
  for (int i = 0; i < hashes; ++i) {
    out[i] = base + (uint64_t)i * seg + ((h ^ (h >> 33)) & (seg - 1));
    h += step;
  }
}

// Segment length used by legacy (version <= 7) manifests without a fixed
// segment_length: the power-of-two floor of clamp(cells / H, 1, 4096).
ZX_HD uint64_t legacy_segment_length(uint64_t cells, int hashes) {
  uint64_t n = cells / (uint64_t)hashes;
  if (n < 1) n = 1;
  if (n > 4096) n = 4096;
  uint64_t p = 1;
  while ((p << 1) <= n) p <<= 1;
  return p;
}

// Constants of the rolling polynomial hash for k > 32: B^(k-1) and B^-1 mod 2^64.
struct LongKmerConsts {
  uint64_t power;    // B^(k-1)
  uint64_t inverse;  // B^-1
  uint64_t domain;   // splitmix64(k ^ domain tag)
};

ZX_HD LongKmerConsts long_kmer_consts(int k) {
  LongKmerConsts c;
  uint64_t inv = kLongKmerBase;
  for (int i = 0; i < 6; ++i) inv = inv * (2ull - kLongKmerBase * inv);
  uint64_t power = 1, base = kLongKmerBase;
  uint64_t e = (uint64_t)(k - 1);
  while (e) {
    if (e & 1) power *= base;
    base *= base;
    e >>= 1;
  }
  c.power = power;
  c.inverse = inv;
  c.domain = splitmix64((uint64_t)k ^ kLongKmerDomain);
  return c;
}

// Open-closed mod-minimizer geometry: w = k-m+1, t = r + (m-r) % w with
// r = min(4, m), s = min(4, t) minus one when t-s is odd.
struct OcmParams {
  int w, t, s;
};

ZX_HD OcmParams ocm_params(int k, int m) {
  OcmParams p;
  p.w = k - m + 1;
  int r = m < 4 ? m : 4;
  p.t = r + (m - r) % p.w;
  p.s = p.t < 4 ? p.t : 4;
  if ((p.t - p.s) & 1) p.s -= 1;
  return p;
}

}  // namespace zx
