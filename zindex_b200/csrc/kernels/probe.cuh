// Interleaved-ZOR membership probe of one seed (K5 + K6).
//
// Follows Index::lookup_selected (src/power_merge/storage.rs:2761-2925) for
// fingerprint-first banks: one recovery-map probe per seed (abandoned.rs:
// 5-10, 180-205), then per source class the partition bank (partition_id,
// storage.rs:99-101; selected_banks 2717-2745), the H cell positions
// (PositionHash, 3452-3481), the XOR of the H fingerprint-plane rows and a
// compare of every b-bit field with fingerprint(key) (3214-3216,
// 3241-3350, packed_fingerprints.rs:7-126). A hit on group i adds one to
// its member, or XOR-decodes the members' bits (get_bits, 3523-3538;
// 2826-2842). Recovered origins count once per seed whether or not a
// filter also hit them (2769-2787, 2916-2924).
//
// A team of T lanes shares one seed: lane j of the team gathers 16-byte
// chunks j, j+T, ... of the fingerprint plane of each of the H rows.
#pragma once
#include <stdint.h>

#include "../zx_hash.h"
#include "device_index.cuh"

namespace zx {

// Lowest bit of every b-bit field of a 32-bit word.
__device__ __forceinline__ uint32_t field_ones(int b) {
  return b == 32 ? 1u : 0xFFFFFFFFu / ((1u << b) - 1u);
}

// Bit set at the low bit of each b-bit field of `x` that is zero.
__device__ __forceinline__ uint32_t zero_fields(uint32_t x, int b, uint32_t ones) {
#pragma unroll
  for (int s = 1; s < 32; s <<= 1)
    if (s < b) x |= x >> s;
  return ~x & ones;
}

__device__ __forceinline__ uint4 ld_row_chunk(const uint8_t* p) {
  return __ldg(reinterpret_cast<const uint4*>(p));
}

// Little-endian bit field of up to 64 bits inside one row.
__device__ __forceinline__ uint64_t row_bits(const uint8_t* row, uint32_t off, uint32_t width) {
  uint32_t byte = off >> 3, shift = off & 7;
  uint32_t nbytes = (shift + width + 7) >> 3;
  uint64_t lo = 0, hi = 0;
  for (uint32_t i = 0; i < nbytes && i < 8; ++i) lo |= (uint64_t)__ldg(row + byte + i) << (8 * i);
  if (nbytes == 9) hi = __ldg(row + byte + 8);
  uint64_t v = lo >> shift;
  if (shift) v |= hi << (64 - shift);
  return width >= 64 ? v : v & ((1ull << width) - 1);
}

// Recovered origins of a key: an inline origin (list == nullptr, len == 1)
// or a posting list in global memory.
struct RecHit {
  const uint32_t* list;
  uint32_t len;
  uint32_t single;
  __device__ __forceinline__ uint32_t at(uint32_t i) const { return list ? __ldg(list + i) : single; }
};

__device__ __forceinline__ RecHit recovery_lookup(const DevRecovery& rec, uint32_t h) {
  RecHit r{nullptr, 0, 0};
  if (!rec.bits) return r;
  const uint64_t mask = (1ull << rec.bits) - 1;
  uint64_t slot = (uint64_t)(h >> (32 - rec.bits));
  for (uint64_t probes = 0; probes <= mask; ++probes) {
    uint64_t e = __ldg(rec.dir + slot);
    uint32_t value = (uint32_t)e;
    if (value == kRecEmpty) return r;
    if ((uint32_t)(e >> 32) == h) {
      if (!(value & kRecMultiple)) {
        r.single = value;
        r.len = 1;
        return r;
      }
      uint2 g = __ldg(rec.ranges + (value & ~kRecMultiple));
      r.list = rec.origins + g.x;
      r.len = g.y;
      return r;
    }
    slot = (slot + 1) & mask;
  }
  return r;
}

// Whether colour c is among the (sorted) recovered origins.
__device__ __forceinline__ bool rec_contains(const RecHit& r, uint32_t c) {
  if (!r.list) return r.len && r.single == c;
  if (r.len <= 8) {
    for (uint32_t i = 0; i < r.len; ++i)
      if (__ldg(r.list + i) == c) return true;
    return false;
  }
  uint32_t lo = 0, hi = r.len;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    uint32_t v = __ldg(r.list + mid);
    if (v == c) return true;
    if (v < c) lo = mid + 1;
    else hi = mid;
  }
  return false;
}

// Counter sink: per-block shared counters, or global 64-bit counters.
struct Counters {
  uint32_t* smem;   // colours entries, or nullptr
  uint64_t* gmem;   // used when smem is null
  __device__ __forceinline__ void add(uint32_t c) const {
    if (smem) atomicAdd(smem + c, 1u);
    else atomicAdd(reinterpret_cast<unsigned long long*>(gmem + c), 1ull);
  }
};

// Visits every colour hit by the filters for `key` (excluding recovered
// origins, which the caller counts once). Template hook `on_hit(colour)`.
template <class OnHit>
__device__ __forceinline__ void probe_filters(const DevIndex& ix, uint64_t key, int tl, int T,
                                              OnHit&& on_hit) {
  const int H = ix.hashes, b = ix.bits;
  const uint32_t ones = field_ones(b);
  const uint32_t fp = (uint32_t)fingerprint(key, ix.seed, b);
  const uint32_t pattern = fp * ones;
  const uint64_t first = mixsplit(key, ix.seed), step = splitmix64(first);
  const int fields_per_word = 32 / b;
  for (uint32_t ci = 0; ci < ix.classes; ++ci) {
    const DevClass& C = ix.cls[ci];
    if ((uint32_t)tl >= C.fp_chunks) continue;
    const uint32_t part = C.partitions > 1 ? partition_id(key, ix.seed, C.partitions) : 0;
    const uint64_t seg = C.seg;
    const uint64_t count = C.slots / seg - (uint64_t)H + 1;
    const uint64_t base = mulhi64(first, count) * seg;
    const uint8_t* bank = C.data + (uint64_t)part * C.slots * C.row_stride;
    for (uint32_t chunk = tl; chunk < C.fp_chunks; chunk += T) {
      uint4 acc = make_uint4(0, 0, 0, 0);
      for (int i0 = 0; i0 < H; i0 += 4) {
        uint4 v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          int i = i0 + j;
          if (i < H) {
            uint64_t h = first + (uint64_t)i * step;
            uint64_t slot = base + (uint64_t)i * seg + ((h ^ (h >> 33)) & (seg - 1));
            v[j] = ld_row_chunk(bank + slot * C.row_stride + chunk * 16u);
          } else {
            v[j] = make_uint4(0, 0, 0, 0);
          }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc.x ^= v[j].x;
          acc.y ^= v[j].y;
          acc.z ^= v[j].z;
          acc.w ^= v[j].w;
        }
      }
      const uint32_t words[4] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
      for (int wi = 0; wi < 4; ++wi) {
        uint32_t field0 = chunk * (uint32_t)(4 * fields_per_word) + (uint32_t)(wi * fields_per_word);
        if (field0 >= C.groups) break;
        uint32_t hits = zero_fields(words[wi] ^ pattern, b, ones);
        uint32_t valid = C.groups - field0;
        if (valid < (uint32_t)fields_per_word) hits &= (1u << (valid * b)) - 1u;
        while (hits) {
          uint32_t bit = __ffs(hits) - 1;
          hits &= hits - 1;
          uint32_t group = field0 + bit / b;
          uint32_t gc = __ldg(C.group_color + group);
          if (!(gc & kMultiGroup)) {
            on_hit(gc);
            continue;
          }
          const uint32_t* mg = C.multi + 3 * (gc & ~kMultiGroup);
          uint32_t off = __ldg(mg), cnt = __ldg(mg + 1), firstm = __ldg(mg + 2);
          uint64_t mask = 0;
          for (int i = 0; i < H; ++i) {
            uint64_t h = first + (uint64_t)i * step;
            uint64_t slot = base + (uint64_t)i * seg + ((h ^ (h >> 33)) & (seg - 1));
            mask ^= row_bits(bank + slot * C.row_stride, off, cnt);
          }
          while (mask) {
            uint32_t mb = __ffsll((long long)mask) - 1;
            mask &= mask - 1;
            on_hit(__ldg(C.members + firstm + mb));
          }
        }
      }
    }
  }
}

// Aggregate probe of one seed: filter hits not covered by the recovery list
// plus every recovered origin, each counted once.
__device__ __forceinline__ void probe_seed(const DevIndex& ix, uint64_t key, int tl, int T,
                                           const Counters& cnt) {
  const RecHit rec = recovery_lookup(ix.rec, recovery_hash(key, ix.seed));
  probe_filters(ix, key, tl, T, [&](uint32_t c) {
    if (rec.len && rec_contains(rec, c)) return;
    cnt.add(c);
  });
  if (tl == 0)
    for (uint32_t i = 0; i < rec.len; ++i) cnt.add(rec.at(i));
}

}  // namespace zx
