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

// Bit set at the top bit of each b-bit field of `x` that is zero, for any
// b in {1,2,4,8,16,32}: adding the low-bits mask carries into a field's top
// bit exactly when the field's low bits are nonzero (no carry crosses a
// field); hi = ones << (b - 1).
__device__ __forceinline__ uint32_t zero_fields_hi(uint32_t x, uint32_t hi) {
  const uint32_t lo = ~hi;
  const uint32_t t = (x & lo) + lo;
  return ~(t | x) & hi;
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
  __device__ __forceinline__ void add(uint32_t c, uint32_t n = 1) const {
    if (smem) atomicAdd(smem + c, n);
    else atomicAdd(reinterpret_cast<unsigned long long*>(gmem + c), (unsigned long long)n);
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

// ---- warp-cooperative probe of a batch of seeds -----------------------------
// The scalar part of each seed (fingerprint, position hash, partition choice,
// recovery probe) is computed once by an owner lane into a shared-memory
// descriptor; teams of T lanes then gather the fingerprint-plane chunks of two
// seeds at a time so each lane keeps 2 * H 16-byte loads in flight.
struct SeedDesc {
  uint64_t first, step;
  const uint32_t* rec_list;
  uint32_t pattern;  // fingerprint replicated over every b-bit field of a word
  uint32_t rec_len, rec_single;
  uint32_t live;  // row-index probe: 1 when the seed is probed (findere skips invalid s-mers)
};

__device__ __forceinline__ bool desc_rec_contains(const SeedDesc& d, uint32_t c) {
  RecHit r{d.rec_list, d.rec_len, d.rec_single};
  return rec_contains(r, c);
}

// Row-address offset (within the class allocation) of row i of a seed.
__device__ __forceinline__ uint64_t row_offset(uint64_t row0, uint64_t h, int i, uint64_t seg,
                                               uint32_t stride) {
  uint32_t low = ((uint32_t)h ^ (uint32_t)(h >> 33)) & (uint32_t)(seg - 1);
  return row0 + ((uint64_t)i * seg + low) * stride;
}

// Fields of one XORed 16-byte chunk equal to the fingerprint -> on_hit(group).
template <class OnGroup>
__device__ __forceinline__ void chunk_hits(const uint4& acc, uint32_t chunk, uint32_t groups, int b,
                                           uint32_t ones, uint32_t pattern, OnGroup&& on_group) {
  const int fpw = 32 / b;
  const uint32_t words[4] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
  for (int wi = 0; wi < 4; ++wi) {
    uint32_t field0 = chunk * (uint32_t)(4 * fpw) + (uint32_t)(wi * fpw);
    if (field0 >= groups) break;
    uint32_t hits = zero_fields(words[wi] ^ pattern, b, ones);
    uint32_t valid = groups - field0;
    if (valid < (uint32_t)fpw) hits &= (1u << (valid * b)) - 1u;
    while (hits) {
      uint32_t bit = __ffs(hits) - 1;
      hits &= hits - 1;
      on_group(field0 + bit / b);
    }
  }
}

// Colours of a hit group (singleton, or XOR-decoded members).
template <class OnHit>
__device__ __forceinline__ void group_hit(const DevClass& C, uint32_t group, const SeedDesc& d,
                                          uint64_t row0, int H, OnHit&& on_hit) {
  uint32_t gc = __ldg(C.group_color + group);
  if (!(gc & kMultiGroup)) {
    on_hit(gc);
    return;
  }
  const uint32_t* mg = C.multi + 3 * (gc & ~kMultiGroup);
  uint32_t off = __ldg(mg), cnt = __ldg(mg + 1), firstm = __ldg(mg + 2);
  uint64_t mask = 0, h = d.first;
  for (int i = 0; i < H; ++i, h += d.step)
    mask ^= row_bits(C.data + row_offset(row0, h, i, C.seg, C.row_stride), off, cnt);
  while (mask) {
    uint32_t mb = __ffsll((long long)mask) - 1;
    mask &= mask - 1;
    on_hit(__ldg(C.members + firstm + mb));
  }
}

// Probes keys[0..n) (shared memory) with the whole warp. Per round of 32
// seeds each lane fills the descriptor of one seed (and its per-class row
// offset of position 0); teams of T lanes then gather two seeds at a time,
// computing row addresses in registers.
__device__ void probe_batch(const DevIndex& ix, const uint64_t* keys, uint32_t n, SeedDesc* desc,
                            uint64_t* row0s, int T, const Counters& cnt, int lane) {
  const int H = ix.hashes, b = ix.bits;
  const uint32_t ones = field_ones(b);
  const uint32_t classes = ix.classes;
  const int team = lane / T, tl = lane % T, nteams = 32 / T;
  for (uint32_t r0 = 0; r0 < n; r0 += 32) {
    const uint32_t m = min(32u, n - r0);
    if ((uint32_t)lane < m) {
      const uint64_t key = keys[r0 + lane];
      SeedDesc d;
      d.first = mixsplit(key, ix.seed);
      d.step = splitmix64(d.first);
      d.pattern = (uint32_t)fingerprint(key, ix.seed, b) * ones;
      RecHit r = recovery_lookup(ix.rec, recovery_hash(key, ix.seed));
      d.rec_list = r.list;
      d.rec_len = r.len;
      d.rec_single = r.single;
      d.live = 1;
      desc[lane] = d;
      for (uint32_t ci = 0; ci < classes; ++ci) {
        const DevClass& C = ix.cls[ci];
        const uint32_t part = C.partitions > 1 ? partition_id(key, ix.seed, C.partitions) : 0;
        const uint64_t count = C.slots / C.seg - (uint64_t)H + 1;
        const uint64_t base = mulhi64(d.first, count) * C.seg;
        row0s[lane * classes + ci] = ((uint64_t)part * C.slots + base) * C.row_stride;
      }
      for (uint32_t i = 0; i < r.len; ++i) cnt.add(r.at(i));
    }
    __syncwarp();
    for (uint32_t ci = 0; ci < classes; ++ci) {
      const DevClass& C = ix.cls[ci];
      if ((uint32_t)tl >= C.fp_chunks) continue;
      const uint64_t seg = C.seg;
      const uint32_t stride = C.row_stride;
      for (uint32_t s = team; s < m; s += 2 * nteams) {
        const uint32_t s2 = s + nteams;
        const bool two = s2 < m;
        const SeedDesc& da = desc[s];
        const SeedDesc& db = desc[two ? s2 : s];
        const uint64_t ra = row0s[s * classes + ci];
        const uint64_t rb = row0s[(two ? s2 : s) * classes + ci];
        for (uint32_t chunk = tl; chunk < C.fp_chunks; chunk += T) {
          uint4 aa = make_uint4(0, 0, 0, 0), ab = make_uint4(0, 0, 0, 0);
          uint64_t ha = da.first, hb = db.first;
          for (int i0 = 0; i0 < H; i0 += 4) {
            uint4 va[4], vb[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int i = i0 + j;
              va[j] = vb[j] = make_uint4(0, 0, 0, 0);
              if (i < H) {
                va[j] = ld_row_chunk(C.data + row_offset(ra, ha, i, seg, stride) + chunk * 16u);
                if (two) vb[j] = ld_row_chunk(C.data + row_offset(rb, hb, i, seg, stride) + chunk * 16u);
                ha += da.step;
                hb += db.step;
              }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              aa.x ^= va[j].x; aa.y ^= va[j].y; aa.z ^= va[j].z; aa.w ^= va[j].w;
              ab.x ^= vb[j].x; ab.y ^= vb[j].y; ab.z ^= vb[j].z; ab.w ^= vb[j].w;
            }
          }
          chunk_hits(aa, chunk, C.groups, b, ones, da.pattern, [&](uint32_t g) {
            group_hit(C, g, da, ra, H, [&](uint32_t c) {
              if (da.rec_len && desc_rec_contains(da, c)) return;
              cnt.add(c);
            });
          });
          if (two)
            chunk_hits(ab, chunk, C.groups, b, ones, db.pattern, [&](uint32_t g) {
              group_hit(C, g, db, rb, H, [&](uint32_t c) {
                if (db.rec_len && desc_rec_contains(db, c)) return;
                cnt.add(c);
              });
            });
        }
      }
    }
    __syncwarp();
  }
}

// ---- row-index probe with bit-plane colour counters -------------------------
// The owner lane of each seed writes, besides the descriptor, the row index
// (partition * slots + cell; below 2^32 because a class holds at most 64 GiB
// of rows of at least 16 bytes) of each of its H cells per class, so a team
// gathers with one multiply-add per row. A lane always covers the same
// fingerprint fields of a class (chunks tl, tl + T, ...), so its hits are
// counted per field in vertical binary counters held in registers (bit p of
// plane k is bit k of the count of field p) and added to the colour counters
// only every few dozen seeds, instead of one shared-memory atomic per hit.
// The first class whose fields of a lane fit one 32-bit dense word (4 x
// chunks per lane <= b) keeps its planes in registers; the next classes, up
// to kMaxSharedPlaneWords dense words per lane in all, keep theirs in the
// warp's shared memory (each lane owns its words: no atomics, no bank
// conflicts), which is what wide rows with many matching fields need (4 KiB
// rows hit by hundreds of colours, or 8 KiB rows of 4-bit fingerprints with a
// 1/16 chance of a false match per group). Hits on multi-member groups,
// every hit of a seed with recovered origins, and hits in the remaining
// classes take the per-hit path (membership decode, recovered-origin
// exclusion).
constexpr int kPlanes = 6;            // register planes: counts up to 63 per field
constexpr uint32_t kPlaneFlush = 31;  // team steps (two seeds each) between flushes
constexpr int kSharedPlanes = 5;      // shared planes: counts up to 31 per field
constexpr uint32_t kSharedFlush = 15; // team steps (two seeds each) between flushes
constexpr uint32_t kMaxSharedPlaneWords = 32;
constexpr uint16_t kNoPlanes = 0xFFFF;

__host__ __device__ __forceinline__ int log2_bits(int b) {
  int l = 0;
  while ((1 << (l + 1)) <= b) ++l;
  return l;
}

// Dense layout of a lane's fields in a class: word q of the lane (its chunk
// q / 4, 32-bit word q % 4 of that chunk) has its field-match flags at bits
// f * b + b - 1 (zero_fields_hi); they move to dense word q / b, bits
// f * b + q % b. Returns the group of dense word d, bit `bit`.
__device__ __forceinline__ uint32_t dense_group(uint32_t bit, uint32_t d, int b, int lb, int tl, int T) {
  const uint32_t r = bit & (uint32_t)(b - 1), f = bit >> lb;
  const uint32_t q = d * (uint32_t)b + r;
  const uint32_t chunk = (uint32_t)tl + (q >> 2) * (uint32_t)T;
  return chunk * (128u >> lb) + (q & 3u) * (32u >> lb) + f;
}

struct LanePlanes {
  uint32_t c[kPlanes];
  uint32_t valid;  // dense positions that are fields of the lane
  uint32_t multi;  // dense positions whose group has several members
  int cls;         // class counted in the planes (-1: none)
  uint32_t steps;
};

__device__ __forceinline__ void plane_add(uint32_t (&c)[kPlanes], uint32_t m) {
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) {
    const uint32_t t = c[k] & m;
    c[k] ^= m;
    m = t;
  }
}

// Dense words a lane needs for class C.
__host__ __device__ __forceinline__ uint32_t plane_words(const DevClass& C, int b, int T) {
  const uint32_t jmax = (C.fp_chunks + (uint32_t)T - 1) / (uint32_t)T;
  return (4u * jmax + (uint32_t)b - 1) / (uint32_t)b;
}

// The register-plane class: the first class needing one dense word.
__host__ __device__ __forceinline__ int register_plane_class(const DevIndex& ix, int T) {
  for (uint32_t ci = 0; ci < ix.classes; ++ci)
    if (plane_words(ix.cls[ci], ix.bits, T) == 1) return (int)ci;
  return -1;
}

// Shared-plane layout: base[c] = first dense word of class c in the warp's
// shared planes (kNoPlanes: not counted there); returns the words per lane.
__host__ __device__ __forceinline__ uint32_t shared_plane_layout(const DevIndex& ix, int T,
                                                                uint16_t* base) {
  const int rc = register_plane_class(ix, T);
  uint32_t used = 0;
  for (uint32_t ci = 0; ci < ix.classes; ++ci) {
    uint16_t b0 = kNoPlanes;
    if ((int)ci != rc) {
      const uint32_t w = plane_words(ix.cls[ci], ix.bits, T);
      if (used + w <= kMaxSharedPlaneWords) {
        b0 = (uint16_t)used;
        used += w;
      }
    }
    if (base) base[ci] = b0;
  }
  return used;
}

// Per-warp shared planes: for each of `words` dense words per lane,
// kSharedPlanes count planes, then the valid and multi-member masks; element
// (word, row) of lane l at ((word * (kSharedPlanes + 2) + row) * 32 + l).
struct SharedPlanes {
  uint32_t* base;
  uint32_t words;
  uint32_t steps;
  __device__ __forceinline__ uint32_t* at(uint32_t word, int row, int lane) const {
    return base + ((size_t)word * (kSharedPlanes + 2) + row) * 32 + lane;
  }
};

__device__ __forceinline__ void shared_plane_add(uint32_t* p, uint32_t m) {
  for (int k = 0; k < kSharedPlanes && m; ++k) {
    const uint32_t c = p[k * 32];
    p[k * 32] = c ^ m;
    m &= c;
  }
}

// Masks of dense word d of a lane in class C: positions that are fields of
// the lane, and those whose group has several members.
__device__ __forceinline__ void plane_masks(const DevClass& C, uint32_t d, int b, int tl, int T,
                                            uint32_t& valid, uint32_t& multi) {
  const int lb = log2_bits(b);
  valid = multi = 0;
  for (uint32_t bit = 0; bit < 32; ++bit) {
    const uint32_t q = d * (uint32_t)b + (bit & (uint32_t)(b - 1));
    if ((uint32_t)tl + (q >> 2) * (uint32_t)T >= C.fp_chunks) continue;
    const uint32_t g = dense_group(bit, d, b, lb, tl, T);
    if (g >= C.groups) continue;
    valid |= 1u << bit;
    if (__ldg(C.group_color + g) & kMultiGroup) multi |= 1u << bit;
  }
}

__device__ __forceinline__ void planes_init(LanePlanes& P, const DevIndex& ix, int tl, int T) {
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) P.c[k] = 0;
  P.cls = -1;
  P.valid = P.multi = 0;
  P.steps = 0;
  P.cls = register_plane_class(ix, T);
  if (P.cls >= 0) plane_masks(ix.cls[P.cls], 0, ix.bits, tl, T, P.valid, P.multi);
}

template <class Sink>
__device__ __forceinline__ void planes_flush(LanePlanes& P, const DevIndex& ix, int tl, int T,
                                             const Sink& cnt) {
  P.steps = 0;
  uint32_t any = 0;
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) any |= P.c[k];
  if (!any) return;
  const DevClass& C = ix.cls[P.cls];
  const int b = ix.bits, lb = log2_bits(b);
  while (any) {
    const uint32_t bit = __ffs(any) - 1;
    any &= any - 1;
    uint32_t v = 0;
#pragma unroll
    for (int k = 0; k < kPlanes; ++k) v |= ((P.c[k] >> bit) & 1u) << k;
    cnt.add(__ldg(C.group_color + dense_group(bit, 0, b, lb, tl, T)), v);
  }
#pragma unroll
  for (int k = 0; k < kPlanes; ++k) P.c[k] = 0;
}

// Zeroes a lane's shared planes and fills its masks (class c owns words
// base[c] .. base[c] + plane_words - 1).
__device__ __forceinline__ void shared_planes_init(SharedPlanes& S, const DevIndex& ix,
                                                   const uint16_t* base, int tl, int T, int lane) {
  S.steps = 0;
  for (uint32_t ci = 0; ci < ix.classes; ++ci) {
    if (base[ci] == kNoPlanes) continue;
    const uint32_t w = plane_words(ix.cls[ci], ix.bits, T);
    for (uint32_t d = 0; d < w; ++d) {
      const uint32_t word = base[ci] + d;
      for (int k = 0; k < kSharedPlanes; ++k) *S.at(word, k, lane) = 0;
      uint32_t valid, multi;
      plane_masks(ix.cls[ci], d, ix.bits, tl, T, valid, multi);
      *S.at(word, kSharedPlanes, lane) = valid;
      *S.at(word, kSharedPlanes + 1, lane) = multi;
    }
  }
}

template <class Sink>
__device__ __forceinline__ void shared_planes_flush(SharedPlanes& S, const DevIndex& ix,
                                                    const uint16_t* base, int tl, int T, int lane,
                                                    const Sink& cnt) {
  S.steps = 0;
  const int b = ix.bits, lb = log2_bits(b);
  for (uint32_t ci = 0; ci < ix.classes; ++ci) {
    if (base[ci] == kNoPlanes) continue;
    const DevClass& C = ix.cls[ci];
    const uint32_t w = plane_words(C, b, T);
    for (uint32_t d = 0; d < w; ++d) {
      uint32_t* p = S.at(base[ci] + d, 0, lane);
      uint32_t any = 0;
      for (int k = 0; k < kSharedPlanes; ++k) any |= p[k * 32];
      if (!any) continue;
      while (any) {
        const uint32_t bit = __ffs(any) - 1;
        any &= any - 1;
        uint32_t v = 0;
        for (int k = 0; k < kSharedPlanes; ++k) v |= ((p[k * 32] >> bit) & 1u) << k;
        cnt.add(__ldg(C.group_color + dense_group(bit, d, b, lb, tl, T)), v);
      }
      for (int k = 0; k < kSharedPlanes; ++k) p[k * 32] = 0;
    }
  }
}

// Colours of a hit group given the seed's H row indices (singleton, or
// XOR-decoded members).
template <class OnHit>
__device__ __forceinline__ void group_hit_rows(const DevClass& C, uint32_t group, const uint32_t* rows,
                                               int H, OnHit&& on_hit) {
  const uint32_t gc = __ldg(C.group_color + group);
  if (!(gc & kMultiGroup)) {
    on_hit(gc);
    return;
  }
  const uint32_t* mg = C.multi + 3 * (gc & ~kMultiGroup);
  const uint32_t off = __ldg(mg), n = __ldg(mg + 1), firstm = __ldg(mg + 2);
  uint64_t mask = 0;
  for (int i = 0; i < H; ++i) mask ^= row_bits(C.data + (uint64_t)rows[i] * C.row_stride, off, n);
  while (mask) {
    const uint32_t mb = __ffsll((long long)mask) - 1;
    mask &= mask - 1;
    on_hit(__ldg(C.members + firstm + mb));
  }
}

// XOR of the H rows' 16-byte chunk at `col` for two seeds (row indices in
// shared memory, 4 per seed at a time; all 8 loads issue before any XOR).
__device__ __forceinline__ void gather_xor2(const uint8_t* col, uint32_t stride, const uint32_t* ra,
                                            const uint32_t* rb, int H, bool va_, bool vb_, uint4& aa,
                                            uint4& ab) {
  aa = ab = make_uint4(0, 0, 0, 0);
  for (int i0 = 0; i0 < H; i0 += 4) {
    const uint4 x = *reinterpret_cast<const uint4*>(ra + i0);
    const uint4 y = *reinterpret_cast<const uint4*>(rb + i0);
    const uint32_t xi[4] = {x.x, x.y, x.z, x.w}, yi[4] = {y.x, y.y, y.z, y.w};
    uint4 va[4], vb[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      va[j] = vb[j] = make_uint4(0, 0, 0, 0);
      if (i0 + j < H) {
        if (va_) va[j] = ld_row_chunk(col + (uint64_t)xi[j] * stride);
        if (vb_) vb[j] = ld_row_chunk(col + (uint64_t)yi[j] * stride);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      aa.x ^= va[j].x; aa.y ^= va[j].y; aa.z ^= va[j].z; aa.w ^= va[j].w;
      ab.x ^= vb[j].x; ab.y ^= vb[j].y; ab.z ^= vb[j].z; ab.w ^= vb[j].w;
    }
  }
}

// Rows per seed and class in shared memory: H rounded up to 4.
__device__ __forceinline__ int padded_hashes(int H) { return (H + 3) & ~3; }

// Probes keys[0..n) in rounds of 32 (seed s of a round is keys[r0 + s]).
// kvalid (nullptr: all valid) marks the keys to probe, bit i of word i / 32.
// Every colour a seed hits (filter hit or recovered origin) goes to
// sink.hit(colour, s), except singleton hits counted in the lane's bit planes
// (flushed through sink.add(colour, count)); on_round(r0, m) runs after each
// round with the warp converged.
// PIPE: compile the two-stage chunk pipeline of shared-plane classes (kernel
// variants with the 255-register budget only; it needs about 40 registers).
template <bool PIPE, class Sink, class OnRound>
__device__ void probe_rows(const DevIndex& ix, const uint64_t* keys, uint32_t n,
                           const uint32_t* kvalid, SeedDesc* desc, uint32_t* rows, int T,
                           LanePlanes& P, SharedPlanes& S, const uint16_t* pbase, const Sink& sink,
                           int lane, OnRound&& on_round) {
  const int H = ix.hashes, Hp = padded_hashes(H), b = ix.bits, lb = log2_bits(b);
  const uint32_t ones = field_ones(b), hi = ones << (b - 1);
  const uint32_t classes = ix.classes;
  const uint32_t per_seed = classes * (uint32_t)Hp;
  const int team = lane / T, tl = lane % T, nteams = 32 / T;
  for (uint32_t r0 = 0; r0 < n; r0 += 32) {
    const uint32_t m = min(32u, n - r0);
    const uint32_t round_valid = kvalid ? kvalid[r0 >> 5] : 0xFFFFFFFFu;
    if ((uint32_t)lane < m) {
      SeedDesc d;
      d.live = (round_valid >> lane) & 1u;
      d.rec_list = nullptr;
      d.rec_len = d.rec_single = 0;
      d.pattern = 0;
      if (d.live) {
        const uint64_t key = keys[r0 + lane];
        d.first = mixsplit(key, ix.seed);
        d.step = splitmix64(d.first);
        d.pattern = (uint32_t)fingerprint(key, ix.seed, b) * ones;
        const RecHit r = recovery_lookup(ix.rec, recovery_hash(key, ix.seed));
        d.rec_list = r.list;
        d.rec_len = r.len;
        d.rec_single = r.single;
        uint32_t* my = rows + lane * per_seed;
        for (uint32_t ci = 0; ci < classes; ++ci) {
          const DevClass& C = ix.cls[ci];
          const uint32_t part = C.partitions > 1 ? partition_id(key, ix.seed, C.partitions) : 0;
          const uint64_t count = C.slots / C.seg - (uint64_t)H + 1;
          const uint32_t seg = (uint32_t)C.seg;
          const uint32_t row0 =
              (uint32_t)((uint64_t)part * C.slots + mulhi64(d.first, count) * C.seg);
          uint64_t h = d.first;
          for (int i = 0; i < H; ++i, h += d.step)
            my[ci * Hp + i] =
                row0 + (uint32_t)i * seg + (((uint32_t)h ^ (uint32_t)(h >> 33)) & (seg - 1));
        }
        for (uint32_t i = 0; i < r.len; ++i) sink.hit(r.at(i), (uint32_t)lane);
      }
      desc[lane] = d;
    }
    __syncwarp();
    for (uint32_t s = team; s < m; s += 2 * nteams) {
      const uint32_t s2 = s + nteams;
      const bool two = s2 < m;
      const SeedDesc& da = desc[s];
      const SeedDesc& db = desc[two ? s2 : s];
      const bool va = da.live != 0, vb = two && db.live != 0;
      const uint32_t pa = da.pattern, pb = db.pattern;
      const bool slow_a = da.rec_len != 0, slow_b = vb && db.rec_len != 0;
      for (uint32_t ci = 0; ci < classes; ++ci) {
        const DevClass& C = ix.cls[ci];
        if ((uint32_t)tl >= C.fp_chunks) continue;
        const uint32_t stride = C.row_stride;
        const uint32_t* ra = rows + s * per_seed + ci * Hp;
        const uint32_t* rb = rows + (two ? s2 : s) * per_seed + ci * Hp;
        if ((int)ci == P.cls) {
          // Plane class: this lane's fields fit one dense word.
          uint32_t xa = 0, xb = 0;
          uint32_t q0 = 0;
          for (uint32_t chunk = tl; chunk < C.fp_chunks; chunk += T, q0 += 4) {
            uint4 aa, ab;
            gather_xor2(C.data + chunk * 16u, stride, ra, rb, H, va, vb, aa, ab);
            const uint32_t wa[4] = {aa.x, aa.y, aa.z, aa.w}, wb[4] = {ab.x, ab.y, ab.z, ab.w};
#pragma unroll
            for (int w = 0; w < 4; ++w) {
              const uint32_t sh = (uint32_t)(b - 1) - ((q0 + (uint32_t)w) & (uint32_t)(b - 1));
              xa |= zero_fields_hi(wa[w] ^ pa, hi) >> sh;
              xb |= zero_fields_hi(wb[w] ^ pb, hi) >> sh;
            }
          }
          xa = va ? (xa & P.valid) : 0u;
          xb = vb ? (xb & P.valid) : 0u;
          const uint32_t slowa = slow_a ? xa : (xa & P.multi);
          const uint32_t slowb = slow_b ? xb : (xb & P.multi);
          plane_add(P.c, xa & ~slowa);
          plane_add(P.c, xb & ~slowb);
          for (uint32_t x = slowa; x; x &= x - 1)
            group_hit_rows(C, dense_group(__ffs(x) - 1, 0, b, lb, tl, T), ra, H, [&](uint32_t c) {
              if (da.rec_len && desc_rec_contains(da, c)) return;
              sink.hit(c, s);
            });
          for (uint32_t x = slowb; x; x &= x - 1)
            group_hit_rows(C, dense_group(__ffs(x) - 1, 0, b, lb, tl, T), rb, H, [&](uint32_t c) {
              if (db.rec_len && desc_rec_contains(db, c)) return;
              sink.hit(c, s2);
            });
          continue;
        }
        if (S.words && pbase[ci] != kNoPlanes) {
          // Shared planes: each dense word is committed once the lane's
          // chunks have filled it.
          const uint32_t wbase = pbase[ci];
          uint32_t xa = 0, xb = 0, dcur = 0;
          auto commit = [&](uint32_t d) {
            const uint32_t word = wbase + d;
            const uint32_t valid = *S.at(word, kSharedPlanes, lane);
            const uint32_t multi = *S.at(word, kSharedPlanes + 1, lane);
            const uint32_t ma = va ? (xa & valid) : 0u, mb = vb ? (xb & valid) : 0u;
            const uint32_t slowa = slow_a ? ma : (ma & multi);
            const uint32_t slowb = slow_b ? mb : (mb & multi);
            uint32_t* p = S.at(word, 0, lane);
            shared_plane_add(p, ma & ~slowa);
            shared_plane_add(p, mb & ~slowb);
            for (uint32_t x = slowa; x; x &= x - 1)
              group_hit_rows(C, dense_group(__ffs(x) - 1, d, b, lb, tl, T), ra, H, [&](uint32_t c) {
                if (da.rec_len && desc_rec_contains(da, c)) return;
                sink.hit(c, s);
              });
            for (uint32_t x = slowb; x; x &= x - 1)
              group_hit_rows(C, dense_group(__ffs(x) - 1, d, b, lb, tl, T), rb, H, [&](uint32_t c) {
                if (db.rec_len && desc_rec_contains(db, c)) return;
                sink.hit(c, s2);
              });
          };
          // Match flags of one chunk (XORed rows of both seeds) into the
          // dense words, committing each word when the next one starts.
          auto consume = [&](const uint4& aa, const uint4& ab, uint32_t q0) {
            const uint32_t wa[4] = {aa.x, aa.y, aa.z, aa.w}, wb[4] = {ab.x, ab.y, ab.z, ab.w};
#pragma unroll
            for (int w = 0; w < 4; ++w) {
              const uint32_t q = q0 + (uint32_t)w;
              const uint32_t d = q >> lb;
              if (d != dcur) {
                commit(dcur);
                xa = xb = 0;
                dcur = d;
              }
              const uint32_t sh = (uint32_t)(b - 1) - (q & (uint32_t)(b - 1));
              xa |= zero_fields_hi(wa[w] ^ pa, hi) >> sh;
              xb |= zero_fields_hi(wb[w] ^ pb, hi) >> sh;
            }
          };
          if (PIPE && H <= 4) {
            // Up to 4 rows: two stages of row chunks in registers, the next
            // chunk's loads issued before the current chunk is compared.
            const uint4 ia = *reinterpret_cast<const uint4*>(ra);
            const uint4 ib = *reinterpret_cast<const uint4*>(rb);
            const uint32_t xi[4] = {ia.x, ia.y, ia.z, ia.w}, yi[4] = {ib.x, ib.y, ib.z, ib.w};
            uint4 a0[4], b0[4], a1[4], b1[4];
            auto load = [&](uint4 (&la)[4], uint4 (&lb4)[4], uint32_t chunk) {
              const uint8_t* col = C.data + chunk * 16u;
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                la[j] = lb4[j] = make_uint4(0, 0, 0, 0);
                if (j < H) {
                  if (va) la[j] = ld_row_chunk(col + (uint64_t)xi[j] * stride);
                  if (vb) lb4[j] = ld_row_chunk(col + (uint64_t)yi[j] * stride);
                }
              }
            };
            auto fold = [&](const uint4 (&la)[4], const uint4 (&lb4)[4], uint32_t q0) {
              uint4 aa = la[0], ab = lb4[0];
#pragma unroll
              for (int j = 1; j < 4; ++j) {
                aa.x ^= la[j].x; aa.y ^= la[j].y; aa.z ^= la[j].z; aa.w ^= la[j].w;
                ab.x ^= lb4[j].x; ab.y ^= lb4[j].y; ab.z ^= lb4[j].z; ab.w ^= lb4[j].w;
              }
              consume(aa, ab, q0);
            };
            uint32_t chunk = tl, q0 = 0;
            if (chunk < C.fp_chunks) load(a0, b0, chunk);
            while (chunk < C.fp_chunks) {
              const uint32_t c1 = chunk + T;
              if (c1 < C.fp_chunks) load(a1, b1, c1);
              fold(a0, b0, q0);
              if (c1 >= C.fp_chunks) break;
              const uint32_t c2 = c1 + T;
              if (c2 < C.fp_chunks) load(a0, b0, c2);
              fold(a1, b1, q0 + 4);
              chunk = c2;
              q0 += 8;
            }
          } else {
            uint32_t q0 = 0;
            for (uint32_t chunk = tl; chunk < C.fp_chunks; chunk += T, q0 += 4) {
              uint4 aa, ab;
              gather_xor2(C.data + chunk * 16u, stride, ra, rb, H, va, vb, aa, ab);
              consume(aa, ab, q0);
            }
          }
          commit(dcur);
          continue;
        }
        for (uint32_t chunk = tl; chunk < C.fp_chunks; chunk += T) {
          uint4 aa, ab;
          gather_xor2(C.data + chunk * 16u, stride, ra, rb, H, va, vb, aa, ab);
          if (va)
            chunk_hits(aa, chunk, C.groups, b, ones, pa, [&](uint32_t g) {
              group_hit_rows(C, g, ra, H, [&](uint32_t c) {
                if (da.rec_len && desc_rec_contains(da, c)) return;
                sink.hit(c, s);
              });
            });
          if (vb)
            chunk_hits(ab, chunk, C.groups, b, ones, pb, [&](uint32_t g) {
              group_hit_rows(C, g, rb, H, [&](uint32_t c) {
                if (db.rec_len && desc_rec_contains(db, c)) return;
                sink.hit(c, s2);
              });
            });
        }
      }
      if (P.cls >= 0 && ++P.steps == kPlaneFlush) planes_flush(P, ix, tl, T, sink);
      if (S.words && ++S.steps == kSharedFlush) shared_planes_flush(S, ix, pbase, tl, T, lane, sink);
    }
    __syncwarp();
    on_round(r0, m);
  }
}

// Colour counting sink of the ordinary modes.
struct CountSink {
  Counters cnt;
  __device__ __forceinline__ void hit(uint32_t c, uint32_t) const { cnt.add(c); }
  __device__ __forceinline__ void add(uint32_t c, uint32_t n) const { cnt.add(c, n); }
};

// ---- findere ----------------------------------------------------------------
// Scores::score, findere branch (query_stream.rs:670-689; findere.rs:74-105): a
// colour scores a k-window when all z + 1 s-mers of the window hit it. A warp
// probes the s-mers of a tile's windows w0 .. w0 + nw - 1 (positions 0 .. nw +
// z - 1, s-mer i starting at base w0 + i) in rounds of 32; each hit sets bit s
// of the colour's round mask (an OR, so a colour hit by the filter and by
// recovery counts once, the union of lookup_selected). After each round a
// sweep counts, per colour, the positions that end a run of at least z + 1
// consecutive hits, carrying the run length (saturated at z) into the next
// round. Windows are the features: total = valid k-windows.
struct FindereSink {
  uint32_t* mask;     // colours round masks of this warp
  uint32_t* touched;  // shared state: bit c set at colour c's first hit of a round (else null)
  __device__ __forceinline__ void hit(uint32_t c, uint32_t s) const {
    const uint32_t old = atomicOr(mask + c, 1u << s);
    if (touched && !old) atomicOr(touched + (c >> 5), 1u << (c & 31));
  }
  __device__ __forceinline__ void add(uint32_t, uint32_t) const {}
};

// One colour's round: positions ending a run of at least z + 1 hits (m: the
// round's hit mask, r: the run carried in), and the run carried out.
__device__ __forceinline__ uint32_t findere_round(uint32_t m, uint32_t r, int z, uint32_t len,
                                                  uint32_t* carried) {
  uint32_t y = m;
  for (int t = 1; t <= z && y; ++t) y &= t < 32 ? (m << t) : 0u;
  uint32_t n = __popc(y);
  const uint32_t lead = m == 0xFFFFFFFFu ? 32u : (uint32_t)(__ffs(~m) - 1);
  const int lo = max(0, z - (int)r), hi2 = min(z, (int)lead);
  if (hi2 > lo) n += (uint32_t)(hi2 - lo);
  if (lead >= len) {
    *carried = min((uint32_t)z, r + len);
  } else {
    const uint32_t mm = len == 32 ? m : (m << (32 - len));
    *carried = min((uint32_t)z, (uint32_t)__clz(~mm));
  }
  return n;
}

// Sweeps the round masks of positions r0 .. r0 + len - 1 (bit i = r0 + i):
// counts the positions whose run of consecutive hits is at least z + 1 long
// and clears the masks; run[c] carries the run length at the round's end (0
// after the tile's last round). SHARED: the warp's masks and run lengths are
// in shared memory (the caller synchronised the warp after the hits).
template <bool SHARED>
__device__ __forceinline__ void findere_sweep(uint32_t* mask, uint32_t* run, uint32_t colors, int z,
                                              uint32_t len, bool last, const Counters& cnt,
                                              int lane) {
  if constexpr (SHARED) {
    // Only the colours hit this round (touched) or carrying a run (runbits)
    // can count or change: lane l takes words l, l + 32, ... of the bitmaps.
    uint32_t* touched = run + colors;
    uint32_t* runbits = touched + (colors + 31) / 32;
    for (uint32_t wd = (uint32_t)lane; wd < (colors + 31) / 32; wd += 32) {
      uint32_t bits = touched[wd] | runbits[wd], carry = 0;
      touched[wd] = 0;
      while (bits) {
        const uint32_t bit = __ffs(bits) - 1;
        bits &= bits - 1;
        const uint32_t c = wd * 32 + bit;
        const uint32_t m = mask[c], r = run[c];
        uint32_t nr = 0, n = 0;
        if (m) {
          mask[c] = 0u;
          n = findere_round(m, r, z, len, &nr);
        }
        if (last) nr = 0;
        run[c] = nr;
        if (nr) carry |= 1u << bit;
        if (n) cnt.add(c, n);
      }
      runbits[wd] = carry;
    }
  } else {
    // Global masks are set by L2 atomics of every lane: read them past L1 and
    // clear them atomically. run[c] belongs to lane c % 32.
    for (uint32_t c = (uint32_t)lane; c < colors; c += 32) {
      uint32_t m = __ldcg(mask + c);
      const uint32_t r = run[c];
      if (!m) {
        if (r) run[c] = 0;
        continue;
      }
      m = atomicExch(mask + c, 0u);
      uint32_t nr;
      const uint32_t n = findere_round(m, r, z, len, &nr);
      run[c] = last ? 0u : nr;
      if (n) cnt.add(c, n);
    }
  }
}

// ---- asynchronous staged gather (cp.async.bulk + mbarrier) ------------------
// One lane arms a stage's mbarrier with the byte count, all lanes issue 1-D
// bulk copies of fingerprint-plane row slices (16-byte aligned, multiples of
// 16 bytes) into a per-warp shared-memory ring, and the warp XORs and compares
// the landed slices while the next stages are in flight. Waits are bounded:
// on expiry the warp raises bit 0 of *err and stops probing.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the completion of the phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 22); ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
// Waits until at most n of this thread's committed groups are pending.
__device__ __forceinline__ void cp_async_wait(uint32_t n) {
  switch (n) {
    case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
    case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
    case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
    case 3: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
    case 4: asm volatile("cp.async.wait_group 4;" ::: "memory"); break;
    case 5: asm volatile("cp.async.wait_group 5;" ::: "memory"); break;
    case 6: asm volatile("cp.async.wait_group 6;" ::: "memory"); break;
    default: asm volatile("cp.async.wait_group 7;" ::: "memory"); break;
  }
}

struct StageRing {
  uint8_t* mem;       // stages * stage_bytes
  uint64_t* bars;     // stages mbarriers
  uint32_t stage_bytes, stages;
  uint32_t phases;    // parity bit per stage
  uint32_t pending;   // stage bits with copies in flight
  bool bulk;          // true: one bulk copy per row slice; false: 16-byte cp.async per lane
};

// Probes keys[0..n) with staged bulk gathers. desc/row0s hold 64 seeds.
__device__ bool probe_batch_async(const DevIndex& ix, const uint64_t* keys, uint32_t n,
                                  SeedDesc* desc, uint64_t* row0s, StageRing& ring,
                                  const Counters& cnt, int lane, uint32_t* err) {
  const int H = ix.hashes, b = ix.bits;
  const uint32_t ones = field_ones(b);
  const uint32_t classes = ix.classes;
  for (uint32_t r0 = 0; r0 < n; r0 += 64) {
    const uint32_t m = min(64u, n - r0);
    for (uint32_t q = lane; q < m; q += 32) {
      const uint64_t key = keys[r0 + q];
      SeedDesc d;
      d.first = mixsplit(key, ix.seed);
      d.step = splitmix64(d.first);
      d.pattern = (uint32_t)fingerprint(key, ix.seed, b) * ones;
      RecHit r = recovery_lookup(ix.rec, recovery_hash(key, ix.seed));
      d.rec_list = r.list;
      d.rec_len = r.len;
      d.rec_single = r.single;
      d.live = 1;
      desc[q] = d;
      for (uint32_t ci = 0; ci < classes; ++ci) {
        const DevClass& C = ix.cls[ci];
        const uint32_t part = C.partitions > 1 ? partition_id(key, ix.seed, C.partitions) : 0;
        const uint64_t count = C.slots / C.seg - (uint64_t)H + 1;
        const uint64_t base = mulhi64(d.first, count) * C.seg;
        row0s[q * classes + ci] = ((uint64_t)part * C.slots + base) * C.row_stride;
      }
      for (uint32_t i = 0; i < r.len; ++i) cnt.add(r.at(i));
    }
    __syncwarp();
    for (uint32_t ci = 0; ci < classes; ++ci) {
      const DevClass& C = ix.cls[ci];
      const uint32_t rb = C.fp_chunks * 16u;                      // bytes gathered per row
      uint32_t cw = (ring.stage_bytes / (uint32_t)H) & ~15u;      // column tile width
      if (cw > rb) cw = rb;
      const uint32_t tiles = (rb + cw - 1) / cw;                  // column tiles per seed
      const uint32_t items = m * tiles;
      const uint32_t per_stage = ring.stage_bytes / ((uint32_t)H * cw);
      const uint32_t batches = (items + per_stage - 1) / per_stage;
      const uint32_t cpi = cw / 16;                               // chunks per item slot
      auto issue = [&](uint32_t bi) {
        const uint32_t st = bi % ring.stages;
        const uint32_t i0 = bi * per_stage, ni = min(per_stage, items - i0);
        uint8_t* smem = ring.mem + (size_t)st * ring.stage_bytes;
        if (!ring.bulk) {
          // Per-lane 16-byte copies: triple t = (item, row, chunk).
          const uint32_t triples = ni * (uint32_t)H * cpi;
          for (uint32_t t = lane; t < triples; t += 32) {
            const uint32_t c = t % cpi, ri = t / cpi, i = ri % (uint32_t)H, li = ri / (uint32_t)H;
            const uint32_t it = i0 + li, sd = it / tiles, col0 = (it % tiles) * cw;
            if (col0 + c * 16 >= rb) continue;
            const SeedDesc& d = desc[sd];
            const uint64_t h = d.first + (uint64_t)i * d.step;
            cp_async16(smem + ((size_t)li * H + i) * cw + c * 16,
                       C.data + row_offset(row0s[sd * classes + ci], h, (int)i, C.seg,
                                           C.row_stride) + col0 + c * 16);
          }
          cp_async_commit();
          return;
        }
        // Order this lane's earlier generic reads of the stage before the
        // async-proxy writes that will overwrite it.
        fence_proxy_async_smem();
        if (lane == 0) {
          uint32_t bytes = 0;
          for (uint32_t it = i0; it < i0 + ni; ++it) {
            uint32_t col0 = (it % tiles) * cw;
            bytes += (uint32_t)H * min(cw, rb - col0);
          }
          mbar_arrive_expect(ring.bars + st, bytes);
        }
        __syncwarp();
        for (uint32_t li = lane; li < ni; li += 32) {
          const uint32_t it = i0 + li, s = it / tiles, col0 = (it % tiles) * cw;
          const uint32_t w = min(cw, rb - col0);
          const SeedDesc& d = desc[s];
          const uint64_t row0 = row0s[s * classes + ci];
          uint64_t h = d.first;
          for (int i = 0; i < H; ++i, h += d.step)
            bulk_copy_g2s(smem + ((size_t)li * H + i) * cw,
                          C.data + row_offset(row0, h, i, C.seg, C.row_stride) + col0, w,
                          ring.bars + st);
        }
        ring.pending |= 1u << st;
      };
      const uint32_t prologue = min(ring.stages, batches);
      for (uint32_t bi = 0; bi < prologue; ++bi) issue(bi);
      for (uint32_t bi = 0; bi < batches; ++bi) {
        const uint32_t st = bi % ring.stages;
        if (ring.bulk) {
          const bool ok = mbar_wait(ring.bars + st, (ring.phases >> st) & 1u);
          if (__any_sync(0xFFFFFFFFu, !ok)) {
            if (lane == 0) atomicOr(err, 1u);
            return false;
          }
          ring.phases ^= 1u << st;
          ring.pending &= ~(1u << st);
        } else {
          // Batches bi .. min(bi + stages, batches) - 1 are committed; keep
          // all but the oldest in flight.
          cp_async_wait(min(ring.stages, batches - bi) - 1);
          __syncwarp();
        }
        const uint32_t i0 = bi * per_stage, ni = min(per_stage, items - i0);
        const uint8_t* smem = ring.mem + (size_t)st * ring.stage_bytes;
        for (uint32_t pair = lane; pair < ni * cpi; pair += 32) {
          const uint32_t li = pair / cpi, c = pair % cpi;
          const uint32_t it = i0 + li, s = it / tiles, col0 = (it % tiles) * cw;
          if (col0 + c * 16 >= rb) continue;
          uint4 acc = make_uint4(0, 0, 0, 0);
          for (int i = 0; i < H; ++i) {
            const uint4 v = *reinterpret_cast<const uint4*>(smem + ((size_t)li * H + i) * cw + c * 16);
            acc.x ^= v.x; acc.y ^= v.y; acc.z ^= v.z; acc.w ^= v.w;
          }
          const SeedDesc& d = desc[s];
          const uint64_t row0 = row0s[s * classes + ci];
          chunk_hits(acc, col0 / 16 + c, C.groups, b, ones, d.pattern, [&](uint32_t g) {
            group_hit(C, g, d, row0, H, [&](uint32_t col) {
              if (d.rec_len && desc_rec_contains(d, col)) return;
              cnt.add(col);
            });
          });
        }
        __syncwarp();
        if (bi + ring.stages < batches) issue(bi + ring.stages);
      }
    }
    __syncwarp();
  }
  return true;
}

// Bounded drain of stages still in flight (after an error).
__device__ __forceinline__ void ring_drain(StageRing& ring) {
  for (uint32_t st = 0; st < ring.stages; ++st)
    if (ring.pending & (1u << st)) {
      mbar_wait(ring.bars + st, (ring.phases >> st) & 1u);
      ring.phases ^= 1u << st;
    }
  ring.pending = 0;
}

}  // namespace zx
