// Device-resident index layout (HBM) shared by the query kernels.
//
// Banks: one allocation per source class holding its P hash partitions back
// to back; partition p, slot s starts at data + (p * slots + s) * row_stride.
// row_stride is the reference row (ceil(row_bits / 8) bytes, fingerprint plane
// first, membership plane after it, storage.rs:1721-1754) padded to a multiple
// of 16 bytes, so every row begins on a 128-bit boundary and the fingerprint
// plane is gathered with 16-byte vector loads.
//
// Recovery map: open-addressed directory of 64-bit entries (hash << 32 |
// value) with the first probe slot taken from the high hash bits, a load
// factor of at most 1/2, inline origins below 2^31 and (start, length)
// postings otherwise (the semantics of OriginMap::get, abandoned.rs:180-205).
#pragma once
#include <stdint.h>

namespace zx {

constexpr uint32_t kRecEmpty = 0xFFFFFFFFu;
constexpr uint32_t kRecMultiple = 0x80000000u;
constexpr uint32_t kMultiGroup = 0x80000000u;
constexpr int kMaxClasses = 64;

struct DevClass {
  const uint8_t* data;         // partitions * slots * row_stride bytes
  const uint32_t* group_color;  // G entries: colour id, or kMultiGroup | multi index
  const uint32_t* multi;        // per multi group: {membership bit offset, member count, first}
  const uint32_t* members;      // member colour ids of multi groups
  uint64_t slots;               // cells per partition bank
  uint64_t seg;                 // segment length
  uint32_t partitions;          // power of two
  uint32_t groups;              // G
  uint32_t row_stride;          // bytes, multiple of 16
  uint32_t fp_chunks;           // 16-byte chunks covering the fingerprint plane
};

struct DevRecovery {
  const uint64_t* dir;       // capacity entries
  const uint2* ranges;       // {start, length} postings
  const uint32_t* origins;   // posting storage
  uint32_t bits;             // log2(capacity); 0 when the map is empty
};

struct __align__(16) DevIndex {
  DevClass cls[kMaxClasses];
  DevRecovery rec;
  uint64_t seed;
  uint32_t classes;
  uint32_t colors;
  int hashes;
  int bits;  // fingerprint bits
};

}  // namespace zx
