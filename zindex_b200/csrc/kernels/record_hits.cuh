// Per-record hit selection for the per-record report with a threshold
// (RecordScores::write_record, src/power_merge/storage.rs:3109-3146): colour c
// of record r is reported when its count is non-zero, the record's total is
// non-zero and count / total >= min_ratio. The division is the IEEE double
// division rounded to nearest, as on the host, so the selection is exact.
//
// counts: records x colours (row-major), totals: records. One warp per record
// walks its row in 32-colour steps; a ballot gives each hit its place, so the
// hits of a record come out in colour order.
#pragma once
#include <cstdint>

namespace zx {

__device__ __forceinline__ bool record_hit(uint64_t count, uint64_t total, double min_ratio) {
  return count != 0 && total != 0 && __ddiv_rn((double)count, (double)total) >= min_ratio;
}

// hits[r] = number of reported colours of record r (r < records); hits[records] = 0.
__global__ void count_record_hits_kernel(const uint64_t* __restrict__ counts,
                                         const unsigned long long* __restrict__ totals,
                                         uint64_t records, uint32_t colors, double min_ratio,
                                         uint64_t* __restrict__ hits) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t first = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (first == 0 && lane == 0) hits[records] = 0;
  for (uint64_t r = first; r < records; r += warps) {
    const uint64_t t = totals[r];
    const uint64_t* row = counts + r * colors;
    uint32_t n = 0;
    for (uint32_t c0 = 0; c0 < colors; c0 += 32) {
      const uint32_t c = c0 + lane;
      const bool h = c < colors && record_hit(row[c], t, min_ratio);
      n += __popc(__ballot_sync(0xffffffffu, h));
    }
    if (lane == 0) hits[r] = n;
  }
}

// Writes the hits of record r at first[r] .. first[r+1]-1 (first: exclusive
// scan of the counts above), colour ids and counts in colour order.
__global__ void write_record_hits_kernel(const uint64_t* __restrict__ counts,
                                         const unsigned long long* __restrict__ totals,
                                         uint64_t records, uint32_t colors, double min_ratio,
                                         const uint64_t* __restrict__ first,
                                         uint32_t* __restrict__ hit_colors,
                                         uint64_t* __restrict__ hit_counts) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < records;
       r += warps) {
    const uint64_t t = totals[r];
    const uint64_t* row = counts + r * colors;
    uint64_t at = first[r];
    for (uint32_t c0 = 0; c0 < colors; c0 += 32) {
      const uint32_t c = c0 + lane;
      const uint64_t v = c < colors ? row[c] : 0;
      const bool h = c < colors && record_hit(v, t, min_ratio);
      const uint32_t m = __ballot_sync(0xffffffffu, h);
      if (h) {
        const uint64_t i = at + __popc(m & ((1u << lane) - 1));
        hit_colors[i] = c;
        hit_counts[i] = v;
      }
      at += __popc(m);
    }
  }
}

}  // namespace zx
