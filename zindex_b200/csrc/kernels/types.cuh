// Plain parameter structs shared by the host runtime and the query kernels.
#pragma once
#include <stdint.h>

#include "../zx_hash.h"
#include "device_index.cuh"

namespace zx {

// Bits of a query's device error word.
constexpr uint32_t kErrWait = 1u;     // a bounded wait expired (staged gather)
constexpr uint32_t kErrOffsets = 2u;  // a record's offsets decrease, leave the bases, or span 2^31

struct SeedParams {
  int mode;        // 0 kmers, 1 minimizers, 2 modimizers, 3 findere
  int k;           // window span (k-mer length, minimizer window, findere k)
  int m;           // minimizer length
  int klen;        // length of the hashed k-mer: k, or k - z for findere s-mers
  uint64_t seed;
  uint64_t sampling;
  OcmParams ocm;
  LongKmerConsts lk;
  int spaced;       // 1: keys are mapped through `pattern` (k-mers and minimizers)
  SpacedSeed pattern;
  // Randstrobemers over k-mers (strobe_max 0 = off): each window is linked to
  // a partner window strobe_min..strobe_max downstream in the same run.
  uint32_t strobe_min, strobe_max;
};

struct Tile {
  uint32_t record;  // record index in the batch
  uint32_t w0;      // first window start (record coordinates)
  uint32_t nw;      // windows in this tile
  uint32_t task;    // findere: first window of the enclosing 16,384-window task
};

struct QueryLaunch {
  int team;           // lanes per seed (1..32, power of two), register gather
  int warps;          // warps per block
  int blocks;         // grid size
  int smem_counters;  // 1: per-block shared counters; 0: global atomics
  int stage_bytes;    // > 0: staged gather with this stage size per warp
  int stages;         // stages in each warp's ring (staged gather)
  int bulk;           // staged gather: 1 = bulk copy per row slice, 0 = 16-byte cp.async
  int min_blocks;     // register budget: 1 (255 registers; row-index form with the chunk
                      // pipeline), 2 or 3 resident 256-thread blocks per SM
  int planes;         // register gather: 1 = row indices + bit-plane colour counters, 0 = descriptors
  int cut;            // host batches: pipelined chunks (copy of chunk i+1 overlaps chunk i), 1..64
  int split;          // minimizers: 1 = seeds extracted by their own kernel into per-tile slots,
                      // then probed by a kernel without the extraction scratch (more warps per SM)
  int wide;           // 1 = wide-row form: seeds extracted into a dense list, probed by blocks
                      // whose threads own fixed 16-byte chunks of every row (wide_probe.cuh)
  int order;          // wide-row form: 1 = each round's seeds sorted by their first hash, so
                      // consecutive seeds read neighbouring rows of every class (2: and the
                      // blocks take interleaved seeds)
};

}  // namespace zx
