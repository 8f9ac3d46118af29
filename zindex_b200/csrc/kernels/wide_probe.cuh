// Wide-row probe: the whole block is one team (K5 for rows of thousands of
// colours).
//
// Same arithmetic as probe_rows (Index::lookup_selected, src/power_merge/
// storage.rs:2761-2925: per class the partition bank, the H cells of
// PositionHash, the XOR of the H fingerprint-plane rows, a compare of every
// b-bit field with fingerprint(key), membership decode of multi-member groups;
// recovered origins counted once per seed, 2769-2787 and 2916-2924), laid out
// for indexes whose rows span many 16-byte chunks (2,048 colours at b = 16:
// 4 KiB per cell; 16,384 colours at b = 4: 8 KiB):
//
// * Seeds come from a dense key list (extract_dense_kernel appends every
//   tile's seeds; aggregate counts do not depend on their order).
// * A block takes 256 seeds at a time. Thread i computes seed i's fingerprint
//   pattern and the row index of each of its H cells per class into shared
//   memory, then the block walks the seeds: thread t owns the 16-byte
//   chunks t, t + T, ... of the concatenated fingerprint planes of all
//   classes, so a warp reads 512 contiguous bytes of every row and each
//   thread's field-match flags always land in the same few dense words. The
//   flags are counted in bit planes held in registers (vertical binary
//   counters, 63 per field) and added to the colour counters every 63 seeds.
// * A recovered origin c is counted when the filter did not hit it: the
//   seed's owner thread re-reads c's own field in the seed's H cells (and its
//   membership bit for a multi-member group). Filter hits plus recovered
//   origins the filter missed is the union lookup_selected counts, and no
//   filter hit has to be checked against the recovery list.
// * Hits on multi-member groups take the per-hit membership decode.
//
// Needs b >= 4 (one dense word per chunk) and at most J chunks per thread.
#pragma once
#include <stdint.h>

#include "query_kernels.cuh"

namespace zx {

constexpr int kWideSeeds = 256;      // seeds per descriptor round of a block
constexpr int kWidePlanes = 6;       // register planes: counts up to 63 per field
constexpr uint32_t kWideFlush = 63;  // seeds between plane flushes
// Ordered rounds: a counting sort of a round's dense key list by the top
// kOrderBits bits of each key's first hash (every class's row index grows
// with the first hash). Keys keep no particular order within a bucket.
constexpr int kOrderBits = 16;
constexpr uint32_t kOrderBuckets = 1u << kOrderBits;

// Colour location for recovered-origin point probes: cls_member = class |
// member index << 8 (member index within a multi-member group, 0 for
// singletons; ~0 for a colour in no bank), group = the colour's group.
struct ColorLoc {
  uint32_t cls_member;
  uint32_t group;
};

// Shared memory of the dense extraction per warp: one tile's keys (and the
// staging of long k-mer hashes) and, for minimizers, the open-closed
// minimizer scratch; no probe descriptors. The block adds the 256-entry inner
// hash table.
struct DenseSmem {
  static __host__ __device__ size_t warp_bytes(int mode, int k) {
    size_t b = FusedSmem::key_bytes(mode, k, false);
    if (mode == 1) b += 2 * FusedSmem::ocm_entries(k) * sizeof(Rank16) + (kTileWindows + 1) * 4 + 16;
    return (b + 15) / 16 * 16;
  }
  static __host__ __device__ size_t total(int mode, int k, int warps) {
    return 256 * 8 + (size_t)warps * warp_bytes(mode, k);
  }
};

// Largest s < n with first[s] <= x (first[] non-decreasing, first[0] <= x):
// the segment holding tile or round x, empty segments sharing its start
// coming before it.
__device__ __forceinline__ uint32_t segment_of(const uint32_t* __restrict__ first, uint32_t n,
                                               uint32_t x) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(first + mid) <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Per-round tables of a wide-row query.
// Segmented (several requests in one launch): per extraction round, segment
// s's keys sit at out[(max(seg_tiles[s], tile_lo) - tile_lo) * kTileWindows
// ...], their number in cursor[s]; the probe's rounds of 256 seeds never
// straddle segments (round_first[s] = first round of segment s). nseg = 0:
// one unsegmented list, one cursor.
struct WideRound {
  const uint32_t* seg_tiles = nullptr;    // first tile of each segment (nseg + 1)
  unsigned long long* cursor = nullptr;   // keys of each segment in this round
  const uint32_t* round_first = nullptr;  // first probe round of each segment (nseg + 1)
  unsigned long long* totals = nullptr;   // seeds of each segment
  uint32_t nseg = 0;
  uint32_t tile_lo = 0;                   // first tile of the extraction round
  // Unsegmented: 1 = blocks take interleaved seeds (see the probe loop).
  uint32_t interleave = 0;
  // Segmented per-record reports: colours reported when count / total >=
  // min_ratio (> 0 turns on threshold pruning); tile_hi ends the round.
  double min_ratio = 0.0;
  uint32_t tile_hi = 0;
};

// Smallest count c with c / total >= ratio in IEEE double division: the
// report's own test (minimum_matches, src/power_merge/record_query.rs:12-26).
__device__ __forceinline__ uint64_t minimum_matches(uint64_t total, double ratio) {
  if (total == 0 || ratio == 0.0) return 0;
  uint64_t lo = 0, hi = total;
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (__ddiv_rn((double)mid, (double)total) >= ratio) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Threshold pruning: a chunk's fields are checked every kPruneStep seeds.
constexpr uint32_t kPruneStep = 16;

__device__ __forceinline__ uint64_t wide_seg_base(const WideRound& sg, uint32_t s) {
  const uint32_t t = __ldg(sg.seg_tiles + s);
  return (uint64_t)(t > sg.tile_lo ? t - sg.tile_lo : 0u) * kTileWindows;
}

// round_first[] of a segmented round: exclusive scan of each segment's
// ceil(keys / 256) probe rounds (one block).
__global__ void wide_rounds_kernel(const unsigned long long* __restrict__ cursor, uint32_t nseg,
                                   uint32_t* __restrict__ round_first) {
  __shared__ uint32_t part[1024];
  const uint32_t T = blockDim.x, tid = threadIdx.x;
  const uint32_t per = (nseg + T - 1) / T;
  const uint32_t lo = min(nseg, tid * per), hi = min(nseg, lo + per);
  uint32_t sum = 0;
  for (uint32_t s = lo; s < hi; ++s) sum += (uint32_t)((cursor[s] + kWideSeeds - 1) / kWideSeeds);
  part[tid] = sum;
  __syncthreads();
  for (uint32_t off = 1; off < T; off <<= 1) {
    const uint32_t v = tid >= off ? part[tid - off] : 0u;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  uint32_t run = tid ? part[tid - 1] : 0u;
  for (uint32_t s = lo; s < hi; ++s) {
    round_first[s] = run;
    run += (uint32_t)((cursor[s] + kWideSeeds - 1) / kWideSeeds);
  }
  if (tid == T - 1) round_first[nseg] = part[T - 1];
}

// Appends the seeds of tiles [tile_lo, tile_hi) (tile_hi 0 = to the end) to
// out[], one atomic cursor bump per warp and tile. out holds at least
// (tile_hi - tile_lo) * kTileWindows keys. Segmented (sg.nseg > 0): each
// tile's seeds go to its segment's part of out[] and cursor.
template <int MODE>
__global__ void extract_dense_kernel(BatchView bv, SeedParams sp, uint64_t* __restrict__ out,
                                     unsigned long long* __restrict__ cursor, int warps_per_block,
                                     WideRound sg) {
  extern __shared__ __align__(16) uint8_t smem[];
  uint64_t* inner = reinterpret_cast<uint64_t*>(smem);
  uint8_t* p = smem + 256 * 8;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t* wbase = p + (size_t)warp * DenseSmem::warp_bytes(MODE, sp.k);
  uint64_t* keys = reinterpret_cast<uint64_t*>(wbase);
  uint8_t* ocm = wbase + FusedSmem::key_bytes(MODE, sp.k, false);
  build_inner_table(sp, inner);
  __syncthreads();
  uint32_t ntiles = *bv.ntiles;
  if (bv.tile_hi && bv.tile_hi < ntiles) ntiles = bv.tile_hi;
  const uint32_t warps_total = gridDim.x * warps_per_block;
  for (uint32_t t = bv.tile_lo + blockIdx.x * warps_per_block + warp; t < ntiles;
       t += warps_total) {
    const uint32_t n = extract_tile<MODE>(bv, sp, bv.tiles[t], keys, ocm, inner, lane);
    __syncwarp();
    unsigned long long at = 0;
    uint64_t* dst = out;
    unsigned long long* cur = cursor;
    if (sg.nseg) {
      const uint32_t seg = segment_of(sg.seg_tiles, sg.nseg, t);
      dst = out + wide_seg_base(sg, seg);
      cur = sg.cursor + seg;
    }
    if (lane == 0 && n) at = atomicAdd(cur, (unsigned long long)n);
    at = __shfl_sync(0xFFFFFFFFu, at, 0);
    for (uint32_t i = lane; i < n; i += 32) dst[at + i] = keys[i];
    __syncwarp();
  }
}

__device__ __forceinline__ uint32_t order_bucket(uint64_t key, uint64_t seed) {
  return (uint32_t)(mixsplit(key, seed) >> (64 - kOrderBits));
}

// Ordered rounds, step 1: keys per bucket (hist zeroed before).
__global__ void order_count_kernel(const uint64_t* __restrict__ keys,
                                   const unsigned long long* __restrict__ nkeys, uint64_t seed,
                                   uint32_t* __restrict__ hist) {
  const uint64_t n = *nkeys;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(hist + order_bucket(keys[i], seed), 1u);
}

// Step 2 (one block of 1,024 threads): the buckets' first places, in place.
__global__ void order_scan_kernel(uint32_t* __restrict__ hist) {
  __shared__ uint32_t part[1024];
  const uint32_t T = blockDim.x, tid = threadIdx.x, per = kOrderBuckets / T;
  uint32_t sum = 0;
  for (uint32_t j = 0; j < per; ++j) sum += hist[tid * per + j];
  part[tid] = sum;
  __syncthreads();
  for (uint32_t off = 1; off < T; off <<= 1) {
    const uint32_t v = tid >= off ? part[tid - off] : 0u;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  uint32_t run = tid ? part[tid - 1] : 0u;
  for (uint32_t j = 0; j < per; ++j) {
    const uint32_t c = hist[tid * per + j];
    hist[tid * per + j] = run;
    run += c;
  }
}

// Step 3: every key to its bucket's next place in out[].
__global__ void order_scatter_kernel(const uint64_t* __restrict__ keys,
                                     const unsigned long long* __restrict__ nkeys, uint64_t seed,
                                     uint32_t* __restrict__ next, uint64_t* __restrict__ out) {
  const uint64_t n = *nkeys;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    out[atomicAdd(next + order_bucket(k, seed), 1u)] = k;
  }
}

// Shared memory of the wide probe: DevIndex copy, colour counters (optional),
// then per seed of a round its fingerprint pattern and row indices (classes x
// H rounded up to 4).
struct WideSmem {
  static __host__ __device__ size_t rows_per_seed(uint32_t classes, int hashes) {
    return (size_t)classes * (size_t)((hashes + 3) & ~3);
  }
  static __host__ __device__ size_t total(uint32_t colors, uint32_t classes, int hashes,
                                          int smem_counters) {
    return FusedSmem::ix_bytes + FusedSmem::counter_bytes(colors, smem_counters) +
           (size_t)kWideSeeds * 4 + (size_t)kWideSeeds * rows_per_seed(classes, hashes) * 4;
  }
};

struct WideCounters {
  uint32_t* smem;
  uint64_t* gmem;  // the current segment's counters when smem is null
  __device__ __forceinline__ void add(uint32_t c, uint32_t n) const {
    if (smem) atomicAdd(smem + c, n);
    else atomicAdd(reinterpret_cast<unsigned long long*>(gmem + c), (unsigned long long)n);
  }
};

// Group of dense bit p of a chunk (chunk-local group 0 = first field): word
// p % b of the chunk, field p / b of that word.
__device__ __forceinline__ uint32_t wide_group(uint32_t g0, uint32_t p, int b, int lb) {
  return g0 + (p & (uint32_t)(b - 1)) * (32u >> lb) + (p >> lb);
}

// J: chunks per thread; S: seeds per step; HQ: rows loaded per seed and chunk
// before the XOR (J * S * HQ 16-byte loads in flight per thread); MAXT: the
// largest block (256, or 288 so that rows a few partial chunks over 256 or
// 512 keep one or two chunks per thread).
template <int J, int S, int HQ, int MINB, int MAXT = 256>
__global__ void __launch_bounds__(MAXT, MINB)
    wide_probe_kernel(const DevIndex* __restrict__ gix, const ColorLoc* __restrict__ color_loc,
                      const uint64_t* __restrict__ keys,
                      const unsigned long long* __restrict__ nkeys, int smem_counters,
                      uint32_t team_threads, uint32_t* __restrict__ partial,
                      uint64_t* __restrict__ counts, unsigned long long* __restrict__ total,
                      WideRound sg) {
  extern __shared__ __align__(16) uint8_t smem[];
  DevIndex* six = reinterpret_cast<DevIndex*>(smem);
  uint8_t* p = smem + FusedSmem::ix_bytes;
  const uint32_t colors = gix->colors, classes = gix->classes;
  uint32_t* scount = nullptr;
  if (smem_counters) {
    scount = reinterpret_cast<uint32_t*>(p);
    p += FusedSmem::counter_bytes(colors, 1);
  }
  uint32_t* pattern = reinterpret_cast<uint32_t*>(p);
  uint32_t* rows = pattern + kWideSeeds;
  load_index_smem(gix, six);
  if (scount)
    for (uint32_t c = threadIdx.x; c < colors; c += blockDim.x) scount[c] = 0;
  __syncthreads();
  const DevIndex& ix = *six;
  WideCounters cnt{scount, counts};
  const int H = ix.hashes, Hp = (H + 3) & ~3, b = ix.bits, lb = log2_bits(b);
  const uint32_t ones = field_ones(b), hi = ones << (b - 1);
  const uint32_t fmask = b == 32 ? 0xFFFFFFFFu : (1u << b) - 1u;
  const uint32_t per_seed = classes * (uint32_t)Hp;
  const uint32_t T = blockDim.x, tid = threadIdx.x;
  // Teams of TT threads (the whole block for wide rows; fewer threads for
  // rows of few chunks, each team then walking its own share of the round's
  // seeds). Thread tt of a team owns chunks tt, tt + TT, ...
  const uint32_t TT = team_threads && team_threads < T ? team_threads : T;
  const uint32_t tt = tid % TT, team = tid / TT, teams = T / TT;

  // The chunks this thread owns, their class and masks (a chunk pruned in a
  // per-record report loses its row pointer and field mask until the next
  // segment sets them up again).
  const uint8_t* col[J];
  uint32_t stride[J], roff[J], g0[J], valid[J], multi[J], cls[J];
  uint32_t planes[J][kWidePlanes];
#pragma unroll
  for (int j = 0; j < J; ++j)
#pragma unroll
    for (int k = 0; k < kWidePlanes; ++k) planes[j][k] = 0;
  auto setup_chunks = [&]() {
#pragma unroll
  for (int j = 0; j < J; ++j) {
    col[j] = nullptr;
    stride[j] = roff[j] = g0[j] = valid[j] = multi[j] = cls[j] = 0;
    uint32_t g = tt + (uint32_t)j * TT, start = 0;
    for (uint32_t ci = 0; ci < classes; ++ci) {
      const DevClass& C = ix.cls[ci];
      if (g < start + C.fp_chunks) {
        const uint32_t k = g - start;
        col[j] = C.data + (uint64_t)k * 16u;
        stride[j] = C.row_stride;
        roff[j] = ci * (uint32_t)Hp;
        cls[j] = ci;
        g0[j] = k * (128u >> lb);
        for (uint32_t bit = 0; bit < 32; ++bit) {
          if ((bit & (uint32_t)(b - 1)) >= 4u) continue;
          const uint32_t grp = wide_group(g0[j], bit, b, lb);
          if (grp >= C.groups) continue;
          valid[j] |= 1u << bit;
          if (__ldg(C.group_color + grp) & kMultiGroup) multi[j] |= 1u << bit;
        }
        break;
      }
      start += C.fp_chunks;
    }
  }
  };
  setup_chunks();

  auto flush = [&]() {
#pragma unroll
    for (int j = 0; j < J; ++j) {
      uint32_t any = 0;
#pragma unroll
      for (int k = 0; k < kWidePlanes; ++k) any |= planes[j][k];
      if (!any) continue;
      const DevClass& C = ix.cls[cls[j]];
      while (any) {
        const uint32_t bit = __ffs(any) - 1;
        any &= any - 1;
        uint32_t v = 0;
#pragma unroll
        for (int k = 0; k < kWidePlanes; ++k) v |= ((planes[j][k] >> bit) & 1u) << k;
        cnt.add(__ldg(C.group_color + wide_group(g0[j], bit, b, lb)), v);
      }
#pragma unroll
      for (int k = 0; k < kWidePlanes; ++k) planes[j][k] = 0;
    }
  };

  unsigned long long seeds = 0;
  uint32_t steps = 0;
  // Threshold pruning (record_query.rs:28-107, exact): in a per-record report
  // a colour is reported only with at least `need` of its record's seeds.
  // Its final count is at most its block counter plus the segment's seeds
  // this team has not probed yet (the other rounds' hits are at most their
  // seeds), so once no field of a chunk can reach `need` the thread stops
  // loading that chunk for the rest of the segment. Counts of pruned
  // colours stay below the threshold, so the reported hits are unchanged.
  // Chunks of multi-member groups are never pruned; segments split across
  // extraction rounds and global counters turn pruning off.
  uint32_t alive = (1u << J) - 1u;
  uint64_t need = 0, seg_total = 0, seen = 0;  // seen: this team's seeds flushed in the segment
  bool prune = false;
  uint32_t flush_at = kWideFlush;  // seeds between flushes (kPruneStep while pruning)
  auto prune_chunks = [&]() {
    const uint64_t rest = seg_total - seen;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      if (!((alive >> j) & 1u) || !col[j] || multi[j]) continue;
      const DevClass& C = ix.cls[cls[j]];
      uint32_t best = 0;
      for (uint32_t x = valid[j]; x; x &= x - 1) {
        const uint32_t c = __ldg(C.group_color + wide_group(g0[j], __ffs(x) - 1, b, lb));
        best = max(best, scount[c]);
      }
      if ((uint64_t)best + rest < need) {
        alive &= ~(1u << j);
        col[j] = nullptr;
        valid[j] = 0;
      }
    }
  };
  // Segmented: the block's counters belong to one segment at a time. They
  // go to that segment's counts when the block moves on (a plain add when
  // the segment has one round, so this block is its only writer).
  uint32_t cur = 0xFFFFFFFFu;
  auto leave_segment = [&]() {
    flush();
    steps = 0;
    if (!scount) return;
    __syncthreads();
    if (cur != 0xFFFFFFFFu) {
      uint64_t* out = counts + (uint64_t)cur * colors;
      const bool owner = __ldg(sg.round_first + cur + 1) - __ldg(sg.round_first + cur) == 1u;
      for (uint32_t c = tid; c < colors; c += T) {
        const uint32_t v = scount[c];
        if (!v) continue;
        if (owner) out[c] += v;
        else atomicAdd(reinterpret_cast<unsigned long long*>(out + c), (unsigned long long)v);
        scount[c] = 0;
      }
    }
    __syncthreads();
  };
  // Rounds of 256 seeds. Unsegmented, contiguous: round r is seeds 256r ..
  // 256r + 255 of the dense list, round-robin over the blocks (in an ordered
  // list each block walks its own neighbourhood of rows). Unsegmented,
  // interleaved: block b takes the seeds b, b + G, b + 2G, ... (G blocks), so
  // all blocks work on neighbouring seeds at the same time. Segmented: rounds
  // of 256 consecutive seeds of one segment, round-robin over the blocks.
  const uint64_t G = gridDim.x;
  const bool inter = !sg.nseg && sg.interleave;
  const uint64_t nk = sg.nseg ? 0 : *nkeys;
  const uint64_t mine = !inter || nk <= blockIdx.x ? 0 : (nk - blockIdx.x + G - 1) / G;
  const uint64_t nrounds = sg.nseg ? (uint64_t)__ldg(sg.round_first + sg.nseg)
                           : inter ? (mine + kWideSeeds - 1) / kWideSeeds
                                   : (nk + kWideSeeds - 1) / kWideSeeds;
  for (uint64_t r = inter ? 0 : blockIdx.x; r < nrounds; r += inter ? 1 : G) {
    uint64_t base, kstride = 1;  // seed i of the round: keys[base + i * kstride]
    uint32_t n;
    if (sg.nseg) {
      const uint32_t seg = segment_of(sg.round_first, sg.nseg, (uint32_t)r);
      const uint64_t k = (uint64_t)((uint32_t)r - __ldg(sg.round_first + seg)) * kWideSeeds;
      const uint64_t have = sg.cursor[seg];
      base = wide_seg_base(sg, seg) + k;
      n = have - k < (uint64_t)kWideSeeds ? (uint32_t)(have - k) : (uint32_t)kWideSeeds;
      if (seg != cur) {  // uniform across the block
        leave_segment();
        cur = seg;
        cnt.gmem = counts + (uint64_t)seg * colors;
        if (alive != (1u << J) - 1u) setup_chunks();
        alive = (1u << J) - 1u;
        seen = 0;
        prune = false;
        flush_at = kWideFlush;
        if (sg.min_ratio > 0.0 && scount && __ldg(sg.seg_tiles + seg) >= sg.tile_lo &&
            __ldg(sg.seg_tiles + seg + 1) <= sg.tile_hi) {
          seg_total = have;  // the whole segment is in this round
          need = minimum_matches(have, sg.min_ratio);
          prune = need > 0;
          if (prune) flush_at = kPruneStep;
        }
      }
      if (tid == 0) atomicAdd(sg.totals + seg, (unsigned long long)n);
    } else if (inter) {
      base = r * kWideSeeds * G + blockIdx.x;
      kstride = G;
      const uint64_t left = mine - r * kWideSeeds;
      n = left < (uint64_t)kWideSeeds ? (uint32_t)left : (uint32_t)kWideSeeds;
    } else {
      base = r * kWideSeeds;
      n = nk - base < (uint64_t)kWideSeeds ? (uint32_t)(nk - base) : (uint32_t)kWideSeeds;
    }
    // Descriptors: pattern and row indices of each seed; recovered origins
    // the filter misses are counted by the seed's owner.
    for (uint32_t i = tid; i < n; i += T) {
      const uint64_t key = keys[base + (uint64_t)i * kstride];
      const uint64_t first = mixsplit(key, ix.seed), step = splitmix64(first);
      const uint32_t fp = (uint32_t)fingerprint(key, ix.seed, b);
      pattern[i] = fp * ones;
      uint32_t* my = rows + i * per_seed;
      for (uint32_t ci = 0; ci < classes; ++ci) {
        const DevClass& C = ix.cls[ci];
        const uint32_t part = C.partitions > 1 ? partition_id(key, ix.seed, C.partitions) : 0;
        const uint64_t count = C.slots / C.seg - (uint64_t)H + 1;
        const uint32_t seg = (uint32_t)C.seg;
        const uint32_t row0 = (uint32_t)((uint64_t)part * C.slots + mulhi64(first, count) * C.seg);
        uint64_t h = first;
        for (int r = 0; r < H; ++r, h += step)
          my[ci * Hp + r] = row0 + (uint32_t)r * seg + (((uint32_t)h ^ (uint32_t)(h >> 33)) & (seg - 1));
      }
      const RecHit rec = recovery_lookup(ix.rec, recovery_hash(key, ix.seed));
      for (uint32_t o = 0; o < rec.len; ++o) {
        const uint32_t c = rec.at(o);
        const ColorLoc loc = color_loc[c];
        bool hit = false;
        if (loc.cls_member != 0xFFFFFFFFu) {
          const uint32_t ci = loc.cls_member & 0xFFu, mi = loc.cls_member >> 8, g = loc.group;
          const DevClass& C = ix.cls[ci];
          const uint32_t* rr = my + ci * Hp;
          uint64_t fx = 0;
          for (int r = 0; r < H; ++r)
            fx ^= row_bits(C.data + (uint64_t)rr[r] * C.row_stride, g * (uint32_t)b, (uint32_t)b);
          hit = (uint32_t)fx == (fp & fmask);
          const uint32_t gc = __ldg(C.group_color + g);
          if (hit && (gc & kMultiGroup)) {
            const uint32_t* mg = C.multi + 3 * (gc & ~kMultiGroup);
            const uint32_t off = __ldg(mg), w = __ldg(mg + 1);
            uint64_t mx = 0;
            for (int r = 0; r < H; ++r) mx ^= row_bits(C.data + (uint64_t)rr[r] * C.row_stride, off, w);
            hit = (mx >> mi) & 1u;
          }
        }
        if (!hit) cnt.add(c, 1);
      }
    }
    if (tid == 0 && !sg.nseg) seeds += n;
    __syncthreads();
    const uint32_t per = (n + teams - 1) / teams;
    const uint32_t first_seed = min(n, team * per), end_seed = min(n, first_seed + per);
    for (uint32_t s0 = first_seed; s0 < end_seed; s0 += S) {
      uint4 acc[J][S];
#pragma unroll
      for (int j = 0; j < J; ++j)
#pragma unroll
        for (int s = 0; s < S; ++s) acc[j][s] = make_uint4(0, 0, 0, 0);
      for (int i0 = 0; i0 < H; i0 += HQ) {
        uint4 v[J][S][HQ];
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const uint32_t sd = min(s0 + (uint32_t)s, end_seed - 1);
          const bool live = s0 + (uint32_t)s < end_seed;
#pragma unroll
          for (int j = 0; j < J; ++j) {
            uint32_t ri[HQ];
#pragma unroll
            for (int q = 0; q < HQ; q += 4) {
              const uint4 r4 = *reinterpret_cast<const uint4*>(rows + sd * per_seed + roff[j] + i0 + q);
              ri[q] = r4.x; ri[q + 1] = r4.y; ri[q + 2] = r4.z; ri[q + 3] = r4.w;
            }
#pragma unroll
            for (int q = 0; q < HQ; ++q) {
              v[j][s][q] = make_uint4(0, 0, 0, 0);
              if (live && col[j] && i0 + q < H)
                v[j][s][q] = ld_row_chunk(col[j] + (uint64_t)ri[q] * stride[j]);
            }
          }
        }
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
          for (int s = 0; s < S; ++s)
#pragma unroll
            for (int q = 0; q < HQ; ++q) {
              acc[j][s].x ^= v[j][s][q].x; acc[j][s].y ^= v[j][s][q].y;
              acc[j][s].z ^= v[j][s][q].z; acc[j][s].w ^= v[j][s][q].w;
            }
      }
#pragma unroll
      for (int s = 0; s < S; ++s) {
        const uint32_t sd = s0 + (uint32_t)s;
        if (sd >= end_seed) continue;
        const uint32_t pat = pattern[sd];
#pragma unroll
        for (int j = 0; j < J; ++j) {
          const uint32_t w4[4] = {acc[j][s].x, acc[j][s].y, acc[j][s].z, acc[j][s].w};
          uint32_t d = 0;
#pragma unroll
          for (int w = 0; w < 4; ++w) d |= zero_fields_hi(w4[w] ^ pat, hi) >> (uint32_t)(b - 1 - w);
          d &= valid[j];
          const uint32_t slow = d & multi[j];
          uint32_t m = d & ~slow;
#pragma unroll
          for (int k = 0; k < kWidePlanes; ++k) {
            const uint32_t t = planes[j][k] & m;
            planes[j][k] ^= m;
            m = t;
          }
          for (uint32_t x = slow; x; x &= x - 1) {
            const DevClass& C = ix.cls[cls[j]];
            const uint32_t g = wide_group(g0[j], __ffs(x) - 1, b, lb);
            const uint32_t gc = __ldg(C.group_color + g);
            const uint32_t* mg = C.multi + 3 * (gc & ~kMultiGroup);
            const uint32_t off = __ldg(mg), w = __ldg(mg + 1), firstm = __ldg(mg + 2);
            const uint32_t* rr = rows + sd * per_seed + roff[j];
            uint64_t mx = 0;
            for (int r = 0; r < H; ++r) mx ^= row_bits(C.data + (uint64_t)rr[r] * C.row_stride, off, w);
            while (mx) {
              const uint32_t mb = __ffsll((long long)mx) - 1;
              mx &= mx - 1;
              cnt.add(__ldg(C.members + firstm + mb), 1);
            }
          }
        }
        if (++steps == flush_at) {
          flush();
          seen += steps;
          steps = 0;
          if (prune) prune_chunks();
        }
      }
    }
    __syncthreads();
  }
  if (sg.nseg) {
    leave_segment();
    return;
  }
  flush();
  if (tid == 0 && seeds) atomicAdd(total, seeds);
  __syncthreads();
  if (scount)
    for (uint32_t c = threadIdx.x; c < colors; c += blockDim.x)
      partial[(uint64_t)blockIdx.x * colors + c] = scount[c];
}

}  // namespace zx
