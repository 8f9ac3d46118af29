// Batched query kernels: tile planning, the fused seed-extraction + probe
// kernel and the per-colour counter reduction.
//
// A batch is many records of uneven length (bases concatenated, offsets[r]
// .. offsets[r+1]). Records are cut into tiles of at most kTileWindows
// windows (a device work list built by plan_tiles); one warp extracts the
// seeds of a tile into shared memory and then probes them with teams of T
// lanes. Counters live in shared memory per block and are reduced at the end
// (the aggregate matches[] of query_ordinary, query_stream.rs:280-300, and
// flush, storage.rs:3545-3598).
#pragma once
#include <stdint.h>

#include "device_index.cuh"
#include "probe.cuh"
#include "seeds.cuh"

namespace zx {

constexpr uint32_t kTileWindows = 256;
constexpr uint32_t kFindereTask = 16384;  // src/findere.rs:13-16
// Findere indexes of up to this many colours keep each warp's round masks and
// run lengths in shared memory (8 bytes per colour and warp).
constexpr uint32_t kFindereSmemColors = 512;
constexpr uint32_t kSplitTiles = 1u << 18;  // tiles per round of a split minimizer query
// Randstrobemer seeds of a tile (strobes.cuh): its windows' positions plus up
// to kStrobeExtra minimizer positions past a record's last window start.
constexpr uint32_t kStrobeExtra = 64;
constexpr uint32_t kStrobeSlot = 256 + kStrobeExtra;

// Windows of record r: k-windows fully inside the record. A record whose
// offsets decrease, pass the end of the bases or span 2^31 bases or more has
// no windows and sets kErrOffsets (the query then fails with ZX_EINVAL), so
// no tile ever points outside the batch.
__device__ __forceinline__ uint32_t record_windows(const uint64_t* offsets, uint64_t r, int span,
                                                   uint64_t nbases, uint32_t* err) {
  const uint64_t a = offsets[r], b = offsets[r + 1];
  if (a > b || b > nbases || b - a >= (1ull << 31)) {
    if (err) atomicOr(err, kErrOffsets);
    return 0u;
  }
  const uint64_t len = b - a;
  return len >= (uint64_t)span ? (uint32_t)(len - span + 1) : 0u;
}

// Tiles per record. Findere tiles never cross a 16,384-window task.
__device__ __forceinline__ uint32_t record_tiles(uint32_t w, int findere) {
  if (!findere) return (w + kTileWindows - 1) / kTileWindows;
  const uint32_t full = w / kFindereTask, rest = w % kFindereTask;
  return full * (kFindereTask / kTileWindows) + (rest + kTileWindows - 1) / kTileWindows;
}

__global__ void count_tiles_kernel(const uint64_t* __restrict__ offsets, uint64_t records,
                                   uint64_t nbases, int span, int findere,
                                   uint32_t* __restrict__ counts, uint32_t* __restrict__ err) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < records;
       r += (uint64_t)gridDim.x * blockDim.x) {
    counts[r] = record_tiles(record_windows(offsets, r, span, nbases, err), findere);
  }
}

__global__ void fill_tiles_kernel(const uint64_t* __restrict__ offsets, uint64_t records,
                                  uint64_t nbases, int span, const uint32_t* __restrict__ first,
                                  Tile* __restrict__ tiles) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < records;
       r += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t w = record_windows(offsets, r, span, nbases, nullptr);
    uint32_t t = first[r];
    for (uint32_t w0 = 0; w0 < w;) {
      uint32_t task = (w0 / kFindereTask) * kFindereTask;
      uint32_t end = min(w, min(w0 + kTileWindows, task + kFindereTask));
      tiles[t++] = Tile{(uint32_t)r, w0, end - w0, task};
      w0 = end;
    }
  }
}

// Small batches (a few thousand records, up to 1 MiB of bases): one block
// packs the bases and plans the tiles (count, scan and fill), so the query is
// two launches instead of six.
constexpr uint32_t kSmallRecords = 4096;
constexpr uint64_t kSmallBases = 1ull << 20;

__global__ void __launch_bounds__(1024)
    small_plan_kernel(const uint8_t* __restrict__ bases, uint64_t nbases,
                      uint64_t* __restrict__ packed, uint32_t* __restrict__ invalid,
                      uint64_t words, const uint64_t* __restrict__ offsets, uint32_t records,
                      int span, int findere, uint32_t* __restrict__ tile_first,
                      Tile* __restrict__ tiles, uint32_t* __restrict__ err) {
  __shared__ uint32_t sums[1024];
  const uint32_t T = blockDim.x, tid = threadIdx.x;
  for (uint64_t w = tid; w < words; w += T) pack_word(bases, nbases, packed, invalid, w);
  // Each thread plans a contiguous run of records: their tile counts, a
  // block scan of the runs' sums, then the tiles.
  const uint32_t per = (records + T - 1) / T;
  const uint32_t lo = min(records, tid * per), hi = min(records, lo + per);
  uint32_t mine = 0;
  for (uint32_t r = lo; r < hi; ++r)
    mine += record_tiles(record_windows(offsets, r, span, nbases, err), findere);
  sums[tid] = mine;
  __syncthreads();
  for (uint32_t off = 1; off < T; off <<= 1) {
    const uint32_t v = tid >= off ? sums[tid - off] : 0u;
    __syncthreads();
    sums[tid] += v;
    __syncthreads();
  }
  uint32_t t = tid ? sums[tid - 1] : 0u;
  for (uint32_t r = lo; r < hi; ++r) {
    tile_first[r] = t;
    const uint32_t w = record_windows(offsets, r, span, nbases, nullptr);
    for (uint32_t w0 = 0; w0 < w;) {
      const uint32_t task = (w0 / kFindereTask) * kFindereTask;
      const uint32_t end = min(w, min(w0 + kTileWindows, task + kFindereTask));
      tiles[t++] = Tile{r, w0, end - w0, task};
      w0 = end;
    }
  }
  if (tid == T - 1) tile_first[records] = sums[T - 1];
}

struct BatchView {
  PackedView pv;
  const uint64_t* offsets;
  const Tile* tiles;
  const uint32_t* ntiles;  // device scalar
  uint32_t* fstate;        // findere: per warp of the grid, colours round masks then run lengths
  // Segmented launch (several requests in one launch, each with its own
  // counters): 0, or the number of segments; segment s owns blocks
  // seg_blocks[s] .. seg_blocks[s+1]-1 and tiles seg_tiles[s] .. seg_tiles[s+1]-1.
  uint32_t segments;
  const uint32_t* seg_blocks;
  const uint32_t* seg_tiles;
  // Tile range of a launch over part of the list: tiles tile_lo .. tile_hi-1
  // (tile_hi 0 = to the end). Seeds extracted beforehand (MODE 4): tile t's
  // keys are prekeys[(t - tile_lo) * stride ...], prekey_count[t - tile_lo] of
  // them (stride = prekey_stride, or kTileWindows when 0).
  uint32_t tile_lo, tile_hi;
  const uint64_t* prekeys;
  const uint32_t* prekey_count;
  uint32_t prekey_stride;
};

// Shared memory of the fused kernel, in order: DevIndex copy, counters,
// inner hash table (minimizers), then per warp: keys[2 * kTileWindows], 32
// seed descriptors, 32 x classes row offsets, minimizer scratch (pre, suf,
// pos).
struct FusedSmem {
  static constexpr size_t ix_bytes = (sizeof(DevIndex) + 15) / 16 * 16;
  static constexpr size_t map_bytes = (kMaxClasses * 2 + 15) / 16 * 16;  // shared-plane bases
  static __host__ __device__ size_t counter_bytes(uint32_t colors, int smem_counters) {
    return smem_counters ? ((size_t)colors * 4 + 15) / 16 * 16 : 0;
  }
  static __host__ __device__ size_t ocm_entries(int k) { return kTileWindows + (size_t)k + 1; }
  // Seed descriptors plus, per gather form: row offsets of position 0 for
  // 64 seeds x classes (8 bytes each; descriptor and staged gathers) or the
  // row indices of 32 seeds x classes x H rounded up to 4 (4 bytes each;
  // row-index gather with bit-plane counters).
  static __host__ __device__ size_t probe_bytes(uint32_t classes, int hashes = 4, int planes = 0) {
    const size_t rows = planes ? 32 * 4 * (size_t)classes * (size_t)((hashes + 3) & ~3)
                               : 64 * 8 * (size_t)classes;
    return 64 * sizeof(SeedDesc) + rows;
  }
  static __host__ __device__ size_t ring_bytes(int stage_bytes, int stages) {
    return stage_bytes > 0 ? (size_t)stage_bytes * stages + 8 * 8 : 0;
  }
  static __host__ __device__ size_t shared_plane_bytes(uint32_t words) {
    return (size_t)words * (kSharedPlanes + 2) * 32 * 4;
  }
  // Key buffer of a warp: one tile's keys, plus the lane-run staging of the
  // polynomial k-mer hashes (modes 0 and 2 with k > 32) and of findere s-mers.
  // Randstrobemer seeds (probed in mode 4): one tile's slot of kStrobeSlot.
  static __host__ __device__ size_t key_bytes(int mode, int k, bool strobes = false) {
    if (strobes) return (size_t)kStrobeSlot * 8;
    const bool staged = mode == 3 || ((mode == 0 || mode == 2) && k > 32);
    return (staged ? 2 : 1) * (size_t)kTileWindows * 8;
  }
  // Findere round masks and run lengths of a warp in shared memory (indexes
  // of up to kFindereSmemColors colours; else in the global scratch).
  static __host__ __device__ size_t findere_state_bytes(uint32_t colors) {
    return colors <= kFindereSmemColors ? (size_t)colors * 8 + (size_t)(colors + 31) / 32 * 8 : 0;
  }
  static __host__ __device__ size_t warp_bytes(int mode, int k, uint32_t classes, int stage_bytes = 0,
                                               int stages = 0, int hashes = 4, int planes = 0,
                                               uint32_t shared_words = 0, bool strobes = false,
                                               uint32_t colors = 0) {
    size_t b = key_bytes(mode, k, strobes) + probe_bytes(classes, hashes, planes) +
               ring_bytes(stage_bytes, stages) + shared_plane_bytes(shared_words);
    if (mode == 1) b += 2 * ocm_entries(k) * sizeof(Rank16) + (kTileWindows + 1) * 4 + 16;
    // Findere: valid bits of up to 512 s-mer positions, then the round state.
    if (mode == 3) b += 64 + findere_state_bytes(colors);
    return (b + 15) / 16 * 16;
  }
  // Findere always runs the row-index probe without a staged ring.
  // shared_words: shared-plane words per lane (shared_plane_layout).
  static __host__ __device__ size_t total(int mode, int k, uint32_t colors, uint32_t classes,
                                          int hashes, const QueryLaunch& l,
                                          uint32_t shared_words = 0, bool strobes = false) {
    const bool fin = mode == 3;
    return ix_bytes + map_bytes + counter_bytes(colors, l.smem_counters) +
           (mode == 1 ? 256 * 8 : 0) +
           (size_t)l.warps * warp_bytes(mode, k, classes, fin ? 0 : l.stage_bytes, l.stages, hashes,
                                        fin ? 1 : l.planes, shared_words, strobes, colors);
  }
  // Shared-plane words per lane a launch uses (0 unless the row-index form
  // counts in planes).
  static __host__ __device__ uint32_t shared_words(int mode, const DevIndex& ix,
                                                   const QueryLaunch& l) {
    if (mode == 3 || !l.planes || l.stage_bytes > 0) return 0;
    return shared_plane_layout(ix, l.team, nullptr);
  }
};

// Extracts the seeds of one tile into `keys`; returns their number.
template <int MODE>
__device__ __forceinline__ uint32_t extract_tile(const BatchView& bv, const SeedParams& sp,
                                                 const Tile& t, uint64_t* keys, uint8_t* ocm,
                                                 const uint64_t* inner, int lane) {
  const uint64_t rb = bv.offsets[t.record];
  uint32_t n;
  if (MODE == 1) {
    if (sp.k == sp.m) {
      n = tile_ocm_full(bv.pv, rb, t.w0, t.nw, sp.m, keys, lane);
    } else {
      Rank16* pre = reinterpret_cast<Rank16*>(ocm);
      Rank16* suf = pre + FusedSmem::ocm_entries(sp.k);
      uint32_t* pos = reinterpret_cast<uint32_t*>(suf + FusedSmem::ocm_entries(sp.k));
      n = tile_ocm(bv.pv, rb, t.w0, t.nw, sp, inner, pre, suf, pos, keys, lane);
    }
  } else if (sp.klen <= 32) {
    n = tile_kmers_short(bv.pv, rb, t.w0, t.nw, sp.klen, MODE == 2, sp.seed, sp.sampling, keys,
                         lane);
  } else {
    n = tile_kmers_long(bv.pv, rb, t.w0, t.nw, sp.klen, sp.lk, MODE == 2, sp.seed, sp.sampling,
                        keys, keys + kTileWindows, lane);
  }
  // Spaced seeds (anchors.rs:265-281; k-mer and minimizer indexes, patterns of
  // width k or m <= 31): the plain canonical keys, selected first, are mapped
  // through the pattern.
  if (MODE <= 1 && sp.spaced) {
    __syncwarp();
    for (uint32_t i = lane; i < n; i += 32) keys[i] = spaced_canonical(sp.pattern, keys[i]);
  }
  return n;
}

__device__ __forceinline__ void load_index_smem(const DevIndex* __restrict__ gix, DevIndex* six) {
  const uint4* src = reinterpret_cast<const uint4*>(gix);
  uint4* dst = reinterpret_cast<uint4*>(six);
  for (uint32_t i = threadIdx.x; i < sizeof(DevIndex) / 16; i += blockDim.x) dst[i] = src[i];
}

__device__ __forceinline__ void build_inner_table(const SeedParams& sp, uint64_t* inner) {
  if (sp.mode != 1) return;
  const int s = sp.ocm.s;
  for (uint32_t v = threadIdx.x; v < (1u << (2 * s)); v += blockDim.x)
    inner[v] = mixsplit(canonical_encoded(v, s), sp.seed ^ kInnerHashSeed);
}

// Fused extraction + probe over the tile list (one instantiation per seed
// mode). partial: gridDim.x x colors block counters (smem_counters); counts:
// global counters (used directly when smem_counters == 0). total: seeds.
template <int MODE, int MINB, int VARIANT>
__global__ void __launch_bounds__(256, MINB) fused_query_kernel(const DevIndex* __restrict__ gix,
                                                          BatchView bv, SeedParams sp,
                                                          QueryLaunch lc,
                                                          uint32_t* __restrict__ partial,
                                                          uint64_t* __restrict__ counts,
                                                          unsigned long long* __restrict__ total,
                                                          uint32_t* __restrict__ err) {
  extern __shared__ __align__(16) uint8_t smem[];
  DevIndex* six = reinterpret_cast<DevIndex*>(smem);
  uint16_t* pbase = reinterpret_cast<uint16_t*>(smem + FusedSmem::ix_bytes);
  uint8_t* p = smem + FusedSmem::ix_bytes + FusedSmem::map_bytes;
  uint32_t* scount = nullptr;
  const uint32_t colors = gix->colors, classes = gix->classes;
  if (lc.smem_counters) {
    scount = reinterpret_cast<uint32_t*>(p);
    p += FusedSmem::counter_bytes(colors, 1);
  }
  uint64_t* inner = nullptr;
  if (MODE == 1) {
    inner = reinterpret_cast<uint64_t*>(p);
    p += 256 * 8;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int hashes = gix->hashes;
  // Findere always runs the row-index probe (VARIANT 2) without a ring.
  constexpr bool ROWS = VARIANT == 2 || MODE == 3;
  const int stage_bytes = MODE == 3 ? 0 : lc.stage_bytes;
  const uint32_t swords = VARIANT == 2 ? FusedSmem::shared_words(MODE, *gix, lc) : 0u;
  const size_t wstride = FusedSmem::warp_bytes(MODE, sp.k, classes, stage_bytes, lc.stages, hashes,
                                               ROWS, swords, sp.strobe_max != 0, colors);
  uint8_t* wbase = p + (size_t)warp * wstride;
  uint64_t* keys = reinterpret_cast<uint64_t*>(wbase);
  SeedDesc* desc = reinterpret_cast<SeedDesc*>(wbase + FusedSmem::key_bytes(MODE, sp.k, sp.strobe_max != 0));
  uint64_t* row0s = reinterpret_cast<uint64_t*>(desc + 64);
  uint8_t* ring_base = wbase + FusedSmem::key_bytes(MODE, sp.k, sp.strobe_max != 0) + FusedSmem::probe_bytes(classes, hashes, ROWS);
  uint8_t* ocm = ring_base + FusedSmem::ring_bytes(stage_bytes, lc.stages);
  if (MODE == 3 && colors <= kFindereSmemColors) {
    // Masks, run lengths, then the touched and run bitmaps of this warp.
    uint32_t* fst = reinterpret_cast<uint32_t*>(ocm + 64);
    for (uint32_t c = lane; c < 2 * colors + 2 * ((colors + 31) / 32); c += 32) fst[c] = 0;
    __syncwarp();
  }
  SharedPlanes splanes{reinterpret_cast<uint32_t*>(wbase + wstride - FusedSmem::shared_plane_bytes(swords)),
                       swords, 0u};
  StageRing ring{ring_base + 64, reinterpret_cast<uint64_t*>(ring_base), (uint32_t)lc.stage_bytes,
                 (uint32_t)lc.stages, 0u, 0u, lc.bulk != 0};
  constexpr bool STAGED = VARIANT == 1;
  if (STAGED && lc.bulk) {
    if (lane == 0) {
      for (int st = 0; st < lc.stages; ++st) mbar_init(ring.bars + st, 1);
      mbar_fence_init();
    }
    __syncwarp();
  }

  load_index_smem(gix, six);
  if (MODE == 1) build_inner_table(sp, inner);
  if (scount)
    for (uint32_t c = threadIdx.x; c < colors; c += blockDim.x) scount[c] = 0;
  __syncthreads();
  const DevIndex& ix = *six;
  LanePlanes planes;
  if (ROWS) planes_init(planes, ix, lane % lc.team, lc.team);
  if (MODE == 3) planes.cls = -1;  // findere: every hit goes to the position masks
  if (swords) {
    if (threadIdx.x == 0) shared_plane_layout(ix, lc.team, pbase);
    __syncthreads();
    shared_planes_init(splanes, ix, pbase, lane % lc.team, lc.team, lane);
    __syncwarp();
  }
  const uint32_t wpb = blockDim.x >> 5;
  const uint32_t gwarp = blockIdx.x * wpb + warp;
  // Tile range of this warp: the whole list, or its block's segment.
  uint32_t t_first = bv.tile_lo + gwarp, t_end = *bv.ntiles, t_stride = gridDim.x * wpb, seg = 0;
  if (bv.tile_hi && bv.tile_hi < t_end) t_end = bv.tile_hi;
  if (bv.segments) {
    uint32_t lo = 0, hi = bv.segments;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (bv.seg_blocks[mid] <= blockIdx.x) lo = mid;
      else hi = mid;
    }
    seg = lo;
    t_first = bv.seg_tiles[seg] + (blockIdx.x - bv.seg_blocks[seg]) * wpb + warp;
    t_end = bv.seg_tiles[seg + 1];
    t_stride = (bv.seg_blocks[seg + 1] - bv.seg_blocks[seg]) * wpb;
  }
  const Counters cnt{scount, counts + (uint64_t)seg * colors};
  unsigned long long seeds = 0;
  for (uint32_t t = t_first; t < t_end; t += t_stride) {
    const Tile tile = bv.tiles[t];
    if constexpr (MODE == 3) {
      // Findere: s-mers of positions 0 .. nw + z - 1, windows are the features.
      const int z = sp.k - sp.klen;
      const uint32_t npos = tile.nw + (uint32_t)z;
      const uint64_t rb = bv.offsets[tile.record];
      uint32_t* kvalid = reinterpret_cast<uint32_t*>(ocm);
      tile_smers(bv.pv, rb, tile.w0, npos, sp.klen, sp.lk, keys, kvalid, lane);
      for (uint32_t i0 = 0; i0 < tile.nw; i0 += 32) {
        const uint32_t i = i0 + lane;
        const bool ok = i < tile.nw && bv.pv.valid(rb + tile.w0 + i, (uint32_t)sp.k);
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, ok);
        if (lane == 0) seeds += __popc(bal);
      }
      const bool fshared = colors <= kFindereSmemColors;
      uint32_t* fmask = fshared ? reinterpret_cast<uint32_t*>(ocm + 64)
                                : bv.fstate + (uint64_t)gwarp * 2 * colors;
      uint32_t* frun = fmask + colors;
      const FindereSink fs{fmask, fshared ? frun + colors : nullptr};
      probe_rows<MINB == 1>(ix, keys, npos, kvalid, desc, reinterpret_cast<uint32_t*>(row0s), lc.team, planes,
                 splanes, pbase, fs, lane, [&](uint32_t r0, uint32_t m) {
                   __syncwarp();
                   if (fshared) findere_sweep<true>(fmask, frun, colors, z, m, r0 + m >= npos, cnt, lane);
                   else findere_sweep<false>(fmask, frun, colors, z, m, r0 + m >= npos, cnt, lane);
                   __syncwarp();
                 });
      continue;
    } else {
    uint32_t n;
    if constexpr (MODE == 4) {
      // Seeds extracted beforehand into this tile's slot.
      const uint64_t slot =
          (uint64_t)(t - bv.tile_lo) * (bv.prekey_stride ? bv.prekey_stride : kTileWindows);
      n = bv.prekey_count[t - bv.tile_lo];
      for (uint32_t i = lane; i < n; i += 32) keys[i] = bv.prekeys[slot + i];
    } else {
      n = extract_tile<MODE>(bv, sp, tile, keys, ocm, inner, lane);
    }
    __syncwarp();
    seeds += n;
    if (STAGED) {
      if (!probe_batch_async(ix, keys, n, desc, row0s, ring, cnt, lane, err)) {
        ring_drain(ring);
        break;
      }
    } else if (VARIANT == 2) {
      probe_rows<MINB == 1>(ix, keys, n, nullptr, desc, reinterpret_cast<uint32_t*>(row0s), lc.team, planes,
                 splanes, pbase, CountSink{cnt}, lane, [](uint32_t, uint32_t) {});
    } else {
      probe_batch(ix, keys, n, desc, row0s, lc.team, cnt, lane);
    }
    }
  }
  if (ROWS && planes.cls >= 0)
    planes_flush(planes, ix, lane % lc.team, lc.team, CountSink{cnt});
  if (swords)
    shared_planes_flush(splanes, ix, pbase, lane % lc.team, lc.team, lane, CountSink{cnt});
  if (lane == 0 && seeds) atomicAdd(total + seg, seeds);
  __syncthreads();
  if (scount)
    for (uint32_t c = threadIdx.x; c < colors; c += blockDim.x)
      partial[(uint64_t)blockIdx.x * colors + c] = scount[c];
}

// counts[c] += sum over blocks of partial[block][c].
__global__ void reduce_counters_kernel(const uint32_t* __restrict__ partial, uint32_t blocks,
                                       uint32_t colors, uint64_t* __restrict__ counts) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < colors; c += gridDim.x * blockDim.x) {
    uint64_t s = 0;
    for (uint32_t b = 0; b < blocks; ++b) s += partial[(uint64_t)b * colors + c];
    counts[c] += s;
  }
}

// Segmented launches: counts[s][c] += sum over the blocks of segment s of
// partial[block][c].
__global__ void reduce_segments_kernel(const uint32_t* __restrict__ partial,
                                       const uint32_t* __restrict__ seg_blocks, uint32_t segments,
                                       uint32_t colors, uint64_t* __restrict__ counts) {
  const uint64_t n = (uint64_t)segments * colors;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t sgm = (uint32_t)(i / colors), c = (uint32_t)(i % colors);
    uint64_t sum = 0;
    for (uint32_t b = seg_blocks[sgm]; b < seg_blocks[sgm + 1]; ++b)
      sum += partial[(uint64_t)b * colors + c];
    counts[i] += sum;
  }
}

// seg_tiles[s] = tile_first[seg_records[s]] for s <= segments (record-first
// tile offsets of a planned batch; tile_first[records] is the tile total).
__global__ void segment_tiles_kernel(const uint32_t* __restrict__ tile_first,
                                     const uint64_t* __restrict__ seg_records, uint32_t segments,
                                     uint32_t* __restrict__ seg_tiles) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s <= segments; s += gridDim.x * blockDim.x)
    seg_tiles[s] = tile_first[seg_records[s]];
}

// Extraction only (testing and inspection): tile t's keys go to
// out[t * kTileWindows ...], their number to out_count[t].
template <int MODE>
__global__ void extract_kernel(BatchView bv, SeedParams sp, uint64_t* __restrict__ out,
                               uint32_t* __restrict__ out_count, int warps_per_block) {
  extern __shared__ __align__(16) uint8_t smem[];
  uint64_t* inner = reinterpret_cast<uint64_t*>(smem);
  uint8_t* p = smem + 256 * 8;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t* wbase = p + (size_t)warp * FusedSmem::warp_bytes(MODE, sp.k, 0, 0, 0, 4, 0, 0,
                                                            sp.strobe_max != 0);
  uint64_t* keys = reinterpret_cast<uint64_t*>(wbase);
  uint8_t* ocm = wbase + FusedSmem::key_bytes(MODE, sp.k, sp.strobe_max != 0) + FusedSmem::probe_bytes(0);
  build_inner_table(sp, inner);
  __syncthreads();
  // Tiles tile_lo .. tile_hi-1 (tile_hi 0 = to the end); tile t's slot is t - tile_lo.
  uint32_t ntiles = *bv.ntiles;
  if (bv.tile_hi && bv.tile_hi < ntiles) ntiles = bv.tile_hi;
  const uint32_t warps_total = gridDim.x * warps_per_block;
  for (uint32_t t = bv.tile_lo + blockIdx.x * warps_per_block + warp; t < ntiles;
       t += warps_total) {
    uint32_t n = extract_tile<MODE>(bv, sp, bv.tiles[t], keys, ocm, inner, lane);
    __syncwarp();
    const uint64_t slot = (uint64_t)(t - bv.tile_lo) * kTileWindows;
    for (uint32_t i = lane; i < n; i += 32) out[slot + i] = keys[i];
    if (lane == 0) out_count[t - bv.tile_lo] = n;
    __syncwarp();
  }
}

}  // namespace zx
