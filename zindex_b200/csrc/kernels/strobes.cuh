// Randstrobemer seeds on the GPU (the Linker, src/anchors.rs:182-256, over
// the candidates of scan, src/anchors.rs:265-353).
//
// Per ACGT run the reference links candidates in position order: every
// canonical k-mer (k-mer indexes), or the run's selected minimizer positions
// sorted and deduplicated (minimizer indexes). Each candidate's partner is the
// first candidate strobe_min..strobe_max bases downstream in the same run
// whose strobe hash differs from it in the fewest of its low 8 bits (the
// candidate itself when there is none); the seed is (h >> 1) + (partner >> 1).
//
// On the device this takes two kernels over the planned tiles:
// * strobe_anchor_kernel marks every candidate in a table indexed by base:
//   bit p of `anchors` when a candidate starts at base p, hashes[p] its strobe
//   hash. A minimizer position selected by several windows is written by each
//   of them with the same value, so the table holds every selected position
//   once, in position order: the reference's sort and deduplication.
// * strobe_link_kernel links each tile's own positions (its windows' starts;
//   the record's last tile also the positions past its last window start,
//   which only minimizer windows select): a forward scan of the table that
//   stops at strobe_max, at the record's end and at the first invalid base
//   (a run break), for any strobe_max. A tile's seeds go to its slot of
//   kStrobeSlot keys, in position order.
#pragma once
#include <stdint.h>

#include "query_kernels.cuh"

namespace zx {

// Shared memory of the anchor kernel: the inner hash table (minimizers),
// then per warp the open-closed minimizer scratch.
struct StrobeSmem {
  static __host__ __device__ size_t warp_bytes(int mode, int k) {
    if (mode != 1) return 0;
    const size_t b = 2 * FusedSmem::ocm_entries(k) * sizeof(Rank16) + (kTileWindows + 1) * 4 + 16;
    return (b + 15) / 16 * 16;
  }
  static __host__ __device__ size_t total(int mode, int k, int warps) {
    return (mode == 1 ? 256 * 8 : 0) + (size_t)warps * warp_bytes(mode, k);
  }
};

__device__ __forceinline__ void strobe_mark(const PackedView& pv, const SeedParams& sp, uint64_t p,
                                            int len, uint32_t* __restrict__ anchors,
                                            uint64_t* __restrict__ hashes) {
  uint64_t key = canonical_at(pv, p, len);
  if (sp.spaced) key = spaced_canonical(sp.pattern, key);
  hashes[p] = strobe_hash(key);
  atomicOr(anchors + (p >> 5), 1u << (p & 31));
}

// MODE 0: k-mer candidates (every valid window). MODE 1: minimizer
// candidates (every window's selected position; every valid m-mer when
// k == m). `anchors` is zeroed before the launch.
template <int MODE>
__global__ void strobe_anchor_kernel(BatchView bv, SeedParams sp, uint32_t* __restrict__ anchors,
                                     uint64_t* __restrict__ hashes, int warps_per_block) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* inner = nullptr;
  uint8_t* wbase = smem;
  if (MODE == 1) {
    inner = reinterpret_cast<uint64_t*>(smem);
    wbase = smem + 256 * 8 + (size_t)warp * StrobeSmem::warp_bytes(1, sp.k);
    build_inner_table(sp, inner);
    __syncthreads();
  }
  const bool plain = MODE == 0 || sp.k == sp.m;
  const int len = MODE == 0 ? sp.klen : sp.m;
  const uint32_t ntiles = *bv.ntiles;
  const uint32_t warps_total = gridDim.x * warps_per_block;
  for (uint32_t t = blockIdx.x * warps_per_block + warp; t < ntiles; t += warps_total) {
    const Tile tile = bv.tiles[t];
    const uint64_t rb = bv.offsets[tile.record];
    if (plain) {
      for (uint32_t i = lane; i < tile.nw; i += 32) {
        const uint64_t p = rb + tile.w0 + i;
        if (bv.pv.valid(p, (uint32_t)len)) strobe_mark(bv.pv, sp, p, len, anchors, hashes);
      }
      continue;
    }
    Rank16* pre = reinterpret_cast<Rank16*>(wbase);
    Rank16* suf = pre + FusedSmem::ocm_entries(sp.k);
    uint32_t* pos = reinterpret_cast<uint32_t*>(suf + FusedSmem::ocm_entries(sp.k));
    tile_ocm_select(bv.pv, rb, tile.w0, tile.nw, sp, inner, pre, suf, pos, lane);
    // Windows w0 .. w0 + nw - 1 (index 0 is the previous tile's last window).
    for (uint32_t i = 1 + lane; i <= tile.nw; i += 32)
      if (pos[i] != 0xFFFFFFFFu)
        strobe_mark(bv.pv, sp, rb + tile.w0 - 1 + pos[i], len, anchors, hashes);
    __syncwarp();
  }
}

// Seeds of every tile into slots[t * kStrobeSlot ...], their number in
// slot_count[t]. len: candidate length (k, or m); extra: positions past a
// record's last window start that can hold candidates (w - 1 for open-closed
// minimizers with k > m, else 0; at most kStrobeExtra).
__global__ void strobe_link_kernel(BatchView bv, SeedParams sp, const uint32_t* __restrict__ anchors,
                                   const uint64_t* __restrict__ hashes, int len, uint32_t extra,
                                   uint64_t* __restrict__ slots, uint32_t* __restrict__ slot_count) {
  const int lane = threadIdx.x & 31;
  const uint32_t ntiles = *bv.ntiles;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint64_t dmin = sp.strobe_min, dmax = sp.strobe_max;
  auto is_anchor = [&](uint64_t p) { return (__ldg(anchors + (p >> 5)) >> (p & 31)) & 1u; };
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += warps) {
    const Tile tile = bv.tiles[t];
    const uint64_t rb = bv.offsets[tile.record];
    const uint64_t rlen = bv.offsets[tile.record + 1] - rb;
    const uint64_t windows = rlen >= (uint64_t)sp.k ? rlen - sp.k + 1 : 0;
    // Positions of this tile: its windows' starts, and for the record's
    // last tile the candidate positions past them.
    uint64_t end = tile.w0 + tile.nw;
    if (end == windows && extra) end = min(end + extra, rlen >= (uint64_t)len ? rlen - len + 1 : 0);
    uint64_t* out = slots + (uint64_t)t * kStrobeSlot;
    uint32_t count = 0;
    for (uint64_t q0 = tile.w0; q0 < end; q0 += 32) {
      const uint64_t q = q0 + lane;
      bool keep = false;
      uint64_t key = 0;
      if (q < end && is_anchor(rb + q)) {
        const uint64_t h = __ldg(hashes + rb + q);
        uint64_t partner = h;
        int fewest = 9;
        for (uint64_t d = 1; d <= dmax; ++d) {
          const uint64_t c = q + d;
          // The record ends, or a base of the run does: no more partners.
          if (c + len > rlen || (bv.pv.inv32(rb + c + len - 1) & 1u)) break;
          if (d < dmin || !is_anchor(rb + c)) continue;
          const uint64_t hc = __ldg(hashes + rb + c);
          const int x = __popcll((h ^ hc) & 0xFFull);
          if (x < fewest) {
            fewest = x;
            partner = hc;
            if (!fewest) break;
          }
        }
        key = (h >> 1) + (partner >> 1);
        keep = true;
      }
      count = warp_append(out, count, keep, key, lane);
    }
    if (lane == 0) slot_count[t] = count;
  }
}

}  // namespace zx
