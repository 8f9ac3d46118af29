// Seed extraction on sm_100a: one warp per tile of k-windows of one record.
//
// Input is the batch packed by pack_kernel: packed[w] holds bases 32w..32w+31
// as 2-bit codes, first base in the two most significant bits; invalid[w] has
// bit i set when base 32w+i is not A/C/G/T (either case). Every kernel below
// reproduces the reference extractors bit for bit:
//   canonical k-mers, k <= 32 ......... src/lib.rs:645-681
//   polynomial k-mer hashes, k > 32 ... src/lib.rs:683-731
//   open-closed mod-minimizers ........ utils/ocm-minimizers/src/implementation.rs:89-346
//   modimizers ........................ src/lib.rs:796-806
//   findere s-mers .................... src/lib.rs:632-640, src/findere.rs:178-233
#pragma once
#include <stdint.h>

#include "../zx_hash.h"
#include "types.cuh"

namespace zx {

// Byte -> 2-bit code, 4 for anything that is not A/C/G/T.
__device__ __forceinline__ uint32_t dev_code(uint8_t b) { return encode_base(b); }

// K0: ASCII bases -> packed 2-bit words + invalid masks. Word w covers bases
// 32w..32w+31; positions past `n` are marked invalid.
__device__ __forceinline__ void pack_word(const uint8_t* __restrict__ bases, uint64_t n,
                                          uint64_t* __restrict__ packed,
                                          uint32_t* __restrict__ invalid, uint64_t w) {
  {
    uint64_t base = w * 32, v = 0;
    uint32_t inv = 0;
    if (base + 32 <= n && (((uintptr_t)(bases + base)) & 15) == 0) {
      uint4 a = *reinterpret_cast<const uint4*>(bases + base);
      uint4 b = *reinterpret_cast<const uint4*>(bases + base + 16);
      uint32_t x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        uint32_t c = dev_code((uint8_t)(x[i >> 2] >> (8 * (i & 3))));
        inv |= (uint32_t)(c > 3) << i;
        v |= (uint64_t)(c & 3) << (62 - 2 * i);
      }
    } else {
      for (int i = 0; i < 32; ++i) {
        uint32_t c = base + i < n ? dev_code(bases[base + i]) : 4;
        inv |= (uint32_t)(c > 3) << i;
        v |= (uint64_t)(c & 3) << (62 - 2 * i);
      }
    }
    packed[w] = v;
    invalid[w] = inv;
  }
}

__global__ void pack_kernel(const uint8_t* __restrict__ bases, uint64_t n,
                            uint64_t* __restrict__ packed, uint32_t* __restrict__ invalid,
                            uint64_t words) {
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < words;
       w += (uint64_t)gridDim.x * blockDim.x)
    pack_word(bases, n, packed, invalid, w);
}

struct PackedView {
  const uint64_t* packed;
  const uint32_t* invalid;

  // The 32 bases starting at global position p, first base most significant.
  __device__ __forceinline__ uint64_t bits32(uint64_t p) const {
    uint64_t w = p >> 5;
    uint32_t r = (uint32_t)(p & 31);
    uint64_t hi = __ldg(packed + w);
    if (!r) return hi;
    uint64_t lo = __ldg(packed + w + 1);
    return (hi << (2 * r)) | (lo >> (64 - 2 * r));
  }
  // Invalid flags of the 32 bases starting at p (bit i = base p+i).
  __device__ __forceinline__ uint32_t inv32(uint64_t p) const {
    uint64_t w = p >> 5;
    uint32_t r = (uint32_t)(p & 31);
    uint64_t m = (uint64_t)__ldg(invalid + w) | ((uint64_t)__ldg(invalid + w + 1) << 32);
    return (uint32_t)(m >> r);
  }
  // True when bases [p, p+len) are all A/C/G/T.
  __device__ __forceinline__ bool valid(uint64_t p, uint32_t len) const {
    while (len >= 32) {
      if (inv32(p)) return false;
      p += 32;
      len -= 32;
    }
    return len == 0 || (inv32(p) & ((1u << len) - 1)) == 0;
  }
  __device__ __forceinline__ uint32_t code(uint64_t p) const {
    return (uint32_t)(__ldg(packed + (p >> 5)) >> (62 - 2 * (p & 31))) & 3;
  }
  // Forward 2-bit value of the len <= 32 bases at p.
  __device__ __forceinline__ uint64_t fwd(uint64_t p, int len) const {
    uint64_t v = bits32(p);
    return len == 32 ? v : v >> (64 - 2 * len);
  }
  // Bases with code >= 2 (G or T) among the len bases at p.
  __device__ __forceinline__ uint32_t gt_count(uint64_t p, uint32_t len) const {
    uint32_t c = 0;
    while (len >= 32) {
      c += __popcll(bits32(p) & 0xAAAAAAAAAAAAAAAAull);
      p += 32;
      len -= 32;
    }
    if (len) c += __popcll((bits32(p) >> (64 - 2 * len)) & 0xAAAAAAAAAAAAAAAAull);
    return c;
  }
};

// Reverse complement of a len-base forward value (len <= 32).
__device__ __forceinline__ uint64_t revcomp(uint64_t fwd, int len) {
  uint64_t y = __brevll(~fwd);
  y = ((y >> 1) & 0x5555555555555555ull) | ((y & 0x5555555555555555ull) << 1);
  return len == 32 ? y : y >> (64 - 2 * len);
}

__device__ __forceinline__ uint64_t canonical_at(const PackedView& pv, uint64_t p, int len) {
  uint64_t f = pv.fwd(p, len), r = revcomp(f, len);
  return f < r ? f : r;
}

// Appends the keys selected by `keep` (one per lane, order = lane order) to
// the warp buffer; returns the new count (warp-uniform).
__device__ __forceinline__ uint32_t warp_append(uint64_t* buf, uint32_t count, bool keep,
                                                uint64_t key, int lane) {
  uint32_t ballot = __ballot_sync(0xFFFFFFFFu, keep);
  if (keep) buf[count + __popc(ballot & ((1u << lane) - 1))] = key;
  return count + __popc(ballot);
}

// Canonical k-mers (k <= 32) of windows [w0, w0+nw) of the record starting at
// global base `rb`: one window per lane per round, in window order.
__device__ __forceinline__ uint32_t tile_kmers_short(const PackedView& pv, uint64_t rb, uint32_t w0,
                                                     uint32_t nw, int k, bool modimizer,
                                                     uint64_t seed, uint64_t sampling,
                                                     uint64_t* buf, int lane) {
  uint32_t count = 0;
  for (uint32_t i0 = 0; i0 < nw; i0 += 32) {
    uint32_t i = i0 + lane;
    bool keep = false;
    uint64_t key = 0;
    if (i < nw) {
      uint64_t p = rb + w0 + i;
      if (pv.valid(p, k)) {
        key = canonical_at(pv, p, k);
        keep = !modimizer || mixsplit(key, seed) % sampling == 0;
      }
    }
    count = warp_append(buf, count, keep, key, lane);
  }
  return count;
}

// Polynomial hashes (k > 32): each lane rolls over a contiguous run of
// windows, restarting with a direct evaluation after invalid bases. Lane runs
// are staged in `tmp` (nw entries) and concatenated in lane order.
__device__ __forceinline__ uint32_t tile_kmers_long(const PackedView& pv, uint64_t rb, uint32_t w0,
                                                    uint32_t nw, int k, const LongKmerConsts& lk,
                                                    bool modimizer, uint64_t seed,
                                                    uint64_t sampling, uint64_t* buf,
                                                    uint64_t* tmp, int lane) {
  const uint32_t per = (nw + 31) / 32;
  const uint32_t a = min(nw, per * lane), e = min(nw, a + per);
  uint32_t n = 0;
  bool live = false;
  uint64_t f = 0, r = 0;
  for (uint32_t i = a; i < e; ++i) {
    uint64_t p = rb + w0 + i;
    if (live) {
      if (pv.inv32(p + k - 1) & 1) {
        live = false;
        continue;
      }
      uint64_t o = pv.code(p - 1), c = pv.code(p + k - 1);
      f = (f - (o + 1) * lk.power) * kLongKmerBase + (c + 1);
      r = (r - (4 - o)) * lk.inverse + (4 - c) * lk.power;
    } else {
      if (!pv.valid(p, k)) continue;
      live = true;
      f = 0;
      r = 0;
      uint64_t wgt = 1;
      for (int q = 0; q < k; ++q) {
        uint64_t c = pv.code(p + q);
        f = f * kLongKmerBase + (c + 1);
        r += (4 - c) * wgt;
        wgt *= kLongKmerBase;
      }
    }
    uint64_t key = splitmix64((f < r ? f : r) ^ lk.domain);
    if (!modimizer || mixsplit(key, seed) % sampling == 0) tmp[a + n++] = key;
  }
  uint32_t incl = n;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= d) incl += v;
  }
  uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  for (uint32_t j = 0; j < n; ++j) buf[incl - n + j] = tmp[a + j];
  __syncwarp();
  return total;
}

// ---- findere s-mers ----------------------------------------------------------
// The canonical s-mer (s = klen bases) at every position w0 + i, i < npos, of
// the record starting at global base rb, by position: keys[i], and bit i % 32
// of valid[i / 32] set when its s bases are all A/C/G/T (scan_canonical_kmers
// per ACGT run, lib.rs:645-731, as findere scans them, findere.rs:178-233).
// k > 32 uses the polynomial hash, each lane rolling over a contiguous range.
__device__ __forceinline__ void tile_smers(const PackedView& pv, uint64_t rb, uint32_t w0,
                                           uint32_t npos, int s, const LongKmerConsts& lk,
                                           uint64_t* keys, uint32_t* valid, int lane) {
  if (s <= 32) {
    for (uint32_t i0 = 0; i0 < npos; i0 += 32) {
      const uint32_t i = i0 + lane;
      bool ok = false;
      if (i < npos) {
        const uint64_t p = rb + w0 + i;
        ok = pv.valid(p, s);
        if (ok) keys[i] = canonical_at(pv, p, s);
      }
      const uint32_t bits = __ballot_sync(0xFFFFFFFFu, ok);
      if (lane == 0) valid[i0 >> 5] = bits;
    }
    __syncwarp();
    return;
  }
  for (uint32_t w = lane; w < (npos + 31) / 32; w += 32) valid[w] = 0;
  __syncwarp();
  const uint32_t per = (npos + 31) / 32;
  const uint32_t a = min(npos, per * lane), e = min(npos, a + per);
  bool live = false;
  uint64_t f = 0, r = 0;
  for (uint32_t i = a; i < e; ++i) {
    const uint64_t p = rb + w0 + i;
    if (live) {
      if (pv.inv32(p + s - 1) & 1) {
        live = false;
        continue;
      }
      const uint64_t o = pv.code(p - 1), c = pv.code(p + s - 1);
      f = (f - (o + 1) * lk.power) * kLongKmerBase + (c + 1);
      r = (r - (4 - o)) * lk.inverse + (4 - c) * lk.power;
    } else {
      if (!pv.valid(p, s)) continue;
      live = true;
      f = 0;
      r = 0;
      uint64_t wgt = 1;
      for (int q = 0; q < s; ++q) {
        const uint64_t c = pv.code(p + q);
        f = f * kLongKmerBase + (c + 1);
        r += (4 - c) * wgt;
        wgt *= kLongKmerBase;
      }
    }
    keys[i] = splitmix64((f < r ? f : r) ^ lk.domain);
    atomicOr(valid + (i >> 5), 1u << (i & 31));
  }
  __syncwarp();
}

// ---- open-closed mod-minimizers -------------------------------------------
struct Rank16 {
  uint64_t hash;
  uint32_t cls;
  uint16_t left, right;  // tile-local anchor indices of the tied extremes
};

__device__ __forceinline__ bool rank_lt(const Rank16& a, const Rank16& b) {
  return a.cls != b.cls ? a.cls < b.cls : a.hash < b.hash;
}
// a lies left of b; equal ranks keep the leftmost and rightmost positions.
__device__ __forceinline__ Rank16 rank_min(const Rank16& a, const Rank16& b) {
  if (rank_lt(a, b)) return a;
  if (rank_lt(b, a)) return b;
  Rank16 r = a;
  r.right = b.right;
  return r;
}

constexpr uint32_t kOcmTile = 256;  // windows per minimizer tile

// Selected minimizer positions of windows w0 - 1 .. w0 + nw - 1 (nw <=
// kOcmTile): pos[i] is window w0 - 1 + i's selected m-mer, as an index j
// into the tile's anchors (record position w0 - 1 + j), or ~0 for an invalid
// window. pre/suf hold at least nw + W entries each; inner is the
// 4^s-entry inner hash table; pos holds nw + 1 entries.
__device__ void tile_ocm_select(const PackedView& pv, uint64_t rb, uint32_t w0, uint32_t nw,
                                const SeedParams& sp, const uint64_t* inner, Rank16* pre,
                                Rank16* suf, uint32_t* pos, int lane) {
  const int k = sp.k, t = sp.ocm.t, s = sp.ocm.s, w = sp.ocm.w;
  const uint32_t W = (uint32_t)(k - t + 1);
  // Anchor index j <-> anchor position w0 - 1 + j (record coordinates).
  const uint32_t anchors = nw + W;
  const uint64_t smask = (1ull << (2 * s)) - 1;
  for (uint32_t j = lane; j < anchors; j += 32) {
    Rank16 rk;
    rk.left = rk.right = (uint16_t)j;
    rk.cls = 3;
    rk.hash = ~0ull;
    if (w0 + j >= 1) {
      uint64_t p = rb + w0 + j - 1;
      uint64_t tf = pv.fwd(p, t);
      uint64_t lo = ~0ull, h0 = 0, hm = 0, hl = 0;
      for (int q = 0; q <= t - s; ++q) {
        uint64_t h = inner[(tf >> (2 * (t - s - q))) & smask];
        lo = h < lo ? h : lo;
        if (q == 0) h0 = h;
        if (q == (t - s) / 2) hm = h;
        if (q == t - s) hl = h;
      }
      rk.cls = hm == lo ? 0 : ((h0 == lo || hl == lo) ? 1 : 2);
      uint64_t tr = revcomp(tf, t);
      rk.hash = mixsplit(tf < tr ? tf : tr, sp.seed);
    }
    suf[j] = rk;
  }
  __syncwarp();
  // Block prefix / suffix minima over blocks of W anchors.
  for (uint32_t b0 = lane * W; b0 < anchors; b0 += 32 * W) {
    uint32_t b1 = min(anchors, b0 + W);
    Rank16 acc = suf[b0];
    pre[b0] = acc;
    for (uint32_t j = b0 + 1; j < b1; ++j) {
      acc = rank_min(acc, suf[j]);
      pre[j] = acc;
    }
    for (uint32_t j = b1 - 1; j-- > b0;) suf[j] = rank_min(suf[j], suf[j + 1]);
  }
  __syncwarp();
  // Selected positions of windows w0-1 .. w0+nw-1 (index i <-> window w0-1+i).
  for (uint32_t i = lane; i <= nw; i += 32) {
    uint32_t sel = 0xFFFFFFFFu;
    if (w0 + i >= 1) {
      uint64_t st = rb + w0 + i - 1;
      if (pv.valid(st, k)) {
        Rank16 best = (i % W == 0) ? suf[i] : rank_min(suf[i], pre[i + W - 1]);
        uint32_t anchor = pv.gt_count(st, k) > (uint32_t)k / 2 ? best.right : best.left;
        sel = i + (anchor - i) % (uint32_t)w;  // anchor index offset from window index
      }
    }
    pos[i] = sel;
  }
  __syncwarp();
}

// Minimizers of windows [w0, w0+nw) (nw <= kOcmTile), buffers as for
// tile_ocm_select. Emits in window order, dropping repeats of the previous
// window's selected position within a run.
__device__ uint32_t tile_ocm(const PackedView& pv, uint64_t rb, uint32_t w0, uint32_t nw,
                             const SeedParams& sp, const uint64_t* inner, Rank16* pre,
                             Rank16* suf, uint32_t* pos, uint64_t* buf, int lane) {
  const int m = sp.m;
  tile_ocm_select(pv, rb, w0, nw, sp, inner, pre, suf, pos, lane);
  uint32_t count = 0;
  for (uint32_t i0 = 1; i0 <= nw; i0 += 32) {
    uint32_t i = i0 + lane;
    bool keep = false;
    uint64_t key = 0;
    if (i <= nw && pos[i] != 0xFFFFFFFFu && pos[i] != pos[i - 1]) {
      keep = true;
      key = canonical_at(pv, rb + w0 - 1 + pos[i], m);
    }
    count = warp_append(buf, count, keep, key, lane);
  }
  return count;
}

// Full-m-mer special case (k == m): every canonical m-mer.
__device__ __forceinline__ uint32_t tile_ocm_full(const PackedView& pv, uint64_t rb, uint32_t w0,
                                                  uint32_t nw, int m, uint64_t* buf, int lane) {
  return tile_kmers_short(pv, rb, w0, nw, m, false, 0, 1, buf, lane);
}

}  // namespace zx
