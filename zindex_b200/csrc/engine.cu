// Host runtime of the GPU query path (see engine.h).
//
// Index loading restates Index::load_mode (src/power_merge/storage.rs:
// 2273-2707) for fingerprint-first banks: the manifest is validated, every
// bank stream is decoded (bank_io.rs:235-292) and checked against its header
// (validate_bank_header, storage.rs:2208-2231), and the recovery file is
// decoded (abandoned_io.rs:4-130) into the device directory described in
// kernels/device_index.cuh. All banks stay resident ("--query-memory all",
// storage.rs:3745-3766): HBM holds the whole filter payload.
#include "engine.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "kernels/query_kernels.cuh"
#include "kernels/record_hits.cuh"
#include "kernels/strobes.cuh"
#include "kernels/wide_probe.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>

#include "host/error.h"
#include "host/zstd_io.h"
#include "zx_hash.h"

namespace zx {

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) raise(kECuda, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

uint64_t round_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

template <class T>
void dev_alloc(T** p, uint64_t count, const char* what) {
  *p = nullptr;
  if (!count) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    raise(kENoMem, std::string("device allocation failed for ") + what + ": " +
                       cudaGetErrorString(e));
  }
}

template <class T>
void host_alloc(T** p, uint64_t count) {
  *p = nullptr;
  if (!count) count = 1;
  cuda_check(cudaMallocHost((void**)p, count * sizeof(T)), "cudaMallocHost");
}

__global__ void repack_rows_kernel(const uint8_t* __restrict__ src, uint64_t rows,
                                   uint32_t row_bytes, uint32_t stride, uint8_t* __restrict__ dst) {
  uint64_t total = rows * stride;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t r = i / stride;
    uint32_t c = (uint32_t)(i % stride);
    dst[i] = c < row_bytes ? src[r * row_bytes + c] : 0;
  }
}

// Legacy interleaved rows (ZORPOW1: group g's fingerprint in the low b bits of
// its field at offset_g, membership bits after it; storage.rs:2864-2914) moved
// into the device's fingerprint-first rows (fingerprint at g*b, membership at
// G*b + offset_g - g*b; storage.rs:1721-1754). The move is a fixed bit
// permutation of the row, and XOR commutes with it, so the query kernels read
// legacy indexes unchanged. One warp per row; fields are ORed into the
// zeroed destination row.
__global__ void repack_legacy_kernel(const uint8_t* __restrict__ src, uint64_t rows,
                                     uint32_t row_bytes, uint32_t stride,
                                     const uint2* __restrict__ fields, uint32_t groups, int b,
                                     uint8_t* __restrict__ dst) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t r = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); r < rows;
       r += warps) {
    const uint8_t* in = src + r * row_bytes;
    uint32_t* out = reinterpret_cast<uint32_t*>(dst + r * stride);
    for (uint32_t w = lane; w < stride / 4; w += 32) out[w] = 0;
    __syncwarp();
    auto put = [&](uint64_t bit, uint32_t width, uint64_t v) {
      while (width) {
        const uint32_t sh = (uint32_t)(bit & 31), n = min(width, 32 - sh);
        const uint32_t part = (uint32_t)(v & ((1ull << n) - 1));
        if (part) atomicOr(out + (bit >> 5), part << sh);
        v >>= n;
        bit += n;
        width -= n;
      }
    };
    for (uint32_t g = lane; g < groups; g += 32) {
      const uint2 f = fields[g];  // {offset, width}
      put((uint64_t)g * b, (uint32_t)b, row_bits(in, f.x, (uint32_t)b));
      if (f.y > (uint32_t)b)
        put((uint64_t)groups * b + f.x - (uint64_t)g * b, f.y - b, row_bits(in, f.x + b, f.y - b));
    }
    __syncwarp();
  }
}

using FusedFn = void (*)(const DevIndex*, BatchView, SeedParams, QueryLaunch, uint32_t*, uint64_t*,
                        unsigned long long*, uint32_t*);
using ExtractFn = void (*)(BatchView, SeedParams, uint64_t*, uint32_t*, int);

template <int MINB, int VARIANT>
FusedFn fused_mode(int mode) {
  switch (mode) {
    case 1: return fused_query_kernel<1, MINB, VARIANT>;
    case 2: return fused_query_kernel<2, MINB, VARIANT>;
    default: return fused_query_kernel<0, MINB, VARIANT>;
  }
}

// Kernel variant: seed mode x register budget (2 or 3 resident 256-thread
// blocks per SM) x gather (register teams with per-hit counter updates,
// staged ring, or register teams with bit-plane counters).
FusedFn fused_for(int mode, const QueryLaunch& l) {
  // Findere has one form: the row-index probe with per-colour position masks.
  if (mode == 3) return l.min_blocks == 3 ? fused_query_kernel<3, 3, 2> : fused_query_kernel<3, 2, 2>;
  // Probe of seeds extracted beforehand (split minimizer queries): row-index form only.
  if (mode == 4)
    return l.min_blocks == 1   ? fused_query_kernel<4, 1, 2>
           : l.min_blocks == 3 ? fused_query_kernel<4, 3, 2>
                               : fused_query_kernel<4, 2, 2>;
  const int v = l.stage_bytes > 0 ? 1 : (l.planes ? 2 : 0);
  // One resident block per SM: the row-index form with the chunk pipeline.
  if (l.min_blocks == 1 && v == 2) return fused_mode<1, 2>(mode);
  if (l.min_blocks == 3) {
    if (v == 1) return fused_mode<3, 1>(mode);
    return v == 2 ? fused_mode<3, 2>(mode) : fused_mode<3, 0>(mode);
  }
  if (v == 1) return fused_mode<2, 1>(mode);
  return v == 2 ? fused_mode<2, 2>(mode) : fused_mode<2, 0>(mode);
}

// Small batches with at most this many colours count with global atomics
// into the caller's counters (flushed planes make them rare).
constexpr size_t kSmallColors = 1024;

using WideFn = void (*)(const DevIndex*, const ColorLoc*, const uint64_t*,
                       const unsigned long long*, int, uint32_t, uint32_t*, uint64_t*,
                       unsigned long long*, WideRound);
using DenseExtractFn = void (*)(BatchView, SeedParams, uint64_t*, unsigned long long*, int,
                                WideRound);

// Wide-row probe variant: J chunks per thread, S seeds per step, HQ rows
// loaded per seed and chunk (16 loads in flight per thread).
// Blocks of up to 288 threads (9 warps) keep rows a few partial chunks over
// 256 or 512 at one or two chunks per thread; their register budget (96 at
// two blocks per SM) holds 16 loads in flight for one chunk, 8 for two.
WideFn wide_fn(int J, int HQ, int T) {
  if (J == 1)
    return HQ == 8 ? wide_probe_kernel<1, 2, 8, 2, 288> : wide_probe_kernel<1, 4, 4, 2, 288>;
  if (J == 2 && T > 256)
    return HQ == 8 ? wide_probe_kernel<2, 1, 8, 2, 288> : wide_probe_kernel<2, 1, 4, 2, 288>;
  if (J == 2) return HQ == 8 ? wide_probe_kernel<2, 1, 8, 2> : wide_probe_kernel<2, 2, 4, 2>;
  if (J == 3) return wide_probe_kernel<3, 1, 4, 2>;
  return wide_probe_kernel<4, 1, 4, 2>;
}

DenseExtractFn dense_extract_for(int mode) {
  switch (mode) {
    case 1: return extract_dense_kernel<1>;
    case 2: return extract_dense_kernel<2>;
    default: return extract_dense_kernel<0>;
  }
}

ExtractFn extract_for(int mode) {
  switch (mode) {
    case 1: return extract_kernel<1>;
    case 2: return extract_kernel<2>;
    default: return extract_kernel<0>;
  }
}

// ---- homopolymer compression of a batch (lib.rs:211-222, applied per ACGT
// run by scan_index_features, lib.rs:574-589): inside a run of A/C/G/T a base
// equal to the one before it is dropped; other bytes are kept as separators.
// Offsets are not trusted here (the tile planner reports bad ones): a start
// past the bases is ignored and positions are read at min(offset, nbases).
__global__ void hp_mark_starts_kernel(const uint64_t* __restrict__ offsets, uint64_t records,
                                      uint64_t nbases, uint32_t* __restrict__ starts) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < records;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = offsets[r];
    if (p < nbases) atomicOr(starts + (p >> 5), 1u << (p & 31));
  }
}

__global__ void hp_keep_kernel(const uint8_t* __restrict__ bases, uint64_t nbases,
                               const uint32_t* __restrict__ starts, uint32_t* __restrict__ keep) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= nbases;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t k = 0;
    if (i < nbases) {
      const uint32_t c = encode_base(bases[i]);
      const bool start = (starts[i >> 5] >> (i & 31)) & 1u;
      k = c > 3 || start || i == 0 || encode_base(bases[i - 1]) != c;
    }
    keep[i] = k;
  }
}

__global__ void hp_compact_kernel(const uint8_t* __restrict__ bases, uint64_t nbases,
                                  const uint32_t* __restrict__ pos, uint8_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nbases;
       i += (uint64_t)gridDim.x * blockDim.x)
    if (pos[i + 1] != pos[i]) out[pos[i]] = bases[i];
}

__global__ void hp_offsets_kernel(const uint64_t* __restrict__ offsets, uint64_t records,
                                  uint64_t nbases, const uint32_t* __restrict__ pos,
                                  uint64_t* __restrict__ out) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r <= records;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t o = offsets[r];
    // An offset past the bases stays invalid for the tile planner.
    out[r] = o <= nbases ? pos[o] : ~0ull;
  }
}

// offsets[i] -= base (chunk-relative record offsets after a raw copy).
__global__ void rebase_offsets_kernel(uint64_t* __restrict__ offsets, uint64_t n, uint64_t base) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    offsets[i] -= base;
}

uint64_t le64(const uint8_t* p) {
  uint64_t v = 0;
  for (int i = 7; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}

struct RecoveryRecords {
  std::vector<uint32_t> hashes;
  std::vector<uint64_t> starts;  // hashes + 1
  std::vector<uint32_t> origins;
};

// AbandonedReader (src/power_merge/abandoned_io.rs:4-130) with its checks.
RecoveryRecords read_recovery(const std::string& dir, const Manifest& m) {
  RecoveryRecords r;
  std::vector<uint8_t> raw = read_file_bytes(dir + "/abandoned.zormap.zst");
  std::vector<uint8_t> d = zstd_decode_all(raw.data(), raw.size());
  check_format(d.size() >= 8, "invalid abandoned map magic");
  bool delta = !memcmp(d.data(), "ZORABN2\0", 8);
  check_format(delta || !memcmp(d.data(), "ZORABN1\0", 8), "invalid abandoned map magic");
  size_t p = 8;
  auto var = [&]() -> uint32_t {
    uint32_t v = 0;
    for (int shift = 0; shift <= 28; shift += 7) {
      check_format(p < d.size(), "truncated abandoned map");
      uint8_t byte = d[p++];
      check_format(shift != 28 || byte <= 15, "abandoned variable integer overflow");
      v |= (uint32_t)(byte & 127) << shift;
      if (!(byte & 128)) return v;
    }
    raise(kEFormat, "abandoned variable integer overflow");
  };
  auto u32 = [&]() -> uint32_t {
    check_format(p + 4 <= d.size(), "truncated abandoned map");
    uint32_t v = (uint32_t)d[p] | ((uint32_t)d[p + 1] << 8) | ((uint32_t)d[p + 2] << 16) |
                 ((uint32_t)d[p + 3] << 24);
    p += 4;
    return v;
  };
  const uint64_t colors = m.colors.size();
  r.hashes.reserve(m.abandoned_hashes);
  r.starts.reserve(m.abandoned_hashes + 1);
  r.origins.reserve(m.abandoned_origins);
  uint32_t prev = 0;
  for (uint64_t rec = 0; rec < m.abandoned_hashes; ++rec) {
    uint32_t h;
    if (delta) {
      uint32_t dh = var();
      check_format(rec == 0 || dh != 0, "unsorted/duplicate abandoned hashes");
      check_format((uint64_t)prev + dh <= 0xFFFFFFFFull, "abandoned hash delta overflow");
      h = prev + dh;
    } else {
      h = u32();
    }
    check_format(rec == 0 || prev < h, "unsorted/duplicate abandoned hashes");
    prev = h;
    uint32_t count = delta ? var() : u32();
    check_format(count > 0 && count <= colors, "invalid abandoned origin count");
    check_format(count <= m.abandoned_origins - r.origins.size(),
                 "abandoned origins exceed manifest");
    r.hashes.push_back(h);
    r.starts.push_back(r.origins.size());
    uint32_t po = 0;
    for (uint32_t c = 0; c < count; ++c) {
      uint32_t o;
      if (delta) {
        uint32_t dd = var();
        check_format(c == 0 || dd != 0, "duplicate abandoned origins");
        check_format((uint64_t)po + dd <= 0xFFFFFFFFull, "abandoned origin delta overflow");
        o = po + dd;
      } else {
        o = u32();
      }
      check_format(o < colors, "invalid abandoned dataset ID");
      check_format(c == 0 || o > po, "unsorted/duplicate abandoned origins");
      r.origins.push_back(o);
      po = o;
    }
  }
  check_format(r.origins.size() == m.abandoned_origins,
               "abandoned origin count differs from manifest");
  check_format(p == d.size(), "unexpected abandoned map data");
  r.starts.push_back(r.origins.size());
  return r;
}

}  // namespace

// ---- allocation-free query: scratch in a static device array ---------------
// For callers that cannot allocate device memory (see zx_query_device_noalloc
// in include/zindex.h). One 64 MiB array per GPU that loads the library, held
// until process exit; its device address is resolved once per device. The
// first kNoAllocErrorSlots words are error words: every engine that uses the
// entry point owns one of them (taken on its first call, returned when the
// engine is released), so one index's status never reports or clears
// another's. The batch scratch starts after them.
constexpr uint64_t kNoAllocScratchBytes = 64ull << 20;
constexpr uint32_t kNoAllocErrorSlots = 1024;
constexpr uint64_t kNoAllocErrorBytes = kNoAllocErrorSlots * 4;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[256] = {};
std::vector<bool> g_noalloc_slot_used[256];

// Device address of the static scratch on the current device (set-up on first
// use per device; this device must be current).
void* noalloc_scratch(int device) {
  check(device >= 0 && device < 256, kEInval, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
    g_noalloc_ptr[device] = p;
  }
  return g_noalloc_ptr[device];
}

// Takes a free error slot of this device and clears its word (synchronously:
// this runs once per engine, on its first allocation-free call).
int noalloc_take_slot(int device) {
  uint32_t* words = static_cast<uint32_t*>(noalloc_scratch(device));
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  auto& used = g_noalloc_slot_used[device];
  if (used.empty()) used.assign(kNoAllocErrorSlots, false);
  for (uint32_t i = 0; i < kNoAllocErrorSlots; ++i)
    if (!used[i]) {
      cuda_check(cudaMemset(words + i, 0, 4), "memset");
      used[i] = true;
      return (int)i;
    }
  raise(kENoMem, "more than " + std::to_string(kNoAllocErrorSlots) +
                     " open indexes use the allocation-free query on this device");
}

void noalloc_return_slot(int device, int slot) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (device >= 0 && device < 256 && slot >= 0 && (size_t)slot < g_noalloc_slot_used[device].size())
    g_noalloc_slot_used[device][slot] = false;
}
}  // namespace

void Engine::query_device_noalloc(const uint8_t* bases, uint64_t nbases, const uint64_t* offsets,
                                  uint64_t records, bool recover, uint64_t* counts,
                                  unsigned long long* total, cudaStream_t s) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  check_not_strobes();
  check(records < (1ull << 31), kEInval, "too many records for one query");
  check(!m_.homopolymer_compression, kEUnsupported,
        "the allocation-free query does not run homopolymer compression (the compressed batch "
        "needs scratch of its own): use zx_query_device");
  uint8_t* base = static_cast<uint8_t*>(noalloc_scratch(device_));
  if (noalloc_slot_ < 0) noalloc_slot_ = noalloc_take_slot(device_);
  // This engine's error word. It is never cleared per call: a bit set by an
  // earlier asynchronous call stays until zx_query_status reads it.
  uint32_t* err = reinterpret_cast<uint32_t*>(base) + noalloc_slot_;
  base += kNoAllocErrorBytes;
  const uint64_t words = nbases / 32 + 2;
  const uint64_t tiles = nbases / kTileWindows + nbases / kFindereTask + records + 16;
  // Register gather, colour counts added straight into the caller's counters.
  QueryLaunch l = fused_launch(launch_);
  l.smem_counters = 0;
  l.stage_bytes = 0;
  l.blocks = 0;
  l.split = 0;
  const size_t smem = fused_smem_bytes(l);
  FusedFn fn = fused_for(sp_.mode, l);
  cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute");
  int per_sm = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, l.warps * 32, smem),
             "occupancy");
  uint64_t want = (tiles + l.warps - 1) / l.warps;
  int blocks = (int)std::min<uint64_t>((uint64_t)std::max(1, per_sm) * sms_, std::max<uint64_t>(want, 1));
  l.blocks = blocks;
  const uint64_t fstate_bytes =
      m_.index_mode == kFindere && m_.colors.size() > kFindereSmemColors
          ? (uint64_t)blocks * l.warps * 2 * m_.colors.size() * 4
          : 0;
  // Scratch layout, every region 256-byte aligned.
  size_t scan_bytes = 0;
  cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t*)nullptr,
                                           (uint32_t*)nullptr, (int)(records + 1)),
             "scan size");
  uint64_t at = 0;
  auto carve = [&](uint64_t bytes) {
    uint64_t off = at;
    at = round_up(at + bytes, 256);
    return base + off;
  };
  uint64_t* packed = reinterpret_cast<uint64_t*>(carve(words * 8));
  uint32_t* invalid = reinterpret_cast<uint32_t*>(carve(words * 4));
  uint32_t* tile_counts = reinterpret_cast<uint32_t*>(carve((records + 1) * 4));
  uint32_t* tile_first = reinterpret_cast<uint32_t*>(carve((records + 1) * 4));
  Tile* tile_list = reinterpret_cast<Tile*>(carve(tiles * sizeof(Tile)));
  void* scan_tmp = carve(scan_bytes);
  uint32_t* fstate = fstate_bytes ? reinterpret_cast<uint32_t*>(carve(fstate_bytes)) : nullptr;
  if (at > kNoAllocScratchBytes - kNoAllocErrorBytes)
    raise(kEInval, "batch needs " + std::to_string(at) + " bytes of scratch; the allocation-free "
                   "query holds at most " + std::to_string(kNoAllocScratchBytes - kNoAllocErrorBytes) +
                   " bytes (about 0.4 byte per base + 28 bytes per record): split the batch");
  // The array keeps the previous call's contents: reset what must start at zero.
  if (fstate) cuda_check(cudaMemsetAsync(fstate, 0, fstate_bytes, s), "memset");
  cuda_check(cudaMemsetAsync(tile_counts + records, 0, 4, s), "memset");
  int grid = (int)std::min<uint64_t>((words + 255) / 256, (uint64_t)sms_ * 16);
  pack_kernel<<<std::max(grid, 1), 256, 0, s>>>(bases, nbases, packed, invalid, words);
  cuda_check(cudaGetLastError(), "pack_kernel");
  const int findere = m_.index_mode == kFindere;
  int rgrid = std::max(1, (int)std::min<uint64_t>((records + 255) / 256, (uint64_t)sms_ * 16));
  if (records) {
    count_tiles_kernel<<<rgrid, 256, 0, s>>>(offsets, records, nbases, span(), findere,
                                             tile_counts, err);
    cuda_check(cudaGetLastError(), "count_tiles_kernel");
  }
  size_t tmp = scan_bytes;
  cuda_check(cub::DeviceScan::ExclusiveSum(scan_tmp, tmp, tile_counts, tile_first,
                                           (int)(records + 1), s),
             "tile scan");
  if (records) {
    fill_tiles_kernel<<<rgrid, 256, 0, s>>>(offsets, records, nbases, span(), tile_first,
                                            tile_list);
    cuda_check(cudaGetLastError(), "fill_tiles_kernel");
  }
  BatchView bv{PackedView{packed, invalid}, offsets, tile_list, tile_first + records, fstate};
  fn<<<blocks, l.warps * 32, smem, s>>>(recover ? d_ix_rec_ : d_ix_norec_, bv, sp_, l, nullptr,
                                        counts, total, err);
  cuda_check(cudaGetLastError(), "fused_query_kernel");
}

Workspace::~Workspace() {
  release_graphs();
  void* dev[] = {bases,      offsets,  packed,    invalid,  tile_counts, tile_first,
                 tiles,      scan_tmp, partial,   counts,   total,       keys_out,
                 keys_count, error,    fstate,    hp_starts, hp_keep,    hp_pos,
                 hp_bases,   hp_offsets, hp_scan_tmp, seg_blocks, seg_tiles, seg_records,
                 rec_counts, rec_totals, rec_hits, rec_first, rec_scan_tmp, hit_colors,
                 hit_counts, split_keys, split_counts, wide_cursor, wide_keys2,
                 wide_seg_cursor, wide_round_first, wide_keys_alt[0], wide_keys_alt[1],
                 wide_hist[0], wide_hist[1], strobe_anchors, strobe_hashes, strobe_slots,
                 strobe_count};
  for (void* p : dev)
    if (p) cudaFree(p);
  void* host[] = {h_bases, h_offsets, h_counts, h_total, h_seg_blocks, h_seg_records};
  for (void* p : host)
    if (p) cudaFreeHost(p);
  if (seg_staged) cudaEventDestroy(seg_staged);
  for (cudaEvent_t e : {wide_fork, wide_ext[0], wide_ext[1], wide_probe[0], wide_probe[1]})
    if (e) cudaEventDestroy(e);
  if (aux_stream) cudaStreamDestroy(aux_stream);
  for (cudaEvent_t e : chunk_events) cudaEventDestroy(e);
  if (copy_stream) cudaStreamDestroy(copy_stream);
  if (stream) cudaStreamDestroy(stream);
}

void Workspace::release_graphs() {
  for (auto& g : graphs) cudaGraphExecDestroy(g.second);
  graphs.clear();
}

Engine::Engine(const std::string& dir, const OpenOptions& options) {
  // A failed load (corrupt bank, short file, no memory) returns every device
  // allocation made so far: the destructor does not run for a constructor
  // that throws.
  try {
    load(dir, options);
  } catch (...) {
    release();
    throw;
  }
}

Engine::~Engine() { release(); }

void Engine::release() {
  ws_.reset();
  cudaSetDevice(device_);
  if (noalloc_slot_ >= 0) {
    // The engine's calls are done with the slot once the device is idle.
    cudaDeviceSynchronize();
    noalloc_return_slot(device_, noalloc_slot_);
    noalloc_slot_ = -1;
  }
  if (ev_begin_) cudaEventDestroy(ev_begin_);
  if (ev_end_) cudaEventDestroy(ev_end_);
  ev_begin_ = ev_end_ = nullptr;
  for (void* p : allocations_) cudaFree(p);
  allocations_.clear();
  if (d_ix_rec_) cudaFree(d_ix_rec_);
  if (d_ix_norec_) cudaFree(d_ix_norec_);
  d_ix_rec_ = d_ix_norec_ = nullptr;
  if (d_color_loc_) cudaFree(d_color_loc_);
  d_color_loc_ = nullptr;
}

int Engine::span() const { return (int)m_.k; }

namespace {

// Bank pieces from the host ring to the device: straight into the resident
// rows when the padded stride equals the row (fingerprint-first banks of
// 16-byte multiple rows), else through a device stage and the repack kernel.
// One stream: a piece's copy and repack run in order; events tell the
// decoder when a ring slot may be rewritten.
struct UploadSink : PieceSink {
  static constexpr int kSlots = 6;
  cudaStream_t stream = nullptr;
  cudaEvent_t done[kSlots] = {};
  bool pending[kSlots] = {};
  uint8_t* ring[kSlots] = {};
  uint8_t* stage[kSlots] = {};
  uint64_t piece_cap = 0;
  int sms = 1;
  // Current bank.
  uint8_t* dst = nullptr;
  uint64_t row_bytes = 0;
  uint32_t stride = 0;
  bool legacy = false;
  const uint2* fields = nullptr;
  uint32_t groups = 0;
  int bits = 0;

  void consume(int slot, uint64_t offset, uint64_t len) override {
    const uint64_t rows = len / row_bytes, r0 = offset / row_bytes;
    check(len % row_bytes == 0 && offset % row_bytes == 0, kEFormat, "bank piece splits a row");
    if (!legacy && stride == row_bytes) {
      cuda_check(cudaMemcpyAsync(dst + offset, ring[slot], len, cudaMemcpyHostToDevice, stream),
                 "bank upload");
    } else {
      cuda_check(cudaMemcpyAsync(stage[slot], ring[slot], len, cudaMemcpyHostToDevice, stream),
                 "bank upload");
      if (!legacy)
        repack_rows_kernel<<<sms * 8, 256, 0, stream>>>(stage[slot], rows, (uint32_t)row_bytes,
                                                        stride, dst + r0 * stride);
      else
        repack_legacy_kernel<<<sms * 8, 256, 0, stream>>>(stage[slot], rows, (uint32_t)row_bytes,
                                                          stride, fields, groups, bits,
                                                          dst + r0 * stride);
      cuda_check(cudaGetLastError(), "repack kernel");
    }
    cuda_check(cudaEventRecord(done[slot], stream), "cudaEventRecord");
    pending[slot] = true;
  }
  void drain(int slot) override {
    if (!pending[slot]) return;
    pending[slot] = false;
    cuda_check(cudaEventSynchronize(done[slot]), "bank upload");
  }
  ~UploadSink() {
    if (stream) cudaStreamSynchronize(stream);
    for (int i = 0; i < kSlots; ++i) {
      if (done[i]) cudaEventDestroy(done[i]);
      if (ring[i]) cudaFreeHost(ring[i]);
      if (stage[i]) cudaFree(stage[i]);
    }
    if (stream) cudaStreamDestroy(stream);
  }
};

}  // namespace

void Engine::load(const std::string& dir, const OpenOptions& options) {
  const auto t_start = std::chrono::steady_clock::now();
  m_ = load_manifest(dir);
  device_ = options.device;
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  cudaDeviceProp prop;
  cuda_check(cudaGetDeviceProperties(&prop, device_), "cudaGetDeviceProperties");
  sms_ = prop.multiProcessorCount;
  check(m_.classes.size() <= (size_t)kMaxClasses, kEUnsupported, "too many source classes");
  check(m_.index_mode != kFindere || m_.findere_z <= 224, kEUnsupported,
        "findere z above 224 is not supported by the GPU query path");

  // Seed parameters from the manifest (the query takes every setting from it).
  sp_.mode = m_.index_mode;
  sp_.k = (int)m_.k;
  sp_.m = (int)m_.minimizer_size;
  sp_.klen = m_.index_mode == kFindere ? (int)(m_.k - m_.findere_z) : (int)m_.k;
  sp_.seed = m_.seed;
  sp_.sampling = m_.modimizer_sampling;
  if (m_.index_mode == kMinimizers && m_.k != m_.minimizer_size)
    sp_.ocm = ocm_params((int)m_.k, (int)m_.minimizer_size);
  else
    sp_.ocm = OcmParams{1, (int)m_.minimizer_size, 1};
  if (sp_.klen > 32) sp_.lk = long_kmer_consts(sp_.klen);
  sp_.spaced = 0;
  if (m_.has_seed_pattern) {
    check_format(parse_spaced_seed(m_.seed_pattern.c_str(), &sp_.pattern), "invalid seed pattern");
    sp_.spaced = 1;
  }
  sp_.strobe_min = sp_.strobe_max = 0;
  if (m_.has_randstrobemers) {
    // Candidates of k-mer (k <= 32) or minimizer indexes; a minimizer window
    // can select up to w - 1 positions past a record's last window start.
    check((m_.index_mode == kKmers && m_.k <= 32) ||
              (m_.index_mode == kMinimizers && m_.minimizer_size <= 32 &&
               m_.k - m_.minimizer_size <= kStrobeExtra),
          kEUnsupported,
          "the GPU query path links randstrobemers over k-mers with k <= 32 and over "
          "minimizers with m <= 32 and k - m <= 64");
    check(m_.strobe_max < (1ull << 31), kEUnsupported, "randstrobemer distances below 2^31");
    sp_.strobe_min = (uint32_t)m_.strobe_min;
    sp_.strobe_max = (uint32_t)m_.strobe_max;
  }

  // Memory admission: banks (padded rows) + recovery directory.
  uint64_t need = 0;
  for (auto& b : m_.banks) need += b.slots * round_up(b.row_bytes(), 16);
  need += m_.abandoned_recovery ? m_.abandoned_hashes * 8 * 4 + m_.abandoned_origins * 4 : 0;
  size_t free_b = 0, total_b = 0;
  cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  uint64_t budget = options.hbm_budget
                        ? options.hbm_budget
                        : (free_b > (4ull << 30) ? free_b - (4ull << 30) : free_b / 2);
  if (need > budget)
    raise(kENoMem, "index needs " + std::to_string(need) + " bytes of HBM, budget is " +
                       std::to_string(budget));

  const int threads = options.threads > 0 ? options.threads
                                          : (int)std::max(1u, std::thread::hardware_concurrency());
  const int b = m_.fingerprint_bits;
  host_ix_ = DevIndex{};
  host_ix_.seed = m_.seed;
  host_ix_.classes = (uint32_t)m_.classes.size();
  host_ix_.colors = (uint32_t)m_.colors.size();
  host_ix_.hashes = m_.hashes;
  host_ix_.bits = b;

  // The recovery map is read and decoded on its own thread while the banks
  // stream in.
  RecoveryRecords rr;
  std::string rr_error;
  int rr_code = kOk;
  double recovery_s = 0;
  std::thread recovery_thread;
  if (m_.abandoned_recovery && m_.abandoned_hashes)
    recovery_thread = std::thread([&] {
      const auto t0 = std::chrono::steady_clock::now();
      try {
        rr = read_recovery(dir, m_);
      } catch (const Error& e) {
        rr_code = e.code;
        rr_error = e.what();
      } catch (const std::exception& e) {
        rr_code = kEFormat;
        rr_error = e.what();
      }
      recovery_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
  struct Joiner {
    std::thread& t;
    ~Joiner() {
      if (t.joinable()) t.join();
    }
  } joiner{recovery_thread};

  // Bank streaming: a pinned ring of 32 MiB pieces (row-aligned) filled by
  // the frame decoders and drained by asynchronous copies.
  const auto t_banks = std::chrono::steady_clock::now();
  UploadSink up;
  up.sms = sms_;
  uint64_t max_row = 16;
  for (auto& bm : m_.banks) max_row = std::max<uint64_t>(max_row, bm.row_bytes());
  up.piece_cap = std::max<uint64_t>(32ull << 20, max_row);
  cuda_check(cudaStreamCreateWithFlags(&up.stream, cudaStreamNonBlocking), "cudaStreamCreate");
  for (int i = 0; i < UploadSink::kSlots; ++i) {
    cuda_check(cudaEventCreateWithFlags(&up.done[i], cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaHostAlloc((void**)&up.ring[i], up.piece_cap, cudaHostAllocDefault),
               "pinned bank ring");
  }
  for (size_t ci = 0; ci < m_.classes.size(); ++ci) {
    const auto& banks = m_.classes[ci];
    const BankMeta& first = m_.banks[banks[0]];
    const uint64_t G = first.groups.size(), row_bytes = first.row_bytes();
    const uint32_t stride = (uint32_t)round_up(row_bytes, 16);
    DevClass& C = host_ix_.cls[ci];
    C.slots = first.slots;
    C.seg = m_.segment_for(first.slots);
    C.partitions = (uint32_t)banks.size();
    C.groups = (uint32_t)G;
    C.row_stride = stride;
    C.fp_chunks = (uint32_t)((first.lookup_bytes(b) + 15) / 16);
    // The kernels address rows by 32-bit row index (partition * slots + cell):
    // at least 16 bytes per row, so at most 64 GiB per class.
    check((uint64_t)banks.size() * first.slots * stride < (1ull << 36), kEUnsupported,
          "a source class larger than 64 GiB is not supported by the device layout");
    // Legacy banks: each group's {offset, width} for the row permutation.
    uint2* d_fields = nullptr;
    bool any_legacy = false;
    for (size_t bi : banks) any_legacy |= !m_.banks[bi].fingerprint_first;
    if (any_legacy) {
      std::vector<uint2> fields(G);
      for (uint64_t g = 0; g < G; ++g) {
        const GroupMeta& gm = first.groups[g];
        check_format(gm.width >= (uint64_t)b && gm.width - b <= 63 &&
                         gm.offset + gm.width <= first.row_bits,
                     "invalid group field in a legacy bank");
        fields[g] = make_uint2((uint32_t)gm.offset, (uint32_t)gm.width);
      }
      dev_alloc(&d_fields, G, "legacy field table");
      allocations_.push_back(d_fields);
      cuda_check(cudaMemcpy(d_fields, fields.data(), G * sizeof(uint2), cudaMemcpyHostToDevice),
                 "upload");
    }
    uint8_t* data = nullptr;
    dev_alloc(&data, (uint64_t)banks.size() * first.slots * stride, "bank payload");
    allocations_.push_back(data);
    resident_bytes_ += (uint64_t)banks.size() * first.slots * stride;
    for (size_t pi = 0; pi < banks.size(); ++pi) {
      const BankMeta& bm = m_.banks[banks[pi]];
      const uint64_t bytes = bm.slots * row_bytes;
      up.dst = data + pi * bm.slots * stride;
      up.row_bytes = row_bytes;
      up.stride = stride;
      up.legacy = !bm.fingerprint_first;
      up.fields = d_fields;
      up.groups = (uint32_t)G;
      up.bits = b;
      if (up.legacy || stride != row_bytes)
        for (int i = 0; i < UploadSink::kSlots; ++i)
          if (!up.stage[i]) dev_alloc(&up.stage[i], up.piece_cap, "bank staging");
      uint8_t header[40];
      const uint64_t piece = up.piece_cap / row_bytes * row_bytes;
      stream_bank(dir + "/" + bm.file, header, bytes, piece, up.ring, UploadSink::kSlots, threads,
                  up);
      check_format(!memcmp(header, bm.fingerprint_first ? "ZORPOW3\0" : "ZORPOW1\0", 8),
                   "invalid bank magic");
      check_format(le64(header + 8) == bm.slots && le64(header + 16) == bm.row_bits &&
                       le64(header + 24) == bm.groups.size() && le64(header + 32) == bytes,
                   "bank header differs from manifest");
    }
    // Group -> colour table, multi-member decode table.
    std::vector<uint32_t> gc(G), multi, members;
    for (uint64_t g = 0; g < G; ++g) {
      const GroupMeta& gm = first.groups[g];
      if (gm.members.size() == 1) {
        gc[g] = gm.members[0];
        continue;
      }
      check(gm.members.size() <= 63, kEFormat, "invalid membership width");
      gc[g] = kMultiGroup | (uint32_t)(multi.size() / 3);
      multi.push_back((uint32_t)(G * b + gm.offset - g * b));
      multi.push_back((uint32_t)gm.members.size());
      multi.push_back((uint32_t)members.size());
      members.insert(members.end(), gm.members.begin(), gm.members.end());
    }
    uint32_t *d_gc, *d_multi, *d_members;
    dev_alloc(&d_gc, gc.size(), "group table");
    dev_alloc(&d_multi, multi.size(), "multi table");
    dev_alloc(&d_members, members.size(), "member table");
    allocations_.push_back(d_gc);
    allocations_.push_back(d_multi);
    allocations_.push_back(d_members);
    cuda_check(cudaMemcpy(d_gc, gc.data(), gc.size() * 4, cudaMemcpyHostToDevice), "upload");
    if (!multi.empty()) {
      cuda_check(cudaMemcpy(d_multi, multi.data(), multi.size() * 4, cudaMemcpyHostToDevice),
                 "upload");
      cuda_check(cudaMemcpy(d_members, members.data(), members.size() * 4, cudaMemcpyHostToDevice),
                 "upload");
    }
    C.data = data;
    C.group_color = d_gc;
    C.multi = d_multi;
    C.members = d_members;
  }
  {
    // Colour -> (class, member index, group) for the wide probe's
    // recovered-origin point probes; a colour in no bank stays ~0.
    std::vector<ColorLoc> loc(std::max<size_t>(m_.colors.size(), 1), ColorLoc{0xFFFFFFFFu, 0u});
    for (size_t ci = 0; ci < m_.classes.size(); ++ci) {
      const BankMeta& first = m_.banks[m_.classes[ci][0]];
      for (uint64_t g = 0; g < first.groups.size(); ++g) {
        const auto& mem = first.groups[g].members;
        for (size_t mi = 0; mi < mem.size(); ++mi)
          if (mem[mi] < m_.colors.size())
            loc[mem[mi]] = ColorLoc{(uint32_t)ci | ((uint32_t)mi << 8), (uint32_t)g};
      }
    }
    dev_alloc(&d_color_loc_, loc.size(), "colour locations");
    cuda_check(cudaMemcpy(d_color_loc_, loc.data(), loc.size() * sizeof(ColorLoc),
                          cudaMemcpyHostToDevice),
               "upload");
  }
  cuda_check(cudaStreamSynchronize(up.stream), "bank upload");
  cuda_check(cudaDeviceSynchronize(), "bank upload");
  banks_load_s_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_banks).count();

  // Recovery directory.
  if (recovery_thread.joinable()) recovery_thread.join();
  recovery_load_s_ = recovery_s;
  if (rr_code != kOk) raise(rr_code, rr_error);
  if (m_.abandoned_recovery && m_.abandoned_hashes) {
    const uint64_t n = rr.hashes.size();
    check(n < (1ull << 31), kEUnsupported, "too many abandoned hashes for the device directory");
    check(rr.origins.size() < (1ull << 32), kEUnsupported, "too many abandoned origins");
    uint64_t cap = 4;
    while (cap < 2 * n) cap <<= 1;
    uint32_t bits = 0;
    while ((1ull << bits) < cap) ++bits;
    std::vector<uint64_t> dir_entries(cap, (uint64_t)kRecEmpty);
    std::vector<uint2> ranges;
    for (uint64_t i = 0; i < n; ++i) {
      uint32_t h = rr.hashes[i];
      uint64_t len = rr.starts[i + 1] - rr.starts[i];
      uint32_t value;
      if (len == 1 && rr.origins[rr.starts[i]] < kRecMultiple) {
        value = rr.origins[rr.starts[i]];
      } else {
        value = kRecMultiple | (uint32_t)ranges.size();
        ranges.push_back(make_uint2((uint32_t)rr.starts[i], (uint32_t)len));
      }
      uint64_t slot = h >> (32 - bits), mask = cap - 1;
      while ((uint32_t)dir_entries[slot] != kRecEmpty) slot = (slot + 1) & mask;
      dir_entries[slot] = ((uint64_t)h << 32) | value;
    }
    uint64_t* d_dir;
    uint2* d_ranges;
    uint32_t* d_origins;
    dev_alloc(&d_dir, cap, "recovery directory");
    dev_alloc(&d_ranges, ranges.size(), "recovery ranges");
    dev_alloc(&d_origins, rr.origins.size(), "recovery origins");
    allocations_.push_back(d_dir);
    allocations_.push_back(d_ranges);
    allocations_.push_back(d_origins);
    resident_bytes_ += cap * 8 + ranges.size() * 8 + rr.origins.size() * 4;
    cuda_check(cudaMemcpy(d_dir, dir_entries.data(), cap * 8, cudaMemcpyHostToDevice), "upload");
    if (!ranges.empty())
      cuda_check(cudaMemcpy(d_ranges, ranges.data(), ranges.size() * 8, cudaMemcpyHostToDevice),
                 "upload");
    cuda_check(cudaMemcpy(d_origins, rr.origins.data(), rr.origins.size() * 4,
                          cudaMemcpyHostToDevice),
               "upload");
    host_ix_.rec = DevRecovery{d_dir, d_ranges, d_origins, bits};
  }
  dev_alloc(&d_ix_rec_, 1, "index table");
  dev_alloc(&d_ix_norec_, 1, "index table");
  cuda_check(cudaMemcpy(d_ix_rec_, &host_ix_, sizeof(DevIndex), cudaMemcpyHostToDevice), "upload");
  DevIndex norec = host_ix_;
  norec.rec = DevRecovery{nullptr, nullptr, nullptr, 0};
  cuda_check(cudaMemcpy(d_ix_norec_, &norec, sizeof(DevIndex), cudaMemcpyHostToDevice), "upload");
  launch_ = default_launch();
  ws_ = make_workspace();
  load_s_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
}

uint64_t Engine::gather_sector_bytes_per_seed() const {
  uint64_t s = 0;
  for (uint32_t c = 0; c < host_ix_.classes; ++c) {
    const DevClass& C = host_ix_.cls[c];
    const uint64_t len = (uint64_t)C.fp_chunks * 16;
    const uint64_t at0 = (len + 31) / 32, at16 = (16 + len + 31) / 32;
    // Sectors per row, times 2 so the average over both row phases stays exact.
    const uint64_t twice = C.row_stride % 32 == 0 ? 2 * at0 : at0 + at16;
    s += (uint64_t)m_.hashes * twice * 16;
  }
  return s;
}

uint64_t Engine::gather_bytes_per_seed() const {
  uint64_t s = 0;
  for (auto& cls : m_.classes) s += (uint64_t)m_.hashes * m_.banks[cls[0]].lookup_bytes(m_.fingerprint_bits);
  return s;
}

QueryLaunch Engine::default_launch() const {
  QueryLaunch l = default_fused_launch();
  // Rows of 16 chunks (256 bytes of fingerprint planes per cell over all
  // classes) and more: the block-team probe over ordered rounds, one 16-byte
  // chunk per thread for rows of up to 256 chunks (teams of fewer threads
  // than the block below 128 chunks; 4 warps at 128), up to four beyond;
  // colour counters in shared memory while they leave room for two blocks
  // per SM. Measured on B200: C2's 16-chunk rows 19.75 ms in 4-warp blocks
  // (22.68 ms in 8-warp blocks, 23.64 ms for the fused kernel), C3 124.3 ms
  // in 9-warp blocks against 212.3 ms.
  if (wide_eligible(8) && wide_chunks() >= 16) {
    const uint32_t nc = wide_chunks();
    l.wide = 1;
    l.order = 1;
    l.warps = nc <= 128 ? 4 : ((nc > 256 && nc <= 288) || (nc > 512 && nc <= 576) ? 9 : 8);
    l.smem_counters = 1;
    if (m_.colors.size() > 16384 || fused_smem_bytes(l) > 110 * 1024) l.smem_counters = 0;
  }
  return l;
}

QueryLaunch Engine::fused_launch(const QueryLaunch& l) const {
  if (!l.wide) return l;
  QueryLaunch f = default_fused_launch();
  f.cut = l.cut;
  return f;
}

QueryLaunch Engine::default_fused_launch() const {
  uint32_t chunks = 1;
  for (uint32_t c = 0; c < host_ix_.classes; ++c) chunks = std::max(chunks, host_ix_.cls[c].fp_chunks);
  int team = 1;
  while (team < 32 && (uint32_t)team < chunks) team <<= 1;
  // Row-index gather with bit-plane counters, 8 warps per block, 2 resident
  // blocks per SM: teams of up to 16 lanes (one 16-byte chunk each) measured
  // fastest on B200 for 256-byte fingerprint rows (22.8 ms against 40.6 ms
  // for the per-hit form on 1.2e8 seeds); wider rows use teams of 8 or 16
  // and count in shared planes. Shared memory above
  // 110 KB per block moves the colour counters to global atomics (flushed
  // planes make them rare), then halves the warps; the per-hit form is the
  // last fallback.
  QueryLaunch l;
  // Measured on B200 over 14 index geometries (the planner's training set)
  // and the wide-row workloads: rows of up to 16 chunks run best with one
  // chunk per lane, rows of 17-64 chunks with teams of 8, wider rows with
  // whole-warp teams (512-chunk rows: 64 ms against 142 ms with teams of 16).
  l.team = chunks <= 16 ? team : (chunks <= 64 ? 8 : 32);
  l.warps = 8;
  l.smem_counters = m_.colors.size() <= 16384 ? 1 : 0;
  l.blocks = 0;  // 0: fill the device (occupancy-derived)
  l.stage_bytes = 0;  // register gather by default (fastest measured on B200 for small rows)
  l.stages = 2;
  l.bulk = 0;
  l.min_blocks = 2;
  l.planes = 1;
  l.cut = 4;
  l.wide = 0;
  l.order = 0;
  // Minimizer seeds are extracted by a kernel of their own: the probe kernel
  // then needs no extraction scratch and keeps twice the warps resident
  // (C3 slice on B200: 22.3 ms against 36.7 ms for the fused kernel).
  l.split = m_.index_mode == kMinimizers ? 1 : 0;
  // Wide rows: fewer warps per block keep several blocks per SM (measured on
  // 8 KiB rows of 16,384 colours: 2 warps x 3 blocks 64 ms, against 78 ms for
  // the per-hit form); colour counters go to global atomics above 2,048
  // colours, since flushed planes make them rare.
  const size_t budget = 110 * 1024;
  if (fused_smem_bytes(l) > budget && l.smem_counters && m_.colors.size() > 2048)
    l.smem_counters = 0;
  if (fused_smem_bytes(l) > budget) l.warps = 4;
  if (fused_smem_bytes(l) > budget) l.warps = 2;
  if (fused_smem_bytes(l) > budget) {
    l.warps = 8;
    l.planes = 0;
    l.team = std::min(team, 8);
    l.min_blocks = 3;
  }
  return l;
}

uint32_t Engine::wide_chunks() const {
  uint32_t n = 0;
  for (uint32_t c = 0; c < host_ix_.classes; ++c) n += host_ix_.cls[c].fp_chunks;
  return n;
}

bool Engine::wide_eligible(int warps) const {
  const uint32_t max_j = warps == 9 ? 2u : 4u;
  return m_.fingerprint_bits >= 4 && sp_.mode >= 0 && sp_.mode <= 2 && !sp_.strobe_max &&
         (warps == 4 || warps == 8 || warps == 9) && wide_chunks() <= max_j * (uint32_t)warps * 32u &&
         WideSmem::total((uint32_t)m_.colors.size(), host_ix_.classes, m_.hashes, 0) <= 200 * 1024;
}

bool Engine::wide_form(const QueryLaunch& l) const { return l.wide && wide_eligible(l.warps); }

void Engine::wide_shape(const QueryLaunch& l, int& J, int& HQ, uint32_t* team) const {
  const uint32_t T = (uint32_t)l.warps * 32u, nc = wide_chunks();
  // Rows of at most half a block of chunks: teams of the next power of two of
  // threads, one chunk each; wider rows: the whole block.
  uint32_t tt = T;
  if (2 * nc <= T) {
    tt = 1;
    while (tt < nc) tt <<= 1;
  }
  if (team) *team = tt;
  J = (int)((nc + tt - 1) / tt);
  const int Hp = (m_.hashes + 3) & ~3;
  HQ = Hp % 8 == 0 && J <= 2 ? 8 : 4;
}

void Engine::check_not_strobes() const {
  check(!sp_.strobe_max, kEUnsupported,
        "randstrobemer indexes score each record's two strands: query them through host-buffer "
        "calls (zx_query_host, zx_query_file, zx_query_per_record, per-record reports)");
}

int Engine::kernel_mode(const QueryLaunch& l) const {
  return l.split && sp_.mode == kMinimizers && l.planes == 1 && l.stage_bytes == 0 ? 4 : sp_.mode;
}

size_t Engine::fused_smem_bytes(const QueryLaunch& l) const {
  if (wide_form(l))
    return WideSmem::total((uint32_t)m_.colors.size(), host_ix_.classes, m_.hashes,
                           l.smem_counters);
  const int mode = kernel_mode(l);
  return FusedSmem::total(mode, sp_.k, (uint32_t)m_.colors.size(), host_ix_.classes, m_.hashes, l,
                          FusedSmem::shared_words(mode, host_ix_, l), sp_.strobe_max != 0);
}

int Engine::max_blocks(const QueryLaunch& l) const {
  if (cached_blocks_ && cached_for_.team == l.team && cached_for_.warps == l.warps &&
      cached_for_.smem_counters == l.smem_counters && cached_for_.stage_bytes == l.stage_bytes &&
      cached_for_.stages == l.stages && cached_for_.bulk == l.bulk &&
      cached_for_.min_blocks == l.min_blocks && cached_for_.planes == l.planes &&
      cached_for_.cut == l.cut && cached_for_.split == l.split && cached_for_.wide == l.wide)
    return cached_blocks_;
  int per_sm = 0;
  size_t smem = fused_smem_bytes(l);
  if (wide_form(l)) {
    int J, HQ;
    wide_shape(l, J, HQ);
    WideFn fn = wide_fn(J, HQ, l.warps * 32);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, l.warps * 32, smem),
               "occupancy");
  } else {
    FusedFn fn = fused_for(kernel_mode(l), l);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn,
                                                             l.warps * 32, smem),
               "occupancy");
  }
  const_cast<Engine*>(this)->cached_blocks_ = std::max(1, per_sm) * sms_;
  const_cast<Engine*>(this)->cached_for_ = l;
  return cached_blocks_;
}

void Engine::set_timing(bool on) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  if (on && !ev_begin_) {
    cuda_check(cudaEventCreate(&ev_begin_), "cudaEventCreate");
    cuda_check(cudaEventCreate(&ev_end_), "cudaEventCreate");
  }
  timing_ = on;
}

float Engine::last_fused_ms() {
  check(ev_end_ != nullptr, kEInval, "kernel timing is not enabled");
  cuda_check(cudaEventSynchronize(ev_end_), "timing");
  float ms = 0;
  cuda_check(cudaEventElapsedTime(&ms, ev_begin_, ev_end_), "timing");
  return ms;
}

void Engine::set_launch(const QueryLaunch& l) {
  check(l.team >= 1 && l.team <= 32 && (l.team & (l.team - 1)) == 0, kEInval,
        "team size must be a power of two in 1..32");
  check((l.warps >= 1 && l.warps <= 8) || (l.wide && l.warps == 9), kEInval,
        "warps per block must be in 1..8 (or 9 for the wide-row form)");
  check(l.smem_counters == 0 || m_.colors.size() <= 16384, kEInval,
        "shared-memory counters support at most 16384 colours");
  check(l.stage_bytes == 0 || (l.stage_bytes % 16 == 0 && l.stage_bytes >= 16 * m_.hashes &&
                                l.stage_bytes <= 65536 && l.stages >= 1 && l.stages <= 8),
        kEInval, "staged gather needs 16-byte multiple stages of at least 16*H bytes, 1..8 stages");
  check(m_.index_mode != kFindere || l.stage_bytes == 0, kEInval,
        "findere indexes use the register gather only");
  check(l.min_blocks >= 1 && l.min_blocks <= 3, kEInval, "min_blocks must be 1, 2 or 3");
  check(l.min_blocks != 1 || (l.planes == 1 && l.stage_bytes == 0), kEInval,
        "min_blocks 1 (255 registers) is compiled for the row-index form (planes 1) only");
  check(l.planes == 0 || l.planes == 1, kEInval, "planes must be 0 or 1");
  check(l.cut >= 1 && l.cut <= 64, kEInval, "cut must be in 1..64");
  check(l.split == 0 || l.split == 1, kEInval, "split must be 0 or 1");
  check(l.wide == 0 || l.wide == 1, kEInval, "wide must be 0 or 1");
  check(l.order >= 0 && l.order <= 2, kEInval, "order must be 0, 1 or 2");
  check(!l.wide || wide_eligible(l.warps), kEInval,
        "the wide-row form needs fingerprints of at least 4 bits, a k-mer, minimizer or "
        "modimizer index without strobes, 4, 8 or 9 warps per block and rows of at most "
        "4 x 32 x warps chunks (2 x 288 with 9 warps)");
  check(l.warps * 32 * l.min_blocks <= 2048 || l.warps <= 8, kEInval, "too many threads");
  check(fused_smem_bytes(l) <= 227 * 1024, kEInval, "launch needs too much shared memory");
  std::lock_guard<std::mutex> lock(mu_);
  launch_ = l;
  ws_->release_graphs();
}

std::unique_ptr<Workspace> Engine::make_workspace() {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  auto ws = std::make_unique<Workspace>();
  ws->device = device_;
  cuda_check(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  return ws;
}

void Engine::ensure_capacity(Workspace& ws, uint64_t nbases, uint64_t records, bool segmented) {
  const uint64_t colors = m_.colors.size();
  // Split minimizer and wide-row queries: key slots allocated before any graph capture.
  if (kernel_mode(launch_) == 4 || wide_form(launch_)) ensure_split_capacity(ws);
  const bool rounds = nbases / kTileWindows + records + nbases / kFindereTask + 1 > kSplitTiles;
  if (wide_form(launch_) && rounds) ensure_wide_pipeline(ws);
  if (wide_form(launch_) && launch_.order && !segmented) {
    ensure_order_capacity(ws, 0);
    if (rounds) ensure_order_capacity(ws, 1);
  }
  if (nbases > ws.cap_bases || !ws.bases) {
    uint64_t cap = std::max<uint64_t>({nbases, ws.cap_bases * 3 / 2, 4096});
    cap = round_up(cap, 4096);
    if (ws.bases) cudaFree(ws.bases);
    if (ws.packed) cudaFree(ws.packed);
    if (ws.invalid) cudaFree(ws.invalid);
    dev_alloc(&ws.bases, cap + 64, "batch bases");
    dev_alloc(&ws.packed, cap / 32 + 8, "packed bases");
    dev_alloc(&ws.invalid, cap / 32 + 8, "invalid masks");
    ws.cap_bases = cap;
    ws.cap_tiles = 0;
    ws.release_graphs();
  }
  if (records > ws.cap_records || !ws.offsets) {
    uint64_t cap = std::max<uint64_t>({records, ws.cap_records * 3 / 2, 1024});
    if (ws.offsets) cudaFree(ws.offsets);
    if (ws.tile_counts) cudaFree(ws.tile_counts);
    if (ws.tile_first) cudaFree(ws.tile_first);
    if (ws.scan_tmp) cudaFree(ws.scan_tmp);
    dev_alloc(&ws.offsets, cap + 1, "record offsets");
    dev_alloc(&ws.tile_counts, cap + 1, "tile counts");
    dev_alloc(&ws.tile_first, cap + 1, "tile offsets");
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, ws.tile_counts, ws.tile_first, (int)(cap + 1));
    dev_alloc((uint8_t**)&ws.scan_tmp, tmp, "scan scratch");
    ws.scan_tmp_bytes = tmp;
    ws.cap_records = cap;
    ws.cap_tiles = 0;
    ws.release_graphs();
  }
  uint64_t tiles = ws.cap_bases / kTileWindows + ws.cap_bases / kFindereTask + ws.cap_records + 16;
  if (tiles > ws.cap_tiles) {
    if (ws.tiles) cudaFree(ws.tiles);
    dev_alloc(&ws.tiles, tiles, "tiles");
    ws.cap_tiles = tiles;
    ws.release_graphs();
  }
  if (m_.index_mode == kFindere) {
    const uint64_t need = (uint64_t)max_blocks(launch_) * launch_.warps * 2 * std::max<uint64_t>(colors, 1);
    if (need > ws.cap_fstate) {
      if (ws.fstate) cudaFree(ws.fstate);
      dev_alloc(&ws.fstate, need, "findere colour state");
      ws.cap_fstate = need;
      ws.release_graphs();
    }
  }
  uint64_t partial = (uint64_t)max_blocks(launch_) * colors;
  if (partial > ws.cap_partial) {
    if (ws.partial) cudaFree(ws.partial);
    dev_alloc(&ws.partial, partial, "block counters");
    ws.cap_partial = partial;
    ws.release_graphs();
  }
  if (colors > ws.cap_colors || !ws.counts) {
    if (ws.counts) cudaFree(ws.counts);
    if (ws.total) cudaFree(ws.total);
    dev_alloc(&ws.counts, colors, "counts");
    dev_alloc(&ws.total, 1, "total");
    if (!ws.error) {
      dev_alloc(&ws.error, 1, "error word");
      cuda_check(cudaMemset(ws.error, 0, 4), "memset");
    }
    ws.cap_colors = colors;
    ws.release_graphs();
  }
}

void Engine::ensure_host_capacity(Workspace& ws, uint64_t nbases, uint64_t records) {
  if (nbases > ws.cap_h_bases || !ws.h_bases) {
    if (ws.h_bases) cudaFreeHost(ws.h_bases);
    uint64_t cap = round_up(std::max<uint64_t>({nbases, ws.cap_h_bases * 3 / 2, 4096}), 4096);
    host_alloc(&ws.h_bases, cap);
    ws.cap_h_bases = cap;
  }
  if (records + 1 > ws.cap_h_records || !ws.h_offsets) {
    if (ws.h_offsets) cudaFreeHost(ws.h_offsets);
    uint64_t cap = std::max<uint64_t>({records + 1, ws.cap_h_records * 3 / 2, 1024});
    host_alloc(&ws.h_offsets, cap);
    ws.cap_h_records = cap;
  }
  if (!ws.h_counts) {
    host_alloc(&ws.h_counts, std::max<uint64_t>(m_.colors.size(), 1));
    host_alloc(&ws.h_total, 1);
  }
}

void Engine::compress_homopolymers(Workspace& ws, const uint8_t*& bases, uint64_t nbases,
                                   const uint64_t*& offsets, uint64_t records, cudaStream_t s) {
  check(nbases < (1ull << 31) - 1, kEInval,
        "homopolymer-compressed queries take batches below 2^31 bases: split the batch");
  if (nbases > ws.cap_hp_bases || !ws.hp_bases) {
    const uint64_t cap = round_up(std::max<uint64_t>({nbases, ws.cap_hp_bases * 3 / 2, 4096}), 4096);
    for (void* p : {(void*)ws.hp_starts, (void*)ws.hp_keep, (void*)ws.hp_pos, (void*)ws.hp_bases,
                    ws.hp_scan_tmp})
      if (p) cudaFree(p);
    dev_alloc(&ws.hp_starts, cap / 32 + 2, "homopolymer record starts");
    dev_alloc(&ws.hp_keep, cap + 1, "homopolymer flags");
    dev_alloc(&ws.hp_pos, cap + 1, "homopolymer positions");
    dev_alloc(&ws.hp_bases, cap + 64, "compressed bases");
    size_t tmp = 0;
    cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, tmp, ws.hp_keep, ws.hp_pos, (int)(cap + 1)),
               "scan size");
    dev_alloc((uint8_t**)&ws.hp_scan_tmp, tmp, "homopolymer scan scratch");
    ws.hp_scan_bytes = tmp;
    ws.cap_hp_bases = cap;
    ws.release_graphs();
  }
  if (records + 1 > ws.cap_hp_records || !ws.hp_offsets) {
    const uint64_t cap = std::max<uint64_t>({records + 1, ws.cap_hp_records * 3 / 2, 1024});
    if (ws.hp_offsets) cudaFree(ws.hp_offsets);
    dev_alloc(&ws.hp_offsets, cap, "compressed offsets");
    ws.cap_hp_records = cap;
    ws.release_graphs();
  }
  const int bgrid = std::max(1, (int)std::min<uint64_t>((nbases + 256) / 256, (uint64_t)sms_ * 16));
  const int rgrid = std::max(1, (int)std::min<uint64_t>((records + 256) / 256, (uint64_t)sms_ * 16));
  cuda_check(cudaMemsetAsync(ws.hp_starts, 0, (nbases / 32 + 2) * 4, s), "memset");
  if (records) hp_mark_starts_kernel<<<rgrid, 256, 0, s>>>(offsets, records, nbases, ws.hp_starts);
  hp_keep_kernel<<<bgrid, 256, 0, s>>>(bases, nbases, ws.hp_starts, ws.hp_keep);
  cuda_check(cudaGetLastError(), "hp_keep_kernel");
  size_t tmp = ws.hp_scan_bytes;
  cuda_check(cub::DeviceScan::ExclusiveSum(ws.hp_scan_tmp, tmp, ws.hp_keep, ws.hp_pos,
                                           (int)(nbases + 1), s),
             "homopolymer scan");
  hp_compact_kernel<<<bgrid, 256, 0, s>>>(bases, nbases, ws.hp_pos, ws.hp_bases);
  hp_offsets_kernel<<<rgrid, 256, 0, s>>>(offsets, records, nbases, ws.hp_pos, ws.hp_offsets);
  cuda_check(cudaGetLastError(), "hp_offsets_kernel");
  bases = ws.hp_bases;
  offsets = ws.hp_offsets;
}

void Engine::plan_tiles(Workspace& ws, const uint64_t* offsets, uint64_t records,
                        uint64_t nbases, cudaStream_t s) {
  const int findere = m_.index_mode == kFindere;
  int grid = (int)std::min<uint64_t>((records + 255) / 256, (uint64_t)sms_ * 16);
  grid = std::max(grid, 1);
  cuda_check(cudaMemsetAsync(ws.tile_counts + records, 0, 4, s), "memset");
  if (records) {
    count_tiles_kernel<<<grid, 256, 0, s>>>(offsets, records, nbases, span(), findere,
                                            ws.tile_counts, ws.error);
    cuda_check(cudaGetLastError(), "count_tiles_kernel");
  }
  size_t tmp = ws.scan_tmp_bytes;
  cuda_check(cub::DeviceScan::ExclusiveSum(ws.scan_tmp, tmp, ws.tile_counts, ws.tile_first,
                                           (int)(records + 1), s),
             "tile scan");
  if (records) {
    fill_tiles_kernel<<<grid, 256, 0, s>>>(offsets, records, nbases, span(), ws.tile_first,
                                           ws.tiles);
    cuda_check(cudaGetLastError(), "fill_tiles_kernel");
  }
}

void Engine::enqueue(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                     const uint64_t* offsets, uint64_t records, bool recover, uint64_t* counts,
                     unsigned long long* total, cudaStream_t s) {
  if (m_.homopolymer_compression) compress_homopolymers(ws, bases, nbases, offsets, records, s);
  const uint64_t words = nbases / 32 + 2;
  QueryLaunch l = launch_;
  // Small batches: one block packs and plans (one launch for pack, count,
  // scan and fill), and with few colours the fused kernel adds into the
  // caller's counters (no reduction launch).
  const bool small = records <= kSmallRecords && nbases <= kSmallBases && !wide_form(l) &&
                     kernel_mode(l) != 4;
  if (small) {
    small_plan_kernel<<<1, 1024, 0, s>>>(bases, nbases, ws.packed, ws.invalid, words, offsets,
                                         (uint32_t)records, span(), m_.index_mode == kFindere,
                                         ws.tile_first, ws.tiles, ws.error);
    cuda_check(cudaGetLastError(), "small_plan_kernel");
    if (m_.colors.size() <= kSmallColors) l.smem_counters = 0;
  } else {
    int grid = (int)std::min<uint64_t>((words + 255) / 256, (uint64_t)sms_ * 16);
    pack_kernel<<<std::max(grid, 1), 256, 0, s>>>(bases, nbases, ws.packed, ws.invalid, words);
    cuda_check(cudaGetLastError(), "pack_kernel");
    plan_tiles(ws, offsets, records, nbases, s);
  }
  const int kmode = kernel_mode(l);
  const size_t smem = fused_smem_bytes(l);
  const int blocks_cap = max_blocks(l);
  uint64_t tiles_bound = nbases / kTileWindows + records + nbases / kFindereTask + 1;
  uint64_t want = (tiles_bound + l.warps - 1) / l.warps;
  int blocks = l.blocks > 0 ? std::min(l.blocks, blocks_cap)
                            : (int)std::min<uint64_t>((uint64_t)blocks_cap, std::max<uint64_t>(want, 1));
  l.blocks = blocks;
  BatchView bv{PackedView{ws.packed, ws.invalid}, offsets, ws.tiles, ws.tile_first + records,
               ws.fstate};
  // Findere round state: in shared memory for up to kFindereSmemColors
  // colours, else in this zeroed scratch.
  if (m_.index_mode == kFindere && m_.colors.size() > kFindereSmemColors)
    cuda_check(cudaMemsetAsync(ws.fstate, 0,
                               (uint64_t)blocks * l.warps * 2 * m_.colors.size() * 4, s),
               "memset");
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  cuda_check(cudaStreamIsCapturing(s, &capturing), "cudaStreamIsCapturing");
  const bool timed = timing_ && capturing == cudaStreamCaptureStatusNone;
  if (timed) cuda_check(cudaEventRecord(ev_begin_, s), "cudaEventRecord");
  FusedFn fn = fused_for(kmode, l);
  // The dynamic shared-memory limit is a property of the kernel function, shared by
  // every engine in the process: set it for this launch's size every time.
  cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute");
  const uint32_t colors = (uint32_t)m_.colors.size();
  auto reduce = [&] {
    if (!l.smem_counters) return;
    reduce_counters_kernel<<<std::max(1u, (colors + 255) / 256), 256, 0, s>>>(ws.partial, blocks,
                                                                               colors, counts);
    cuda_check(cudaGetLastError(), "reduce_counters_kernel");
  };
  if (wide_form(l)) {
    run_wide(ws, bv, tiles_bound, recover, counts, total, 0, s);
    if (timed) cuda_check(cudaEventRecord(ev_end_, s), "cudaEventRecord");
    return;
  }
  if (kmode != 4) {
    fn<<<blocks, l.warps * 32, smem, s>>>(recover ? d_ix_rec_ : d_ix_norec_, bv, sp_, l, ws.partial,
                                          counts, total, ws.error);
    cuda_check(cudaGetLastError(), "fused_query_kernel");
    if (timed) cuda_check(cudaEventRecord(ev_end_, s), "cudaEventRecord");
    reduce();
    return;
  }
  // Split minimizer query: rounds of up to kSplitTiles tiles; per round the
  // extraction kernel fills each tile's key slot, the probe kernel (no
  // extraction scratch, so more warps per SM) counts them, and the block
  // counters are added up. The rounds cover the host's tile bound; tiles past
  // the planned count are skipped on the device.
  ensure_split_capacity(ws);
  const int ewarps = 4;
  const size_t esmem = 256 * 8 + ewarps * FusedSmem::warp_bytes(kMinimizers, sp_.k, 0);
  ExtractFn efn = extract_for(kMinimizers);
  cuda_check(cudaFuncSetAttribute(efn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)esmem),
             "cudaFuncSetAttribute");
  const int egrid = (int)std::min<uint64_t>((kSplitTiles + ewarps - 1) / ewarps,
                                            (uint64_t)sms_ * 8);
  for (uint64_t lo = 0; lo < tiles_bound; lo += kSplitTiles) {
    BatchView rb = bv;
    rb.tile_lo = (uint32_t)lo;
    rb.tile_hi = (uint32_t)std::min<uint64_t>(lo + kSplitTiles, tiles_bound);
    rb.prekeys = ws.split_keys;
    rb.prekey_count = ws.split_counts;
    efn<<<egrid, ewarps * 32, esmem, s>>>(rb, sp_, ws.split_keys, ws.split_counts, ewarps);
    cuda_check(cudaGetLastError(), "extract_kernel");
    fn<<<blocks, l.warps * 32, smem, s>>>(recover ? d_ix_rec_ : d_ix_norec_, rb, sp_, l,
                                          ws.partial, counts, total, ws.error);
    cuda_check(cudaGetLastError(), "fused_query_kernel");
    reduce();
  }
  if (timed) cuda_check(cudaEventRecord(ev_end_, s), "cudaEventRecord");
}

void Engine::run_wide(Workspace& ws, const BatchView& bv, uint64_t tiles_bound, bool recover,
                      uint64_t* counts, unsigned long long* total, uint32_t segments,
                      cudaStream_t s, double prune_ratio) {
  // Rounds of up to kSplitTiles tiles; per round the extraction kernel
  // appends the tiles' seeds to one dense list (segmented: each segment's
  // seeds to its own part of it), the wide probe counts them, and the block
  // counters are added up (segmented: each block adds its counters to the
  // segment it leaves).
  const QueryLaunch& l = launch_;
  ensure_split_capacity(ws);
  const size_t smem = fused_smem_bytes(l);
  const int blocks_cap = max_blocks(l);
  int J, HQ;
  uint32_t wteam = 0;
  wide_shape(l, J, HQ, &wteam);
  WideFn wfn = wide_fn(J, HQ, l.warps * 32);
  cuda_check(cudaFuncSetAttribute(wfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute");
  const int ewarps = 4;
  const size_t esmem = DenseSmem::total(sp_.mode, sp_.k, ewarps);
  DenseExtractFn efn = dense_extract_for(sp_.mode);
  cuda_check(cudaFuncSetAttribute(efn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)esmem),
             "cudaFuncSetAttribute");
  const int egrid = (int)std::min<uint64_t>((kSplitTiles + ewarps - 1) / ewarps,
                                            (uint64_t)sms_ * 8);
  // A tile holds at most 256 seeds: one probe round.
  const int wblocks = l.blocks > 0 ? std::min(l.blocks, blocks_cap)
                                   : (int)std::min<uint64_t>(blocks_cap, std::max<uint64_t>(tiles_bound, 1));
  const uint32_t colors = (uint32_t)m_.colors.size();
  const uint64_t rounds = (tiles_bound + kSplitTiles - 1) / kSplitTiles;
  // Several rounds: extraction (compute-bound) of round r + 1 runs on the
  // auxiliary stream beside the probe (memory-bound) of round r, the rounds
  // alternating between two key lists; events order each list's reuse.
  const bool overlap = rounds > 1;
  if (overlap) ensure_wide_pipeline(ws);
  cudaStream_t xs = overlap ? ws.aux_stream : s;
  if (overlap) {
    cuda_check(cudaEventRecord(ws.wide_fork, s), "cudaEventRecord");
    cuda_check(cudaStreamWaitEvent(xs, ws.wide_fork, 0), "cudaStreamWaitEvent");
  }
  for (uint64_t r = 0; r < rounds; ++r) {
    const int b = overlap ? (int)(r & 1) : 0;
    uint64_t* keys = b ? ws.wide_keys2 : ws.split_keys;
    BatchView rb = bv;
    rb.tile_lo = (uint32_t)(r * kSplitTiles);
    rb.tile_hi = (uint32_t)std::min<uint64_t>((r + 1) * kSplitTiles, tiles_bound);
    WideRound sg;
    if (segments) {
      sg.seg_tiles = ws.seg_tiles;
      sg.cursor = ws.wide_seg_cursor + (uint64_t)b * ws.cap_segments;
      sg.round_first = ws.wide_round_first + (uint64_t)b * ws.cap_segments;
      sg.totals = total;
      sg.nseg = segments;
      sg.tile_lo = rb.tile_lo;
      sg.tile_hi = rb.tile_hi;
      sg.min_ratio = prune_ratio;
    }
    const bool ordered = l.order && !segments;
    if (ordered) ensure_order_capacity(ws, b);
    sg.interleave = !segments && l.order == 2 ? 1u : 0u;
    if (overlap && r >= 2)
      cuda_check(cudaStreamWaitEvent(xs, ws.wide_probe[b], 0), "cudaStreamWaitEvent");
    if (segments)
      cuda_check(cudaMemsetAsync(sg.cursor, 0, segments * 8ull, xs), "memset");
    else
      cuda_check(cudaMemsetAsync(ws.wide_cursor + b, 0, 8, xs), "memset");
    efn<<<egrid, ewarps * 32, esmem, xs>>>(rb, sp_, keys, ws.wide_cursor + b, ewarps, sg);
    cuda_check(cudaGetLastError(), "extract_dense_kernel");
    const uint64_t* probe_keys = keys;
    if (ordered) {
      // Counting sort of the round's keys by their first hash's top bits
      // (row-address order of every class), the key count read on the device.
      const int ogrid = sms_ * 8;
      cuda_check(cudaMemsetAsync(ws.wide_hist[b], 0, kOrderBuckets * 4, xs), "memset");
      order_count_kernel<<<ogrid, 256, 0, xs>>>(keys, ws.wide_cursor + b, host_ix_.seed,
                                                ws.wide_hist[b]);
      cuda_check(cudaGetLastError(), "order_count_kernel");
      order_scan_kernel<<<1, 1024, 0, xs>>>(ws.wide_hist[b]);
      cuda_check(cudaGetLastError(), "order_scan_kernel");
      order_scatter_kernel<<<ogrid, 256, 0, xs>>>(keys, ws.wide_cursor + b, host_ix_.seed,
                                                  ws.wide_hist[b], ws.wide_keys_alt[b]);
      cuda_check(cudaGetLastError(), "order_scatter_kernel");
      probe_keys = ws.wide_keys_alt[b];
    }
    if (segments) {
      wide_rounds_kernel<<<1, 1024, 0, xs>>>(sg.cursor, segments,
                                             const_cast<uint32_t*>(sg.round_first));
      cuda_check(cudaGetLastError(), "wide_rounds_kernel");
    }
    if (overlap) {
      cuda_check(cudaEventRecord(ws.wide_ext[b], xs), "cudaEventRecord");
      cuda_check(cudaStreamWaitEvent(s, ws.wide_ext[b], 0), "cudaStreamWaitEvent");
    }
    wfn<<<wblocks, l.warps * 32, smem, s>>>(recover ? d_ix_rec_ : d_ix_norec_, d_color_loc_,
                                            probe_keys, ws.wide_cursor + b, l.smem_counters,
                                            wteam, ws.partial, counts, segments ? nullptr : total,
                                            sg);
    cuda_check(cudaGetLastError(), "wide_probe_kernel");
    if (l.smem_counters && !segments) {
      reduce_counters_kernel<<<std::max(1u, (colors + 255) / 256), 256, 0, s>>>(
          ws.partial, wblocks, colors, counts);
      cuda_check(cudaGetLastError(), "reduce_counters_kernel");
    }
    if (overlap) cuda_check(cudaEventRecord(ws.wide_probe[b], s), "cudaEventRecord");
  }
}

void Engine::ensure_order_capacity(Workspace& ws, int b) {
  if (ws.wide_keys_alt[b]) return;
  dev_alloc(&ws.wide_keys_alt[b], (uint64_t)kSplitTiles * kTileWindows, "round keys in order");
  dev_alloc(&ws.wide_hist[b], kOrderBuckets, "round order buckets");
  ws.release_graphs();
}

void Engine::ensure_strobe_capacity(Workspace& ws, uint64_t nbases, uint64_t tiles) {
  if (nbases > ws.cap_strobe_bases || !ws.strobe_anchors) {
    const uint64_t cap = std::max<uint64_t>({nbases, ws.cap_strobe_bases * 3 / 2, 4096});
    if (ws.strobe_anchors) cudaFree(ws.strobe_anchors);
    if (ws.strobe_hashes) cudaFree(ws.strobe_hashes);
    ws.strobe_anchors = nullptr;
    ws.strobe_hashes = nullptr;
    dev_alloc(&ws.strobe_anchors, cap / 32 + 2, "strobe candidates");
    dev_alloc(&ws.strobe_hashes, cap + 1, "strobe hashes");
    ws.cap_strobe_bases = cap;
    ws.release_graphs();
  }
  if (tiles > ws.cap_strobe_tiles || !ws.strobe_slots) {
    const uint64_t cap = std::max<uint64_t>({tiles, ws.cap_strobe_tiles * 3 / 2, 1024});
    if (ws.strobe_slots) cudaFree(ws.strobe_slots);
    if (ws.strobe_count) cudaFree(ws.strobe_count);
    ws.strobe_slots = nullptr;
    ws.strobe_count = nullptr;
    dev_alloc(&ws.strobe_slots, cap * kStrobeSlot, "strobe seeds");
    dev_alloc(&ws.strobe_count, cap, "strobe seed counts");
    ws.cap_strobe_tiles = cap;
    ws.release_graphs();
  }
}

void Engine::link_strobes(Workspace& ws, const BatchView& bv, uint64_t nbases, cudaStream_t s) {
  cuda_check(cudaMemsetAsync(ws.strobe_anchors, 0, (nbases / 32 + 2) * 4, s), "memset");
  const int warps = 4;
  const int mode = sp_.mode == kMinimizers ? 1 : 0;
  const size_t smem = StrobeSmem::total(mode, sp_.k, warps);
  auto afn = mode == 1 ? strobe_anchor_kernel<1> : strobe_anchor_kernel<0>;
  cuda_check(cudaFuncSetAttribute(afn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute");
  const int grid = sms_ * 8;
  afn<<<grid, warps * 32, smem, s>>>(bv, sp_, ws.strobe_anchors, ws.strobe_hashes, warps);
  cuda_check(cudaGetLastError(), "strobe_anchor_kernel");
  const int len = mode == 1 ? sp_.m : sp_.klen;
  const uint32_t extra = mode == 1 && sp_.k != sp_.m ? (uint32_t)sp_.ocm.w - 1 : 0u;
  strobe_link_kernel<<<grid, 256, 0, s>>>(bv, sp_, ws.strobe_anchors, ws.strobe_hashes, len,
                                          extra, ws.strobe_slots, ws.strobe_count);
  cuda_check(cudaGetLastError(), "strobe_link_kernel");
}

void Engine::ensure_segment_capacity(Workspace& ws, uint32_t segments) {
  if (segments + 1 > ws.cap_segments || !ws.seg_blocks) {
    const uint64_t c = std::max<uint64_t>(segments + 1, 256);
    for (void* p : {(void*)ws.seg_blocks, (void*)ws.seg_tiles, (void*)ws.seg_records,
                    (void*)ws.wide_seg_cursor, (void*)ws.wide_round_first})
      if (p) cudaFree(p);
    for (void* p : {(void*)ws.h_seg_blocks, (void*)ws.h_seg_records})
      if (p) cudaFreeHost(p);
    ws.wide_seg_cursor = nullptr;
    ws.wide_round_first = nullptr;
    dev_alloc(&ws.seg_blocks, c, "segment blocks");
    dev_alloc(&ws.seg_tiles, c, "segment tiles");
    dev_alloc(&ws.seg_records, c, "segment records");
    host_alloc(&ws.h_seg_blocks, c);
    host_alloc(&ws.h_seg_records, c);
    ws.cap_segments = c;
  }
  if (wide_form(launch_) && !ws.wide_seg_cursor) {
    dev_alloc(&ws.wide_seg_cursor, 2 * ws.cap_segments, "segment key cursors");
    dev_alloc(&ws.wide_round_first, 2 * ws.cap_segments, "segment probe rounds");
  }
  if (!ws.seg_staged)
    cuda_check(cudaEventCreateWithFlags(&ws.seg_staged, cudaEventDisableTiming), "cudaEventCreate");
}

void Engine::ensure_wide_pipeline(Workspace& ws) {
  if (ws.aux_stream) return;
  dev_alloc(&ws.wide_keys2, kSplitTiles * kTileWindows, "second dense key list");
  cuda_check(cudaStreamCreateWithFlags(&ws.aux_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  for (cudaEvent_t* e : {&ws.wide_fork, &ws.wide_ext[0], &ws.wide_ext[1], &ws.wide_probe[0],
                         &ws.wide_probe[1]})
    cuda_check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
  ws.release_graphs();
}

void Engine::ensure_split_capacity(Workspace& ws) {
  if (ws.split_keys) return;
  dev_alloc(&ws.split_keys, kSplitTiles * kTileWindows, "split key slots");
  dev_alloc(&ws.split_counts, kSplitTiles, "split key counts");
  dev_alloc(&ws.wide_cursor, 2, "dense key cursors");
  ws.release_graphs();
}

uint64_t Engine::tiles_for_length(uint64_t len) const {
  const uint64_t span = (uint64_t)this->span();
  if (len < span) return 0;
  const uint64_t w = len - span + 1;
  if (m_.index_mode != kFindere) return (w + kTileWindows - 1) / kTileWindows;
  return (w / kFindereTask) * (kFindereTask / kTileWindows) +
         (w % kFindereTask + kTileWindows - 1) / kTileWindows;
}

void Engine::query_segments(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                            const uint64_t* offsets, uint64_t records, const uint64_t* seg_records,
                            const uint64_t* est_tiles, uint32_t segments, bool recover,
                            uint64_t* counts, unsigned long long* totals, cudaStream_t s,
                            int warps, double prune_ratio) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  check(segments > 0, kEInval, "a segmented query needs at least one segment");
  check(warps >= 0 && warps <= 8, kEInval, "warps per block must be in 1..8");
  check(seg_records[0] == 0 && seg_records[segments] == records, kEInval,
        "segments must span the records");
  for (uint32_t i = 0; i < segments; ++i)
    check(seg_records[i] <= seg_records[i + 1], kEInval, "segment records must be non-decreasing");
  ensure_capacity(ws, nbases, records, true);
  ensure_segment_capacity(ws, segments);
  // The pinned staging is reused: wait until the previous call's copies ran.
  cuda_check(cudaEventSynchronize(ws.seg_staged), "segment staging");
  if (wide_form(launch_)) {
    // Wide-row indexes: one wide-form query over the whole batch, each
    // request's seeds in its own part of the key lists and its own counters.
    for (uint32_t i = 0; i <= segments; ++i) ws.h_seg_records[i] = seg_records[i];
    cuda_check(cudaMemcpyAsync(ws.seg_records, ws.h_seg_records, (segments + 1) * 8ull,
                               cudaMemcpyHostToDevice, s),
               "H2D");
    cuda_check(cudaEventRecord(ws.seg_staged, s), "cudaEventRecord");
    if (m_.homopolymer_compression) compress_homopolymers(ws, bases, nbases, offsets, records, s);
    const uint64_t words = nbases / 32 + 2;
    int grid = (int)std::min<uint64_t>((words + 255) / 256, (uint64_t)sms_ * 16);
    pack_kernel<<<std::max(grid, 1), 256, 0, s>>>(bases, nbases, ws.packed, ws.invalid, words);
    cuda_check(cudaGetLastError(), "pack_kernel");
    plan_tiles(ws, offsets, records, nbases, s);
    segment_tiles_kernel<<<(segments + 256) / 256, 256, 0, s>>>(ws.tile_first, ws.seg_records,
                                                                segments, ws.seg_tiles);
    cuda_check(cudaGetLastError(), "segment_tiles_kernel");
    BatchView bv{PackedView{ws.packed, ws.invalid}, offsets, ws.tiles, ws.tile_first + records,
                 ws.fstate};
    const uint64_t tiles_bound = nbases / kTileWindows + records + nbases / kFindereTask + 1;
    run_wide(ws, bv, tiles_bound, recover, counts, totals, segments, s, prune_ratio);
    return;
  }
  QueryLaunch l = fused_launch(launch_);
  l.split = 0;  // every segment extracts its own tiles in the fused kernel
  if (warps > 0 && warps < l.warps) l.warps = warps;
  // Randstrobemer indexes: the segments' seeds are linked beforehand
  // (strobes.cuh) and probed from their tile slots (mode 4, row-index form).
  const bool strobes = sp_.strobe_max != 0;
  if (strobes) {
    l.planes = 1;
    l.stage_bytes = 0;
    uint64_t tiles = 0;
    for (uint32_t i = 0; i < segments; ++i) tiles += est_tiles[i];
    check(tiles <= kSplitTiles, kEInval,
          "a randstrobemer query holds at most 262,144 tiles (about 64 Mbases) per launch");
    ensure_strobe_capacity(ws, nbases, std::max<uint64_t>(tiles, 1));
  }
  const int cap = max_blocks(l);
  const uint32_t wpb = (uint32_t)l.warps;
  // Grid shares: proportional to the estimated tiles, at least one block,
  // at most one warp per tile.
  uint64_t est_total = 0;
  for (uint32_t i = 0; i < segments; ++i) est_total += est_tiles[i];
  uint32_t blocks = 0;
  for (uint32_t i = 0; i < segments; ++i) {
    ws.h_seg_blocks[i] = blocks;
    uint64_t share = est_total ? est_tiles[i] * (uint64_t)cap / est_total : 1;
    share = std::min<uint64_t>(share, (est_tiles[i] + wpb - 1) / wpb);
    blocks += (uint32_t)std::max<uint64_t>(share, 1);
    ws.h_seg_records[i] = seg_records[i];
  }
  ws.h_seg_blocks[segments] = blocks;
  ws.h_seg_records[segments] = seg_records[segments];
  const uint64_t colors = m_.colors.size();
  if (l.smem_counters && (uint64_t)blocks * colors > ws.cap_partial) {
    if (ws.partial) cudaFree(ws.partial);
    dev_alloc(&ws.partial, (uint64_t)blocks * colors, "block counters");
    ws.cap_partial = (uint64_t)blocks * colors;
    ws.release_graphs();
  }
  if (m_.index_mode == kFindere && (uint64_t)blocks * wpb * 2 * colors > ws.cap_fstate) {
    if (ws.fstate) cudaFree(ws.fstate);
    dev_alloc(&ws.fstate, (uint64_t)blocks * wpb * 2 * colors, "findere colour state");
    ws.cap_fstate = (uint64_t)blocks * wpb * 2 * colors;
    ws.release_graphs();
  }
  cuda_check(cudaMemcpyAsync(ws.seg_blocks, ws.h_seg_blocks, (segments + 1) * 4ull,
                             cudaMemcpyHostToDevice, s),
             "H2D");
  cuda_check(cudaMemcpyAsync(ws.seg_records, ws.h_seg_records, (segments + 1) * 8ull,
                             cudaMemcpyHostToDevice, s),
             "H2D");
  cuda_check(cudaEventRecord(ws.seg_staged, s), "cudaEventRecord");
  if (m_.homopolymer_compression) compress_homopolymers(ws, bases, nbases, offsets, records, s);
  const uint64_t words = nbases / 32 + 2;
  {
    int grid = (int)std::min<uint64_t>((words + 255) / 256, (uint64_t)sms_ * 16);
    pack_kernel<<<std::max(grid, 1), 256, 0, s>>>(bases, nbases, ws.packed, ws.invalid, words);
    cuda_check(cudaGetLastError(), "pack_kernel");
  }
  plan_tiles(ws, offsets, records, nbases, s);
  segment_tiles_kernel<<<(segments + 256) / 256, 256, 0, s>>>(ws.tile_first, ws.seg_records,
                                                              segments, ws.seg_tiles);
  cuda_check(cudaGetLastError(), "segment_tiles_kernel");
  l.blocks = (int)blocks;
  const int kmode = strobes ? 4 : sp_.mode;
  const size_t smem = strobes ? FusedSmem::total(4, sp_.k, (uint32_t)colors, host_ix_.classes,
                                                 m_.hashes, l,
                                                 FusedSmem::shared_words(4, host_ix_, l), true)
                              : fused_smem_bytes(l);
  BatchView bv{PackedView{ws.packed, ws.invalid}, offsets, ws.tiles, ws.tile_first + records,
               ws.fstate, segments, ws.seg_blocks, ws.seg_tiles};
  if (strobes) {
    link_strobes(ws, bv, nbases, s);
    bv.prekeys = ws.strobe_slots;
    bv.prekey_count = ws.strobe_count;
    bv.prekey_stride = kStrobeSlot;
  }
  if (m_.index_mode == kFindere && colors > kFindereSmemColors)
    cuda_check(cudaMemsetAsync(ws.fstate, 0, (uint64_t)blocks * wpb * 2 * colors * 4, s), "memset");
  FusedFn fn = fused_for(kmode, l);
  cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute");
  fn<<<blocks, l.warps * 32, smem, s>>>(recover ? d_ix_rec_ : d_ix_norec_, bv, sp_, l, ws.partial,
                                        counts, totals, ws.error);
  cuda_check(cudaGetLastError(), "fused_query_kernel");
  if (l.smem_counters) {
    const uint64_t n = (uint64_t)segments * colors;
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, sms_ * 8ull));
    reduce_segments_kernel<<<grid, 256, 0, s>>>(ws.partial, ws.seg_blocks, segments,
                                                (uint32_t)colors, counts);
    cuda_check(cudaGetLastError(), "reduce_segments_kernel");
  }
}

void Engine::record_groups(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                           const uint64_t* offsets, uint64_t records, bool recover,
                           double prune_ratio,
                           const std::function<void(uint64_t, uint64_t)>& on_group) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  check(offsets[0] == 0 && offsets[records] == nbases, kEInval, "offsets must span the bases");
  for (uint64_t r = 0; r < records; ++r)  // groups are cut and sized on the host
    check(offsets[r] <= offsets[r + 1], kEInval, "offsets must be non-decreasing");
  const uint64_t colors = std::max<uint64_t>(m_.colors.size(), 1);
  // Group size: the group's counters (records x colours x 8 bytes), the extra
  // block counters (one block per short record, colours x 4 bytes each) and,
  // for findere, the extra per-warp colour state stay within 256 MiB each.
  const uint64_t budget = 256ull << 20;
  uint64_t gmax = budget / (colors * 8);
  if (m_.index_mode == kFindere) gmax = std::min<uint64_t>(gmax, budget / (colors * 8 * launch_.warps));
  gmax = std::max<uint64_t>(1, std::min<uint64_t>(gmax, 1ull << 20));
  // Randstrobemer groups: one launch's tile slots and a candidate table of
  // 8 bytes per base (64 Mi bases).
  const bool strobes = sp_.strobe_max != 0;
  const uint64_t group_bases = strobes ? (64ull << 20) : (256ull << 20);
  if (gmax > ws.cap_rec_totals || !ws.rec_counts) {
    for (void* p : {(void*)ws.rec_counts, (void*)ws.rec_totals, (void*)ws.rec_hits,
                    (void*)ws.rec_first, ws.rec_scan_tmp})
      if (p) cudaFree(p);
    ws.rec_counts = nullptr;
    ws.rec_totals = nullptr;
    ws.rec_hits = ws.rec_first = nullptr;
    ws.rec_scan_tmp = nullptr;
    dev_alloc(&ws.rec_counts, gmax * colors, "record counters");
    dev_alloc(&ws.rec_totals, gmax, "record totals");
    dev_alloc(&ws.rec_hits, gmax + 1, "record hit counts");
    dev_alloc(&ws.rec_first, gmax + 1, "record hit offsets");
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, ws.rec_hits, ws.rec_first, (int)(gmax + 1));
    dev_alloc((uint8_t**)&ws.rec_scan_tmp, tmp, "record hit scan scratch");
    ws.rec_scan_bytes = tmp;
    ws.cap_rec_counts = gmax * colors;
    ws.cap_rec_totals = gmax;
  }
  cudaStream_t s = ws.stream;
  // Page-locked caller bases are copied directly, pageable ones through the
  // workspace's pinned staging.
  cudaPointerAttributes attr;
  bool direct = false;
  if (nbases && cudaPointerGetAttributes(&attr, bases) == cudaSuccess)
    direct = attr.type == cudaMemoryTypeHost;
  else
    cudaGetLastError();
  std::vector<uint64_t> seg, est;
  for (uint64_t r0 = 0; r0 < records;) {
    // (Strobe groups count a tile for every record, as the launch's estimate does.)
    auto tiles_of = [&](uint64_t r) {
      const uint64_t t = tiles_for_length(offsets[r + 1] - offsets[r]);
      return strobes ? std::max<uint64_t>(1, t) : t;
    };
    uint64_t r1 = r0 + 1, tiles = tiles_of(r0);
    while (r1 < records && r1 - r0 < gmax && offsets[r1 + 1] - offsets[r0] <= group_bases) {
      const uint64_t next = tiles_of(r1);
      if (strobes && tiles + next > kSplitTiles) break;
      tiles += next;
      ++r1;
    }
    const uint64_t n = r1 - r0, b0 = offsets[r0], nb = offsets[r1] - b0;
    ensure_capacity(ws, nb, n, true);
    ensure_host_capacity(ws, nb, n);
    seg.resize(n + 1);
    est.resize(n);
    for (uint64_t i = 0; i <= n; ++i) {
      seg[i] = i;
      ws.h_offsets[i] = offsets[r0 + i] - b0;
    }
    for (uint64_t i = 0; i < n; ++i)
      est[i] = std::max<uint64_t>(1, tiles_for_length(offsets[r0 + i + 1] - offsets[r0 + i]));
    if (nb) {
      const uint8_t* src = bases + b0;
      if (!direct) {
        memcpy(ws.h_bases, src, nb);
        src = ws.h_bases;
      }
      cuda_check(cudaMemcpyAsync(ws.bases, src, nb, cudaMemcpyHostToDevice, s), "H2D");
    }
    cuda_check(cudaMemcpyAsync(ws.offsets, ws.h_offsets, (n + 1) * 8, cudaMemcpyHostToDevice, s),
               "H2D");
    cuda_check(cudaMemsetAsync(ws.rec_counts, 0, n * colors * 8, s), "memset");
    cuda_check(cudaMemsetAsync(ws.rec_totals, 0, n * 8, s), "memset");
    // Short records: warps per block near the mean tiles per record.
    int warps = 0;
    const uint64_t mean = (tiles + n - 1) / n;
    if (mean < (uint64_t)launch_.warps) warps = mean <= 2 ? 2 : (mean <= 4 ? 4 : 8);
    query_segments(ws, ws.bases, nb, ws.offsets, n, seg.data(), est.data(), (uint32_t)n, recover,
                   ws.rec_counts, ws.rec_totals, s, warps, prune_ratio);
    on_group(r0, n);
    cuda_check(cudaStreamSynchronize(s), "per-record query");
    check_error_word(ws);
    r0 = r1;
  }
}

void Engine::query_per_record(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                              const uint64_t* offsets, uint64_t records, bool recover,
                              uint64_t* counts, uint64_t* totals) {
  const uint64_t colors = m_.colors.size();
  cudaStream_t s = ws.stream;
  auto run = [&](const uint8_t* b, uint64_t* c, uint64_t* t) {
    record_groups(ws, b, nbases, offsets, records, recover, 0.0, [&](uint64_t r0, uint64_t n) {
      cuda_check(cudaMemcpyAsync(c + r0 * colors, ws.rec_counts, n * colors * 8,
                                 cudaMemcpyDeviceToHost, s),
                 "D2H");
      cuda_check(cudaMemcpyAsync(t + r0, ws.rec_totals, n * 8, cudaMemcpyDeviceToHost, s), "D2H");
    });
  };
  run(bases, counts, totals);
  if (!sp_.strobe_max) return;
  // Randstrobemers: the reverse-complement strand too, and per record and
  // colour the larger count (PreparedRead::new, query_stream.rs:516-534;
  // Scores::score, query_stream.rs:690-701).
  std::vector<uint8_t> rc(nbases);
  reverse_complement_records(bases, offsets, records, rc.data());
  std::vector<uint64_t> rcounts(records * colors), rtotals(records);
  run(rc.data(), rcounts.data(), rtotals.data());
  for (uint64_t r = 0; r < records; ++r)
    check(rtotals[r] == totals[r], kEFormat, "canonical anchor counts must agree across strands");
  for (uint64_t i = 0; i < records * colors; ++i) counts[i] = std::max(counts[i], rcounts[i]);
}

void reverse_complement_records(const uint8_t* bases, const uint64_t* offsets, uint64_t records,
                                uint8_t* out) {
  // reverse_complement (src/anchors.rs:257-263): ACGT of either case become
  // the upper-case complement, every other byte stays a separator.
  static const struct Table {
    uint8_t t[256];
    Table() {
      for (int i = 0; i < 256; ++i) t[i] = (uint8_t)i;
      t['A'] = t['a'] = 'T';
      t['C'] = t['c'] = 'G';
      t['G'] = t['g'] = 'C';
      t['T'] = t['t'] = 'A';
    }
  } table;
  for (uint64_t r = 0; r < records; ++r) {
    const uint64_t a = offsets[r], b = offsets[r + 1];
    for (uint64_t i = a; i < b; ++i) out[a + (b - 1 - i)] = table.t[bases[i]];
  }
}

void Engine::query_strobes_host(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                                const uint64_t* offsets, uint64_t records, bool recover,
                                uint64_t* counts, uint64_t* total) {
  check(offsets[0] == 0 && offsets[records] == nbases, kEInval, "offsets must span the bases");
  const uint64_t colors = std::max<uint64_t>(m_.colors.size(), 1);
  const uint64_t step = std::max<uint64_t>(1, (32ull << 20) / colors);
  std::vector<uint64_t> c, t, rel;
  std::fill(counts, counts + m_.colors.size(), 0);
  *total = 0;
  for (uint64_t r0 = 0; r0 < records; r0 += step) {
    const uint64_t n = std::min(step, records - r0), b0 = offsets[r0];
    rel.resize(n + 1);
    for (uint64_t r = 0; r <= n; ++r) rel[r] = offsets[r0 + r] - b0;
    check(rel[n] <= nbases - b0, kEInval, "offsets must be non-decreasing");
    c.resize(n * m_.colors.size());
    t.resize(n);
    query_per_record(ws, bases + b0, rel[n], rel.data(), n, recover, c.data(), t.data());
    for (uint64_t r = 0; r < n; ++r) {
      *total += t[r];
      for (uint64_t i = 0; i < m_.colors.size(); ++i) counts[i] += c[r * m_.colors.size() + i];
    }
  }
}

void Engine::query_record_hits(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                               const uint64_t* offsets, uint64_t records, bool recover,
                               double min_ratio, RecordHits& out) {
  check(min_ratio > 0.0 && min_ratio <= 1.0, kEInval, "hit selection needs min_ratio in (0, 1]");
  const uint32_t colors = (uint32_t)m_.colors.size();
  cudaStream_t s = ws.stream;
  out.totals.assign(records, 0);
  out.first.assign(records + 1, 0);
  out.colors.clear();
  out.counts.clear();
  // Threshold pruning in the wide-row form: colours that cannot reach the
  // ratio may stop counting early (their counts stay below it).
  record_groups(ws, bases, nbases, offsets, records, recover, min_ratio,
                [&](uint64_t r0, uint64_t n) {
    const int grid = (int)std::min<uint64_t>((n + 7) / 8, (uint64_t)sms_ * 16);
    count_record_hits_kernel<<<grid, 256, 0, s>>>(ws.rec_counts, ws.rec_totals, n, colors,
                                                  min_ratio, ws.rec_hits);
    cuda_check(cudaGetLastError(), "count_record_hits_kernel");
    size_t tmp = ws.rec_scan_bytes;
    cuda_check(cub::DeviceScan::ExclusiveSum(ws.rec_scan_tmp, tmp, ws.rec_hits, ws.rec_first,
                                             (int)(n + 1), s),
               "scan");
    uint64_t hits = 0;
    cuda_check(cudaMemcpyAsync(&hits, ws.rec_first + n, 8, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "per-record hits");
    if (hits > ws.cap_hits || !ws.hit_colors) {
      if (ws.hit_colors) cudaFree(ws.hit_colors);
      if (ws.hit_counts) cudaFree(ws.hit_counts);
      ws.hit_colors = nullptr;
      ws.hit_counts = nullptr;
      const uint64_t cap = std::max<uint64_t>({hits, ws.cap_hits * 3 / 2, 4096});
      dev_alloc(&ws.hit_colors, cap, "record hits");
      dev_alloc(&ws.hit_counts, cap, "record hit counts");
      ws.cap_hits = cap;
    }
    if (hits)
      write_record_hits_kernel<<<grid, 256, 0, s>>>(ws.rec_counts, ws.rec_totals, n, colors,
                                                    min_ratio, ws.rec_first, ws.hit_colors,
                                                    ws.hit_counts);
    cuda_check(cudaGetLastError(), "write_record_hits_kernel");
    const uint64_t base = out.colors.size();
    out.colors.resize(base + hits);
    out.counts.resize(base + hits);
    if (hits) {
      cuda_check(cudaMemcpyAsync(out.colors.data() + base, ws.hit_colors, hits * 4,
                                 cudaMemcpyDeviceToHost, s),
                 "D2H");
      cuda_check(cudaMemcpyAsync(out.counts.data() + base, ws.hit_counts, hits * 8,
                                 cudaMemcpyDeviceToHost, s),
                 "D2H");
    }
    cuda_check(cudaMemcpyAsync(out.first.data() + r0, ws.rec_first, (n + 1) * 8,
                               cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaMemcpyAsync(out.totals.data() + r0, ws.rec_totals, n * 8,
                               cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaStreamSynchronize(s), "per-record hits");
    // Group-relative offsets to global ones (first[r0 + n] is the next group's base).
    for (uint64_t i = 0; i <= n; ++i) out.first[r0 + i] += base;
  });
}

static void raise_error_word(uint32_t err) {
  if (err & kErrOffsets)
    raise(kEInval, "record offsets must be non-decreasing, end within the bases and span fewer "
                   "than 2^31 bases (offending records were skipped; counts are incomplete)");
  if (err) raise(kETimeout, "a bounded device wait expired during the query");
}

void Engine::check_error_word(Workspace& ws) {
  uint32_t err = 0;
  cuda_check(cudaMemcpy(&err, ws.error, 4, cudaMemcpyDeviceToHost), "error word");
  if (err) {
    cuda_check(cudaMemset(ws.error, 0, 4), "memset");
    raise_error_word(err);
  }
}

uint32_t Engine::take_noalloc_error() {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  if (noalloc_slot_ < 0) return 0;
  uint32_t* err = static_cast<uint32_t*>(noalloc_scratch(device_)) + noalloc_slot_;
  uint32_t v = 0;
  cuda_check(cudaMemcpy(&v, err, 4, cudaMemcpyDeviceToHost), "error word");
  if (v) cuda_check(cudaMemset(err, 0, 4), "memset");
  return v;
}

uint32_t Engine::take_error(Workspace& ws) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  uint32_t err = 0;
  if (!ws.error) return 0;
  cuda_check(cudaMemcpy(&err, ws.error, 4, cudaMemcpyDeviceToHost), "error word");
  if (err) cuda_check(cudaMemset(ws.error, 0, 4), "memset");
  return err;
}

void Engine::query_device(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                          const uint64_t* offsets, uint64_t records, bool recover,
                          uint64_t* counts, unsigned long long* total, cudaStream_t s,
                          bool use_graph) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  check_not_strobes();
  ensure_capacity(ws, nbases, records);
  if (!use_graph) {
    enqueue(ws, bases, nbases, offsets, records, recover, counts, total, s);
    return;
  }
  auto key = std::make_tuple((const void*)bases, nbases, (const void*)offsets, records,
                             (void*)counts, (void*)total, (int)recover);
  auto it = ws.graphs.find(key);
  if (it == ws.graphs.end()) {
    cudaStream_t cap;
    cuda_check(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaGraph_t graph;
    cuda_check(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      enqueue(ws, bases, nbases, offsets, records, recover, counts, total, cap);
    } catch (...) {
      cudaStreamEndCapture(cap, &graph);
      cudaStreamDestroy(cap);
      throw;
    }
    cuda_check(cudaStreamEndCapture(cap, &graph), "end capture");
    cudaGraphExec_t exec;
    cuda_check(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
    cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    it = ws.graphs.emplace(key, exec).first;
  }
  cuda_check(cudaGraphLaunch(it->second, s), "graph launch");
}

void Engine::query_host(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                        const uint64_t* offsets, uint64_t records, bool recover, uint64_t* counts,
                        uint64_t* total) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  if (sp_.strobe_max) {
    query_strobes_host(ws, bases, nbases, offsets, records, recover, counts, total);
    return;
  }
  // Offsets are checked per record by the tile planner on the device
  // (kErrOffsets): a host pass over a million records cost about 1 ms.
  check(offsets[0] == 0 && offsets[records] == nbases, kEInval, "offsets must span the bases");
  // Chunks: record-aligned cuts near multiples of nbases / cut, at least
  // 1 MiB of bases each.
  const uint64_t min_chunk = 1ull << 20;
  uint64_t cut = std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)launch_.cut,
                                                          nbases / min_chunk));
  std::vector<uint64_t> bounds{0};  // record index of each chunk start, then records
  for (uint64_t c = 1; c < cut; ++c) {
    const uint64_t target = nbases / cut * c;
    const uint64_t r = (uint64_t)(std::lower_bound(offsets, offsets + records + 1, target) - offsets);
    if (r > bounds.back() && r < records) bounds.push_back(r);
  }
  bounds.push_back(records);
  const uint64_t chunks = bounds.size() - 1;
  // Chunk copies must stay inside the batch whatever the interior offsets.
  for (uint64_t c = 0; c < chunks; ++c)
    check(offsets[bounds[c]] <= offsets[bounds[c + 1]] && offsets[bounds[c + 1]] <= nbases, kEInval,
          "offsets must be non-decreasing");
  ensure_capacity(ws, nbases, records + chunks);
  ensure_host_capacity(ws, nbases, records + chunks);
  const uint64_t colors = m_.colors.size();
  cudaStream_t s = ws.stream;
  if (!ws.copy_stream)
    cuda_check(cudaStreamCreateWithFlags(&ws.copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  while (ws.chunk_events.size() < chunks) {
    cudaEvent_t e;
    cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    ws.chunk_events.push_back(e);
  }
  // The copy stream must not overwrite buffers the previous query still reads.
  cuda_check(cudaEventRecord(ws.chunk_events[0], s), "cudaEventRecord");
  cuda_check(cudaStreamWaitEvent(ws.copy_stream, ws.chunk_events[0], 0), "cudaStreamWaitEvent");
  // Page-locked caller bases are copied directly; pageable ones through the
  // workspace's pinned staging, chunk by chunk.
  auto pinned = [](const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return a.type == cudaMemoryTypeHost;
  };
  const bool direct = nbases && pinned(bases);
  const bool direct_offsets = pinned(offsets);
  cuda_check(cudaMemsetAsync(ws.counts, 0, colors * 8, s), "memset");
  cuda_check(cudaMemsetAsync(ws.total, 0, 8, s), "memset");
  for (uint64_t c = 0; c < chunks; ++c) {
    const uint64_t r0 = bounds[c], r1 = bounds[c + 1], b0 = offsets[r0], nb = offsets[r1] - b0;
    // The chunk's records + 1 absolute offsets, made chunk-relative on the
    // device after the copy.
    const uint64_t* h_off = offsets + r0;
    if (!direct_offsets) {
      memcpy(ws.h_offsets + r0 + c, offsets + r0, (r1 - r0 + 1) * 8);
      h_off = ws.h_offsets + r0 + c;
    }
    const uint8_t* src = bases + b0;
    if (!direct && nb) {
      memcpy(ws.h_bases + b0, bases + b0, nb);
      src = ws.h_bases + b0;
    }
    if (nb)
      cuda_check(cudaMemcpyAsync(ws.bases + b0, src, nb, cudaMemcpyHostToDevice, ws.copy_stream),
                 "H2D");
    cuda_check(cudaMemcpyAsync(ws.offsets + r0 + c, h_off, (r1 - r0 + 1) * 8,
                               cudaMemcpyHostToDevice, ws.copy_stream),
               "H2D");
    if (b0) {
      const uint64_t n = r1 - r0 + 1;
      rebase_offsets_kernel<<<(int)std::min<uint64_t>((n + 255) / 256, (uint64_t)sms_ * 4), 256, 0,
                              ws.copy_stream>>>(ws.offsets + r0 + c, n, b0);
      cuda_check(cudaGetLastError(), "rebase_offsets_kernel");
    }
    cuda_check(cudaEventRecord(ws.chunk_events[c], ws.copy_stream), "cudaEventRecord");
    cuda_check(cudaStreamWaitEvent(s, ws.chunk_events[c], 0), "cudaStreamWaitEvent");
    enqueue(ws, ws.bases + b0, nb, ws.offsets + r0 + c, r1 - r0, recover, ws.counts, ws.total, s);
  }
  cuda_check(cudaMemcpyAsync(ws.h_counts, ws.counts, colors * 8, cudaMemcpyDeviceToHost, s), "D2H");
  cuda_check(cudaMemcpyAsync(ws.h_total, ws.total, 8, cudaMemcpyDeviceToHost, s), "D2H");
  cuda_check(cudaStreamSynchronize(s), "query");
  check_error_word(ws);
  memcpy(counts, ws.h_counts, colors * 8);
  *total = *ws.h_total;
}

void Engine::query_host_plain(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                              const uint64_t* offsets, uint64_t records, bool recover,
                              uint64_t* counts, uint64_t* total) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  if (sp_.strobe_max) {
    query_strobes_host(ws, bases, nbases, offsets, records, recover, counts, total);
    return;
  }
  check(offsets[0] == 0 && offsets[records] == nbases, kEInval, "offsets must span the bases");
  for (uint64_t r = 0; r < records; ++r)  // records are sliced on the host here
    check(offsets[r] <= offsets[r + 1], kEInval, "offsets must be non-decreasing");
  ensure_capacity(ws, nbases, records);
  ensure_host_capacity(ws, nbases, records);
  const uint64_t colors = m_.colors.size();
  cudaStream_t s = ws.stream;
  memcpy(ws.h_bases, bases, nbases);
  cuda_check(cudaMemcpyAsync(ws.bases, ws.h_bases, nbases, cudaMemcpyHostToDevice, s), "H2D");
  cuda_check(cudaMemsetAsync(ws.counts, 0, colors * 8, s), "memset");
  cuda_check(cudaMemsetAsync(ws.total, 0, 8, s), "memset");
  // One record per launch sequence, default tiles: each record is its own batch.
  for (uint64_t r = 0; r < records; ++r) {
    ws.h_offsets[2 * (r % 2)] = 0;
    ws.h_offsets[2 * (r % 2) + 1] = offsets[r + 1] - offsets[r];
    uint64_t* d_off = ws.offsets + 2 * (r % 2);
    cuda_check(cudaMemcpyAsync(d_off, ws.h_offsets + 2 * (r % 2), 16, cudaMemcpyHostToDevice, s),
               "H2D");
    enqueue(ws, ws.bases + offsets[r], offsets[r + 1] - offsets[r], d_off, 1, recover, ws.counts,
            ws.total, s);
    if (r % 2 == 1) cuda_check(cudaStreamSynchronize(s), "plain query");
  }
  cuda_check(cudaMemcpyAsync(ws.h_counts, ws.counts, colors * 8, cudaMemcpyDeviceToHost, s), "D2H");
  cuda_check(cudaMemcpyAsync(ws.h_total, ws.total, 8, cudaMemcpyDeviceToHost, s), "D2H");
  cuda_check(cudaStreamSynchronize(s), "plain query");
  check_error_word(ws);
  memcpy(counts, ws.h_counts, colors * 8);
  *total = *ws.h_total;
}

void Engine::extract_host(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                          const uint64_t* offsets, uint64_t records, std::vector<uint64_t>& keys) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  check(offsets[0] == 0 && offsets[records] == nbases, kEInval, "offsets must span the bases");
  check(m_.index_mode != kFindere, kEUnsupported,
        "seed extraction output is defined for k-mer, minimizer and modimizer indexes");
  ensure_capacity(ws, nbases, records);
  ensure_host_capacity(ws, nbases, records);
  cudaStream_t s = ws.stream;
  memcpy(ws.h_bases, bases, nbases);
  memcpy(ws.h_offsets, offsets, (records + 1) * 8);
  cuda_check(cudaMemcpyAsync(ws.bases, ws.h_bases, nbases, cudaMemcpyHostToDevice, s), "H2D");
  cuda_check(cudaMemcpyAsync(ws.offsets, ws.h_offsets, (records + 1) * 8, cudaMemcpyHostToDevice, s),
             "H2D");
  const uint8_t* d_bases = ws.bases;
  const uint64_t* d_offsets = ws.offsets;
  if (m_.homopolymer_compression) compress_homopolymers(ws, d_bases, nbases, d_offsets, records, s);
  const uint64_t words = nbases / 32 + 2;
  pack_kernel<<<std::max<int>(1, (int)std::min<uint64_t>((words + 255) / 256, sms_ * 16ull)), 256, 0, s>>>(
      d_bases, nbases, ws.packed, ws.invalid, words);
  cuda_check(cudaGetLastError(), "pack_kernel");
  plan_tiles(ws, d_offsets, records, nbases, s);
  uint32_t ntiles = 0;
  cuda_check(cudaMemcpyAsync(&ntiles, ws.tile_first + records, 4, cudaMemcpyDeviceToHost, s), "D2H");
  cuda_check(cudaStreamSynchronize(s), "tiles");
  if (ntiles == 0) {
    keys.clear();
    return;
  }
  if (sp_.strobe_max) {
    // Randstrobemer seeds of the forward strand, records and positions in order.
    ensure_strobe_capacity(ws, nbases, ntiles);
    BatchView bv{PackedView{ws.packed, ws.invalid}, d_offsets, ws.tiles, ws.tile_first + records,
                 nullptr};
    link_strobes(ws, bv, nbases, s);
    std::vector<uint64_t> all((uint64_t)ntiles * kStrobeSlot);
    std::vector<uint32_t> cnt(ntiles);
    cuda_check(cudaMemcpyAsync(all.data(), ws.strobe_slots, all.size() * 8, cudaMemcpyDeviceToHost,
                               s),
               "D2H");
    cuda_check(cudaMemcpyAsync(cnt.data(), ws.strobe_count, ntiles * 4ull, cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaStreamSynchronize(s), "extract");
    check_error_word(ws);
    keys.clear();
    for (uint32_t t = 0; t < ntiles; ++t)
      keys.insert(keys.end(), all.begin() + (uint64_t)t * kStrobeSlot,
                  all.begin() + (uint64_t)t * kStrobeSlot + cnt[t]);
    return;
  }
  uint64_t need = (uint64_t)ntiles * kTileWindows;
  if (need > ws.cap_keys) {
    if (ws.keys_out) cudaFree(ws.keys_out);
    if (ws.keys_count) cudaFree(ws.keys_count);
    dev_alloc(&ws.keys_out, need, "extracted keys");
    dev_alloc(&ws.keys_count, ntiles, "extracted counts");
    ws.cap_keys = need;
  }
  const int warps = 4;
  size_t smem = 256 * 8 + warps * FusedSmem::warp_bytes(sp_.mode, sp_.k, 0, 0, 0, 4, 0, 0,
                                                        sp_.strobe_max != 0);
  ExtractFn efn = extract_for(sp_.mode);
  cudaFuncSetAttribute(efn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  BatchView bv{PackedView{ws.packed, ws.invalid}, d_offsets, ws.tiles, ws.tile_first + records,
               nullptr};
  int grid = (int)std::min<uint64_t>((ntiles + warps - 1) / warps, (uint64_t)sms_ * 8);
  efn<<<grid, warps * 32, smem, s>>>(bv, sp_, ws.keys_out, ws.keys_count, warps);
  cuda_check(cudaGetLastError(), "extract_kernel");
  std::vector<uint64_t> all(need);
  std::vector<uint32_t> cnt(ntiles);
  cuda_check(cudaMemcpyAsync(all.data(), ws.keys_out, need * 8, cudaMemcpyDeviceToHost, s), "D2H");
  cuda_check(cudaMemcpyAsync(cnt.data(), ws.keys_count, ntiles * 4ull, cudaMemcpyDeviceToHost, s),
             "D2H");
  cuda_check(cudaStreamSynchronize(s), "extract");
  check_error_word(ws);
  keys.clear();
  for (uint32_t t = 0; t < ntiles; ++t)
    keys.insert(keys.end(), all.begin() + (uint64_t)t * kTileWindows,
                all.begin() + (uint64_t)t * kTileWindows + cnt[t]);
}

}  // namespace zx
