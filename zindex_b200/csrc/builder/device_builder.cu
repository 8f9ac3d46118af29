// Index construction on the GPU (zx_build --device): the same index directory
// as the host builder (builder.cpp), built with the device doing the work that
// grows with the collection.
//
// Per batch of datasets: the genomes are generated in place (synthetic
// collections; synth.h's generator is host/device code) or copied in, and the
// query path's kernels pack them and cut them into tiles; every tile's seeds
// are appended to its dataset's own region (an atomic cursor per dataset), a
// radix sort per dataset and a block-per-dataset compaction give the distinct
// keys (scan_index_features + sort/dedup of storage.rs:500-882). A first pass
// only counts them (unique_kmers, which fixes the bank layout: BuildConfig::
// slots, mod.rs:319-337, promotion and partitions, shared with the host
// builder); the second pass builds the filters.
//
// Filters (one per dataset and hash partition) are built as the reference's
// ZOR construction builds them (zorindex.rs:634-841): every key's H cells of
// PositionHash are counted and XORed into the cell arrays (one device pass
// over all keys), then ONE DEVICE THREAD PER FILTER peels the hypergraph —
// pop a cell of degree one, take its key, remove the key from its cells —
// over keys sorted by their first segment, so the cells a thread touches
// stay within a window of H segments and the peel moves along the filter like
// a wave. When no cell of degree one is left the thread abandons the first
// key still active in that order (the reference abandons the first active key
// of a minimum-degree cell; any choice gives a valid index, and on segment-
// sorted keys this one abandons fewer keys: 0.5 % instead of 0.8 % at load
// 0.9 with H = 8 in a CPU experiment), and the abandoned keys go to the
// recovery file with their dataset. Cells are then assigned in reverse peel
// order (value = fingerprint XOR the key's other cells) and packed into the
// fingerprint-first rows (pack_ram_rows, storage.rs:1721-1754) with atomic
// ORs. Every loop is bounded; a bound that trips sets an error word and the
// build fails.
//
// Scope: singleton groups (no --groups), k-mer, minimizer and modimizer
// indexes, with or without a spaced-seed pattern; no homopolymer compression,
// randstrobemers or legacy layout (the host builder covers those).
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/block/block_scan.cuh>
#include <thread>

#include "../host/error.h"
#include "../host/fastx.h"
#include "../kernels/query_kernels.cuh"
#include "../zx_hash.h"
#include "builder_internal.h"
#include "synth.h"

namespace zx {
namespace {

using build::Context;

void cu(cudaError_t e, const char* what) {
  if (e != cudaSuccess) raise(kECuda, std::string(what) + ": " + cudaGetErrorString(e));
}

// Device buffer that grows (never shrinks) and frees itself.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  void need(size_t count, const char* what) {
    if (count <= n && p) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) {
      cudaGetLastError();
      raise(kENoMem, std::string("device allocation failed for ") + what);
    }
    n = std::max<size_t>(count, 1);
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

// Builder error bits (beside the tile planner's kErrOffsets).
constexpr uint32_t kErrPeel = 8u, kErrQueue = 16u, kErrKey = 32u;

// Synthetic genomes of a batch: base i belongs to the dataset d with
// start[d] <= i < start[d + 1]; genome[d] is its genome number.
__global__ void synth_kernel(bool pool, uint64_t seed, const uint64_t* __restrict__ start,
                             const uint64_t* __restrict__ genome, uint32_t datasets,
                             uint64_t nbases, uint8_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nbases;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = datasets;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (start[mid] <= i) lo = mid;
      else hi = mid;
    }
    out[i] = (uint8_t)synth::synth_base(pool, seed, genome[lo], i - start[lo]);
  }
}

// Seeds of every tile appended to its dataset's region: region[d] + cursor[d].
template <int MODE>
__global__ void extract_region_kernel(BatchView bv, SeedParams sp,
                                      const uint32_t* __restrict__ rec_dataset,
                                      const uint64_t* __restrict__ region,
                                      unsigned long long* __restrict__ cursor,
                                      uint64_t* __restrict__ out, int warps_per_block) {
  extern __shared__ __align__(16) uint8_t smem[];
  uint64_t* inner = reinterpret_cast<uint64_t*>(smem);
  uint8_t* p = smem + 256 * 8;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t* wbase = p + (size_t)warp * FusedSmem::warp_bytes(MODE, sp.k, 0, 0, 0, 4, 0, 0, false);
  uint64_t* keys = reinterpret_cast<uint64_t*>(wbase);
  uint8_t* ocm = wbase + FusedSmem::key_bytes(MODE, sp.k, false) + FusedSmem::probe_bytes(0);
  build_inner_table(sp, inner);
  __syncthreads();
  const uint32_t ntiles = *bv.ntiles;
  const uint32_t warps_total = gridDim.x * warps_per_block;
  for (uint32_t t = blockIdx.x * warps_per_block + warp; t < ntiles; t += warps_total) {
    const Tile tile = bv.tiles[t];
    const uint32_t n = extract_tile<MODE>(bv, sp, tile, keys, ocm, inner, lane);
    __syncwarp();
    const uint32_t d = rec_dataset[tile.record];
    unsigned long long at = 0;
    if (lane == 0 && n) at = atomicAdd(cursor + d, (unsigned long long)n);
    at = __shfl_sync(0xFFFFFFFFu, at, 0);
    for (uint32_t i = lane; i < n; i += 32) out[region[d] + at + i] = keys[i];
    __syncwarp();
  }
}

// One block per dataset: distinct keys of its sorted region. counts[d]
// receives their number; with `out`, they are written to out[dense[d]...].
template <int THREADS>
__global__ void unique_kernel(const uint64_t* __restrict__ sorted, const uint64_t* __restrict__ region,
                              const unsigned long long* __restrict__ cursor,
                              const uint64_t* __restrict__ dense, uint64_t* __restrict__ counts,
                              uint64_t* __restrict__ out) {
  using Scan = cub::BlockScan<uint32_t, THREADS>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ uint64_t running;
  const uint32_t d = blockIdx.x;
  const uint64_t a = region[d], n = cursor[d];
  if (threadIdx.x == 0) running = 0;
  __syncthreads();
  for (uint64_t c0 = 0; c0 < n; c0 += THREADS) {
    const uint64_t i = c0 + threadIdx.x;
    uint32_t flag = 0;
    uint64_t k = 0;
    if (i < n) {
      k = sorted[a + i];
      flag = i == 0 || sorted[a + i - 1] != k;
    }
    uint32_t rank = 0, sum = 0;
    Scan(tmp).ExclusiveSum(flag, rank, sum);
    if (out && flag) out[dense[d] + running + rank] = k;
    __syncthreads();
    if (threadIdx.x == 0) running += sum;
    __syncthreads();
  }
  if (threadIdx.x == 0) counts[d] = running;
}

// Sort key of each distinct key: partition << 32 | first segment, so a
// dataset's keys fall into its partitions' filters, each in segment order.
__global__ void order_kernel(const uint64_t* __restrict__ keys, uint64_t n,
                             const uint64_t* __restrict__ dense, const uint32_t* __restrict__ parts,
                             const uint64_t* __restrict__ local_slots, uint32_t datasets,
                             uint64_t seed, int H, uint64_t seg, uint64_t* __restrict__ order,
                             unsigned long long* __restrict__ hist, uint32_t max_parts) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = datasets;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (dense[mid] <= i) lo = mid;
      else hi = mid;
    }
    const uint64_t key = keys[i];
    const uint32_t P = parts[lo];
    const uint32_t p = P > 1 ? partition_id(key, seed, P) : 0;
    const uint64_t count = local_slots[lo] / seg - (uint64_t)H + 1;
    const uint64_t base = mulhi64(mixsplit(key, seed), count);
    order[i] = ((uint64_t)p << 32) | base;
    atomicAdd(hist + (uint64_t)lo * max_parts + p, 1ull);
  }
}

struct Filter {
  uint64_t key0;      // first key in the batch's filter-ordered key array
  uint64_t cell0;     // first cell in the arena
  uint8_t* rows;      // payload of the filter's (class, partition)
  uint32_t nkeys;
  uint32_t slots;     // cells (local slots)
  uint32_t row_bytes;
  uint32_t column;
  uint32_t dataset;   // global dataset id
  uint32_t pad;
};

__device__ __forceinline__ uint32_t filter_of(const Filter* f, uint32_t nf, uint64_t i, bool cells) {
  uint32_t lo = 0, hi = nf;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if ((cells ? f[mid].cell0 : f[mid].key0) <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Degrees and key-index XORs of every cell.
__global__ void accumulate_kernel(const Filter* __restrict__ f, uint32_t nf,
                                  const uint64_t* __restrict__ keys, uint64_t n, uint64_t seed,
                                  int H, uint64_t seg, uint32_t* __restrict__ deg,
                                  uint32_t* __restrict__ xr) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const Filter F = f[filter_of(f, nf, i, false)];
    const uint32_t e = (uint32_t)(i - F.key0);
    uint64_t pos[kMaxHashes];
    positions(keys[i], seed, F.slots, H, seg, pos);
    for (int h = 0; h < H; ++h) {
      atomicAdd(deg + F.cell0 + pos[h], 1u);
      atomicXor(xr + F.cell0 + pos[h], e);
    }
  }
}

// One thread per filter: peel in segment order, abandoning the first active
// key whenever no cell of degree one is left. stack[key0 + j] = (key, cell)
// in peel order, cell ~0 for an abandoned key.
__global__ void peel_kernel(const Filter* __restrict__ f, uint32_t nf,
                            const uint64_t* __restrict__ keys, uint64_t seed, int H, uint64_t seg,
                            uint32_t* __restrict__ deg, uint32_t* __restrict__ xr,
                            uint32_t* __restrict__ queue, uint8_t* __restrict__ state,
                            uint2* __restrict__ stack, uint32_t* __restrict__ abandoned,
                            uint32_t* __restrict__ err) {
  const uint32_t fi = blockIdx.x * blockDim.x + threadIdx.x;
  if (fi >= nf) return;
  const Filter F = f[fi];
  uint32_t* D = deg + F.cell0;
  uint32_t* X = xr + F.cell0;
  uint32_t* Q = queue + F.cell0;
  const uint64_t* K = keys + F.key0;
  uint8_t* S = state + F.key0;
  uint2* ST = stack + F.key0;
  const uint32_t n = F.nkeys, M = F.slots;
  uint32_t top = 0;
  for (uint32_t s = 0; s < M; ++s)
    if (D[s] == 1) Q[top++] = s;
  uint32_t sp = 0, cursor = 0, nab = 0;
  const uint64_t limit = 2ull * ((uint64_t)M + n) + 64;
  uint64_t pos[kMaxHashes];
  for (uint64_t it = 0; sp < n; ++it) {
    if (it > limit) {
      atomicOr(err, kErrPeel);
      break;
    }
    uint32_t e;
    if (top) {
      const uint32_t s = Q[--top];
      if (D[s] != 1) continue;
      e = X[s];
      if (e >= n || S[e]) {
        atomicOr(err, kErrKey);
        break;
      }
      S[e] = 1;
      ST[sp++] = make_uint2(e, s);
    } else {
      while (cursor < n && S[cursor]) ++cursor;
      if (cursor >= n) {
        atomicOr(err, kErrKey);
        break;
      }
      e = cursor;
      S[e] = 2;
      ST[sp++] = make_uint2(e, 0xFFFFFFFFu);
      ++nab;
    }
    positions(K[e], seed, M, H, seg, pos);
    // A key's H cells lie in H different segments, so they are distinct: the
    // degrees and XORs of 8 cells are loaded together, then updated.
    bool full = false;
    for (int h0 = 0; h0 < H && !full; h0 += 8) {
      uint32_t dv[8], xv[8], tv[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        tv[i] = h0 + i < H ? (uint32_t)pos[h0 + i] : 0u;
        if (h0 + i < H) {
          dv[i] = D[tv[i]];
          xv[i] = X[tv[i]];
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if (h0 + i >= H) continue;
        X[tv[i]] = xv[i] ^ e;
        D[tv[i]] = dv[i] - 1;
        if (dv[i] == 2) {
          if (top >= M) {
            full = true;
            break;
          }
          Q[top++] = tv[i];
        }
      }
    }
    if (full) {
      atomicOr(err, kErrQueue);
      break;
    }
  }
  abandoned[fi] = nab;
}

// One thread per filter: cell values in reverse peel order (the cell array
// is the degree array, zero after the peel).
__global__ void assign_kernel(const Filter* __restrict__ f, uint32_t nf,
                              const uint64_t* __restrict__ keys, uint64_t seed, int H, uint64_t seg,
                              int bits, uint32_t* __restrict__ cells,
                              const uint2* __restrict__ stack) {
  const uint32_t fi = blockIdx.x * blockDim.x + threadIdx.x;
  if (fi >= nf) return;
  const Filter F = f[fi];
  uint32_t* C = cells + F.cell0;
  const uint64_t* K = keys + F.key0;
  const uint2* ST = stack + F.key0;
  uint64_t pos[kMaxHashes];
  for (uint32_t j = F.nkeys; j-- > 0;) {
    const uint2 es = ST[j];
    if (es.y == 0xFFFFFFFFu) continue;
    const uint64_t key = K[es.x];
    uint32_t v = (uint32_t)fingerprint(key, seed, bits);
    positions(key, seed, F.slots, H, seg, pos);
    // The key's cells are distinct: 8 of them are loaded together.
    for (int h0 = 0; h0 < H; h0 += 8) {
      uint32_t cv[8];
#pragma unroll
      for (int i = 0; i < 8; ++i)
        cv[i] = h0 + i < H && (uint32_t)pos[h0 + i] != es.y ? C[pos[h0 + i]] : 0u;
#pragma unroll
      for (int i = 0; i < 8; ++i) v ^= cv[i];
    }
    C[es.y] = v;
  }
}

// Cell values ORed into the rows: b bits at row s, bit column * b.
__global__ void pack_rows_kernel(const Filter* __restrict__ f, uint32_t nf, uint64_t ncells,
                                 const uint32_t* __restrict__ cells, int bits) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ncells;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = cells[i];
    if (!v) continue;
    const Filter F = f[filter_of(f, nf, i, true)];
    const uint64_t s = i - F.cell0;
    const uint64_t bit = s * F.row_bytes * 8 + (uint64_t)F.column * bits;
    uint32_t* w = reinterpret_cast<uint32_t*>(F.rows) + (bit >> 5);
    const uint32_t sh = (uint32_t)(bit & 31);
    atomicOr(w, v << sh);
    if (sh + bits > 32) atomicOr(w + 1, v >> (32 - sh));
  }
}

// Abandoned keys -> (recovery hash, dataset) at out[first[filter] + k].
__global__ void abandoned_kernel(const Filter* __restrict__ f, uint32_t nf, uint64_t n,
                                 const uint64_t* __restrict__ keys, const uint2* __restrict__ stack,
                                 uint64_t seed, const uint64_t* __restrict__ first,
                                 unsigned int* __restrict__ fill, uint2* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 es = stack[i];
    if (es.y != 0xFFFFFFFFu) continue;
    const uint32_t fi = filter_of(f, nf, i, false);
    const Filter& F = f[fi];
    const uint32_t at = atomicAdd(fill + fi, 1u);
    out[first[fi] + at] = make_uint2(recovery_hash(keys[F.key0 + es.x], seed), F.dataset);
  }
}

int grid_for(uint64_t n, int sms) {
  return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 16));
}

struct Batch {
  uint32_t d0 = 0, d1 = 0;  // datasets [d0, d1)
  uint64_t bases = 0;
};

// The device side of one pass over the datasets.
class DeviceBuilder {
 public:
  DeviceBuilder(Context& bc) : bc_(bc) {
    cu(cudaSetDevice(bc.opt.gpu), "cudaSetDevice");
    cudaDeviceProp prop;
    cu(cudaGetDeviceProperties(&prop, bc.opt.gpu), "cudaGetDeviceProperties");
    sms_ = prop.multiProcessorCount;
    cu(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking), "cudaStreamCreate");
    const FeatureParams& fp = bc.fp;
    sp_ = SeedParams{};
    sp_.mode = fp.mode;
    sp_.k = fp.k;
    sp_.m = fp.m;
    sp_.klen = fp.k;
    sp_.seed = fp.seed;
    sp_.sampling = fp.sampling;
    sp_.ocm = fp.mode == 1 && fp.k != fp.m ? ocm_params(fp.k, fp.m) : OcmParams{1, fp.m, 1};
    if (sp_.klen > 32) sp_.lk = long_kmer_consts(sp_.klen);
    sp_.spaced = fp.spaced ? 1 : 0;
    if (fp.spaced) sp_.pattern = fp.pattern;
    err_.need(1, "error word");
    cu(cudaMemset(err_.p, 0, 4), "memset");
  }
  ~DeviceBuilder() {
    if (s_) cudaStreamDestroy(s_);
  }

  // Seconds per build phase, summed over batches (measured at stream
  // synchronisations when the build is not quiet).
  enum Phase { kExtract, kSort, kUnique, kOrder, kAccumulate, kPeel, kPack, kAbandoned, kPhases };
  void report(FILE* f) const {
    static const char* names[kPhases] = {"extract", "sort", "unique", "order", "accumulate",
                                         "peel", "assign+pack", "abandoned"};
    fprintf(f, "device phases:");
    for (int i = 0; i < kPhases; ++i) fprintf(f, " %s %.2fs", names[i], phase_[i]);
    fprintf(f, "\n");
  }

  // Bases of dataset d (its records' bases for file inputs).
  uint64_t dataset_bases(uint32_t d) {
    if (!bc_.opt.synth.empty()) return synth::genome_length(bc_.spec, d);
    return file_batch(d).bases.size();
  }

  // Extracts, sorts and deduplicates the seeds of datasets [d0, d1): unique
  // counts in `unique`, occurrences in `occ`; with `dense_out`, the distinct
  // keys are left in raw_ at batch-relative dense offsets (dense_start of the
  // dataset minus that of the batch's first dataset), datasets in order.
  void distinct(const Batch& b, std::vector<uint64_t>& unique, std::vector<uint64_t>& occ,
                bool dense_out, const std::vector<uint64_t>* dense_start) {
    const uint32_t nd = b.d1 - b.d0;
    tick();
    // Records: one per synthetic genome; the files' records otherwise.
    std::vector<uint64_t> rec_off{0}, region(nd + 1, 0), genome(nd);
    std::vector<uint32_t> rec_ds;
    bases_.need(b.bases + 64, "bases");
    const bool synth = !bc_.opt.synth.empty();
    for (uint32_t j = 0; j < nd; ++j) {
      const uint32_t d = b.d0 + j;
      genome[j] = d;
      if (synth) {
        region[j + 1] = region[j] + synth::genome_length(bc_.spec, d);
        rec_off.push_back(region[j + 1]);
        rec_ds.push_back(j);
      } else {
        const RecordBatch& rb = file_batch(d);
        cu(cudaMemcpyAsync(bases_.p + region[j], rb.bases.data(), rb.bases.size(),
                           cudaMemcpyHostToDevice, s_),
           "H2D");
        for (size_t r = 0; r < rb.records(); ++r) {
          rec_off.push_back(region[j] + rb.offsets[r + 1]);
          rec_ds.push_back(j);
        }
        region[j + 1] = region[j] + rb.bases.size();
      }
    }
    const uint64_t nbases = region[nd];
    const uint64_t records = rec_ds.size();
    check(nbases == b.bases, kEInval, "batch size mismatch");
    d_region_.need(nd + 1, "regions");
    d_genome_.need(nd, "genomes");
    d_rec_off_.need(records + 1, "record offsets");
    d_rec_ds_.need(std::max<uint64_t>(records, 1), "record datasets");
    cu(cudaMemcpyAsync(d_region_.p, region.data(), (nd + 1) * 8, cudaMemcpyHostToDevice, s_), "H2D");
    cu(cudaMemcpyAsync(d_genome_.p, genome.data(), nd * 8, cudaMemcpyHostToDevice, s_), "H2D");
    cu(cudaMemcpyAsync(d_rec_off_.p, rec_off.data(), (records + 1) * 8, cudaMemcpyHostToDevice, s_),
       "H2D");
    if (records)
      cu(cudaMemcpyAsync(d_rec_ds_.p, rec_ds.data(), records * 4, cudaMemcpyHostToDevice, s_), "H2D");
    if (synth) {
      synth_kernel<<<grid_for(nbases, sms_), 256, 0, s_>>>(bc_.spec.kind != "uniform", bc_.spec.seed,
                                                          d_region_.p, d_genome_.p, nd, nbases,
                                                          bases_.p);
      cu(cudaGetLastError(), "synth_kernel");
    }
    // Pack and tile plan (the query path's kernels).
    const uint64_t words = nbases / 32 + 2;
    packed_.need(words, "packed bases");
    invalid_.need(words, "invalid masks");
    pack_kernel<<<grid_for(words, sms_), 256, 0, s_>>>(bases_.p, nbases, packed_.p, invalid_.p, words);
    cu(cudaGetLastError(), "pack_kernel");
    tile_counts_.need(records + 1, "tile counts");
    tile_first_.need(records + 1, "tile offsets");
    cu(cudaMemsetAsync(tile_counts_.p + records, 0, 4, s_), "memset");
    if (records)
      count_tiles_kernel<<<grid_for(records, sms_), 256, 0, s_>>>(d_rec_off_.p, records, nbases,
                                                                  bc_.fp.k, 0, tile_counts_.p, err_.p);
    size_t tmp = 0;
    cu(cub::DeviceScan::ExclusiveSum(nullptr, tmp, tile_counts_.p, tile_first_.p, (int)(records + 1)),
       "scan size");
    scan_tmp_.need(tmp, "scan scratch");
    cu(cub::DeviceScan::ExclusiveSum(scan_tmp_.p, tmp, tile_counts_.p, tile_first_.p,
                                     (int)(records + 1), s_),
       "tile scan");
    uint32_t ntiles = 0;
    cu(cudaMemcpyAsync(&ntiles, tile_first_.p + records, 4, cudaMemcpyDeviceToHost, s_), "D2H");
    cu(cudaStreamSynchronize(s_), "tile plan");
    tiles_.need(std::max<uint32_t>(ntiles, 1), "tiles");
    if (records)
      fill_tiles_kernel<<<grid_for(records, sms_), 256, 0, s_>>>(d_rec_off_.p, records, nbases,
                                                                 bc_.fp.k, tile_first_.p, tiles_.p);
    // Seeds into each dataset's region (capacity: its bases).
    raw_.need(nbases + 1, "seed regions");
    sorted_.need(nbases + 1, "sorted seeds");
    cursor_.need(nd, "cursors");
    cu(cudaMemsetAsync(cursor_.p, 0, nd * 8, s_), "memset");
    BatchView bv{};
    bv.pv = PackedView{packed_.p, invalid_.p};
    bv.offsets = d_rec_off_.p;
    bv.tiles = tiles_.p;
    bv.ntiles = tile_first_.p + records;
    const int ewarps = 4;
    const size_t esmem = 256 * 8 + ewarps * FusedSmem::warp_bytes(sp_.mode, sp_.k, 0);
    auto efn = sp_.mode == 1 ? extract_region_kernel<1>
                             : (sp_.mode == 2 ? extract_region_kernel<2> : extract_region_kernel<0>);
    cu(cudaFuncSetAttribute(efn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)esmem),
       "cudaFuncSetAttribute");
    efn<<<std::max(1, std::min<int>((int)((ntiles + ewarps - 1) / ewarps), sms_ * 8)), ewarps * 32,
          esmem, s_>>>(bv, sp_, d_rec_ds_.p, d_region_.p, cursor_.p, raw_.p, ewarps);
    cu(cudaGetLastError(), "extract_region_kernel");
    std::vector<unsigned long long> cur(nd);
    cu(cudaMemcpyAsync(cur.data(), cursor_.p, nd * 8, cudaMemcpyDeviceToHost, s_), "D2H");
    cu(cudaStreamSynchronize(s_), "extraction");
    tock(kExtract);
    // Radix sort of each dataset's region.
    uint64_t largest = 1;
    for (auto c : cur) largest = std::max<uint64_t>(largest, c);
    check(largest < (1ull << 31), kEUnsupported, "a dataset of 2^31 seeds or more");
    size_t sbytes = 0;
    cu(cub::DeviceRadixSort::SortKeys(nullptr, sbytes, raw_.p, sorted_.p, (int)largest), "sort size");
    sort_tmp_.need(sbytes, "sort scratch");
    for (uint32_t j = 0; j < nd; ++j) {
      if (!cur[j]) continue;
      size_t bytes = sort_tmp_.n;
      cu(cub::DeviceRadixSort::SortKeys(sort_tmp_.p, bytes, raw_.p + region[j],
                                        sorted_.p + region[j], (int)cur[j], 0, 64, s_),
         "sort");
    }
    tock(kSort);
    d_counts_.need(nd, "counts");
    d_dense_.need(nd + 1, "dense offsets");
    std::vector<uint64_t> local_dense(nd, 0);
    if (dense_out) {
      for (uint32_t j = 0; j < nd; ++j)
        local_dense[j] = (*dense_start)[b.d0 + j] - (*dense_start)[b.d0];
      cu(cudaMemcpyAsync(d_dense_.p, local_dense.data(), nd * 8, cudaMemcpyHostToDevice, s_), "H2D");
    }
    unique_kernel<256><<<nd, 256, 0, s_>>>(sorted_.p, d_region_.p, cursor_.p, d_dense_.p,
                                           d_counts_.p, dense_out ? raw_.p : nullptr);
    cu(cudaGetLastError(), "unique_kernel");
    std::vector<uint64_t> cnt(nd);
    cu(cudaMemcpyAsync(cnt.data(), d_counts_.p, nd * 8, cudaMemcpyDeviceToHost, s_), "D2H");
    cu(cudaStreamSynchronize(s_), "unique");
    tock(kUnique);
    for (uint32_t j = 0; j < nd; ++j) {
      unique[b.d0 + j] = cnt[j];
      occ[b.d0 + j] = cur[j];
    }
    check_error();
  }

  // Builds the filters of datasets [d0, d1) (distinct keys dense in raw_, from
  // distinct(..., dense_out)) and packs them into the device rows.
  void construct(const Batch& b, const std::vector<uint64_t>& dense_start,
                 const std::vector<std::vector<uint8_t*>>& rows) {
    auto& groups = bc_.groups;
    auto& classes = bc_.classes;
    const uint32_t nd = b.d1 - b.d0;
    const uint64_t k0 = dense_start[b.d0], n = dense_start[b.d1] - k0;
    const int H = bc_.H;
    const uint64_t seg = bc_.opt.segment_length, seed = bc_.fp.seed;
    if (!n) return;
    tick();
    // Per-dataset filter geometry.
    std::vector<uint64_t> dense(nd + 1), local(nd);
    std::vector<uint32_t> parts(nd);
    uint32_t maxp = 1;
    for (uint32_t j = 0; j < nd; ++j) {
      const build::Group& g = groups[b.d0 + j];
      const build::ClassLayout& cl = classes[g.cls];
      dense[j] = dense_start[b.d0 + j] - k0;
      local[j] = cl.local_slots;
      parts[j] = (uint32_t)cl.partitions;
      maxp = std::max(maxp, parts[j]);
    }
    dense[nd] = n;
    d_dense_.need(nd + 1, "dense offsets");
    d_local_.need(nd, "slots");
    d_parts_.need(nd, "partitions");
    cu(cudaMemcpyAsync(d_dense_.p, dense.data(), (nd + 1) * 8, cudaMemcpyHostToDevice, s_), "H2D");
    cu(cudaMemcpyAsync(d_local_.p, local.data(), nd * 8, cudaMemcpyHostToDevice, s_), "H2D");
    cu(cudaMemcpyAsync(d_parts_.p, parts.data(), nd * 4, cudaMemcpyHostToDevice, s_), "H2D");
    hist_.need((uint64_t)nd * maxp, "partition counts");
    cu(cudaMemsetAsync(hist_.p, 0, (uint64_t)nd * maxp * 8, s_), "memset");
    // raw_ holds the batch's distinct keys at [0, n); their order keys go to
    // order_, sorted to order_sorted_, and the keys in filter order to keys_.
    const uint64_t* kin = raw_.p;
    order_.need(n, "order keys");
    order_sorted_.need(n, "sorted order keys");
    keys_.need(n, "filter keys");
    order_kernel<<<grid_for(n, sms_), 256, 0, s_>>>(kin, n, d_dense_.p, d_parts_.p, d_local_.p, nd,
                                                    seed, H, seg, order_.p, hist_.p, maxp);
    cu(cudaGetLastError(), "order_kernel");
    uint64_t largest = 1;
    for (uint32_t j = 0; j < nd; ++j) largest = std::max<uint64_t>(largest, dense[j + 1] - dense[j]);
    size_t sbytes = 0;
    cu(cub::DeviceRadixSort::SortPairs(nullptr, sbytes, order_.p, order_sorted_.p, kin, keys_.p,
                                       (int)largest),
       "sort size");
    sort_tmp_.need(sbytes, "sort scratch");
    for (uint32_t j = 0; j < nd; ++j) {
      const uint64_t m = dense[j + 1] - dense[j];
      if (!m) continue;
      int end_bit = 32;
      while ((1u << (end_bit - 32)) < parts[j]) ++end_bit;
      size_t bytes = sort_tmp_.n;
      cu(cub::DeviceRadixSort::SortPairs(sort_tmp_.p, bytes, order_.p + dense[j],
                                         order_sorted_.p + dense[j], kin + dense[j],
                                         keys_.p + dense[j], (int)m, 0, end_bit, s_),
         "sort");
    }
    std::vector<unsigned long long> hist((uint64_t)nd * maxp);
    cu(cudaMemcpyAsync(hist.data(), hist_.p, hist.size() * 8, cudaMemcpyDeviceToHost, s_), "D2H");
    cu(cudaStreamSynchronize(s_), "filter order");
    tock(kOrder);
    // Filter table: dataset-major, partitions in order (the keys' order).
    std::vector<Filter> filters;
    uint64_t cells = 0;
    for (uint32_t j = 0; j < nd; ++j) {
      const build::Group& g = groups[b.d0 + j];
      const build::ClassLayout& cl = classes[g.cls];
      uint64_t at = dense[j];
      for (uint32_t p = 0; p < parts[j]; ++p) {
        const uint64_t m = hist[(uint64_t)j * maxp + p];
        Filter F{};
        F.key0 = at;
        F.cell0 = cells;
        F.rows = rows[g.cls][p];
        F.nkeys = (uint32_t)m;
        F.slots = (uint32_t)cl.local_slots;
        F.row_bytes = (uint32_t)((cl.row_bits + 7) / 8);
        F.column = (uint32_t)g.column;
        F.dataset = b.d0 + j;
        check(cl.local_slots < (1ull << 32) && m < (1ull << 32), kEUnsupported,
              "a filter of 2^32 cells or keys");
        filters.push_back(F);
        at += m;
        cells += cl.local_slots;
      }
      check(at == dense[j + 1], kEInval, "partition counts do not add up");
    }
    const uint32_t nf = (uint32_t)filters.size();
    d_filters_.need(nf, "filters");
    cu(cudaMemcpyAsync(d_filters_.p, filters.data(), nf * sizeof(Filter), cudaMemcpyHostToDevice, s_),
       "H2D");
    deg_.need(cells, "cell degrees");
    xr_.need(cells, "cell xors");
    queue_.need(cells, "peel queues");
    state_.need(n, "key states");
    stack_.need(n, "peel stacks");
    nab_.need(nf, "abandoned counts");
    cu(cudaMemsetAsync(deg_.p, 0, cells * 4, s_), "memset");
    cu(cudaMemsetAsync(xr_.p, 0, cells * 4, s_), "memset");
    cu(cudaMemsetAsync(state_.p, 0, n, s_), "memset");
    accumulate_kernel<<<grid_for(n, sms_), 256, 0, s_>>>(d_filters_.p, nf, keys_.p, n, seed, H, seg,
                                                         deg_.p, xr_.p);
    cu(cudaGetLastError(), "accumulate_kernel");
    tock(kAccumulate);
    const int pb = 32, pg = (int)((nf + pb - 1) / pb);
    peel_kernel<<<pg, pb, 0, s_>>>(d_filters_.p, nf, keys_.p, seed, H, seg, deg_.p, xr_.p, queue_.p,
                                   state_.p, stack_.p, nab_.p, err_.p);
    cu(cudaGetLastError(), "peel_kernel");
    tock(kPeel);
    assign_kernel<<<pg, pb, 0, s_>>>(d_filters_.p, nf, keys_.p, seed, H, seg, bc_.b, deg_.p,
                                     stack_.p);
    cu(cudaGetLastError(), "assign_kernel");
    pack_rows_kernel<<<grid_for(cells, sms_), 256, 0, s_>>>(d_filters_.p, nf, cells, deg_.p, bc_.b);
    cu(cudaGetLastError(), "pack_rows_kernel");
    std::vector<uint32_t> nab(nf);
    cu(cudaMemcpyAsync(nab.data(), nab_.p, nf * 4, cudaMemcpyDeviceToHost, s_), "D2H");
    cu(cudaStreamSynchronize(s_), "construction");
    tock(kPack);
    check_error();
    std::vector<uint64_t> first(nf + 1, 0);
    for (uint32_t i = 0; i < nf; ++i) {
      first[i + 1] = first[i] + nab[i];
      groups[filters[i].dataset].abandoned += nab[i];
    }
    if (first[nf] && !bc_.opt.drop_abandoned) {
      d_first_.need(nf + 1, "abandoned offsets");
      fill_.need(nf, "abandoned fill");
      lost_.need(first[nf], "abandoned keys");
      cu(cudaMemcpyAsync(d_first_.p, first.data(), (nf + 1) * 8, cudaMemcpyHostToDevice, s_), "H2D");
      cu(cudaMemsetAsync(fill_.p, 0, nf * 4, s_), "memset");
      abandoned_kernel<<<grid_for(n, sms_), 256, 0, s_>>>(d_filters_.p, nf, n, keys_.p, stack_.p, seed,
                                                          d_first_.p, fill_.p, lost_.p);
      cu(cudaGetLastError(), "abandoned_kernel");
      std::vector<uint2> lost(first[nf]);
      cu(cudaMemcpyAsync(lost.data(), lost_.p, lost.size() * 8, cudaMemcpyDeviceToHost, s_), "D2H");
      cu(cudaStreamSynchronize(s_), "abandoned keys");
      for (const uint2& x : lost) bc_.abandoned.push_back(build::Abandoned{x.x, x.y, 1});
    }
    tock(kAbandoned);
  }

  cudaStream_t stream() const { return s_; }

 private:
  void check_error() {
    uint32_t e = 0;
    cu(cudaMemcpy(&e, err_.p, 4, cudaMemcpyDeviceToHost), "error word");
    if (e & kErrOffsets) raise(kEInval, "a dataset record of 2^31 bases or more");
    if (e) raise(kEInval, "device filter construction failed a bound (error word " +
                              std::to_string(e) + ")");
  }
  const RecordBatch& file_batch(uint32_t d) {
    if (cached_ != d) {
      file_ = read_fastx(bc_.inputs[d].path, false);
      cached_ = d;
    }
    return file_;
  }

  void tick() {
    if (bc_.opt.quiet) return;
    cu(cudaStreamSynchronize(s_), "phase timing");
    tp_ = std::chrono::steady_clock::now();
  }
  void tock(Phase i) {
    if (bc_.opt.quiet) return;
    cu(cudaStreamSynchronize(s_), "phase timing");
    const auto now = std::chrono::steady_clock::now();
    phase_[i] += std::chrono::duration<double>(now - tp_).count();
    tp_ = now;
  }

  Context& bc_;
  double phase_[kPhases] = {};
  std::chrono::steady_clock::time_point tp_;
  int sms_ = 1;
  cudaStream_t s_ = nullptr;
  SeedParams sp_{};
  RecordBatch file_;
  uint32_t cached_ = 0xFFFFFFFFu;
  DevBuf<uint8_t> bases_;
  DevBuf<uint64_t> packed_, d_region_, d_genome_, d_rec_off_, raw_, sorted_, d_counts_, d_dense_,
      d_local_, order_, order_sorted_, keys_, d_first_;
  DevBuf<uint32_t> invalid_, tile_counts_, tile_first_, d_rec_ds_, d_parts_, deg_, xr_, queue_,
      nab_, err_;
  DevBuf<unsigned long long> cursor_, hist_;
  DevBuf<unsigned int> fill_;
  DevBuf<Tile> tiles_;
  DevBuf<uint8_t> scan_tmp_, sort_tmp_, state_;
  DevBuf<uint2> stack_, lost_;
  DevBuf<Filter> d_filters_;
};

}  // namespace

void build_index_device(const BuildOptions& opt) {
  using namespace build;
  Context bc;
  prepare(opt, bc);
  const FeatureParams& fp = bc.fp;
  check(opt.groups.empty(), kEUnsupported, "the device builder builds singleton groups only");
  check(fp.mode >= 0 && fp.mode <= 2, kEUnsupported,
        "the device builder builds k-mer, minimizer and modimizer indexes");
  check(!fp.homopolymer && !fp.strobes && !opt.legacy_layout, kEUnsupported,
        "the device builder does not do homopolymer compression, randstrobemers or the legacy "
        "layout");
  check(bc.H <= kMaxHashes, kEInval, "invalid hash count");
  const size_t C = bc.inputs.size();
  DeviceBuilder dev(bc);
  // Batches of datasets by bases (every device buffer scales with them).
  size_t free_b = 0, total_b = 0;
  cu(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  std::vector<uint64_t> lengths(C);
  for (size_t d = 0; d < C; ++d) lengths[d] = dev.dataset_bases((uint32_t)d);
  auto batches = [&](uint64_t cap_bases) {
    std::vector<Batch> out;
    Batch cur;
    for (size_t d = 0; d < C; ++d) {
      if (cur.d1 > cur.d0 && cur.bases + lengths[d] > cap_bases) {
        out.push_back(cur);
        cur = Batch{(uint32_t)d, (uint32_t)d, 0};
      }
      cur.d1 = (uint32_t)d + 1;
      cur.bases += lengths[d];
    }
    if (cur.d1 > cur.d0) out.push_back(cur);
    return out;
  };
  // Pass 1: distinct keys per dataset (about 17 bytes of device memory per
  // base: bases, packed bases, two seed regions).
  const uint64_t cap1 = std::min<uint64_t>((free_b - (free_b >> 3)) / 20, (1ull << 31) - 64);
  std::vector<uint64_t> unique(C, 0);
  for (const Batch& b : batches(cap1)) dev.distinct(b, unique, bc.occurrences, false, nullptr);
  if (!opt.quiet)
    fprintf(stderr, "counted distinct keys of %zu datasets in %.3fs\n", C, seconds_since(bc.t0));
  // Layout, shared with the host builder.
  bc.groups.resize(C);
  for (size_t d = 0; d < C; ++d) {
    Group& g = bc.groups[d];
    g.members = {(uint32_t)d};
    g.width = (uint64_t)bc.b;
    g.cardinality = unique[d];
    g.slots = config_slots(opt, bc.H, g.cardinality);
  }
  plan_layout(bc, false);
  // Device rows of every (class, partition).
  std::vector<std::vector<uint8_t*>> rows(bc.classes.size());
  std::vector<std::unique_ptr<DevBuf<uint8_t>>> row_bufs;
  uint64_t row_total = 0;
  for (size_t ci = 0; ci < bc.classes.size(); ++ci) {
    const ClassLayout& cl = bc.classes[ci];
    const uint64_t bytes = cl.local_slots * ((cl.row_bits + 7) / 8);
    for (uint64_t p = 0; p < cl.partitions; ++p) {
      row_bufs.push_back(std::make_unique<DevBuf<uint8_t>>());
      row_bufs.back()->need(bytes + 16, "bank rows");
      cu(cudaMemsetAsync(row_bufs.back()->p, 0, bytes + 16, dev.stream()), "memset");
      rows[ci].push_back(row_bufs.back()->p);
      row_total += bytes;
    }
  }
  // Pass 2: distinct keys again (dense, per dataset), then the filters. Device
  // memory per base: about 17 bytes for extraction, 24 per distinct key for
  // ordering, and 12 per cell (cells are at most about twice the keys, except
  // for tiny promoted datasets) plus 9 per key for the peel.
  std::vector<uint64_t> dense(C + 1, 0);
  for (size_t d = 0; d < C; ++d) dense[d + 1] = dense[d] + unique[d];
  cu(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  uint64_t max_cells = 1;
  for (auto& g : bc.groups) max_cells = std::max<uint64_t>(max_cells, bc.classes[g.cls].source_slots);
  const uint64_t usable = free_b - (free_b >> 3);
  uint64_t cap2 = std::min<uint64_t>(usable / 90, (1ull << 31) - 64);
  check(cap2 > max_cells / 4, kENoMem, "not enough device memory for the largest filter");
  std::vector<uint64_t> occ_again(C, 0), unique_again(C, 0);
  for (const Batch& b : batches(cap2)) {
    dev.distinct(b, unique_again, occ_again, true, &dense);
    dev.construct(b, dense, rows);
  }
  for (size_t d = 0; d < C; ++d)
    check(unique_again[d] == unique[d], kEInval, "distinct keys differ between passes");
  if (!opt.quiet) {
    fprintf(stderr, "constructed %zu filters in %.3fs (%llu bytes of rows on the device)\n", C,
            seconds_since(bc.t0), (unsigned long long)row_total);
    dev.report(stderr);
  }
  const double t_write = seconds_since(bc.t0);
  // Bank payloads streamed from the device, one writer per bank, each through
  // its own pinned buffer.
  constexpr uint64_t kPiece = 64ull << 20;
  write_index(
      bc,
      [&](size_t ci, uint64_t part, FramedWriter& w) {
        cu(cudaSetDevice(opt.gpu), "cudaSetDevice");
        uint8_t* pinned = nullptr;
        cu(cudaMallocHost((void**)&pinned, kPiece), "cudaMallocHost");
        struct PinnedFree {
          uint8_t* p;
          ~PinnedFree() { cudaFreeHost(p); }
        } pinned_free{pinned};
        const ClassLayout& cl = bc.classes[ci];
        const uint64_t bytes = cl.local_slots * ((cl.row_bits + 7) / 8);
        for (uint64_t at = 0; at < bytes; at += kPiece) {
          const uint64_t len = std::min(kPiece, bytes - at);
          cu(cudaMemcpy(pinned, rows[ci][part] + at, len, cudaMemcpyDeviceToHost), "D2H rows");
          w.write(pinned, len);
        }
      },
      bc.threads);
  if (!opt.quiet)
    fprintf(stderr, "wrote the index in %.3fs (%zu abandoned keys)\n", seconds_since(bc.t0) - t_write,
            bc.abandoned.size());
}

}  // namespace zx
