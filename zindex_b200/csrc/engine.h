// Host runtime of the GPU query path: loads an index directory into HBM and
// runs batched queries on one device.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "host/manifest.h"
#include "kernels/device_index.cuh"
#include "kernels/types.cuh"

namespace zx {
struct ColorLoc;
struct BatchView;
}

namespace zx {

struct OpenOptions {
  int device = 0;
  uint64_t hbm_budget = 0;  // bytes the resident index may take; 0 = free memory - 4 GiB
  int threads = 0;          // host threads for decompression; 0 = hardware concurrency
};

// Device buffers of one in-flight batch. One workspace serves one stream at a
// time; the serving loop keeps one per slot.
struct Workspace {
  int device = 0;
  uint8_t* bases = nullptr;
  uint64_t* offsets = nullptr;
  uint64_t* packed = nullptr;
  uint32_t* invalid = nullptr;
  uint32_t* tile_counts = nullptr;  // records + 1
  uint32_t* tile_first = nullptr;   // records + 1 (last entry = tile total)
  Tile* tiles = nullptr;
  void* scan_tmp = nullptr;
  size_t scan_tmp_bytes = 0;
  uint32_t* partial = nullptr;
  uint64_t* counts = nullptr;
  unsigned long long* total = nullptr;
  uint32_t* error = nullptr;        // bit 0: a bounded device wait expired
  uint64_t* keys_out = nullptr;     // extraction-only output
  uint32_t* keys_count = nullptr;
  uint32_t* fstate = nullptr;       // findere: per grid warp, colour round masks + run lengths
  // Homopolymer compression of the batch (indexes built with it).
  uint32_t* hp_starts = nullptr;    // record-start bits
  uint32_t* hp_keep = nullptr;      // keep flag per base (+1)
  uint32_t* hp_pos = nullptr;       // exclusive scan of the flags
  uint8_t* hp_bases = nullptr;      // compressed bases
  uint64_t* hp_offsets = nullptr;   // compressed record offsets
  void* hp_scan_tmp = nullptr;
  size_t hp_scan_bytes = 0;
  uint64_t cap_fstate = 0, cap_hp_bases = 0, cap_hp_records = 0;
  // Segmented launches (several requests per launch).
  uint32_t* seg_blocks = nullptr;   // segments + 1
  uint32_t* seg_tiles = nullptr;    // segments + 1
  uint64_t* seg_records = nullptr;  // segments + 1
  uint32_t* h_seg_blocks = nullptr;   // pinned staging
  uint64_t* h_seg_records = nullptr;  // pinned staging
  uint64_t cap_segments = 0;
  cudaEvent_t seg_staged = nullptr;   // the last segmented call's staging copies are done
  // Split minimizer queries: key slots of one round of tiles.
  uint64_t* split_keys = nullptr;
  uint32_t* split_counts = nullptr;
  unsigned long long* wide_cursor = nullptr;  // wide-row queries: keys in the dense lists (2)
  // Segmented wide-row queries, per key list: keys of each segment and the
  // first probe round of each segment (2 x cap_segments each).
  unsigned long long* wide_seg_cursor = nullptr;
  uint32_t* wide_round_first = nullptr;
  // Ordered wide-row rounds, per key list: the keys in bucket order and the
  // buckets' counts / next places.
  uint64_t* wide_keys_alt[2] = {};
  uint32_t* wide_hist[2] = {};
  // Randstrobemer queries: candidate bits and strobe hashes per base, each
  // tile's linked seeds (kStrobeSlot per tile) and their numbers.
  uint32_t* strobe_anchors = nullptr;
  uint64_t* strobe_hashes = nullptr;
  uint64_t* strobe_slots = nullptr;
  uint32_t* strobe_count = nullptr;
  uint64_t cap_strobe_bases = 0, cap_strobe_tiles = 0;
  uint64_t* wide_keys2 = nullptr;  // second dense key list (rounds alternate)
  cudaStream_t aux_stream = nullptr;  // wide-row queries: extraction beside the probe
  cudaEvent_t wide_fork = nullptr, wide_ext[2] = {}, wide_probe[2] = {};
  // Per-record queries: counters of one record group (records x colours).
  uint64_t* rec_counts = nullptr;
  unsigned long long* rec_totals = nullptr;
  uint64_t cap_rec_counts = 0, cap_rec_totals = 0;
  // Thresholded reports: per-record hit counts, their scan and the hits.
  uint64_t* rec_hits = nullptr;    // group records + 1
  uint64_t* rec_first = nullptr;   // group records + 1
  void* rec_scan_tmp = nullptr;
  size_t rec_scan_bytes = 0;
  uint32_t* hit_colors = nullptr;
  uint64_t* hit_counts = nullptr;
  uint64_t cap_hits = 0;
  // Pinned host staging.
  uint8_t* h_bases = nullptr;
  uint64_t* h_offsets = nullptr;
  uint64_t* h_counts = nullptr;
  unsigned long long* h_total = nullptr;
  uint64_t cap_bases = 0, cap_records = 0, cap_tiles = 0, cap_partial = 0, cap_colors = 0,
           cap_keys = 0, cap_h_bases = 0, cap_h_records = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;       // host-buffer queries: chunk copies
  std::vector<cudaEvent_t> chunk_events;    // one per pipelined chunk
  // Graph cache: one instantiated graph per (input pointers, sizes, recover).
  std::map<std::tuple<const void*, uint64_t, const void*, uint64_t, void*, void*, int>,
           cudaGraphExec_t>
      graphs;
  ~Workspace();
  void release_graphs();
};

// Reverse complement of every record of a host batch, records in place.
void reverse_complement_records(const uint8_t* bases, const uint64_t* offsets, uint64_t records,
                                uint8_t* out);

class Engine {
 public:
  Engine(const std::string& dir, const OpenOptions& options);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  const Manifest& manifest() const { return m_; }
  // Seconds of the load: total, the bank streaming (read, decode, upload) and
  // the recovery map (read and decoded concurrently with the banks).
  double load_seconds() const { return load_s_; }
  double banks_load_seconds() const { return banks_load_s_; }
  double recovery_load_seconds() const { return recovery_load_s_; }
  int device() const { return device_; }
  uint64_t resident_bytes() const { return resident_bytes_; }
  int span() const;  // k-window span of the index mode
  const SeedParams& seed_params() const { return sp_; }
  // Launch configuration used by the batched kernels (tunable).
  QueryLaunch launch() const { return launch_; }
  void set_launch(const QueryLaunch& l);
  QueryLaunch default_launch() const;
  // The fused kernel's default launch (segmented and allocation-free queries
  // run the fused kernel; a wide-row launch maps to it, keeping its cut).
  QueryLaunch default_fused_launch() const;
  QueryLaunch fused_launch(const QueryLaunch& l) const;
  // Wide-row form (kernels/wide_probe.cuh): fingerprint chunks over all
  // classes, whether an index and block size admit it, and the kernel shape.
  uint32_t wide_chunks() const;
  bool wide_eligible(int warps) const;
  bool wide_form(const QueryLaunch& l) const;
  void wide_shape(const QueryLaunch& l, int& J, int& HQ, uint32_t* team = nullptr) const;
  size_t fused_smem_bytes(const QueryLaunch& l) const;
  int max_blocks(const QueryLaunch& l) const;
  // Bytes of fingerprint planes gathered per seed, summed over classes.
  uint64_t gather_bytes_per_seed() const;
  // The same gather counted in 32-byte DRAM sectors: per class H rows of
  // fp_chunks 16-byte chunks, each row starting at row * stride (rows of a
  // 16-byte-odd stride alternate between sector offsets 0 and 16).
  uint64_t gather_sector_bytes_per_seed() const;

  std::unique_ptr<Workspace> make_workspace();
  // Sizes a workspace's device buffers for segmented batches up to these
  // sizes (the request server's slots).
  void reserve(Workspace& ws, uint64_t nbases, uint64_t records) {
    ensure_capacity(ws, nbases, records, true);
  }
  Workspace& default_workspace() { return *ws_; }

  // Asynchronous query of a batch resident on the device. counts (colors
  // entries) and total are accumulated, not cleared. use_graph replays a
  // captured CUDA graph when the same batch shape was seen before.
  void query_device(Workspace& ws, const uint8_t* bases, uint64_t nbases, const uint64_t* offsets,
                    uint64_t records, bool recover, uint64_t* counts, unsigned long long* total,
                    cudaStream_t stream, bool use_graph);
  // As query_device, but every scratch buffer comes from one static device
  // array (no device allocation at all); see zx_query_device_noalloc.
  void query_device_noalloc(const uint8_t* bases, uint64_t nbases, const uint64_t* offsets,
                            uint64_t records, bool recover, uint64_t* counts,
                            unsigned long long* total, cudaStream_t stream);
  // Synchronous query of host buffers (bases, records + 1 offsets).
  void query_host(Workspace& ws, const uint8_t* bases, uint64_t nbases, const uint64_t* offsets,
                  uint64_t records, bool recover, uint64_t* counts, uint64_t* total);
  // One record per launch (the plain form), host buffers, synchronous.
  void query_host_plain(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                        const uint64_t* offsets, uint64_t records, bool recover, uint64_t* counts,
                        uint64_t* total);
  // Kernel timing: when enabled, non-graph launches record CUDA events around
  // the fused query kernel on its stream; last_fused_ms() waits for and
  // returns the most recent interval.
  void set_timing(bool on);
  float last_fused_ms();
  // Device error word of a workspace (read and cleared); nonzero means a
  // bounded wait expired and the query's counts are incomplete.
  uint32_t take_error(Workspace& ws);
  // This engine's error word in the allocation-free query's scratch (read
  // and cleared; 0 if that entry point was never used by this engine).
  uint32_t take_noalloc_error();
  // Asynchronous query of several requests coalesced into one launch: the
  // batch's records are the requests' records back to back, request s owning
  // records seg_records[s] .. seg_records[s+1]-1 (host array, segments + 1
  // entries). counts (segments x colours) and totals (segments) are
  // accumulated, not cleared. est_tiles[s] (host) sizes each request's share
  // of the grid; any positive estimate gives exact results. warps > 0
  // overrides the launch's warps per block (short requests leave most warps
  // of a block idle).
  void query_segments(Workspace& ws, const uint8_t* bases, uint64_t nbases, const uint64_t* offsets,
                      uint64_t records, const uint64_t* seg_records, const uint64_t* est_tiles,
                      uint32_t segments, bool recover, uint64_t* counts,
                      unsigned long long* totals, cudaStream_t stream, int warps = 0,
                      double prune_ratio = 0.0);
  // Per-record query of host records (--records): counts (records x colours,
  // row-major) and totals (records) receive each record's own result, exactly
  // as if the record were queried alone. Records run in groups whose device
  // counters fit a fixed budget, one segment per record in a segmented launch.
  void query_per_record(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                        const uint64_t* offsets, uint64_t records, bool recover, uint64_t* counts,
                        uint64_t* totals);
  // Randstrobemer indexes (k-mer strobes on the GPU): aggregate of host
  // records = the sum over records of the per-colour maximum of the two
  // strands' counts; *total = forward anchors.
  void query_strobes_host(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                          const uint64_t* offsets, uint64_t records, bool recover,
                          uint64_t* counts, uint64_t* total);
  bool strobes() const { return sp_.strobe_max != 0; }
  // Raises ZX_EUNSUPPORTED for randstrobemer indexes (entry points that
  // count one strand of device batches).
  void check_not_strobes() const;
  // Per-record hits for a report with min_ratio in (0, 1]: totals (records)
  // and, for record r, the colours hit_colors[first[r] .. first[r+1]) with
  // their counts, in colour order: those with count > 0 and count / total >=
  // min_ratio. Selected on the device; only the hits are copied back.
  struct RecordHits {
    std::vector<uint64_t> totals, first;
    std::vector<uint32_t> colors;
    std::vector<uint64_t> counts;
  };
  void query_record_hits(Workspace& ws, const uint8_t* bases, uint64_t nbases,
                         const uint64_t* offsets, uint64_t records, bool recover, double min_ratio,
                         RecordHits& out);
  // Upper bound of the tiles of one record of `len` bases.
  uint64_t tiles_for_length(uint64_t len) const;
  // Seeds of host records in record/window order (extraction only).
  void extract_host(Workspace& ws, const uint8_t* bases, uint64_t nbases, const uint64_t* offsets,
                    uint64_t records, std::vector<uint64_t>& keys);

 private:
  void load(const std::string& dir, const OpenOptions& options);
  void release();  // frees every device allocation and event of the engine
  // Device buffers of a query of nbases / records (segmented queries do not
  // sort their rounds: no ordered-round buffers).
  void ensure_capacity(Workspace& ws, uint64_t nbases, uint64_t records, bool segmented = false);
  // Homopolymer compression on the device (lib.rs:211-222 per ACGT run):
  // replaces (bases, offsets) by the compressed batch in the workspace.
  void compress_homopolymers(Workspace& ws, const uint8_t*& bases, uint64_t nbases,
                             const uint64_t*& offsets, uint64_t records, cudaStream_t s);
  void ensure_host_capacity(Workspace& ws, uint64_t nbases, uint64_t records);
  void enqueue(Workspace& ws, const uint8_t* bases, uint64_t nbases, const uint64_t* offsets,
               uint64_t records, bool recover, uint64_t* counts, unsigned long long* total,
               cudaStream_t stream);
  void plan_tiles(Workspace& ws, const uint64_t* offsets, uint64_t records, uint64_t nbases,
                  cudaStream_t stream);
  void check_error_word(Workspace& ws);
  // Kernel form of a launch: the seed mode, or 4 (probe of pre-extracted
  // seeds) for split minimizer queries.
  int kernel_mode(const QueryLaunch& l) const;
  void ensure_split_capacity(Workspace& ws);
  // Wide-row queries of several rounds: the second key list, the auxiliary
  // stream and the events of the extraction / probe pipeline.
  void ensure_wide_pipeline(Workspace& ws);
  // Ordered wide-row rounds: sort buffers of key list b (0 or 1).
  void ensure_order_capacity(Workspace& ws, int b);
  // Wide-row form over the planned tiles of a packed batch: rounds of up to
  // kSplitTiles tiles, each a dense extraction and a wide probe. segments = 0:
  // one query into counts / *total; segments > 0: a segmented query, request
  // s into counts + s x colours and total[s] (the segment tables and their
  // per-round cursors already in ws).
  // prune_ratio > 0 (segmented per-record reports): threshold pruning of the
  // colours that cannot reach count / total >= prune_ratio.
  void run_wide(Workspace& ws, const BatchView& bv, uint64_t tiles_bound, bool recover,
                uint64_t* counts, unsigned long long* total, uint32_t segments, cudaStream_t s,
                double prune_ratio = 0.0);
  // Device tables of a segmented launch for `segments` requests.
  void ensure_segment_capacity(Workspace& ws, uint32_t segments);
  // Randstrobemer seeds of a planned batch (strobes.cuh): candidates, then
  // each tile's linked seeds into ws.strobe_slots / strobe_count.
  void ensure_strobe_capacity(Workspace& ws, uint64_t nbases, uint64_t tiles);
  void link_strobes(Workspace& ws, const BatchView& bv, uint64_t nbases, cudaStream_t s);
  // Runs host records in device groups (one segment per record): after each
  // group's launch, on_group(r0, n) enqueues its read-back on ws.stream; the
  // stream is then synchronised and the error word checked.
  // prune_ratio > 0: the groups' counts are only exact for the colours with
  // count / total >= prune_ratio (the others may stop early, below it).
  void record_groups(Workspace& ws, const uint8_t* bases, uint64_t nbases, const uint64_t* offsets,
                     uint64_t records, bool recover, double prune_ratio,
                     const std::function<void(uint64_t, uint64_t)>& on_group);

  Manifest m_;
  int device_ = 0;
  int sms_ = 0;
  SeedParams sp_{};
  QueryLaunch launch_{};
  DevIndex host_ix_{};
  DevIndex* d_ix_rec_ = nullptr;    // with recovery
  DevIndex* d_ix_norec_ = nullptr;  // recovery disabled
  ColorLoc* d_color_loc_ = nullptr;  // colour -> class, member, group (wide probe)
  std::vector<void*> allocations_;
  uint64_t resident_bytes_ = 0;
  std::unique_ptr<Workspace> ws_;
  std::mutex mu_;
  bool timing_ = false;
  cudaEvent_t ev_begin_ = nullptr, ev_end_ = nullptr;
  int cached_blocks_ = 0;
  int noalloc_slot_ = -1;  // error word of the allocation-free query, once used
  double load_s_ = 0, banks_load_s_ = 0, recovery_load_s_ = 0;
  QueryLaunch cached_for_{};
};

// CUDA error check that throws zx::Error(kECuda).
void cuda_check(cudaError_t e, const char* what);

}  // namespace zx
