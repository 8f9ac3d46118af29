/*
 * zindex.h — C ABI of the B200 Zindex query path (libzindex_b200.so).
 *
 * The reference (Malfoy/Zindex, crate `zorindex`) is a Rust program with no
 * FFI; its query entry points are library functions called by the CLI. Each
 * declaration below names the reference function or behaviour it replaces
 * (paths relative to the reference project). Plain pointers and sizes only:
 * no CUDA or torch types cross this boundary except the opaque `stream`
 * argument of zx_query_device (a cudaStream_t passed as void*).
 *
 * Errors: every int-returning function returns ZX_OK (0) or one of the ZX_E*
 * codes; zx_last_error() returns the calling thread's last message. No
 * exception crosses the boundary. Ownership: the library owns the index and
 * its device memory; the caller owns every buffer it passes in.
 * Threading: an index handle may be shared; each query call uses a private
 * workspace unless stated otherwise.
 */
#ifndef ZINDEX_B200_H
#define ZINDEX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZX_OK 0
#define ZX_EINVAL 1       /* invalid argument */
#define ZX_EFORMAT 2      /* malformed index, manifest or query input */
#define ZX_EIO 3          /* file system error */
#define ZX_ENOMEM 4       /* HBM / host memory exhausted, or admission refused */
#define ZX_ECUDA 5        /* CUDA runtime error */
#define ZX_ETIMEOUT 6     /* a bounded device wait expired */
#define ZX_EUNSUPPORTED 7 /* index feature the GPU path does not implement */

typedef struct zx_index zx_index;

typedef struct zx_info {
  uint32_t version;           /* manifest "version" */
  uint32_t k;                 /* window span: k-mer length / minimizer window */
  uint32_t hashes;            /* H */
  uint32_t fingerprint_bits;  /* b */
  uint32_t index_mode;        /* 0 kmers, 1 minimizers, 2 modimizers, 3 findere */
  uint32_t minimizer_size;    /* m */
  uint64_t seed;
  uint64_t colors;
  uint64_t banks;
  uint64_t classes;           /* source size classes */
  uint64_t resident_bytes;    /* HBM held by the index */
  uint64_t gather_bytes_per_seed; /* fingerprint-plane bytes read per seed, all classes */
  uint64_t gather_sector_bytes_per_seed; /* the same reads in whole 32-byte DRAM sectors */
  uint64_t abandoned_hashes;
  int recovery;               /* manifest abandoned_recovery */
  double load_s;              /* zx_open wall time */
  double load_banks_s;        /* bank files read, decoded and uploaded (overlapped) */
  double load_recovery_s;     /* recovery map read and decoded (concurrent with the banks) */
} zx_info;

typedef struct zx_launch {
  int team;           /* register gather: lanes sharing one seed, 1..32 (power of two) */
  int warps;          /* warps per block, 1..8 */
  int blocks;         /* grid size; 0 = fill the device */
  int smem_counters;  /* 1 = per-block shared colour counters, 0 = global atomics */
  int stage_bytes;    /* > 0: staged gather, bytes per ring stage (multiple of 16) */
  int stages;         /* stages per warp ring for the staged gather, 1..8 */
  int bulk;           /* staged gather: 1 = cp.async.bulk per row slice, 0 = 16-byte cp.async */
  int min_blocks;     /* kernel variant register budget: 2 or 3 resident 256-thread blocks, or 1
                         (255 registers; planes 1 only: pipelines the row loads of wide rows) */
  int planes;         /* register gather: 1 = per-seed row indices and per-lane bit-plane colour
                         counters, 0 = per-seed descriptors and one counter update per hit */
  int cut;            /* host-buffer queries: the batch is cut at record boundaries into this many
                         chunks (1..64) whose host-to-device copies overlap the previous chunk's
                         kernels; chunks below 1 MiB of bases are merged */
  int split;          /* minimizer indexes: 1 = seeds are extracted by a kernel of their own into
                         per-tile slots and probed by a kernel without the extraction scratch
                         (more resident warps); applies to the row-index form (planes 1, no
                         staged gather) and is ignored elsewhere */
  int wide;           /* 1 = wide-row form (fingerprint bits >= 4, k-mer, minimizer and
                         modimizer indexes with rows of at most 4 x warps x 32 chunks): seeds
                         are extracted into a dense list and probed by blocks whose threads
                         each own fixed 16-byte chunks of every row, counting in registers;
                         team, planes, stage_bytes and split are then unused */
  int order;          /* wide-row form, unsegmented queries: 1 = each round's seeds are sorted
                         by their first hash before the probe (every class's row index grows
                         with it, so consecutive seeds read neighbouring rows), each block
                         probing runs of 256 consecutive seeds; 2 = sorted, and block b
                         probes seeds b, b + blocks, ... (all blocks on neighbouring seeds);
                         0 = extraction order; ignored elsewhere. Counts do not depend on it */
} zx_launch;

/* Thread-local message of the last failed call on this thread. */
const char* zx_last_error(void);

/* Load and validate an index directory and make it resident in HBM of
 * `device`. Replaces Index::load_mode / load_with_recovery
 * (src/power_merge/storage.rs:2273-2707) and the bank readers
 * (bank_io.rs:235-292, abandoned_io.rs:4-130). hbm_budget = 0 admits the
 * index if it fits in free device memory minus 4 GiB; otherwise the index must
 * fit in hbm_budget bytes (ZX_ENOMEM if not). */
int zx_open(const char* index_dir, int device, uint64_t hbm_budget, zx_index** out);

/* Release the index and its device memory. */
void zx_close(zx_index* index);

/* Index geometry (manifest fields, storage.rs:132-214). */
int zx_index_info(const zx_index* index, zx_info* out);

/* Name and unique_kmers of colour c (manifest colors[c], storage.rs:57-63). */
const char* zx_color_name(const zx_index* index, uint64_t color);
uint64_t zx_color_unique_kmers(const zx_index* index, uint64_t color);

/* Aggregate query of a FASTA/FASTQ file (plain, gzip or zstd): the hot path
 * of query_command_with_memory (storage.rs:3731-3767; query_aggregate,
 * query_stream.rs:864-946). counts receives one 64-bit match count per colour
 * (matches[] of print_aggregate); *total the number of query features (the
 * ratio denominator, total_features); *probes the feature probes
 * (stack_probes). recover = 0 disables abandoned-key recovery
 * (query_command_with_recovery, storage.rs:3722-3729). */
int zx_query_file(zx_index* index, const char* query_path, int recover, uint64_t* counts,
                  uint64_t* total, uint64_t* probes);

/* Aggregate query of records in host memory: record r is
 * bases[offsets[r] .. offsets[r+1]) (raw sequence bytes; non-ACGT bytes split
 * seeds as the reference parser's split_non_actg does, src/lib.rs:27-33).
 * Batched: all records go through one launch sequence. */
int zx_query_host(zx_index* index, const uint8_t* bases, const uint64_t* offsets,
                  uint64_t records, int recover, uint64_t* counts, uint64_t* total);

/* As zx_query_host, but one record per launch sequence with default tiles
 * (the plain GPU form, kept for comparison). */
int zx_query_host_plain(zx_index* index, const uint8_t* bases, const uint64_t* offsets,
                        uint64_t records, int recover, uint64_t* counts, uint64_t* total);

/* Per-record query of records in host memory (the counting step of
 * query_records_command_with_memory, storage.rs:3626-3720, and of the
 * findere branch's Scorer per record): counts (records x colours, row-major)
 * receives each record's match counts and totals (records) its feature count,
 * each exactly as a query of that record alone would give. */
int zx_query_per_record(zx_index* index, const uint8_t* bases, const uint64_t* offsets,
                        uint64_t records, int recover, uint64_t* counts, uint64_t* totals);

/* Per-record report of a FASTA/FASTQ file: `zorindex query --records`
 * (query_records_command_with_memory, storage.rs:3626-3720). Records are read
 * by the rules of read_batches (src/power_merge/records.rs:150-290) and
 * reported in input order; compact = 0 writes RecordFormat::Tsv, 1
 * RecordFormat::Compact (src/power_merge/record_output.rs:13-62) with the
 * colour selection of RecordScores::write_record (storage.rs:3109-3146).
 * min_ratio must be in [0, 1] and batch_records (--record-batch-size) > 0.
 * As in the reference the batch size does not change the output; the GPU
 * path sizes its own steps (with min_ratio > 0 the reported colours are
 * selected on the device and only they are copied back). out_path NULL =
 * stdout. */
int zx_query_records_report(zx_index* index, const char* query_path, int recover,
                            double min_ratio, int compact, uint64_t batch_records,
                            const char* out_path);

/* Asynchronous query of a batch already in device memory of the index's GPU.
 * d_bases / d_offsets / d_counts / d_total are device pointers; counts and
 * total are ACCUMULATED (the caller zeroes them). stream is a cudaStream_t
 * (NULL = the legacy default stream). use_graph != 0 captures the launch
 * sequence as a CUDA graph on first use of a batch shape and replays it after.
 * Uses the index's shared workspace: callers serialise calls per index. */
int zx_query_device(zx_index* index, const uint8_t* d_bases, uint64_t nbases,
                    const uint64_t* d_offsets, uint64_t records, int recover,
                    uint64_t* d_counts, uint64_t* d_total, void* stream, int use_graph);

/* Allocation-free variant of zx_query_device. No counterpart in the
 * reference: it exists for callers that cannot allocate device memory while
 * querying, such as a host process whose HBM is already fully reserved by its
 * own allocator or by resident indexes, or latency-critical loops that must
 * not enter the driver's allocator (cudaMalloc / cudaFree can synchronise the
 * device). It performs no cudaMalloc, cudaFree or allocating library call:
 * its scratch (packed bases, tile plan, scan workspace) lives in one
 * file-scope device array of 64 MiB per GPU that loads the library, held
 * until process exit. The first call on a device resolves that array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture. Limit: about 0.4 byte per base plus 28 bytes per record must fit in
 * 64 MiB (for example 150 Mbp cannot, 100 Mbp of short reads can); larger
 * batches return ZX_EINVAL with the needed size. Colour counts are added into
 * d_counts / d_total (caller-zeroed) with global atomics. Every call shares
 * the one array, so calls that overlap on the GPU (different streams, or
 * different indexes on the same GPU) race: serialise them. Asynchronous on
 * `stream` (a cudaStream_t; NULL = legacy default stream). Errors found on
 * the device (invalid record offsets) are kept in an error word of this
 * index inside the array (up to 1024 open indexes per GPU use the call; the
 * first call of an index takes its word and clears it, synchronously): later
 * calls do not clear it, and zx_query_status of this index reports and clears
 * it. */
int zx_query_device_noalloc(zx_index* index, const uint8_t* d_bases, uint64_t nbases,
                            const uint64_t* d_offsets, uint64_t records, int recover,
                            uint64_t* d_counts, uint64_t* d_total, void* stream);

/* Seeds of host records, in record and window order, as the reference's
 * scan_index_features emits them (src/lib.rs:574-642). *count receives the
 * total number of seeds; at most cap are written. */
int zx_extract_seeds(zx_index* index, const uint8_t* bases, const uint64_t* offsets,
                     uint64_t records, uint64_t* out, uint64_t cap, uint64_t* count);

/* Launch configuration of the batched kernels (autotuner / planner hook;
 * never changes results). */
int zx_get_launch(const zx_index* index, zx_launch* out);
int zx_set_launch(zx_index* index, const zx_launch* launch);
int zx_default_launch(const zx_index* index, zx_launch* out);
/* The default launch of the fused kernel's forms (wide = 0): what a launch
 * that leaves the wide-row form starts from; the same as zx_default_launch
 * for indexes whose default is not the wide-row form. */
int zx_default_fused_launch(const zx_index* index, zx_launch* out);

/* Status of the asynchronous zx_query_device / zx_query_device_noalloc calls
 * of this index since the last status call: ZX_OK; ZX_EINVAL when record
 * offsets of any of them were invalid
 * (decreasing, past the bases, or a record of 2^31 bases or more: those
 * records were skipped, counts incomplete); ZX_ETIMEOUT when a bounded device
 * wait expired. The device error words are cleared. Synchronous calls report
 * these directly. */
int zx_query_status(zx_index* index);

/* Measurement hook: with timing on, zx_query_device calls made with
 * use_graph == 0 record CUDA events around the fused extraction+probe kernel
 * on the launch stream; zx_last_kernel_ms waits for the last such kernel and
 * returns its duration in milliseconds. */
int zx_set_timing(zx_index* index, int on);
int zx_last_kernel_ms(zx_index* index, float* ms);

/* Several requests coalesced into one asynchronous launch on `stream`, each
 * with its own counters: the batch's records are the requests' records back
 * to back, request s owning records seg_records[s] .. seg_records[s+1]-1
 * (host array of segments + 1 entries, seg_records[segments] == records).
 * counts (device, segments x colours, request-major) and totals (device,
 * segments) are accumulated, not cleared. Each request's counts equal those
 * of querying it alone (query_stream.rs:280-300 per request). Replaces one
 * query_command_with_memory call per query file (storage.rs:3731) when many
 * files are answered by one resident index. */
int zx_query_segments(zx_index* index, const uint8_t* bases, uint64_t nbases,
                      const uint64_t* offsets, uint64_t records, const uint64_t* seg_records,
                      uint32_t segments, int recover, uint64_t* counts, uint64_t* totals,
                      void* stream);

/* Request server over a resident index (no reference counterpart: the
 * reference answers one query file per process run, zorindex.rs:341-343).
 * Requests from any thread are copied at submit, queued, admitted into a
 * batch when one of `slots` batch slots is free and the batch still has room
 * in the slot's device buffers (slot_bases bases, slot_records records,
 * slot_requests requests, sized at start), and answered by one segmented
 * launch per batch; slots run on their own streams, so batches overlap.
 * Results are those of each request queried alone. The index must outlive
 * the server; other calls on the index serialise with its launches. */
typedef struct zx_server zx_server;

typedef struct zx_server_options {
  int slots;              /* batches in flight, 1..16 (0 = 3) */
  uint64_t slot_bases;    /* bases per batch (0 = 64 Mi) */
  uint64_t slot_records;  /* records per batch (0 = 1 Mi) */
  uint32_t slot_requests; /* requests per batch (0 = 512) */
} zx_server_options;

typedef struct zx_server_report {
  uint64_t submitted, completed, failed, batches, seeds, bases;
  double p50_s, p99_s, mean_s, max_s; /* submit-to-completion latency */
  double elapsed_s;                   /* since start or the last reset */
  uint64_t device_bytes;              /* device memory held by the slots */
  uint64_t pinned_bytes;              /* page-locked host memory: the request ring
                                         ((slots + 2) x slot_bases) and the slots */
} zx_server_report;

int zx_server_start(zx_index* index, const zx_server_options* options, zx_server** out);
/* Queue one request (host buffers, copied before returning into the server's
 * page-locked ring, waiting while the ring is full); ZX_EINVAL if it
 * does not fit one batch slot. */
int zx_server_submit(zx_server* server, const uint8_t* bases, const uint64_t* offsets,
                     uint64_t records, int recover, uint64_t* ticket);
/* Wait up to timeout_ms (< 0: forever); ZX_ETIMEOUT if not done yet (the
 * ticket stays valid). On success the counts (colours entries), total and
 * latency are written and the ticket is released. */
int zx_server_wait(zx_server* server, uint64_t ticket, int timeout_ms, uint64_t* counts,
                   uint64_t* total, double* latency_s);
int zx_server_stats(zx_server* server, int reset, zx_server_report* out);
/* Finish every queued request, then stop (pending results are dropped). */
void zx_server_stop(zx_server* server);

/* Learned launch planner network (no reference counterpart: the reference
 * has no launch configuration to choose). A two-layer FP32 perceptron,
 * y = w2 . relu(W1 x + b1) + b2, trained on the GPU by the library's own
 * forward, backward and Adam kernels; parameters in the order W1 (hidden x
 * inputs, row-major), b1, w2, b2. Host arrays: x is n x inputs row-major,
 * targets and outputs n. Inputs 1..32, hidden units 1..64. */
typedef struct zx_mlp zx_mlp;
int zx_mlp_create(int device, int inputs, int hidden, uint64_t seed, zx_mlp** out);
void zx_mlp_destroy(zx_mlp* mlp);
uint64_t zx_mlp_param_count(const zx_mlp* mlp);
int zx_mlp_get_params(zx_mlp* mlp, float* params);
int zx_mlp_set_params(zx_mlp* mlp, const float* params, uint64_t count);
/* Loss (1/2n) sum (y - t)^2 and its gradient (param_count entries, may be NULL). */
int zx_mlp_loss_grad(zx_mlp* mlp, const float* x, const float* targets, uint64_t n, float* loss,
                     float* grad);
/* Full-batch Adam steps; *loss receives the loss after the last step. */
int zx_mlp_train(zx_mlp* mlp, const float* x, const float* targets, uint64_t n, int epochs,
                 float lr, float* loss);
int zx_mlp_predict(zx_mlp* mlp, const float* x, uint64_t n, float* out);

/* Write the aggregate report exactly as print_aggregate does
 * (storage.rs:3817-3844): stdout-style TSV
 * "color\tmatches\tratio\tunique_kmers" with rows whose ratio >= min_ratio to
 * out_path (NULL = stdout), and the "#query\t..." statistics line to stderr
 * when stats != 0. query_label is printed as the query path. */
int zx_write_aggregate(const zx_index* index, const char* query_label, const uint64_t* counts,
                       uint64_t total, uint64_t probes, double min_ratio, double seconds,
                       const char* out_path, int stats);

#ifdef __cplusplus
}
#endif

#endif /* ZINDEX_B200_H */
