// TEST INFRASTRUCTURE ONLY. The oracle is the checker for the CUDA query path
// and the timed CPU baseline; the product never links, loads or runs it.
//
// C entry points of liboracle.so, a CPU restatement of the Zindex (zorindex)
// query algorithm. Each function names the reference code it follows.
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// splitmix64 (utils/ocm-minimizers/src/lib.rs:47-53).
uint64_t oracle_splitmix64(uint64_t x);

// Seed extraction of one sequence chunk exactly as scan_index_features
// (src/lib.rs:574-642) would emit it, including the split at non-ACGT bytes.
// mode: 0 kmers, 1 minimizers (open-closed mod), 2 modimizers, 3 findere.
// Writes at most `cap` keys; *count receives the full number of keys.
int oracle_features(const uint8_t* seq, size_t len, int mode, int k, int m, uint64_t seed,
                    uint64_t sampling, int findere_z, int homopolymer, uint64_t* out, size_t cap,
                    size_t* count);

// Window-by-window open-closed mod-minimizer reference
// (src/open_closed_minimizers.rs:43-85), for an all-ACGT `seq`.
int oracle_ocm_slow(const uint8_t* seq, size_t len, int k, int m, uint64_t seed, uint64_t* pos_out,
                    uint64_t* key_out, size_t cap, size_t* count);

// Aggregate query of a FASTA/FASTQ file against an index directory
// (query_command_with_memory, src/power_merge/storage.rs:3731-3767).
// counts must hold `colors` entries. Returns 0 or a nonzero error; the message
// is available from oracle_last_error().
int oracle_query_file(const char* index_dir, const char* query_path, int threads, int recover,
                      uint64_t* counts, size_t colors, uint64_t* total, uint64_t* probes);

// Same query over sequences already in memory: record r spans
// bases[offsets[r] .. offsets[r+1]).
int oracle_query_records(const char* index_dir, const uint8_t* bases, const uint64_t* offsets,
                         size_t records, int threads, int recover, uint64_t* counts, size_t colors,
                         uint64_t* total, uint64_t* probes);

// Number of colours of an index (manifest "colors").
int oracle_index_colors(const char* index_dir, size_t* colors);

// Render the aggregate TSV of print_aggregate (storage.rs:3817-3844) into buf.
int oracle_format_aggregate(const char* index_dir, const uint64_t* counts, uint64_t total,
                            double min_ratio, char* buf, size_t cap, size_t* written);

// Resident index handle for repeated timed queries (the CPU baseline).
typedef struct oracle_index oracle_index;
int oracle_open(const char* index_dir, int recover, oracle_index** out);
void oracle_close(oracle_index* index);
// Query of in-memory records with `threads` workers; *seconds receives the
// query time (parsing of records into seeds + lookup), index load excluded.
int oracle_query_handle(oracle_index* index, const uint8_t* bases, const uint64_t* offsets,
                        size_t records, int threads, uint64_t* counts, size_t colors,
                        uint64_t* total, double* seconds);
// The same query with the reference's lookup_batch blocks, 4-ahead row
// prefetch and AVX2 fingerprint screens (the timed CPU baseline; same
// counts). oracle_fast_serves: 1 when the index takes that path (ordinary
// modes over fingerprint-first banks), else the scalar lookup runs.
int oracle_query_handle_fast(oracle_index* index, const uint8_t* bases, const uint64_t* offsets,
                             size_t records, int threads, uint64_t* counts, size_t colors,
                             uint64_t* total, double* seconds);
int oracle_fast_serves(oracle_index* index);

// Per-record report of a query file as `zorindex query --records` prints it
// (query_records_command_with_memory, src/power_merge/storage.rs:3626-3720):
// TSV (compact = 0) or compact rows; *written = its bytes (copied up to cap
// when buf is not NULL).
int oracle_query_records_report(const char* index_dir, const char* query_path, int recover,
                                double min_ratio, int compact, char* buf, size_t cap,
                                size_t* written);

/* Per-record report over an open index: records split across `threads`
 * workers; *seconds covers reading, querying and formatting. */
int oracle_records_report_handle(oracle_index* index, const char* query_path, double min_ratio,
                                 int compact, int threads, char* buf, size_t cap,
                                 size_t* written, double* seconds);

/* Spaced seed (anchors.rs:15-90): the projection and canonical key of a
 * 2-bit key under a '#'/'_' pattern. */
int oracle_pattern_canonical(const char* pattern, uint64_t key, uint64_t* projected,
                             uint64_t* canonical);

/* Randstrobemers (anchors.rs:129-347): the XXH64 strobe hash of one u64, and
 * the seeds of a sequence with an optional pattern and strobe linking. */
uint64_t oracle_strobe_hash(uint64_t v);
/* PositionHash::positions (storage.rs:3452-3481; segment 0 = legacy length)
 * and abandoned::hash (abandoned.rs:5-10). */
void oracle_positions(uint64_t key, uint64_t seed, uint64_t cells, int hashes, uint64_t segment,
                      uint64_t* out);
uint32_t oracle_abandoned_hash(uint64_t key, uint64_t seed);
void oracle_link_strobes(const uint64_t* positions, const uint64_t* hashes, size_t n,
                         uint64_t dmin, uint64_t dmax, uint64_t* out);
int oracle_features_anchored(const uint8_t* seq, size_t len, int mode, int k, int m, uint64_t seed,
                             int homopolymer, const char* pattern, uint64_t strobe_min,
                             uint64_t strobe_max, uint64_t* out, size_t cap, size_t* count);

const char* oracle_last_error(void);

#ifdef __cplusplus
}
#endif
