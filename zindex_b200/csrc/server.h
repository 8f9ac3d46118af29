// Request server over a resident index: continuous batching of query
// requests into segmented launches (one launch serves many requests, each
// with its own counters).
//
// The reference answers one query file per process run (query_command,
// zorindex.rs:341-343; query_stream.rs:163-452). A server keeps the filters
// resident in HBM and accepts requests from any thread:
//
// * admission: a request's bases are copied at submit, on the submitting
//   thread, into a page-locked ring shared by the slots (submit waits while
//   the ring is full: back-pressure), and the request is queued; it is
//   admitted into a batch when a slot is free and the batch still has room
//   (bases, records, requests) in the slot's device buffers, which are sized
//   once at start (their bytes are the server's device memory budget);
// * continuous batching: whenever a slot is free the scheduler takes the
//   queued requests in arrival order that fit (same recovery flag) and
//   launches them at once; requests that arrive while others run are taken
//   by the next free slot, so batches grow with load;
// * overlap: every slot has its own CUDA stream; the scheduler only issues
//   asynchronous copies from the ring (one per run of ring-adjacent
//   requests), so the copies of one batch overlap the kernels of another;
// * latency: submit-to-completion time of every request (p50/p99 in stats()).
//
// Results are exactly those of a query of the request alone (integer counts;
// the segmented launch gives each request its own blocks and counters).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "host/span_ring.h"

namespace zx {

struct ServerOptions {
  int slots = 3;                     // batches in flight (one stream each)
  uint64_t slot_bases = 64ull << 20;  // bases per batch
  uint64_t slot_records = 1ull << 20; // records per batch
  uint32_t slot_requests = 512;       // requests per batch
};

struct ServerStats {
  uint64_t submitted = 0, completed = 0, failed = 0, batches = 0, seeds = 0, bases = 0;
  double p50_s = 0, p99_s = 0, mean_s = 0, max_s = 0;
  double elapsed_s = 0;       // since start or the last reset
  uint64_t device_bytes = 0;  // device memory held by the slots
  uint64_t pinned_bytes = 0;  // page-locked host memory of the ring and the slots
};

class Server {
 public:
  // `index_mu` serialises the server's launch preparation with other users of
  // the engine.
  Server(Engine& engine, std::mutex& index_mu, const ServerOptions& options);
  ~Server();
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  // Queues a request (host buffers, copied before returning); returns its ticket.
  uint64_t submit(const uint8_t* bases, uint64_t nbases, const uint64_t* offsets, uint64_t records,
                  bool recover);
  // Waits up to timeout_ms (< 0: forever) for a request; false on timeout.
  // On success copies its counts (colours entries) and total and forgets it.
  bool wait(uint64_t ticket, int timeout_ms, uint64_t* counts, uint64_t* total, double* latency_s);
  ServerStats stats(bool reset);

 private:
  using Clock = std::chrono::steady_clock;
  struct Request {
    uint64_t id = 0;
    uint64_t nbases = 0;
    uint64_t ring_off = 0;          // the bases' span in the ring
    uint64_t span = 0;              // its ring span id (0: no span, no bases)
    std::vector<uint64_t> offsets;  // records + 1, from 0
    bool recover = true;
    uint64_t est_tiles = 0;
    Clock::time_point arrival;
    bool done = false;
    std::string error;
    std::vector<uint64_t> counts;
    uint64_t total = 0;
    double latency = 0;
  };
  struct Slot {
    std::unique_ptr<Workspace> ws;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    uint8_t* d_bases = nullptr;
    uint64_t* d_offsets = nullptr;
    uint64_t* d_counts = nullptr;
    unsigned long long* d_totals = nullptr;
    uint64_t* h_offsets = nullptr;
    uint64_t* h_counts = nullptr;
    unsigned long long* h_totals = nullptr;
    std::vector<std::shared_ptr<Request>> batch;
    bool busy = false;
  };

  void run();
  bool launch(Slot& slot);
  void finish(Slot& slot, const std::string& error);
  void release(Slot& slot);
  // Ring spans: reserve waits until n contiguous bytes of the ring are free
  // and returns (offset, span id); release frees a span.
  std::pair<uint64_t, uint64_t> ring_reserve(uint64_t n);
  void ring_release(uint64_t span);

  Engine& engine_;
  std::mutex& index_mu_;
  ServerOptions opt_;
  uint64_t colors_ = 0;
  uint64_t device_bytes_ = 0;
  std::vector<Slot> slots_;

  std::mutex ring_mu_;
  std::condition_variable ring_cv_;
  uint8_t* ring_ = nullptr;  // page-locked request bases
  uint64_t ring_cap_ = 0;
  SpanRing spans_;
  bool ring_stop_ = false;
  uint64_t pinned_bytes_ = 0;

  std::mutex mu_;  // queue, requests, stats
  std::condition_variable cv_submit_, cv_done_;
  std::deque<std::shared_ptr<Request>> queue_;
  std::map<uint64_t, std::shared_ptr<Request>> requests_;
  uint64_t next_id_ = 1;
  bool stop_ = false;
  std::vector<double> latencies_;
  uint64_t submitted_ = 0, completed_ = 0, failed_ = 0, batches_ = 0, seeds_ = 0, bases_ = 0;
  Clock::time_point since_;
  std::thread thread_;
};

}  // namespace zx
