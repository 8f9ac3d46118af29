// Request server: continuous batching over segmented launches (see server.h).
#include "server.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "host/error.h"

namespace zx {

namespace {

template <class T>
T* device_array(uint64_t count, const char* what) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, std::max<uint64_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    raise(kENoMem, std::string("server: device allocation failed for ") + what + ": " +
                       cudaGetErrorString(e));
  }
  return static_cast<T*>(p);
}

template <class T>
T* pinned_array(uint64_t count) {
  void* p = nullptr;
  cuda_check(cudaMallocHost(&p, std::max<uint64_t>(count, 1) * sizeof(T)), "cudaMallocHost");
  return static_cast<T*>(p);
}

}  // namespace

Server::Server(Engine& engine, std::mutex& index_mu, const ServerOptions& options)
    : engine_(engine), index_mu_(index_mu), opt_(options) {
  engine_.check_not_strobes();
  check(opt_.slots >= 1 && opt_.slots <= 16, kEInval, "server slots must be in 1..16");
  check(opt_.slot_bases >= 1024 && opt_.slot_records >= 1 && opt_.slot_requests >= 1, kEInval,
        "server slot capacities must be positive (at least 1024 bases)");
  check(opt_.slot_bases < (1ull << 31), kEInval, "server slots hold fewer than 2^31 bases");
  colors_ = engine_.manifest().colors.size();
  cuda_check(cudaSetDevice(engine_.device()), "cudaSetDevice");
  size_t free_before = 0, total_mem = 0, free_after = 0;
  cuda_check(cudaMemGetInfo(&free_before, &total_mem), "cudaMemGetInfo");
  slots_.resize((size_t)opt_.slots);
  try {
    std::lock_guard<std::mutex> lock(index_mu_);
    for (auto& s : slots_) {
      s.ws = engine_.make_workspace();
      engine_.reserve(*s.ws, opt_.slot_bases, opt_.slot_records);
      s.stream = s.ws->stream;
      cuda_check(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming), "cudaEventCreate");
      s.d_bases = s.ws->bases;
      s.d_offsets = s.ws->offsets;
      s.d_counts = device_array<uint64_t>((uint64_t)opt_.slot_requests * colors_, "counts");
      s.d_totals = device_array<unsigned long long>(opt_.slot_requests, "totals");
      s.h_offsets = pinned_array<uint64_t>(opt_.slot_records + 1);
      s.h_counts = pinned_array<uint64_t>((uint64_t)opt_.slot_requests * colors_);
      s.h_totals = pinned_array<unsigned long long>(opt_.slot_requests);
    }
  } catch (...) {
    for (auto& s : slots_) release(s);
    throw;
  }
  // The ring holds every slot's batch and two more, so submitters rarely wait
  // while batches run.
  ring_cap_ = (uint64_t)(opt_.slots + 2) * opt_.slot_bases;
  spans_ = SpanRing(ring_cap_);
  try {
    ring_ = pinned_array<uint8_t>(ring_cap_);
  } catch (...) {
    for (auto& s : slots_) release(s);
    throw;
  }
  pinned_bytes_ = ring_cap_ + (uint64_t)opt_.slots *
                                  ((opt_.slot_records + 1) * 8 +
                                   (uint64_t)opt_.slot_requests * (colors_ + 1) * 8);
  cuda_check(cudaMemGetInfo(&free_after, &total_mem), "cudaMemGetInfo");
  device_bytes_ = free_before > free_after ? free_before - free_after : 0;
  since_ = Clock::now();
  thread_ = std::thread([this] { run(); });
}

void Server::release(Slot& s) {
  if (s.done) cudaEventDestroy(s.done);
  if (s.d_counts) cudaFree(s.d_counts);
  if (s.d_totals) cudaFree(s.d_totals);
  for (void* p : {(void*)s.h_offsets, (void*)s.h_counts, (void*)s.h_totals})
    if (p) cudaFreeHost(p);
  s = Slot{};
}

std::pair<uint64_t, uint64_t> Server::ring_reserve(uint64_t n) {
  std::unique_lock<std::mutex> lk(ring_mu_);
  uint64_t off = 0, id = 0;
  for (;;) {
    check(!ring_stop_, kEInval, "server is stopping");
    if (spans_.reserve(n, &off, &id)) return {off, id};
    ring_cv_.wait(lk);
  }
}

void Server::ring_release(uint64_t span) {
  if (!span) return;
  {
    std::lock_guard<std::mutex> lk(ring_mu_);
    spans_.release(span);
  }
  ring_cv_.notify_all();
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  {
    std::lock_guard<std::mutex> lk(ring_mu_);
    ring_stop_ = true;
  }
  ring_cv_.notify_all();
  cv_submit_.notify_all();
  if (thread_.joinable()) thread_.join();
  cudaSetDevice(engine_.device());
  for (auto& s : slots_) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    release(s);
  }
  if (ring_) cudaFreeHost(ring_);
}

uint64_t Server::submit(const uint8_t* bases, uint64_t nbases, const uint64_t* offsets,
                        uint64_t records, bool recover) {
  check(offsets && (bases || nbases == 0), kEInval, "null argument");
  check(offsets[0] == 0 && offsets[records] == nbases, kEInval, "offsets must span the bases");
  if (nbases > opt_.slot_bases || records > opt_.slot_records)
    raise(kEInval, "request exceeds one batch slot of the server (" +
                       std::to_string(opt_.slot_bases) + " bases, " +
                       std::to_string(opt_.slot_records) + " records): split it");
  auto r = std::make_shared<Request>();
  r->arrival = Clock::now();
  r->offsets.assign(offsets, offsets + records + 1);
  r->recover = recover;
  for (uint64_t i = 0; i < records; ++i) {
    check(offsets[i] <= offsets[i + 1], kEInval, "offsets must not decrease");
    r->est_tiles += engine_.tiles_for_length(offsets[i + 1] - offsets[i]);
  }
  r->nbases = nbases;
  if (nbases) {
    const auto span = ring_reserve(nbases);
    r->ring_off = span.first;
    r->span = span.second;
    memcpy(ring_ + r->ring_off, bases, nbases);
  }
  uint64_t id;
  {
    std::lock_guard<std::mutex> lk(mu_);
    if (stop_) {
      ring_release(r->span);
      raise(kEInval, "server is stopping");
    }
    id = next_id_++;
    r->id = id;
    queue_.push_back(r);
    requests_[id] = r;
    ++submitted_;
  }
  cv_submit_.notify_one();
  return id;
}

bool Server::wait(uint64_t ticket, int timeout_ms, uint64_t* counts, uint64_t* total,
                  double* latency_s) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = requests_.find(ticket);
  check(it != requests_.end(), kEInval, "unknown or already collected ticket");
  std::shared_ptr<Request> r = it->second;
  auto ready = [&] { return r->done; };
  if (timeout_ms < 0) cv_done_.wait(lk, ready);
  else if (!cv_done_.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return false;
  requests_.erase(ticket);
  if (!r->error.empty()) raise(kECuda, "request failed: " + r->error);
  if (counts) std::copy(r->counts.begin(), r->counts.end(), counts);
  if (total) *total = r->total;
  if (latency_s) *latency_s = r->latency;
  return true;
}

ServerStats Server::stats(bool reset) {
  std::lock_guard<std::mutex> lk(mu_);
  ServerStats st;
  st.submitted = submitted_;
  st.completed = completed_;
  st.failed = failed_;
  st.batches = batches_;
  st.seeds = seeds_;
  st.bases = bases_;
  st.device_bytes = device_bytes_;
  st.pinned_bytes = pinned_bytes_;
  st.elapsed_s = std::chrono::duration<double>(Clock::now() - since_).count();
  if (!latencies_.empty()) {
    std::vector<double> v = latencies_;
    std::sort(v.begin(), v.end());
    auto rank = [&](double q) {  // nearest rank
      size_t k = (size_t)std::ceil(q * (double)v.size());
      return v[std::min(v.size(), std::max<size_t>(k, 1)) - 1];
    };
    st.p50_s = rank(0.50);
    st.p99_s = rank(0.99);
    double sum = 0;
    for (double x : v) sum += x;
    st.mean_s = sum / (double)v.size();
    st.max_s = v.back();
  }
  if (reset) {
    latencies_.clear();
    submitted_ = completed_ = failed_ = batches_ = seeds_ = bases_ = 0;
    since_ = Clock::now();
  }
  return st;
}

// Takes the queued requests that fit one slot (arrival order, same recovery
// flag) and launches them as one segmented query. False when none is queued.
bool Server::launch(Slot& s) {
  std::vector<std::shared_ptr<Request>> batch;
  uint64_t nb = 0, nr = 0;
  {
    std::lock_guard<std::mutex> lk(mu_);
    if (queue_.empty()) return false;
    const bool rec = queue_.front()->recover;
    while (!queue_.empty() && batch.size() < opt_.slot_requests) {
      const auto& r = queue_.front();
      const uint64_t rb = r->nbases, rr = r->offsets.size() - 1;
      if (r->recover != rec || nb + rb > opt_.slot_bases || nr + rr > opt_.slot_records) break;
      batch.push_back(r);
      queue_.pop_front();
      nb += rb;
      nr += rr;
    }
  }
  const uint32_t n = (uint32_t)batch.size();
  std::vector<uint64_t> seg_records(n + 1), est(n);
  uint64_t at = 0, rec0 = 0;
  s.h_offsets[0] = 0;
  // Copies from the ring: one per run of requests adjacent in it.
  struct Copy {
    uint64_t dst, src, len;
  };
  std::vector<Copy> copies;
  for (uint32_t i = 0; i < n; ++i) {
    const Request& r = *batch[i];
    if (r.nbases) {
      if (!copies.empty() && copies.back().src + copies.back().len == r.ring_off &&
          copies.back().dst + copies.back().len == at)
        copies.back().len += r.nbases;
      else
        copies.push_back(Copy{at, r.ring_off, r.nbases});
    }
    const uint64_t rr = r.offsets.size() - 1;
    for (uint64_t j = 1; j <= rr; ++j) s.h_offsets[rec0 + j] = at + r.offsets[j];
    seg_records[i] = rec0;
    est[i] = r.est_tiles;
    at += r.nbases;
    rec0 += rr;
  }
  seg_records[n] = rec0;
  s.batch = std::move(batch);
  s.busy = true;
  try {
    std::lock_guard<std::mutex> lock(index_mu_);
    for (const Copy& c : copies)
      cuda_check(cudaMemcpyAsync(s.d_bases + c.dst, ring_ + c.src, c.len, cudaMemcpyHostToDevice,
                                 s.stream),
                 "H2D");
    cuda_check(cudaMemcpyAsync(s.d_offsets, s.h_offsets, (nr + 1) * 8, cudaMemcpyHostToDevice,
                               s.stream),
               "H2D");
    cuda_check(cudaMemsetAsync(s.d_counts, 0, (uint64_t)n * colors_ * 8, s.stream), "memset");
    cuda_check(cudaMemsetAsync(s.d_totals, 0, (uint64_t)n * 8, s.stream), "memset");
    engine_.query_segments(*s.ws, s.d_bases, nb, s.d_offsets, nr, seg_records.data(), est.data(),
                           n, s.batch.front()->recover, s.d_counts, s.d_totals, s.stream);
    cuda_check(cudaMemcpyAsync(s.h_counts, s.d_counts, (uint64_t)n * colors_ * 8,
                               cudaMemcpyDeviceToHost, s.stream),
               "D2H");
    cuda_check(cudaMemcpyAsync(s.h_totals, s.d_totals, (uint64_t)n * 8, cudaMemcpyDeviceToHost,
                               s.stream),
               "D2H");
    cuda_check(cudaEventRecord(s.done, s.stream), "cudaEventRecord");
  } catch (const std::exception& e) {
    cudaStreamSynchronize(s.stream);
    finish(s, e.what());
  }
  return true;
}

void Server::finish(Slot& s, const std::string& error) {
  const auto now = Clock::now();
  {
    std::lock_guard<std::mutex> lk(mu_);
    ++batches_;
    for (size_t i = 0; i < s.batch.size(); ++i) {
      Request& r = *s.batch[i];
      r.latency = std::chrono::duration<double>(now - r.arrival).count();
      r.error = error;
      if (error.empty()) {
        r.counts.assign(s.h_counts + i * colors_, s.h_counts + (i + 1) * colors_);
        r.total = s.h_totals[i];
        ++completed_;
        seeds_ += r.total;
        bases_ += r.nbases;
        latencies_.push_back(r.latency);
      } else {
        ++failed_;
      }
      r.done = true;
    }
  }
  // The batch's copies have run: its ring spans are free.
  for (const auto& r : s.batch) ring_release(r->span);
  s.batch.clear();
  s.busy = false;
  cv_done_.notify_all();
}

void Server::run() {
  cudaSetDevice(engine_.device());
  for (;;) {
    bool progress = false, busy = false;
    for (auto& s : slots_) {
      if (!s.busy) continue;
      const cudaError_t q = cudaEventQuery(s.done);
      if (q == cudaSuccess) {
        finish(s, "");
        progress = true;
      } else if (q != cudaErrorNotReady) {
        cudaGetLastError();
        finish(s, cudaGetErrorString(q));
        progress = true;
      } else {
        busy = true;
      }
    }
    for (auto& s : slots_) {
      if (s.busy) continue;
      if (!launch(s)) break;
      progress = true;
      busy = true;
    }
    std::unique_lock<std::mutex> lk(mu_);
    if (stop_ && queue_.empty() && !busy) break;
    if (progress) continue;
    if (busy) cv_submit_.wait_for(lk, std::chrono::microseconds(20));
    else cv_submit_.wait(lk, [&] { return stop_ || !queue_.empty(); });
  }
}

}  // namespace zx
