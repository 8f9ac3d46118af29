// extern "C" boundary (include/zindex.h). Converts zx::Error and CUDA
// failures into status codes plus a thread-local message.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/zindex.h"
#include "engine.h"
#include "host/error.h"
#include "planner.h"
#include "server.h"
#include "host/fastx.h"
#include "host/record_report.h"
#include <thread>

struct zx_index {
  std::unique_ptr<zx::Engine> engine;
  std::mutex mu;  // guards the shared workspace
  std::unique_ptr<zx::Workspace> seg_ws;  // zx_query_segments
};

struct zx_server {
  std::unique_ptr<zx::Server> server;
};

struct zx_mlp {
  std::unique_ptr<zx::Mlp> net;
};

namespace {

thread_local std::string g_last_error;

template <class F>
int guarded(F&& body) {
  try {
    body();
    g_last_error.clear();
    return ZX_OK;
  } catch (const zx::Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host memory exhausted";
    return ZX_ENOMEM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return ZX_EINVAL;
  }
}

void fill_launch(const zx::QueryLaunch& l, zx_launch* out) {
  out->team = l.team;
  out->warps = l.warps;
  out->blocks = l.blocks;
  out->smem_counters = l.smem_counters;
  out->stage_bytes = l.stage_bytes;
  out->stages = l.stages;
  out->bulk = l.bulk;
  out->min_blocks = l.min_blocks;
  out->planes = l.planes;
  out->cut = l.cut;
  out->split = l.split;
  out->wide = l.wide;
  out->order = l.order;
}

}  // namespace

extern "C" {

const char* zx_last_error(void) { return g_last_error.c_str(); }

int zx_open(const char* index_dir, int device, uint64_t hbm_budget, zx_index** out) {
  return guarded([&] {
    zx::check(index_dir && out, zx::kEInval, "null argument");
    *out = nullptr;
    zx::OpenOptions o;
    o.device = device;
    o.hbm_budget = hbm_budget;
    auto ix = std::make_unique<zx_index>();
    ix->engine = std::make_unique<zx::Engine>(index_dir, o);
    *out = ix.release();
  });
}

void zx_close(zx_index* index) { delete index; }

int zx_index_info(const zx_index* index, zx_info* out) {
  return guarded([&] {
    zx::check(index && out, zx::kEInval, "null argument");
    const zx::Manifest& m = index->engine->manifest();
    memset(out, 0, sizeof *out);
    out->version = m.version;
    out->k = (uint32_t)m.k;
    out->hashes = (uint32_t)m.hashes;
    out->fingerprint_bits = (uint32_t)m.fingerprint_bits;
    out->index_mode = (uint32_t)m.index_mode;
    out->minimizer_size = (uint32_t)m.minimizer_size;
    out->seed = m.seed;
    out->colors = m.colors.size();
    out->banks = m.banks.size();
    out->classes = m.classes.size();
    out->resident_bytes = index->engine->resident_bytes();
    out->gather_bytes_per_seed = index->engine->gather_bytes_per_seed();
    out->gather_sector_bytes_per_seed = index->engine->gather_sector_bytes_per_seed();
    out->abandoned_hashes = m.abandoned_hashes;
    out->recovery = m.abandoned_recovery ? 1 : 0;
    out->load_s = index->engine->load_seconds();
    out->load_banks_s = index->engine->banks_load_seconds();
    out->load_recovery_s = index->engine->recovery_load_seconds();
  });
}

const char* zx_color_name(const zx_index* index, uint64_t color) {
  if (!index || color >= index->engine->manifest().colors.size()) return nullptr;
  return index->engine->manifest().colors[color].name.c_str();
}

uint64_t zx_color_unique_kmers(const zx_index* index, uint64_t color) {
  if (!index || color >= index->engine->manifest().colors.size()) return 0;
  return index->engine->manifest().colors[color].unique_kmers;
}

int zx_query_host(zx_index* index, const uint8_t* bases, const uint64_t* offsets,
                  uint64_t records, int recover, uint64_t* counts, uint64_t* total) {
  return guarded([&] {
    zx::check(index && offsets && counts && total && (bases || !offsets[records]), zx::kEInval,
              "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    auto& e = *index->engine;
    e.query_host(e.default_workspace(), bases, offsets[records], offsets, records, recover != 0,
                 counts, total);
  });
}

int zx_query_host_plain(zx_index* index, const uint8_t* bases, const uint64_t* offsets,
                        uint64_t records, int recover, uint64_t* counts, uint64_t* total) {
  return guarded([&] {
    zx::check(index && offsets && counts && total && (bases || !offsets[records]), zx::kEInval,
              "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    auto& e = *index->engine;
    e.query_host_plain(e.default_workspace(), bases, offsets[records], offsets, records,
                       recover != 0, counts, total);
  });
}

int zx_query_file(zx_index* index, const char* query_path, int recover, uint64_t* counts,
                  uint64_t* total, uint64_t* probes) {
  return guarded([&] {
    zx::check(index && query_path && counts && total, zx::kEInval, "null argument");
    zx::RecordBatch batch = zx::read_fastx(query_path, false);
    std::lock_guard<std::mutex> lock(index->mu);
    auto& e = *index->engine;
    e.query_host(e.default_workspace(), batch.bases.data(), batch.bases.size(),
                 batch.offsets.data(), batch.records(), recover != 0, counts, total);
    if (probes) *probes = *total;
  });
}

int zx_query_per_record(zx_index* index, const uint8_t* bases, const uint64_t* offsets,
                        uint64_t records, int recover, uint64_t* counts, uint64_t* totals) {
  return guarded([&] {
    zx::check(index && offsets && (counts || !records) && (totals || !records) &&
                  (bases || !offsets[records]),
              zx::kEInval, "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    auto& e = *index->engine;
    e.query_per_record(e.default_workspace(), bases, offsets[records], offsets, records,
                       recover != 0, counts, totals);
  });
}

int zx_query_records_report(zx_index* index, const char* query_path, int recover,
                            double min_ratio, int compact, uint64_t batch_records,
                            const char* out_path) {
  return guarded([&] {
    zx::check(index && query_path, zx::kEInval, "null argument");
    zx::check(min_ratio >= 0.0 && min_ratio <= 1.0, zx::kEInval, "--min-ratio must be in [0, 1]");
    zx::check(batch_records > 0, zx::kEInval, "record batch size must be positive");
    zx::check(compact == 0 || compact == 1, zx::kEInval, "format must be 0 (tsv) or 1 (compact)");
    const zx::RecordFormat format = compact ? zx::RecordFormat::kCompact : zx::RecordFormat::kTsv;
    zx::RecordBatch rb = zx::read_named_records(query_path);
    std::lock_guard<std::mutex> lock(index->mu);
    auto& e = *index->engine;
    const auto& colors = e.manifest().colors;
    const uint64_t C = std::max<uint64_t>(colors.size(), 1);
    const uint64_t records = rb.records();
    // With a threshold the reported colours are selected on the device and
    // only they are copied back; with min_ratio 0 every colour is reported and
    // the dense counts come back, at most 256 MiB of them per step. The step
    // (like the reference's record batch size) does not change the output.
    const bool sparse = min_ratio > 0.0 && !e.strobes();
    const uint64_t step = sparse ? (1ull << 18) : std::max<uint64_t>(1, (32ull << 20) / C);
    FILE* f = out_path ? fopen(out_path, "wb") : stdout;
    if (!f) zx::raise(zx::kEIo, std::string("cannot create ") + out_path);
    struct Closer {
      FILE* f;
      bool own;
      ~Closer() {
        if (own) fclose(f);
      }
    } closer{f, out_path != nullptr};
    std::string head = zx::record_header(format);
    head += '\n';
    bool write_ok = fwrite(head.data(), 1, head.size(), f) == head.size();
    // Step i's report is formatted and written on a second thread while the
    // GPU runs step i + 1.
    std::vector<uint64_t> counts[2], totals[2];
    zx::Engine::RecordHits hits[2];
    std::vector<uint64_t> rel;
    std::vector<std::string> text[2];
    const uint64_t formatters = std::max(1u, std::thread::hardware_concurrency());
    std::thread writer;
    auto join = [&] {
      if (writer.joinable()) writer.join();
    };
    try {
      uint64_t i = 0;
      for (uint64_t r0 = 0; r0 < records; r0 += step, ++i) {
        const uint64_t n = std::min(step, records - r0), b = i & 1, b0 = rb.offsets[r0];
        rel.resize(n + 1);
        for (uint64_t r = 0; r <= n; ++r) rel[r] = rb.offsets[r0 + r] - b0;
        if (sparse) {
          e.query_record_hits(e.default_workspace(), rb.bases.data() + b0, rel[n], rel.data(), n,
                              recover != 0, min_ratio, hits[b]);
        } else {
          counts[b].resize(n * colors.size());
          totals[b].resize(n);
          e.query_per_record(e.default_workspace(), rb.bases.data() + b0, rel[n], rel.data(), n,
                             recover != 0, counts[b].data(), totals[b].data());
        }
        join();
        writer = std::thread([&, b, r0, n] {
          // Records are formatted by up to `formatters` threads in contiguous
          // runs (a dense report writes every colour of every record) and
          // written in input order.
          auto format_range = [&](uint64_t lo, uint64_t hi, std::string& t) {
            t.clear();
            for (uint64_t r = lo; r < hi; ++r) {
              if (sparse) {
                const auto& h = hits[b];
                zx::append_record_hits(t, format, rb.names[r0 + r], h.totals[r],
                                       h.colors.data() + h.first[r], h.counts.data() + h.first[r],
                                       h.first[r + 1] - h.first[r], colors);
              } else {
                zx::append_record(t, format, rb.names[r0 + r], totals[b][r],
                                  counts[b].data() + r * colors.size(), colors, min_ratio);
              }
            }
          };
          const uint64_t cells = n * (sparse ? 1 : colors.size());
          const uint64_t parts =
              std::max<uint64_t>(1, std::min<uint64_t>({formatters, n, cells / 65536 + 1}));
          std::vector<std::string>& pieces = text[b];
          pieces.resize(parts);
          std::vector<std::thread> pool;
          for (uint64_t i = 1; i < parts; ++i)
            pool.emplace_back(format_range, n * i / parts, n * (i + 1) / parts,
                              std::ref(pieces[i]));
          format_range(0, n / parts, pieces[0]);
          for (auto& th : pool) th.join();
          for (const std::string& t : pieces)
            if (fwrite(t.data(), 1, t.size(), f) != t.size()) write_ok = false;
        });
      }
      join();
    } catch (...) {
      join();
      throw;
    }
    if (fflush(f) != 0) write_ok = false;
    zx::check(write_ok, zx::kEIo, "writing the per-record report failed");
  });
}

int zx_query_device(zx_index* index, const uint8_t* d_bases, uint64_t nbases,
                    const uint64_t* d_offsets, uint64_t records, int recover,
                    uint64_t* d_counts, uint64_t* d_total, void* stream, int use_graph) {
  return guarded([&] {
    zx::check(index && d_offsets && d_counts && d_total, zx::kEInval, "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    auto& e = *index->engine;
    e.query_device(e.default_workspace(), d_bases, nbases, d_offsets, records, recover != 0,
                   d_counts, reinterpret_cast<unsigned long long*>(d_total),
                   static_cast<cudaStream_t>(stream), use_graph != 0);
  });
}

int zx_query_device_noalloc(zx_index* index, const uint8_t* d_bases, uint64_t nbases,
                            const uint64_t* d_offsets, uint64_t records, int recover,
                            uint64_t* d_counts, uint64_t* d_total, void* stream) {
  return guarded([&] {
    zx::check(index && d_offsets && d_counts && d_total, zx::kEInval, "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    index->engine->query_device_noalloc(d_bases, nbases, d_offsets, records, recover != 0,
                                        d_counts, reinterpret_cast<unsigned long long*>(d_total),
                                        static_cast<cudaStream_t>(stream));
  });
}

int zx_extract_seeds(zx_index* index, const uint8_t* bases, const uint64_t* offsets,
                     uint64_t records, uint64_t* out, uint64_t cap, uint64_t* count) {
  return guarded([&] {
    zx::check(index && offsets && count, zx::kEInval, "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    auto& e = *index->engine;
    std::vector<uint64_t> keys;
    e.extract_host(e.default_workspace(), bases, offsets[records], offsets, records, keys);
    *count = keys.size();
    if (out) memcpy(out, keys.data(), std::min<uint64_t>(cap, keys.size()) * 8);
  });
}

int zx_get_launch(const zx_index* index, zx_launch* out) {
  return guarded([&] {
    zx::check(index && out, zx::kEInval, "null argument");
    fill_launch(index->engine->launch(), out);
  });
}

int zx_default_launch(const zx_index* index, zx_launch* out) {
  return guarded([&] {
    zx::check(index && out, zx::kEInval, "null argument");
    fill_launch(index->engine->default_launch(), out);
  });
}

int zx_default_fused_launch(const zx_index* index, zx_launch* out) {
  return guarded([&] {
    zx::check(index && out, zx::kEInval, "null argument");
    fill_launch(index->engine->default_fused_launch(), out);
  });
}

int zx_set_launch(zx_index* index, const zx_launch* l) {
  return guarded([&] {
    zx::check(index && l, zx::kEInval, "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    index->engine->set_launch(
        zx::QueryLaunch{l->team, l->warps, l->blocks, l->smem_counters, l->stage_bytes, l->stages,
                        l->bulk, l->min_blocks, l->planes, l->cut, l->split, l->wide,
                        l->order});
  });
}

int zx_query_status(zx_index* index) {
  return guarded([&] {
    zx::check(index, zx::kEInval, "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    auto& e = *index->engine;
    const uint32_t err = e.take_error(e.default_workspace()) | e.take_noalloc_error();
    if (err & zx::kErrOffsets)
      zx::raise(zx::kEInval, "record offsets of an asynchronous query were invalid (decreasing, "
                             "past the bases or spanning 2^31 bases); those records were skipped");
    if (err) zx::raise(zx::kETimeout, "a bounded device wait expired during a query");
  });
}

int zx_set_timing(zx_index* index, int on) {
  return guarded([&] {
    zx::check(index, zx::kEInval, "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    index->engine->set_timing(on != 0);
  });
}

int zx_last_kernel_ms(zx_index* index, float* ms) {
  return guarded([&] {
    zx::check(index && ms, zx::kEInval, "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    *ms = index->engine->last_fused_ms();
  });
}

int zx_query_segments(zx_index* index, const uint8_t* bases, uint64_t nbases,
                      const uint64_t* offsets, uint64_t records, const uint64_t* seg_records,
                      uint32_t segments, int recover, uint64_t* counts, uint64_t* totals,
                      void* stream) {
  return guarded([&] {
    zx::check(index && offsets && seg_records && counts && totals && (bases || nbases == 0),
              zx::kEInval, "null argument");
    std::lock_guard<std::mutex> lock(index->mu);
    auto& e = *index->engine;
    e.check_not_strobes();
    if (!index->seg_ws) index->seg_ws = e.make_workspace();
    // Grid shares from the record counts (the lengths stay on the device).
    std::vector<uint64_t> est(segments);
    for (uint32_t s = 0; s < segments; ++s) est[s] = seg_records[s + 1] - seg_records[s] + 1;
    e.query_segments(*index->seg_ws, bases, nbases, offsets, records, seg_records, est.data(),
                     segments, recover != 0, counts, reinterpret_cast<unsigned long long*>(totals),
                     static_cast<cudaStream_t>(stream));
  });
}

int zx_server_start(zx_index* index, const zx_server_options* options, zx_server** out) {
  return guarded([&] {
    zx::check(index && out, zx::kEInval, "null argument");
    *out = nullptr;
    zx::ServerOptions o;
    if (options) {
      if (options->slots) o.slots = options->slots;
      if (options->slot_bases) o.slot_bases = options->slot_bases;
      if (options->slot_records) o.slot_records = options->slot_records;
      if (options->slot_requests) o.slot_requests = options->slot_requests;
    }
    auto sv = std::make_unique<zx_server>();
    sv->server = std::make_unique<zx::Server>(*index->engine, index->mu, o);
    *out = sv.release();
  });
}

int zx_server_submit(zx_server* server, const uint8_t* bases, const uint64_t* offsets,
                     uint64_t records, int recover, uint64_t* ticket) {
  return guarded([&] {
    zx::check(server && offsets && ticket, zx::kEInval, "null argument");
    *ticket = server->server->submit(bases, offsets[records], offsets, records, recover != 0);
  });
}

int zx_server_wait(zx_server* server, uint64_t ticket, int timeout_ms, uint64_t* counts,
                   uint64_t* total, double* latency_s) {
  return guarded([&] {
    zx::check(server, zx::kEInval, "null argument");
    if (!server->server->wait(ticket, timeout_ms, counts, total, latency_s))
      zx::raise(zx::kETimeout, "request not finished yet");
  });
}

int zx_server_stats(zx_server* server, int reset, zx_server_report* out) {
  return guarded([&] {
    zx::check(server && out, zx::kEInval, "null argument");
    const zx::ServerStats st = server->server->stats(reset != 0);
    out->submitted = st.submitted;
    out->completed = st.completed;
    out->failed = st.failed;
    out->batches = st.batches;
    out->seeds = st.seeds;
    out->bases = st.bases;
    out->p50_s = st.p50_s;
    out->p99_s = st.p99_s;
    out->mean_s = st.mean_s;
    out->max_s = st.max_s;
    out->elapsed_s = st.elapsed_s;
    out->device_bytes = st.device_bytes;
    out->pinned_bytes = st.pinned_bytes;
  });
}

void zx_server_stop(zx_server* server) { delete server; }

int zx_mlp_create(int device, int inputs, int hidden, uint64_t seed, zx_mlp** out) {
  return guarded([&] {
    zx::check(out != nullptr, zx::kEInval, "null argument");
    *out = nullptr;
    auto m = std::make_unique<zx_mlp>();
    m->net = std::make_unique<zx::Mlp>(device, inputs, hidden, seed);
    *out = m.release();
  });
}

void zx_mlp_destroy(zx_mlp* mlp) { delete mlp; }

uint64_t zx_mlp_param_count(const zx_mlp* mlp) { return mlp ? mlp->net->param_count() : 0; }

int zx_mlp_get_params(zx_mlp* mlp, float* params) {
  return guarded([&] {
    zx::check(mlp && params, zx::kEInval, "null argument");
    const std::vector<float> p = mlp->net->params();
    std::copy(p.begin(), p.end(), params);
  });
}

int zx_mlp_set_params(zx_mlp* mlp, const float* params, uint64_t count) {
  return guarded([&] {
    zx::check(mlp && params, zx::kEInval, "null argument");
    mlp->net->set_params(params, count);
  });
}

int zx_mlp_loss_grad(zx_mlp* mlp, const float* x, const float* targets, uint64_t n, float* loss,
                     float* grad) {
  return guarded([&] {
    zx::check(mlp && x && targets && loss, zx::kEInval, "null argument");
    *loss = mlp->net->loss_grad(x, targets, n, grad);
  });
}

int zx_mlp_train(zx_mlp* mlp, const float* x, const float* targets, uint64_t n, int epochs,
                 float lr, float* loss) {
  return guarded([&] {
    zx::check(mlp && x && targets && loss, zx::kEInval, "null argument");
    *loss = mlp->net->train(x, targets, n, epochs, lr);
  });
}

int zx_mlp_predict(zx_mlp* mlp, const float* x, uint64_t n, float* out) {
  return guarded([&] {
    zx::check(mlp && x && out, zx::kEInval, "null argument");
    mlp->net->predict(x, n, out);
  });
}

int zx_write_aggregate(const zx_index* index, const char* query_label, const uint64_t* counts,
                       uint64_t total, uint64_t probes, double min_ratio, double seconds,
                       const char* out_path, int stats) {
  return guarded([&] {
    zx::check(index && counts, zx::kEInval, "null argument");
    const zx::Manifest& m = index->engine->manifest();
    if (stats)
      fprintf(stderr,
              "#query\t%s\tk=%llu\tindex_mode=%s\ttotal_features=%llu\tstack_probes=%llu\t"
              "bank_probes=%llu\telapsed_s=%.6f\n",
              query_label ? query_label : "", (unsigned long long)m.k,
              zx::index_mode_label(m.index_mode), (unsigned long long)total,
              (unsigned long long)probes, (unsigned long long)(probes * m.classes.size()),
              seconds);
    FILE* f = out_path ? fopen(out_path, "w") : stdout;
    if (!f) zx::raise(zx::kEIo, std::string("cannot create ") + out_path);
    fputs("color\tmatches\tratio\tunique_kmers\n", f);
    for (size_t c = 0; c < m.colors.size(); ++c) {
      double ratio = total == 0 ? 0.0 : (double)counts[c] / (double)total;
      if (!(ratio >= min_ratio)) continue;
      fprintf(f, "%s\t%llu\t%.8f\t%llu\n", m.colors[c].name.c_str(), (unsigned long long)counts[c],
              ratio, (unsigned long long)m.colors[c].unique_kmers);
    }
    if (out_path) fclose(f);
    else fflush(f);
  });
}

}  // extern "C"
