// zorindex: command-line drop-in for the reference CLI's query side
// (src/bin/zorindex.rs:161-196 QueryArgs, 426-450 query_command) running on
// the GPU through include/zindex.h, plus `build` (the host-side builder).
//
//   zorindex [-t T] query -i DIR -q FILE [-a MIN_RATIO] [-r [-F tsv|compact] [-B N]]
//                         [-M subindex|all] [--device N]
//   zorindex [-t T] build -f FOF -o DIR [build options, see zx_build]
//
// stdout carries the aggregate TSV of print_aggregate (storage.rs:3817-3844),
// or with -r the per-record report (record_output.rs:13-62); stderr the
// "#query" statistics line (aggregate only) and query_timings.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/zindex.h"
#include "../builder/builder.h"
#include "../host/error.h"

namespace {

int usage() {
  fprintf(stderr,
          "usage: zorindex [-t THREADS] query -i DIR -q FILE [-a MIN_RATIO]\n"
          "                [-r [-F tsv|compact] [-B RECORDS]] [-M subindex|all] [--device N]\n"
          "       zorindex [-t THREADS] build -f FOF -o DIR [-k K] [-m M] [-H H] [-b BITS]\n"
          "                [-s SEED] [-i MODE] [-z Z] [-d D] [-c] [-p PATTERN] [-S SCALE] [-L SEG]\n"
          "                [-D MIN_DOCS]\n"
          "                [-N MAX] [-X SIZE] [-R] [--groups 0,1;2,3]\n");
  return 2;
}

int query(int argc, char** argv, int) {
  std::string dir, path;
  double min_ratio = 0.0;
  int device = 0;
  bool records = false, format_given = false;
  int compact = 0;
  long long batch = 4096;
  for (int i = 0; i < argc; ++i) {
    std::string a = argv[i];
    auto val = [&]() -> const char* {
      if (i + 1 >= argc) {
        fprintf(stderr, "error: %s needs a value\n", a.c_str());
        exit(2);
      }
      return argv[++i];
    };
    if (a == "-i" || a == "--index") dir = val();
    else if (a == "-q" || a == "--query") path = val();
    else if (a == "-a" || a == "--min-ratio") min_ratio = atof(val());
    else if (a == "-M" || a == "--query-memory") {
      std::string v = val();
      if (v != "subindex" && v != "all") return usage();
    } else if (a == "-B" || a == "--record-batch-size") {
      char* end = nullptr;
      const char* v = val();
      batch = strtoll(v, &end, 10);
      if (!*v || *end || batch < 0) return usage();
    } else if (a == "-F" || a == "--output-format") {
      std::string v = val();
      if (v == "tsv") compact = 0;
      else if (v == "compact") compact = 1;
      else return usage();
      format_given = true;
    } else if (a == "--device") device = atoi(val());
    else if (a == "-r" || a == "--records") records = true;
    else return usage();
  }
  if (dir.empty() || path.empty()) return usage();
  if (format_given && !records) {  // clap: output_format requires records
    fprintf(stderr, "error: --output-format requires --records\n");
    return 2;
  }
  if (!(min_ratio >= 0.0 && min_ratio <= 1.0)) {
    fprintf(stderr, "Error: --min-ratio must be in [0, 1]\n");
    return 1;
  }
  auto t0 = std::chrono::steady_clock::now();
  zx_index* ix = nullptr;
  if (zx_open(dir.c_str(), device, 0, &ix) != ZX_OK) {
    fprintf(stderr, "Error: loading %s: %s\n", dir.c_str(), zx_last_error());
    return 1;
  }
  double load_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (records) {
    auto t1 = std::chrono::steady_clock::now();
    int rc = zx_query_records_report(ix, path.c_str(), 1, min_ratio, compact, (uint64_t)batch,
                                     nullptr);
    double query_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
    if (rc != ZX_OK) fprintf(stderr, "Error: %s\n", zx_last_error());
    else fprintf(stderr, "query_timings\tload_s=%.6f\tquery_s=%.6f\n", load_s, query_s);
    zx_close(ix);
    return rc == ZX_OK ? 0 : 1;
  }
  zx_info info;
  zx_index_info(ix, &info);
  std::vector<uint64_t> counts(info.colors);
  uint64_t total = 0, probes = 0;
  auto t1 = std::chrono::steady_clock::now();
  int rc = zx_query_file(ix, path.c_str(), 1, counts.data(), &total, &probes);
  double query_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
  if (rc != ZX_OK) {
    fprintf(stderr, "Error: %s\n", zx_last_error());
    zx_close(ix);
    return 1;
  }
  rc = zx_write_aggregate(ix, path.c_str(), counts.data(), total, probes, min_ratio, query_s,
                          nullptr, 1);
  fprintf(stderr, "query_timings\tload_s=%.6f\tquery_s=%.6f\n", load_s, query_s);
  zx_close(ix);
  return rc == ZX_OK ? 0 : 1;
}

uint64_t parse_size(const std::string& v) {
  struct {
    const char* s;
    uint64_t scale;
  } units[] = {{"GiB", 1ull << 30}, {"MiB", 1ull << 20}, {"KiB", 1ull << 10}, {"B", 1}};
  for (auto& u : units) {
    size_t n = strlen(u.s);
    if (v.size() > n && v.compare(v.size() - n, n, u.s) == 0)
      return std::stoull(v.substr(0, v.size() - n)) * u.scale;
  }
  return std::stoull(v);
}

int build(int argc, char** argv, int threads) {
  zx::BuildOptions o;
  o.threads = threads;
  std::string mode = "kmers";
  for (int i = 0; i < argc; ++i) {
    std::string a = argv[i];
    auto val = [&]() -> std::string {
      if (i + 1 >= argc) {
        fprintf(stderr, "error: %s needs a value\n", a.c_str());
        exit(2);
      }
      return argv[++i];
    };
    if (a == "-f" || a == "--fof") o.fof = val();
    else if (a == "-o" || a == "--output") o.output = val();
    else if (a == "-k" || a == "--k") o.features.k = std::stoi(val());
    else if (a == "-m" || a == "--minimizer-size") o.features.m = std::stoi(val());
    else if (a == "-H" || a == "--hashes") o.hashes = std::stoi(val());
    else if (a == "-b" || a == "--fingerprint-bits") o.fingerprint_bits = std::stoi(val());
    else if (a == "-s" || a == "--seed") o.features.seed = std::stoull(val());
    else if (a == "-i" || a == "--index-mode") mode = val();
    else if (a == "-z" || a == "--findere-z") o.features.z = std::stoi(val());
    else if (a == "-d" || a == "--modimizer-sampling") o.features.sampling = std::stoull(val());
    else if (a == "-c" || a == "--homopolymer-compression") o.features.homopolymer = true;
    else if (a == "-p" || a == "--seed-pattern") o.features.seed_pattern = val();
    else if (a == "-r" || a == "--randstrobemers") o.features.strobes = true;
    else if (a == "-l" || a == "--strobe-min") o.features.strobe_min = std::stoull(val());
    else if (a == "-u" || a == "--strobe-max") o.features.strobe_max = std::stoull(val());
    else if (a == "-S" || a == "--slot-scale") o.slot_scale = std::stod(val());
    else if (a == "-L" || a == "--segment-length") o.segment_length = std::stoull(val());
    else if (a == "-D" || a == "--min-subindex-documents") o.min_subindex_documents = std::stoull(val());
    else if (a == "-N" || a == "--max-subindexes") o.max_subindexes = std::stoll(val());
    else if (a == "-X" || a == "--max-subindex-size") o.max_subindex_size = parse_size(val());
    else if (a == "-R" || a == "--drop-abandoned") o.drop_abandoned = true;
    else if (a == "--groups") o.groups = val();
    else if (a == "--synth") o.synth = val();
    else return usage();
  }
  if (mode == "kmers") o.features.mode = 0;
  else if (mode == "minimizers") o.features.mode = 1;
  else if (mode == "modimizers") o.features.mode = 2;
  else if (mode == "findere") o.features.mode = 3;
  else return usage();
  if ((o.fof.empty() && o.synth.empty()) || o.output.empty()) return usage();
  try {
    zx::build_index(o);
  } catch (const std::exception& e) {
    fprintf(stderr, "Error: %s\n", e.what());
    return 1;
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  int i = 1, threads = 0;
  while (i < argc && argv[i][0] == '-') {
    std::string a = argv[i];
    if ((a == "-t" || a == "--threads") && i + 1 < argc) {
      threads = atoi(argv[i + 1]);
      i += 2;
    } else {
      return usage();
    }
  }
  if (i >= argc) return usage();
  std::string cmd = argv[i];
  if (cmd == "query") return query(argc - i - 1, argv + i + 1, threads);
  if (cmd == "build") return build(argc - i - 1, argv + i + 1, threads);
  return usage();
}
