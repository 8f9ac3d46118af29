// zx_build: command line of the index builder, with the option letters of
// `zorindex build` (src/bin/zorindex.rs:57-150; merge options mod.rs:143-222).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../host/error.h"
#include "builder.h"

static uint64_t parse_size(const std::string& v) {
  struct {
    const char* suffix;
    uint64_t scale;
  } units[] = {{"GiB", 1ull << 30}, {"MiB", 1ull << 20}, {"KiB", 1ull << 10}, {"B", 1}};
  for (auto& u : units) {
    size_t n = strlen(u.suffix);
    if (v.size() > n && v.compare(v.size() - n, n, u.suffix) == 0)
      return std::stoull(v.substr(0, v.size() - n)) * u.scale;
  }
  return std::stoull(v);
}

int main(int argc, char** argv) {
  zx::BuildOptions o;
  std::string mode = "kmers";
  bool have_m = false;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto val = [&]() -> std::string {
      if (i + 1 >= argc) {
        fprintf(stderr, "missing value for %s\n", a.c_str());
        exit(2);
      }
      return argv[++i];
    };
    if (a == "-f" || a == "--fof") o.fof = val();
    else if (a == "-o" || a == "--output") o.output = val();
    else if (a == "-k" || a == "--k") o.features.k = std::stoi(val());
    else if (a == "-m" || a == "--minimizer-size") {
      o.features.m = std::stoi(val());
      have_m = true;
    } else if (a == "-H" || a == "--hashes") o.hashes = std::stoi(val());
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
    else if (a == "--legacy-layout") o.legacy_layout = true;
    else if (a == "-S" || a == "--slot-scale") o.slot_scale = std::stod(val());
    else if (a == "-L" || a == "--segment-length") o.segment_length = std::stoull(val());
    else if (a == "-D" || a == "--min-subindex-documents") o.min_subindex_documents = std::stoull(val());
    else if (a == "-N" || a == "--max-subindexes") o.max_subindexes = std::stoll(val());
    else if (a == "-X" || a == "--max-subindex-size") o.max_subindex_size = parse_size(val());
    else if (a == "-R" || a == "--drop-abandoned") o.drop_abandoned = true;
    else if (a == "-t" || a == "--threads") o.threads = std::stoi(val());
    else if (a == "--groups") o.groups = val();
    else if (a == "--synth") o.synth = val();
    else if (a == "-q" || a == "--quiet") o.quiet = true;
    else if (a == "--device") o.device = true;
    else if (a == "--gpu") o.gpu = std::stoi(val());
    else {
      fprintf(stderr,
              "usage: zx_build -f FOF -o DIR [-k K] [-m M] [-H H] [-b BITS] [-s SEED]\n"
              "  [-i kmers|minimizers|modimizers|findere] [-z Z] [-d D] [-c] [-p PATTERN] [-S SCALE]\n"
              "  [-L SEG] [-D MIN_DOCS] [-N MAX_SUBINDEXES] [-X MAX_SIZE] [-R] [-t THREADS]\n"
              "  [--groups 0,1;2,3] [--device [--gpu N]]\n");
      return 2;
    }
  }
  if (mode == "kmers") o.features.mode = 0;
  else if (mode == "minimizers") o.features.mode = 1;
  else if (mode == "modimizers") o.features.mode = 2;
  else if (mode == "findere") o.features.mode = 3;
  else {
    fprintf(stderr, "unknown index mode %s\n", mode.c_str());
    return 2;
  }
  if (o.features.mode == 1 && !have_m) {
    fprintf(stderr, "minimizer indexes require --minimizer-size\n");
    return 2;
  }
  if ((o.fof.empty() && o.synth.empty()) || o.output.empty()) {
    fprintf(stderr, "zx_build needs -f FOF and -o DIR\n");
    return 2;
  }
  try {
    zx::build_index(o);
  } catch (const std::exception& e) {
    fprintf(stderr, "Error: %s\n", e.what());
    return 1;
  }
  return 0;
}
