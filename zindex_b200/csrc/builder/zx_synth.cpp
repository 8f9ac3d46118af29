// zx_synth: seeded synthetic genomes and query reads for the benchmark
// workloads (no datasets are available offline). Every base is a pure
// function of (seed, genome, position), so reads can be sampled from a genome
// without materialising it.
//
//   zx_synth genomes --kind uniform|pool --colors N --min-len A --max-len B
//                    --seed S --out DIR          (writes DIR/g<i>.fa, DIR/fof.tsv)
//   zx_synth reads   --kind fragment|short|long --colors N --min-len A --max-len B
//                    --seed S --reads R [--length L] [--sourced F] [--subst P]
//                    [--n-runs F] [--format fasta|raw] --out FILE
//
// uniform genomes: genome i = dna(len, seed + i) with dna(n, s)[j] =
//   "ACGT"[splitmix64(j ^ s) & 3] (the reference tests' helper).
// pool genomes: lengths log-uniform in [A, B]; each 100 kbp block is, with
//   probability 0.3, a copy of one of 50 seeded 100 kbp core segments, else
//   i.i.d. uniform bases.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../zx_hash.h"
#include "synth.h"

using zx::splitmix64;
using zx::synth::genome_base;
using zx::synth::genome_length;
using zx::synth::unit;
using Spec = zx::synth::GenomeSpec;

namespace {

const char kAcgt[] = "ACGT";

void write_genomes(const Spec& s, const std::string& dir) {
  std::string fof = dir + "/fof.tsv";
  FILE* f = fopen(fof.c_str(), "w");
  if (!f) {
    perror(fof.c_str());
    exit(1);
  }
  for (uint64_t g = 0; g < s.colors; ++g)
    fprintf(f, "g%llu\t%s/g%llu.fa\n", (unsigned long long)g, dir.c_str(), (unsigned long long)g);
  fclose(f);
  unsigned threads = std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      std::vector<char> buf;
      for (uint64_t g = t; g < s.colors; g += threads) {
        uint64_t n = genome_length(s, g);
        buf.clear();
        char head[64];
        int hn = snprintf(head, sizeof head, ">g%llu\n", (unsigned long long)g);
        buf.insert(buf.end(), head, head + hn);
        for (uint64_t p = 0; p < n; ++p) {
          buf.push_back(genome_base(s, g, p));
          if (p % 80 == 79 || p + 1 == n) buf.push_back('\n');
        }
        std::string path = dir + "/g" + std::to_string(g) + ".fa";
        FILE* o = fopen(path.c_str(), "wb");
        fwrite(buf.data(), 1, buf.size(), o);
        fclose(o);
      }
    });
  for (auto& th : pool) th.join();
}

struct ReadSpec {
  std::string kind = "short";
  uint64_t reads = 1000, length = 150;
  double sourced = 0.7, subst = 0.005, n_runs = 0.0;
  uint64_t seed = 7;
};

// FASTA output, or with raw = true OUT.bases (concatenated sequences) and
// OUT.offsets (reads + 1 little-endian u64 offsets).
void write_reads(const Spec& s, const ReadSpec& r, const std::string& out, bool raw) {
  FILE* f = fopen(raw ? (out + ".bases").c_str() : out.c_str(), "wb");
  FILE* fo = raw ? fopen((out + ".offsets").c_str(), "wb") : nullptr;
  if (!f || (raw && !fo)) {
    perror(out.c_str());
    exit(1);
  }
  uint64_t at = 0;
  if (raw) fwrite(&at, 8, 1, fo);
  std::string seq;
  for (uint64_t i = 0; i < r.reads; ++i) {
    uint64_t h = splitmix64(r.seed ^ splitmix64(0x72656164ull + i));
    uint64_t len = r.length;
    if (r.kind == "long") {
      // Lognormal lengths, median `length`, sigma 1, clipped to 100..100000.
      double u1 = unit(splitmix64(h ^ 1)), u2 = unit(splitmix64(h ^ 2));
      double z = std::sqrt(-2.0 * std::log(u1 > 0 ? u1 : 1e-300)) * std::cos(6.283185307179586 * u2);
      double l = std::exp(std::log((double)r.length) + z);
      len = (uint64_t)std::min(100000.0, std::max(100.0, l));
    }
    seq.clear();
    bool sourced;
    if (r.kind == "fragment") sourced = i == 0;  // record 0 comes from genome 0
    else sourced = unit(splitmix64(h ^ 3)) < r.sourced;
    if (sourced) {
      uint64_t g = r.kind == "fragment" ? 0 : splitmix64(h ^ 4) % s.colors;
      uint64_t glen = genome_length(s, g);
      if (glen < len) len = glen;
      uint64_t off = splitmix64(h ^ 5) % (glen - len + 1);
      for (uint64_t p = 0; p < len; ++p) {
        char b = genome_base(s, g, off + p);
        uint64_t q = splitmix64(h ^ splitmix64(0x737562ull + p));
        if (unit(q) < r.subst) {
          int c = (int)(strchr(kAcgt, b) - kAcgt);
          b = kAcgt[(c + 1 + (int)((q >> 8) % 3)) & 3];
        }
        seq.push_back(b);
      }
    } else {
      for (uint64_t p = 0; p < len; ++p) seq.push_back(kAcgt[splitmix64(h ^ splitmix64(0x726e64ull + p)) & 3]);
    }
    if (r.n_runs > 0 && unit(splitmix64(h ^ 6)) < r.n_runs && seq.size() > 1) {
      uint64_t run = 1 + splitmix64(h ^ 7) % 50;
      uint64_t at = splitmix64(h ^ 8) % seq.size();
      for (uint64_t p = at; p < at + run && p < seq.size(); ++p) seq[p] = 'N';
    }
    if (raw) {
      fwrite(seq.data(), 1, seq.size(), f);
      at += seq.size();
      fwrite(&at, 8, 1, fo);
      continue;
    }
    fprintf(f, ">r%llu\n", (unsigned long long)i);
    fwrite(seq.data(), 1, seq.size(), f);
    fputc('\n', f);
  }
  fclose(f);
  if (fo) fclose(fo);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: zx_synth genomes|reads [options]\n");
    return 2;
  }
  std::string cmd = argv[1], out;
  bool raw = false;
  Spec s;
  ReadSpec r;
  for (int i = 2; i + 1 < argc; i += 2) {
    std::string a = argv[i], v = argv[i + 1];
    if (a == "--kind") {
      if (cmd == "genomes") s.kind = v;
      else r.kind = v;
    } else if (a == "--genome-kind") s.kind = v;
    else if (a == "--colors") s.colors = std::stoull(v);
    else if (a == "--min-len") s.min_len = std::stoull(v);
    else if (a == "--max-len") s.max_len = std::stoull(v);
    else if (a == "--seed") s.seed = std::stoull(v);
    else if (a == "--read-seed") r.seed = std::stoull(v);
    else if (a == "--reads") r.reads = std::stoull(v);
    else if (a == "--length") r.length = std::stoull(v);
    else if (a == "--sourced") r.sourced = std::stod(v);
    else if (a == "--subst") r.subst = std::stod(v);
    else if (a == "--n-runs") r.n_runs = std::stod(v);
    else if (a == "--out") out = v;
    else if (a == "--format") raw = v == "raw";
    else {
      fprintf(stderr, "unknown option %s\n", a.c_str());
      return 2;
    }
  }
  if (out.empty()) {
    fprintf(stderr, "--out is required\n");
    return 2;
  }
  if (cmd == "genomes") write_genomes(s, out);
  else if (cmd == "reads") write_reads(s, r, out, raw);
  else {
    fprintf(stderr, "unknown command %s\n", cmd.c_str());
    return 2;
  }
  return 0;
}
