// TEST INFRASTRUCTURE ONLY — the oracle.
//
// A CPU restatement of the Zindex (`zorindex`, Malfoy/Zindex) query path, used
// (1) by tests/ as the parity checker for the CUDA path and (2) by bench.py's
// cpu_baseline leg and `--impl reference` arm as the timed CPU baseline (the
// reference itself is Rust and cannot be compiled on these machines). The
// product never links, loads or executes this file.
//
// It is written independently of the product sources: its own hashing, FASTA
// parsing, manifest reading, bank decoding, recovery map and lookup. Every
// function cites the reference code it restates.
//
// Parity pins (checked by tests/test_oracle_golden.py): splitmix64 known answers
// (src/lib.rs:1152-1161), the mixsplit relation (1174-1181), encode_full_kmer
// values (966-975), k-mer counts with N and lowercase (986-1001), the k>32
// window formula (821-868), the slow open-closed minimizer reference against
// the rolling scan for all odd k <= 65, m <= 31 (open_closed_minimizers.rs:
// 87-130), packed-screen semantics (packed_fingerprints.rs:128-242) and the
// README's distinct k-mer counts of the bundled bacteria (README.md:60-62);
// spaced-seed validation and projection (anchors.rs:751-773, 841-855) and the
// randstrobemer strobe hash and upstream strobealign iterator witnesses
// (anchors.rs:824-825, 951-986) in tests/test_oracle_golden.py and
// tests/test_strobes_oracle.py; per-record reports by the reference's identity
// (power_merge_cli.rs:1170-1230) and quoting test (record_output.rs:90-112) in
// tests/test_records_oracle.py.
#include "zx_oracle.h"

#include <immintrin.h>
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <functional>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

// --- libzstd public streaming API (zstd.h is not installed; libzstd.so.1 is) ---
extern "C" {
typedef struct ZSTD_DCtx_s ZSTD_DStream;
typedef struct {
  const void* src;
  size_t size;
  size_t pos;
} ZSTD_inBuffer;
typedef struct {
  void* dst;
  size_t size;
  size_t pos;
} ZSTD_outBuffer;
ZSTD_DStream* ZSTD_createDStream(void);
size_t ZSTD_freeDStream(ZSTD_DStream*);
size_t ZSTD_initDStream(ZSTD_DStream*);
size_t ZSTD_decompressStream(ZSTD_DStream*, ZSTD_outBuffer*, ZSTD_inBuffer*);
unsigned ZSTD_isError(size_t);
const char* ZSTD_getErrorName(size_t);
}

namespace {

thread_local std::string g_error;

struct OracleError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

[[noreturn]] void fail(const std::string& msg) { throw OracleError(msg); }
void ensure(bool ok, const char* msg) {
  if (!ok) fail(msg);
}

// ---------------------------------------------------------------- hashing ---
// utils/ocm-minimizers/src/lib.rs:42-53
uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
uint64_t mixsplit(uint64_t key, uint64_t seed) { return splitmix64(key + seed); }

// utils/ocm-minimizers/src/lib.rs:7-15; -1 marks a non-ACGT byte.
int encode_base(uint8_t b) {
  switch (b) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return -1;
  }
}

// utils/ocm-minimizers/src/lib.rs:23-40
uint64_t encode_full(const uint8_t* s, size_t n) {
  uint64_t v = 0;
  for (size_t i = 0; i < n; ++i) v = (v << 2) | (uint64_t)encode_base(s[i]);
  return v;
}
uint64_t canonical_encoded(uint64_t encoded, size_t k) {
  uint64_t v = encoded, rc = 0;
  for (size_t i = 0; i < k; ++i) {
    rc = (rc << 2) | ((v & 3) ^ 3);
    v >>= 2;
  }
  return std::min(encoded, rc);
}

// ------------------------------------------------------------- extraction ---
using Emit = std::vector<uint64_t>;

// src/lib.rs:685-731 (k > 32): rolling polynomial hash of both strands.
void scan_long_kmers(const uint8_t* seq, size_t n, size_t k, Emit& out) {
  const uint64_t B = 0x9e3779b185ebca87ull;
  uint64_t inverse = B;
  for (int i = 0; i < 6; ++i) inverse = inverse * (2ull - B * inverse);
  uint64_t power = 1, base = B;
  for (size_t e = k - 1; e; e >>= 1) {
    if (e & 1) power *= base;
    base *= base;
  }
  const uint64_t domain = splitmix64((uint64_t)k ^ 0x6b6d65722d763031ull);
  uint64_t fwd = 0, rev = 0, weight = 1;
  size_t seen = 0;
  for (size_t p = 0; p < n; ++p) {
    int c = encode_base(seq[p]);
    if (c < 0) {
      fwd = rev = 0;
      weight = 1;
      seen = 0;
      continue;
    }
    uint64_t value = (uint64_t)c + 1, comp = 4 - (uint64_t)c;
    if (seen < k) {
      fwd = fwd * B + value;
      rev = rev + comp * weight;
      weight *= B;
      ++seen;
    } else {
      uint64_t out_code = (uint64_t)encode_base(seq[p - k]);
      fwd = (fwd - (out_code + 1) * power) * B + value;
      rev = (rev - (4 - out_code)) * inverse + comp * power;
    }
    if (seen == k) out.push_back(splitmix64(std::min(fwd, rev) ^ domain));
  }
}

// src/lib.rs:645-681 (k <= 32), dispatching to the long form above 32.
void scan_canonical_kmers(const uint8_t* seq, size_t n, size_t k, Emit& out) {
  if (k == 0 || n < k) return;
  if (k > 32) {
    scan_long_kmers(seq, n, k, out);
    return;
  }
  const uint64_t mask = k == 32 ? ~0ull : ((1ull << (2 * k)) - 1);
  const unsigned shift = (unsigned)(2 * (k - 1));
  uint64_t fwd = 0, rev = 0;
  size_t seen = 0;
  for (size_t p = 0; p < n; ++p) {
    int c = encode_base(seq[p]);
    if (c < 0) {
      fwd = rev = 0;
      seen = 0;
      continue;
    }
    fwd = ((fwd << 2) | (uint64_t)c) & mask;
    rev = (rev >> 2) | ((uint64_t)(c ^ 3) << shift);
    if (++seen >= k) out.push_back(std::min(fwd, rev));
  }
}

struct OcmGeom {
  size_t w, t, s;
};
// utils/ocm-minimizers/src/implementation.rs:89-98
OcmGeom ocm_geom(size_t k, size_t m) {
  OcmGeom g;
  g.w = k - m + 1;
  size_t r = std::min<size_t>(4, m);
  g.t = r + (m - r) % g.w;
  g.s = std::min<size_t>(4, g.t);
  if ((g.t - g.s) & 1) g.s -= 1;
  return g;
}

struct Rank {
  uint8_t cls;
  uint64_t hash;
  bool operator<(const Rank& o) const { return cls != o.cls ? cls < o.cls : hash < o.hash; }
  bool operator==(const Rank& o) const { return cls == o.cls && hash == o.hash; }
};

// One all-ACGT run of length >= k: implementation.rs:141-236. The sliding
// minima follow the queue formulation of scan_run_scalar (implementation.rs
// tests), which the reference asserts equal to the portable ring scan.
void ocm_scan_run(const uint8_t* seq, size_t n, size_t k, size_t m, uint64_t seed,
                  std::vector<std::pair<size_t, uint64_t>>& out) {
  if (k == m) {
    for (size_t p = 0; p + m <= n; ++p)
      out.emplace_back(p, canonical_encoded(encode_full(seq + p, m), m));
    return;
  }
  const OcmGeom g = ocm_geom(k, m);
  const size_t inner_len = g.t - g.s + 1, anchor_len = k - g.t + 1;
  const uint64_t inner_seed = seed ^ 0xC6BC279692B5CC83ull;
  // Inner s-mer hashes and anchor ranks for every position of the run.
  std::vector<uint64_t> inner(n >= g.s ? n - g.s + 1 : 0);
  for (size_t p = 0; p < inner.size(); ++p)
    inner[p] = mixsplit(canonical_encoded(encode_full(seq + p, g.s), g.s), inner_seed);
  const size_t anchors = n - g.t + 1;
  std::vector<Rank> rank(anchors);
  for (size_t p = 0; p < anchors; ++p) {
    uint64_t mn = ~0ull;
    for (size_t j = 0; j < inner_len; ++j) mn = std::min(mn, inner[p + j]);
    uint8_t cls = inner[p + (g.t - g.s) / 2] == mn ? 0
                  : (inner[p] == mn || inner[p + g.t - g.s] == mn) ? 1
                                                                   : 2;
    rank[p] = Rank{cls, mixsplit(canonical_encoded(encode_full(seq + p, g.t), g.t), seed)};
  }
  std::deque<size_t> left, right;  // candidate anchor positions, ranks nondecreasing
  size_t gt = 0;
  bool have_prev = false;
  size_t prev = 0;
  for (size_t end = 0; end < n; ++end) {
    gt += encode_base(seq[end]) >= 2;
    if (end >= k) gt -= encode_base(seq[end - k]) >= 2;
    if (end + 1 < g.t) continue;
    const size_t p = end + 1 - g.t;
    const size_t start = (p + 1 >= anchor_len) ? p + 1 - anchor_len : 0;
    while (!left.empty() && left.front() < start) left.pop_front();
    while (!right.empty() && right.front() < start) right.pop_front();
    while (!left.empty() && rank[p] < rank[left.back()]) left.pop_back();
    while (!right.empty() && !(rank[right.back()] < rank[p])) right.pop_back();
    left.push_back(p);
    right.push_back(p);
    if (end + 1 < k) continue;
    const size_t wstart = end + 1 - k;
    const size_t anchor = gt > k / 2 ? right.front() : left.front();
    const size_t pos = wstart + (anchor - wstart) % g.w;
    if (!have_prev || prev != pos) {
      out.emplace_back(pos, canonical_encoded(encode_full(seq + pos, m), m));
      prev = pos;
      have_prev = true;
    }
  }
}

// implementation.rs:108-128: split at non-ACGT, scan runs of length >= k.
void ocm_scan(const uint8_t* seq, size_t n, size_t k, size_t m, uint64_t seed, Emit& keys) {
  if (k == 0 || (k & 1) == 0 || m == 0 || m > 31 || m > k) return;
  std::vector<std::pair<size_t, uint64_t>> out;
  size_t start = 0;
  while (start < n) {
    size_t end = start;
    while (end < n && encode_base(seq[end]) >= 0) ++end;
    if (end - start >= k) {
      out.clear();
      ocm_scan_run(seq + start, end - start, k, m, seed, out);
      for (auto& e : out) keys.push_back(e.second);
    }
    start = end + 1;
  }
}

// src/lib.rs:211-222
std::vector<uint8_t> homopolymer_compress(const uint8_t* seq, size_t n) {
  std::vector<uint8_t> r;
  r.reserve(n);
  int prev = -2;
  for (size_t i = 0; i < n; ++i) {
    int c = encode_base(seq[i]);
    if (c < 0 || c != prev) r.push_back(c < 0 ? seq[i] : (uint8_t)"ACGT"[c]);
    prev = c < 0 ? -2 : c;
  }
  return r;
}

struct Features {
  int mode = 0;  // 0 kmers, 1 minimizers, 2 modimizers, 3 findere
  size_t k = 31, m = 21;
  uint64_t seed = 69, sampling = 16;
  size_t z = 10;
  bool homopolymer = false;
  int scheme = 1;  // 1 open-closed-mod (0 = simd: not restated, third-party)
  // Spaced seed (src/anchors.rs:10-90): 2 bits per pattern base, '#' = 3;
  // width 0 = none.
  uint64_t pattern_mask = 0;
  size_t pattern_width = 0;
  // Randstrobemers (src/anchors.rs:92-110): strobe-start distance range.
  bool strobes = false;
  size_t strobe_min = 0, strobe_max = 0;
};

// SpacedSeed::from_str (src/anchors.rs:15-42).
bool parse_pattern(const std::string& p, uint64_t* mask, size_t* width) {
  if (p.empty() || p.size() > 31) return false;
  bool any = false;
  uint64_t m = 0;
  for (size_t i = 0; i < p.size(); ++i) {
    if (p[i] != '#' && p[i] != '_') return false;
    if (p[i] != p[p.size() - 1 - i]) return false;
    any |= p[i] == '#';
    m = (m << 2) | (p[i] == '#' ? 3 : 0);
  }
  if (!any) return false;
  *mask = m;
  *width = p.size();
  return true;
}

// SpacedSeed::project_portable and ::canonical (src/anchors.rs:72-90).
uint64_t pattern_project(uint64_t mask, size_t width, uint64_t key) {
  uint64_t r = 0;
  for (size_t i = width; i-- > 0;)
    if (mask & (3ull << (2 * i))) r = (r << 2) | ((key >> (2 * i)) & 3);
  return r;
}
uint64_t pattern_canonical(uint64_t mask, size_t width, uint64_t key) {
  return canonical_encoded(pattern_project(mask, width, key),
                           (size_t)__builtin_popcountll(mask) / 2);
}

// strobe_hash (src/anchors.rs:136-151): XXH64 of one little-endian u64 with
// seed 0 (the published short-input rounds and avalanche).
uint64_t strobe_hash(uint64_t v) {
  auto rotl = [](uint64_t x, int r) { return (x << r) | (x >> (64 - r)); };
  const uint64_t p1 = 0x9E3779B185EBCA87ull, p2 = 0xC2B2AE3D27D4EB4Full,
                 p3 = 0x165667B19E3779F9ull, p4 = 0x85EBCA77C2B2AE63ull,
                 p5 = 0x27D4EB2F165667C5ull;
  uint64_t h = (p5 + 8) ^ (rotl(v * p2, 31) * p1);
  h = rotl(h, 27) * p1 + p4;
  h ^= h >> 33;
  h *= p2;
  h ^= h >> 29;
  h *= p3;
  return h ^ (h >> 32);
}

// Linker (src/anchors.rs:182-256) restated as a direct loop: candidates of
// one run in position order; each anchor emits (anchor.hash / 2) +
// (partner.hash / 2) for the first later candidate at distance in
// [dmin, dmax] with the fewest differing low 8 hash bits (the anchor itself
// when there is none).
void link_strobes(const std::vector<std::pair<size_t, uint64_t>>& cand, size_t dmin, size_t dmax,
                  Emit& keys) {
  for (size_t i = 0; i < cand.size(); ++i) {
    const uint64_t a = cand[i].second;
    uint64_t partner = a;
    int best = 99;
    for (size_t j = i + 1; j < cand.size(); ++j) {
      const size_t d = cand[j].first - cand[i].first;
      if (d > dmax) break;
      if (d < dmin) continue;
      const int rank = __builtin_popcountll((a ^ cand[j].second) & 255);
      if (rank < best) {
        best = rank;
        partner = cand[j].second;
        if (rank == 0) break;
      }
    }
    keys.push_back(a / 2 + partner / 2);
  }
}

// anchors::scan with randstrobemers (src/anchors.rs:265-347) on one ACGT run:
// the candidates are the run's canonical k-mers (position = window start) or
// its selected minimizer positions (sorted, one per position), hashed by
// strobe_hash of the plain key, or of its spaced-seed key under a pattern.
void scan_run_strobes(const uint8_t* seq, size_t n, const Features& f, Emit& keys);

// scan_plain_features_uncompressed (src/lib.rs:608-642) on one ACGT run,
// then the spaced-seed mapping of anchors::scan (src/anchors.rs:265-281).
void scan_run_features(const uint8_t* seq, size_t n, const Features& f, Emit& keys) {
  if (f.strobes && f.mode <= 1) {
    scan_run_strobes(seq, n, f, keys);
    return;
  }
  const size_t first = keys.size();
  switch (f.mode) {
    case 0:
      scan_canonical_kmers(seq, n, f.k, keys);
      break;
    case 1:
      ocm_scan(seq, n, f.k, f.m, f.seed, keys);
      break;
    case 2: {  // src/lib.rs:796-806
      Emit all;
      scan_canonical_kmers(seq, n, f.k, all);
      for (uint64_t key : all)
        if (mixsplit(key, f.seed) % f.sampling == 0) keys.push_back(key);
      break;
    }
    case 3:
      if (n >= f.k) scan_canonical_kmers(seq, n, f.k - f.z, keys);
      break;
  }
  if (f.pattern_width && f.mode <= 1)
    for (size_t i = first; i < keys.size(); ++i)
      keys[i] = pattern_canonical(f.pattern_mask, f.pattern_width, keys[i]);
}

void scan_run_strobes(const uint8_t* seq, size_t n, const Features& f, Emit& keys) {
  std::vector<std::pair<size_t, uint64_t>> cand;
  if (f.mode == 1) {
    if (n >= f.k && (f.k & 1) && f.m >= 1 && f.m <= 31 && f.m <= f.k)
      ocm_scan_run(seq, n, f.k, f.m, f.seed, cand);
    std::sort(cand.begin(), cand.end(),
              [](const auto& a, const auto& b) { return a.first < b.first; });
    cand.erase(std::unique(cand.begin(), cand.end(),
                           [](const auto& a, const auto& b) { return a.first == b.first; }),
               cand.end());
  } else {
    Emit plain;
    scan_canonical_kmers(seq, n, f.k, plain);
    for (size_t i = 0; i < plain.size(); ++i) cand.emplace_back(i, plain[i]);
  }
  for (auto& c : cand) {
    if (f.pattern_width) c.second = pattern_canonical(f.pattern_mask, f.pattern_width, c.second);
    c.second = strobe_hash(c.second);
  }
  link_strobes(cand, f.strobe_min, f.strobe_max, keys);
}

// Calls visit(run, len) for every maximal ACGT run of a sequence, after the
// optional homopolymer compression of the run (the parser delivers ACGT runs,
// src/lib.rs:27-33, and scan_index_features compresses each, 574-589).
template <class V>
void for_each_run(const uint8_t* seq, size_t n, bool homopolymer, V&& visit) {
  size_t start = 0;
  while (start < n) {
    size_t end = start;
    while (end < n && encode_base(seq[end]) >= 0) ++end;
    if (end > start) {
      if (homopolymer) {
        auto c = homopolymer_compress(seq + start, end - start);
        visit(c.data(), c.size());
      } else {
        visit(seq + start, end - start);
      }
    }
    start = end + 1;
  }
}

// ---------------------------------------------------------------- input ---
std::vector<uint8_t> read_file(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) fail("cannot open " + path + ": " + strerror(errno));
  std::vector<uint8_t> data;
  uint8_t buf[1 << 16];
  size_t got;
  while ((got = fread(buf, 1, sizeof buf, f)) > 0) data.insert(data.end(), buf, buf + got);
  fclose(f);
  return data;
}

std::vector<uint8_t> zstd_decode(const std::vector<uint8_t>& in) {
  std::vector<uint8_t> out;
  ZSTD_DStream* ds = ZSTD_createDStream();
  ZSTD_initDStream(ds);
  ZSTD_inBuffer ib{in.data(), in.size(), 0};
  std::vector<uint8_t> chunk(1 << 20);
  size_t last = 0;
  for (;;) {
    ZSTD_outBuffer ob{chunk.data(), chunk.size(), 0};
    last = ZSTD_decompressStream(ds, &ob, &ib);
    if (ZSTD_isError(last)) {
      std::string msg = ZSTD_getErrorName(last);
      ZSTD_freeDStream(ds);
      fail("zstd: " + msg);
    }
    out.insert(out.end(), chunk.data(), chunk.data() + ob.pos);
    // Done once all input is consumed and the output was not filled up.
    if (ib.pos == ib.size && ob.pos < ob.size) break;
  }
  ZSTD_freeDStream(ds);
  ensure(last == 0, "zstd: truncated stream");
  return out;
}

// Decoded bytes of a possibly compressed input (gzip by zlib, zstd by libzstd).
std::vector<uint8_t> read_decoded(const std::string& path) {
  std::vector<uint8_t> raw = read_file(path);
  if (raw.size() >= 4 && raw[0] == 0x28 && raw[1] == 0xb5 && raw[2] == 0x2f && raw[3] == 0xfd)
    return zstd_decode(raw);
  if (raw.size() >= 2 && raw[0] == 0x1f && raw[1] == 0x8b) {
    gzFile g = gzopen(path.c_str(), "rb");
    if (!g) fail("cannot open " + path);
    std::vector<uint8_t> out;
    uint8_t buf[1 << 16];
    int got;
    while ((got = gzread(g, buf, sizeof buf)) > 0) out.insert(out.end(), buf, buf + got);
    int err = 0;
    gzerror(g, &err);
    gzclose(g);
    if (got < 0 || (err != Z_OK && err != Z_STREAM_END)) fail("corrupt gzip stream " + path);
    return out;
  }
  return raw;
}

// FASTA/FASTQ records as in helicase with ignore_headers/dna_string: FASTA
// sequence lines are joined, line ends (LF or CRLF) removed; FASTQ is
// 4-line records whose quality must match the sequence length.
void parse_fastx(const std::vector<uint8_t>& d, std::vector<std::vector<uint8_t>>& records) {
  size_t i = 0, n = d.size();
  auto line_end = [&](size_t from) {
    size_t e = from;
    while (e < n && d[e] != '\n') ++e;
    return e;
  };
  auto trimmed = [&](size_t a, size_t e) { return (e > a && d[e - 1] == '\r') ? e - 1 : e; };
  while (i < n && (d[i] == '\n' || d[i] == '\r')) ++i;
  if (i == n) return;
  if (d[i] == '>') {
    while (i < n) {
      ensure(d[i] == '>', "malformed FASTA record");
      size_t e = line_end(i);
      i = e < n ? e + 1 : n;
      std::vector<uint8_t> seq;
      while (i < n && d[i] != '>') {
        size_t le = line_end(i);
        size_t te = trimmed(i, le);
        seq.insert(seq.end(), d.begin() + i, d.begin() + te);
        i = le < n ? le + 1 : n;
      }
      records.push_back(std::move(seq));
    }
  } else if (d[i] == '@') {
    while (i < n) {
      if (d[i] == '\n' || d[i] == '\r') {
        ++i;
        continue;
      }
      ensure(d[i] == '@', "malformed FASTQ record");
      size_t e = line_end(i);
      ensure(e < n, "truncated FASTQ header");
      i = e + 1;
      size_t se = line_end(i);
      size_t ste = trimmed(i, se);
      std::vector<uint8_t> seq(d.begin() + i, d.begin() + ste);
      ensure(se < n, "truncated FASTQ record");
      i = se + 1;
      ensure(i < n && d[i] == '+', "malformed FASTQ separator");
      size_t pe = line_end(i);
      ensure(pe < n, "truncated FASTQ record");
      i = pe + 1;
      size_t qe = line_end(i);
      size_t qte = trimmed(i, qe);
      ensure(qte - i == seq.size(), "truncated FASTQ quality");
      i = qe < n ? qe + 1 : n;
      records.push_back(std::move(seq));
    }
  } else {
    fail("input is neither FASTA nor FASTQ");
  }
}

// ------------------------------------------------------------------ json ---
struct Json {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  bool b = false;
  bool is_int = false;
  uint64_t u = 0;
  bool neg = false;
  double d = 0;
  std::string s;
  std::vector<Json> a;
  std::vector<std::pair<std::string, Json>> o;
  const Json* get(const char* key) const {
    for (auto& kv : o)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
  uint64_t as_u64() const {
    ensure(kind == Num && is_int && !neg, "expected an unsigned integer in manifest");
    return u;
  }
  double as_f64() const {
    ensure(kind == Num, "expected a number in manifest");
    return d;
  }
};

struct JsonParser {
  const char* p;
  const char* e;
  void ws() {
    while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
  }
  Json parse() {
    ws();
    ensure(p < e, "unexpected end of manifest");
    Json v;
    if (*p == '{') {
      v.kind = Json::Obj;
      ++p;
      ws();
      if (*p == '}') {
        ++p;
        return v;
      }
      for (;;) {
        ws();
        Json key = parse();
        ensure(key.kind == Json::Str, "manifest object key");
        ws();
        ensure(p < e && *p == ':', "manifest ':'");
        ++p;
        v.o.emplace_back(key.s, parse());
        ws();
        ensure(p < e, "manifest object");
        if (*p == ',') {
          ++p;
          continue;
        }
        ensure(*p == '}', "manifest '}'");
        ++p;
        return v;
      }
    }
    if (*p == '[') {
      v.kind = Json::Arr;
      ++p;
      ws();
      if (*p == ']') {
        ++p;
        return v;
      }
      for (;;) {
        v.a.push_back(parse());
        ws();
        ensure(p < e, "manifest array");
        if (*p == ',') {
          ++p;
          continue;
        }
        ensure(*p == ']', "manifest ']'");
        ++p;
        return v;
      }
    }
    if (*p == '"') {
      v.kind = Json::Str;
      ++p;
      while (p < e && *p != '"') {
        if (*p == '\\') {
          ++p;
          ensure(p < e, "manifest string escape");
          char c = *p++;
          switch (c) {
            case 'n': v.s += '\n'; break;
            case 't': v.s += '\t'; break;
            case 'r': v.s += '\r'; break;
            case 'b': v.s += '\b'; break;
            case 'f': v.s += '\f'; break;
            case 'u': {
              ensure(e - p >= 4, "manifest \\u escape");
              unsigned cp = (unsigned)strtoul(std::string(p, 4).c_str(), nullptr, 16);
              p += 4;
              if (cp >= 0xD800 && cp < 0xDC00 && e - p >= 6 && p[0] == '\\' && p[1] == 'u') {
                unsigned lo = (unsigned)strtoul(std::string(p + 2, 4).c_str(), nullptr, 16);
                p += 6;
                cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
              }
              if (cp < 0x80) v.s += (char)cp;
              else if (cp < 0x800) {
                v.s += (char)(0xC0 | (cp >> 6));
                v.s += (char)(0x80 | (cp & 0x3F));
              } else if (cp < 0x10000) {
                v.s += (char)(0xE0 | (cp >> 12));
                v.s += (char)(0x80 | ((cp >> 6) & 0x3F));
                v.s += (char)(0x80 | (cp & 0x3F));
              } else {
                v.s += (char)(0xF0 | (cp >> 18));
                v.s += (char)(0x80 | ((cp >> 12) & 0x3F));
                v.s += (char)(0x80 | ((cp >> 6) & 0x3F));
                v.s += (char)(0x80 | (cp & 0x3F));
              }
              break;
            }
            default: v.s += c;
          }
        } else {
          v.s += *p++;
        }
      }
      ensure(p < e, "unterminated manifest string");
      ++p;
      return v;
    }
    if (e - p >= 4 && !strncmp(p, "true", 4)) {
      v.kind = Json::Bool;
      v.b = true;
      p += 4;
      return v;
    }
    if (e - p >= 5 && !strncmp(p, "false", 5)) {
      v.kind = Json::Bool;
      p += 5;
      return v;
    }
    if (e - p >= 4 && !strncmp(p, "null", 4)) {
      p += 4;
      return v;
    }
    v.kind = Json::Num;
    const char* s = p;
    if (*p == '-') {
      v.neg = true;
      ++p;
    }
    bool integral = true;
    while (p < e && ((*p >= '0' && *p <= '9') || *p == '.' || *p == 'e' || *p == 'E' ||
                     *p == '+' || *p == '-')) {
      if (*p == '.' || *p == 'e' || *p == 'E') integral = false;
      ++p;
    }
    std::string text(s, p);
    ensure(!text.empty(), "manifest value");
    v.d = strtod(text.c_str(), nullptr);
    if (integral) {
      v.is_int = true;
      v.u = strtoull(text.c_str() + (v.neg ? 1 : 0), nullptr, 10);
    }
    return v;
  }
};

// ----------------------------------------------------------------- index ---
struct Group {
  std::vector<uint32_t> members;
  size_t width = 0, offset = 0;
};
struct Bank {
  size_t slots = 0, row_bits = 0, source_slots = 0, component = 0;
  size_t partition = 0, partitions = 1;
  bool fp_first = false;
  std::string file;
  std::vector<Group> groups;
  std::vector<uint8_t> data;
  size_t row_bytes() const { return (row_bits + 7) / 8; }
};
struct Color {
  std::string name;
  uint64_t unique = 0;
};

// OriginMap (src/power_merge/abandoned.rs:28-225): open addressing over
// 32-bit hashes, first slot from the high bits, linear probing.
struct OriginMap {
  struct Entry {
    uint32_t hash;
    uint32_t value;
  };
  static constexpr uint32_t kEmpty = 0xFFFFFFFFu, kMultiple = 1u << 31;
  std::vector<Entry> dir;
  std::vector<std::pair<size_t, size_t>> ranges;
  std::vector<uint32_t> origins;
  unsigned bits = 0;
  size_t first_slot(uint32_t key) const {
    return bits <= 32 ? (size_t)(key >> (32 - bits)) : ((size_t)key << (bits - 32));
  }
  void build(const std::vector<std::pair<uint32_t, std::vector<uint32_t>>>& recs) {
    size_t n = recs.size();
    if (n == 0) return;
    size_t cap = std::max<size_t>((n * 4 + 2) / 3, 4);
    size_t c = 1;
    while (c < cap) c <<= 1;
    dir.assign(c, Entry{0, kEmpty});
    bits = (unsigned)__builtin_ctzll(c);
    for (auto& r : recs) {
      uint32_t value;
      if (r.second.size() == 1 && r.second[0] < kMultiple) {
        value = r.second[0];
      } else {
        value = kMultiple | (uint32_t)ranges.size();
        ranges.emplace_back(origins.size(), r.second.size());
        origins.insert(origins.end(), r.second.begin(), r.second.end());
      }
      size_t slot = first_slot(r.first);
      while (dir[slot].value != kEmpty) slot = (slot + 1) & (c - 1);
      dir[slot] = Entry{r.first, value};
    }
  }
  // Returns the origins of `key` as [ptr, ptr+len).
  const uint32_t* get(uint32_t key, size_t* len) const {
    *len = 0;
    if (dir.empty()) return nullptr;
    size_t mask = dir.size() - 1, slot = first_slot(key);
    for (;;) {
      const Entry& e = dir[slot];
      if (e.value == kEmpty) return nullptr;
      if (e.hash == key) {
        if (!(e.value & kMultiple)) {
          *len = 1;
          return &e.value;
        }
        auto& r = ranges[e.value & ~kMultiple];
        *len = r.second;
        return origins.data() + r.first;
      }
      slot = (slot + 1) & mask;
    }
  }
};

struct Index {
  uint32_t version = 0;
  size_t k = 0, hashes = 0, bits = 0, m = 0;
  bool has_segment = false;
  size_t segment = 0;
  uint64_t seed = 0;
  Features f;
  bool recovery = false;
  std::vector<Color> colors;
  std::vector<Bank> banks;
  std::vector<std::vector<size_t>> classes;  // bank ids per source class, partition order
  OriginMap recover;
};

uint64_t get_bits(const uint8_t* row, size_t offset, size_t width) {
  // src/power_merge/storage.rs:3523-3538 (little-endian bit order).
  uint64_t v = 0;
  for (size_t i = 0; i < width; ++i) {
    size_t bit = offset + i;
    v |= (uint64_t)((row[bit >> 3] >> (bit & 7)) & 1) << i;
  }
  return v;
}

uint64_t read_u64le(const uint8_t* p) {
  uint64_t v = 0;
  for (int i = 7; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}

// Bank file: magic, u64 LE slots/row_bits/groups/payload, payload
// (validate_bank_header, storage.rs:2208-2231; zstd frames, bank_io.rs).
void load_bank(const std::string& dir, Bank& b) {
  std::vector<uint8_t> raw = read_file(dir + "/" + b.file);
  std::vector<uint8_t> dec =
      (raw.size() >= 4 && raw[0] == 0x28 && raw[1] == 0xb5) ? zstd_decode(raw) : raw;
  size_t expected = b.slots * b.row_bytes();
  ensure(dec.size() >= 40, "short bank file");
  ensure(!memcmp(dec.data(), b.fp_first ? "ZORPOW3\0" : "ZORPOW1\0", 8), "invalid bank magic");
  ensure(read_u64le(&dec[8]) == b.slots && read_u64le(&dec[16]) == b.row_bits &&
             read_u64le(&dec[24]) == b.groups.size() && read_u64le(&dec[32]) == expected,
         "bank header differs from manifest");
  ensure(dec.size() == 40 + expected, "unexpected bank data");
  b.data.assign(dec.begin() + 40, dec.end());
}

// abandoned_io.rs:4-130 (ZORABN2 varint deltas, or ZORABN1 u32 LE).
void load_recovery(const std::string& dir, Index& ix, size_t hashes, size_t assoc) {
  std::vector<uint8_t> raw = read_file(dir + "/abandoned.zormap.zst");
  std::vector<uint8_t> d =
      (raw.size() >= 4 && raw[0] == 0x28 && raw[1] == 0xb5) ? zstd_decode(raw) : raw;
  ensure(d.size() >= 8, "invalid abandoned map magic");
  bool delta = !memcmp(d.data(), "ZORABN2\0", 8);
  ensure(delta || !memcmp(d.data(), "ZORABN1\0", 8), "invalid abandoned map magic");
  size_t p = 8;
  auto var = [&]() -> uint32_t {
    uint32_t v = 0;
    for (int shift = 0; shift <= 28; shift += 7) {
      ensure(p < d.size(), "truncated abandoned map");
      uint8_t byte = d[p++];
      ensure(shift != 28 || byte <= 15, "abandoned variable integer overflow");
      v |= (uint32_t)(byte & 127) << shift;
      if (!(byte & 128)) return v;
    }
    fail("abandoned variable integer overflow");
  };
  auto u32 = [&]() -> uint32_t {
    ensure(p + 4 <= d.size(), "truncated abandoned map");
    uint32_t v = (uint32_t)d[p] | ((uint32_t)d[p + 1] << 8) | ((uint32_t)d[p + 2] << 16) |
                 ((uint32_t)d[p + 3] << 24);
    p += 4;
    return v;
  };
  std::vector<std::pair<uint32_t, std::vector<uint32_t>>> recs;
  recs.reserve(hashes);
  uint32_t prev = 0;
  size_t total = 0;
  for (size_t r = 0; r < hashes; ++r) {
    uint32_t h = delta ? prev + var() : u32();
    ensure(r == 0 || h > prev, "unsorted/duplicate abandoned hashes");
    prev = h;
    uint32_t count = delta ? var() : u32();
    ensure(count > 0 && count <= ix.colors.size(), "invalid abandoned origin count");
    std::vector<uint32_t> origins(count);
    uint32_t po = 0;
    for (uint32_t c = 0; c < count; ++c) {
      uint32_t o = delta ? po + var() : u32();
      ensure(o < ix.colors.size(), "invalid abandoned dataset ID");
      ensure(c == 0 || o > po, "unsorted/duplicate abandoned origins");
      origins[c] = po = o;
    }
    total += count;
    recs.emplace_back(h, std::move(origins));
  }
  ensure(total == assoc, "abandoned origin count differs from manifest");
  ensure(p == d.size(), "unexpected abandoned map data");
  ix.recover.build(recs);
}

std::unique_ptr<Index> load_index(const std::string& dir, bool recover, bool payload = true) {
  auto ix = std::make_unique<Index>();
  std::vector<uint8_t> text = read_file(dir + "/manifest.json");
  JsonParser jp{(const char*)text.data(), (const char*)text.data() + text.size()};
  Json m = jp.parse();
  ensure(m.kind == Json::Obj, "manifest is not an object");
  auto req = [&](const char* key) -> const Json& {
    const Json* v = m.get(key);
    if (!v) fail(std::string("manifest lacks ") + key);
    return *v;
  };
  ix->version = (uint32_t)req("version").as_u64();
  ensure(ix->version >= 2 && ix->version <= 10, "unsupported power-of-two index format");
  ix->k = req("k").as_u64();
  ix->hashes = req("hashes").as_u64();
  ix->seed = req("seed").as_u64();
  ix->bits = req("fingerprint_bits").as_u64();
  ensure(ix->hashes >= 2 && ix->hashes <= 32, "invalid hash count");
  const Json* seg = m.get("segment_length");
  if (seg && seg->kind != Json::Null) {
    ix->has_segment = true;
    ix->segment = seg->as_u64();
  }
  ix->f.mode = (int)req("index_mode").as_u64();
  ix->f.k = ix->k;
  ix->f.m = req("minimizer_size").as_u64();
  ix->f.seed = ix->seed;
  ix->f.sampling = req("modimizer_sampling").as_u64();
  ix->f.z = req("findere_z").as_u64();
  const Json* hp = m.get("homopolymer_compression");
  ix->f.homopolymer = hp && hp->kind == Json::Bool && hp->b;
  const Json* sch = m.get("minimizer_scheme");
  ix->f.scheme = (sch && sch->kind == Json::Str && sch->s == "open-closed-mod") ? 1 : 0;
  ensure(!(ix->f.mode == 1 && ix->f.scheme == 0), "simd minimizer scheme is not restated");
  const Json* sp = m.get("seed_pattern");
  if (sp && sp->kind != Json::Null) {
    // FeatureConfig::validate_anchors (src/lib.rs:177-206).
    ensure(sp->kind == Json::Str && parse_pattern(sp->s, &ix->f.pattern_mask, &ix->f.pattern_width),
           "invalid seed pattern");
    ensure(ix->f.mode == 0 || ix->f.mode == 1,
           "spaced seeds and randstrobemers require --index-mode kmers or minimizers");
    ensure(ix->f.pattern_width == (ix->f.mode == 1 ? ix->f.m : ix->f.k),
           "seed pattern width must match k (or m in minimizer mode)");
  }
  const Json* rs = m.get("randstrobemers");
  if (rs && rs->kind != Json::Null) {
    // Manifest::features (storage.rs:240-256), RandstrobeConfig::validate
    // (anchors.rs:98-110), FeatureConfig::validate_anchors (lib.rs:177-206).
    const Json* scheme = m.get("randstrobe_scheme");
    ensure(ix->version >= 6 && scheme && scheme->kind == Json::Str &&
               scheme->s == "strobealign-popcount8-symmetric64-downstream-v1",
           "unsupported legacy/custom randstrobemer extraction; rebuild this index with the "
           "current downstream scheme");
    ensure(ix->f.mode == 0 || ix->f.mode == 1,
           "spaced seeds and randstrobemers require --index-mode kmers or minimizers");
    const Json* lo = rs->get("min_distance");
    const Json* hi = rs->get("max_distance");
    ensure(lo && hi, "manifest: randstrobemers");
    ix->f.strobes = true;
    ix->f.strobe_min = lo->as_u64();
    ix->f.strobe_max = hi->as_u64();
    ensure(ix->f.strobe_min > 0, "randstrobemer minimum distance must be greater than zero");
    ensure(ix->f.strobe_min <= ix->f.strobe_max,
           "randstrobemer minimum distance must not exceed maximum distance");
  }
  const Json* ar = m.get("abandoned_recovery");
  bool recovery = !ar || (ar->kind == Json::Bool && ar->b);
  ix->recovery = recover && recovery;
  for (auto& c : req("colors").a) {
    Color col;
    col.name = c.get("name")->s;
    col.unique = c.get("unique_kmers")->as_u64();
    ix->colors.push_back(col);
  }
  for (auto& bj : req("banks").a) {
    Bank b;
    b.file = bj.get("file")->s;
    b.slots = bj.get("slots")->as_u64();
    b.row_bits = bj.get("row_bits")->as_u64();
    const Json* ff = bj.get("fingerprint_first");
    b.fp_first = ff && ff->kind == Json::Bool && ff->b;
    const Json* comp = bj.get("component");
    b.component = comp ? comp->as_u64() : 0;
    b.source_slots = b.slots;
    const Json* rt = bj.get("routing");
    if (rt && rt->kind == Json::Obj) {
      b.source_slots = rt->get("source_slots")->as_u64();
      b.partition = rt->get("partition")->as_u64();
      b.partitions = rt->get("partitions")->as_u64();
    }
    for (auto& gj : bj.get("groups")->a) {
      Group g;
      for (auto& mm : gj.get("members")->a) g.members.push_back((uint32_t)mm.as_u64());
      g.width = gj.get("width")->as_u64();
      g.offset = gj.get("offset")->as_u64();
      b.groups.push_back(std::move(g));
    }
    ix->banks.push_back(std::move(b));
  }
  // Source classes: consecutive banks sharing (component, source_slots).
  for (size_t i = 0; i < ix->banks.size();) {
    size_t j = i + 1;
    while (j < ix->banks.size() && ix->banks[j].component == ix->banks[i].component &&
           ix->banks[j].source_slots == ix->banks[i].source_slots)
      ++j;
    std::vector<size_t> cls;
    for (size_t q = i; q < j; ++q) {
      ensure(ix->banks[q].partition == q - i && ix->banks[q].partitions == j - i,
             "invalid/duplicate/missing hash partition");
      cls.push_back(q);
    }
    ix->classes.push_back(cls);
    i = j;
  }
  if (payload) {
    for (auto& b : ix->banks) load_bank(dir, b);
    if (ix->recovery) {
      size_t hashes = req("abandoned_hashes").as_u64();
      size_t assoc = req("abandoned_origins").as_u64();
      if (hashes) load_recovery(dir, *ix, hashes, assoc);
    }
  }
  return ix;
}

// PositionHash::positions (storage.rs:3452-3481): the H cells of a key in a
// bank of `cells` slots; segment 0 = the legacy length, the power-of-two
// floor of clamp(cells / H, 1, 4096).
void positions(uint64_t key, uint64_t seed, uint64_t cells, size_t hashes, uint64_t segment,
               uint64_t* out) {
  uint64_t len = segment;
  if (!len) {
    uint64_t n = std::min<uint64_t>(std::max<uint64_t>(cells / hashes, 1), 4096);
    len = 1;
    while (len * 2 <= n) len *= 2;
  }
  const uint64_t first = mixsplit(key, seed), step = splitmix64(first);
  const uint64_t count = cells / len - hashes + 1;
  const uint64_t base = (uint64_t)(((unsigned __int128)first * count) >> 64) * len;
  uint64_t h = first;
  for (size_t i = 0; i < hashes; ++i) {
    out[i] = base + i * len + ((h ^ (h >> 33)) & (len - 1));
    h += step;
  }
}

// abandoned::hash (abandoned.rs:5-10).
uint32_t abandoned_hash(uint64_t key, uint64_t seed) {
  return (uint32_t)(splitmix64(key ^ seed ^ 0xD6E8FEB86659FD93ull) >> 32);
}

// lookup_selected (storage.rs:2761-2925) for one key: every colour hit by a
// filter or by the recovery map, each at most once, appended to `hits`.
void lookup(const Index& ix, uint64_t key, std::vector<uint32_t>& hits) {
  hits.clear();
  size_t rlen = 0;
  const uint32_t* rec = ix.recovery ? ix.recover.get(abandoned_hash(key, ix.seed), &rlen) : nullptr;
  const uint64_t fp = splitmix64(key ^ ix.seed ^ 0x8E2D4F6A9B13C5D7ull) & ((1ull << ix.bits) - 1);
  uint64_t slots[32];
  std::vector<uint8_t> row;
  for (auto& cls : ix.classes) {
    const Bank* bp = &ix.banks[cls[0]];
    if (cls.size() > 1)
      bp = &ix.banks[cls[splitmix64(key ^ ix.seed ^ 0x34B61D8F29A7C053ull) & (cls.size() - 1)]];
    const Bank& b = *bp;
    positions(key, ix.seed, b.slots, ix.hashes, ix.has_segment ? ix.segment : 0, slots);
    const size_t rb = b.row_bytes(), G = b.groups.size(), bits = ix.bits;
    auto hit = [&](uint32_t c) { hits.push_back(c); };
    if (b.fp_first) {
      size_t lookup_bytes = (G * bits + 7) / 8;
      row.assign(lookup_bytes, 0);
      for (size_t i = 0; i < ix.hashes; ++i) {
        const uint8_t* r = b.data.data() + slots[i] * rb;
        for (size_t j = 0; j < lookup_bytes; ++j) row[j] ^= r[j];
      }
      for (size_t g = 0; g < G; ++g) {
        if (get_bits(row.data(), g * bits, bits) != fp) continue;
        const Group& gr = b.groups[g];
        if (gr.members.size() == 1) {
          hit(gr.members[0]);
          continue;
        }
        size_t off = G * bits + gr.offset - g * bits;
        uint64_t mask = 0;
        for (size_t i = 0; i < ix.hashes; ++i)
          mask ^= get_bits(b.data.data() + slots[i] * rb, off, gr.width - bits);
        while (mask) {
          hit(gr.members[__builtin_ctzll(mask)]);
          mask &= mask - 1;
        }
      }
    } else {
      row.assign(rb, 0);
      for (size_t i = 0; i < ix.hashes; ++i) {
        const uint8_t* r = b.data.data() + slots[i] * rb;
        for (size_t j = 0; j < rb; ++j) row[j] ^= r[j];
      }
      for (auto& gr : b.groups) {
        uint64_t v = get_bits(row.data(), gr.offset, gr.width);
        if ((v & ((1ull << bits) - 1)) != fp) continue;
        if (gr.members.size() == 1) {
          hit(gr.members[0]);
          continue;
        }
        uint64_t mask = v >> bits;
        while (mask) {
          hit(gr.members[__builtin_ctzll(mask)]);
          mask &= mask - 1;
        }
      }
    }
  }
  // Recovery union: an origin counts once whether or not a filter also hit it.
  for (size_t i = 0; i < rlen; ++i) {
    uint32_t o = rec[i];
    if (std::find(hits.begin(), hits.end(), o) == hits.end()) hits.push_back(o);
  }
}

struct Work {
  // Ordinary modes: keys of all records. Findere: s-mer keys per task.
  std::vector<uint64_t> keys;
  std::vector<std::pair<size_t, size_t>> tasks;  // findere task key ranges
  uint64_t total = 0, probes = 0;
};

// Seeds of one record (a sequence that may hold non-ACGT bytes).
void prepare_record(const Features& f, const uint8_t* seq, size_t n, Work& w) {
  for_each_run(seq, n, f.homopolymer, [&](const uint8_t* run, size_t len) {
    if (f.mode != 3) {
      size_t before = w.keys.size();
      scan_run_features(run, len, f, w.keys);
      w.total += w.keys.size() - before;
      w.probes += w.keys.size() - before;
      return;
    }
    // Findere (findere.rs:178-233, query_stream.rs:488-515): tasks of
    // 16,384 k-windows carrying k-1 bases of context.
    if (len < f.k) return;
    size_t windows = len - f.k + 1;
    w.total += windows;
    for (size_t start = 0; start < windows; start += 16384) {
      size_t owned = std::min<size_t>(16384, windows - start);
      size_t first = w.keys.size();
      scan_canonical_kmers(run + start, owned + f.k - 1, f.k - f.z, w.keys);
      w.tasks.emplace_back(first, w.keys.size());
      w.probes += w.keys.size() - first;
    }
  });
}

// ------------------------------------------------- fast CPU baseline path ---
// The reference's own speed measures for the aggregate lookup, restated for
// the timed CPU baseline (the scalar lookup above stays the checker):
// lookup_batch (storage.rs:2929-2978) takes blocks of 32 weighted keys,
// computes every selected bank's H positions for the whole block, and
// prefetches the rows of key i + 4 (prefetch_lookup, 3014-3054: every 64
// bytes of the fingerprint plane, and the recovery bucket) while key i is
// looked up; fingerprint_matches_rows (3241-3350) screens 8/16/32-bit fields
// with AVX2 XOR + compare + movemask, packed_fingerprints::matches_rows
// (7-126) screens 2/4-bit fields by XOR, fold and and-not over 256 bits, and
// 1-bit fields are read 64 at a time. Counts follow WeightedScores
// (3083-3101): a hit adds the key's weight; recovered origins' counters are
// read before the filter hits and raised afterwards only if unchanged
// (lookup_selected, 2778-2787, 2916-2924).
namespace fastpath {

template <class Hit>
void screen_bytes_scalar(const uint8_t* const* rows, size_t H, size_t bits, uint64_t fp,
                         size_t byte0, size_t len, Hit& hit) {
  const size_t width = bits / 8;
  for (size_t byte = byte0; byte + width <= len; byte += width) {
    uint64_t v = 0;
    for (size_t i = 0; i < H; ++i) {
      uint64_t x = 0;
      memcpy(&x, rows[i] + byte, width);
      v ^= x;
    }
    if (v == fp) hit(byte / width);
  }
}

template <size_t B, class Hit>
void screen_packed_scalar(const uint8_t* const* rows, size_t H, uint64_t fp, size_t count,
                          size_t base, Hit& hit) {
  const uint64_t ones = ~0ull / ((1ull << B) - 1), target = ones * fp;
  auto fold = [&](uint64_t diff) {
    uint64_t f = diff | (diff >> 1);
    if (B == 4) f |= f >> 2;
    return ~f & ones;
  };
  auto emit = [&](uint64_t m, size_t at) {
    for (; m; m &= m - 1) hit(at + (size_t)__builtin_ctzll(m) / B);
  };
  while (count - base >= 64 / B) {
    uint64_t v = 0;
    for (size_t i = 0; i < H; ++i) {
      uint64_t x;
      memcpy(&x, rows[i] + base * B / 8, 8);
      v ^= x;
    }
    emit(fold(v ^ target), base);
    base += 64 / B;
  }
  if (base != count) {
    const size_t bytes = ((count - base) * B + 7) / 8;
    uint64_t v = 0;
    for (size_t i = 0; i < H; ++i) {
      uint64_t x = 0;
      memcpy(&x, rows[i] + base * B / 8, bytes);
      v ^= x;
    }
    emit(fold(v ^ target) & (~0ull >> (64 - (count - base) * B)), base);
  }
}

template <class Hit>
__attribute__((target("avx2"))) void screen_bytes_avx2(const uint8_t* const* rows, size_t H,
                                                       size_t bits, uint64_t fp, size_t len,
                                                       Hit& hit) {
  const __m256i target = bits == 8    ? _mm256_set1_epi8((char)fp)
                         : bits == 16 ? _mm256_set1_epi16((short)fp)
                                      : _mm256_set1_epi32((int)fp);
  const uint32_t keep = bits == 8 ? 0xFFFFFFFFu : (bits == 16 ? 0x55555555u : 0x11111111u);
  const size_t end = len / 32 * 32;
  for (size_t byte = 0; byte < end; byte += 32) {
    __m256i v = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(rows[0] + byte));
    for (size_t i = 1; i < H; ++i)
      v = _mm256_xor_si256(v, _mm256_loadu_si256(reinterpret_cast<const __m256i*>(rows[i] + byte)));
    const __m256i eq = bits == 8    ? _mm256_cmpeq_epi8(v, target)
                       : bits == 16 ? _mm256_cmpeq_epi16(v, target)
                                    : _mm256_cmpeq_epi32(v, target);
    for (uint32_t m = (uint32_t)_mm256_movemask_epi8(eq) & keep; m; m &= m - 1)
      hit((byte + (size_t)__builtin_ctz(m)) / (bits / 8));
  }
  screen_bytes_scalar(rows, H, bits, fp, end, len, hit);
}

template <size_t B, class Hit>
__attribute__((target("avx2"))) void screen_packed_avx2(const uint8_t* const* rows, size_t H,
                                                        uint64_t fp, size_t count, Hit& hit) {
  const uint64_t ones = ~0ull / ((1ull << B) - 1);
  const __m256i target = _mm256_set1_epi64x((long long)(ones * fp));
  const __m256i low = _mm256_set1_epi64x((long long)ones);
  size_t base = 0;
  while (count - base >= 256 / B) {
    const size_t byte = base * B / 8;
    __m256i v = _mm256_setzero_si256();
    for (size_t i = 0; i < H; ++i)
      v = _mm256_xor_si256(v, _mm256_loadu_si256(reinterpret_cast<const __m256i*>(rows[i] + byte)));
    const __m256i diff = _mm256_xor_si256(v, target);
    __m256i f = _mm256_or_si256(diff, _mm256_srli_epi64(diff, 1));
    if (B == 4) f = _mm256_or_si256(f, _mm256_srli_epi64(f, 2));
    const __m256i m = _mm256_andnot_si256(f, low);
    if (!_mm256_testz_si256(m, m)) {
      alignas(32) uint64_t w[4];
      _mm256_store_si256(reinterpret_cast<__m256i*>(w), m);
      for (int q = 0; q < 4; ++q)
        for (uint64_t x = w[q]; x; x &= x - 1)
          hit(base + (size_t)q * (64 / B) + (size_t)__builtin_ctzll(x) / B);
    }
    base += 256 / B;
  }
  screen_packed_scalar<B>(rows, H, fp, count, base, hit);
}

template <class Hit>
void screen(const uint8_t* const* rows, size_t H, size_t bits, uint64_t fp, size_t G, bool avx2,
            Hit& hit) {
  if (bits == 2 || bits == 4) {
    if (avx2) bits == 2 ? screen_packed_avx2<2>(rows, H, fp, G, hit)
                        : screen_packed_avx2<4>(rows, H, fp, G, hit);
    else bits == 2 ? screen_packed_scalar<2>(rows, H, fp, G, 0, hit)
                   : screen_packed_scalar<4>(rows, H, fp, G, 0, hit);
    return;
  }
  if (bits == 1) {
    for (size_t base = 0; base < G; base += 64) {
      const size_t len = (std::min<size_t>(G - base, 64) + 7) / 8;
      uint64_t v = 0;
      for (size_t i = 0; i < H; ++i) {
        uint64_t x = 0;
        memcpy(&x, rows[i] + base / 8, len);
        v ^= x;
      }
      const size_t rem = std::min<size_t>(G - base, 64);
      uint64_t m = (fp == 1 ? v : ~v) & (~0ull >> (64 - rem));
      for (; m; m &= m - 1) hit(base + (size_t)__builtin_ctzll(m));
    }
    return;
  }
  const size_t len = G * bits / 8;
  if (avx2) screen_bytes_avx2(rows, H, bits, fp, len, hit);
  else screen_bytes_scalar(rows, H, bits, fp, 0, len, hit);
}

struct Scratch {
  std::vector<uint64_t> pos;            // block x classes x H cells
  std::vector<const Bank*> bank;        // block x classes selected banks
  std::vector<const uint8_t*> rows;     // H row starts of one key and class
  std::vector<uint64_t> snap;           // recovered origins' counters
};

inline void prefetch_key(const Index& ix, uint64_t key, const Bank* const* banks,
                         const uint64_t* pos) {
  if (ix.recovery && !ix.recover.dir.empty())
    __builtin_prefetch(&ix.recover.dir[ix.recover.first_slot(abandoned_hash(key, ix.seed))]);
  for (size_t ci = 0; ci < ix.classes.size(); ++ci) {
    const Bank& b = *banks[ci];
    const size_t rb = b.row_bytes(), bytes = (b.groups.size() * ix.bits + 7) / 8;
    for (size_t i = 0; i < ix.hashes; ++i)
      for (size_t byte = 0; byte < bytes; byte += 64)
        __builtin_prefetch(b.data.data() + pos[ci * ix.hashes + i] * rb + byte);
  }
}

void lookup_weighted(const Index& ix, uint64_t key, uint64_t weight, const Bank* const* banks,
                     const uint64_t* pos, bool avx2, Scratch& s, uint64_t* counts) {
  size_t rlen = 0;
  const uint32_t* rec = ix.recovery ? ix.recover.get(abandoned_hash(key, ix.seed), &rlen) : nullptr;
  s.snap.resize(rlen);
  for (size_t i = 0; i < rlen; ++i) s.snap[i] = counts[rec[i]];
  const uint64_t fp = splitmix64(key ^ ix.seed ^ 0x8E2D4F6A9B13C5D7ull) & ((1ull << ix.bits) - 1);
  s.rows.resize(ix.hashes);
  for (size_t ci = 0; ci < ix.classes.size(); ++ci) {
    const Bank& b = *banks[ci];
    const size_t rb = b.row_bytes(), G = b.groups.size(), bits = ix.bits;
    for (size_t i = 0; i < ix.hashes; ++i) s.rows[i] = b.data.data() + pos[ci * ix.hashes + i] * rb;
    auto hit = [&](size_t g) {
      const Group& gr = b.groups[g];
      if (gr.members.size() == 1) {
        counts[gr.members[0]] += weight;
        return;
      }
      const size_t off = G * bits + gr.offset - g * bits;
      uint64_t mask = 0;
      for (size_t i = 0; i < ix.hashes; ++i) mask ^= get_bits(s.rows[i], off, gr.width - bits);
      for (; mask; mask &= mask - 1) counts[gr.members[__builtin_ctzll(mask)]] += weight;
    };
    screen(s.rows.data(), ix.hashes, bits, fp, G, avx2, hit);
  }
  for (size_t i = 0; i < rlen; ++i)
    if (counts[rec[i]] == s.snap[i]) counts[rec[i]] += weight;
}

// Weighted keys (sorted, distinct) of one block into counts.
void lookup_block_batch(const Index& ix, const std::vector<std::pair<uint64_t, uint64_t>>& kw,
                        bool avx2, Scratch& s, uint64_t* counts) {
  constexpr size_t kBlock = 32, kAhead = 4;
  const size_t C = ix.classes.size(), H = ix.hashes;
  for (size_t b0 = 0; b0 < kw.size(); b0 += kBlock) {
    const size_t n = std::min(kBlock, kw.size() - b0);
    s.pos.resize(n * C * H);
    s.bank.resize(n * C);
    for (size_t j = 0; j < n; ++j) {
      const uint64_t key = kw[b0 + j].first;
      for (size_t ci = 0; ci < C; ++ci) {
        const auto& cls = ix.classes[ci];
        const Bank* bp = &ix.banks[cls[0]];
        if (cls.size() > 1)
          bp = &ix.banks[cls[splitmix64(key ^ ix.seed ^ 0x34B61D8F29A7C053ull) & (cls.size() - 1)]];
        s.bank[j * C + ci] = bp;
        positions(key, ix.seed, bp->slots, H, ix.has_segment ? ix.segment : 0,
                  &s.pos[(j * C + ci) * H]);
      }
    }
    for (size_t j = 0; j < std::min(n, kAhead); ++j)
      prefetch_key(ix, kw[b0 + j].first, &s.bank[j * C], &s.pos[j * C * H]);
    for (size_t j = 0; j < n; ++j) {
      if (j + kAhead < n)
        prefetch_key(ix, kw[b0 + j + kAhead].first, &s.bank[(j + kAhead) * C],
                     &s.pos[(j + kAhead) * C * H]);
      lookup_weighted(ix, kw[b0 + j].first, kw[b0 + j].second, &s.bank[j * C], &s.pos[j * C * H],
                      avx2, s, counts);
    }
  }
}

// Indexes the fast path serves: ordinary (non-findere) modes over
// fingerprint-first banks.
bool serves(const Index& ix) {
  if (ix.f.mode == 3 || ix.hashes > 32) return false;
  for (auto& b : ix.banks)
    if (!b.fp_first) return false;
  return true;
}

}  // namespace fastpath

// Set for the duration of one oracle_query_handle_fast call (the baseline's
// calls do not overlap).
bool g_fast_lookup = false;

void run_query(const Index& ix, const Work& w, int threads, std::vector<uint64_t>& counts) {
  const size_t C = ix.colors.size();
  counts.assign(C, 0);
  if (threads < 1) threads = 1;
  std::vector<std::vector<uint64_t>> part(threads, std::vector<uint64_t>(C, 0));
  std::vector<std::thread> pool;
  if (ix.f.mode != 3) {
    // query_feature_range (record_query.rs:337-404): 32 Ki-key blocks,
    // sorted, with repeated keys folded into weights.
    const size_t block = 32 * 1024;
    size_t blocks = (w.keys.size() + block - 1) / block;
    std::atomic<size_t> next{0};
    for (int t = 0; t < threads; ++t)
      pool.emplace_back([&, t] {
        std::vector<uint32_t> hits;
        std::vector<uint64_t> keys;
        if (g_fast_lookup && fastpath::serves(ix)) {
          const bool avx2 = __builtin_cpu_supports("avx2");
          fastpath::Scratch s;
          std::vector<std::pair<uint64_t, uint64_t>> kw;
          for (size_t bi; (bi = next.fetch_add(1)) < blocks;) {
            size_t a = bi * block, e = std::min(w.keys.size(), a + block);
            keys.assign(w.keys.begin() + a, w.keys.begin() + e);
            std::sort(keys.begin(), keys.end());
            kw.clear();
            for (size_t i = 0; i < keys.size();) {
              size_t j = i + 1;
              while (j < keys.size() && keys[j] == keys[i]) ++j;
              kw.emplace_back(keys[i], j - i);
              i = j;
            }
            fastpath::lookup_block_batch(ix, kw, avx2, s, part[t].data());
          }
          return;
        }
        for (size_t bi; (bi = next.fetch_add(1)) < blocks;) {
          size_t a = bi * block, e = std::min(w.keys.size(), a + block);
          keys.assign(w.keys.begin() + a, w.keys.begin() + e);
          std::sort(keys.begin(), keys.end());
          for (size_t i = 0; i < keys.size();) {
            size_t j = i + 1;
            while (j < keys.size() && keys[j] == keys[i]) ++j;
            lookup(ix, keys[i], hits);
            for (uint32_t c : hits) part[t][c] += j - i;
            i = j;
          }
        }
      });
  } else {
    // Scores::score findere branch (query_stream.rs:670-689): a colour
    // counts a k-window when z+1 consecutive s-mers of a task hit it.
    std::atomic<size_t> next{0};
    for (int t = 0; t < threads; ++t)
      pool.emplace_back([&, t] {
        std::vector<uint32_t> hits;
        std::vector<size_t> last(C, SIZE_MAX), run(C, 0);
        std::vector<uint32_t> touched;
        for (size_t ti; (ti = next.fetch_add(1)) < w.tasks.size();) {
          for (uint32_t c : touched) last[c] = SIZE_MAX;
          touched.clear();
          auto [a, e] = w.tasks[ti];
          for (size_t p = a; p < e; ++p) {
            lookup(ix, w.keys[p], hits);
            size_t pos = p - a;
            for (uint32_t c : hits) {
              run[c] = (last[c] != SIZE_MAX && last[c] + 1 == pos) ? run[c] + 1 : 1;
              if (last[c] == SIZE_MAX) touched.push_back(c);
              last[c] = pos;
              if (run[c] > ix.f.z) part[t][c] += 1;
            }
          }
        }
      });
  }
  for (auto& th : pool) th.join();
  for (auto& p : part)
    for (size_t c = 0; c < C; ++c) counts[c] += p[c];
}

// ------------------------------------------------------- per-record query ---
// query_records_command_with_memory (src/power_merge/storage.rs:3626-3720).

struct NamedRecord {
  std::string name;
  std::vector<uint8_t> seq;
};

// std::str::from_utf8 acceptance: decodes each sequence and rejects
// overlong forms, surrogates and code points above U+10FFFF.
bool utf8_ok(const std::string& s) {
  size_t i = 0;
  while (i < s.size()) {
    const unsigned char c = (unsigned char)s[i];
    const int len = c < 0x80 ? 1 : (c >> 5) == 6 ? 2 : (c >> 4) == 14 ? 3 : (c >> 3) == 30 ? 4 : 0;
    if (!len || i + len > s.size()) return false;
    uint32_t cp = len == 1 ? c : c & (0x7f >> len);
    for (int j = 1; j < len; ++j) {
      const unsigned char d = (unsigned char)s[i + j];
      if ((d >> 6) != 2) return false;
      cp = cp << 6 | (d & 0x3f);
    }
    static const uint32_t least[5] = {0, 0, 0x80, 0x800, 0x10000};
    if (cp < least[len] || cp > 0x10ffff || (cp >= 0xd800 && cp <= 0xdfff)) return false;
    i += len;
  }
  return true;
}

// read_batches (src/power_merge/records.rs:150-290): trailing whitespace of a
// line is dropped and empty lines are skipped; the first line decides FASTQ
// ('@') or FASTA; the identifier is the header up to the first whitespace;
// sequence lines may not contain whitespace; FASTQ qualities are consumed by
// length; identifiers must be UTF-8 and at least one record is required.
std::vector<NamedRecord> parse_named_records(const std::vector<uint8_t>& d) {
  std::vector<NamedRecord> out;
  size_t i = 0;
  auto next_line = [&](std::string& line) {
    if (i >= d.size()) return false;
    size_t e = i;
    while (e < d.size() && d[e] != '\n') ++e;
    line.assign((const char*)d.data() + i, e - i);
    i = e < d.size() ? e + 1 : e;
    return true;
  };
  auto is_ws = [](char c) {
    return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v';
  };
  auto ident = [&](const std::string& line, const char* what) {
    size_t e = 1;
    while (e < line.size() && !is_ws(line[e])) ++e;
    std::string id = line.substr(1, e - 1);
    ensure(!id.empty(), (std::string("empty ") + what + " identifier").c_str());
    ensure(utf8_ok(id), (std::string("invalid ") + what + " identifier").c_str());
    return id;
  };
  int fastq = -1;
  std::string line;
  bool have = false;
  while (next_line(line)) {
    while (!line.empty() && is_ws(line.back())) line.pop_back();
    if (line.empty()) continue;
    if (fastq == 1 || (fastq == -1 && line[0] == '@')) {
      fastq = 1;
      ensure(line[0] == '@', "expected FASTQ identifier");
      NamedRecord r;
      r.name = ident(line, "FASTQ");
      for (;;) {
        ensure(next_line(line), "truncated FASTQ sequence");
        while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
        if (!line.empty() && line[0] == '+') break;
        for (char c : line) ensure(!is_ws(c), "whitespace inside FASTQ sequence");
        r.seq.insert(r.seq.end(), line.begin(), line.end());
      }
      size_t q = 0;
      while (q < r.seq.size()) {
        ensure(next_line(line), "truncated FASTQ quality");
        while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
        q += line.size();
        ensure(q <= r.seq.size(), "FASTQ sequence and quality lengths differ");
      }
      out.push_back(std::move(r));
      continue;
    }
    fastq = 0;
    if (line[0] == '>') {
      NamedRecord r;
      r.name = ident(line, "FASTA");
      out.push_back(std::move(r));
      have = true;
    } else {
      ensure(have, "--records requires FASTA or FASTQ");
      for (char c : line) ensure(!is_ws(c), "whitespace inside FASTA sequence");
      out.back().seq.insert(out.back().seq.end(), line.begin(), line.end());
    }
  }
  ensure(!out.empty(), "no FASTA/FASTQ records");
  return out;
}

// write_field (src/power_merge/record_output.rs:64-80): CSV quoting of names
// holding a tab, CR, LF or quote.
void write_field(std::string& out, const std::string& v) {
  if (v.find_first_of("\t\r\n\"") == std::string::npos) {
    out += v;
    return;
  }
  out += '"';
  for (char c : v) {
    out += c;
    if (c == '"') out += '"';
  }
  out += '"';
}

const char* records_header(bool compact) {
  return compact ? "query_id\tvalid_kmers\thits"
                 : "query_id\tdataset_id\tdataset_name\tmatches\tqueried_seeds\tratio";
}

// RecordScores::write_record (storage.rs:3109-3146) and
// RecordFormat::write_record (record_output.rs:21-62): with min_ratio 0 every
// colour is reported, otherwise the touched colours in id order whose ratio
// reaches min_ratio.
void format_record(const Index& ix, const std::string& name, uint64_t total,
                   const std::vector<uint64_t>& counts, double min_ratio, bool compact,
                   std::string& out) {
  std::vector<std::pair<size_t, uint64_t>> hits;
  for (size_t c = 0; c < counts.size(); ++c) {
    if (min_ratio > 0.0 && (total == 0 || counts[c] == 0)) continue;
    double ratio = total == 0 ? 0.0 : (double)counts[c] / (double)total;
    if (ratio >= min_ratio) hits.emplace_back(c, counts[c]);
  }
  char buf[96];
  if (compact) {
    out += name;
    snprintf(buf, sizeof buf, "\t%llu\t", (unsigned long long)total);
    out += buf;
    for (size_t i = 0; i < hits.size(); ++i) {
      snprintf(buf, sizeof buf, i ? ",%zu:%llu" : "%zu:%llu", hits[i].first,
               (unsigned long long)hits[i].second);
      out += buf;
    }
    out += '\n';
    return;
  }
  for (auto& h : hits) {
    write_field(out, name);
    snprintf(buf, sizeof buf, "\t%zu\t", h.first);
    out += buf;
    write_field(out, ix.colors[h.first].name);
    double ratio = total == 0 ? 0.0 : (double)h.second / (double)total;
    snprintf(buf, sizeof buf, "\t%llu\t%llu\t%.8f\n", (unsigned long long)h.second,
             (unsigned long long)total, ratio);
    out += buf;
  }
  if (hits.empty()) {
    write_field(out, name);
    snprintf(buf, sizeof buf, "\t.\t.\t0\t%llu\t0.00000000\n", (unsigned long long)total);
    out += buf;
  }
}

// reverse_complement (src/anchors.rs:257-263): reversed, ACGT complemented
// (upper case), every other byte kept as a separator.
std::vector<uint8_t> reverse_complement(const uint8_t* seq, size_t n) {
  std::vector<uint8_t> r(n);
  for (size_t i = 0; i < n; ++i) {
    const uint8_t b = seq[n - 1 - i];
    const int c = encode_base(b);
    r[i] = c < 0 ? b : (uint8_t)"TGCA"[c];
  }
  return r;
}

// Counts of one record queried alone. Randstrobemer indexes extract both
// strands (PreparedRead::new, query_stream.rs:516-534) and keep per colour
// the larger strand count (Scores::score, query_stream.rs:690-701); total =
// forward anchors, probes = anchors of both strands.
void record_counts(const Index& ix, const uint8_t* seq, size_t n, std::vector<uint64_t>& counts,
                   uint64_t& total, uint64_t& probes) {
  Work w;
  prepare_record(ix.f, seq, n, w);
  run_query(ix, w, 1, counts);
  total = w.total;
  probes = w.probes;
  if (!ix.f.strobes) return;
  std::vector<uint8_t> rc = reverse_complement(seq, n);
  Work wr;
  prepare_record(ix.f, rc.data(), rc.size(), wr);
  ensure(wr.keys.size() == w.keys.size(), "canonical anchor counts must agree across strands");
  std::vector<uint64_t> reverse;
  run_query(ix, wr, 1, reverse);
  for (size_t c = 0; c < counts.size(); ++c) counts[c] = std::max(counts[c], reverse[c]);
  probes += wr.probes;
}

// Aggregate counts of records seq(r), r < records: one pass over all seeds,
// or for randstrobemer indexes the per-record strand maxima summed (records
// spread over `threads` workers).
void query_many(const Index& ix, size_t records,
                const std::function<std::pair<const uint8_t*, size_t>(size_t)>& seq, int threads,
                std::vector<uint64_t>& counts, uint64_t& total, uint64_t& probes) {
  if (!ix.f.strobes) {
    Work w;
    for (size_t r = 0; r < records; ++r) {
      auto sq = seq(r);
      prepare_record(ix.f, sq.first, sq.second, w);
    }
    run_query(ix, w, threads, counts);
    total = w.total;
    probes = w.probes;
    return;
  }
  const size_t C = ix.colors.size(), T = (size_t)std::max(1, threads);
  std::vector<std::vector<uint64_t>> part(T, std::vector<uint64_t>(C, 0));
  std::vector<uint64_t> tot(T, 0), prb(T, 0);
  std::vector<std::string> err(T);
  std::vector<std::thread> pool;
  for (size_t t = 0; t < T; ++t)
    pool.emplace_back([&, t] {
      try {
        std::vector<uint64_t> c;
        for (size_t r = records * t / T; r < records * (t + 1) / T; ++r) {
          auto sq = seq(r);
          uint64_t a = 0, b = 0;
          record_counts(ix, sq.first, sq.second, c, a, b);
          for (size_t i = 0; i < C; ++i) part[t][i] += c[i];
          tot[t] += a;
          prb[t] += b;
        }
      } catch (const std::exception& e) {
        err[t] = e.what();
      }
    });
  for (auto& th : pool) th.join();
  for (auto& e : err) ensure(e.empty(), e.c_str());
  counts.assign(C, 0);
  total = probes = 0;
  for (size_t t = 0; t < T; ++t) {
    for (size_t i = 0; i < C; ++i) counts[i] += part[t][i];
    total += tot[t];
    probes += prb[t];
  }
}

// Per-record counts and totals of named records (each record queried alone).
std::string query_records_output(const Index& ix, const std::vector<NamedRecord>& recs,
                                 double min_ratio, bool compact) {
  std::string out = records_header(compact);
  out += '\n';
  for (auto& r : recs) {
    std::vector<uint64_t> counts;
    uint64_t total = 0, probes = 0;
    record_counts(ix, r.seq.data(), r.seq.size(), counts, total, probes);
    format_record(ix, r.name, total, counts, min_ratio, compact, out);
  }
  return out;
}

int guarded(const std::function<void()>& body) {
  try {
    body();
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

std::string format_aggregate(const Index& ix, const uint64_t* counts, uint64_t total,
                             double min_ratio) {
  std::string out = "color\tmatches\tratio\tunique_kmers\n";
  char buf[64];
  for (size_t c = 0; c < ix.colors.size(); ++c) {
    double ratio = total == 0 ? 0.0 : (double)counts[c] / (double)total;
    if (!(ratio >= min_ratio)) continue;
    out += ix.colors[c].name;
    snprintf(buf, sizeof buf, "\t%llu\t%.8f\t%llu\n", (unsigned long long)counts[c], ratio,
             (unsigned long long)ix.colors[c].unique);
    out += buf;
  }
  return out;
}

const char* mode_label(int mode) {
  static const char* labels[] = {"kmers", "minimizers", "modimizers", "findere"};
  return mode >= 0 && mode < 4 ? labels[mode] : "?";
}

}  // namespace

extern "C" {

uint64_t oracle_splitmix64(uint64_t x) { return splitmix64(x); }

const char* oracle_last_error(void) { return g_error.c_str(); }

int oracle_features(const uint8_t* seq, size_t len, int mode, int k, int m, uint64_t seed,
                    uint64_t sampling, int findere_z, int homopolymer, uint64_t* out, size_t cap,
                    size_t* count) {
  return guarded([&] {
    Features f;
    f.mode = mode;
    f.k = (size_t)k;
    f.m = (size_t)m;
    f.seed = seed;
    f.sampling = sampling;
    f.z = (size_t)findere_z;
    f.homopolymer = homopolymer != 0;
    Emit keys;
    for_each_run(seq, len, f.homopolymer,
                 [&](const uint8_t* run, size_t n) { scan_run_features(run, n, f, keys); });
    *count = keys.size();
    memcpy(out, keys.data(), std::min(cap, keys.size()) * 8);
  });
}

uint64_t oracle_strobe_hash(uint64_t v) { return strobe_hash(v); }

void oracle_positions(uint64_t key, uint64_t seed, uint64_t cells, int hashes, uint64_t segment,
                      uint64_t* out) {
  positions(key, seed, cells, (size_t)hashes, segment, out);
}

uint32_t oracle_abandoned_hash(uint64_t key, uint64_t seed) { return abandoned_hash(key, seed); }

// Links candidates (ascending positions, their strobe hashes) into keys.
void oracle_link_strobes(const uint64_t* positions, const uint64_t* hashes, size_t n,
                         uint64_t dmin, uint64_t dmax, uint64_t* out) {
  std::vector<std::pair<size_t, uint64_t>> cand(n);
  for (size_t i = 0; i < n; ++i) cand[i] = {(size_t)positions[i], hashes[i]};
  Emit keys;
  link_strobes(cand, dmin, dmax, keys);
  memcpy(out, keys.data(), keys.size() * 8);
}

// Seeds of a sequence with a spaced-seed pattern ("" = none) and, when
// strobe_max > 0, randstrobemers linked over [strobe_min, strobe_max].
int oracle_features_anchored(const uint8_t* seq, size_t len, int mode, int k, int m, uint64_t seed,
                             int homopolymer, const char* pattern, uint64_t strobe_min,
                             uint64_t strobe_max, uint64_t* out, size_t cap, size_t* count) {
  return guarded([&] {
    Features f;
    f.mode = mode;
    f.k = (size_t)k;
    f.m = (size_t)m;
    f.seed = seed;
    f.homopolymer = homopolymer != 0;
    if (pattern && *pattern)
      ensure(parse_pattern(pattern, &f.pattern_mask, &f.pattern_width), "invalid seed pattern");
    if (strobe_max) {
      f.strobes = true;
      f.strobe_min = strobe_min;
      f.strobe_max = strobe_max;
    }
    Emit keys;
    for_each_run(seq, len, f.homopolymer,
                 [&](const uint8_t* run, size_t n) { scan_run_features(run, n, f, keys); });
    *count = keys.size();
    memcpy(out, keys.data(), std::min(cap, keys.size()) * 8);
  });
}

// Spaced-seed key of a 2-bit key under a pattern (anchors.rs:86-90); returns
// ZX error when the pattern is invalid.
int oracle_pattern_canonical(const char* pattern, uint64_t key, uint64_t* projected,
                             uint64_t* canonical) {
  return guarded([&] {
    uint64_t mask = 0;
    size_t width = 0;
    ensure(parse_pattern(pattern, &mask, &width), "invalid seed pattern");
    *projected = pattern_project(mask, width, key);
    *canonical = pattern_canonical(mask, width, key);
  });
}

int oracle_ocm_slow(const uint8_t* seq, size_t len, int k, int m, uint64_t seed,
                    uint64_t* pos_out, uint64_t* key_out, size_t cap, size_t* count) {
  return guarded([&] {
    // open_closed_minimizers.rs:43-85: evaluate every candidate per window.
    OcmGeom g = ocm_geom((size_t)k, (size_t)m);
    std::vector<std::pair<size_t, uint64_t>> res;
    for (size_t st = 0; st + (size_t)k <= len; ++st) {
      const uint8_t* win = seq + st;
      Rank best{255, 0};
      std::vector<size_t> tied;
      for (size_t p = 0; p + g.t <= (size_t)k; ++p) {
        std::vector<uint64_t> hs;
        for (size_t q = 0; q + g.s <= g.t; ++q)
          hs.push_back(mixsplit(canonical_encoded(encode_full(win + p + q, g.s), g.s),
                                seed ^ 0xC6BC279692B5CC83ull));
        uint64_t mn = *std::min_element(hs.begin(), hs.end());
        uint8_t cls = hs[(g.t - g.s) / 2] == mn ? 0 : (hs.front() == mn || hs.back() == mn) ? 1 : 2;
        Rank r{cls, mixsplit(canonical_encoded(encode_full(win + p, g.t), g.t), seed)};
        if (r < best) {
          best = r;
          tied.assign(1, p);
        } else if (r == best) {
          tied.push_back(p);
        }
      }
      size_t gt = 0;
      for (size_t i = 0; i < (size_t)k; ++i) gt += encode_base(win[i]) >= 2;
      size_t anchor = gt > (size_t)k / 2 ? tied.back() : tied.front();
      size_t pos = st + anchor % g.w;
      if (res.empty() || res.back().first != pos)
        res.emplace_back(pos, canonical_encoded(encode_full(seq + pos, m), m));
    }
    *count = res.size();
    for (size_t i = 0; i < std::min(cap, res.size()); ++i) {
      pos_out[i] = res[i].first;
      key_out[i] = res[i].second;
    }
  });
}

int oracle_index_colors(const char* index_dir, size_t* colors) {
  return guarded([&] { *colors = load_index(index_dir, false, false)->colors.size(); });
}

int oracle_query_file(const char* index_dir, const char* query_path, int threads, int recover,
                      uint64_t* counts, size_t colors, uint64_t* total, uint64_t* probes) {
  return guarded([&] {
    auto ix = load_index(index_dir, recover != 0);
    ensure(colors == ix->colors.size(), "colour count differs from the index");
    std::vector<std::vector<uint8_t>> records;
    parse_fastx(read_decoded(query_path), records);
    std::vector<uint64_t> out;
    query_many(
        *ix, records.size(),
        [&](size_t r) { return std::make_pair((const uint8_t*)records[r].data(), records[r].size()); },
        threads, out, *total, *probes);
    memcpy(counts, out.data(), colors * 8);
  });
}

int oracle_query_records(const char* index_dir, const uint8_t* bases, const uint64_t* offsets,
                         size_t records, int threads, int recover, uint64_t* counts, size_t colors,
                         uint64_t* total, uint64_t* probes) {
  return guarded([&] {
    auto ix = load_index(index_dir, recover != 0);
    ensure(colors == ix->colors.size(), "colour count differs from the index");
    std::vector<uint64_t> out;
    query_many(
        *ix, records,
        [&](size_t r) { return std::make_pair(bases + offsets[r], (size_t)(offsets[r + 1] - offsets[r])); },
        threads, out, *total, *probes);
    memcpy(counts, out.data(), colors * 8);
  });
}

int oracle_format_aggregate(const char* index_dir, const uint64_t* counts, uint64_t total,
                            double min_ratio, char* buf, size_t cap, size_t* written) {
  return guarded([&] {
    auto ix = load_index(index_dir, false, false);
    std::string s = format_aggregate(*ix, counts, total, min_ratio);
    *written = s.size();
    memcpy(buf, s.data(), std::min(cap, s.size()));
  });
}

// Timed CPU query used by the baseline: index load excluded (like the
// reference's query_s), parsing + extraction + lookup included. Returns the
// query seconds through *seconds.
int oracle_query_timed(const char* index_dir, const uint8_t* bases, const uint64_t* offsets,
                       size_t records, int threads, uint64_t* counts, size_t colors,
                       uint64_t* total, double* seconds) {
  return guarded([&] {
    auto ix = load_index(index_dir, true);
    ensure(colors == ix->colors.size(), "colour count differs from the index");
    auto t0 = std::chrono::steady_clock::now();
    std::vector<uint64_t> out;
    uint64_t probes = 0;
    query_many(
        *ix, records,
        [&](size_t r) { return std::make_pair(bases + offsets[r], (size_t)(offsets[r + 1] - offsets[r])); },
        threads, out, *total, probes);
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    memcpy(counts, out.data(), colors * 8);
  });
}

// Per-record report of a query file (TSV or compact), as
// `zorindex query --records` prints it.
int oracle_query_records_report(const char* index_dir, const char* query_path, int recover,
                                double min_ratio, int compact, char* buf, size_t cap,
                                size_t* written) {
  return guarded([&] {
    auto ix = load_index(index_dir, recover != 0);
    std::string s = query_records_output(*ix, parse_named_records(read_decoded(query_path)),
                                         min_ratio, compact != 0);
    *written = s.size();
    if (buf) memcpy(buf, s.data(), std::min(cap, s.size()));
  });
}

struct oracle_index {
  std::unique_ptr<Index> ix;
};

int oracle_open(const char* index_dir, int recover, oracle_index** out) {
  return guarded([&] {
    auto h = std::make_unique<oracle_index>();
    h->ix = load_index(index_dir, recover != 0);
    *out = h.release();
  });
}

void oracle_close(oracle_index* index) { delete index; }

int oracle_query_handle_fast(oracle_index* h, const uint8_t* bases, const uint64_t* offsets,
                             size_t records, int threads, uint64_t* counts, size_t colors,
                             uint64_t* total, double* seconds) {
  g_fast_lookup = true;
  const int rc = oracle_query_handle(h, bases, offsets, records, threads, counts, colors, total,
                                     seconds);
  g_fast_lookup = false;
  return rc;
}

int oracle_fast_serves(oracle_index* h) { return fastpath::serves(*h->ix) ? 1 : 0; }

int oracle_query_handle(oracle_index* h, const uint8_t* bases, const uint64_t* offsets,
                        size_t records, int threads, uint64_t* counts, size_t colors,
                        uint64_t* total, double* seconds) {
  return guarded([&] {
    const Index& ix = *h->ix;
    ensure(colors == ix.colors.size(), "colour count differs from the index");
    auto t0 = std::chrono::steady_clock::now();
    std::vector<uint64_t> out;
    uint64_t probes = 0;
    query_many(
        ix, records,
        [&](size_t r) { return std::make_pair(bases + offsets[r], (size_t)(offsets[r + 1] - offsets[r])); },
        threads, out, *total, probes);
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    memcpy(counts, out.data(), colors * 8);
  });
}

// Per-record report of a query file over a resident index, records split
// across `threads` workers in contiguous runs (the report keeps input order);
// *seconds covers reading, querying and formatting (not the index load).
int oracle_records_report_handle(oracle_index* h, const char* query_path, double min_ratio,
                                 int compact, int threads, char* buf, size_t cap,
                                 size_t* written, double* seconds) {
  return guarded([&] {
    const Index& ix = *h->ix;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<NamedRecord> recs = parse_named_records(read_decoded(query_path));
    const size_t T = (size_t)std::max(1, std::min<int>(threads, (int)recs.size()));
    std::vector<std::string> parts(T);
    std::vector<std::thread> pool;
    for (size_t t = 0; t < T; ++t)
      pool.emplace_back([&, t] {
        const size_t a = recs.size() * t / T, b = recs.size() * (t + 1) / T;
        for (size_t r = a; r < b; ++r) {
          std::vector<uint64_t> counts;
          uint64_t total = 0, probes = 0;
          record_counts(ix, recs[r].seq.data(), recs[r].seq.size(), counts, total, probes);
          format_record(ix, recs[r].name, total, counts, min_ratio, compact != 0, parts[t]);
        }
      });
    for (auto& th : pool) th.join();
    std::string s = records_header(compact != 0);
    s += '\n';
    for (auto& p : parts) s += p;
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *written = s.size();
    if (buf) memcpy(buf, s.data(), std::min(cap, s.size()));
  });
}

}  // extern "C"

#ifdef ZX_ORACLE_MAIN
// zx_oracle query -i DIR -q FILE [-a RATIO] [-t THREADS]: the aggregate TSV of
// `zorindex query` on stdout and its #query line on stderr.
int main(int argc, char** argv) {
  std::string dir, query, format = "tsv";
  double ratio = 0;
  bool records = false;
  int threads = (int)std::thread::hardware_concurrency();
  for (int i = 2; i < argc; ++i) {
    std::string a = argv[i];
    if (a == "-r") {
      records = true;
      continue;
    }
    if (i + 1 >= argc) break;
    if (a == "-i") dir = argv[++i];
    else if (a == "-q") query = argv[++i];
    else if (a == "-a") ratio = atof(argv[++i]);
    else if (a == "-t") threads = atoi(argv[++i]);
    else if (a == "-F") format = argv[++i];
  }
  if (records && !dir.empty() && !query.empty()) {
    try {
      auto ix = load_index(dir, true);
      std::string s = query_records_output(*ix, parse_named_records(read_decoded(query)), ratio,
                                           format == "compact");
      fwrite(s.data(), 1, s.size(), stdout);
      return 0;
    } catch (const std::exception& e) {
      fprintf(stderr, "error: %s\n", e.what());
      return 1;
    }
  }
  if (argc < 2 || std::string(argv[1]) != "query" || dir.empty() || query.empty()) {
    fprintf(stderr, "usage: zx_oracle query -i DIR -q FILE [-a RATIO] [-t THREADS] [-r [-F tsv|compact]]\n");
    return 2;
  }
  try {
    auto ix = load_index(dir, true);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::vector<uint8_t>> records;
    parse_fastx(read_decoded(query), records);
    std::vector<uint64_t> counts;
    uint64_t total = 0, probes = 0;
    query_many(
        *ix, records.size(),
        [&](size_t r) { return std::make_pair((const uint8_t*)records[r].data(), records[r].size()); },
        threads, counts, total, probes);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    fprintf(stderr,
            "#query\t%s\tk=%zu\tindex_mode=%s\ttotal_features=%llu\tstack_probes=%llu\t"
            "bank_probes=%llu\telapsed_s=%.6f\n",
            query.c_str(), ix->k, mode_label(ix->f.mode), (unsigned long long)total,
            (unsigned long long)probes, (unsigned long long)(probes * ix->classes.size()), secs);
    fputs(format_aggregate(*ix, counts.data(), total, ratio).c_str(), stdout);
    return 0;
  } catch (const std::exception& e) {
    fprintf(stderr, "Error: %s\n", e.what());
    return 1;
  }
}
#endif
