// Index builder: see builder.h. Reference construction stages restated here:
// BuildConfig::slots (src/power_merge/mod.rs:319-337), group values
// fp | membership << b (storage.rs:1301-1308), promotion layout
// (layout.rs:7-115), hash partitioning (storage.rs:1524-1642), peeling with
// "first active key in a minimum-degree cell" cycle breaking
// (src/bin/zorindex.rs:634-841), fingerprint-first row packing
// (storage.rs:1721-1878) and the ZORABN2 recovery file (storage.rs:1882-2128).
// The phases shared with the device builder are in namespace zx::build
// (builder_internal.h).
#include "builder_internal.h"

#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <thread>

#include "../host/error.h"
#include "../host/fastx.h"
#include "../host/json.h"
#include "../host/zstd_io.h"
#include "../zx_hash.h"
#include "synth.h"

namespace zx {
namespace build {
namespace {

std::string strip_name(const std::string& path) {
  std::string name = path.substr(path.find_last_of('/') == std::string::npos
                                     ? 0
                                     : path.find_last_of('/') + 1);
  for (const char* ext : {".zstd", ".zst", ".gzip", ".gz", ".xz", ".bz2", ".bz", ".bzip2",
                          ".fasta", ".fastq", ".fna", ".fa", ".fq", ".fas"}) {
    size_t n = strlen(ext);
    if (name.size() >= n && name.compare(name.size() - n, n, ext) == 0)
      name = name.substr(0, name.size() - n);
  }
  return name.empty() ? "color" : name;
}

// read_fof (src/lib.rs:329-372).
std::vector<Input> read_fof(const std::string& path) {
  std::ifstream in(path);
  if (!in) raise(kEIo, "cannot open " + path);
  std::vector<Input> out;
  std::string line;
  while (std::getline(in, line)) {
    size_t a = line.find_first_not_of(" \t\r\n");
    if (a == std::string::npos || line[a] == '#') continue;
    size_t b = line.find_last_not_of(" \t\r\n");
    std::string t = line.substr(a, b - a + 1);
    Input input;
    size_t tab = t.find('\t');
    if (tab != std::string::npos) {
      auto trim = [](std::string s) {
        size_t x = s.find_first_not_of(" \t"), y = s.find_last_not_of(" \t");
        return x == std::string::npos ? std::string() : s.substr(x, y - x + 1);
      };
      input.name = trim(t.substr(0, tab));
      std::string rest = t.substr(tab + 1);
      size_t tab2 = rest.find('\t');
      input.path = trim(tab2 == std::string::npos ? rest : rest.substr(0, tab2));
    } else {
      std::istringstream ss(t);
      std::string x, y;
      ss >> x >> y;
      if (!y.empty()) {
        input.name = x;
        input.path = y;
      } else {
        input.path = x;
        input.name = strip_name(x);
      }
    }
    check(!input.name.empty(), kEInval, "file of files has an empty color name");
    out.push_back(input);
  }
  check(!out.empty(), kEInval, "file of files contains no inputs");
  return out;
}

int ilog2(uint64_t v) { return 63 - __builtin_clzll(v); }

// ZOR construction of one filter: peel the H-uniform hypergraph, abandon
// keys when the peel stalls, assign cells in reverse peel order so every
// kept key's H cells XOR to its value. Returns the abandoned key indices.
std::vector<uint32_t> construct_filter(const std::vector<uint64_t>& keys,
                                       const std::vector<uint64_t>& values, uint64_t slots,
                                       int H, uint64_t seg, uint64_t seed,
                                       std::vector<uint64_t>& cells) {
  const size_t n = keys.size();
  check(slots <= 0xFFFFFFFFull, kEInval, "filter too large for 32-bit cell ids");
  check(n < 0xFFFFFFFFull, kEInval, "too many keys in one filter");
  std::vector<uint32_t> pos(n * (size_t)H);
  std::vector<uint32_t> deg(slots, 0), xr(slots, 0);
  uint64_t tmp[kMaxHashes];
  for (size_t e = 0; e < n; ++e) {
    positions(keys[e], seed, slots, H, seg, tmp);
    for (int i = 0; i < H; ++i) {
      uint32_t s = (uint32_t)tmp[i];
      pos[e * H + i] = s;
      ++deg[s];
      xr[s] ^= (uint32_t)e;
    }
  }
  std::vector<uint8_t> state(n, 0);  // 0 active, 1 peeled, 2 abandoned
  std::vector<std::pair<uint32_t, uint32_t>> stack;
  stack.reserve(n);
  std::vector<uint32_t> queue;
  for (uint64_t s = 0; s < slots; ++s)
    if (deg[s] == 1) queue.push_back((uint32_t)s);
  std::vector<std::vector<uint32_t>> buckets;  // cycle-break phase only
  bool breaking = false;
  auto remove_edge = [&](uint32_t e) {
    for (int i = 0; i < H; ++i) {
      uint32_t s = pos[(size_t)e * H + i];
      --deg[s];
      xr[s] ^= e;
      if (deg[s] == 1) queue.push_back(s);
      else if (breaking && deg[s] >= 2) {
        if (buckets.size() <= deg[s]) buckets.resize(deg[s] + 1);
        buckets[deg[s]].push_back(s);
      }
    }
  };
  auto drain = [&] {
    while (!queue.empty()) {
      uint32_t s = queue.back();
      queue.pop_back();
      if (deg[s] != 1) continue;
      uint32_t e = xr[s];
      state[e] = 1;
      stack.emplace_back(e, s);
      remove_edge(e);
    }
  };
  drain();
  std::vector<uint32_t> abandoned;
  if (stack.size() < n) {
    // Cyclic core: adjacency of the remaining keys, then repeatedly abandon
    // the first active key of a minimum-degree cell and keep peeling.
    breaking = true;
    std::vector<uint32_t> start(slots + 1, 0);
    for (size_t e = 0; e < n; ++e)
      if (!state[e])
        for (int i = 0; i < H; ++i) ++start[pos[e * H + i] + 1];
    for (uint64_t s = 0; s < slots; ++s) start[s + 1] += start[s];
    std::vector<uint32_t> adj(start[slots]), fill(start.begin(), start.end() - 1);
    for (size_t e = 0; e < n; ++e)
      if (!state[e])
        for (int i = 0; i < H; ++i) adj[fill[pos[e * H + i]]++] = (uint32_t)e;
    for (uint64_t s = 0; s < slots; ++s)
      if (deg[s] >= 2) {
        if (buckets.size() <= deg[s]) buckets.resize(deg[s] + 1);
        buckets[deg[s]].push_back((uint32_t)s);
      }
    size_t d = 2;
    while (stack.size() + abandoned.size() < n) {
      if (d >= buckets.size()) d = 2;
      while (d < buckets.size() && buckets[d].empty()) ++d;
      check(d < buckets.size(), kEInval, "peeling made no progress");
      uint32_t s = buckets[d].back();
      buckets[d].pop_back();
      if (deg[s] != d) continue;
      uint32_t victim = UINT32_MAX;
      for (uint32_t q = start[s]; q < start[s + 1]; ++q)
        if (state[adj[q]] == 0) {
          victim = adj[q];
          break;
        }
      if (victim == UINT32_MAX) continue;
      state[victim] = 2;
      abandoned.push_back(victim);
      remove_edge(victim);
      drain();
      d = 2;
    }
  }
  cells.assign(slots, 0);
  for (size_t i = stack.size(); i-- > 0;) {
    uint32_t e = stack[i].first, s = stack[i].second;
    uint64_t v = values[e];
    for (int h = 0; h < H; ++h) {
      uint32_t p = pos[(size_t)e * H + h];
      if (p != s) v ^= cells[p];
    }
    cells[s] = v;
  }
  std::sort(abandoned.begin(), abandoned.end());
  return abandoned;
}

// OR `width` bits of `value` into a little-endian bit stream at `bit`, with
// atomic word updates so groups sharing a row can be packed concurrently.
inline void or_bits(uint64_t* words, uint64_t bit, uint64_t width, uint64_t value) {
  if (width < 64) value &= (1ull << width) - 1;
  if (!value) return;
  uint64_t w = bit >> 6, sh = bit & 63;
  __atomic_fetch_or(&words[w], value << sh, __ATOMIC_RELAXED);
  if (sh && sh + width > 64) __atomic_fetch_or(&words[w + 1], value >> (64 - sh), __ATOMIC_RELAXED);
}

void write_var(std::vector<uint8_t>& out, uint32_t v) {
  while (v >= 128) {
    out.push_back((uint8_t)(v | 128));
    v >>= 7;
  }
  out.push_back((uint8_t)v);
}



}  // namespace

uint64_t next_pow2(uint64_t v) {
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

double seconds_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}

uint64_t config_slots(const BuildOptions& opt, int H, uint64_t cardinality) {
  double needed = std::ceil(std::max<double>((double)cardinality, 1.0) * opt.slot_scale);
  uint64_t s = (uint64_t)needed;
  s = std::max<uint64_t>(s, next_pow2((uint64_t)H));
  s = std::max<uint64_t>(s, opt.segment_length * next_pow2((uint64_t)H));
  return next_pow2(s);
}

void prepare(const BuildOptions& opt, Context& bc) {
  bc.opt = opt;
  bc.t0 = std::chrono::steady_clock::now();
  bc.threads = opt.threads > 0 ? opt.threads : (int)std::thread::hardware_concurrency();
  const int H = bc.H = opt.hashes, b = bc.b = opt.fingerprint_bits;
  FeatureParams& fp = bc.fp;
  fp = opt.features;
  check(H >= 2 && H <= kMaxHashes, kEInval, "invalid hash count");
  check(b == 1 || b == 2 || b == 4 || b == 8 || b == 16 || b == 32, kEInval,
        "fingerprint bits must be 1, 2, 4, 8, 16 or 32");
  check((opt.segment_length & (opt.segment_length - 1)) == 0 && opt.segment_length >= 1 &&
            opt.segment_length <= 4096,
        kEInval, "segment length must be a power of two in 1..=4096");
  check((opt.max_subindex_size & (opt.max_subindex_size - 1)) == 0 && opt.max_subindex_size,
        kEInval, "--max-subindex-size must be a non-zero power of two");
  switch (fp.mode) {
    case 0: case 2: check(fp.k > 0, kEInval, "k must be positive"); break;
    case 1:
      check(fp.k >= 1 && fp.k <= 255 && (fp.k & 1) && fp.m >= 1 && fp.m <= 31 && fp.m <= fp.k,
            kEInval, "invalid minimizer window/length");
      break;
    case 3: check(fp.z < fp.k, kEInval, "--findere-z must be smaller than query k"); break;
    default: raise(kEInval, "invalid index mode");
  }
  if (!fp.seed_pattern.empty()) {
    // SpacedSeed::from_str (src/anchors.rs:15-42), FeatureConfig::validate_anchors
    // (src/lib.rs:177-206).
    check(parse_spaced_seed(fp.seed_pattern.c_str(), &fp.pattern), kEInval,
          "seed pattern must be 1..=31 symmetric '#'/'_' characters with at least one '#'");
    check(fp.mode == 0 || fp.mode == 1, kEInval,
          "spaced seeds and randstrobemers require --index-mode kmers or minimizers");
    check(fp.pattern.width == (fp.mode == 1 ? fp.m : fp.k), kEInval,
          "seed pattern width must match k (or m in minimizer mode)");
    fp.spaced = true;
  }
  if (fp.strobes) {
    // RandstrobeConfig defaults and checks (src/bin/zorindex.rs:471-484,
    // src/anchors.rs:98-110): distances default to the strobe length (k, or
    // m in minimizer mode) and three times it.
    check(fp.mode == 0 || fp.mode == 1, kEInval,
          "spaced seeds and randstrobemers require --index-mode kmers or minimizers");
    const uint64_t length = (uint64_t)(fp.mode == 1 ? fp.m : fp.k);
    if (!fp.strobe_min) fp.strobe_min = length;
    if (!fp.strobe_max) fp.strobe_max = 3 * length;
    check(fp.strobe_min <= fp.strobe_max, kEInval,
          "randstrobemer minimum distance must not exceed maximum distance");
  }
  struct stat st;
  check(stat(opt.output.c_str(), &st) != 0, kEInval,
        ("output " + opt.output + " already exists; choose a new directory").c_str());

  auto& inputs = bc.inputs;
  auto& spec = bc.spec;
  if (!opt.synth.empty()) {
    check(synth::parse_spec(opt.synth, spec), kEInval, "invalid --synth specification");
    for (uint64_t c = 0; c < spec.colors; ++c)
      inputs.push_back(Input{"g" + std::to_string(c), "synthetic:" + opt.synth + ":" + std::to_string(c)});
  } else {
    inputs = read_fof(opt.fof);
  }
  bc.occurrences.assign(inputs.size(), 0);
}

void plan_layout(Context& bc, bool host_rows) {
  // Promotion of undersized size classes.
  const BuildOptions& opt = bc.opt;
  const int H = bc.H;
  auto& groups = bc.groups;
  auto& classes = bc.classes;
  auto& class_order = bc.class_order;
  std::map<uint64_t, std::pair<uint64_t, uint64_t>> sizes;
  for (auto& g : groups) {
    sizes[g.slots].first += g.members.size();
    sizes[g.slots].second += g.width;
  }
  std::vector<uint64_t> bs, bd, bw;
  for (auto& kv : sizes) {
    bs.push_back(kv.first);
    bd.push_back(kv.second.first);
    bw.push_back(kv.second.second);
  }
  std::vector<uint64_t> targets =
      promotion_targets(bs, bd, bw, opt.min_subindex_documents, opt.max_subindexes);
  std::map<uint64_t, uint64_t> promote;
  size_t& promoted = bc.promoted;
  promoted = 0;
  for (size_t i = 0; i < bs.size(); ++i) promote[bs[i]] = targets[i];
  for (auto& g : groups) {
    uint64_t t = promote[g.slots];
    promoted += t > g.slots;
    g.slots = t;
  }

  // Classes (one per final slot count), columns ordered by width then first
  // member (ColumnOrder::Width, storage.rs:1644-1660), hash partitions.
  std::map<uint64_t, size_t> class_of;
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    auto it = class_of.find(groups[gi].slots);
    if (it == class_of.end()) {
      it = class_of.emplace(groups[gi].slots, classes.size()).first;
      classes.emplace_back();
      classes.back().source_slots = groups[gi].slots;
    }
    classes[it->second].groups.push_back(gi);
  }
  // Banks in increasing source-slot order.
  class_order.assign(classes.size(), 0);
  for (size_t i = 0; i < classes.size(); ++i) class_order[i] = i;
  std::sort(class_order.begin(), class_order.end(),
            [&](size_t a, size_t c) { return classes[a].source_slots < classes[c].source_slots; });
  const uint64_t min_local = opt.segment_length * next_pow2((uint64_t)H);
  bool& partitioned = bc.partitioned;
  partitioned = false;
  for (auto& cl : classes) {
    std::sort(cl.groups.begin(), cl.groups.end(), [&](size_t a, size_t c) {
      if (groups[a].width != groups[c].width) return groups[a].width < groups[c].width;
      return groups[a].members[0] < groups[c].members[0];
    });
    uint64_t off = 0;
    for (size_t col = 0; col < cl.groups.size(); ++col) {
      Group& g = groups[cl.groups[col]];
      g.column = col;
      g.offset = off;
      off += g.width;
    }
    cl.row_bits = off;
    uint64_t row_bytes = (off + 7) / 8;
    cl.local_slots = cl.source_slots;
    if ((unsigned __int128)cl.source_slots * row_bytes > opt.max_subindex_size) {
      while ((unsigned __int128)cl.local_slots * row_bytes > opt.max_subindex_size)
        cl.local_slots /= 2;
      check(cl.local_slots >= min_local, kEInval,
            "--max-subindex-size is too small for this row width; raise the cap");
      partitioned = true;
    }
    cl.partitions = cl.source_slots / cl.local_slots;
    if (host_rows) {
      size_t words = (size_t)((cl.local_slots * row_bytes + 7) / 8 + 2);
      cl.rows.assign(cl.partitions, std::vector<uint64_t>(words, 0));
    }
  }
  for (size_t ci = 0; ci < classes.size(); ++ci)
    for (size_t gi : classes[ci].groups) groups[gi].cls = ci;

}

void write_index(Context& bc, const PayloadFn& payload_fn, int payload_threads) {
  const BuildOptions& opt = bc.opt;
  auto& groups = bc.groups;
  auto& classes = bc.classes;
  const FeatureParams& fp = bc.fp;
  const int H = bc.H, b = bc.b;
  const auto t0 = bc.t0;
  const size_t C = bc.inputs.size();
  const auto& inputs = bc.inputs;
  const auto& occurrences = bc.occurrences;
  const bool partitioned = bc.partitioned;
  const size_t promoted = bc.promoted;
  // Staging directory, renamed into place at the end (storage.rs:466-475).
  std::string stage = opt.output + ".building";
  mkdir(stage.c_str(), 0755);
  struct BankOut {
    size_t cls;
    uint64_t partition;
    std::string file;
  };
  std::vector<BankOut> banks;
  for (size_t ci : bc.class_order) {
    const ClassLayout& cl = classes[ci];
    for (uint64_t p = 0; p < cl.partitions; ++p) {
      char name[128];
      if (cl.partitions > 1)
        snprintf(name, sizeof name, "bank-%d-part-%llu-of-%llu.zorbank.zst",
                 ilog2(cl.source_slots), (unsigned long long)p,
                 (unsigned long long)cl.partitions);
      else
        snprintf(name, sizeof name, "bank-%d.zorbank.zst", ilog2(cl.source_slots));
      banks.push_back({ci, p, name});
    }
  }
  parallel_for(banks.size(), payload_threads, [&](size_t bi) {
    const ClassLayout& cl = classes[banks[bi].cls];
    const uint64_t row_bytes = (cl.row_bits + 7) / 8, payload = cl.local_slots * row_bytes;
    FramedWriter w(stage + "/" + banks[bi].file, opt.zstd_level);
    uint8_t header[40];
    memcpy(header, opt.legacy_layout ? "ZORPOW1\0" : "ZORPOW3\0", 8);
    uint64_t fields[4] = {cl.local_slots, cl.row_bits, cl.groups.size(), payload};
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 8; ++j) header[8 + 8 * i + j] = (uint8_t)(fields[i] >> (8 * j));
    w.write(header, 40);
    payload_fn(banks[bi].cls, banks[bi].partition, w);
    w.finish();
  });

  // Recovery map: origins of every abandoned hash, unioned across groups.
  uint64_t hashes = 0, associations = 0;
  if (!opt.drop_abandoned) {
    std::vector<Abandoned>& all = bc.abandoned;
    std::sort(all.begin(), all.end(),
              [](const Abandoned& a, const Abandoned& c) { return a.hash < c.hash; });
    std::vector<uint8_t> out;
    out.insert(out.end(), (const uint8_t*)"ZORABN2\0", (const uint8_t*)"ZORABN2\0" + 8);
    uint32_t prev_hash = 0;
    std::vector<uint32_t> origins;
    for (size_t i = 0; i < all.size();) {
      size_t j = i;
      origins.clear();
      while (j < all.size() && all[j].hash == all[i].hash) {
        const Group& g = groups[all[j].group];
        for (uint64_t mask = all[j].mask; mask; mask &= mask - 1)
          origins.push_back(g.members[__builtin_ctzll(mask)]);
        ++j;
      }
      std::sort(origins.begin(), origins.end());
      origins.erase(std::unique(origins.begin(), origins.end()), origins.end());
      write_var(out, all[i].hash - prev_hash);
      prev_hash = all[i].hash;
      write_var(out, (uint32_t)origins.size());
      uint32_t po = 0;
      for (uint32_t o : origins) {
        write_var(out, o - po);
        po = o;
      }
      ++hashes;
      associations += origins.size();
      i = j;
    }
    write_zstd_file(stage + "/abandoned.zormap.zst", out.data(), out.size(), 3);
  }

  // manifest.json in the field order of the reference's Manifest.
  JsonValue m = JsonValue::object();
  m.set("version", JsonValue::uint(partitioned ? 9 : 8));
  m.set("abandoned_recovery", JsonValue::boolean(!opt.drop_abandoned));
  m.set("abandoned_file", opt.drop_abandoned ? JsonValue::null()
                                             : JsonValue::str("abandoned.zormap.zst"));
  m.set("abandoned_hashes", JsonValue::uint(hashes));
  m.set("abandoned_origins", JsonValue::uint(associations));
  m.set("backend", JsonValue::str("zor"));
  m.set("k", JsonValue::uint((uint64_t)fp.k));
  m.set("hashes", JsonValue::uint((uint64_t)H));
  m.set("segment_length", JsonValue::uint(opt.segment_length));
  m.set("seed", JsonValue::uint(fp.seed));
  m.set("fingerprint_bits", JsonValue::uint((uint64_t)b));
  m.set("index_mode", JsonValue::uint((uint64_t)fp.mode));
  m.set("minimizer_size", JsonValue::uint((uint64_t)fp.m));
  m.set("minimizer_scheme", JsonValue::str("open-closed-mod"));
  m.set("homopolymer_compression", JsonValue::boolean(fp.homopolymer));
  m.set("seed_pattern", fp.spaced ? JsonValue::str(fp.seed_pattern) : JsonValue::null());
  if (fp.strobes) {
    JsonValue rs = JsonValue::object();
    rs.set("min_distance", JsonValue::uint(fp.strobe_min));
    rs.set("max_distance", JsonValue::uint(fp.strobe_max));
    m.set("randstrobemers", rs);
    m.set("randstrobe_scheme", JsonValue::str("strobealign-popcount8-symmetric64-downstream-v1"));
  } else {
    m.set("randstrobemers", JsonValue::null());
    m.set("randstrobe_scheme", JsonValue::null());
  }
  m.set("modimizer_sampling", JsonValue::uint(fp.sampling));
  m.set("findere_z", JsonValue::uint((uint64_t)fp.z));
  m.set("sketch_size", JsonValue::uint(128));
  m.set("sketch_method", JsonValue::str("none: explicit groups or singletons"));
  m.set("merge_planner", JsonValue::str("naive"));
  m.set("column_order", JsonValue::str("width"));
  m.set("column_order_method", JsonValue::str("width-then-dataset-id-v1"));
  m.set("planning_pair_evaluations", JsonValue::uint(0));
  m.set("planning_possible_pair_evaluations", JsonValue::uint(0));
  m.set("merge_reverts_enabled", JsonValue::boolean(false));
  m.set("construction_cell_storage", JsonValue::str("two-pass-memory-packed-no-scratch"));
  m.set("construction_abandoned_storage",
        JsonValue::str(opt.drop_abandoned ? "omitted" : "memory"));
  m.set("slot_scale", JsonValue::real(opt.slot_scale));
  m.set("min_subindex_documents", JsonValue::uint(opt.min_subindex_documents));
  if (opt.max_subindexes >= 0) m.set("max_subindexes", JsonValue::uint((uint64_t)opt.max_subindexes));
  m.set("max_subindex_size", JsonValue::uint(opt.max_subindex_size));
  m.set("promoted_groups", JsonValue::uint(promoted));
  uint64_t logical = 0;
  for (auto& g : groups) logical += g.slots * g.width;
  m.set("singleton_logical_bits", JsonValue::uint(logical));
  m.set("predicted_logical_bits", JsonValue::uint(logical));
  m.set("planned_groups", JsonValue::uint(groups.size()));
  m.set("rejected_groups", JsonValue::uint(0));
  m.set("overflow_groups", JsonValue::uint(0));
  uint64_t verified = 0;
  for (auto& g : groups) verified += g.cardinality - (opt.drop_abandoned ? g.abandoned : 0);
  m.set("exact_group_verifications", JsonValue::uint(verified));
  m.set("sketch_seconds", JsonValue::real(0.0));
  m.set("plan_seconds", JsonValue::real(0.0));
  m.set("build_seconds", JsonValue::real(seconds_since(t0)));
  m.set("input_document_count", JsonValue::uint(C));
  JsonValue colors = JsonValue::array();
  for (size_t c = 0; c < C; ++c) {
    JsonValue col = JsonValue::object();
    col.set("name", JsonValue::str(inputs[c].name));
    col.set("path", JsonValue::str(inputs[c].path));
    col.set("occurrences", JsonValue::uint(occurrences[c]));
    uint64_t unique = 0;
    for (auto& g : groups)
      if (g.members.size() == 1 && g.members[0] == c) unique = g.cardinality;
    col.set("unique_kmers", JsonValue::uint(unique));
    colors.arr.push_back(std::move(col));
  }
  // unique_kmers of grouped datasets: distinct keys carrying their bit.
  for (auto& g : groups)
    if (g.members.size() > 1)
      for (size_t i = 0; i < g.members.size(); ++i) {
        uint64_t n = 0;
        for (uint64_t mask : g.masks) n += (mask >> i) & 1;
        colors.arr[g.members[i]].obj[3].second = JsonValue::uint(n);
      }
  m.set("colors", std::move(colors));
  JsonValue bank_list = JsonValue::array();
  for (auto& bo : banks) {
    const ClassLayout& cl = classes[bo.cls];
    JsonValue bj = JsonValue::object();
    bj.set("file", JsonValue::str(bo.file));
    bj.set("slots", JsonValue::uint(cl.local_slots));
    bj.set("row_bits", JsonValue::uint(cl.row_bits));
    JsonValue gl = JsonValue::array();
    for (size_t gi : cl.groups) {
      const Group& g = groups[gi];
      JsonValue gj = JsonValue::object();
      JsonValue mem = JsonValue::array();
      for (uint32_t c : g.members) mem.arr.push_back(JsonValue::uint(c));
      gj.set("members", std::move(mem));
      gj.set("width", JsonValue::uint(g.width));
      gj.set("offset", JsonValue::uint(g.offset));
      gj.set("union_cardinality", JsonValue::uint(g.cardinality));
      gj.set("fallback_keys", JsonValue::uint(opt.drop_abandoned ? 0 : g.abandoned));
      gj.set("abandoned_keys", JsonValue::uint(g.abandoned));
      gl.arr.push_back(std::move(gj));
    }
    bj.set("groups", std::move(gl));
    bj.set("fingerprint_first", JsonValue::boolean(!opt.legacy_layout));
    if (cl.partitions > 1) {
      JsonValue rt = JsonValue::object();
      rt.set("source_slots", JsonValue::uint(cl.source_slots));
      rt.set("partition", JsonValue::uint(bo.partition));
      rt.set("partitions", JsonValue::uint(cl.partitions));
      bj.set("routing", std::move(rt));
    }
    bank_list.arr.push_back(std::move(bj));
  }
  m.set("banks", std::move(bank_list));
  std::string text = json_write_pretty(m);
  write_file_bytes(stage + "/manifest.json", text.data(), text.size());
  check(rename(stage.c_str(), opt.output.c_str()) == 0, kEIo, "cannot move the built index into place");
  if (!opt.quiet) {
    uint64_t abandoned = 0, bytes = 0;
    for (auto& g : groups) abandoned += g.abandoned;
    for (auto& bo : banks)
      bytes += classes[bo.cls].local_slots * ((classes[bo.cls].row_bits + 7) / 8);
    fprintf(stderr,
            "built %s in %.3fs: banks=%zu, groups=%zu, stack_bytes=%llu, abandoned_keys=%llu, "
            "abandoned_hashes=%llu\n",
            opt.output.c_str(), seconds_since(t0), banks.size(), groups.size(),
            (unsigned long long)bytes, (unsigned long long)abandoned, (unsigned long long)hashes);
  }
}

}  // namespace build

std::vector<uint64_t> promotion_targets(const std::vector<uint64_t>& slots,
                                        const std::vector<uint64_t>& docs,
                                        const std::vector<uint64_t>& widths, uint64_t minimum,
                                        int64_t maximum) {
  const size_t n = slots.size();
  bool all_big = true;
  for (uint64_t d : docs) all_big &= d >= minimum;
  if ((minimum == 1 || all_big) && (maximum < 0 || (int64_t)n <= maximum)) return slots;
  uint64_t total = 0;
  for (uint64_t d : docs) total += d;
  minimum = std::min(minimum, total);
  using Cost = unsigned __int128;
  auto bank_cost = [&](size_t end, uint64_t width) {
    return (Cost)slots[end - 1] * (Cost)((width + 7) / 8) * 8;
  };
  std::vector<uint64_t> targets(n, 0);
  if (maximum >= 0 && (int64_t)n > maximum) {
    size_t limit = (size_t)maximum;
    struct Cell {
      bool ok = false;
      Cost cost = 0;
      size_t start = 0;
    };
    std::vector<std::vector<Cell>> best(limit + 1, std::vector<Cell>(n + 1));
    best[0][0] = Cell{true, 0, 0};
    for (size_t count = 1; count <= limit; ++count)
      for (size_t end = count; end <= n; ++end) {
        uint64_t d = 0, w = 0;
        for (size_t s = end; s-- > 0;) {
          d += docs[s];
          w += widths[s];
          if (d < minimum || !best[count - 1][s].ok) continue;
          Cost c = best[count - 1][s].cost + bank_cost(end, w);
          Cell& cur = best[count][end];
          if (!cur.ok || c < cur.cost || (c == cur.cost && s < cur.start)) cur = Cell{true, c, s};
        }
      }
    size_t count = 0;
    Cost bestc = 0;
    for (size_t c = 1; c <= limit; ++c)
      if (best[c][n].ok && (!count || best[c][n].cost < bestc)) {
        count = c;
        bestc = best[c][n].cost;
      }
    check(count > 0, kEInval, "no feasible bounded subindex layout");
    for (size_t end = n; end > 0; --count) {
      size_t s = best[count][end].start;
      for (size_t i = s; i < end; ++i) targets[i] = slots[end - 1];
      end = s;
    }
    return targets;
  }
  struct Cell {
    bool ok = false;
    Cost cost = 0;
    uint64_t banks = 0;
    size_t start = 0;
  };
  std::vector<Cell> best(n + 1);
  best[0] = Cell{true, 0, 0, 0};
  for (size_t end = 1; end <= n; ++end) {
    uint64_t d = 0, w = 0;
    for (size_t s = end; s-- > 0;) {
      d += docs[s];
      w += widths[s];
      if (d < minimum || !best[s].ok) continue;
      Cell cand{true, best[s].cost + bank_cost(end, w), best[s].banks + 1, s};
      Cell& cur = best[end];
      bool better = !cur.ok || cand.cost < cur.cost ||
                    (cand.cost == cur.cost &&
                     (cand.banks < cur.banks || (cand.banks == cur.banks && s < cur.start)));
      if (better) cur = cand;
    }
  }
  for (size_t end = n; end > 0;) {
    check(best[end].ok, kEInval, "no feasible minimum-document layout");
    size_t s = best[end].start;
    for (size_t i = s; i < end; ++i) targets[i] = slots[end - 1];
    end = s;
  }
  return targets;
}

// Programs linked without device_builder.cu (the zorindex command line) get
// this definition; zx_build links the device builder's.
__attribute__((weak)) void build_index_device(const BuildOptions&) {
  raise(kEUnsupported, "this program was built without the device builder: use zx_build --device");
}

void build_index(const BuildOptions& opt) {
  if (opt.device) {
    build_index_device(opt);
    return;
  }
  using namespace build;
  Context bc;
  prepare(opt, bc);
  const auto t0 = bc.t0;
  const int threads = bc.threads;
  const int H = bc.H, b = bc.b;
  const FeatureParams& fp = bc.fp;
  const auto& inputs = bc.inputs;
  const auto& spec = bc.spec;
  auto& occurrences = bc.occurrences;
  const size_t C = inputs.size();
  std::vector<std::vector<uint64_t>> keys(C);
  parallel_for(C, threads, [&](size_t c) {
    std::vector<uint64_t> k;
    if (!opt.synth.empty()) {
      std::vector<uint8_t> g;
      synth::genome(spec, c, g);
      cpu::sequence_features(g.data(), g.size(), fp, k);
    } else {
      RecordBatch rb = read_fastx(inputs[c].path, false);
      for (size_t r = 0; r < rb.records(); ++r)
        cpu::sequence_features(rb.bases.data() + rb.offsets[r], rb.offsets[r + 1] - rb.offsets[r],
                               fp, k);
    }
    occurrences[c] = k.size();
    std::sort(k.begin(), k.end());
    k.erase(std::unique(k.begin(), k.end()), k.end());
    keys[c] = std::move(k);
  });
  if (!opt.quiet) fprintf(stderr, "extracted %zu datasets in %.3fs\n", C, seconds_since(t0));

  // Groups: explicit multi-member groups, singletons for everything else.
  auto& groups = bc.groups;
  std::vector<int> grouped(C, 0);
  if (!opt.groups.empty()) {
    std::stringstream ss(opt.groups);
    std::string part;
    while (std::getline(ss, part, ';')) {
      Group g;
      std::stringstream ps(part);
      std::string id;
      while (std::getline(ps, id, ',')) {
        size_t c = std::stoul(id);
        check(c < C && !grouped[c], kEInval, "invalid or repeated dataset in --groups");
        grouped[c] = 1;
        g.members.push_back((uint32_t)c);
      }
      std::sort(g.members.begin(), g.members.end());
      check(!g.members.empty() && g.members.size() <= (size_t)(64 - b), kEInval,
            "invalid group size");
      groups.push_back(std::move(g));
    }
  }
  for (size_t c = 0; c < C; ++c)
    if (!grouped[c]) {
      Group g;
      g.members.push_back((uint32_t)c);
      groups.push_back(std::move(g));
    }
  const uint64_t fp_mask = (1ull << b) - 1;
  parallel_for(groups.size(), threads, [&](size_t gi) {
    Group& g = groups[gi];
    g.width = (uint64_t)b + (g.members.size() == 1 ? 0 : g.members.size());
    if (g.members.size() == 1) {
      g.keys = std::move(keys[g.members[0]]);  // singleton: no membership masks
    } else {
      std::vector<std::pair<uint64_t, uint64_t>> all;
      for (size_t i = 0; i < g.members.size(); ++i)
        for (uint64_t key : keys[g.members[i]]) all.emplace_back(key, 1ull << i);
      std::sort(all.begin(), all.end());
      for (size_t i = 0; i < all.size();) {
        size_t j = i;
        uint64_t mask = 0;
        while (j < all.size() && all[j].first == all[i].first) mask |= all[j++].second;
        g.keys.push_back(all[i].first);
        g.masks.push_back(mask);
        i = j;
      }
    }
    g.cardinality = g.keys.size();
    g.slots = config_slots(opt, H, g.cardinality);
  });
  for (auto& k : keys) std::vector<uint64_t>().swap(k);

  plan_layout(bc, true);
  auto& classes = bc.classes;
  // Construction jobs: one per (group, partition).
  struct Job {
    size_t group;
    uint64_t partition;
  };
  std::vector<Job> jobs;
  for (size_t gi = 0; gi < groups.size(); ++gi)
    for (uint64_t p = 0; p < classes[groups[gi].cls].partitions; ++p) jobs.push_back({gi, p});
  std::vector<std::vector<Abandoned>> dropped(jobs.size());
  std::vector<uint64_t> dropped_count(jobs.size(), 0);
  // Largest filters first for load balance.
  std::sort(jobs.begin(), jobs.end(), [&](const Job& a, const Job& c) {
    return groups[a.group].cardinality > groups[c.group].cardinality;
  });
  parallel_for(jobs.size(), threads, [&](size_t ji) {
    const Job& job = jobs[ji];
    Group& g = groups[job.group];
    ClassLayout& cl = classes[g.cls];
    std::vector<uint64_t> k, v;
    for (size_t i = 0; i < g.keys.size(); ++i) {
      if (cl.partitions > 1 &&
          partition_id(g.keys[i], fp.seed, (uint32_t)cl.partitions) != job.partition)
        continue;
      k.push_back(g.keys[i]);
      v.push_back(fingerprint(g.keys[i], fp.seed, b) |
                  (g.members.size() == 1 ? 0 : g.masks[i] << b));
    }
    std::vector<uint64_t> cells;
    std::vector<uint32_t> lost =
        construct_filter(k, v, cl.local_slots, H, opt.segment_length, fp.seed, cells);
    dropped_count[ji] = lost.size();
    if (!opt.drop_abandoned)
      for (uint32_t e : lost)
        dropped[ji].push_back(Abandoned{recovery_hash(k[e], fp.seed), (uint32_t)job.group,
                                        g.members.size() == 1 ? 1 : v[e] >> b});
    // Fingerprint-first packing into this partition's rows (legacy: the
    // group's whole field, fingerprint in its low bits, at its offset).
    const uint64_t G = cl.groups.size(), row_bytes = (cl.row_bits + 7) / 8;
    const uint64_t mem_off = G * (uint64_t)b + g.offset - g.column * (uint64_t)b;
    uint64_t* words = cl.rows[job.partition].data();
    for (uint64_t s = 0; s < cl.local_slots; ++s) {
      uint64_t cell = cells[s];
      if (!cell) continue;
      uint64_t base = s * row_bytes * 8;
      if (opt.legacy_layout) {
        or_bits(words, base + g.offset, (uint64_t)b, cell & fp_mask);
        if (g.width > (uint64_t)b) or_bits(words, base + g.offset + b, g.width - b, cell >> b);
        continue;
      }
      or_bits(words, base + g.column * (uint64_t)b, (uint64_t)b, cell & fp_mask);
      if (g.width > (uint64_t)b) or_bits(words, base + mem_off, g.width - b, cell >> b);
    }
  });
  for (size_t ji = 0; ji < jobs.size(); ++ji) groups[jobs[ji].group].abandoned += dropped_count[ji];
  if (!opt.quiet) fprintf(stderr, "constructed %zu filters in %.3fs\n", jobs.size(), seconds_since(t0));

  for (auto& d : dropped) bc.abandoned.insert(bc.abandoned.end(), d.begin(), d.end());

  write_index(
      bc,
      [&](size_t ci, uint64_t part, FramedWriter& w) {
        const ClassLayout& cl = classes[ci];
        w.write(cl.rows[part].data(), cl.local_slots * ((cl.row_bits + 7) / 8));
      },
      threads);
}

}  // namespace zx
