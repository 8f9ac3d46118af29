#include "manifest.h"

#include <algorithm>
#include <cstdio>
#include <fstream>
#include <map>
#include <set>
#include <sstream>

#include "../zx_hash.h"
#include "error.h"

namespace zx {

const char* index_mode_label(int mode) {
  switch (mode) {
    case kKmers: return "kmers";
    case kMinimizers: return "minimizers";
    case kModimizers: return "modimizers";
    case kFindere: return "findere";
    default: return "unknown";
  }
}

static int ilog2(uint64_t v) { return 63 - __builtin_clzll(v); }
static bool is_pow2(uint64_t v) { return v && !(v & (v - 1)); }

// BankMeta::expected_filename / filename (storage.rs:104-130).
std::string BankMeta::expected_filename() const {
  char buf[128];
  if (routed)
    snprintf(buf, sizeof buf, "bank-%d-part-%llu-of-%llu.zorbank.zst", ilog2(source_slots),
             (unsigned long long)partition, (unsigned long long)partitions);
  else
    snprintf(buf, sizeof buf, "bank-%d.zorbank.zst", ilog2(slots));
  std::string name = buf;
  if (component != 0) name = "component-" + std::to_string(component) + "-" + name;
  return name;
}

uint64_t Manifest::segment_for(uint64_t slots) const {
  return has_segment_length ? segment_length : legacy_segment_length(slots, hashes);
}

namespace {

const JsonValue& need(const JsonValue& o, const char* key) {
  const JsonValue* v = o.find(key);
  if (!v) raise(kEFormat, std::string("manifest: missing field ") + key);
  return *v;
}
uint64_t as_u64(const JsonValue& v, const char* what) {
  if (v.kind != JsonValue::Int || v.neg) raise(kEFormat, std::string("manifest: ") + what);
  return v.u;
}
uint64_t u64_field(const JsonValue& o, const char* key) { return as_u64(need(o, key), key); }
uint64_t u64_or(const JsonValue& o, const char* key, uint64_t dflt) {
  const JsonValue* v = o.find(key);
  return (v && !v->is_null()) ? as_u64(*v, key) : dflt;
}
bool bool_or(const JsonValue& o, const char* key, bool dflt) {
  const JsonValue* v = o.find(key);
  if (!v || v->is_null()) return dflt;
  if (v->kind != JsonValue::Bool) raise(kEFormat, std::string("manifest: ") + key);
  return v->b;
}
std::string str_field(const JsonValue& o, const char* key) {
  const JsonValue& v = need(o, key);
  if (v.kind != JsonValue::Str) raise(kEFormat, std::string("manifest: ") + key);
  return v.s;
}

}  // namespace

void validate_manifest(Manifest& m) {
  check_format(m.version >= 1 && m.version <= 10, "unsupported power-of-two index format");
  check(m.version >= 2, kEUnsupported,
        "index format version 1 (embedded legacy recovery records) is not supported; rebuild");
  check_format(m.hashes >= 2 && m.hashes <= kMaxHashes, "invalid hash count");
  if (m.version >= 9) {
    check_format(!m.has_segment_length ||
                     (is_pow2(m.segment_length) && m.segment_length <= 4096),
                 "invalid/missing segment length for index version");
  } else if (m.version == 8) {
    check_format(m.has_segment_length && is_pow2(m.segment_length) && m.segment_length <= 4096,
                 "invalid/missing segment length for index version");
  } else {
    check_format(!m.has_segment_length, "invalid/missing segment length for index version");
  }
  int b = m.fingerprint_bits;
  check_format(b == 1 || b == 2 || b == 4 || b == 8 || b == 16 || b == 32,
               "invalid fingerprint width");
  check_format(m.colors.size() <= 0xFFFFFFFFull, "dataset IDs must fit in 32 bits");
  check_format(m.abandoned_recovery == m.has_abandoned_file,
               "inconsistent abandoned recovery metadata");
  check_format(m.abandoned_recovery || (m.abandoned_hashes == 0 && m.abandoned_origins == 0),
               "disabled recovery has abandoned records");
  if (m.has_randstrobemers) {
    // Manifest::features (storage.rs:240-256), RandstrobeConfig::validate
    // (anchors.rs:98-110), FeatureConfig::validate_anchors (lib.rs:177-206).
    check_format(m.version >= 6 &&
                     m.randstrobe_scheme == "strobealign-popcount8-symmetric64-downstream-v1",
                 "unsupported legacy/custom randstrobemer extraction; rebuild this index with the "
                 "current downstream scheme");
    check_format(m.index_mode == kKmers || m.index_mode == kMinimizers,
                 "spaced seeds and randstrobemers require --index-mode kmers or minimizers");
    check_format(m.strobe_min > 0, "randstrobemer minimum distance must be greater than zero");
    check_format(m.strobe_min <= m.strobe_max,
                 "randstrobemer minimum distance must not exceed maximum distance");
  }
  if (m.has_seed_pattern) {
    // FeatureConfig::validate_anchors (src/lib.rs:177-206) and SpacedSeed::from_str
    // (src/anchors.rs:15-42).
    SpacedSeed sp;
    check_format(parse_spaced_seed(m.seed_pattern.c_str(), &sp),
                 "seed pattern must be 1..=31 symmetric '#'/'_' characters with at least one '#'");
    check_format(m.index_mode == kKmers || m.index_mode == kMinimizers,
                 "spaced seeds and randstrobemers require --index-mode kmers or minimizers");
    const uint64_t length = m.index_mode == kMinimizers ? m.minimizer_size : m.k;
    check_format((uint64_t)sp.width == length,
                 "seed pattern width must match k (or m in minimizer mode)");
  }
  switch (m.index_mode) {
    case kFindere:
      check_format(m.k > 0 && m.findere_z < m.k, "--findere-z must be smaller than query k");
      break;
    case kKmers:
    case kModimizers:
      check_format(m.k > 0, "invalid k");
      break;
    case kMinimizers:
      check_format(m.k >= 1 && m.k <= 255 && (m.k & 1) && m.minimizer_size <= m.k,
                   "invalid minimizer window");
      check(m.minimizer_scheme == 1, kEUnsupported,
            "the simd minimizer scheme (third-party simd-minimizers) is not supported; use "
            "open-closed-mod");
      break;
    default:
      raise(kEFormat, "unsupported index mode");
  }
  check_format(m.minimizer_size >= 1 && m.minimizer_size <= 31 && m.modimizer_sampling > 0,
               "invalid feature parameters");

  const size_t C = m.colors.size();
  std::vector<int> seen_class(C, -1);
  std::vector<std::pair<size_t, size_t>> first_group(C, {SIZE_MAX, 0});
  m.classes.clear();
  std::pair<uint64_t, uint64_t> previous{0, 0};
  uint64_t next_partition = 0, partition_count = 1;
  size_t first_class_bank = 0;
  for (size_t id = 0; id < m.banks.size(); ++id) {
    BankMeta& bank = m.banks[id];
    check_format(bank.component == 0 || m.version >= 10, "unsupported index component");
    check_format(!bank.fingerprint_first || m.version >= 3, "unsupported bank layout");
    if (!bank.routed) bank.source_slots = bank.slots;
    check_format(is_pow2(bank.slots) && bank.slots >= (uint64_t)m.hashes &&
                     is_pow2(bank.source_slots),
                 "invalid bank size/order");
    uint64_t partition = bank.routed ? bank.partition : 0;
    uint64_t partitions = bank.routed ? bank.partitions : 1;
    check_format(!bank.routed || (m.version >= 9 && partitions > 1 && is_pow2(partitions) &&
                                  bank.slots * partitions == bank.source_slots),
                 "invalid hash partition geometry");
    std::pair<uint64_t, uint64_t> group{bank.component, bank.source_slots};
    if (group != previous) {
      check_format(group > previous && (previous == std::make_pair<uint64_t, uint64_t>(0, 0) ||
                                        next_partition == partition_count),
                   "invalid/incomplete partition order");
      previous = group;
      next_partition = 0;
      partition_count = partitions;
      first_class_bank = id;
      m.classes.emplace_back();
    }
    check_format(partitions == partition_count && partition == next_partition &&
                     partition < partitions,
                 "invalid/duplicate/missing hash partition");
    ++next_partition;
    m.classes.back().push_back(id);
    if (m.has_segment_length)
      check_format(bank.slots % m.segment_length == 0 &&
                       bank.slots / m.segment_length >= (uint64_t)m.hashes,
                   "subindex too small for fixed segment geometry");
    check_format(bank.file == bank.expected_filename(), "invalid bank file name");
    uint64_t offset = 0;
    std::set<uint32_t> local;
    for (size_t g = 0; g < bank.groups.size(); ++g) {
      GroupMeta& gm = bank.groups[g];
      check_format(!gm.members.empty() && gm.members.size() <= (size_t)(64 - b),
                   "invalid membership width");
      uint64_t width = (uint64_t)b + (gm.members.size() == 1 ? 0 : gm.members.size());
      check_format(gm.offset == offset && gm.width == width, "invalid group bit layout");
      offset += width;
      for (uint32_t c : gm.members) {
        check_format(c < C && local.insert(c).second &&
                         (seen_class[c] < 0 || seen_class[c] == (int)(m.classes.size() - 1)),
                     "invalid/duplicate dataset mapping");
        if (partition == 0) {
          seen_class[c] = (int)(m.classes.size() - 1);
          first_group[c] = {id, g};
        } else {
          check_format(first_group[c].first != SIZE_MAX, "missing partition dataset");
          const auto& fg = m.banks[first_group[c].first].groups[first_group[c].second];
          check_format(fg.members == gm.members, "inconsistent partition dataset mapping");
        }
      }
      check_format(gm.fallback_keys <= gm.union_cardinality, "invalid fallback count");
      check_format(gm.has_abandoned, "missing abandoned equation count");
      check_format(gm.abandoned_keys <= gm.union_cardinality,
                   "invalid abandoned equation count");
      check_format(gm.fallback_keys == (m.abandoned_recovery ? gm.abandoned_keys : 0),
                   "inconsistent abandoned equation count");
    }
    check_format(offset == bank.row_bits && offset > 0, "invalid row width");
    if (partition > 0) {
      const BankMeta& first = m.banks[first_class_bank];
      size_t members = 0;
      for (auto& gm : first.groups) members += gm.members.size();
      check_format(first.row_bits == bank.row_bits && first.groups.size() == bank.groups.size() &&
                       local.size() == members,
                   "incomplete partition dataset mapping");
    }
  }
  bool all_seen = std::all_of(seen_class.begin(), seen_class.end(), [](int v) { return v >= 0; });
  check_format(!m.banks.empty() && all_seen && next_partition == partition_count,
               "incomplete dataset mapping");
}

Manifest load_manifest(const std::string& dir) {
  std::ifstream in(dir + "/manifest.json", std::ios::binary);
  if (!in) raise(kEIo, "cannot open " + dir + "/manifest.json");
  std::stringstream ss;
  ss << in.rdbuf();
  JsonValue j = json_parse(ss.str());
  check_format(j.kind == JsonValue::Obj, "manifest: not a JSON object");
  Manifest m;
  m.version = (uint32_t)u64_field(j, "version");
  check_format(str_field(j, "backend") == "zor", "unsupported power-of-two index format");
  m.abandoned_recovery = bool_or(j, "abandoned_recovery", true);
  const JsonValue* af = j.find("abandoned_file");
  m.has_abandoned_file = af && !af->is_null();
  if (m.has_abandoned_file)
    check_format(af->kind == JsonValue::Str && af->s == "abandoned.zormap.zst",
                 "invalid abandoned map filename");
  m.abandoned_hashes = u64_or(j, "abandoned_hashes", 0);
  m.abandoned_origins = u64_or(j, "abandoned_origins", 0);
  m.k = u64_field(j, "k");
  m.hashes = (int)u64_field(j, "hashes");
  const JsonValue* sl = j.find("segment_length");
  m.has_segment_length = sl && !sl->is_null();
  if (m.has_segment_length) m.segment_length = as_u64(*sl, "segment_length");
  m.seed = u64_field(j, "seed");
  m.fingerprint_bits = (int)u64_field(j, "fingerprint_bits");
  m.index_mode = (int)u64_field(j, "index_mode");
  m.minimizer_size = u64_field(j, "minimizer_size");
  const JsonValue* sch = j.find("minimizer_scheme");
  m.minimizer_scheme = 0;
  if (sch && !sch->is_null()) {
    check_format(sch->kind == JsonValue::Str && (sch->s == "simd" || sch->s == "open-closed-mod"),
                 "manifest: minimizer_scheme");
    m.minimizer_scheme = sch->s == "open-closed-mod" ? 1 : 0;
  }
  m.homopolymer_compression = bool_or(j, "homopolymer_compression", false);
  const JsonValue* sp = j.find("seed_pattern");
  m.has_seed_pattern = sp && !sp->is_null();
  if (m.has_seed_pattern) {
    check_format(sp->kind == JsonValue::Str, "manifest: seed_pattern");
    m.seed_pattern = sp->s;
  }
  const JsonValue* rs = j.find("randstrobemers");
  m.has_randstrobemers = rs && !rs->is_null();
  if (m.has_randstrobemers) {
    m.strobe_min = u64_field(*rs, "min_distance");
    m.strobe_max = u64_field(*rs, "max_distance");
    const JsonValue* sch = j.find("randstrobe_scheme");
    if (sch && sch->kind == JsonValue::Str) m.randstrobe_scheme = sch->s;
  }
  m.modimizer_sampling = u64_field(j, "modimizer_sampling");
  m.findere_z = u64_field(j, "findere_z");
  for (auto& c : need(j, "colors").arr) {
    ColorMeta cm;
    cm.name = str_field(c, "name");
    const JsonValue* p = c.find("path");
    if (p && p->kind == JsonValue::Str) cm.path = p->s;
    cm.occurrences = u64_or(c, "occurrences", 0);
    cm.unique_kmers = u64_field(c, "unique_kmers");
    m.colors.push_back(std::move(cm));
  }
  for (auto& bj : need(j, "banks").arr) {
    BankMeta b;
    b.component = u64_or(bj, "component", 0);
    b.file = str_field(bj, "file");
    b.slots = u64_field(bj, "slots");
    b.row_bits = u64_field(bj, "row_bits");
    b.fingerprint_first = bool_or(bj, "fingerprint_first", false);
    const JsonValue* rt = bj.find("routing");
    if (rt && !rt->is_null()) {
      b.routed = true;
      b.source_slots = u64_field(*rt, "source_slots");
      b.partition = u64_field(*rt, "partition");
      b.partitions = u64_field(*rt, "partitions");
    }
    for (auto& gj : need(bj, "groups").arr) {
      GroupMeta g;
      for (auto& mm : need(gj, "members").arr) {
        uint64_t id = as_u64(mm, "members");
        check_format(id <= 0xFFFFFFFFull, "dataset IDs must fit in 32 bits");
        g.members.push_back((uint32_t)id);
      }
      g.width = u64_field(gj, "width");
      g.offset = u64_field(gj, "offset");
      g.union_cardinality = u64_field(gj, "union_cardinality");
      g.fallback_keys = u64_field(gj, "fallback_keys");
      const JsonValue* ak = gj.find("abandoned_keys");
      g.has_abandoned = ak && !ak->is_null();
      if (g.has_abandoned) g.abandoned_keys = as_u64(*ak, "abandoned_keys");
      b.groups.push_back(std::move(g));
    }
    m.banks.push_back(std::move(b));
  }
  validate_manifest(m);
  return m;
}

}  // namespace zx
