// CPU seed extraction used by the index builder (construction runs on the
// host, as the reference builder does). The query path never calls this: it
// extracts seeds with the sm_100a kernels in kernels/seeds.cuh.
//
// Semantics follow scan_index_features (src/lib.rs:574-642): canonical k-mers
// (645-681), k > 32 polynomial hashes (683-731), open-closed mod-minimizers
// (utils/ocm-minimizers/src/implementation.rs:108-236), modimizers (796-806),
// findere s-mers (632-640) and homopolymer compression (211-222).
#pragma once
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../zx_hash.h"

namespace zx {

struct FeatureParams {
  int mode = 0;  // 0 kmers, 1 minimizers (open-closed mod), 2 modimizers, 3 findere
  int k = 31, m = 21;
  uint64_t seed = 69, sampling = 16;
  int z = 10;
  bool homopolymer = false;
  // Spaced seed (k-mer and minimizer modes): the selected canonical keys are
  // mapped through the pattern (src/anchors.rs:265-281).
  std::string seed_pattern;
  bool spaced = false;
  SpacedSeed pattern;
  // Randstrobemers (src/anchors.rs:92-110, 182-347): each candidate seed is
  // linked to a partner starting strobe_min..strobe_max bases downstream.
  bool strobes = false;
  uint64_t strobe_min = 0, strobe_max = 0;
};

namespace cpu {

inline void kmers_short(const uint8_t* s, size_t n, int k, std::vector<uint64_t>& out) {
  const uint64_t mask = k == 32 ? ~0ull : ((1ull << (2 * k)) - 1);
  const int shift = 2 * (k - 1);
  uint64_t f = 0, r = 0;
  int seen = 0;
  for (size_t i = 0; i < n; ++i) {
    uint32_t c = encode_base(s[i]);
    if (c > 3) {
      f = r = 0;
      seen = 0;
      continue;
    }
    f = ((f << 2) | c) & mask;
    r = (r >> 2) | ((uint64_t)(c ^ 3) << shift);
    if (++seen >= k) out.push_back(f < r ? f : r);
  }
}

// Direct (non-rolling) evaluation of both strand polynomials at each valid
// window start, rolled forward with B^(k-1) and B^-1.
inline void kmers_long(const uint8_t* s, size_t n, int k, std::vector<uint64_t>& out) {
  const LongKmerConsts kc = long_kmer_consts(k);
  size_t i = 0;
  while (i < n) {
    while (i < n && encode_base(s[i]) > 3) ++i;
    size_t j = i;
    while (j < n && encode_base(s[j]) <= 3) ++j;
    if (j - i >= (size_t)k) {
      uint64_t f = 0, r = 0, w = 1;
      for (int q = 0; q < k; ++q) {
        uint32_t c = encode_base(s[i + q]);
        f = f * kLongKmerBase + (c + 1);
        r += (4 - c) * w;
        w *= kLongKmerBase;
      }
      out.push_back(splitmix64((f < r ? f : r) ^ kc.domain));
      for (size_t p = i + k; p < j; ++p) {
        uint64_t o = encode_base(s[p - k]), c = encode_base(s[p]);
        f = (f - (o + 1) * kc.power) * kLongKmerBase + (c + 1);
        r = (r - (4 - o)) * kc.inverse + (4 - c) * kc.power;
        out.push_back(splitmix64((f < r ? f : r) ^ kc.domain));
      }
    }
    i = j;
  }
}

inline void kmers(const uint8_t* s, size_t n, int k, std::vector<uint64_t>& out) {
  if (k <= 0 || n < (size_t)k) return;
  if (k <= 32) kmers_short(s, n, k, out);
  else kmers_long(s, n, k, out);
}

struct AnchorRank {
  uint64_t hash;
  uint32_t cls, left, right;
};
inline bool rank_less(const AnchorRank& a, const AnchorRank& b) {
  return a.cls != b.cls ? a.cls < b.cls : a.hash < b.hash;
}
inline bool rank_equal(const AnchorRank& a, const AnchorRank& b) {
  return a.cls == b.cls && a.hash == b.hash;
}
// a lies to the left of b.
inline AnchorRank rank_combine(const AnchorRank& a, const AnchorRank& b) {
  if (rank_less(a, b)) return a;
  if (rank_less(b, a)) return b;
  AnchorRank r = a;
  r.right = b.right;
  return r;
}

// Open-closed mod-minimizers of one all-ACGT run (n >= k).
// positions (optional) receives the run offset of each emitted minimizer.
inline void ocm_run(const uint8_t* s, size_t n, int k, int m, uint64_t seed,
                    std::vector<uint64_t>& out, std::vector<uint64_t>* positions = nullptr) {
  auto canon = [&](size_t p, int len) {
    uint64_t v = 0;
    for (int q = 0; q < len; ++q) v = (v << 2) | encode_base(s[p + q]);
    return canonical_encoded(v, len);
  };
  if (k == m) {
    for (size_t p = 0; p + m <= n; ++p) {
      out.push_back(canon(p, m));
      if (positions) positions->push_back(p);
    }
    return;
  }
  const OcmParams g = ocm_params(k, m);
  const size_t W = (size_t)(k - g.t + 1);  // anchors per window
  const size_t anchors = n - g.t + 1;
  std::vector<uint64_t> inner(n - g.s + 1);
  for (size_t p = 0; p < inner.size(); ++p) inner[p] = mixsplit(canon(p, g.s), seed ^ kInnerHashSeed);
  std::vector<AnchorRank> rank(anchors);
  for (size_t p = 0; p < anchors; ++p) {
    uint64_t lo = ~0ull;
    for (int q = 0; q <= g.t - g.s; ++q) lo = inner[p + q] < lo ? inner[p + q] : lo;
    uint32_t cls = inner[p + (g.t - g.s) / 2] == lo ? 0
                   : (inner[p] == lo || inner[p + g.t - g.s] == lo) ? 1 : 2;
    rank[p] = AnchorRank{mixsplit(canon(p, g.t), seed), cls, (uint32_t)p, (uint32_t)p};
  }
  // Block minima (van Herk / Gil-Werman) over blocks of W anchors.
  std::vector<AnchorRank> pre(anchors), suf(anchors);
  for (size_t b0 = 0; b0 < anchors; b0 += W) {
    size_t b1 = b0 + W < anchors ? b0 + W : anchors;
    pre[b0] = rank[b0];
    for (size_t p = b0 + 1; p < b1; ++p) pre[p] = rank_combine(pre[p - 1], rank[p]);
    suf[b1 - 1] = rank[b1 - 1];
    for (size_t p = b1 - 1; p-- > b0;) suf[p] = rank_combine(rank[p], suf[p + 1]);
  }
  std::vector<int> gt(n + 1, 0);
  for (size_t p = 0; p < n; ++p) gt[p + 1] = gt[p] + (encode_base(s[p]) >= 2);
  bool have = false;
  size_t prev = 0;
  for (size_t st = 0; st + k <= n; ++st) {
    size_t a = st, b = st + W - 1;  // anchor range [a, b]
    // An aligned window is exactly one block; otherwise it straddles two.
    AnchorRank best = (a % W == 0) ? suf[a] : rank_combine(suf[a], pre[b]);
    int g_count = gt[st + k] - gt[st];
    size_t anchor = g_count > k / 2 ? best.right : best.left;
    size_t pos = st + (anchor - st) % (size_t)g.w;
    if (!have || pos != prev) {
      out.push_back(canon(pos, m));
      if (positions) positions->push_back(pos);
      prev = pos;
      have = true;
    }
  }
}

// Links the candidates of one run (offsets ascending, one per offset) into
// randstrobemer keys, one per candidate in order: the partner is the first
// candidate strobe_min..strobe_max bases downstream with the fewest differing
// low 8 hash bits, or the candidate itself (Linker, src/anchors.rs:182-256).
inline void link_run(const std::vector<uint64_t>& offsets, const std::vector<uint64_t>& hashes,
                     uint64_t dmin, uint64_t dmax, std::vector<uint64_t>& out) {
  const size_t n = hashes.size();
  for (size_t i = 0; i < n; ++i) {
    size_t pick = i;
    int fewest = 9;
    for (size_t j = i + 1; j < n && offsets[j] - offsets[i] <= dmax && fewest; ++j) {
      if (offsets[j] - offsets[i] < dmin) continue;
      const int d = __builtin_popcountll((hashes[i] ^ hashes[j]) & 0xFF);
      if (d < fewest) fewest = d, pick = j;
    }
    out.push_back((hashes[i] >> 1) + (hashes[pick] >> 1));
  }
}

inline void ocm(const uint8_t* s, size_t n, int k, int m, uint64_t seed,
                std::vector<uint64_t>& out) {
  if (k <= 0 || !(k & 1) || m <= 0 || m > 31 || m > k) return;
  size_t i = 0;
  while (i < n) {
    size_t j = i;
    while (j < n && encode_base(s[j]) <= 3) ++j;
    if (j - i >= (size_t)k) ocm_run(s + i, j - i, k, m, seed, out);
    i = j + 1;
  }
}

inline std::vector<uint8_t> homopolymer(const uint8_t* s, size_t n) {
  std::vector<uint8_t> r;
  r.reserve(n);
  uint32_t prev = 5;
  for (size_t i = 0; i < n; ++i) {
    uint32_t c = encode_base(s[i]);
    if (c > 3 || c != prev) r.push_back(c > 3 ? s[i] : (uint8_t)"ACGT"[c]);
    prev = c > 3 ? 5 : c;
  }
  return r;
}

// Features of one ACGT run (already homopolymer-compressed when requested).
inline void run_features(const uint8_t* s, size_t n, const FeatureParams& f,
                         std::vector<uint64_t>& out) {
  if (f.strobes && f.mode <= 1) {
    // Candidates: every canonical k-mer (offset = window start) or the
    // run's selected minimizers, sorted by offset, one per offset.
    std::vector<uint64_t> keys, offsets;
    if (f.mode == 0) {
      kmers(s, n, f.k, keys);
      for (size_t i = 0; i < keys.size(); ++i) offsets.push_back(i);
    } else if (n >= (size_t)f.k && (f.k & 1) && f.m >= 1 && f.m <= 31 && f.m <= f.k) {
      std::vector<uint64_t> raw, at;
      ocm_run(s, n, f.k, f.m, f.seed, raw, &at);
      std::vector<size_t> order(raw.size());
      for (size_t i = 0; i < order.size(); ++i) order[i] = i;
      std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return at[a] < at[b]; });
      for (size_t i : order)
        if (offsets.empty() || at[i] != offsets.back()) {
          offsets.push_back(at[i]);
          keys.push_back(raw[i]);
        }
    }
    for (uint64_t& k : keys) k = strobe_hash(f.spaced ? spaced_canonical(f.pattern, k) : k);
    link_run(offsets, keys, f.strobe_min, f.strobe_max, out);
    return;
  }
  const size_t first = out.size();
  switch (f.mode) {
    case 0: kmers(s, n, f.k, out); break;
    case 1: ocm(s, n, f.k, f.m, f.seed, out); break;
    case 2: {
      size_t before = out.size();
      kmers(s, n, f.k, out);
      size_t w = before;
      for (size_t i = before; i < out.size(); ++i)
        if (mixsplit(out[i], f.seed) % f.sampling == 0) out[w++] = out[i];
      out.resize(w);
      break;
    }
    case 3:
      if (n >= (size_t)f.k) kmers(s, n, f.k - f.z, out);
      break;
  }
  if (f.spaced && f.mode <= 1)
    for (size_t i = first; i < out.size(); ++i) out[i] = spaced_canonical(f.pattern, out[i]);
}

// Features of a sequence that may contain non-ACGT bytes.
inline void sequence_features(const uint8_t* s, size_t n, const FeatureParams& f,
                              std::vector<uint64_t>& out) {
  size_t i = 0;
  while (i < n) {
    size_t j = i;
    while (j < n && encode_base(s[j]) <= 3) ++j;
    if (j > i) {
      if (f.homopolymer) {
        std::vector<uint8_t> c = homopolymer(s + i, j - i);
        run_features(c.data(), c.size(), f, out);
      } else {
        run_features(s + i, j - i, f, out);
      }
    }
    i = j + 1;
  }
}

}  // namespace cpu
}  // namespace zx
