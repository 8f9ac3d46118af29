"""The request server's staging ring (zindex_b200/csrc/host/span_ring.h) on
the CPU through a compiled harness.

The server copies each request's bases into a page-locked ring at submit and
frees the span when the request's batch has completed; batches complete out
of order. Random reserve/release sequences check that every span lies inside
the ring, that live spans never overlap, that an empty ring takes any span
that fits, that a refused span really has no room under the placement rule
(after the newest span, or at the start; a freed span comes back only when
every older span is freed), and that freeing everything brings the whole
ring back.
"""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HOST = ROOT / "zindex_b200" / "csrc" / "host"

HARNESS = r"""
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <vector>
#include "span_ring.h"

static int fail(const char* what, unsigned long long a, unsigned long long b) {
  printf("FAIL %s %llu %llu\n", what, a, b);
  return 1;
}

int main(int argc, char** argv) {
  const uint64_t cap = strtoull(argv[1], nullptr, 10);
  const int ops = atoi(argv[2]);
  std::mt19937_64 rng(strtoull(argv[3], nullptr, 10));
  zx::SpanRing ring(cap);
  std::map<uint64_t, std::pair<uint64_t, uint64_t>> live;  // id -> (off, len)
  std::vector<uint64_t> order;                              // live ids, oldest first
  // The ring's own span list: spans in id order, freed ones stay until every
  // older span is freed.
  struct M { uint64_t id, off, len; bool freed; };
  std::vector<M> model;
  uint64_t placed = 0, refused = 0, wraps = 0, last_off = 0;
  for (int i = 0; i < ops; ++i) {
    const bool take = live.empty() || rng() % 100 < 55;
    if (take) {
      const uint64_t n = 1 + rng() % (cap / 2);
      uint64_t off = 0, id = 0;
      const bool was_empty = live.empty();
      if (ring.reserve(n, &off, &id)) {
        if (off + n > cap) return fail("outside", off, n);
        for (auto& kv : live) {
          const uint64_t o = kv.second.first, l = kv.second.second;
          if (off < o + l && o < off + n) return fail("overlap", off, o);
        }
        if (!live.empty() && off < last_off) ++wraps;
        live[id] = {off, n};
        order.push_back(id);
        model.push_back(M{id, off, n, false});
        last_off = off;
        ++placed;
      } else {
        if (was_empty) return fail("empty ring refused", n, cap);
        // Refused: no room after the newest span nor at the start (before
        // the oldest), nor in the gap of a wrapped ring.
        const uint64_t head = model.front().off, tail = model.back().off + model.back().len;
        if (tail > head) {
          if (cap - tail >= n || head >= n) return fail("refused with room", n, tail);
        } else if (head - tail >= n) {
          return fail("refused with a gap", n, head - tail);
        }
        ++refused;
      }
    } else {
      const size_t k = rng() % order.size();
      const uint64_t id = order[k];
      ring.release(id);
      live.erase(id);
      order.erase(order.begin() + k);
      for (auto& m : model)
        if (m.id == id) m.freed = true;
      while (!model.empty() && model.front().freed) model.erase(model.begin());
      ring.release(id);  // a second release is ignored
    }
    if (ring.live() != model.size()) return fail("span count", ring.live(), model.size());
  }
  for (uint64_t id : order) ring.release(id);
  if (!ring.empty()) return fail("not empty", ring.live(), 0);
  uint64_t off = 0, id = 0;
  if (!ring.reserve(cap, &off, &id) || off != 0) return fail("whole ring", off, cap);
  uint64_t tmp = 0;
  if (ring.reserve(0, &off, &tmp) || ring.reserve(cap + 1, &off, &tmp)) return fail("sizes", 0, 0);
  printf("OK %llu %llu %llu\n", (unsigned long long)placed, (unsigned long long)refused,
         (unsigned long long)wraps);
  return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("ring")
    (d / "h.cpp").write_text(HARNESS)
    exe = d / "h"
    subprocess.run(["g++", "-O1", "-std=c++17", f"-I{HOST}", "-o", str(exe), str(d / "h.cpp")],
                   check=True)
    return exe


@pytest.mark.parametrize("cap,seed", [(1000, 1), (4096, 2), (65536, 3), (17, 4)])
def test_span_ring_random_sequences(harness, cap, seed):
    out = subprocess.run([str(harness), str(cap), "20000", str(seed)], capture_output=True,
                         text=True)
    assert out.returncode == 0, out.stdout
    status, placed, refused, wraps = out.stdout.split()
    assert status == "OK"
    # The sequences exercise all three outcomes.
    assert int(placed) > 1000 and int(refused) > 100 and int(wraps) > 100
