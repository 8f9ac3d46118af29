"""The per-record report writer (zindex_b200/csrc/host/record_report.cpp) on the
CPU: its fixed-point ratios must equal correctly rounded `{:.8}` formatting
(Rust's, record_output.rs:47-52; Python's format is correctly rounded too) for
every count / total, including exact ties, and its rows must follow
RecordFormat::write_record (record_output.rs:21-62).

The writer is compiled here into a small harness (g++) that reads
"count total" lines and prints one TSV row per line.
"""
import random
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HOST = ROOT / "zindex_b200" / "csrc" / "host"

HARNESS = r"""
#include <cstdio>
#include <iostream>
#include "record_report.h"
int main() {
  std::vector<zx::ColorMeta> colors(2);
  colors[0].name = "a";
  colors[1].name = "b\"c";
  unsigned long long c, t;
  std::string out;
  while (std::cin >> c >> t) {
    out.clear();
    const uint64_t counts[2] = {c, 0};
    zx::append_record(out, zx::RecordFormat::kTsv, "q", t, counts, colors, 1e-300);
    const uint32_t ids[2] = {0, 1};
    const uint64_t hits[2] = {c, 7};
    zx::append_record_hits(out, zx::RecordFormat::kCompact, "q", t, ids, hits, 2, colors);
    fputs(out.c_str(), stdout);
  }
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("fmt")
    src = d / "h.cpp"
    src.write_text(HARNESS)
    exe = d / "h"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{HOST}", "-o", str(exe), str(src),
                    str(HOST / "record_report.cpp")], check=True)
    return exe


def _pairs():
    rng = random.Random(11)
    pairs = [(1, 1), (0, 5), (1, 3), (2, 3), (1, 512), (3, 512), (5, 1024), (1, 2 ** 20),
             (1, 10 ** 9), (10 ** 9 - 1, 10 ** 9), (123456789, 987654321), (1, 7), (6, 7)]
    # Exact ties at the eighth decimal: count / total = (2j+1) / (2 * 10^8) with a
    # power-of-two denominator (e.g. 1/512 = 0.001953125).
    for e in range(9, 40):
        for c in (1, 3, 5, 7, 11, 1023):
            if c < 2 ** e:
                pairs.append((c, 2 ** e))
    for _ in range(20000):
        t = rng.choice([rng.randint(1, 300), rng.randint(1, 10 ** 6), rng.randint(1, 10 ** 12)])
        pairs.append((rng.randint(0, t), t))
    return pairs


def test_ratios_and_rows_match_correct_rounding(harness):
    pairs = _pairs()
    text = "".join(f"{c} {t}\n" for c, t in pairs)
    out = subprocess.run([str(harness)], input=text, capture_output=True, text=True, check=True)
    lines = out.stdout.splitlines()
    want = []
    for c, t in pairs:
        if c > 0:
            want.append(f"q\t0\ta\t{c}\t{t}\t{c / t:.8f}")
        else:
            want.append(f"q\t.\t.\t0\t{t}\t0.00000000")
        want.append(f"q\t{t}\t0:{c},1:7")
    assert len(lines) == len(want)
    for got, exp in zip(lines, want):
        assert got == exp
