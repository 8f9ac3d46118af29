"""The product's manifest reader on the CPU (zindex_b200/csrc/host/
manifest.cpp) through a compiled harness: a valid index loads, and manifests
the reference refuses are refused (Manifest::features and validate,
storage.rs:132-259; SpacedSeed and RandstrobeConfig checks, anchors.rs:15-42,
98-110; FeatureConfig::validate_anchors, lib.rs:177-206).
"""
import json
import shutil
import subprocess
from pathlib import Path

import pytest

import helpers

ROOT = Path(__file__).resolve().parents[1]
HOST = ROOT / "zindex_b200" / "csrc" / "host"

HARNESS = r"""
#include <cstdio>
#include "error.h"
#include "manifest.h"
int main(int argc, char** argv) {
  try {
    zx::Manifest m = zx::load_manifest(argv[1]);
    printf("OK\t%zu\t%d\t%s\t%llu\t%llu\n", m.colors.size(), (int)m.has_seed_pattern,
           m.seed_pattern.c_str(), (unsigned long long)m.strobe_min,
           (unsigned long long)m.strobe_max);
  } catch (const zx::Error& e) {
    printf("ERROR\t%d\t%s\n", e.code, e.what());
  }
}
"""


@pytest.fixture(scope="module")
def harness(native, tmp_path_factory):
    d = tmp_path_factory.mktemp("manifest")
    (d / "h.cpp").write_text(HARNESS)
    exe = d / "h"
    subprocess.run(["g++", "-O1", "-std=c++17", f"-I{HOST}", "-o", str(exe), str(d / "h.cpp"),
                    str(HOST / "manifest.cpp"), str(HOST / "json.cpp")], check=True)
    fof = helpers.make_genomes(d / "g", 3, 3000, 4)
    ix = helpers.build_index(fof, d / "ix", k=15, H=3, b=8, pattern="###_#_#_#_#_###")
    return exe, ix


def _load(exe, ix):
    out = subprocess.run([str(exe), str(ix)], capture_output=True, text=True, check=True)
    return out.stdout.strip().split("\t")


def test_valid_manifest_loads(harness):
    exe, ix = harness
    r = _load(exe, ix)
    assert r[:4] == ["OK", "3", "1", "###_#_#_#_#_###"]


@pytest.mark.parametrize("changes,code,message", [
    ({"seed_pattern": "##_"}, 2, "seed pattern must be 1..=31 symmetric"),
    ({"seed_pattern": "#_#_#"}, 2, "seed pattern width must match k"),
    ({"index_mode": 3, "findere_z": 5}, 2, "require --index-mode kmers or minimizers"),
    ({"randstrobemers": {"min_distance": 6, "max_distance": 5},
      "randstrobe_scheme": "strobealign-popcount8-symmetric64-downstream-v1"}, 2,
     "minimum distance must not exceed maximum"),
    ({"randstrobemers": {"min_distance": 0, "max_distance": 5},
      "randstrobe_scheme": "strobealign-popcount8-symmetric64-downstream-v1"}, 2,
     "minimum distance must be greater than zero"),
    ({"randstrobemers": {"min_distance": 2, "max_distance": 5},
      "randstrobe_scheme": "custom"}, 2, "unsupported legacy/custom randstrobemer extraction"),
    ({"fingerprint_bits": 3}, 2, "invalid fingerprint width"),
])
def test_refused_manifests(harness, tmp_path, changes, code, message):
    exe, ix = harness
    bad = tmp_path / "bad"
    shutil.copytree(ix, bad)
    m = json.loads((bad / "manifest.json").read_text())
    m.update(changes)
    (bad / "manifest.json").write_text(json.dumps(m))
    r = _load(exe, bad)
    assert r[0] == "ERROR" and int(r[1]) in (code, 7), r
    assert message in r[2], r
