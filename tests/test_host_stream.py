"""The streamed bank decoder (zindex_b200/csrc/host/zstd_io.cpp: stream_bank)
on the CPU through a compiled harness whose sink copies every piece into host
memory: for several piece sizes (frames straddling pieces), ring sizes and
thread counts the reassembled payload equals a whole-stream decode of the same
file, and damaged files are refused.
"""
import subprocess
from pathlib import Path

import pytest

import helpers

ROOT = Path(__file__).resolve().parents[1]
HOST = ROOT / "zindex_b200" / "csrc" / "host"

HARNESS = r"""
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "error.h"
#include "zstd_io.h"
struct Copy : zx::PieceSink {
  std::vector<uint8_t>* out;
  uint8_t* const* ring;
  std::vector<int> busy;
  void consume(int slot, uint64_t offset, uint64_t len) override {
    if (busy[slot]) throw zx::Error(1, "slot reused before it was drained");
    memcpy(out->data() + offset, ring[slot], len);
    busy[slot] = 1;
  }
  void drain(int slot) override { busy[slot] = 0; }
};
int main(int argc, char** argv) {
  const std::string path = argv[1];
  const uint64_t payload = std::stoull(argv[2]), piece = std::stoull(argv[3]);
  const int slots = std::stoi(argv[4]), threads = std::stoi(argv[5]);
  const bool compare = argc > 6;  // also decode the whole stream and compare
  try {
    std::vector<uint8_t> whole;
    if (compare) {
      std::vector<uint8_t> file = zx::read_file_bytes(path);
      whole = zx::zstd_decode_all(file.data(), file.size());
    }
    std::vector<std::vector<uint8_t>> ring_mem(slots, std::vector<uint8_t>(piece));
    std::vector<uint8_t*> ring(slots);
    for (int i = 0; i < slots; ++i) ring[i] = ring_mem[i].data();
    std::vector<uint8_t> got(payload);
    Copy sink;
    sink.out = &got;
    sink.ring = ring.data();
    sink.busy.assign(slots, 0);
    uint8_t header[40];
    zx::stream_bank(path, header, payload, piece, ring.data(), slots, threads, sink);
    if (!compare) {
      printf("STREAMED\n");
      return 0;
    }
    const bool same = whole.size() == payload + 40 && !memcmp(whole.data(), header, 40) &&
                      !memcmp(whole.data() + 40, got.data(), payload);
    printf(same ? "SAME\n" : "DIFFERENT\n");
  } catch (const zx::Error& e) {
    printf("ERROR\t%d\t%s\n", e.code, e.what());
  }
}
"""


@pytest.fixture(scope="module")
def setup(native, tmp_path_factory):
    d = tmp_path_factory.mktemp("stream")
    (d / "h.cpp").write_text(HARNESS)
    exe = d / "h"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{HOST}", "-o", str(exe), str(d / "h.cpp"),
                    str(HOST / "zstd_io.cpp"), "-lz", "-l:libzstd.so.1", "-lpthread"], check=True)
    fof = helpers.make_genomes(d / "g", 20, 1_000_000, 3)
    ix = helpers.build_index(fof, d / "ix", k=31, H=4, b=16)   # 40-byte rows, several frames
    import json

    bank = json.loads((ix / "manifest.json").read_text())["banks"][0]
    payload = bank["slots"] * ((bank["row_bits"] + 7) // 8)
    return exe, ix / bank["file"], payload, (bank["row_bits"] + 7) // 8


def _run(exe, path, payload, piece, slots, threads, compare=True):
    args = [str(exe), str(path), str(payload), str(piece), str(slots), str(threads)]
    out = subprocess.run(args + (["compare"] if compare else []), capture_output=True, text=True,
                         check=True, timeout=120)
    return out.stdout.strip()


@pytest.mark.parametrize("rows_per_piece,slots,threads", [
    (110_000, 3, 1), (110_000, 6, 8), (123_457, 3, 4), (400_000, 4, 16), (10_000_000, 3, 2)])
def test_streamed_payload_equals_whole_decode(setup, rows_per_piece, slots, threads):
    exe, bank, payload, row = setup
    assert payload > (32 << 20)  # several 4 MiB frames and pieces
    piece = min(rows_per_piece * row, payload)
    assert _run(exe, bank, payload, piece, slots, threads) == "SAME"


def test_pieces_below_one_frame_are_refused(setup):
    exe, bank, payload, row = setup
    r = _run(exe, bank, payload, 1000 * row, 3, 2, compare=False)
    assert r.startswith("ERROR\t1\t"), r


def test_damaged_banks_are_refused(setup, tmp_path):
    exe, bank, payload, row = setup
    data = bytearray(bank.read_bytes())
    bad = tmp_path / "bad.zst"
    data[len(data) // 3] ^= 0xFF
    bad.write_bytes(bytes(data))
    assert _run(exe, bank, payload, 110_000 * row, 4, 4, compare=False) == "STREAMED"
    r = _run(exe, bad, payload, 110_000 * row, 4, 4, compare=False)
    assert r.startswith("ERROR\t2\t"), r
    short = tmp_path / "short.zst"
    short.write_bytes(bank.read_bytes()[: bank.stat().st_size // 2])
    r = _run(exe, short, payload, 110_000 * row, 4, 4, compare=False)
    assert r.startswith("ERROR\t2\t"), r
