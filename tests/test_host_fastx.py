"""The product's host-side query readers on the CPU (zindex_b200/csrc/host/
fastx.cpp), compiled into a small harness: the aggregate reader (split at
records, headers and qualities ignored, LF/CRLF, gzip) and the strict named
record reader of per-record reports (records.rs:150-290), including its error
messages, which must be the reference's. Compressed inputs: gzip, zstd, xz and
bzip2, single and concatenated streams, as the reference's reader decodes them
(src/lib.rs:283-321; its test of identical features from every format,
src/lib.rs:1214-1283).
"""
import bz2
import gzip
import lzma
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HOST = ROOT / "zindex_b200" / "csrc" / "host"

HARNESS = r"""
#include <cstdio>
#include <string>
#include "error.h"
#include "fastx.h"
int main(int argc, char** argv) {
  const std::string mode = argv[1], path = argv[2];
  try {
    zx::RecordBatch b = mode == "named" ? zx::read_named_records(path) : zx::read_fastx(path, true);
    for (size_t r = 0; r < b.records(); ++r) {
      std::string seq(b.bases.begin() + b.offsets[r], b.bases.begin() + b.offsets[r + 1]);
      printf("%s\t%s\n", r < b.names.size() ? b.names[r].c_str() : "", seq.c_str());
    }
  } catch (const zx::Error& e) {
    printf("ERROR\t%d\t%s\n", e.code, e.what());
  }
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("fastx")
    (d / "h.cpp").write_text(HARNESS)
    exe = d / "h"
    subprocess.run(["g++", "-O1", "-std=c++17", f"-I{HOST}", "-o", str(exe), str(d / "h.cpp"),
                    str(HOST / "fastx.cpp"), str(HOST / "zstd_io.cpp"), "-lz", "-l:libzstd.so.1",
                    "-l:liblzma.so.5", "-l:libbz2.so.1.0", "-lpthread"], check=True)
    return exe


def run(harness, tmp_path, mode, data: bytes, gz=False):
    p = tmp_path / ("q.fa.gz" if gz else "q.fa")
    p.write_bytes(gzip.compress(data) if gz else data)
    out = subprocess.run([str(harness), mode, str(p)], capture_output=True, check=True)
    return out.stdout.decode().splitlines()


def test_aggregate_reader(harness, tmp_path):
    data = b">r1 desc\r\nACGT\r\nNNac\r\n>r2\n\n>r3\nGG\n"
    want = ["r1\tACGTNNac", "r2\t", "r3\tGG"]
    assert run(harness, tmp_path, "plain", data) == want
    assert run(harness, tmp_path, "plain", data, gz=True) == want
    fq = b"@a x\nACGT\n+\nIIII\n@b\nAC\n+b\nII\n"
    assert run(harness, tmp_path, "plain", fq) == ["a\tACGT", "b\tAC"]


def test_named_reader_accepts_reference_layouts(harness, tmp_path):
    fq = b"@r1 d\r\nAC\r\nGT\r\n+\r\nII\r\nII\r\n\r\n@r2\n\n+\n"
    assert run(harness, tmp_path, "named", fq) == ["r1\tACGT", "r2\t"]
    fa = b"\n>q\"1\" x  \nAC  \n\nGT\n>e\n"
    assert run(harness, tmp_path, "named", fa) == ['q"1"\tACGT', "e\t"]


@pytest.mark.parametrize("text,message", [
    (b"ACGT\n", "--records requires FASTA or FASTQ"),
    (b"", "no FASTA/FASTQ records"),
    (b">r1\nAC GT\n", "whitespace inside FASTA sequence"),
    (b">\nACGT\n", "empty FASTA identifier"),
    (b"@r1\nACGT\n+\nII\n", "truncated FASTQ quality"),
    (b"@r1\nACGT\n+\nIIIII\n", "FASTQ sequence and quality lengths differ"),
    (b"@r1\nACGT\n", "truncated FASTQ sequence"),
    (b">r\xff\nACGT\n", "invalid FASTA identifier"),
])
def test_named_reader_errors(harness, tmp_path, text, message):
    lines = run(harness, tmp_path, "named", text)
    assert len(lines) == 1 and lines[0].startswith("ERROR\t2\t"), lines
    assert lines[0].split("\t", 2)[2] == message


def _zstd(data: bytes) -> bytes:
    import pyarrow as pa

    return pa.compress(data, codec="zstd", asbytes=True)


@pytest.mark.parametrize("codec", ["gz", "zst", "xz", "bz2"])
def test_compressed_inputs_read_like_plain(harness, tmp_path, codec):
    data = b">r1 d\nACGTNN\nacgt\n>r2\n" + b"ACGT" * 20000 + b"\n>r3\nTTTT\n"
    pack = {"gz": gzip.compress, "xz": lzma.compress, "bz2": bz2.compress, "zst": _zstd}[codec]
    want = run(harness, tmp_path, "plain", data)
    half = data.index(b">r2")
    for blob in (pack(data), pack(data[:half]) + pack(data[half:])):  # one and two streams
        p = tmp_path / f"q.fa.{codec}"
        p.write_bytes(blob)
        out = subprocess.run([str(harness), "plain", str(p)], capture_output=True, check=True)
        assert out.stdout.decode().splitlines() == want
    p.write_bytes(pack(data)[:-7])  # truncated
    out = subprocess.run([str(harness), "plain", str(p)], capture_output=True, check=True)
    assert out.stdout.decode().startswith("ERROR\t2\t"), out.stdout
