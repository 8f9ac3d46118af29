"""Compressed query files through zx_query_file on the GPU: plain, gzip,
zstd, xz and bzip2 inputs give the same counts, and the oracle's on the plain
file (the reference reads every format through one decoder, src/lib.rs:283-321,
and tests identical features from each, src/lib.rs:1214-1283)."""
import bz2
import gzip
import lzma

import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu


def test_compressed_query_files_match_plain(gpu, oracle, tmp_path):
    import pyarrow as pa

    import zindex_b200 as zx

    fof = helpers.make_genomes(tmp_path / "genomes", colors=4, length=20000, seed=41)
    index = helpers.build_index(fof, tmp_path / "index", k=31, H=4, b=8)
    genomes = [helpers.dna(20000, 41 + c) for c in range(4)]
    reads = helpers.sample_reads(genomes, np.random.default_rng(3), 300, 150, n_runs=0.1)
    plain = helpers.write_fasta(tmp_path / "q.fa", reads)
    data = plain.read_bytes()
    files = {"plain": plain}
    for ext, pack in (("gz", gzip.compress), ("xz", lzma.compress), ("bz2", bz2.compress),
                      ("zst", lambda d: pa.compress(d, codec="zstd", asbytes=True))):
        files[ext] = tmp_path / f"q.fa.{ext}"
        files[ext].write_bytes(pack(data))
    want, want_total, _ = oracle.query_file(index, plain)
    with zx.Index(index) as ix:
        for name, path in files.items():
            got, total, _ = ix.query_file(path)
            assert total == want_total, name
            np.testing.assert_array_equal(got, want)
