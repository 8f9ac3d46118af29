"""Randstrobemer queries on the GPU against the oracle.

Candidates (every canonical k-mer, or the selected minimizer positions of a
run, once each) are marked in a per-base table on the device and each tile's
candidates are linked by a forward scan of it (partners strobe_min..
strobe_max bases downstream in the same run, for distances above 256 too,
across tile boundaries); the reverse-complement strand is queried too, and
every record keeps per colour the larger strand count (query_stream.rs:
516-534, 690-701). Aggregates, per-record counts and per-record reports must
equal the oracle's, for k-mer and minimizer strobes, spaced seeds and
homopolymer compression.
"""
import numpy as np
import pytest

from helpers import build_index, dna, make_genomes, sample_reads

pytestmark = pytest.mark.gpu

_INDEXES = {}


def strobe_index(tmp_path_factory, k=21, lo=None, hi=None, pattern=None, homopolymer=False,
                 mode="kmers", m=None):
    key = (k, lo, hi, pattern, homopolymer, mode, m)
    if key not in _INDEXES:
        import subprocess

        import helpers

        d = tmp_path_factory.mktemp("strobe")
        fof = make_genomes(d / "g", 5, 12000, 61)
        args = [str(helpers.ZX_BUILD), "-f", str(fof), "-o", str(d / "ix"), "-q", "-r", "-i", mode,
                "-k", str(k), "-H", "4", "-b", "8"]
        if lo:
            args += ["-l", str(lo)]
        if hi:
            args += ["-u", str(hi)]
        if pattern:
            args += ["-p", pattern]
        if homopolymer:
            args += ["-c"]
        if m:
            args += ["-m", str(m)]
        subprocess.run(args, check=True)
        _INDEXES[key] = (d / "ix", [dna(12000, 61 + c) for c in range(5)])
    return _INDEXES[key]


def reads_for(genomes, n=200, length=180, seed=3):
    rng = np.random.default_rng(seed)
    reads = sample_reads(genomes, rng, n, length, n_runs=0.15, lower=0.02)
    return reads + [b"", b"ACG", genomes[2][:3000], genomes[0][5000:5900] + b"NNNN" + genomes[1][:700]]


CASES = [
    dict(k=21),
    dict(k=31, lo=5, hi=200),
    dict(k=15, pattern="##_#_#_#_#_#_##"),
    dict(k=25, homopolymer=True, lo=10, hi=90),
    dict(k=21, lo=300, hi=1200),                      # distances above 256
    dict(mode="minimizers", k=31, m=15),
    dict(mode="minimizers", k=31, m=19, lo=20, hi=400),
    dict(mode="minimizers", k=21, m=21),              # k == m: every m-mer
    dict(mode="minimizers", k=31, m=15, pattern="#####_###_#####"),
    dict(mode="minimizers", k=29, m=13, lo=100, hi=2000, homopolymer=True),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_strobe_aggregate_and_per_record_match_oracle(gpu, oracle, tmp_path_factory, tmp_path, case):
    import zindex_b200 as zx

    ix, genomes = strobe_index(tmp_path_factory, **case)
    reads = reads_for(genomes)
    bases, offsets = zx.pack_records(reads)
    want, want_total = oracle.query_records(ix, bases, offsets)
    with zx.Index(ix) as index:
        got, total = index.query_records(bases, offsets)
        assert total == want_total
        np.testing.assert_array_equal(got, want)
        counts, totals = index.query_per_record(bases, offsets)
        np.testing.assert_array_equal(counts.sum(axis=0, dtype=np.uint64), want)
        for r in (0, 7, len(reads) - 1, len(reads) - 2):
            b = np.frombuffer(reads[r], dtype=np.uint8)
            w, wt = oracle.query_records(ix, b, np.array([0, len(b)], dtype=np.uint64))
            assert totals[r] == wt
            np.testing.assert_array_equal(counts[r], w)
        q = tmp_path / "q.fa"
        with open(q, "wb") as f:
            for i, r in enumerate(reads):
                f.write(b">r%d\n" % i + r + b"\n")
        for fmt, ratio in (("tsv", 0.0), ("compact", 0.3)):
            out = tmp_path / f"{fmt}.txt"
            index.query_records_report(q, out, min_ratio=ratio, fmt=fmt)
            assert out.read_bytes() == oracle.records_report(ix, q, min_ratio=ratio, fmt=fmt)


def test_strobe_indexes_refuse_single_strand_device_paths(gpu, tmp_path_factory):
    import torch

    import zindex_b200 as zx

    ix, _ = strobe_index(tmp_path_factory, k=21)
    with zx.Index(ix) as index:
        dev = torch.device("cuda", 0)
        d_bases = torch.zeros(100, dtype=torch.uint8, device=dev)
        d_off = torch.tensor([0, 100], dtype=torch.int64, device=dev)
        d_counts = torch.zeros(index.colors, dtype=torch.int64, device=dev)
        d_total = torch.zeros(1, dtype=torch.int64, device=dev)
        with pytest.raises(zx.ZxError):
            index.query_device(d_bases.data_ptr(), 100, d_off.data_ptr(), 1, d_counts.data_ptr(),
                               d_total.data_ptr())
    mix, _ = strobe_index(tmp_path_factory, k=31, mode="minimizers", m=15)
    with zx.Index(mix) as index:
        with pytest.raises(zx.ZxError):
            index.query_device(d_bases.data_ptr(), 100, d_off.data_ptr(), 1, d_counts.data_ptr(),
                               d_total.data_ptr())
