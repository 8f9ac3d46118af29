"""Per-record queries (`zorindex query --records`) on the GPU against the oracle.

The report bytes of the C ABI (zx_query_records_report) and of the CLI must
equal the oracle's report for every seed mode, both formats, several
min_ratio thresholds and record batch sizes; the per-record counts
(zx_query_per_record) must equal a query of each record alone, also when the
records span several device groups (many colours).
"""
import subprocess

import numpy as np
import pytest

import helpers
from helpers import ZORINDEX, build_index, dna, make_genomes, sample_reads

pytestmark = pytest.mark.gpu

_INDEXES = {}


def index_for(tmp_path_factory, colors=5, length=12000, seed=81, **opts):
    key = (colors, length, seed, tuple(sorted(opts.items())))
    if key not in _INDEXES:
        d = tmp_path_factory.mktemp("rix")
        fof = make_genomes(d / "genomes", colors, length, seed)
        build_index(fof, d / "index", **opts)
        _INDEXES[key] = (d / "index", [dna(length, seed + c) for c in range(colors)])
    return _INDEXES[key]


def query_file(path, genomes, n=300, seed=5, fastq=False):
    rng = np.random.default_rng(seed)
    reads = sample_reads(genomes, rng, n, 150, n_runs=0.1, lower=0.01)
    reads += [b"", b"ACG", genomes[0][:5000], b"N" * 80, genomes[-1][200:260] + b"NN" + genomes[-1][:90]]
    names = [f"read{i}" for i in range(len(reads))]
    names[1] = 'read"1"'
    with open(path, "wb") as f:
        for name, r in zip(names, reads):
            if fastq:
                f.write(b"@" + name.encode() + b" x\n" + r + b"\n+\n" + b"I" * len(r) + b"\n")
            else:
                f.write(b">" + name.encode() + b" desc\n")
                for j in range(0, len(r), 70):
                    f.write(r[j: j + 70] + b"\n")
    return path, reads


MODES = [
    dict(mode="kmers", k=31, H=4, b=8),
    dict(mode="kmers", k=45, H=3, b=4),
    dict(mode="minimizers", k=31, m=19, H=4, b=8),
    dict(mode="modimizers", k=31, d=8, H=2, b=16),
    dict(mode="findere", k=31, z=10, H=4, b=8),
    dict(mode="kmers", k=31, H=4, b=8, homopolymer=True),
    dict(mode="minimizers", k=31, m=15, H=4, b=8, pattern="##_##_###_##_##"),
]


@pytest.mark.parametrize("opts", MODES, ids=lambda o: "-".join(f"{k}{v}" for k, v in o.items()))
def test_report_matches_oracle(gpu, oracle, tmp_path_factory, tmp_path, opts):
    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, **opts)
    q, _ = query_file(tmp_path / "q.fa", genomes)
    with zx.Index(ix) as index:
        for fmt in ("tsv", "compact"):
            for min_ratio in (0.0, 1e-9, 0.4, 1.0):
                out = tmp_path / f"out-{fmt}-{min_ratio}.tsv"
                index.query_records_report(q, out, min_ratio=min_ratio, fmt=fmt)
                want = oracle.records_report(ix, q, min_ratio=min_ratio, fmt=fmt)
                assert out.read_bytes() == want, (fmt, min_ratio)
        out = tmp_path / "norec.tsv"
        index.query_records_report(q, out, recover=False)
        assert out.read_bytes() == oracle.records_report(ix, q, recover=False)


@pytest.mark.parametrize("colors,opts", [(4096, dict(k=31, H=8, b=4)),
                                         (2048, dict(k=25, H=3, b=16, groups="4,5,6"))],
                         ids=["c4096-H8-b4", "c2048-H3-b16-multi"])
def test_wide_row_report_with_threshold_pruning(gpu, oracle, tmp_path_factory, tmp_path, colors,
                                                opts):
    """Per-record reports on wide-row indexes: with min_ratio > 0 the wide
    probe stops loading the row chunks whose colours can no longer reach the
    threshold (exact pruning), and the report bytes still equal the oracle's
    (colours below the threshold are not reported, whatever their partial
    counts). Long records take several probe rounds (no pruning across
    blocks); a multi-member group's chunks are never pruned."""
    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, colors=colors, length=3000, seed=91, min_docs=1,
                            **opts)
    q, _ = query_file(tmp_path / "q.fa", genomes, n=400, seed=9)
    with zx.Index(ix) as index:
        assert index.launch()["wide"] == 1
        for fmt in ("compact", "tsv"):
            for min_ratio in (1e-9, 0.3, 0.8, 1.0):
                out = tmp_path / f"w-{fmt}-{min_ratio}.tsv"
                index.query_records_report(q, out, min_ratio=min_ratio, fmt=fmt)
                want = oracle.records_report(ix, q, min_ratio=min_ratio, fmt=fmt)
                assert out.read_bytes() == want, (fmt, min_ratio)


def test_batch_sizes_fastq_and_cli(gpu, oracle, tmp_path_factory, tmp_path):
    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, mode="kmers", k=31, H=4, b=8)
    fa, _ = query_file(tmp_path / "q.fa", genomes, n=200, seed=8)
    fq, _ = query_file(tmp_path / "q.fq", genomes, n=200, seed=8, fastq=True)
    want = oracle.records_report(ix, fa, fmt="compact", min_ratio=0.2)
    with zx.Index(ix) as index:
        for batch in (1, 3, 4096):
            out = tmp_path / f"b{batch}.txt"
            index.query_records_report(fq, out, fmt="compact", min_ratio=0.2, batch=batch)
            assert out.read_bytes() == want, batch
    run = lambda *a: subprocess.run([str(ZORINDEX), "query", "-i", str(ix), *a],
                                    capture_output=True)
    r = run("-q", str(fa), "-r", "-F", "compact", "-a", "0.2", "-B", "3")
    assert r.returncode == 0, r.stderr
    assert r.stdout == want
    r = run("-q", str(fa), "--records")
    assert r.returncode == 0 and r.stdout == oracle.records_report(ix, fa)
    assert run("-q", str(fa), "-F", "compact").returncode == 2   # requires --records
    assert run("-q", str(fa), "-r", "-B", "0").returncode == 1   # batch must be positive
    assert run("-q", str(fa), "-r", "-a", "1.5").returncode == 1
    bad = tmp_path / "bad.fa"
    bad.write_bytes(b"ACGT\n")
    r = run("-q", str(bad), "-r")
    assert r.returncode == 1 and b"--records requires FASTA or FASTQ" in r.stderr


@pytest.mark.parametrize("opts,colors,n", [
    (dict(mode="kmers", k=25, H=3, b=16), 2048, 17000),   # 16,384 records per device group
    (dict(mode="findere", k=31, z=10, H=4, b=8), 2048, 4500),  # 2,048-4,096 records per group
])
def test_per_record_counts_across_groups(gpu, oracle, tmp_path_factory, opts, colors, n):
    """Each record's counts equal a query of the record alone, also when the
    records run in several device groups; the column sums equal the aggregate."""
    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, colors=colors, length=1500, seed=91, **opts)
    rng = np.random.default_rng(3)
    reads = sample_reads(genomes, rng, n, 120, n_runs=0.05)
    bases, offsets = zx.pack_records(reads)
    with zx.Index(ix) as index:
        counts, totals = index.query_per_record(bases, offsets)
        assert counts.shape == (n, colors)
        pick = list(range(0, n, max(1, n // 40))) + [n - 1]
        for r in pick:
            b = np.frombuffer(reads[r], dtype=np.uint8)
            want, want_total = oracle.query_records(ix, b, np.array([0, len(b)], dtype=np.uint64))
            assert totals[r] == want_total, r
            np.testing.assert_array_equal(counts[r], want)
        # Column sums: the aggregate of all records.
        agg, agg_total = index.query_records(bases, offsets)
        np.testing.assert_array_equal(counts.sum(axis=0, dtype=np.uint64), agg)
        assert int(totals.sum()) == agg_total


def test_per_record_small_cases(gpu, oracle, tmp_path_factory):
    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, mode="kmers", k=31, H=4, b=8)
    with zx.Index(ix) as index:
        counts, totals = index.query_per_record(np.zeros(0, np.uint8), np.zeros(1, np.uint64))
        assert counts.shape == (0, index.colors) and totals.shape == (0,)
        reads = [b"", genomes[2][:31], genomes[2][:30], b"N" * 40]
        bases, offsets = zx.pack_records(reads)
        counts, totals = index.query_per_record(bases, offsets)
        assert list(totals) == [0, 1, 0, 0]
        assert counts[1][2] == 1 and counts.sum() == counts[1].sum()
        bases, offsets = zx.pack_records([b"", b""])   # a group without bases
        counts, totals = index.query_per_record(bases, offsets)
        assert list(totals) == [0, 0] and counts.sum() == 0
        # Page-locked inputs and caller-owned page-locked outputs.
        import torch

        reads = [genomes[r % 5][r * 37: r * 37 + 150] for r in range(200)]
        bases, offsets = zx.pack_records(reads)
        want_c, want_t = index.query_per_record(bases, offsets)
        pb = torch.from_numpy(bases).pin_memory().numpy()
        po = torch.from_numpy(offsets.view(np.int64)).pin_memory().numpy().view(np.uint64)
        pc = torch.zeros((200, index.colors), dtype=torch.int64).pin_memory().numpy().view(np.uint64)
        pt = torch.zeros(200, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
        got_c, got_t = index.query_per_record(pb, po, counts=pc, totals=pt)
        assert got_c is pc and got_t is pt
        np.testing.assert_array_equal(pc, want_c)
        np.testing.assert_array_equal(pt, want_t)
        with pytest.raises(ValueError):
            index.query_per_record(bases, offsets, counts=np.zeros((3, 3), np.uint64))
