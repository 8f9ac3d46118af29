"""Parity of the CUDA query path with the oracle (bit-exact counts and totals).

Every test here runs the GPU through the C ABI (libzindex_b200.so) and compares
with the oracle's restatement of the reference query on the same index and
query records. Indexes are built by zx_build from seeded synthetic genomes.
"""
import subprocess

import numpy as np
import pytest

import helpers
from helpers import build_index, dna, make_genomes, sample_reads

pytestmark = pytest.mark.gpu

_INDEXES = {}


def index_for(tmp_path_factory, colors=6, length=30000, seed=5, **opts):
    key = (colors, length, seed, tuple(sorted(opts.items())))
    if key not in _INDEXES:
        d = tmp_path_factory.mktemp("ix")
        fof = make_genomes(d / "genomes", colors, length, seed)
        build_index(fof, d / "index", **opts)
        genomes = [dna(length, seed + c) for c in range(colors)]
        _INDEXES[key] = (d / "index", genomes)
    return _INDEXES[key]


def reads_for(genomes, seed=11, n=300, length=150, **kw):
    rng = np.random.default_rng(seed)
    return sample_reads(genomes, rng, n, length, **kw)


def gpu_vs_oracle(oracle, index_dir, records, recover=True, plain=False):
    import zindex_b200 as zx

    bases, offsets = zx.pack_records(records)
    want, want_total = oracle.query_records(index_dir, bases, offsets, recover=recover)
    with zx.Index(index_dir) as ix:
        # Both register-gather forms: per-hit counter updates and bit-plane counters.
        for planes in ((0,) if plain else (0, 1)):
            ix.set_launch(planes=planes)
            got, total = ix.query_records(bases, offsets, recover=recover, plain=plain)
            assert total == want_total
            np.testing.assert_array_equal(got, want)
    return got, total


KMER_CASES = [
    dict(k=31, H=4, b=8),
    dict(k=21, H=3, b=4),
    dict(k=32, H=2, b=16),
    dict(k=33, H=4, b=8),
    dict(k=63, H=8, b=2),
    dict(k=15, H=16, b=1),
    dict(k=27, H=32, b=32),
]


@pytest.mark.parametrize("case", KMER_CASES, ids=lambda c: "k{k}-H{H}-b{b}".format(**c))
def test_kmers_match_oracle(gpu, oracle, tmp_path_factory, case):
    ix, genomes = index_for(tmp_path_factory, mode="kmers", **case)
    gpu_vs_oracle(oracle, ix, reads_for(genomes, n_runs=0.1, lower=0.01))


@pytest.mark.parametrize("H", [2, 3, 4, 8, 16, 32])
@pytest.mark.parametrize("b", [1, 2, 4, 8, 16, 32])
def test_hash_and_width_sweep(gpu, oracle, tmp_path_factory, H, b):
    ix, genomes = index_for(tmp_path_factory, colors=5, length=8000, mode="kmers", k=25, H=H, b=b)
    gpu_vs_oracle(oracle, ix, reads_for(genomes, n=120, length=120))


MIN_CASES = [
    dict(k=49, m=31, H=3, b=16),
    dict(k=31, m=21, H=4, b=8),
    dict(k=19, m=12, H=4, b=8),
    dict(k=15, m=15, H=4, b=8),
    dict(k=9, m=5, H=3, b=4),
    dict(k=101, m=31, H=4, b=8),
]


@pytest.mark.parametrize("case", MIN_CASES, ids=lambda c: "k{k}-m{m}".format(**c))
def test_minimizers_match_oracle(gpu, oracle, tmp_path_factory, case):
    ix, genomes = index_for(tmp_path_factory, mode="minimizers", **case)
    gpu_vs_oracle(oracle, ix, reads_for(genomes, length=600, n=120, n_runs=0.2, lower=0.01))


@pytest.mark.parametrize("case", [dict(k=31, d=4), dict(k=49, d=8), dict(k=21, d=1)],
                         ids=lambda c: "k{k}-d{d}".format(**c))
def test_modimizers_match_oracle(gpu, oracle, tmp_path_factory, case):
    ix, genomes = index_for(tmp_path_factory, mode="modimizers", H=4, b=8, **case)
    gpu_vs_oracle(oracle, ix, reads_for(genomes, length=400, n=150, n_runs=0.1))


FINDERE_CASES = [
    dict(k=31, z=10, H=4, b=8),
    dict(k=25, z=3, H=3, b=4),
    dict(k=21, z=1, H=2, b=16),
    dict(k=45, z=8, H=4, b=8),   # s = 37: polynomial hash of long s-mers
    dict(k=31, z=30, H=8, b=1),  # s = 1
]


@pytest.mark.parametrize("case", FINDERE_CASES, ids=lambda c: "k{k}-z{z}-H{H}-b{b}".format(**c))
def test_findere_matches_oracle(gpu, oracle, tmp_path_factory, case):
    ix, genomes = index_for(tmp_path_factory, colors=6, length=20000, mode="findere", **case)
    reads = reads_for(genomes, n=150, length=300, n_runs=0.2, lower=0.05)
    g = genomes[1]
    # Records across a 16,384-window findere task, shorter than k, exactly k, with N.
    reads += [g[:18000], g[100:100 + case["k"] - 1], g[200:200 + case["k"]], b"",
              g[300:600] + b"N" + g[600:900], b"ACGT" * 50]
    gpu_vs_oracle(oracle, ix, reads)


def test_findere_groups_and_recovery(gpu, oracle, tmp_path_factory):
    ix, genomes = index_for(tmp_path_factory, colors=8, length=15000, seed=31, mode="findere",
                            k=31, z=6, H=4, b=4, groups="0,1,2;3,5;6,7")
    reads = reads_for(genomes, n=300, length=250)
    gpu_vs_oracle(oracle, ix, reads, recover=True)
    gpu_vs_oracle(oracle, ix, reads, recover=False)


def test_findere_noalloc_equals_device_query(gpu, oracle, tmp_path_factory):
    import torch

    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, colors=6, length=20000, mode="findere", k=31, z=10,
                            H=4, b=8)
    reads = reads_for(genomes, n=200, length=200)
    bases, offsets = zx.pack_records(reads)
    want, want_total = oracle.query_records(ix, bases, offsets)
    dev = torch.device("cuda", 0)
    d_bases = torch.from_numpy(bases).to(dev)
    d_off = torch.from_numpy(offsets.view(np.int64)).to(dev)
    with zx.Index(ix) as index:
        for _ in range(2):
            counts = torch.zeros(index.colors, dtype=torch.int64, device=dev)
            total = torch.zeros(1, dtype=torch.int64, device=dev)
            index.query_device_noalloc(d_bases.data_ptr(), len(bases), d_off.data_ptr(), len(reads),
                                       counts.data_ptr(), total.data_ptr())
            torch.cuda.synchronize(dev)
            assert int(total.item()) == want_total
            np.testing.assert_array_equal(counts.cpu().numpy().astype(np.uint64), want)


@pytest.mark.parametrize("mode,opts", [
    ("kmers", dict(k=21, H=4, b=8)),
    ("kmers", dict(k=41, H=3, b=8)),
    ("minimizers", dict(k=31, m=21, H=4, b=8)),
    ("modimizers", dict(k=25, d=4, H=4, b=8)),
    ("findere", dict(k=31, z=10, H=4, b=8)),
], ids=lambda v: v if isinstance(v, str) else "-".join(f"{a}{b}" for a, b in v.items()))
def test_homopolymer_compression(gpu, oracle, tmp_path_factory, mode, opts):
    ix, genomes = index_for(tmp_path_factory, colors=5, length=15000, seed=41, mode=mode,
                            homopolymer=True, **opts)
    reads = reads_for(genomes, n=200, length=300, n_runs=0.3, lower=0.1)
    g = genomes[0]
    reads += [b"AAAAAAAAAAAACCCCCCCCGGGGGTTTT" * 8, g[:400].replace(b"A", b"AAA"),
              b"acgtNNNNaaaaccccggggtttt" * 10, b"", b"A" * 300]
    gpu_vs_oracle(oracle, ix, reads)
    if mode != "findere":
        import zindex_b200 as zx

        bases, offsets = zx.pack_records(reads)
        with zx.Index(ix) as index:
            got = index.extract_seeds(bases, offsets)
        want = np.concatenate([oracle.features(r, mode=mode, k=opts["k"], m=opts.get("m", 21),
                                               sampling=opts.get("d", 16), homopolymer=True)
                               for r in reads])
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("opts", [
    dict(mode="kmers", k=31, H=4, b=8, groups="0,1,2;3,5"),
    dict(mode="kmers", k=25, H=3, b=1, groups="1,2"),
    dict(mode="kmers", k=31, H=4, b=16, max_size="64KiB"),
    dict(mode="minimizers", k=31, m=21, H=4, b=4, groups="0,4"),
    dict(mode="findere", k=31, z=10, H=4, b=8, groups="2,3,4"),
], ids=lambda o: "-".join(f"{a}{b}" for a, b in o.items()).replace(",", "_").replace(";", "+"))
def test_legacy_interleaved_banks(gpu, oracle, tmp_path_factory, opts):
    """Legacy ZORPOW1 banks are permuted into fingerprint-first rows at load;
    the counts must equal the oracle's, which reads the legacy layout as is."""
    ix, genomes = index_for(tmp_path_factory, colors=7, length=30000, seed=13, legacy=True, **opts)
    import json

    manifest = json.loads((ix / "manifest.json").read_text())
    assert all(not b.get("fingerprint_first", False) for b in manifest["banks"])
    gpu_vs_oracle(oracle, ix, reads_for(genomes, n=300, length=200, n_runs=0.1))


SPLIT_CASES = [
    dict(mode="minimizers", k=31, m=21, H=4, b=8),
    dict(mode="minimizers", k=21, m=21, H=3, b=16),
    dict(mode="minimizers", k=49, m=31, H=3, b=16, homopolymer=True),
    dict(mode="minimizers", k=31, m=15, H=4, b=8, pattern="##_##_###_##_##"),
]


@pytest.mark.parametrize("case", SPLIT_CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_split_minimizer_extraction_matches_oracle(gpu, oracle, tmp_path_factory, case):
    """Split minimizer queries (seeds extracted into per-tile slots by their own
    kernel, then probed) count exactly what the fused kernel and the oracle count."""
    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, colors=6, length=30000, seed=29, **case)
    reads = reads_for(genomes, n=300, length=2500, n_runs=0.1, lower=0.01)
    bases, offsets = zx.pack_records(reads)
    want, want_total = oracle.query_records(ix, bases, offsets)
    with zx.Index(ix) as index:
        for minb in (2, 1, 3):
            index.set_launch(split=1, planes=1, min_blocks=minb)
            assert index.launch()["split"] == 1
            got, total = index.query_records(bases, offsets)
            assert total == want_total, minb
            np.testing.assert_array_equal(got, want)


def test_split_rounds_equal_fused(gpu, tmp_path_factory):
    """A batch of more tiles than one split round (262,144) gives the fused
    kernel's counts, through host buffers and device graphs."""
    import torch

    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, colors=6, length=30000, seed=29, mode="minimizers",
                            k=31, m=21, H=4, b=8)
    rng = np.random.default_rng(5)
    n, length = 300_000, 120
    codes = rng.integers(0, 4, size=n * length, dtype=np.uint8)
    bases = np.frombuffer(b"ACGT", dtype=np.uint8)[codes]
    src = np.frombuffer(b"".join(genomes), dtype=np.uint8)
    for i in range(0, n, 3):  # a third of the reads copied from the genomes
        at = int(rng.integers(0, len(src) - length))
        bases[i * length:(i + 1) * length] = src[at:at + length]
    offsets = np.arange(n + 1, dtype=np.uint64) * length
    with zx.Index(ix) as index:
        index.set_launch(split=0)
        want, want_total = index.query_records(bases, offsets)
    with zx.Index(ix) as index:
        # A fresh index: the first split query is a graph capture.
        index.set_launch(split=1)
        dev = torch.device("cuda", 0)
        d_bases = torch.from_numpy(bases).to(dev)
        d_off = torch.from_numpy(offsets.view(np.int64)).to(dev)
        d_counts = torch.zeros(index.colors, dtype=torch.int64, device=dev)
        d_total = torch.zeros(1, dtype=torch.int64, device=dev)
        stream = torch.cuda.current_stream(dev)
        for _ in range(2):  # the second call replays the captured graph
            d_counts.zero_()
            d_total.zero_()
            index.query_device(d_bases.data_ptr(), len(bases), d_off.data_ptr(), n,
                               d_counts.data_ptr(), d_total.data_ptr(), stream=stream.cuda_stream)
            torch.cuda.synchronize(dev)
            assert int(d_total.item()) == want_total
            np.testing.assert_array_equal(d_counts.cpu().numpy().astype(np.uint64), want)
        got, total = index.query_records(bases, offsets)
        assert total == want_total and total > 0
        np.testing.assert_array_equal(got, want)


SPACED_CASES = [
    dict(mode="kmers", k=21, H=4, b=8, pattern="###_#_##_" + "###" + "_##_#_###"),
    dict(mode="kmers", k=31, H=3, b=16, pattern="#_" * 15 + "#", homopolymer=True),
    dict(mode="kmers", k=15, H=4, b=4, pattern="#" * 15),
    dict(mode="minimizers", k=31, m=15, H=4, b=8, pattern="##_##_###_##_##"),
    dict(mode="minimizers", k=21, m=21, H=2, b=8, pattern="##__" + "#" * 13 + "__##"),
]


@pytest.mark.parametrize("case", SPACED_CASES, ids=lambda c: f"{c['mode']}-k{c['k']}-{c['pattern']}")
def test_spaced_seeds_match_oracle(gpu, oracle, tmp_path_factory, case):
    """Spaced seeds (anchors.rs:265-281): the selected canonical k-mers or
    minimizers mapped through the pattern, counted as the oracle counts them."""
    ix, genomes = index_for(tmp_path_factory, colors=5, length=20000, seed=23, **case)
    reads = reads_for(genomes, n=400, length=180, n_runs=0.1, lower=0.01)
    gpu_vs_oracle(oracle, ix, reads)
    gpu_vs_oracle(oracle, ix, reads, recover=False)


@pytest.mark.parametrize("colors,length,legacy", [
    (16, 1100000, False),  # 32-byte rows (64 MiB): pieces go straight to the resident rows
    (20, 900000, False),   # 40-byte rows (48-byte stride, 40 MiB): staged and repacked
    (20, 900000, True),    # legacy rows: staged and permuted
])
def test_multi_frame_banks_stream_into_hbm(gpu, oracle, tmp_path_factory, colors, length, legacy):
    """Banks of many 4 MiB zstd frames and several 32 MiB upload pieces (frames
    straddle piece boundaries) load to the same filters the oracle reads."""
    import json

    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, colors=colors, length=length, seed=17, k=31, H=4,
                            b=16, legacy=legacy)
    manifest = json.loads((ix / "manifest.json").read_text())
    raw = sum(b["slots"] * ((b["row_bits"] + 7) // 8) for b in manifest["banks"])
    assert raw > (32 << 20), raw
    with zx.Index(ix) as index:
        info = index.info
        assert info.load_s >= info.load_banks_s > 0
    gpu_vs_oracle(oracle, ix, reads_for(genomes, n=400, length=150, n_runs=0.1))


@pytest.mark.parametrize("mode", ["kmers", "findere"])
def test_pipelined_host_chunks_equal_one_pass(gpu, oracle, tmp_path_factory, mode):
    """A host batch cut into record-aligned chunks (copies overlapping the
    previous chunk's kernels) gives the counts of one pass and the oracle's."""
    import zindex_b200 as zx

    opts = dict(mode=mode, k=31, H=4, b=8) if mode == "kmers" else dict(mode=mode, k=31, z=6,
                                                                       H=4, b=8)
    ix, genomes = index_for(tmp_path_factory, colors=6, length=30000, **opts)
    reads = reads_for(genomes, n=24000, length=150, n_runs=0.05)
    bases, offsets = zx.pack_records(reads)
    want, want_total = oracle.query_records(ix, bases, offsets)
    with zx.Index(ix) as index:
        for cut in (1, 3, 64):
            index.set_launch(cut=cut)
            got, total = index.query_records(bases, offsets)
            assert total == want_total, cut
            np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("colors,H,b,groups", [
    (600, 2, 8, "1,2"),         # 38 chunks, H = 2: the chunk pipeline with two rows
    (1500, 4, 4, "0,1,2;7,9"),   # 47 chunks per row: two shared-plane words per lane
    (2048, 3, 16, "5,6,7,8"),    # 256 chunks per row (4 KiB)
])
def test_wide_rows_shared_planes(gpu, oracle, tmp_path_factory, colors, H, b, groups):
    """Rows wider than one register plane word per lane count in shared planes."""
    ix, genomes = index_for(tmp_path_factory, colors=colors, length=3000, seed=61, mode="kmers",
                            k=25, H=H, b=b, groups=groups)
    reads = reads_for(genomes, n=600, length=150, n_runs=0.05)
    gpu_vs_oracle(oracle, ix, reads, recover=True)
    gpu_vs_oracle(oracle, ix, reads, recover=False)
    import zindex_b200 as zx

    bases, offsets = zx.pack_records(reads)
    want, want_total = oracle.query_records(ix, bases, offsets)
    with zx.Index(ix) as index:
        for team, warps, minb in ((32, 8, 2), (16, 4, 2), (8, 2, 2), (32, 4, 1), (8, 4, 1)):
            index.set_launch(team=team, warps=warps, planes=1, smem_counters=0, min_blocks=minb)
            got, total = index.query_records(bases, offsets)
            assert total == want_total
            np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("mode", ["kmers", "homopolymer"])
def test_invalid_offsets_are_reported_and_skipped(gpu, oracle, tmp_path_factory, mode):
    """Decreasing interior offsets (and offsets past the bases) are checked on
    the device: the query fails with ZX_EINVAL, no memory outside the batch is
    touched, and the index keeps answering correctly."""
    import torch

    import zindex_b200 as zx

    opts = dict(mode="kmers", k=31, H=4, b=8, homopolymer=(mode == "homopolymer"))
    ix, genomes = index_for(tmp_path_factory, colors=4, length=20000, seed=71, **opts)
    reads = reads_for(genomes, n=2000, length=150)
    bases, offsets = zx.pack_records(reads)
    bad = offsets.copy()
    bad[5] = bad[7] + 40          # record 5 ends before it starts; record 4 runs long
    bad[9] = len(bases) + 10**9   # an interior offset past the bases
    want, want_total = oracle.query_records(ix, bases, offsets)
    with zx.Index(ix) as index:
        with pytest.raises(zx.ZxError) as err:
            index.query_records(bases, bad)
        assert err.value.code == 1 and "offsets" in str(err.value)
        got, total = index.query_records(bases, offsets)
        assert total == want_total
        np.testing.assert_array_equal(got, want)
        dev = torch.device("cuda", 0)
        d_b = torch.from_numpy(bases).to(dev)
        d_bad = torch.from_numpy(bad.view(np.int64)).to(dev)
        counts = torch.zeros(index.colors, dtype=torch.int64, device=dev)
        total_d = torch.zeros(1, dtype=torch.int64, device=dev)
        for fn in (lambda: index.query_device(d_b.data_ptr(), len(bases), d_bad.data_ptr(),
                                              len(reads), counts.data_ptr(), total_d.data_ptr(),
                                              use_graph=False),
                   lambda: index.query_device_noalloc(d_b.data_ptr(), len(bases), d_bad.data_ptr(),
                                                      len(reads), counts.data_ptr(),
                                                      total_d.data_ptr())):
            try:
                fn()
            except zx.ZxError:
                continue  # refused before any launch
            torch.cuda.synchronize(dev)
            with pytest.raises(zx.ZxError) as err:
                index.query_status()
            assert err.value.code == 1
        got, total = index.query_records(bases, offsets)
        assert total == want_total
        np.testing.assert_array_equal(got, want)


def test_multi_member_groups(gpu, oracle, tmp_path_factory):
    ix, genomes = index_for(tmp_path_factory, colors=8, mode="kmers", k=31, H=4, b=4,
                            groups="0,1,2;3,5;6,7")
    gpu_vs_oracle(oracle, ix, reads_for(genomes, n=400))


def test_hash_partitions(gpu, oracle, tmp_path_factory):
    ix, genomes = index_for(tmp_path_factory, colors=6, length=60000, mode="kmers", k=31, H=4,
                            b=8, max_size="64KiB")
    import json

    manifest = json.loads((ix / "manifest.json").read_text())
    assert any("routing" in b for b in manifest["banks"]), "expected a partitioned class"
    gpu_vs_oracle(oracle, ix, reads_for(genomes, n=400))


def test_promoted_size_classes(gpu, oracle, tmp_path_factory):
    d = tmp_path_factory.mktemp("classes")
    genomes = [dna(n, 77 + i) for i, n in enumerate([3000, 9000, 20000, 70000, 5000])]
    lines = []
    for i, g in enumerate(genomes):
        p = d / f"g{i}.fa"
        helpers.write_fasta(p, [g])
        lines.append(f"g{i}\t{p}")
    (d / "fof.tsv").write_text("\n".join(lines) + "\n")
    ix = build_index(d / "fof.tsv", d / "index", k=31, H=4, b=8, min_docs=1)
    gpu_vs_oracle(oracle, ix, reads_for(genomes, n=300))


def test_recovery_disabled_and_dropped(gpu, oracle, tmp_path_factory):
    ix, genomes = index_for(tmp_path_factory, mode="kmers", k=31, H=4, b=8)
    reads = reads_for(genomes, n=300)
    with_rec, _ = gpu_vs_oracle(oracle, ix, reads, recover=True)
    without, _ = gpu_vs_oracle(oracle, ix, reads, recover=False)
    assert (with_rec >= without).all()
    ix2, genomes2 = index_for(tmp_path_factory, seed=9, mode="kmers", k=31, H=4, b=8,
                              drop_abandoned=True)
    gpu_vs_oracle(oracle, ix2, reads_for(genomes2, n=200))


def test_edge_records(gpu, oracle, tmp_path_factory):
    ix, genomes = index_for(tmp_path_factory, mode="kmers", k=31, H=4, b=8)
    g = genomes[0]
    records = [b"", b"ACGT", g[:30], g[:31], b"N" * 100, g[:500].lower(),
               g[1000:1100] + b"NNN" + g[2000:2100], b"acgtn" * 40, g[:2000],
               bytes(g[5000:5300].replace(b"A", b"R"))]
    gpu_vs_oracle(oracle, ix, records)
    gpu_vs_oracle(oracle, ix, [])


def test_plain_form_equals_batched(gpu, oracle, tmp_path_factory):
    ix, genomes = index_for(tmp_path_factory, mode="kmers", k=31, H=4, b=8)
    reads = reads_for(genomes, n=40, length=300)
    batched, t1 = gpu_vs_oracle(oracle, ix, reads)
    plain, t2 = gpu_vs_oracle(oracle, ix, reads, plain=True)
    np.testing.assert_array_equal(batched, plain)
    assert t1 == t2


@pytest.mark.parametrize("mode,case", [
    ("kmers", dict(k=31)), ("kmers", dict(k=32)), ("kmers", dict(k=45)), ("kmers", dict(k=1)),
    ("minimizers", dict(k=49, m=31)), ("minimizers", dict(k=31, m=15)),
    ("minimizers", dict(k=7, m=7)), ("modimizers", dict(k=31, d=3)),
    ("modimizers", dict(k=40, d=5)),
], ids=lambda v: str(v))
def test_extraction_matches_oracle_in_order(gpu, oracle, tmp_path_factory, mode, case):
    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, colors=2, length=5000, mode=mode, H=4, b=8, **case)
    rng = np.random.default_rng(3)
    records = [helpers.mutate(dna(int(rng.integers(0, 3000)), s), rng, n_runs=3, lower=0.05)
               for s in range(40)]
    records += [b"", b"N" * 50, dna(70000, 99)]
    bases, offsets = zx.pack_records(records)
    with zx.Index(ix) as index:
        got = index.extract_seeds(bases, offsets)
    k = case["k"]
    want = np.concatenate([oracle.features(r, mode=mode, k=k, m=case.get("m", 21),
                                           sampling=case.get("d", 16)) for r in records])
    np.testing.assert_array_equal(got, want)


def test_cli_output_is_byte_identical(gpu, oracle, tmp_path_factory):
    ix, genomes = index_for(tmp_path_factory, mode="kmers", k=31, H=4, b=8)
    q = tmp_path_factory.mktemp("cli") / "q.fa"
    helpers.write_fasta(q, reads_for(genomes, n=100))
    ours = subprocess.run([str(helpers.ZORINDEX), "query", "-i", str(ix), "-q", str(q)],
                          check=True, capture_output=True)
    ref = subprocess.run([str(helpers.ORACLE_DIR / "_build" / "zx_oracle"), "query", "-i", str(ix),
                          "-q", str(q)], check=True, capture_output=True)
    assert ours.stdout == ref.stdout
    ours_stats = [l for l in ours.stderr.decode().splitlines() if l.startswith("#query")][0]
    ref_stats = [l for l in ref.stderr.decode().splitlines() if l.startswith("#query")][0]
    assert ours_stats.split("elapsed_s")[0] == ref_stats.split("elapsed_s")[0]
    for ratio in ("0.001", "0.5"):
        a = subprocess.run([str(helpers.ZORINDEX), "query", "-i", str(ix), "-q", str(q), "-a", ratio],
                           check=True, capture_output=True)
        b = subprocess.run([str(helpers.ORACLE_DIR / "_build" / "zx_oracle"), "query", "-i", str(ix),
                            "-q", str(q), "-a", ratio], check=True, capture_output=True)
        assert a.stdout == b.stdout


def test_device_api_with_graph_replay(gpu, oracle, tmp_path_factory):
    import torch

    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, mode="kmers", k=31, H=4, b=8)
    reads = reads_for(genomes, n=500)
    bases, offsets = zx.pack_records(reads)
    want, want_total = oracle.query_records(ix, bases, offsets)
    dev = torch.device("cuda:0")
    d_bases = torch.from_numpy(bases).to(dev)
    d_off = torch.from_numpy(offsets.view(np.int64)).to(dev)
    with zx.Index(ix) as index:
        for _ in range(3):
            d_counts = torch.zeros(index.colors, dtype=torch.int64, device=dev)
            d_total = torch.zeros(1, dtype=torch.int64, device=dev)
            stream = torch.cuda.current_stream().cuda_stream
            index.query_device(d_bases.data_ptr(), len(bases), d_off.data_ptr(), len(reads),
                               d_counts.data_ptr(), d_total.data_ptr(), stream=stream)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(d_counts.cpu().numpy().astype(np.uint64), want)
            assert int(d_total.item()) == want_total


LAUNCHES = [
    dict(team=1, warps=4, stage_bytes=0), dict(team=2, warps=2, stage_bytes=0),
    dict(team=8, warps=8, stage_bytes=0), dict(team=32, warps=1, stage_bytes=0),
    dict(team=16, warps=3, stage_bytes=0),
    dict(team=1, warps=4, planes=1), dict(team=2, warps=3, planes=1),
    dict(team=8, warps=8, planes=1, min_blocks=2), dict(team=32, warps=1, planes=1),
    dict(team=4, warps=8, planes=1, min_blocks=2), dict(team=16, warps=8, planes=1),
    dict(team=1, warps=4, planes=1, min_blocks=1), dict(team=2, warps=8, planes=1, min_blocks=1),
    dict(warps=4, stage_bytes=8192, stages=2, bulk=1), dict(warps=8, stage_bytes=4096, stages=3, bulk=1),
    dict(warps=2, stage_bytes=64, stages=1, bulk=1), dict(warps=4, stage_bytes=128, stages=4, bulk=1),
    dict(warps=1, stage_bytes=16384, stages=8, bulk=1),
    dict(warps=4, stage_bytes=8192, stages=2, bulk=0), dict(warps=8, stage_bytes=4096, stages=3, bulk=0),
    dict(warps=2, stage_bytes=64, stages=1, bulk=0), dict(warps=4, stage_bytes=128, stages=4, bulk=0),
    dict(warps=1, stage_bytes=16384, stages=8, bulk=0),
]


@pytest.mark.parametrize("launch", LAUNCHES, ids=lambda l: "-".join(f"{k}{v}" for k, v in l.items()))
def test_launch_configurations_do_not_change_results(gpu, oracle, tmp_path_factory, launch):
    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, colors=40, length=4000, mode="kmers", k=31, H=4, b=8)
    reads = reads_for(genomes, n=300)
    bases, offsets = zx.pack_records(reads)
    want, want_total = oracle.query_records(ix, bases, offsets)
    with zx.Index(ix) as index:
        for smem in (0, 1):
            index.set_launch(smem_counters=smem, **launch)
            got, total = index.query_records(bases, offsets)
            np.testing.assert_array_equal(got, want)
            assert total == want_total


@pytest.mark.parametrize("stage_bytes,stages,bulk,planes", [
    (0, 0, 0, 0), (0, 0, 0, 1), (8192, 2, 1, 0), (256, 3, 1, 0), (64, 2, 1, 0), (8192, 2, 0, 0),
    (256, 3, 0, 0), (64, 2, 0, 0)])
def test_gathers_on_wide_partitioned_multiclass_index(gpu, oracle, tmp_path_factory,
                                                      stage_bytes, stages, bulk, planes):
    import zindex_b200 as zx

    d = tmp_path_factory.mktemp("wide")
    lengths = [2000 + 37 * i for i in range(300)] + [40000 + 1000 * i for i in range(12)]
    lines = []
    genomes = []
    for i, n in enumerate(lengths):
        g = dna(n, 500 + i)
        genomes.append(g)
        p = d / f"g{i}.fa"
        helpers.write_fasta(p, [g])
        lines.append(f"g{i}\t{p}")
    (d / "fof.tsv").write_text("\n".join(lines) + "\n")
    ix = build_index(d / "fof.tsv", d / "index", k=31, H=4, b=16, min_docs=1, max_size="256KiB",
                     groups="3,4,5,6;10,11")
    reads = reads_for(genomes, n=400)
    bases, offsets = zx.pack_records(reads)
    want, want_total = oracle.query_records(ix, bases, offsets)
    with zx.Index(ix) as index:
        assert index.info.classes >= 2
        index.set_launch(stage_bytes=stage_bytes, stages=stages or 1, bulk=bulk, planes=planes)
        got, total = index.query_records(bases, offsets)
    np.testing.assert_array_equal(got, want)
    assert total == want_total
