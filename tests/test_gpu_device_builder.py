"""The device builder (zx_build --device) against the host builder.

Both build the same datasets; the bank layout (files, slots, row widths,
groups, partitions) and the per-dataset counts of the manifest must be the
same, the device-built index must answer every query exactly as the oracle
reads it (recovery on and off), and its rows must hold every key that is not
in its recovery file, read by the independent Python reader of the row
format (tests/test_row_format_pin.py). Its filter cells may differ from the
host builder's: the peel order and the abandoned keys are the builder's
choice, and the query reads any valid solution the same way.
"""
import json
import subprocess

import numpy as np
import pytest

import helpers
from test_row_format_pin import get_bits, positions, read_bank, read_recovery, recovery_hash, splitmix64

pytestmark = pytest.mark.gpu

CASES = [
    dict(k=31, H=4, b=8),
    dict(k=25, H=8, b=4, min_docs=1, max_size="16KiB"),
    dict(mode="minimizers", k=31, m=21, H=3, b=16),
    dict(mode="modimizers", k=31, H=4, b=4, d=4),
    dict(k=45, H=5, b=32),
    dict(k=11, H=2, b=1, pattern="####_#_####"),
]

LAYOUT = ("file", "slots", "row_bits", "routing")


def _build(fof, out, device, **opts):
    helpers.build_index(fof, out, **opts)  # host
    return out


def _device_index(fof, out, **opts):
    args = [str(helpers.ZX_BUILD), "-f", str(fof), "-o", str(out), "-q", "--device"]
    flag = {"k": "-k", "m": "-m", "H": "-H", "b": "-b", "mode": "-i", "d": "-d",
            "min_docs": "-D", "max_size": "-X", "pattern": "-p"}
    for key, val in opts.items():
        args += [flag[key], str(val)]
    subprocess.run(args, check=True)
    return out


def _rows_hold_keys(index, keys_of):
    m = json.loads((index / "manifest.json").read_text())
    seed, H, b = m["seed"], m["hashes"], m["fingerprint_bits"]
    rec = (read_recovery(index / m["abandoned_file"], seed)
           if m.get("abandoned_recovery") and m.get("abandoned_hashes") else {})
    routed = {}
    for bank in m["banks"]:
        r = bank.get("routing")
        routed.setdefault(r["source_slots"] if r else bank["slots"], []).append(bank)
    held = lost = 0
    for banks in routed.values():
        banks.sort(key=lambda bk: (bk.get("routing") or {"partition": 0})["partition"])
        payloads = [read_bank(index / bk["file"])[40:] for bk in banks]
        bank, P = banks[0], len(banks)
        rb = (bank["row_bits"] + 7) // 8
        for gi, g in enumerate(bank["groups"]):
            c = g["members"][0]
            for key in sorted(keys_of[c])[:300]:
                part = splitmix64(key ^ seed ^ 0x34B61D8F29A7C053) & (P - 1) if P > 1 else 0
                fp = 0
                for cell in positions(key, seed, bank["slots"], H, m.get("segment_length")):
                    fp ^= get_bits(payloads[part][cell * rb: (cell + 1) * rb], gi * b, b)
                if fp == splitmix64(key ^ seed ^ 0x8E2D4F6A9B13C5D7) & ((1 << b) - 1):
                    held += 1
                else:
                    assert c in rec.get(recovery_hash(key, seed), set()), (key, c)
                    lost += 1
    return held, lost


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_device_builder_matches_host_layout_and_queries(gpu, oracle, tmp_path, case):
    import zindex_b200 as zx

    lengths = [3000, 9000, 25000, 60000, 7000, 40000]
    genomes = [helpers.dna(n, 91 + c) for c, n in enumerate(lengths)]
    lines = []
    for c, g in enumerate(genomes):
        p = helpers.write_fasta(tmp_path / f"g{c}.fa", [g[: len(g) // 3], g[len(g) // 3:]])
        lines.append(f"g{c}\t{p}")
    (tmp_path / "fof.tsv").write_text("\n".join(lines) + "\n")
    fof = tmp_path / "fof.tsv"
    host = _build(fof, tmp_path / "host", False, **case)
    dev = _device_index(fof, tmp_path / "dev", **case)
    mh = json.loads((host / "manifest.json").read_text())
    md = json.loads((dev / "manifest.json").read_text())
    for key in ("version", "k", "hashes", "fingerprint_bits", "index_mode", "segment_length",
                "seed_pattern"):
        assert mh.get(key) == md.get(key), key
    assert [(c["name"], c["occurrences"], c["unique_kmers"]) for c in mh["colors"]] == \
        [(c["name"], c["occurrences"], c["unique_kmers"]) for c in md["colors"]]
    assert [{k: b.get(k) for k in LAYOUT} for b in mh["banks"]] == \
        [{k: b.get(k) for k in LAYOUT} for b in md["banks"]]
    assert [[(g["members"], g["width"], g["offset"]) for g in b["groups"]] for b in mh["banks"]] == \
        [[(g["members"], g["width"], g["offset"]) for g in b["groups"]] for b in md["banks"]]
    reads = helpers.sample_reads(genomes, np.random.default_rng(4), 500, 150, n_runs=0.1)
    bases, offsets = zx.pack_records(reads)
    with zx.Index(dev) as ix:
        for recover in (True, False):
            want, want_total = oracle.query_records(dev, bases, offsets, recover=recover)
            got, total = ix.query_records(bases, offsets, recover=recover)
            assert total == want_total
            np.testing.assert_array_equal(got, want)
    if case.get("mode", "kmers") == "kmers" and "pattern" not in case:
        # Each genome is two records: k-mers across the cut are not indexed.
        keys = [set(int(x) for x in oracle.features(g[: len(g) // 3], mode="kmers", k=case["k"])) |
                set(int(x) for x in oracle.features(g[len(g) // 3:], mode="kmers", k=case["k"]))
                for g in genomes]
        held, lost = _rows_hold_keys(dev, keys)
        assert held > 1000 and lost < held // 10


def test_device_builder_on_the_bundled_bacteria(gpu, oracle, tmp_path):
    """The reference's bundled genomes (gzip FASTA through a file of files):
    the README's unique_kmers and the source genome's 970/970."""
    from test_gpu_bacteria import DATA, GOLDEN, _fof

    import zindex_b200 as zx

    fof, names = _fof(tmp_path)
    dev = _device_index(fof, tmp_path / "dev", k=31)
    m = json.loads((dev / "manifest.json").read_text())
    for c in m["colors"]:
        if c["name"] in GOLDEN["unique_kmers"]:
            assert c["unique_kmers"] == GOLDEN["unique_kmers"][c["name"]]
    with zx.Index(dev) as ix:
        counts, total, _ = ix.query_file(DATA / "query.fa")
    assert total == GOLDEN["query_kmers"]
    assert counts[names.index(GOLDEN["source_genome"])] == GOLDEN["source_matches"]
