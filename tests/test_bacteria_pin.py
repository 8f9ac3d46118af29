"""Pins the oracle to the reference's published bacteria example.

The reference README (lines 60-62) lists, for its bundled genomes, the
distinct indexed 31-mers per dataset (`unique_kmers`) and states that the
source genome of tests/data/bacteria/query.fa matches all 970 query 31-mers
(guaranteed by recovery, README.md:65-66). The expected numbers are committed
in tests/golden/bacteria_readme.json and the genomes are the reference's
bundled files, copied byte for byte into tests/golden/bacteria by
tests/golden/make_bacteria_fixture.py. The false-positive count of the third
row depends on the exact filter cells of the reference builder and is not
pinned.
"""
import gzip
import json
from pathlib import Path

import numpy as np
import pytest

import helpers

REF = Path(__file__).parent / "golden" / "bacteria"
GOLDEN = json.loads((Path(__file__).parent / "golden" / "bacteria_readme.json").read_text())


def fasta_records(path):
    opener = gzip.open if str(path).endswith(".gz") else open
    seq, out = [], []
    with opener(path, "rt") as f:
        for line in f:
            if line.startswith(">"):
                if seq:
                    out.append("".join(seq).encode())
                seq = []
            else:
                seq.append(line.strip())
    if seq:
        out.append("".join(seq).encode())
    return out


def test_unique_kmers_of_the_bundled_genomes(oracle):
    for acc, want in GOLDEN["unique_kmers"].items():
        keys = [oracle.features(r, mode="kmers", k=GOLDEN["k"])
                for r in fasta_records(REF / "genomes" / f"{acc}.fna.gz")]
        assert len(np.unique(np.concatenate(keys))) == want, acc


def test_source_genome_matches_every_query_kmer(oracle, tmp_path):
    lines = [f"{acc}\t{REF / 'genomes' / (acc + '.fna.gz')}" for acc in GOLDEN["unique_kmers"]]
    (tmp_path / "fof.tsv").write_text("\n".join(lines) + "\n")
    index = helpers.build_index(tmp_path / "fof.tsv", tmp_path / "index", k=GOLDEN["k"], H=4, b=8)
    counts, total, _ = oracle.query_file(index, REF / "query.fa")
    names = list(GOLDEN["unique_kmers"])
    assert total == GOLDEN["query_kmers"]
    assert counts[names.index(GOLDEN["source_genome"])] == GOLDEN["source_matches"]
    manifest = json.loads((index / "manifest.json").read_text())
    for c in manifest["colors"]:
        assert c["unique_kmers"] == GOLDEN["unique_kmers"][c["name"]]


@pytest.mark.parametrize("mode", ["kmers", "minimizers"])
def test_oracle_report_meets_the_bacteria_source_truth(oracle, tmp_path, mode):
    """The reference's end-to-end check (utils/scripts/demo.sh:36-43 and
    prepare_bacteria_example.py:144-177) on the oracle's `--records
    --min-ratio 0.8` report: every positive record's source dataset matches
    all of its queried seeds, and the random negative reports nothing."""
    from test_gpu_bacteria import MODES, _check_results, _fof

    fof, names = _fof(tmp_path)
    index = helpers.build_index(fof, tmp_path / "index", **MODES[mode])
    report = oracle.records_report(index, REF / "queries.fa", min_ratio=0.8, fmt="tsv")
    assert _check_results(report.decode(), names) == 20
