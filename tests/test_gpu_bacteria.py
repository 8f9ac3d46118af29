"""The reference's end-to-end truth on its bundled bacteria, on the GPU.

utils/scripts/demo.sh:36-43 of the reference builds a k-mer index (k 31) and a
minimizer index (k 49, m 31) of the ten bundled genomes, queries queries.fa
(a 1-kb fragment of each genome, its reverse complement and a random
negative) with `--records --min-ratio 0.8`, and checks every positive with
prepare_bacteria_example.py --check-results (lines 144-177): the record's
source dataset must match every one of the record's queried seeds. The same
check runs here on the GPU report, which must also equal the oracle's report
byte for byte. The data are the reference's files, copied into
tests/golden/bacteria by tests/golden/make_bacteria_fixture.py.

The README's aggregate example (README.md:58-62) is checked on the columns
that do not depend on the builder's filter cells: the source genome matches
all 970 query 31-mers with ratio 1, and unique_kmers of the first rows.
"""
import csv
import io
import json
from pathlib import Path

import pytest

import helpers

pytestmark = pytest.mark.gpu

DATA = Path(__file__).parent / "golden" / "bacteria"
GOLDEN = json.loads((Path(__file__).parent / "golden" / "bacteria_readme.json").read_text())
MODES = {"kmers": dict(k=31), "minimizers": dict(mode="minimizers", k=49, m=31)}


def _fof(tmp_path):
    lines = []
    for line in (DATA / "samples.fof").read_text().splitlines():
        name, rel = line.split("\t")
        lines.append(f"{name}\t{DATA / rel}")
    (tmp_path / "fof.tsv").write_text("\n".join(lines) + "\n")
    return tmp_path / "fof.tsv", [l.split("\t")[0] for l in lines]


def _check_results(report: str, names):
    """prepare_bacteria_example.py --check-results on a TSV report: one row per
    (record, reported dataset), grouped per record; each positive's source
    must have as many matches as the record has queried seeds."""
    truth = list(csv.DictReader((DATA / "source-truth.tsv").open(newline=""), delimiter="\t"))
    rows = list(csv.DictReader(io.StringIO(report), delimiter="\t"))
    grouped = []
    for row in rows:
        if not grouped or grouped[-1]["query_id"] != row["query_id"]:
            grouped.append({"query_id": row["query_id"], "valid": int(row["queried_seeds"]),
                            "hits": {}})
        assert int(row["queried_seeds"]) == grouped[-1]["valid"], "inconsistent seed counts"
        if row["dataset_id"] != ".":
            grouped[-1]["hits"][int(row["dataset_id"])] = int(row["matches"])
    assert [g["query_id"] for g in grouped] == [t["query_id"] for t in truth]
    positives = 0
    for g, t in zip(grouped, truth):
        if t["document_id"] == "-":
            assert not g["hits"], f"random negative reported {g['hits']}"
            continue
        doc = int(t["document_id"])
        assert names[doc] == t["accession"]
        assert g["valid"] > 0 and g["hits"].get(doc) == g["valid"], (g, t)
        positives += 1
    return positives


@pytest.mark.parametrize("mode", sorted(MODES))
def test_bacteria_source_truth_on_the_gpu(gpu, oracle, tmp_path, mode):
    import zindex_b200 as zx

    fof, names = _fof(tmp_path)
    index = helpers.build_index(fof, tmp_path / "index", **MODES[mode])
    out = tmp_path / "hits.tsv"
    with zx.Index(index) as ix:
        ix.query_records_report(DATA / "queries.fa", out, min_ratio=0.8, fmt="tsv")
    got = out.read_bytes()
    assert got == oracle.records_report(index, DATA / "queries.fa", min_ratio=0.8, fmt="tsv")
    assert _check_results(got.decode(), names) == 20


def test_bacteria_readme_aggregate_on_the_gpu(gpu, oracle, tmp_path):
    import zindex_b200 as zx

    fof, names = _fof(tmp_path)
    index = helpers.build_index(fof, tmp_path / "index", k=GOLDEN["k"])
    with zx.Index(index) as ix:
        counts, total, _ = ix.query_file(DATA / "query.fa")
        text = ix.format_aggregate(counts, total)
    want, want_total, _ = oracle.query_file(index, DATA / "query.fa")
    assert total == want_total == GOLDEN["query_kmers"]
    assert counts.tolist() == want.tolist()
    rows = {r.split("\t")[0]: r.split("\t") for r in text.splitlines()[1:]}
    src = rows[GOLDEN["source_genome"]]
    assert src[1:3] == [str(GOLDEN["source_matches"]), "1.00000000"]
    for name, unique in GOLDEN["unique_kmers"].items():
        assert rows[name][3] == str(unique)
