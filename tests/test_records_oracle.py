"""The oracle's per-record report (`zorindex query --records`) pinned on the CPU.

The reference's own record test (tests/power_merge_cli.rs:1170-1230) states
the contract: every record's row equals an aggregate query of that record
alone, formatted as record_output.rs:21-62 writes it, whatever the record batch
size. Here the expected rows are formatted in Python from the oracle's
aggregate query of each record alone, and the quoting rule is pinned by the
reference's unit test (record_output.rs:90-112). Reader rules and errors follow
read_batches (records.rs:150-290).
"""
import numpy as np
import pytest

import helpers
from helpers import build_index, dna, sample_reads


def _field(v: str) -> str:
    # CSV quoting of record_output.rs:64-80.
    if any(c in v for c in "\t\r\n\""):
        return '"' + v.replace('"', '""') + '"'
    return v


def _expected(per_record, names, colors, min_ratio, fmt):
    out = ["query_id\tvalid_kmers\thits" if fmt == "compact"
           else "query_id\tdataset_id\tdataset_name\tmatches\tqueried_seeds\tratio"]
    for name, (counts, total) in zip(names, per_record):
        hits = []
        for c, n in enumerate(counts):
            n = int(n)
            if min_ratio == 0.0 or (total and n and n / total >= min_ratio):
                hits.append((c, n))
        if fmt == "compact":
            out.append(f"{name}\t{total}\t" + ",".join(f"{c}:{n}" for c, n in hits))
            continue
        for c, n in hits:
            ratio = n / total if total else 0.0
            out.append(f"{_field(name)}\t{c}\t{_field(colors[c])}\t{n}\t{total}\t{ratio:.8f}")
        if not hits:
            out.append(f"{_field(name)}\t.\t.\t0\t{total}\t0.00000000")
    return ("\n".join(out) + "\n").encode()


@pytest.fixture(scope="module")
def small_index(native, tmp_path_factory):
    d = tmp_path_factory.mktemp("rec")
    names = ["a", 'b"quoted"', "c"]
    lines = []
    for c, name in enumerate(names):
        p = d / f"g{c}.fa"
        helpers.write_fasta(p, [dna(4000, 300 + c)])
        lines.append(f"{name}\t{p}")
    (d / "fof.tsv").write_text("\n".join(lines) + "\n")
    return build_index(d / "fof.tsv", d / "index", k=21, H=3, b=8), names


def _records(seed=7, n=40):
    genomes = [dna(4000, 300 + c) for c in range(3)]
    rng = np.random.default_rng(seed)
    reads = sample_reads(genomes, rng, n, 120, n_runs=0.2)
    reads += [b"", b"ACGT", genomes[1][100:1100], b"N" * 50]
    names = [f"r{i}" for i in range(len(reads))]
    names[3] = 'q"x'  # quoted in TSV, raw in compact
    return names, reads


def _write_fasta(path, names, reads):
    with open(path, "wb") as f:
        for name, r in zip(names, reads):
            f.write(b">" + name.encode() + b" description\n")
            for j in range(0, len(r), 60):
                f.write(r[j: j + 60] + b"\n")
    return path


@pytest.mark.parametrize("min_ratio", [0.0, 0.4, 1.0])
@pytest.mark.parametrize("fmt", ["tsv", "compact"])
def test_report_equals_single_record_aggregates(oracle, small_index, tmp_path, min_ratio, fmt):
    index, colors = small_index
    names, reads = _records()
    query = _write_fasta(tmp_path / "q.fa", names, reads)
    per_record = []
    for r in reads:
        bases = np.frombuffer(r, dtype=np.uint8) if r else np.zeros(0, dtype=np.uint8)
        counts, total = oracle.query_records(index, bases, np.array([0, len(r)], dtype=np.uint64))
        per_record.append((counts, total))
    want = _expected(per_record, names, colors, min_ratio, fmt)
    assert oracle.records_report(index, query, min_ratio=min_ratio, fmt=fmt) == want


def test_fastq_crlf_and_multiline(oracle, small_index, tmp_path):
    index, _ = small_index
    names, reads = _records(seed=9, n=12)
    fa = _write_fasta(tmp_path / "q.fa", names, reads)
    fq = tmp_path / "q.fq"
    with open(fq, "wb") as f:
        for name, r in zip(names, reads):
            half = len(r) // 2
            # Multi-line FASTQ sequence and quality, CRLF line ends, blank lines.
            f.write(b"@" + name.encode() + b"\r\n" + r[:half] + b"\r\n" + r[half:] + b"\r\n+\r\n")
            f.write(b"I" * half + b"\r\n" + b"I" * (len(r) - half) + b"\r\n\r\n")
    assert oracle.records_report(index, fq) == oracle.records_report(index, fa)


@pytest.mark.parametrize("text,message", [
    (b"ACGT\n", "--records requires FASTA or FASTQ"),
    (b"", "no FASTA/FASTQ records"),
    (b"\n\n  \n", "no FASTA/FASTQ records"),
    (b">r1\nAC GT\n", "whitespace inside FASTA sequence"),
    (b">\nACGT\n", "empty FASTA identifier"),
    (b"@r1\nACGT\n+\nII\n", "truncated FASTQ quality"),
    (b"@r1\nACGT\n+\nIIIII\n", "FASTQ sequence and quality lengths differ"),
    (b"@r1\nACGT\n", "truncated FASTQ sequence"),
    (b">r\xff\nACGT\n", "invalid FASTA identifier"),
])
def test_reader_errors(oracle, small_index, tmp_path, text, message):
    index, _ = small_index
    q = tmp_path / "bad.fa"
    q.write_bytes(text)
    with pytest.raises(RuntimeError, match=message):
        oracle.records_report(index, q)
