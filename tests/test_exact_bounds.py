"""Membership bounds against exact k-mer sets (CPU): the restated query never
loses a k-mer a document really holds and never counts more than the query's
k-mers, for every fingerprint width, with recovery on. Restates the
reference's canonical-string oracle test (tests/option_coverage_cli.rs:
137-245): shared segments, a reverse-complemented copy, ambiguity breaks,
lowercase, repeated keys, records shorter than k and empty documents.
"""
import numpy as np
import pytest

import helpers
from helpers import dna

K = 31


def _rc(s: bytes) -> bytes:
    return s[::-1].translate(bytes.maketrans(b"ACGTacgt", b"TGCAtgca"))


def exact_kmers(s: bytes):
    """Canonical k-mers of every all-ACGT window (case-insensitive)."""
    out = []
    s = s.upper()
    for i in range(len(s) - K + 1):
        w = s[i:i + K]
        if all(c in b"ACGT" for c in w):
            out.append(min(w, _rc(w)))
    return out


@pytest.mark.parametrize("bits", [1, 2, 4, 8, 16])
def test_counts_bracket_exact_membership(oracle, tmp_path, bits):
    shared = dna(210, 37).upper()
    documents = [
        shared + b"NNN" + dna(90, 11).upper(),
        _rc(shared) + b"NNN" + dna(90, 12).upper(),
        dna(370, 13).upper(),
        b"ACGTNacgt",
        b"NNNNNN",
    ]
    sets = [set(exact_kmers(d)) for d in documents]
    lines = []
    for i, d in enumerate(documents):
        p = tmp_path / f"d{i}.fa"
        p.write_bytes(b">a\n" + d + b"\n")
        lines.append(f"d{i}\t{p}")
    (tmp_path / "fof.tsv").write_text("\n".join(lines) + "\n")
    index = helpers.build_index(tmp_path / "fof.tsv", tmp_path / "ix", k=K, H=4, b=bits,
                                min_docs=1)
    queries = [
        shared.lower(),
        _rc(shared),
        shared[:61] + b"NN" + documents[2][:75],
        dna(150, 999).upper(),
        b"ACGT",
        b"NNNN",
        b"",
        shared[:31] + b"N" + shared[:31] + b"N" + shared[:31],
    ]
    agg_exact = np.zeros(len(documents), dtype=np.uint64)
    for q in queries:
        keys = exact_kmers(q)
        exact = np.array([sum(k in s for k in keys) for s in sets], dtype=np.uint64)
        agg_exact += exact
        b = np.frombuffer(q, dtype=np.uint8) if q else np.zeros(0, dtype=np.uint8)
        got, total = oracle.query_records(index, b, np.array([0, len(q)], dtype=np.uint64))
        assert total == len(keys)
        assert np.all(got >= exact) and np.all(got <= total), (bits, q[:20], got, exact)
    bases = np.frombuffer(b"".join(queries), dtype=np.uint8)
    offsets = np.cumsum([0] + [len(q) for q in queries]).astype(np.uint64)
    agg, _ = oracle.query_records(index, bases, offsets)
    assert np.all(agg >= agg_exact)
