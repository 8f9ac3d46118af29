"""Randstrobemers in the oracle and the builder, pinned on the CPU.

Known answers and properties from the reference's own tests
(src/anchors.rs): the XXH64 strobe hash (824-825), the upstream strobealign
iterator witnesses (951-986), inclusive distances and self fallback
(1040-1062), breaks and homopolymer compression (1016-1038), directional
extraction (988-1014), plus the builder's distinct keys against the oracle's.
These tests pin the checker and the index builder; tests/test_gpu_strobes.py
compares the GPU path with the checker.
"""
import ctypes
import json
from ctypes import POINTER, c_char_p, c_int, c_size_t, c_uint64, c_void_p

import numpy as np
import pytest

import helpers
from helpers import dna

M64 = (1 << 64) - 1


def _lib(oracle):
    lib = oracle.lib
    lib.oracle_strobe_hash.restype = c_uint64
    lib.oracle_strobe_hash.argtypes = [c_uint64]
    lib.oracle_link_strobes.restype = None
    lib.oracle_link_strobes.argtypes = [POINTER(c_uint64), POINTER(c_uint64), c_size_t, c_uint64,
                                        c_uint64, POINTER(c_uint64)]
    lib.oracle_features_anchored.restype = c_int
    lib.oracle_features_anchored.argtypes = [c_void_p, c_size_t, c_int, c_int, c_int, c_uint64,
                                             c_int, c_char_p, c_uint64, c_uint64,
                                             POINTER(c_uint64), c_size_t, POINTER(c_size_t)]
    return lib


def anchored(oracle, seq, mode="kmers", k=9, m=9, seed=69, homopolymer=False, pattern="",
             strobes=None):
    lib = _lib(oracle)
    b = seq if isinstance(seq, bytes) else seq.encode()
    cap = len(b) + 8
    out = np.zeros(cap, dtype=np.uint64)
    n = c_size_t()
    lo, hi = strobes if strobes else (0, 0)
    oracle._check(lib.oracle_features_anchored(
        ctypes.create_string_buffer(b, len(b) + 1), len(b), helpers.MODES[mode], k, m, seed,
        int(homopolymer), pattern.encode(), lo, hi, out.ctypes.data_as(POINTER(c_uint64)), cap,
        ctypes.byref(n)))
    return [int(x) for x in out[: n.value]]


def _encode(seq: bytes) -> int:
    v = 0
    for ch in seq:
        v = (v << 2) | b"ACGT".index(ch)
    return v


def _canonical(v: int, k: int) -> int:
    rc, x = 0, v
    for _ in range(k):
        rc = (rc << 2) | ((x & 3) ^ 3)
        x >>= 2
    return min(v, rc)


def _rc(seq: bytes) -> bytes:
    return seq[::-1].translate(bytes.maketrans(b"ACGT", b"TGCA"))


def test_strobe_hash_known_answer(oracle):
    # anchors.rs:825: XXH64 of one u64 with seed 0.
    assert _lib(oracle).oracle_strobe_hash(0x3332316F6C6C6568) == 0x2D119FCED5EE39CE


# anchors.rs:951-986: keys of the unmodified upstream strobealign iterator on one
# sequence, as (k, low, high, step, count, checksum of the keys in order).
WITNESS_SEQ = b"ACGTTGCACTGATCGATGGCATACCTAGGCTAACGTCGATCTTACGGAATCGCTAGCTGACCATGGTTACG"
WITNESSES = [
    (11, 4, 12, 1, 61, 11859818861789259928),
    (11, 2, 5, 3, 21, 7111390358099897965),
    (21, 7, 15, 1, 51, 7250723734144174666),
]


@pytest.mark.parametrize("k,low,high,step,count,expected", WITNESSES)
def test_linker_matches_upstream_witnesses(oracle, k, low, high, step, count, expected):
    lib = _lib(oracle)
    pos = list(range(0, len(WITNESS_SEQ) - k + 1, step))
    hashes = [lib.oracle_strobe_hash(_canonical(_encode(WITNESS_SEQ[p:p + k]), k)) for p in pos]
    n = len(pos)
    P = (c_uint64 * n)(*pos)
    H = (c_uint64 * n)(*hashes)
    out = (c_uint64 * n)()
    lib.oracle_link_strobes(P, H, n, low * step, high * step, out)
    assert n == count
    checksum = 0
    for key in out:
        checksum = (checksum * 0x9E3779B185EBCA87 + key) & M64
    assert checksum == expected


def test_distances_are_inclusive_and_unpaired_anchors_fall_back_to_self(oracle):
    # anchors.rs:1040-1052 (k 3, distances exactly 5).
    assert anchored(oracle, "AC", k=3, strobes=(5, 5)) == []
    assert len(anchored(oracle, "ACGTACG", k=3, strobes=(5, 5))) == 5
    keys = anchored(oracle, "ACGTACGT", k=3, strobes=(5, 5))
    plain = anchored(oracle, "ACGTACGT", k=3)
    lib = _lib(oracle)
    h = [lib.oracle_strobe_hash(x) for x in plain]
    assert len(keys) == 6
    assert keys[0] == h[0] // 2 + h[5] // 2      # window 0 pairs with window 5
    assert keys[1] == h[1] // 2 + h[1] // 2      # no window 6: falls back to itself


@pytest.mark.parametrize("mode,k", [("kmers", 9), ("minimizers", 31)])
def test_breaks_and_homopolymer_compression(oracle, mode, k):
    # anchors.rs:1016-1038.
    seq = dna(300, 5).upper()
    inp = seq + b"NNN" + seq
    kw = dict(mode=mode, k=k, m=9, pattern="##__#__##", strobes=(9, 40))
    assert anchored(oracle, inp, **kw) == anchored(oracle, seq, **kw) * 2
    expanded = bytes(b for ch in inp for b in (ch, ch, ch))
    compressed = bytes(b for i, b in enumerate(expanded) if i == 0 or b != expanded[i - 1] or
                       b not in b"ACGT")
    assert anchored(oracle, expanded, homopolymer=True, **kw) == anchored(oracle, compressed, **kw)


@pytest.mark.parametrize("mode,k", [("kmers", 11), ("minimizers", 29)])
def test_extraction_is_directional(oracle, mode, k):
    # anchors.rs:988-1014: one key per plain seed, equal counts on both strands,
    # different key sets (partner selection is not canonicalisation).
    seq = dna(1000, 9).upper()
    kw = dict(mode=mode, k=k, m=11)
    fwd = anchored(oracle, seq, strobes=(15, 50), **kw)
    rev = anchored(oracle, _rc(seq), strobes=(15, 50), **kw)
    assert len(fwd) == len(anchored(oracle, seq, **kw)) == len(rev)
    assert sorted(fwd) != sorted(rev)


@pytest.mark.parametrize("mode,extra,pattern", [
    ("kmers", dict(k=21), ""),
    ("kmers", dict(k=15), "##_#_#_#_#_#_##"),
    ("minimizers", dict(k=31, m=15), ""),
    ("minimizers", dict(k=31, m=15), "##_##_###_##_##"),
])
def test_builder_randstrobe_keys_match_oracle(oracle, tmp_path, mode, extra, pattern):
    """The builder's distinct randstrobemer keys per colour (unique_kmers)
    equal the oracle's keys of each genome."""
    d = tmp_path / "rs"
    fof = helpers.make_genomes(d / "g", 3, 8000, 57)
    args = [str(helpers.ZX_BUILD), "-f", str(fof), "-o", str(d / "ix"), "-q", "-r",
            "-l", "9", "-u", "60", "-i", mode, "-H", "3", "-b", "8", "-k", str(extra["k"])]
    if "m" in extra:
        args += ["-m", str(extra["m"])]
    if pattern:
        args += ["-p", pattern]
    import subprocess

    subprocess.run(args, check=True)
    manifest = json.loads((d / "ix" / "manifest.json").read_text())
    assert manifest["randstrobemers"] == {"min_distance": 9, "max_distance": 60}
    for c, col in enumerate(manifest["colors"]):
        keys = anchored(oracle, dna(8000, 57 + c), mode=mode, k=extra["k"], m=extra.get("m", 9),
                        pattern=pattern, strobes=(9, 60))
        assert col["unique_kmers"] == len(set(keys)), (mode, c)


def test_builder_randstrobe_defaults_and_checks(native, tmp_path):
    import subprocess

    fof = helpers.make_genomes(tmp_path / "g", 2, 3000, 5)
    subprocess.run([str(helpers.ZX_BUILD), "-f", str(fof), "-o", str(tmp_path / "a"), "-q", "-r",
                    "-k", "17"], check=True)
    m = json.loads((tmp_path / "a" / "manifest.json").read_text())
    assert m["randstrobemers"] == {"min_distance": 17, "max_distance": 51}
    assert m["randstrobe_scheme"] == "strobealign-popcount8-symmetric64-downstream-v1"
    for i, extra in enumerate((["-l", "6", "-u", "5"], ["-i", "findere", "-z", "5"])):
        with pytest.raises(subprocess.CalledProcessError):
            subprocess.run([str(helpers.ZX_BUILD), "-f", str(fof), "-o", str(tmp_path / f"b{i}"),
                            "-q", "-r", "-k", "17", *extra], check=True)


def test_oracle_query_keeps_the_larger_strand(oracle, tmp_path):
    """A randstrobemer query counts both strands of a record and keeps, per
    colour, the larger count (query_stream.rs:690-701): a record and its
    reverse complement give the same counts, and the aggregate of two records
    is the sum of their per-record counts."""
    import subprocess

    fof = helpers.make_genomes(tmp_path / "g", 3, 6000, 71)
    ix = tmp_path / "ix"
    subprocess.run([str(helpers.ZX_BUILD), "-f", str(fof), "-o", str(ix), "-q", "-r", "-k", "19",
                    "-H", "3", "-b", "8"], check=True)
    g = dna(6000, 72).upper()
    r1, r2 = g[100:700], dna(500, 9).upper()

    def q(*reads):
        import zindex_b200 as zx

        bases, offsets = zx.pack_records(list(reads))
        return oracle.query_records(ix, bases, offsets)

    c1, t1 = q(r1)
    c1r, t1r = q(_rc(r1))
    np.testing.assert_array_equal(c1, c1r)
    assert t1 == t1r == 600 - 19 + 1
    # Every anchor whose partner window lies inside the read is a key of the
    # source genome (partners are only chosen downstream, up to 3k = 57 bases).
    assert t1 - 57 <= c1[1] <= t1
    c2, t2 = q(r2)
    c12, t12 = q(r1, r2)
    np.testing.assert_array_equal(c12, c1 + c2)
    assert t12 == t1 + t2


def test_cli_build_writes_anchor_settings(native, tmp_path):
    """`zorindex build` takes the reference's anchor flags (-c, -p, -r, -l, -u)."""
    import subprocess

    fof = helpers.make_genomes(tmp_path / "g", 2, 3000, 8)
    out = tmp_path / "ix"
    subprocess.run([str(helpers.ZORINDEX), "build", "-f", str(fof), "-o", str(out), "-k", "15",
                    "-c", "-p", "##_#_#_#_#_#_##", "-r", "-l", "4", "-u", "40"], check=True,
                   capture_output=True)
    m = json.loads((out / "manifest.json").read_text())
    assert m["homopolymer_compression"] is True
    assert m["seed_pattern"] == "##_#_#_#_#_#_##"
    assert m["randstrobemers"] == {"min_distance": 4, "max_distance": 40}
