"""The oracle pinned against the reference's own known answers (CPU only).

Each test cites the reference test it mirrors. The reference cannot be built
here (Rust), so these known answers and the reference's independent
window-by-window formulations are what pin the oracle.
"""
import numpy as np
import pytest

from helpers import M64, dna

# src/lib.rs:1152-1161 (splitmix_stable_00..09).
SPLITMIX = [0xE220A8397B1DCDAF, 0x910A2DEC89025CC1, 0x975835DE1C9756CE, 0x1D0B14E4DB018FED,
            0x6E73E372E2338ACA, 0x63033B0CA389C35A, 0xBD64A5D9ADEFE000, 0x63CBE1E459320DD7,
            0x9E5651B0EF953636, 0xAEAF52FEBE706064]


def test_splitmix64_known_answers(oracle):
    assert [oracle.splitmix64(i) for i in range(10)] == SPLITMIX


@pytest.mark.parametrize("seq,value", [("A", 0), ("C", 1), ("G", 2), ("T", 3), ("AC", 1),
                                       ("GT", 11), ("ACGT", 27), ("acgt", 27)])
def test_encode_full_kmer(oracle, seq, value):
    # src/lib.rs:966-975: a k = len(seq) forward value; canonical = min(fwd, rc).
    rc = 0
    for ch in reversed(seq.upper()):
        rc = (rc << 2) | ("ACGT".index(ch) ^ 3)
    assert list(oracle.features(seq, k=len(seq))) == [min(value, rc)]


@pytest.mark.parametrize("seq,k,count", [
    ("ACG", 4, 0), ("ACGT", 4, 1), ("AAAA", 4, 1), ("ACGTA", 3, 3), ("ACGTACGT", 4, 5),
    ("ACGTACGTAA", 5, 6), ("NACGT", 4, 1), ("ACNGTAC", 3, 2), ("ACGTNNACGT", 4, 2),
    ("acgtac", 4, 3), ("AcGtAc", 4, 3), ("ACGT", 1, 4), ("ACGT", 2, 3), ("ACGT", 3, 2),
    ("ACGT", 4, 1), ("AAAAAAAA", 5, 4)])
def test_kmer_counts(oracle, seq, k, count):
    # src/lib.rs:986-1001.
    assert len(oracle.features(seq, k=k)) == count


def _reference_windows(seq: bytes, k: int):
    # src/lib.rs:821-868: independent per-window hash of every all-ACGT window.
    B = 0x9E3779B185EBCA87
    out = []
    for i in range(len(seq) - k + 1):
        w = seq[i:i + k]
        if any(c not in b"ACGTacgt" for c in w):
            continue
        codes = ["ACGT".index(chr(c).upper()) for c in w]
        if k <= 32:
            f = 0
            r = 0
            for c in codes:
                f = (f << 2) | c
            for c in reversed(codes):
                r = (r << 2) | (c ^ 3)
            out.append(min(f, r))
        else:
            f = r = 0
            for c in codes:
                f = (f * B + c + 1) & M64
            for c in reversed(codes):
                r = (r * B + 4 - c) & M64
            dom = _sm((k ^ 0x6B6D65722D763031) & M64)
            out.append(_sm(min(f, r) ^ dom))
    return out


def _sm(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


@pytest.mark.parametrize("k", [1, 31, 32, 33, 49, 64, 65, 127, 255, 256])
def test_arbitrary_k_matches_window_formula(oracle, k):
    seq = bytearray(dna(700, 0))
    seq[80] = ord("N")
    seq[300] = ord("n")
    seq[120:160] = bytes(seq[120:160]).lower()
    seq = bytes(seq)
    assert list(oracle.features(seq, k=k)) == _reference_windows(seq, k)


OCM_SEQS = [dna(190, 0), b"ACGT" * 48, b"A" * 190, b"AAAACCCCGGGGTTTT" * 12]


@pytest.mark.parametrize("seq_id", range(len(OCM_SEQS)))
def test_ocm_rolling_matches_slow_reference(oracle, seq_id):
    # open_closed_minimizers.rs:87-130: every odd k <= 65, m <= 31, seeds 0/69.
    seq = OCM_SEQS[seq_id]
    for k in range(1, 66, 2):
        for m in range(1, min(31, k) + 1):
            for seed in (0, 69):
                _, slow = oracle.ocm_slow(seq, k, m, seed)
                got = oracle.features(seq, mode="minimizers", k=k, m=m, seed=seed)
                assert np.array_equal(got, slow), (k, m, seed)


def test_ocm_reverse_complement_property(oracle):
    seq = dna(190, 0)
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    rc = seq.translate(comp)[::-1]
    for k, m in [(49, 31), (31, 21), (19, 12), (9, 5)]:
        a = sorted(oracle.features(seq, mode="minimizers", k=k, m=m).tolist())
        b = sorted(oracle.features(rc, mode="minimizers", k=k, m=m).tolist())
        assert set(a) == set(b)


def test_ocm_ambiguity_split(oracle):
    # open_closed_minimizers.rs:132-143.
    whole = oracle.features(b"acgtACGTAANNNacgtacgtaa", mode="minimizers", k=9, m=5)
    split = np.concatenate([oracle.features(b"ACGTACGTAA", mode="minimizers", k=9, m=5)] * 2)
    assert np.array_equal(whole, split)


def test_modimizer_sampling_one_keeps_all(oracle):
    # src/lib.rs:1091-1107.
    for seq, k in [(b"ACGTACGT", 3), (b"AAAACCCC", 4), (b"ACGTNACGT", 4), (b"CCCCCCCC", 2)]:
        assert np.array_equal(oracle.features(seq, mode="modimizers", k=k, sampling=1),
                              oracle.features(seq, k=k))


def test_findere_indexes_smers_of_long_runs(oracle):
    seq = dna(100, 4) + b"N" + dna(20, 5)
    got = oracle.features(seq, mode="findere", k=31, z=10)
    want = oracle.features(dna(100, 4), k=21)
    assert np.array_equal(got, want)  # the 20-base run is shorter than k


def test_planner_measurements_and_features():
    """The committed planner training set loads and encodes (no GPU needed)."""
    from zindex_b200 import planner as pl

    rows, defaults = pl.load_rows()
    assert rows and set(defaults) == {r.setting for r in rows}
    x = pl.encode(rows[0].features, rows[0].launch, rows[0].e2e)
    assert x.shape == (len(pl.FEATURES),) and np.isfinite(x).all()


# ---- spaced seeds (src/anchors.rs:751-773 pattern_validation_and_projection) ----
def _encode(seq: str) -> int:
    v = 0
    for ch in seq:
        v = (v << 2) | "ACGT".index(ch)
    return v


def _rc(seq: str) -> str:
    return seq[::-1].translate(str.maketrans("ACGT", "TGCA"))


def _pattern(oracle, pattern, key):
    import ctypes
    from ctypes import POINTER, c_char_p, c_int, c_uint64

    f = oracle.lib.oracle_pattern_canonical
    f.argtypes = [c_char_p, c_uint64, POINTER(c_uint64), POINTER(c_uint64)]
    f.restype = c_int
    proj, canon = c_uint64(), c_uint64()
    rc = f(pattern.encode(), key, ctypes.byref(proj), ctypes.byref(canon))
    return rc, proj.value, canon.value


@pytest.mark.parametrize("invalid", ["", "___", "#x#", "##_", "#" * 31 + "_"])
def test_spaced_seed_pattern_validation(oracle, invalid):
    assert _pattern(oracle, invalid, 0)[0] != 0


def test_spaced_seed_projection_and_canonical(oracle):
    p = "##_##_##"
    rc, proj, _ = _pattern(oracle, p, _encode("ACGTAACG"))
    assert rc == 0 and proj == _encode("ACTACG")
    a, b = "ACATACCG", "ACGTAGCG"
    ca = _pattern(oracle, p, _encode(a))[2]
    assert ca == _pattern(oracle, p, _encode(b))[2]
    assert ca == _pattern(oracle, p, _encode(_rc(a)))[2]


def test_all_retained_pattern_leaves_keys_unchanged(oracle):
    # anchors.rs:841-855: a pattern of only '#' maps every canonical key to itself.
    seq = dna(2000, 77)
    for key in oracle.features(seq, k=9)[:500]:
        assert _pattern(oracle, "#########", int(key))[2] == int(key)


def test_builder_spaced_seed_keys_match_oracle(oracle, tmp_path):
    """The builder's distinct spaced-seed keys per colour (manifest unique_kmers)
    equal the oracle's plain canonical keys mapped through the pattern."""
    import json

    import helpers

    pattern = "##_#_##_#_##"  # width 12 = k, weight 8
    for mode, extra in (("kmers", dict(k=12)), ("minimizers", dict(k=21, m=12))):
        d = tmp_path / mode
        fof = helpers.make_genomes(d / "g", 3, 6000, 91)
        ix = helpers.build_index(fof, d / "ix", mode=mode, H=3, b=8, pattern=pattern, **extra)
        manifest = json.loads((ix / "manifest.json").read_text())
        assert manifest["seed_pattern"] == pattern
        for c, col in enumerate(manifest["colors"]):
            plain = oracle.features(dna(6000, 91 + c), mode=mode, **extra)
            mapped = {_pattern(oracle, pattern, int(k))[2] for k in plain}
            assert col["unique_kmers"] == len(mapped), (mode, c)


def test_builder_rejects_invalid_patterns(native, tmp_path):
    import subprocess

    import helpers

    fof = helpers.make_genomes(tmp_path / "g", 2, 3000, 5)
    for i, (pattern, opts) in enumerate([("##_", dict(k=3)), ("#_#", dict(k=5)),
                                         ("###", dict(mode="findere", k=13, z=10))]):
        with pytest.raises(subprocess.CalledProcessError):
            helpers.build_index(fof, tmp_path / f"ix{i}", pattern=pattern, **opts)


# ---- position hash and recovery hash ----------------------------------------
def _mix(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def test_position_hash_matches_segment_mapping(oracle):
    # storage.rs:4799-4825 (shared_position_hash_matches_original_segment_mapping):
    # the legacy segment length and the cell formula, for H in {2,3,4,8,32}.
    import ctypes
    from ctypes import POINTER, c_int, c_uint64

    f = oracle.lib.oracle_positions
    f.argtypes = [c_uint64, c_uint64, c_uint64, c_int, c_uint64, POINTER(c_uint64)]
    f.restype = None
    for hashes in (2, 3, 4, 8, 32):
        for exponent in range(5, 25):
            cells = 1 << exponent
            for key in (0, 1, 123, M64):
                seed = 69
                length = 1 << (min(max(cells // hashes, 1), 4096).bit_length() - 1)
                count = cells // length - hashes + 1
                h1 = _mix((key + seed) & M64)
                h2 = _mix(h1)
                base = ((h1 * count) >> 64) * length
                h, want = h1, []
                for i in range(hashes):
                    want.append(base + i * length + ((h ^ (h >> 33)) & (length - 1)))
                    h = (h + h2) & M64
                out = (c_uint64 * hashes)()
                f(key, seed, cells, hashes, 0, out)
                assert list(out) == want, (hashes, exponent, key)


def test_recovery_hash_collision(oracle):
    # query_stream.rs:1114-1160: keys 83,843 and 95,900 share the stored
    # 32-bit recovery hash under seed 69; 123 does not.
    from ctypes import c_uint32, c_uint64

    f = oracle.lib.oracle_abandoned_hash
    f.argtypes = [c_uint64, c_uint64]
    f.restype = c_uint32
    assert f(83843, 69) == f(95900, 69)
    assert f(123, 69) != f(83843, 69)
    assert f(83843, 69) == _mix(83843 ^ 69 ^ 0xD6E8FEB86659FD93) >> 32
