"""The GPU's randstrobemer formulation (kernels/strobes.cuh) restated on the
CPU and checked against the oracle's linker (link_strobes: the reference's
Linker, src/anchors.rs:182-256, over one ACGT run's candidates sorted by
position, one per position).

On the device the candidates of a batch are marked in a table indexed by base
(a position that several minimizer windows select is one entry), and each
tile links the candidates it owns - its windows' starts, and for a record's
last tile the positions past its last window start (up to k - m of them for
open-closed minimizers) - by a forward scan of the table that stops at
strobe_max, at the record's end and at the first invalid base. Random
records (ACGT runs split by N, lengths around the 256-window tiles), random
candidate sets of the positions windows can select, and random distances
(above 256 and above the record too) go through that formulation tile by
tile; its seeds, in order, must equal the oracle's per-run linking.
"""
import ctypes

import numpy as np
import pytest

TILE = 256


def device_form(valid, cand, k, length, extra, dmin, dmax):
    """The seeds strobe_link_kernel writes for one record, tiles in order."""
    n = len(valid)
    windows = n - k + 1 if n >= k else 0
    out = []
    for w0 in range(0, windows, TILE):
        end = min(w0 + TILE, windows)
        if end == windows and extra:
            end = min(end + extra, n - length + 1 if n >= length else 0)
        for q in range(w0, end):
            if q not in cand:
                continue
            h = cand[q]
            partner, fewest = h, 9
            for d in range(1, dmax + 1):
                c = q + d
                if c + length > n or not valid[c + length - 1]:
                    break
                if d < dmin or c not in cand:
                    continue
                x = bin((h ^ cand[c]) & 0xFF).count("1")
                if x < fewest:
                    fewest, partner = x, cand[c]
                    if not fewest:
                        break
            out.append((h >> 1) + (partner >> 1))
    return out


def oracle_form(lib, valid, cand, dmin, dmax):
    """The oracle's linking of each ACGT run's candidates, runs in order."""
    out, n, i = [], len(valid), 0
    while i < n:
        if not valid[i]:
            i += 1
            continue
        j = i
        while j < n and valid[j]:
            j += 1
        pos = sorted(p for p in cand if i <= p < j)
        if pos:
            P = np.array(pos, dtype=np.uint64)
            Hs = np.array([cand[p] for p in pos], dtype=np.uint64)
            keys = np.zeros(len(pos), dtype=np.uint64)
            u64p = ctypes.POINTER(ctypes.c_uint64)
            lib.oracle_link_strobes(P.ctypes.data_as(u64p), Hs.ctypes.data_as(u64p),
                                    ctypes.c_size_t(len(pos)), ctypes.c_uint64(dmin),
                                    ctypes.c_uint64(dmax), keys.ctypes.data_as(u64p))
            out.extend(int(x) for x in keys)
        i = j
    return out


def random_record(rng):
    n = int(rng.choice([0, 5, 30, 255, 256, 257, 286, 600, 1024, 1300]))
    n = max(0, n + int(rng.integers(-3, 4)))
    valid = rng.random(n) > 0.004
    for _ in range(int(rng.integers(0, 3))):  # N runs
        if n:
            a = int(rng.integers(0, n))
            valid[a: a + int(rng.integers(1, 40))] = False
    return valid


def candidates(rng, valid, k, length, extra, density):
    """Positions the windows of a record can select: inside a valid k-window
    w, at w .. w + extra (every valid window start for k-mers)."""
    n = len(valid)
    bad = np.concatenate([[0], np.cumsum(~valid)])
    window_ok = [bad[w + k] - bad[w] == 0 for w in range(max(0, n - k + 1))]
    cand = {}
    for w, good in enumerate(window_ok):
        if not good:
            continue
        for p in range(w, w + extra + 1):
            if p not in cand and rng.random() < density:
                cand[p] = int(rng.integers(0, 1 << 63)) * 2 + int(rng.integers(0, 2))
    return cand


@pytest.mark.parametrize("mode,k,length,density", [
    ("kmers", 21, 21, 1.0), ("kmers", 31, 31, 1.0),
    ("minimizers", 31, 15, 0.15), ("minimizers", 49, 31, 0.1), ("minimizers", 25, 25, 1.0),
])
def test_table_scan_equals_the_reference_linker(oracle, mode, k, length, density):
    lib = oracle.lib
    lib.oracle_link_strobes.restype = None
    rng = np.random.default_rng(1000 * k + length + (7 if mode == "minimizers" else 0))
    extra = k - length  # 0 for k-mers and for k == m
    checked = 0
    for case in range(24):
        valid = random_record(rng)
        dmin = int(rng.choice([1, 2, 5, 20, 100]))
        dmax = int(rng.choice([dmin, 40, 256, 300, 1200, 5000])) if case % 3 else dmin + 3
        cand = candidates(rng, valid, k, length, extra,
                          density if mode == "minimizers" else 1.0)
        got = device_form(valid, cand, k, length, extra, dmin, dmax)
        want = oracle_form(lib, valid, cand, dmin, dmax)
        assert got == want, (mode, case, len(valid), dmin, dmax)
        checked += len(want)
    assert checked > 1000
