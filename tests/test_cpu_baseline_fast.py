"""The timed CPU baseline's fast lookup (the reference's lookup_batch blocks,
4-ahead row prefetch and AVX2 screens, restated in the oracle as
oracle_query_handle_fast) gives exactly the scalar checker's counts."""
import ctypes
from ctypes import POINTER, byref, c_double, c_int, c_size_t, c_uint64, c_void_p

import numpy as np
import pytest

import helpers

CASES = [
    dict(k=31, H=4, b=8),
    dict(k=25, H=3, b=16, groups="0,1,2"),
    dict(k=21, H=5, b=32),
    dict(k=27, H=8, b=4, groups="1,3"),
    dict(k=23, H=2, b=2, max_size="16KiB"),
    dict(k=19, H=4, b=1),
    dict(k=33, H=4, b=8, groups="2,3"),
    dict(mode="minimizers", k=31, m=21, H=3, b=16),
    dict(mode="modimizers", k=31, H=4, b=4, d=4),
]


def _lib():
    lib = ctypes.CDLL(str(helpers.ORACLE_LIB))
    P64 = POINTER(c_uint64)
    for name in ("oracle_query_handle", "oracle_query_handle_fast"):
        f = getattr(lib, name)
        f.argtypes = [c_void_p, c_void_p, P64, c_size_t, c_int, P64, c_size_t, P64,
                      POINTER(c_double)]
        f.restype = c_int
    lib.oracle_open.argtypes = [ctypes.c_char_p, c_int, POINTER(c_void_p)]
    lib.oracle_open.restype = c_int
    lib.oracle_close.argtypes = [c_void_p]
    lib.oracle_fast_serves.argtypes = [c_void_p]
    lib.oracle_fast_serves.restype = c_int
    return lib


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
@pytest.mark.parametrize("recover", [1, 0])
def test_fast_lookup_equals_scalar_checker(oracle, tmp_path, case, recover):
    import zindex_b200 as zx

    fof = helpers.make_genomes(tmp_path / "g", colors=7, length=12000, seed=31)
    index = helpers.build_index(fof, tmp_path / "index", **case)
    genomes = [helpers.dna(12000, 31 + c) for c in range(7)]
    reads = helpers.sample_reads(genomes, np.random.default_rng(2), 800, 150, n_runs=0.1)
    reads += reads[:50]  # repeated keys fold into weights
    bases, offsets = zx.pack_records(reads)
    lib = _lib()
    h = c_void_p()
    assert lib.oracle_open(str(index).encode(), recover, byref(h)) == 0
    try:
        assert lib.oracle_fast_serves(h) == 1
        out = []
        for fn in (lib.oracle_query_handle, lib.oracle_query_handle_fast):
            counts = np.zeros(7, dtype=np.uint64)
            total, secs = c_uint64(), c_double()
            assert fn(h, bases.ctypes.data_as(c_void_p), offsets.ctypes.data_as(POINTER(c_uint64)),
                      len(reads), 4, counts.ctypes.data_as(POINTER(c_uint64)), 7, byref(total),
                      byref(secs)) == 0
            out.append((counts, total.value))
        assert out[0][1] == out[1][1] > 0
        np.testing.assert_array_equal(out[0][0], out[1][0])
    finally:
        lib.oracle_close(h)
