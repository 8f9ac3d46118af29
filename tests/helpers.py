"""Shared test helpers: the oracle's ctypes wrapper, seeded sequence
generators and an index-building wrapper around zx_build.

The oracle (oracle/liboracle.so) is the checker: tests compare the CUDA path
against it, never the other way round.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
from ctypes import POINTER, byref, c_char_p, c_double, c_int, c_size_t, c_uint64, c_void_p
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "_build" / "liboracle.so"
ZX_BUILD = ROOT / "zindex_b200" / "_lib" / "zx_build"
ZX_SYNTH = ROOT / "zindex_b200" / "_lib" / "zx_synth"
ZORINDEX = ROOT / "zindex_b200" / "_lib" / "zorindex"
MODES = {"kmers": 0, "minimizers": 1, "modimizers": 2, "findere": 3}
M64 = (1 << 64) - 1


def build_native() -> None:
    from zindex_b200.build import build

    build()
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)


# ---------------------------------------------------------------- oracle ---
class Oracle:
    """ctypes view of oracle/zx_oracle.h."""

    def __init__(self):
        lib = ctypes.CDLL(str(ORACLE_LIB))
        P64 = POINTER(c_uint64)
        lib.oracle_splitmix64.restype = c_uint64
        lib.oracle_splitmix64.argtypes = [c_uint64]
        lib.oracle_features.restype = c_int
        lib.oracle_features.argtypes = [c_void_p, c_size_t, c_int, c_int, c_int, c_uint64, c_uint64,
                                        c_int, c_int, P64, c_size_t, POINTER(c_size_t)]
        lib.oracle_ocm_slow.restype = c_int
        lib.oracle_ocm_slow.argtypes = [c_void_p, c_size_t, c_int, c_int, c_uint64, P64, P64,
                                        c_size_t, POINTER(c_size_t)]
        lib.oracle_query_file.restype = c_int
        lib.oracle_query_file.argtypes = [c_char_p, c_char_p, c_int, c_int, P64, c_size_t, P64, P64]
        lib.oracle_query_records.restype = c_int
        lib.oracle_query_records.argtypes = [c_char_p, c_void_p, P64, c_size_t, c_int, c_int, P64,
                                             c_size_t, P64, P64]
        lib.oracle_index_colors.restype = c_int
        lib.oracle_index_colors.argtypes = [c_char_p, POINTER(c_size_t)]
        lib.oracle_format_aggregate.restype = c_int
        lib.oracle_format_aggregate.argtypes = [c_char_p, P64, c_uint64, c_double, c_char_p,
                                                c_size_t, POINTER(c_size_t)]
        lib.oracle_last_error.restype = c_char_p
        lib.oracle_query_records_report.restype = c_int
        lib.oracle_query_records_report.argtypes = [c_char_p, c_char_p, c_int, c_double, c_int,
                                                    c_char_p, c_size_t, POINTER(c_size_t)]
        lib.oracle_query_timed.restype = c_int
        lib.oracle_query_timed.argtypes = [c_char_p, c_void_p, P64, c_size_t, c_int, P64, c_size_t,
                                           P64, POINTER(c_double)]
        self.lib = lib

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError("oracle: " + self.lib.oracle_last_error().decode())

    def splitmix64(self, x: int) -> int:
        return int(self.lib.oracle_splitmix64(x & M64))

    def features(self, seq, mode="kmers", k=31, m=21, seed=69, sampling=16, z=10,
                 homopolymer=False) -> np.ndarray:
        b = seq.encode() if isinstance(seq, str) else bytes(seq)
        buf = ctypes.create_string_buffer(b, len(b) + 1)
        cap = len(b) + 8
        out = np.zeros(cap, dtype=np.uint64)
        n = c_size_t()
        self._check(self.lib.oracle_features(buf, len(b), MODES[mode], k, m, seed, sampling, z,
                                             int(homopolymer), out.ctypes.data_as(POINTER(c_uint64)),
                                             cap, byref(n)))
        return out[: n.value].copy()

    def ocm_slow(self, seq, k, m, seed):
        b = seq.encode() if isinstance(seq, str) else bytes(seq)
        cap = len(b) + 8
        pos = np.zeros(cap, dtype=np.uint64)
        key = np.zeros(cap, dtype=np.uint64)
        n = c_size_t()
        self._check(self.lib.oracle_ocm_slow(b, len(b), k, m, seed,
                                             pos.ctypes.data_as(POINTER(c_uint64)),
                                             key.ctypes.data_as(POINTER(c_uint64)), cap, byref(n)))
        return pos[: n.value].copy(), key[: n.value].copy()

    def colors(self, index_dir) -> int:
        n = c_size_t()
        self._check(self.lib.oracle_index_colors(str(index_dir).encode(), byref(n)))
        return n.value

    def query_file(self, index_dir, query, threads=4, recover=True):
        colors = self.colors(index_dir)
        counts = np.zeros(colors, dtype=np.uint64)
        total, probes = c_uint64(), c_uint64()
        self._check(self.lib.oracle_query_file(str(index_dir).encode(), str(query).encode(), threads,
                                               int(recover), counts.ctypes.data_as(POINTER(c_uint64)),
                                               colors, byref(total), byref(probes)))
        return counts, int(total.value), int(probes.value)

    def query_records(self, index_dir, bases, offsets, threads=4, recover=True):
        colors = self.colors(index_dir)
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        counts = np.zeros(colors, dtype=np.uint64)
        total, probes = c_uint64(), c_uint64()
        self._check(self.lib.oracle_query_records(
            str(index_dir).encode(), bases.ctypes.data_as(c_void_p),
            offsets.ctypes.data_as(POINTER(c_uint64)), len(offsets) - 1, threads, int(recover),
            counts.ctypes.data_as(POINTER(c_uint64)), colors, byref(total), byref(probes)))
        return counts, int(total.value)

    def records_report(self, index_dir, query, recover=True, min_ratio=0.0,
                       fmt="tsv") -> bytes:
        """Per-record report bytes (`zorindex query --records`) of a query file."""
        n = c_size_t()
        args = (str(index_dir).encode(), str(query).encode(), int(recover), float(min_ratio),
                int(fmt == "compact"))
        self._check(self.lib.oracle_query_records_report(*args, None, 0, byref(n)))
        buf = ctypes.create_string_buffer(max(n.value, 1))
        self._check(self.lib.oracle_query_records_report(*args, buf, n.value, byref(n)))
        return buf.raw[: n.value]

    def format_aggregate(self, index_dir, counts, total, min_ratio=0.0) -> str:
        counts = np.ascontiguousarray(counts, dtype=np.uint64)
        cap = 1 << 22
        buf = ctypes.create_string_buffer(cap)
        n = c_size_t()
        self._check(self.lib.oracle_format_aggregate(str(index_dir).encode(),
                                                     counts.ctypes.data_as(POINTER(c_uint64)),
                                                     total, min_ratio, buf, cap, byref(n)))
        return buf.raw[: n.value].decode()


# ------------------------------------------------------------ sequences ---
def splitmix64_np(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def dna(n: int, seed: int) -> bytes:
    """The reference tests' generator: "ACGT"[splitmix64(i ^ seed) & 3]."""
    with np.errstate(over="ignore"):
        idx = np.arange(n, dtype=np.uint64) ^ np.uint64(seed & M64)
        codes = splitmix64_np(idx) & np.uint64(3)
    return np.frombuffer(b"ACGT", dtype=np.uint8)[codes.astype(np.int64)].tobytes()


def mutate(seq: bytes, rng: np.random.Generator, subst=0.0, n_runs=0, lower=0.0) -> bytes:
    a = np.frombuffer(seq, dtype=np.uint8).copy()
    if subst > 0 and len(a):
        hit = rng.random(len(a)) < subst
        a[hit] = np.frombuffer(b"ACGT", dtype=np.uint8)[rng.integers(0, 4, hit.sum())]
    for _ in range(n_runs):
        if len(a) < 2:
            break
        at = int(rng.integers(0, len(a)))
        a[at: at + int(rng.integers(1, 8))] = ord("N")
    if lower > 0 and len(a):
        lo = rng.random(len(a)) < lower
        a[lo] = a[lo] | 0x20  # ASCII lowercase
    return a.tobytes()


def write_fasta(path: Path, records, width=80) -> Path:
    with open(path, "wb") as f:
        for i, r in enumerate(records):
            f.write(b">r%d\n" % i)
            for j in range(0, len(r), width):
                f.write(r[j: j + width] + b"\n")
            if not r:
                f.write(b"\n")
    return path


def make_genomes(directory: Path, colors: int, length: int, seed: int = 1) -> Path:
    directory.mkdir(parents=True, exist_ok=True)
    lines = []
    for c in range(colors):
        p = directory / f"g{c}.fa"
        write_fasta(p, [dna(length, seed + c)])
        lines.append(f"g{c}\t{p}")
    fof = directory / "fof.tsv"
    fof.write_text("\n".join(lines) + "\n")
    return fof


def build_index(fof: Path, out: Path, **opts) -> Path:
    args = [str(ZX_BUILD), "-f", str(fof), "-o", str(out), "-q"]
    flag = {"k": "-k", "m": "-m", "H": "-H", "b": "-b", "seed": "-s", "mode": "-i", "z": "-z",
            "d": "-d", "scale": "-S", "seg": "-L", "min_docs": "-D", "max_sub": "-N",
            "max_size": "-X", "threads": "-t", "groups": "--groups", "pattern": "-p"}
    for key, val in opts.items():
        if key == "drop_abandoned":
            if val:
                args.append("-R")
            continue
        if key == "homopolymer":
            if val:
                args.append("-c")
            continue
        if key == "legacy":
            if val:
                args.append("--legacy-layout")
            continue
        args += [flag[key], str(val)]
    subprocess.run(args, check=True)
    return out


def sample_reads(genomes, rng, n, length, sourced=0.7, subst=0.005, n_runs=0.0, lower=0.0):
    out = []
    for _ in range(n):
        if rng.random() < sourced:
            g = genomes[int(rng.integers(0, len(genomes)))]
            at = int(rng.integers(0, max(1, len(g) - length)))
            r = g[at: at + length]
        else:
            r = dna(length, int(rng.integers(0, 1 << 62)))
        r = mutate(r, rng, subst=subst, n_runs=1 if rng.random() < n_runs else 0, lower=lower)
        out.append(r)
    return out


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
