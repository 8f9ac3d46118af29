"""In-tree build of the native parts of zindex_b200.

Outputs (all under zindex_b200/_lib/, git-ignored, shipped with the tree):
  libzindex_b200.so  CUDA query path for sm_100a + its extern "C" ABI
  zorindex           command-line drop-in (`zorindex query ...`, `zorindex build ...`)
  zx_build           index builder (construction, host side)
  zx_synth           seeded synthetic genomes / reads for the benchmark workloads

Run `python -m zindex_b200.build` (or call build()). Rebuilds only stale targets.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "_lib"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_SOURCES = ["host/json.cpp", "host/manifest.cpp", "host/zstd_io.cpp", "host/fastx.cpp",
                "host/record_report.cpp"]
CUDA_SOURCES = ["engine.cu", "server.cu", "planner.cu", "capi.cu"]
LIBS = ["-lz", "-l:libzstd.so.1", "-l:liblzma.so.5", "-l:libbz2.so.1.0", "-lpthread"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _headers():
    return list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.cuh")) + [PKG.parent / "include" / "zindex.h"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), file=sys.stderr)
    subprocess.run([str(c) for c in cmd], check=True)


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile every native target; returns the path of libzindex_b200.so."""
    LIB.mkdir(exist_ok=True)
    nvcc = _nvcc()
    heads = _headers()
    objdir = LIB / "obj"
    objdir.mkdir(exist_ok=True)
    host_objs = []
    for src in HOST_SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        if force or _stale(obj, [CSRC / src] + heads):
            _run(["g++", "-O3", "-std=c++17", "-fPIC", "-Wall", "-c", CSRC / src, "-o", obj], verbose)
        host_objs.append(obj)
    cuda_objs = []
    for src in CUDA_SOURCES:
        obj = objdir / (Path(src).stem + ".cu.o")
        if force or _stale(obj, [CSRC / src] + heads):
            _run([nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr", "-c", CSRC / src, "-o", obj], verbose)
        cuda_objs.append(obj)
    so = LIB / "libzindex_b200.so"
    if force or _stale(so, host_objs + cuda_objs):
        _run([nvcc, *ARCH, "-shared", "-o", so, *cuda_objs, *host_objs, *LIBS], verbose)
    cli = LIB / "zorindex"
    cli_src = CSRC / "cli" / "zorindex.cpp"
    build_src = [CSRC / "builder" / "builder.cpp"]
    if force or _stale(cli, [cli_src, so] + build_src + heads):
        _run(["g++", "-O3", "-std=c++17", "-Wall", "-o", cli, cli_src, *build_src, *host_objs,
              f"-L{LIB}", "-lzindex_b200", f"-Wl,-rpath,$ORIGIN", *LIBS], verbose)
    # The device builder (zx_build --device) is CUDA: compiled by nvcc and
    # linked into zx_build only.
    dbo = objdir / "device_builder.cu.o"
    dbs = CSRC / "builder" / "device_builder.cu"
    if force or _stale(dbo, [dbs] + heads):
        _run([nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr", "-c", dbs,
              "-o", dbo], verbose)
    zb = LIB / "zx_build"
    zb_src = [CSRC / "builder" / "zx_build_main.cpp", CSRC / "builder" / "builder.cpp"]
    if force or _stale(zb, zb_src + heads + host_objs + [dbo]):
        _run([nvcc, *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-Wall", "-o", zb, *zb_src, dbo,
              *host_objs, *LIBS], verbose)
    zs = LIB / "zx_synth"
    zs_src = CSRC / "builder" / "zx_synth.cpp"
    if force or _stale(zs, [zs_src] + heads):
        _run(["g++", "-O3", "-std=c++17", "-Wall", "-o", zs, zs_src, "-lpthread"], verbose)
    return so


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
