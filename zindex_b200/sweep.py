"""Geometry sweep of the batched query (hashes, fingerprint bits, colours and
seed modes) on a mixed read-length batch.

Each setting is an index built from seeded synthetic genomes (zx_build) and a
batch of 100,000 reads of 150 bp plus 5,000 long reads (lognormal lengths,
median 2 kbp), 70 % sourced from the genomes with 0.5 % substitutions. For
every setting the default launch is timed on the device-resident batch (CUDA
events around graph replays; median of `reps`), the fused kernel alone with
the engine's own events, and the kernel's algorithmic bytes (seeds x gather
bytes per seed + 8 B per recovery probe + 3/8 B per base) are set against the
measured HBM copy peak. Indexes below the 126 MB L2 are marked: their bound is
the L2, not HBM.

    python -m zindex_b200.sweep --out sweep.json --md sweep.md
"""
from __future__ import annotations

import json
import statistics
import subprocess
import time
from pathlib import Path

import numpy as np

from .tuning import Autotuner, DeviceBatch

BASE = dict(mode="kmers", k=31, H=4, b=8)
POOL = (512, 100_000, 1_000_000)  # colours, min and max genome length
SETTINGS = (
    [(f"H{h}", dict(BASE, H=h), POOL) for h in (2, 4, 8, 16, 32)]
    + [(f"b{b}", dict(BASE, b=b), POOL) for b in (1, 4, 16, 32)]
    + [("c64", BASE, (64, 1_000_000, 4_000_000)),
       ("c4096", BASE, (4096, 20_000, 100_000)),
       ("c16384", BASE, (16384, 5_000, 25_000)),
       ("minimizers-k49-m31", dict(BASE, mode="minimizers", k=49, m=31), POOL),
       ("modimizers-k49-d16", dict(BASE, mode="modimizers", k=49, d=16), POOL),
       ("findere-k31-z10", dict(BASE, mode="findere", z=10), POOL)]
)
L2_BYTES = 126 << 20


def _synth(lib: Path, args, out: Path):
    subprocess.run([str(lib / "zx_synth"), *args, "--out", str(out)], check=True)


def _prepare(lib: Path, work: Path, name: str, opts: dict, pool, seed: int):
    d = work / name
    d.mkdir(parents=True, exist_ok=True)
    colors, lo, hi = pool
    gen = work / f"genomes-{colors}-{lo}-{hi}"
    if not (gen / "fof.tsv").exists():
        gen.mkdir(parents=True, exist_ok=True)
        _synth(lib, ["genomes", "--kind", "pool", "--colors", str(colors), "--min-len", str(lo),
                     "--max-len", str(hi), "--seed", str(seed)], gen)
    index = d / "index"
    build_s = 0.0
    if not (index / "manifest.json").exists():
        flag = {"k": "-k", "m": "-m", "H": "-H", "b": "-b", "mode": "-i", "z": "-z", "d": "-d"}
        args = [str(lib / "zx_build"), "-f", str(gen / "fof.tsv"), "-o", str(index), "-q"]
        for key, val in opts.items():
            args += [flag[key], str(val)]
        t0 = time.perf_counter()
        subprocess.run(args, check=True)
        build_s = time.perf_counter() - t0
    parts = []
    common = ["--genome-kind", "pool", "--colors", str(colors), "--min-len", str(lo), "--max-len",
              str(hi), "--seed", str(seed), "--sourced", "0.7", "--subst", "0.005",
              "--format", "raw"]
    for kind, length, count, rseed in (("short", 150, 100_000, seed + 7),
                                       ("long", 2000, 5_000, seed + 8)):
        out = gen / f"reads-{kind}"
        if not Path(str(out) + ".offsets").exists():
            _synth(lib, ["reads", "--kind", kind, "--length", str(length), "--reads", str(count),
                         "--read-seed", str(rseed), *common], out)
        parts.append((np.fromfile(str(out) + ".bases", dtype=np.uint8),
                      np.fromfile(str(out) + ".offsets", dtype=np.uint64)))
    bases = np.concatenate([p[0] for p in parts])
    offsets = np.concatenate([parts[0][1], parts[1][1][1:] + parts[0][1][-1]])
    return index, bases, offsets, build_s


def _peak():
    root = Path(__file__).resolve().parents[1]
    try:
        return float(json.loads((root / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def run(work: Path, reps: int = 5, settings=SETTINGS, log=print):
    import torch

    import zindex_b200 as zx

    lib = Path(zx.LIB_DIR)
    work.mkdir(parents=True, exist_ok=True)
    peak, peak_kind = _peak()
    rows = []
    for name, opts, pool in settings:
        index, bases, offsets, build_s = _prepare(lib, work, name, opts, pool, 2000)
        torch.zeros(1, device="cuda")
        t0 = time.perf_counter()
        ix = zx.Index(index)
        load_s = time.perf_counter() - t0
        info = ix.info
        batch = DeviceBatch(bases, offsets, ix.colors)
        seeds = batch.seeds(ix)
        step_ms = Autotuner(reps=reps).time_config(ix, batch, dict(ix.launch()))
        ix.set_timing(True)
        kms = []
        for _ in range(reps):
            batch.run(ix, torch.cuda.current_stream(), use_graph=False)
            kms.append(ix.last_kernel_ms())
        ix.set_timing(False)
        kernel_ms = statistics.median(kms)
        rec = 8 if info.abandoned_hashes else 0
        alg = seeds * (info.gather_bytes_per_seed + rec) + len(bases) * 3 // 8
        sec = seeds * (info.gather_sector_bytes_per_seed + (32 if rec else 0)) + len(bases) * 3 // 8
        row = {
            "setting": name, "options": opts, "colors": int(info.colors),
            "genome_len_bp": list(pool[1:]), "classes": int(info.classes),
            "resident_bytes": int(info.resident_bytes),
            "l2_resident": bool(info.resident_bytes < L2_BYTES),
            "bases": int(len(bases)), "records": int(len(offsets) - 1), "seeds": seeds,
            "gather_bytes_per_seed": int(info.gather_bytes_per_seed),
            "sector_bytes_per_seed": int(info.gather_sector_bytes_per_seed),
            "step_ms": step_ms, "seeds_per_s": seeds / (step_ms / 1e3),
            "kernel_ms": kernel_ms, "achieved_gbs": alg / (kernel_ms / 1e3) / 1e9,
            "frac": alg / (kernel_ms / 1e3) / 1e9 / peak,
            "sector_frac": sec / (kernel_ms / 1e3) / 1e9 / peak,
            "launch": ix.launch(), "build_s": build_s, "load_s": load_s,
            "peak_gbs": peak, "peak_kind": peak_kind,
        }
        rows.append(row)
        log(f"{name}: {row['seeds_per_s']:.3e} seeds/s, frac {row['frac']:.3f} "
            f"(sector {row['sector_frac']:.3f}), kernel {kernel_ms:.2f} ms")
        del batch
        ix.close()
        torch.cuda.empty_cache()
    return {"device": torch.cuda.get_device_name(0), "reps": reps, "rows": rows}


def markdown(data) -> str:
    out = ["| setting | colours | classes | resident MB | B/seed (sectors) | seeds | step ms | "
           "seeds/s | kernel ms | GB/s | frac | sector frac | launch (team, warps, planes) |",
           "|---|---|---|---|---|---|---|---|---|---|---|---|---|"]
    for r in data["rows"]:
        lc = r["launch"]
        l2 = " (L2)" if r["l2_resident"] else ""
        out.append(
            f"| {r['setting']} | {r['colors']} | {r['classes']} | {r['resident_bytes'] / 1e6:.0f}{l2} | "
            f"{r['gather_bytes_per_seed']} ({r['sector_bytes_per_seed']}) | {r['seeds']:,} | "
            f"{r['step_ms']:.2f} | {r['seeds_per_s']:.3e} | {r['kernel_ms']:.2f} | "
            f"{r['achieved_gbs']:.0f} | {r['frac']:.3f} | {r['sector_frac']:.3f} | "
            f"{lc['team']}, {lc['warps']}, {lc['planes']} |")
    return "\n".join(out) + "\n"


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="geometry sweep of the batched query")
    ap.add_argument("--work", default="/tmp/zx_sweep")
    ap.add_argument("--out", required=True)
    ap.add_argument("--md", default=None)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--only", default=None, help="comma-separated setting names")
    a = ap.parse_args()
    chosen = SETTINGS if not a.only else [s for s in SETTINGS if s[0] in a.only.split(",")]
    result = run(Path(a.work), a.reps, chosen)
    Path(a.out).write_text(json.dumps(result, indent=1))
    if a.md:
        Path(a.md).write_text(markdown(result))
