"""Launch-configuration autotuner for the batched query kernels.

The fused extraction+probe kernel has three tunables that never change the
results: the team size T (lanes sharing one seed's row gather; the 16-byte
chunks of a fingerprint-plane row are split over the T lanes), the warps per
block, and whether per-colour counters live in shared memory or are global
atomics. The best choice depends on the index geometry (H, b, groups per
class, classes, colours, mode) and on the batch (read-length mix, seed count).

Autotuner.tune() times every candidate on a device-resident batch with CUDA
events (graph replays on the index's stream) and returns the fastest. Every
measurement is also kept as a training row for the learned planner
(zindex_b200.planner).
"""
from __future__ import annotations

import itertools
import json
import statistics
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Sequence

import numpy as np

TEAMS = (2, 4, 8, 16, 32)
WARPS = (2, 4, 8)
STAGE_BYTES = (4096, 8192, 16384)
STAGES = (2, 3, 4)
MIN_BLOCKS = (1, 2, 3)
PLANES = (0, 1)


@dataclass
class Measurement:
    features: Dict[str, float]
    launch: Dict[str, int]
    ms: float
    seeds: int


@dataclass
class Autotuner:
    reps: int = 3
    rows: List[Measurement] = field(default_factory=list)

    @staticmethod
    def candidates(ix, register_gather: bool = True, staged: bool = True) -> List[dict]:
        """Register-gather teams and staged bulk-copy rings, shared-memory
        counters whenever the colours fit (global atomics only otherwise)."""
        smem = 1 if ix.colors <= 16384 else 0
        out = []
        if register_gather:
            for team, warps, minb, planes in itertools.product(TEAMS, WARPS, MIN_BLOCKS, PLANES):
                if minb == 1 and not planes:
                    continue
                out.append({"team": team, "warps": warps, "blocks": 0, "smem_counters": smem,
                            "stage_bytes": 0, "stages": 1, "bulk": 0, "min_blocks": minb,
                            "planes": planes})
        if staged:
            for bulk, stage_bytes, stages, warps in itertools.product(
                    (0, 1), STAGE_BYTES, STAGES, WARPS):
                if stage_bytes < 16 * ix.info.hashes:
                    continue
                out.append({"team": 8, "warps": warps, "blocks": 0, "smem_counters": smem,
                            "stage_bytes": stage_bytes, "stages": stages, "bulk": bulk,
                            "min_blocks": 2, "planes": 0})
        return out

    @staticmethod
    def features(ix, lengths: np.ndarray, seeds: int) -> Dict[str, float]:
        info = ix.info
        return {
            "hashes": float(info.hashes), "bits": float(info.fingerprint_bits),
            "colors": float(info.colors), "mode": float(info.index_mode),
            "classes": float(info.classes),
            "gather_bytes": float(info.gather_bytes_per_seed),
            "len_mean": float(lengths.mean()) if len(lengths) else 0.0,
            "len_var": float(lengths.var()) if len(lengths) else 0.0,
            "seeds": float(seeds),
        }

    def time_config(self, ix, batch, launch: dict) -> float:
        """Median milliseconds of one batch query under `launch`."""
        import torch

        try:
            ix.set_launch(**launch)
        except Exception:
            return float("inf")  # e.g. more shared memory than a block may use
        stream = torch.cuda.current_stream()
        batch.run(ix, stream)  # captures the graph for this configuration
        torch.cuda.synchronize()
        times = []
        for _ in range(self.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.run(ix, stream)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        return statistics.median(times)

    def tune(self, ix, batch, candidates: Optional[Sequence[dict]] = None) -> dict:
        cands = list(candidates) if candidates is not None else self.candidates(ix)
        feats = self.features(ix, batch.lengths, batch.seeds(ix))
        best, best_ms = None, float("inf")
        for launch in cands:
            ms = self.time_config(ix, batch, launch)
            self.rows.append(Measurement(feats, dict(launch), ms, int(feats["seeds"])))
            if ms < best_ms:
                best, best_ms = dict(launch), ms
        ix.set_launch(**best)
        return {"launch": best, "ms": best_ms}

    def save(self, path: Path) -> None:
        path.write_text(json.dumps([m.__dict__ for m in self.rows]))


class DeviceBatch:
    """A read batch resident on the GPU, plus counters, for tuning and serving."""

    def __init__(self, bases: np.ndarray, offsets: np.ndarray, colors: int, device=0):
        import torch

        self.dev = torch.device("cuda", device)
        self.d_bases = torch.from_numpy(np.ascontiguousarray(bases)).to(self.dev)
        self.d_off = torch.from_numpy(np.ascontiguousarray(offsets).view(np.int64)).to(self.dev)
        self.d_counts = torch.zeros(colors, dtype=torch.int64, device=self.dev)
        self.d_total = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.nbases = int(len(bases))
        self.records = int(len(offsets) - 1)
        self.lengths = np.diff(offsets.astype(np.int64))
        self._seeds = None

    def run(self, ix, stream, use_graph: bool = True) -> None:
        self.d_counts.zero_()
        self.d_total.zero_()
        ix.query_device(self.d_bases.data_ptr(), self.nbases, self.d_off.data_ptr(), self.records,
                        self.d_counts.data_ptr(), self.d_total.data_ptr(),
                        stream=stream.cuda_stream, use_graph=use_graph)

    def seeds(self, ix) -> int:
        if self._seeds is None:
            import torch

            self.run(ix, torch.cuda.current_stream())
            torch.cuda.synchronize()
            self._seeds = int(self.d_total.item())
        return self._seeds


# ---- measurement sweep for the learned planner --------------------------------
# Each setting is an index geometry (built from seeded synthetic genomes by
# zx_build) and a read batch (zx_synth). Device rows time every register-gather
# launch on the resident batch; e2e rows time host-buffer queries for each cut
# with the default launch.
SETTINGS = [
    # name, build options, genome spec (colors, min_len, max_len), reads (kind, length, count)
    ("k31-H4-b8-c64-short", dict(mode="kmers", k=31, H=4, b=8), (64, 100_000, 1_000_000), ("short", 150, 200_000)),
    ("k31-H4-b8-c64-long", dict(mode="kmers", k=31, H=4, b=8), (64, 100_000, 1_000_000), ("long", 5000, 6000)),
    ("k31-H3-b16-c256-short", dict(mode="kmers", k=31, H=3, b=16), (256, 50_000, 500_000), ("short", 150, 200_000)),
    ("k31-H8-b4-c512-short", dict(mode="kmers", k=31, H=8, b=4), (512, 20_000, 200_000), ("short", 150, 100_000)),
    ("k31-H8-b4-c512-long", dict(mode="kmers", k=31, H=8, b=4), (512, 20_000, 200_000), ("long", 3000, 5000)),
    ("k25-H4-b4-c1024-short", dict(mode="kmers", k=25, H=4, b=4), (1024, 10_000, 100_000), ("short", 150, 100_000)),
    ("k31-H2-b32-c16-short", dict(mode="kmers", k=31, H=2, b=32), (16, 1_000_000, 4_000_000), ("short", 150, 200_000)),
    ("k31-H4-b8-c2048-short", dict(mode="kmers", k=31, H=4, b=8), (2048, 5_000, 50_000), ("short", 150, 100_000)),
    ("min-k31-m21-H3-b16-c256-long", dict(mode="minimizers", k=31, m=21, H=3, b=16), (256, 100_000, 1_000_000), ("long", 2000, 20_000)),
    ("min-k49-m31-H4-b8-c128-short", dict(mode="minimizers", k=49, m=31, H=4, b=8), (128, 100_000, 1_000_000), ("short", 150, 200_000)),
    ("mod-k31-d4-H4-b8-c256-short", dict(mode="modimizers", k=31, d=4, H=4, b=8), (256, 50_000, 500_000), ("short", 150, 300_000)),
    ("fin-k31-z10-H4-b8-c128-short", dict(mode="findere", k=31, z=10, H=4, b=8), (128, 50_000, 500_000), ("short", 150, 100_000)),
    ("k31-H4-b1-c256-short", dict(mode="kmers", k=31, H=4, b=1), (256, 50_000, 300_000), ("short", 150, 200_000)),
    ("k63-H4-b8-c128-long", dict(mode="kmers", k=63, H=4, b=8), (128, 100_000, 800_000), ("long", 4000, 4000)),
]
REGISTER_LAUNCHES = [dict(team=t, warps=w, min_blocks=mb, planes=pl)
                     for t in (2, 4, 8, 16, 32) for w in (2, 4, 8) for pl in (0, 1)
                     for mb in ((1, 2, 3) if pl else (2, 3))]
CUTS = (1, 2, 4, 8, 16)


def _build_setting(lib_dir: Path, work: Path, name, opts, genomes, reads, seed):
    import subprocess

    d = work / name
    d.mkdir(parents=True, exist_ok=True)
    colors, lo, hi = genomes
    gdir = d / "genomes"
    gdir.mkdir(parents=True, exist_ok=True)
    if not (gdir / "fof.tsv").exists():
        subprocess.run([str(lib_dir / "zx_synth"), "genomes", "--kind", "pool", "--colors",
                        str(colors), "--min-len", str(lo), "--max-len", str(hi), "--seed",
                        str(seed), "--out", str(gdir)], check=True)
    index = d / "index"
    if not (index / "manifest.json").exists():
        flag = {"k": "-k", "m": "-m", "H": "-H", "b": "-b", "mode": "-i", "z": "-z", "d": "-d"}
        args = [str(lib_dir / "zx_build"), "-f", str(gdir / "fof.tsv"), "-o", str(index), "-q"]
        for key, val in opts.items():
            args += [flag[key], str(val)]
        subprocess.run(args, check=True)
    kind, length, count = reads
    rfile = d / "reads"
    if not Path(str(rfile) + ".offsets").exists():
        subprocess.run([str(lib_dir / "zx_synth"), "reads", "--kind", kind, "--genome-kind",
                        "pool", "--colors", str(colors), "--min-len", str(lo), "--max-len",
                        str(hi), "--seed", str(seed), "--read-seed", str(seed + 7), "--reads",
                        str(count), "--length", str(length), "--sourced", "0.7", "--subst",
                        "0.005", "--format", "raw", "--out", str(rfile)], check=True)
    bases = np.fromfile(str(rfile) + ".bases", dtype=np.uint8)
    offsets = np.fromfile(str(rfile) + ".offsets", dtype=np.uint64)
    return index, bases, offsets


def collect(work: Path, out: Path, reps: int = 5, settings=None, log=print) -> dict:
    """Measure every setting; write {"rows": [...]} to `out`."""
    import torch

    import zindex_b200 as zx

    lib_dir = Path(zx.LIB_DIR)
    rows, defaults = [], {}
    for i, (name, opts, genomes, reads) in enumerate(settings or SETTINGS):
        index, bases, offsets = _build_setting(lib_dir, work, name, opts, genomes, reads, 1000 + i)
        with zx.Index(index) as ix:
            batch = DeviceBatch(bases, offsets, ix.colors)
            feats = Autotuner.features(ix, batch.lengths, batch.seeds(ix))
            tuner = Autotuner(reps=reps)
            default = ix.default_launch()
            defaults[name] = dict(default, blocks=0)
            # The fused kernel's launches; a wide-row default is one more row.
            fused = ix.default_fused_launch()
            launches = [dict(fused, **launch, blocks=0, stage_bytes=0, wide=0)
                        for launch in REGISTER_LAUNCHES]
            if default["wide"]:
                launches.append(dict(default, blocks=0))
            for full in launches:
                ms = tuner.time_config(ix, batch, full)
                rows.append({"setting": name, "features": feats, "launch": full, "e2e": False,
                             "ms": ms})
            ix.set_launch(**default)
            h_bases = torch.from_numpy(bases).pin_memory().numpy()
            h_off = torch.from_numpy(offsets.view(np.int64)).pin_memory().numpy().view(np.uint64)
            for cut in CUTS:
                full = dict(default, cut=cut, blocks=0)
                ix.set_launch(**full)
                ix.query_records(h_bases, h_off)
                times = []
                for _ in range(reps):
                    t0 = time.perf_counter()
                    ix.query_records(h_bases, h_off)
                    times.append((time.perf_counter() - t0) * 1e3)
                rows.append({"setting": name, "features": feats, "launch": full, "e2e": True,
                             "ms": statistics.median(times)})
            mine = [r["ms"] for r in rows if r["setting"] == name and not r["e2e"]]
            log(f"{name}: seeds {int(feats['seeds'])}, device ms min {min(mine):.3f} "
                f"max {max(mine):.3f}")
            del batch
            torch.cuda.empty_cache()
    data = {"device": torch.cuda.get_device_name(0), "reps": reps, "defaults": defaults,
            "rows": rows}
    Path(out).write_text(json.dumps(data))
    return data


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="measurement sweep for the learned planner")
    ap.add_argument("--work", default="/tmp/zx_planner")
    ap.add_argument("--out", required=True)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    collect(Path(a.work), Path(a.out), a.reps)
