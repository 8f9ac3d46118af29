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
MIN_BLOCKS = (2, 3)
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
