"""Learned launch planner: a two-layer FP32 perceptron trained on the GPU.

The planner predicts, for an index geometry, a read batch and one candidate
launch configuration, the log of the query time; it then picks the candidate
with the lowest prediction. Two decisions are made per incoming batch:

* the launch configuration of the fused kernel (team size, warps per block,
  register budget, counting form) from device-time measurements, and
* the batch cut of host-buffer queries (how many pipelined chunks the batch is
  split into) from end-to-end measurements with the chosen launch.

The network (hidden 32, ReLU) is trained by the library's own CUDA forward,
backward and Adam kernels (zx_mlp_* in include/zindex.h) on rows measured by
the autotuner (zindex_b200.tuning). Launches and cuts are chosen by
verification: the network ranks all candidates, its top few and the default
are timed on the batch, and the fastest wins, so a plan is never slower than the default
(up to timing noise) and costs a handful of timings instead of an exhaustive
search, which stays the fallback and the measure of its regret. The planner
never changes results: every launch configuration and cut gives the same
counts.
"""
from __future__ import annotations

import ctypes
import json
import math
from ctypes import POINTER, byref, c_float, c_uint64, c_void_p
from dataclasses import dataclass
from pathlib import Path
from typing import Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib

FEATURES = (
    "log2_hashes", "log2_bits", "log2_colors", "classes", "mode_kmers", "mode_minimizers",
    "mode_modimizers", "mode_findere", "log2_gather_bytes", "log2_len_mean", "log2_seeds",
    "log2_team", "log2_warps", "min_blocks", "planes", "smem_counters", "log2_stage_bytes",
    "bulk", "log2_cut", "e2e", "log2_chunks", "team_over_chunks", "plane_word_fits",
    "idle_lanes",
)
DATA = Path(__file__).resolve().parent / "data" / "planner_measurements.json"


def encode(features: Dict[str, float], launch: Dict[str, int], e2e: bool = False) -> np.ndarray:
    """Fixed-scale feature vector (each entry roughly in [0, 1]). Besides the
    raw geometry it carries how a launch meets the rows: 16-byte chunks per
    fingerprint-plane row, team size against chunks, whether a lane's fields
    fit one bit-plane word (4 x chunks per lane <= b), idle lanes."""
    mode = int(features.get("mode", 0))
    hashes, bits = max(1.0, features["hashes"]), max(1.0, features["bits"])
    classes = max(1.0, features.get("classes", 1.0))
    row_bytes = features["gather_bytes"] / (hashes * classes)
    chunks = max(1.0, math.ceil(row_bytes / 16.0))
    team = max(1, launch.get("team", 8))
    per_lane = math.ceil(chunks / team)
    planes = float(launch.get("planes", 0))
    return np.array([
        math.log2(hashes) / 5.0,
        math.log2(bits) / 5.0,
        math.log2(max(1.0, features["colors"])) / 14.0,
        classes / 8.0,
        float(mode == 0), float(mode == 1), float(mode == 2), float(mode == 3),
        math.log2(max(1.0, features["gather_bytes"])) / 16.0,
        math.log2(1.0 + features["len_mean"]) / 17.0,
        math.log2(1.0 + features["seeds"]) / 30.0,
        math.log2(team) / 5.0,
        math.log2(max(1, launch.get("warps", 8))) / 3.0,
        float(launch.get("min_blocks", 2) - 2),
        planes,
        float(launch.get("smem_counters", 1)),
        math.log2(1 + launch.get("stage_bytes", 0)) / 16.0,
        float(launch.get("bulk", 0)),
        math.log2(max(1, launch.get("cut", 1))) / 6.0,
        float(e2e),
        math.log2(chunks) / 8.0,
        max(-5.0, min(5.0, math.log2(team / chunks))) / 5.0,
        planes * float(4 * per_lane <= bits),
        max(0.0, 1.0 - chunks / team),
    ], dtype=np.float32)


def _pf(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_float))


class Mlp:
    """The network on the GPU (zx_mlp_*): y = w2 . relu(W1 x + b1) + b2."""

    def __init__(self, inputs: int, hidden: int = 32, seed: int = 1, device: int = 0):
        lib = _lib.load()
        h = c_void_p()
        _lib.check(lib.zx_mlp_create(int(device), int(inputs), int(hidden), int(seed), byref(h)))
        self._h = h
        self.inputs, self.hidden = inputs, hidden
        self.count = int(lib.zx_mlp_param_count(self._h))

    def params(self) -> np.ndarray:
        p = np.zeros(self.count, dtype=np.float32)
        _lib.check(_lib.load().zx_mlp_get_params(self._h, _pf(p)))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        _lib.check(_lib.load().zx_mlp_set_params(self._h, _pf(p), len(p)))

    def loss_grad(self, x: np.ndarray, t: np.ndarray) -> Tuple[float, np.ndarray]:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(self.count, dtype=np.float32)
        loss = c_float()
        _lib.check(_lib.load().zx_mlp_loss_grad(self._h, _pf(x), _pf(t), len(t), byref(loss),
                                               _pf(g)))
        return float(loss.value), g

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int, lr: float) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = c_float()
        _lib.check(_lib.load().zx_mlp_train(self._h, _pf(x), _pf(t), len(t), int(epochs),
                                           float(lr), byref(loss)))
        return float(loss.value)

    def predict(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros(len(x), dtype=np.float32)
        _lib.check(_lib.load().zx_mlp_predict(self._h, _pf(x), len(x), _pf(y)))
        return y

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().zx_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Row:
    """One measurement: a setting (index + batch features), a launch, e2e or
    device timing, and its milliseconds."""
    setting: str
    features: Dict[str, float]
    launch: Dict[str, int]
    e2e: bool
    ms: float


def load_rows(path: Path = DATA) -> Tuple[List[Row], Dict[str, Dict[str, int]]]:
    """Measured rows and the default launch of each setting."""
    raw = json.loads(Path(path).read_text())
    rows = [Row(r["setting"], r["features"], r["launch"], bool(r["e2e"]), float(r["ms"]))
            for r in raw["rows"] if math.isfinite(r["ms"])]
    return rows, raw["defaults"]


# Margins of the two decisions: launches are taken as predicted; the cut of
# host batches only moves off the default when the network predicts a clear
# win (the default cut was within 2% of the best in the measured settings).
LAUNCH_MARGIN = 0.0
CUT_MARGIN = 0.06
SHORTLIST = 3  # predicted-best launches timed beside the default
POOL = 8  # device launches nearest the default that the network ranks


class Planner:
    """Train on measured rows; choose launch and cut for new batches.

    Targets are relative: for each setting, log(ms) minus the mean log(ms) of
    that setting's rows of the same kind (device or end-to-end), scaled by the
    spread over all rows. Only the ranking of candidates within one batch
    matters for a choice, and relative targets keep the network from spending
    its capacity on the large differences between settings."""

    def __init__(self, hidden: int = 32, seed: int = 1, device: int = 0):
        self.net = Mlp(len(FEATURES), hidden, seed, device)
        self.sigma = 1.0

    def fit(self, rows: Sequence[Row], epochs: int = 3000, lr: float = 3e-3) -> float:
        x = np.stack([encode(r.features, r.launch, r.e2e) for r in rows])
        y = np.log(np.array([r.ms for r in rows], dtype=np.float64))
        groups: Dict[Tuple[str, bool], List[int]] = {}
        for i, r in enumerate(rows):
            groups.setdefault((r.setting, r.e2e), []).append(i)
        rel = np.zeros_like(y)
        for idx in groups.values():
            rel[idx] = y[idx] - y[idx].mean()
        self.sigma = float(rel.std() or 1.0)
        return self.net.train(x, (rel / self.sigma).astype(np.float32), epochs, lr)

    def predict_cost(self, features: Dict[str, float], launches: Sequence[Dict[str, int]],
                     e2e: bool = False) -> np.ndarray:
        """Predicted time of each candidate relative to the batch's typical
        time (only ratios between candidates of one batch are meaningful)."""
        x = np.stack([encode(features, l, e2e) for l in launches])
        return np.exp(self.net.predict(x).astype(np.float64) * self.sigma)

    def choose(self, features: Dict[str, float], launches: Sequence[Dict[str, int]],
               e2e: bool = False, default: Optional[Dict[str, int]] = None,
               margin: float = 0.0, pool: Optional[int] = None) -> Dict[str, int]:
        """The candidate with the lowest predicted time; with `default` given,
        the default unless the pick is predicted faster by more than `margin`
        (a fraction), and for device launches the pick comes from the `pool`
        candidates nearest the default (POOL by default; 0 = all): on the
        committed measurements that untimed pick beats the default (1.024x,
        leave-one-setting-out), the pick among all launches does not."""
        if default is not None:
            if pool is None:
                pool = 0 if e2e else POOL
            if pool:
                dkey = launch_key(default)
                launches = sorted([l for l in launches if launch_key(l) != dkey],
                                  key=lambda l: _launch_distance(l, default))[:pool]
        cands = list(launches) + ([default] if default is not None else [])
        pred = self.predict_cost(features, cands, e2e)
        k = int(np.argmin(pred[: len(launches)]))
        if default is not None and not pred[k] < pred[-1] * (1.0 - margin):
            return dict(default)
        return dict(launches[k])

    def shortlist(self, features: Dict[str, float], launches: Sequence[Dict[str, int]],
                  default: Dict[str, int], k: int = SHORTLIST, e2e: bool = False,
                  pool: Optional[int] = None) -> List[Dict[str, int]]:
        """The k candidates with the lowest predicted time, then the default
        (without duplicates): the launches worth timing on the batch. Device
        launches are ranked among the `pool` candidates nearest the default
        launch (POOL by default; 0 = all): on the committed measurements the
        network ranks that neighbourhood better than it ranks every launch."""
        if pool is None:
            pool = 0 if e2e else POOL
        if pool:
            dkey = launch_key(default)
            launches = sorted([l for l in launches if launch_key(l) != dkey],
                              key=lambda l: _launch_distance(l, default))[:pool]
        order = np.argsort(self.predict_cost(features, launches, e2e))
        out, seen = [], set()
        for i in list(order[:k]):
            key = launch_key(launches[int(i)])
            if key not in seen:
                seen.add(key)
                out.append(dict(launches[int(i)]))
        if launch_key(default) not in seen:
            out.append(dict(default))
        return out

    def save(self, path: Path) -> None:
        Path(path).write_text(json.dumps({
            "features": list(FEATURES), "hidden": self.net.hidden, "sigma": self.sigma,
            "params": self.net.params().tolist()}))

    @classmethod
    def load(cls, path: Path, device: int = 0) -> "Planner":
        d = json.loads(Path(path).read_text())
        if tuple(d["features"]) != FEATURES:
            raise ValueError("planner file was trained on other features")
        p = cls(hidden=int(d["hidden"]), device=device)
        p.sigma = float(d["sigma"])
        p.net.set_params(np.array(d["params"], dtype=np.float32))
        return p




def launch_key(l: Dict[str, int]) -> Tuple:
    return tuple(sorted((k, int(v)) for k, v in l.items() if k != "blocks"))


# A single untimed pick leaves the default only for a predicted win above this.
TOP1_MARGIN = 0.05


def _launch_distance(l: Dict[str, int], d: Dict[str, int]) -> float:
    """Steps between two launches in the default rule's own parameters."""
    step = lambda a, b: abs(np.log2(max(a, 1)) - np.log2(max(b, 1)))
    return (step(l["team"], d["team"]) + step(l["warps"], d["warps"]) +
            abs(l["min_blocks"] - d["min_blocks"]) + 2 * abs(l["planes"] - d["planes"]))


def evaluate(planner: Planner, rows: Sequence[Row], default: Dict[str, int],
             e2e: bool = False, k: int = SHORTLIST) -> Dict[str, float]:
    """Scores the planner on measured rows of one kind, per setting, against
    the exhaustive best (regret) and the default launch (gain); geometric
    means over settings. Device rows: the shortlist is "timed" by reading its
    measured times (the fastest of the k predictions and the default wins),
    and the network's top prediction alone is scored too. End-to-end rows:
    the network's best cut and the default cut, the faster kept."""
    by: Dict[str, List[Row]] = {}
    for r in rows:
        if r.e2e == e2e:
            by.setdefault(r.setting, []).append(r)
    regrets, gains, top_gains, timed = [], [], [], []
    rand_gains, heur_gains, guard_gains, all_gains, near_top = [], [], [], [], []
    rng = np.random.default_rng(12345)
    dkey = launch_key(default)
    for setting, rs in by.items():
        table = {launch_key(r.launch): r for r in rs}
        if dkey not in table:
            continue
        best = min(r.ms for r in rs)
        launches = [r.launch for r in rs]
        if e2e:
            # The network's best cut and the default, timed end to end.
            short = planner.shortlist(rs[0].features, launches, default, 1, e2e=True)
            chosen = min(table[launch_key(l)].ms for l in short)
            timed.append(len(short))
        else:
            short = planner.shortlist(rs[0].features, launches, default, k)
            chosen = min(table[launch_key(l)].ms for l in short)
            top = planner.choose(rs[0].features, launches)
            top_gains.append(table[dkey].ms / table[launch_key(top)].ms)
            guard = planner.choose(rs[0].features, launches, default=default,
                                   margin=TOP1_MARGIN, pool=0)
            guard_gains.append(table[dkey].ms / table[launch_key(guard)].ms)
            # The network ranking every launch (no neighbourhood).
            wide = planner.shortlist(rs[0].features, launches, default, k, pool=0)
            all_gains.append(table[dkey].ms / min(table[launch_key(l)].ms for l in wide))
            timed.append(len(short))
            # The same timing budget without the network: k random candidates
            # plus the default (mean over draws), and the k candidates nearest
            # the default launch in its own parameters (the rule the default
            # follows, one step off in team size, warps or budget).
            others = [l for l in launches if launch_key(l) != dkey]
            draws = []
            for _ in range(64):
                pick = rng.choice(len(others), size=min(k, len(others)), replace=False)
                draws.append(min([table[dkey].ms] + [table[launch_key(others[i])].ms for i in pick]))
            rand_gains.append(float(np.exp(np.mean(np.log(table[dkey].ms / np.array(draws))))))
            near = sorted(others, key=lambda l: _launch_distance(l, default))[:k]
            heur_gains.append(table[dkey].ms / min([table[dkey].ms] +
                                                   [table[launch_key(l)].ms for l in near]))
            # An untimed pick inside the default's neighbourhood, kept only
            # when predicted faster than the default by the margin.
            pick = planner.choose(rs[0].features, launches, default=default, margin=TOP1_MARGIN)
            near_top.append(table[dkey].ms / table[launch_key(pick)].ms)
        regrets.append(chosen / best)
        gains.append(table[dkey].ms / chosen)
    gm = lambda v: float(np.exp(np.mean(np.log(v)))) if v else float("nan")
    return {"settings": len(gains), "regret": gm(regrets) - 1.0, "gain_over_default": gm(gains),
            "worst_gain": min(gains) if gains else float("nan"),
            "top1_gain_over_default": gm(top_gains),
            "top1_guarded_gain_over_default": gm(guard_gains),
            "top1_nearby_guarded_gain_over_default": gm(near_top),
            "random_shortlist_gain_over_default": gm(rand_gains),
            "network_over_all_launches_gain_over_default": gm(all_gains),
            "heuristic_shortlist_gain_over_default": gm(heur_gains),
            "timed_per_setting": float(np.mean(timed)),
            "candidates_per_setting": float(np.mean([len(v) for v in by.values()]))}
