"""zindex_b200 — the Zindex (zorindex) query hot path on NVIDIA B200.

Host-side mirror of the reference's query interface:

* ``Index(index_dir)`` loads and validates an index directory into HBM
  (Index::load_mode, src/power_merge/storage.rs:2273-2707).
* ``Index.query_file(path)`` / ``Index.query_records(bases, offsets)`` return
  per-colour match counts and the feature total, the numbers behind
  ``print_aggregate`` (storage.rs:3817-3844).
* ``query_command(index_dir, query, min_ratio, recover)`` prints the aggregate
  TSV like ``query_command_with_recovery`` (storage.rs:3722-3744).
* ``Server(index)`` answers many query requests from a resident index with
  continuous batching (one segmented launch per batch, per-request counts).

All compute runs in the CUDA kernels of libzindex_b200.so; this module only
moves buffers across the C ABI (include/zindex.h).
"""
from __future__ import annotations

import ctypes
import sys
import time
from ctypes import POINTER, byref, c_uint64, c_void_p
from pathlib import Path
from typing import Optional, Sequence, Tuple, Union

import numpy as np

from . import _lib
from ._lib import ZxError, ZxInfo, ZxLaunch

__all__ = ["Index", "Server", "ZxError", "query_command", "query_records_command", "pack_records",
           "LIB_DIR"]

LIB_DIR = _lib.LIB_DIR
INDEX_MODES = ("kmers", "minimizers", "modimizers", "findere")


def _p64(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_uint64))


def pack_records(records: Sequence[Union[bytes, str]]) -> Tuple[np.ndarray, np.ndarray]:
    """Concatenate sequences into (bases uint8, offsets uint64[n+1])."""
    parts = [r.encode() if isinstance(r, str) else bytes(r) for r in records]
    offsets = np.zeros(len(parts) + 1, dtype=np.uint64)
    if parts:
        offsets[1:] = np.cumsum([len(p) for p in parts], dtype=np.uint64)
    bases = np.frombuffer(b"".join(parts), dtype=np.uint8).copy()
    return bases, offsets


class Index:
    """An index directory made resident in HBM of one GPU."""

    def __init__(self, index_dir: Union[str, Path], device: int = 0, hbm_budget: int = 0):
        lib = _lib.load()
        handle = c_void_p()
        _lib.check(lib.zx_open(str(index_dir).encode(), int(device), int(hbm_budget), byref(handle)))
        self._h = handle
        self.path = Path(index_dir)
        info = ZxInfo()
        _lib.check(lib.zx_index_info(self._h, byref(info)))
        self.info = info
        self.colors = int(info.colors)
        self.names = [lib.zx_color_name(self._h, c).decode() for c in range(self.colors)]
        self.unique_kmers = [int(lib.zx_color_unique_kmers(self._h, c)) for c in range(self.colors)]

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().zx_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- queries --------------------------------------------------------------
    @property
    def mode(self) -> str:
        return INDEX_MODES[self.info.index_mode]

    def query_file(self, path: Union[str, Path], recover: bool = True):
        """(counts uint64[colors], total, probes) for a FASTA/FASTQ file."""
        counts = np.zeros(self.colors, dtype=np.uint64)
        total, probes = c_uint64(), c_uint64()
        _lib.check(_lib.load().zx_query_file(self._h, str(path).encode(), int(recover),
                                            _p64(counts), byref(total), byref(probes)))
        return counts, int(total.value), int(probes.value)

    def query_records(self, bases: np.ndarray, offsets: np.ndarray, recover: bool = True,
                      plain: bool = False):
        """(counts, total) for records bases[offsets[r]:offsets[r+1]] in host memory."""
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        counts = np.zeros(self.colors, dtype=np.uint64)
        total = c_uint64()
        fn = _lib.load().zx_query_host_plain if plain else _lib.load().zx_query_host
        _lib.check(fn(self._h, bases.ctypes.data_as(c_void_p), _p64(offsets), len(offsets) - 1,
                      int(recover), _p64(counts), byref(total)))
        return counts, int(total.value)

    def query_per_record(self, bases: np.ndarray, offsets: np.ndarray, recover: bool = True,
                         counts: Optional[np.ndarray] = None, totals: Optional[np.ndarray] = None):
        """(counts uint64[records, colors], totals uint64[records]): each record
        bases[offsets[r]:offsets[r+1]] counted as if queried alone. `counts` and
        `totals` may be given (C-contiguous uint64 of those shapes, e.g. views of
        page-locked buffers, which the device writes at full PCIe rate)."""
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        records = len(offsets) - 1
        if counts is None:
            counts = np.zeros((records, self.colors), dtype=np.uint64)
        if totals is None:
            totals = np.zeros(records, dtype=np.uint64)
        if (counts.dtype != np.uint64 or counts.shape != (records, self.colors)
                or not counts.flags.c_contiguous or totals.dtype != np.uint64
                or totals.shape != (records,) or not totals.flags.c_contiguous):
            raise ValueError("counts must be uint64[records, colors] and totals uint64[records], "
                             "C-contiguous")
        _lib.check(_lib.load().zx_query_per_record(self._h, bases.ctypes.data_as(c_void_p),
                                                  _p64(offsets), records, int(recover),
                                                  _p64(counts), _p64(totals)))
        return counts, totals

    def query_records_report(self, path: Union[str, Path], out: Union[str, Path, None] = None,
                             min_ratio: float = 0.0, fmt: str = "tsv", batch: int = 4096,
                             recover: bool = True) -> None:
        """Per-record report of a FASTA/FASTQ file (`zorindex query --records`)
        written to `out` (None: stdout); fmt "tsv" or "compact"."""
        if fmt not in ("tsv", "compact"):
            raise ValueError("fmt must be 'tsv' or 'compact'")
        _lib.check(_lib.load().zx_query_records_report(
            self._h, str(path).encode(), int(recover), float(min_ratio), int(fmt == "compact"),
            int(batch), None if out is None else str(out).encode()))

    def query_device(self, d_bases: int, nbases: int, d_offsets: int, records: int,
                     d_counts: int, d_total: int, stream: int = 0, recover: bool = True,
                     use_graph: bool = True) -> None:
        """Enqueue a query of a device-resident batch (raw device pointers)."""
        _lib.check(_lib.load().zx_query_device(self._h, c_void_p(d_bases), nbases,
                                              c_void_p(d_offsets), records, int(recover),
                                              c_void_p(d_counts), c_void_p(d_total),
                                              c_void_p(stream), int(use_graph)))

    def query_device_noalloc(self, d_bases: int, nbases: int, d_offsets: int, records: int,
                             d_counts: int, d_total: int, stream: int = 0,
                             recover: bool = True) -> None:
        """Enqueue a query of a device-resident batch without allocating any
        device memory (scratch in a static 64 MiB array per GPU; calls must not
        overlap on the GPU). For callers that cannot allocate while querying."""
        _lib.check(_lib.load().zx_query_device_noalloc(self._h, c_void_p(d_bases), nbases,
                                                      c_void_p(d_offsets), records, int(recover),
                                                      c_void_p(d_counts), c_void_p(d_total),
                                                      c_void_p(stream)))

    def query_segments(self, d_bases: int, nbases: int, d_offsets: int, records: int,
                       seg_records: np.ndarray, d_counts: int, d_totals: int, stream: int = 0,
                       recover: bool = True) -> None:
        """Enqueue several requests coalesced into one launch: request s owns
        records seg_records[s] .. seg_records[s+1]-1 of the device batch; its
        counts go to row s of d_counts (segments x colours, uint64) and its
        total to d_totals[s]. Each row equals the request queried alone."""
        seg = np.ascontiguousarray(seg_records, dtype=np.uint64)
        _lib.check(_lib.load().zx_query_segments(
            self._h, c_void_p(d_bases), nbases, c_void_p(d_offsets), records, _p64(seg),
            len(seg) - 1, int(recover), c_void_p(d_counts), c_void_p(d_totals), c_void_p(stream)))

    def extract_seeds(self, bases: np.ndarray, offsets: np.ndarray) -> np.ndarray:
        """Seeds of the records in record/window order (extraction only)."""
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        count = c_uint64()
        lib = _lib.load()
        _lib.check(lib.zx_extract_seeds(self._h, bases.ctypes.data_as(c_void_p), _p64(offsets),
                                        len(offsets) - 1, None, 0, byref(count)))
        out = np.zeros(max(1, count.value), dtype=np.uint64)
        _lib.check(lib.zx_extract_seeds(self._h, bases.ctypes.data_as(c_void_p), _p64(offsets),
                                        len(offsets) - 1, _p64(out), len(out), byref(count)))
        return out[: count.value]

    # -- measurement ----------------------------------------------------------
    def set_timing(self, on: bool = True) -> None:
        _lib.check(_lib.load().zx_set_timing(self._h, int(on)))

    def last_kernel_ms(self) -> float:
        ms = ctypes.c_float()
        _lib.check(_lib.load().zx_last_kernel_ms(self._h, byref(ms)))
        return float(ms.value)

    # -- launch configuration -------------------------------------------------
    @staticmethod
    def _launch_dict(l: ZxLaunch) -> dict:
        return {"team": l.team, "warps": l.warps, "blocks": l.blocks,
                "smem_counters": l.smem_counters, "stage_bytes": l.stage_bytes,
                "stages": l.stages, "bulk": l.bulk, "min_blocks": l.min_blocks,
                "planes": l.planes, "cut": l.cut, "split": l.split, "wide": l.wide,
                "order": l.order}

    def launch(self) -> dict:
        l = ZxLaunch()
        _lib.check(_lib.load().zx_get_launch(self._h, byref(l)))
        return self._launch_dict(l)

    def default_launch(self) -> dict:
        l = ZxLaunch()
        _lib.check(_lib.load().zx_default_launch(self._h, byref(l)))
        return self._launch_dict(l)

    def default_fused_launch(self) -> dict:
        """The default launch with the wide-row form off."""
        l = ZxLaunch()
        _lib.check(_lib.load().zx_default_fused_launch(self._h, byref(l)))
        return self._launch_dict(l)

    def set_launch(self, team: int = None, warps: int = None, blocks: int = 0,
                   smem_counters: Optional[int] = None, stage_bytes: Optional[int] = None,
                   stages: Optional[int] = None, bulk: Optional[int] = None,
                   min_blocks: Optional[int] = None, planes: Optional[int] = None,
                   cut: Optional[int] = None, split: Optional[int] = None,
                   wide: Optional[int] = None, order: Optional[int] = None, **_ignored):
        """Change the launch configuration (never changes results); unset
        fields keep their default values (a default 255-register budget,
        min_blocks 1, becomes 2 when the per-hit or staged form is asked for;
        naming a field of the fused kernel's forms - team, planes, stage_bytes,
        split or min_blocks - without `wide` selects the fused kernel)."""
        d = self.default_launch()
        if wide is None:
            fused = any(v is not None for v in (team, planes, stage_bytes, split, min_blocks))
            wide = 0 if fused else d["wide"]
        if not wide and d["wide"]:
            d = self.default_fused_launch()
        if min_blocks is None and d["min_blocks"] == 1 and (planes == 0 or (stage_bytes or 0) > 0):
            d["min_blocks"] = 2
        l = ZxLaunch(int(d["team"] if team is None else team), int(d["warps"] if warps is None else warps),
                     int(blocks), int(d["smem_counters"] if smem_counters is None else smem_counters),
                     int(d["stage_bytes"] if stage_bytes is None else stage_bytes),
                     int(d["stages"] if stages is None else stages),
                     int(d["bulk"] if bulk is None else bulk),
                     int(d["min_blocks"] if min_blocks is None else min_blocks),
                     int(d["planes"] if planes is None else planes),
                     int(d["cut"] if cut is None else cut),
                     int(d["split"] if split is None else split), int(wide),
                     int(d["order"] if order is None else order))
        _lib.check(_lib.load().zx_set_launch(self._h, byref(l)))

    def query_status(self) -> None:
        """Raise if a bounded device wait expired in an asynchronous query."""
        _lib.check(_lib.load().zx_query_status(self._h))

    # -- output ---------------------------------------------------------------
    def format_aggregate(self, counts, total: int, min_ratio: float = 0.0) -> str:
        """The stdout TSV of print_aggregate (storage.rs:3817-3844)."""
        lines = ["color\tmatches\tratio\tunique_kmers"]
        for c in range(self.colors):
            ratio = 0.0 if total == 0 else int(counts[c]) / total
            if ratio >= min_ratio:
                lines.append(f"{self.names[c]}\t{int(counts[c])}\t{ratio:.8f}\t{self.unique_kmers[c]}")
        return "\n".join(lines) + "\n"

    def write_aggregate(self, label: str, counts, total: int, probes: int, min_ratio: float = 0.0,
                        seconds: float = 0.0, out_path: Optional[str] = None, stats: bool = True):
        counts = np.ascontiguousarray(counts, dtype=np.uint64)
        _lib.check(_lib.load().zx_write_aggregate(
            self._h, label.encode(), _p64(counts), int(total), int(probes), float(min_ratio),
            float(seconds), out_path.encode() if out_path else None, int(stats)))


class Server:
    """Request server over a resident Index (see zx_server_start in include/zindex.h).

    submit() copies a request and returns a ticket; wait() returns its
    (counts, total, latency_s). Requests are admitted into batches as batch
    slots free up (continuous batching) and answered by segmented launches on
    per-slot streams. The Index must stay open while the server runs.
    """

    def __init__(self, index: Index, slots: int = 0, slot_bases: int = 0, slot_records: int = 0,
                 slot_requests: int = 0):
        self.index = index
        opts = _lib.ZxServerOptions(int(slots), int(slot_bases), int(slot_records),
                                    int(slot_requests))
        handle = c_void_p()
        _lib.check(_lib.load().zx_server_start(index._h, byref(opts), byref(handle)))
        self._h = handle

    def submit(self, bases: np.ndarray, offsets: np.ndarray, recover: bool = True) -> int:
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        ticket = c_uint64()
        _lib.check(_lib.load().zx_server_submit(self._h, bases.ctypes.data_as(c_void_p),
                                               _p64(offsets), len(offsets) - 1, int(recover),
                                               byref(ticket)))
        return int(ticket.value)

    def wait(self, ticket: int, timeout_ms: int = -1):
        counts = np.zeros(self.index.colors, dtype=np.uint64)
        total, latency = c_uint64(), ctypes.c_double()
        _lib.check(_lib.load().zx_server_wait(self._h, int(ticket), int(timeout_ms), _p64(counts),
                                             byref(total), byref(latency)))
        return counts, int(total.value), float(latency.value)

    def stats(self, reset: bool = False) -> dict:
        st = _lib.ZxServerStats()
        _lib.check(_lib.load().zx_server_stats(self._h, int(reset), byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().zx_server_stop(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def query_records_command(index_dir, query, min_ratio: float = 0.0, recover: bool = True,
                          batch_size: int = 4096, fmt: str = "tsv", device: int = 0) -> None:
    """Print the per-record report, as `zorindex query -i DIR -q FILE -r [-F FMT] [-a R]
    [-B N]` (query_records_command_with_memory, storage.rs:3626-3720)."""
    with Index(index_dir, device=device) as ix:
        t0 = time.perf_counter()
        ix.query_records_report(query, None, min_ratio=min_ratio, fmt=fmt, batch=batch_size,
                                recover=recover)
        print(f"query_timings\tquery_s={time.perf_counter() - t0:.6f}", file=sys.stderr)


def query_command(index_dir, query, min_ratio: float = 0.0, recover: bool = True,
                  device: int = 0) -> None:
    """Print the aggregate query report, as `zorindex query -i DIR -q FILE -a R`."""
    if not 0.0 <= min_ratio <= 1.0:
        raise ValueError("--min-ratio must be in [0, 1]")
    with Index(index_dir, device=device) as ix:
        t0 = time.perf_counter()
        counts, total, probes = ix.query_file(query, recover=recover)
        ix.write_aggregate(str(query), counts, total, probes, min_ratio, time.perf_counter() - t0)
