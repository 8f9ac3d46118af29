"""ctypes binding of libzindex_b200.so (the C ABI in include/zindex.h).

The shared library is built in-tree by zindex_b200.build and loaded from
zindex_b200/_lib/. There is no fallback: if the library is missing or fails to
load, every entry point raises.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_int, c_uint32, c_uint64, c_void_p
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "_lib"
LIB_PATH = LIB_DIR / "libzindex_b200.so"

ZX_OK = 0
ZX_EINVAL = 1
ZX_EFORMAT = 2
ZX_EIO = 3
ZX_ENOMEM = 4
ZX_ECUDA = 5
ZX_ETIMEOUT = 6
ZX_EUNSUPPORTED = 7

# Every symbol include/zindex.h declares.
EXPORTED = (
    "zx_last_error", "zx_open", "zx_close", "zx_index_info", "zx_color_name",
    "zx_color_unique_kmers", "zx_query_file", "zx_query_host", "zx_query_host_plain",
    "zx_query_device", "zx_extract_seeds", "zx_get_launch", "zx_set_launch",
    "zx_default_launch", "zx_write_aggregate", "zx_set_timing", "zx_last_kernel_ms",
    "zx_query_status", "zx_query_device_noalloc", "zx_query_segments", "zx_server_start",
    "zx_server_submit", "zx_server_wait", "zx_server_stats", "zx_server_stop", "zx_mlp_create",
    "zx_mlp_destroy", "zx_mlp_param_count", "zx_mlp_get_params", "zx_mlp_set_params",
    "zx_mlp_loss_grad", "zx_mlp_train", "zx_mlp_predict", "zx_query_per_record",
    "zx_query_records_report", "zx_default_fused_launch",
)


class ZxInfo(ctypes.Structure):
    _fields_ = [
        ("version", c_uint32), ("k", c_uint32), ("hashes", c_uint32),
        ("fingerprint_bits", c_uint32), ("index_mode", c_uint32), ("minimizer_size", c_uint32),
        ("seed", c_uint64), ("colors", c_uint64), ("banks", c_uint64), ("classes", c_uint64),
        ("resident_bytes", c_uint64), ("gather_bytes_per_seed", c_uint64),
        ("gather_sector_bytes_per_seed", c_uint64),
        ("abandoned_hashes", c_uint64), ("recovery", c_int),
        ("load_s", c_double), ("load_banks_s", c_double), ("load_recovery_s", c_double),
    ]


class ZxLaunch(ctypes.Structure):
    _fields_ = [("team", c_int), ("warps", c_int), ("blocks", c_int), ("smem_counters", c_int),
                ("stage_bytes", c_int), ("stages", c_int), ("bulk", c_int), ("min_blocks", c_int),
                ("planes", c_int), ("cut", c_int), ("split", c_int), ("wide", c_int),
                ("order", c_int)]


class ZxServerOptions(ctypes.Structure):
    _fields_ = [("slots", c_int), ("slot_bases", c_uint64), ("slot_records", c_uint64),
                ("slot_requests", c_uint32)]


class ZxServerStats(ctypes.Structure):
    _fields_ = [("submitted", c_uint64), ("completed", c_uint64), ("failed", c_uint64),
                ("batches", c_uint64), ("seeds", c_uint64), ("bases", c_uint64),
                ("p50_s", c_double), ("p99_s", c_double), ("mean_s", c_double),
                ("max_s", c_double), ("elapsed_s", c_double), ("device_bytes", c_uint64),
                ("pinned_bytes", c_uint64)]


class ZxError(RuntimeError):
    """A non-zero status from the C ABI, with the library's message."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


_lib = None


def load() -> ctypes.CDLL:
    """Load libzindex_b200.so (raising if it is absent) and declare signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m zindex_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH))
    P64 = POINTER(c_uint64)
    PF = POINTER(ctypes.c_float)
    sig = {
        "zx_last_error": (c_char_p, []),
        "zx_open": (c_int, [c_char_p, c_int, c_uint64, POINTER(c_void_p)]),
        "zx_close": (None, [c_void_p]),
        "zx_index_info": (c_int, [c_void_p, POINTER(ZxInfo)]),
        "zx_color_name": (c_char_p, [c_void_p, c_uint64]),
        "zx_color_unique_kmers": (c_uint64, [c_void_p, c_uint64]),
        "zx_query_file": (c_int, [c_void_p, c_char_p, c_int, P64, P64, P64]),
        "zx_query_host": (c_int, [c_void_p, c_void_p, P64, c_uint64, c_int, P64, P64]),
        "zx_query_host_plain": (c_int, [c_void_p, c_void_p, P64, c_uint64, c_int, P64, P64]),
        "zx_query_per_record": (c_int, [c_void_p, c_void_p, P64, c_uint64, c_int, P64, P64]),
        "zx_query_records_report": (c_int, [c_void_p, c_char_p, c_int, c_double, c_int,
                                            c_uint64, c_char_p]),
        "zx_query_device": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_uint64, c_int,
                                    c_void_p, c_void_p, c_void_p, c_int]),
        "zx_query_device_noalloc": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_uint64,
                                            c_int, c_void_p, c_void_p, c_void_p]),
        "zx_extract_seeds": (c_int, [c_void_p, c_void_p, P64, c_uint64, P64, c_uint64, P64]),
        "zx_get_launch": (c_int, [c_void_p, POINTER(ZxLaunch)]),
        "zx_set_launch": (c_int, [c_void_p, POINTER(ZxLaunch)]),
        "zx_default_launch": (c_int, [c_void_p, POINTER(ZxLaunch)]),
        "zx_default_fused_launch": (c_int, [c_void_p, POINTER(ZxLaunch)]),
        "zx_set_timing": (c_int, [c_void_p, c_int]),
        "zx_query_status": (c_int, [c_void_p]),
        "zx_last_kernel_ms": (c_int, [c_void_p, POINTER(ctypes.c_float)]),
        "zx_write_aggregate": (c_int, [c_void_p, c_char_p, P64, c_uint64, c_uint64, c_double,
                                       c_double, c_char_p, c_int]),
        "zx_query_segments": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_uint64, P64,
                                      c_uint32, c_int, c_void_p, c_void_p, c_void_p]),
        "zx_server_start": (c_int, [c_void_p, POINTER(ZxServerOptions), POINTER(c_void_p)]),
        "zx_server_submit": (c_int, [c_void_p, c_void_p, P64, c_uint64, c_int, P64]),
        "zx_server_wait": (c_int, [c_void_p, c_uint64, c_int, P64, P64, POINTER(c_double)]),
        "zx_server_stats": (c_int, [c_void_p, c_int, POINTER(ZxServerStats)]),
        "zx_server_stop": (None, [c_void_p]),
        "zx_mlp_create": (c_int, [c_int, c_int, c_int, c_uint64, POINTER(c_void_p)]),
        "zx_mlp_destroy": (None, [c_void_p]),
        "zx_mlp_param_count": (c_uint64, [c_void_p]),
        "zx_mlp_get_params": (c_int, [c_void_p, PF]),
        "zx_mlp_set_params": (c_int, [c_void_p, PF, c_uint64]),
        "zx_mlp_loss_grad": (c_int, [c_void_p, PF, PF, c_uint64, PF, PF]),
        "zx_mlp_train": (c_int, [c_void_p, PF, PF, c_uint64, c_int, ctypes.c_float, PF]),
        "zx_mlp_predict": (c_int, [c_void_p, PF, c_uint64, PF]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != ZX_OK:
        msg = load().zx_last_error()
        raise ZxError(rc, msg.decode() if msg else "unknown error")
