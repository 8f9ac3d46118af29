"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import re
from pathlib import Path

import zindex_b200._lib as zlib

HEADER = Path(__file__).resolve().parents[1] / "include" / "zindex.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zx_[a-z_]+)\s*\(", text)))


def test_header_declares_the_binding_table():
    assert set(declared_symbols()) == set(zlib.EXPORTED)


def test_library_exports_every_declared_symbol(native):
    lib = ctypes.CDLL(str(zlib.LIB_PATH))
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_errors_surface_without_a_gpu_call(native):
    lib = zlib.load()
    handle = ctypes.c_void_p()
    rc = lib.zx_open(b"/nonexistent/index", 0, 0, ctypes.byref(handle))
    assert rc != zlib.ZX_OK
    assert lib.zx_last_error()
