"""The C ABI's public structs as the Python binding declares them.

zindex_b200/_lib.py mirrors zx_info, zx_launch, zx_server_options and
zx_server_report (include/zindex.h) as ctypes structures; a field added or
reordered on one side only would make every call through them read the
wrong bytes. A small C program compiled against the header prints each
struct's size and every field's offset, and they must equal the ctypes
layout.
"""
import ctypes
import subprocess
from pathlib import Path

import pytest

from zindex_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]

STRUCTS = {
    "zx_info": _lib.ZxInfo,
    "zx_launch": _lib.ZxLaunch,
    "zx_server_options": _lib.ZxServerOptions,
    "zx_server_report": _lib.ZxServerStats,
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    d = tmp_path_factory.mktemp("layout")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "zindex.h"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = d / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = d / "layout"
    subprocess.run(["gcc", "-std=c11", f"-I{ROOT / 'include'}", "-o", str(exe), str(src)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    table = {}
    for line in out.splitlines():
        name, field, value = line.split()
        table[(name, field)] = int(value)
    return table


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_ctypes_layout_matches_the_header(c_layout, cname):
    cls = STRUCTS[cname]
    assert ctypes.sizeof(cls) == c_layout[(cname, "size")], cname
    for field, _ in cls._fields_:
        assert getattr(cls, field).offset == c_layout[(cname, field)], (cname, field)
