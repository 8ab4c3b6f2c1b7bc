"""The ctypes mirrors of the C ABI's structs (superman_b200/_lib.py) have the
C layout: for every struct, the size and every field's offset as the C
compiler lays them out from include/superman_b200.h (CPU only: gcc)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from superman_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = [_lib.spb_options, _lib.spb_result, _lib.spb_pipeline_result, _lib.spb_server_config,
           _lib.spb_request_result, _lib.spb_server_stats]


def test_ctypes_structs_match_the_c_layout(tmp_path):
    gcc = shutil.which("gcc") or "/usr/bin/gcc"
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "superman_b200.h"', "int main(void) {"]
    for st in STRUCTS:
        name = st.__name__
        lines.append(f'printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in st._fields_:
            lines.append(f'printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    r = subprocess.run([gcc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True, timeout=120)
    if r.returncode != 0:
        pytest.fail(r.stderr[-2000:])
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        *key, value = line.split()
        got[tuple(key)] = int(value)
    for st in STRUCTS:
        name = st.__name__
        assert got[(name, "size")] == ctypes.sizeof(st), name
        for field, _ in st._fields_:
            assert got[(name, field)] == getattr(st, field).offset, (name, field)
