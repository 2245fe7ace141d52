"""The ctypes mirrors in hytgraph_b200/capi.py have the C layout of
include/hyt/capi.h: for every struct both declare, sizeof and the offset of
every field agree (compiled with gcc against the header, no GPU)."""
from __future__ import annotations

import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _mirrored_structs(capi):
    header = (ROOT / "include" / "hyt" / "capi.h").read_text()
    declared = set(re.findall(r"typedef struct (hyt_\w+) \{", header))
    out = {}
    for name in sorted(declared):
        cls = getattr(capi, name, None)
        if isinstance(cls, type) and issubclass(cls, C.Structure):
            out[name] = cls
    return out


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc is not installed")
def test_ctypes_structs_match_the_c_header(hyt, tmp_path):
    structs = _mirrored_structs(hyt.capi)
    assert len(structs) >= 20, sorted(structs)
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "hyt/capi.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'    printf("{name} size %zu\\n", sizeof({name}));')
        for field, *_ in cls._fields_:
            lines.append(f'    printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        name, key, val = line.split()
        got[(name, key)] = int(val)
    for name, cls in structs.items():
        assert C.sizeof(cls) == got[(name, "size")], name
        for field, *_ in cls._fields_:
            assert getattr(cls, field).offset == got[(name, field)], (name, field)
