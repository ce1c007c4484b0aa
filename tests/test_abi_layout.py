"""CPU: the ctypes mirrors of the C-ABI structs have the header's layout.

Every struct that calamarijoins_b200._lib passes across the boundary is
compiled here by gcc against include/cj_b200.h, and its size and the offset
of each field (by name) are compared with what ctypes lays out. A field
added to the header but not to the binding (or in a different place) fails
this test instead of corrupting memory at run time."""
import ctypes as C
import os
import shutil
import subprocess
import tempfile

import pytest

from calamarijoins_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")

# ctypes mirror -> C type name in include/cj_b200.h
MIRRORS = {
    "ColumnDesc": "cj_column_desc",
    "TableDesc": "cj_table_desc",
    "Attr": "cj_attr",
    "PlanNodeDesc": "cj_plan_node",
    "PlanDesc": "cj_plan_desc",
    "PredNodeC": "cj_pred_node",
    "PredicateC": "cj_predicate",
    "TimingStatsC": "cj_timing_stats",
    "ExecStatsC": "cj_exec_stats",
    "CacheMetaC": "cj_cache_meta",
    "BatchStatsC": "cj_batch_stats",
    "ServerConfigC": "cj_server_config",
    "ServerStatsC": "cj_server_stats",
}


def c_layouts():
    """{C type: (sizeof, {field: offsetof})} as gcc lays the header out."""
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "cj_b200.h"', "int main(void) {"]
    for py, c in MIRRORS.items():
        lines.append(f'    printf("S {c} %zu\\n", sizeof({c}));')
        for name, _ in getattr(_lib, py)._fields_:
            lines.append(f'    printf("F {c} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["    return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        with open(src, "w") as f:
            f.write("\n".join(lines) + "\n")
        res = subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, src, "-o", exe], capture_output=True, text=True)
        assert res.returncode == 0, "a ctypes field name is not in the header:\n" + res.stderr[-3000:]
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    layouts = {}
    for line in out.splitlines():
        parts = line.split()
        if parts[0] == "S":
            layouts.setdefault(parts[1], [0, {}])[0] = int(parts[2])
        else:
            layouts.setdefault(parts[1], [0, {}])[1][parts[2]] = int(parts[3])
    return layouts


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_header():
    layouts = c_layouts()
    for py, c in MIRRORS.items():
        cls = getattr(_lib, py)
        size, offsets = layouts[c]
        assert C.sizeof(cls) == size, f"{py}: ctypes {C.sizeof(cls)} bytes, {c} {size} bytes"
        for name, _ in cls._fields_:
            assert getattr(cls, name).offset == offsets[name], (
                f"{py}.{name}: ctypes offset {getattr(cls, name).offset}, {c} offset {offsets[name]}")
