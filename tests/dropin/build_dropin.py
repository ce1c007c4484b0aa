"""Builds tests/dropin/dropin_harness: the drop-in execute.cpp
(calamarijoins_b200/contest/execute.cpp) compiled against the reference's
own plan.h, plus a driver that runs one serialized plan through
Contest::build_context / execute / destroy_context.

Needs the reference source tree (located by oracle/build_oracle.reference_dir);
the reference's re2 / range-v3 includes are satisfied by oracle/ref_shim.
The binary links libcj_b200.so through an rpath relative to itself.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "dropin_harness")


def build(force: bool = False) -> str | None:
    sys.path.insert(0, ROOT)
    from oracle.build_oracle import reference_dir
    ref = reference_dir()
    if ref is None or not os.path.isfile(os.path.join(ref, "include", "data_model", "plan.h")):
        return None
    import torch
    fmt_inc = os.path.join(os.path.dirname(torch.__file__), "include")
    srcs = [os.path.join(ROOT, "calamarijoins_b200", "contest", "execute.cpp"),
            os.path.join(HERE, "dropin_harness.cpp")]
    lib = os.path.join(ROOT, "calamarijoins_b200", "libcj_b200.so")
    deps = srcs + [lib, os.path.join(ROOT, "include", "cj_b200.h")]
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(p) for p in deps):
        return OUT
    cmd = ["g++", "-std=c++17", "-O2", "-w", "-fpermissive", "-DFMT_HEADER_ONLY",
           "-I", os.path.join(ROOT, "oracle", "ref_shim"), "-I", os.path.join(ref, "include"),
           "-I", fmt_inc, "-I", os.path.join(ROOT, "include"), *srcs, lib,
           "-Wl,-rpath,$ORIGIN/../../calamarijoins_b200", "-o", OUT]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("drop-in build failed:\n" + res.stderr[-4000:])
    return OUT


if __name__ == "__main__":
    print(build("--force" in sys.argv))
