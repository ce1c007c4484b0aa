"""Build recipe for libcj_b200.so (sm_100a CUDA kernels + C++ host engine).

Compiles every source under calamarijoins_b200/csrc with nvcc for
compute_100a / sm_100a and links them, with the static CUDA runtime, into
calamarijoins_b200/libcj_b200.so (in-tree, next to the Python package).

Usage: python -m calamarijoins_b200.build [--force] [--debug]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")
OBJDIR = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libcj_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
            + glob.glob(os.path.join(INCLUDE, "*.h")))


def _compile(src: str, debug: bool) -> str:
    obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
    opt = ["-O0", "-g"] if debug else ["-O3"]
    cmd = [NVCC, "-std=c++17", *opt, *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-Wall",
           "-I", INCLUDE, "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd[1:1] = ["-x", "cu"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr[-6000:]}")
    return obj


def build(force: bool = False, debug: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = _sources()
    newest = max(os.path.getmtime(p) for p in srcs + _headers() + [__file__])
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, debug), srcs))
    cmd = [NVCC, "-shared", *ARCH, "-o", LIB, *objs, "-cudart", "static", "-lrt", "-lpthread", "-ldl"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("link failed:\n" + res.stderr[-6000:])
    if verbose:
        print(LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    a = ap.parse_args(argv)
    build(a.force, a.debug, verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
