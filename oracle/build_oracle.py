"""Build recipe for the oracle (test infrastructure).

Produces
  oracle/libcj_oracle.so            the C restatement (oracle/cj_oracle.c)
  oracle/_ref/libcj_ref_t<N>.so     the reference's own execute()
                                    (CalamariJoins src/execute.cpp), compiled
                                    from its sources with N worker threads,
                                    plus oracle/ref_bridge.cpp

The reference is compiled only when its source tree is present (environment
variable CJ_REFERENCE_DIR, default /root/reference). Its CMake build cannot
run offline (FetchContent of Catch2, abseil, re2, fmt, range-v3, DuckDB), so
this recipe compiles the one translation unit on the join path directly:
fmt comes header-only from PyTorch's include tree, and oracle/ref_shim/
stands in for re2 (unused on the join path), the range-v3 table loader
(unused) and the hard-coded hardware constants. The build targets
x86-64-v3 (AVX2 + SSE4.2 CRC32) instead of -march=native so that the library
also runs on the GPU host, whose CPU model may differ from the build host.
Each thread-count variant is self-contained (-fno-gnu-unique,
-Wl,-Bsymbolic); still, callers load one variant per process.

Usage: python oracle/build_oracle.py [--threads 32,64,...]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_THREADS = (8, 16, 32, 64, 128, 192, 256)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + res.stderr[-4000:])


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "cj_oracle.c")
    hdrs = [os.path.join(HERE, "cj_oracle.h"), os.path.join(HERE, "..", "include", "cj_b200.h")]
    out = os.path.join(HERE, "libcj_oracle.so")
    if force or not _newer(out, [src] + hdrs):
        _run(["gcc", "-O2", "-g", "-std=gnu11", "-shared", "-fPIC", "-Wall", "-Wno-unused-function",
              src, "-o", out])
    return out


def reference_dir() -> str | None:
    ref = os.environ.get("CJ_REFERENCE_DIR", "/root/reference")
    if os.path.isfile(os.path.join(ref, "src", "execute.cpp")):
        return ref
    return None


def build_reference(threads=DEFAULT_THREADS, force: bool = False) -> list[str]:
    ref = reference_dir()
    if ref is None:
        return []
    try:
        import torch  # only for the bundled header-only fmt
        fmt_inc = os.path.join(os.path.dirname(torch.__file__), "include")
    except Exception:  # pragma: no cover
        return []
    outdir = os.path.join(HERE, "_ref")
    os.makedirs(outdir, exist_ok=True)
    sources = [os.path.join(ref, "src", "execute.cpp"), os.path.join(HERE, "ref_bridge.cpp")]
    shim = os.path.join(HERE, "ref_shim")
    deps = sources + [os.path.join(shim, "platform", "hardware.h")]
    built = []
    for t in threads:
        out = os.path.join(outdir, f"libcj_ref_t{t}.so")
        if force or not _newer(out, deps):
            # -fno-gnu-unique -Wl,-Bsymbolic: each variant keeps its own
            # singletons (the worker pool is a function-local static, which
            # GCC would otherwise merge across every loaded variant)
            _run(["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-fpermissive", "-w", "-fno-gnu-unique",
                  "-Wl,-Bsymbolic",
                  "-DFMT_HEADER_ONLY", f"-DSPC__THREAD_COUNT={t}",
                  "-I", shim, "-I", os.path.join(ref, "include"), "-I", fmt_inc,
                  "-shared", "-fPIC", *sources, "-o", out, "-lpthread"])
        built.append(out)
    return built


def build_reference_filter(force: bool = False) -> str | None:
    """oracle/_ref/libcj_ref_filter.so: the reference's scan-filter
    evaluation (src/statement.cpp with include/data_model/inner_column.h)
    behind oracle/ref_filter_bridge.cpp; RE2 is the shim's subset matcher."""
    ref = reference_dir()
    if ref is None:
        return None
    try:
        import torch  # only for the bundled header-only fmt
        fmt_inc = os.path.join(os.path.dirname(torch.__file__), "include")
    except Exception:  # pragma: no cover
        return None
    outdir = os.path.join(HERE, "_ref")
    os.makedirs(outdir, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim")
    sources = [os.path.join(ref, "src", "statement.cpp"), os.path.join(HERE, "ref_filter_bridge.cpp")]
    out = os.path.join(outdir, "libcj_ref_filter.so")
    if force or not _newer(out, sources + [os.path.join(shim, "re2", "re2.h")]):
        _run(["g++", "-std=c++17", "-O2", "-fpermissive", "-w", "-fno-gnu-unique", "-Wl,-Bsymbolic",
              "-DFMT_HEADER_ONLY", "-I", shim, "-I", os.path.join(ref, "include"), "-I", fmt_inc,
              "-shared", "-fPIC", *sources, "-o", out, "-lpthread"])
    return out


def build_reference_cache(force: bool = False) -> str | None:
    """oracle/_ref/libcj_ref_cache.so: the reference's `.tbl` cache reader
    (Table::from_cache, src/build_table.cpp) and writer (DumpTable,
    include/data_access/table.h) behind oracle/ref_cache_bridge.cpp. The
    reference's table.h needs range-v3, absent here: compiled as C++23 with
    oracle/ref_shim_tbl's stand-in over std::ranges, and with the reference's
    own headers ahead of oracle/ref_shim (only its re2 stand-in is used)."""
    ref = reference_dir()
    if ref is None:
        return None
    try:
        import torch  # only for the bundled header-only fmt
        fmt_inc = os.path.join(os.path.dirname(torch.__file__), "include")
    except Exception:  # pragma: no cover
        return None
    outdir = os.path.join(HERE, "_ref")
    os.makedirs(outdir, exist_ok=True)
    sources = [os.path.join(ref, "src", f) for f in ("build_table.cpp", "csv_parser.cpp", "statement.cpp")]
    sources.append(os.path.join(HERE, "ref_cache_bridge.cpp"))
    out = os.path.join(outdir, "libcj_ref_cache.so")
    deps = sources + [os.path.join(HERE, "ref_shim_tbl", "range", "v3", "all.hpp")]
    if force or not _newer(out, deps):
        _run(["g++", "-std=c++23", "-O2", "-fpermissive", "-w", "-fno-gnu-unique", "-Wl,-Bsymbolic",
              "-DFMT_HEADER_ONLY", "-I", os.path.join(HERE, "ref_shim_tbl"), "-I", os.path.join(ref, "include"),
              "-I", os.path.join(HERE, "ref_shim"), "-I", fmt_inc,
              "-shared", "-fPIC", *sources, "-o", out, "-lpthread"])
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", default=",".join(str(t) for t in DEFAULT_THREADS))
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print(build_oracle(a.force))
    for p in build_reference(tuple(int(x) for x in a.threads.split(",")), a.force):
        print(p)
    print(build_reference_filter(a.force))
    print(build_reference_cache(a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
