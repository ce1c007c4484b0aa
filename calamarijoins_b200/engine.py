"""Execution entry points mirroring the reference's Contest namespace.

  build_context()            Contest::build_context   (plan.h:380)
  destroy_context(ctx)       Contest::destroy_context (plan.h:382)
  execute(plan, ctx, stats)  Contest::execute         (plan.h:384; src/execute.cpp:311-325)
  TimingStats                Contest::TimingStats     (plan.h:370-378)

Errors raise CJError carrying the library's status code (the reference
throws std::bad_alloc / std::runtime_error).
"""
from __future__ import annotations

import ctypes as C
import os
import sys
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from ._lib import PAGE_SIZE, check, lib
from .plan import Column, ColumnarTable, DataType, Plan, PlanDescriptor

_finalizing = sys.is_finalizing  # bound now: module globals are gone at exit


@dataclass
class TimingStats:
    hashtable_build_ms: int = 0
    hash_join_probe_ms: int = 0
    nested_loop_join_ms: int = 0
    materialize_ms: int = 0
    setup_ms: int = 0
    total_execution_ms: int = 0
    intermediate_ms: int = 0
    # finer statistics of the call (cj_exec_stats)
    exec: dict = field(default_factory=dict)


class Context:
    """A device context: CUDA device, stream, memory pool (cj_context)."""

    def __init__(self, device: int = -1):
        h = C.c_void_p()
        check(lib().cj_context_create(int(device), C.byref(h)))
        self.handle = h.value

    def close(self):
        if getattr(self, "handle", None):
            lib().cj_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        if not _finalizing():  # at exit the process releases everything
            self.close()

    def set_option(self, option: int, value: int):
        check(lib().cj_context_set_option(self.handle, int(option), int(value)))

    def get_option(self, option: int) -> int:
        v = C.c_int64()
        check(lib().cj_context_get_option(self.handle, int(option), C.byref(v)))
        return v.value

    def memory(self):
        u, r = C.c_uint64(), C.c_uint64()
        check(lib().cj_context_memory(self.handle, C.byref(u), C.byref(r)))
        return u.value, r.value

    def profile(self) -> dict:
        n = C.c_uint64()
        check(lib().cj_profile_count(self.handle, C.byref(n)))
        out = {}
        for i in range(n.value):
            name, launches, us = C.c_char_p(), C.c_uint64(), C.c_double()
            check(lib().cj_profile_entry(self.handle, i, C.byref(name), C.byref(launches), C.byref(us)))
            out[name.value.decode()] = (launches.value, us.value)
        return out

    def profile_reset(self):
        check(lib().cj_profile_reset(self.handle))

    def autotune(self, path: Optional[str] = None, quick: bool = False):
        """Times the hash build and probe per size class and keeps the
        fastest launch parameters (cj_autotune); writes them to `path`."""
        check(lib().cj_autotune(self.handle, os.fsencode(path) if path else None,
                                _lib.CJ_TUNE_QUICK if quick else 0))

    def load_tuning(self, path: str):
        check(lib().cj_tuning_load(self.handle, os.fsencode(path)))

    def tuning(self) -> list:
        """Per size class: (log2 slots per partition, radix-pass CTAs per SM,
        probe CTAs per SM); zeros mean untuned defaults."""
        out = []
        for c in range(6):
            a, b, d = C.c_int32(), C.c_int32(), C.c_int32()
            check(lib().cj_tuning_entry(self.handle, c, C.byref(a), C.byref(b), C.byref(d)))
            out.append((a.value, b.value, d.value))
        return out


class ResidentTable:
    """A table whose pages live in device memory (cj_table)."""

    def __init__(self, ctx: Context, table: ColumnarTable):
        self.ctx = ctx
        self.num_rows = table.num_rows
        self.types = [c.type for c in table.columns]
        keep = []
        cols = (_lib.ColumnDesc * max(len(table.columns), 1))()
        for c, col in enumerate(table.columns):
            ptrs = col.page_pointers()
            keep.append(ptrs)
            cols[c].type = int(col.type)
            cols[c].num_pages = col.num_pages
            cols[c].pages = C.cast(ptrs, C.POINTER(C.c_void_p))
        td = _lib.TableDesc(table.num_rows, len(table.columns), cols)
        h = C.c_void_p()
        check(lib().cj_table_upload(ctx.handle, C.byref(td), C.byref(h)))
        self.handle = h.value
        self._owned = True

    @classmethod
    def from_handle(cls, ctx: Context, handle: int, num_rows: int, types, owned: bool = True) -> "ResidentTable":
        """Wraps a cj_table made elsewhere (a cache file, a catalog entry);
        `owned` False leaves freeing it to its owner."""
        t = cls.__new__(cls)
        t.ctx, t.handle, t.num_rows, t.types, t._owned = ctx, handle, num_rows, [DataType(x) for x in types], owned
        return t

    @classmethod
    def from_cache(cls, ctx: Context, path: str) -> "ResidentTable":
        """Loads one of the reference's `.tbl` cache files into HBM
        (cj_table_load_cache; Table::from_cache, src/build_table.cpp:140-197)."""
        meta = read_cache_meta(path)
        h = C.c_void_p()
        check(lib().cj_table_load_cache(ctx.handle, os.fsencode(path), C.byref(h)))
        return cls.from_handle(ctx, h.value, meta["num_rows"], meta["types"])

    def filter(self, predicate=None, columns=None) -> "ResidentTable":
        """Rows for which `predicate` (a predicate.Statement, or None for
        all rows) holds, projected to `columns` (default: all), as a new
        resident table (cj_table_filter): the predicate is evaluated and the
        pages written on the GPU."""
        from .predicate import PredicateDesc
        cols = list(range(len(self.types))) if columns is None else [int(c) for c in columns]
        arr = (C.c_uint64 * max(len(cols), 1))(*cols)
        pd = PredicateDesc(predicate) if predicate is not None else None
        h, n = C.c_void_p(), C.c_uint64()
        check(lib().cj_table_filter(self.ctx.handle, self.handle, C.byref(pd.desc) if pd else None, len(cols), arr,
                                    C.byref(h), C.byref(n)))
        return ResidentTable.from_handle(self.ctx, h.value, n.value, [self.types[c] for c in cols])

    def download(self) -> ColumnarTable:
        """The table's pages copied back to the host."""
        cols = []
        for c, t in enumerate(self.types):
            p, np_ = C.c_void_p(), C.c_uint64()
            check(lib().cj_table_column_pages(self.handle, c, C.byref(p), C.byref(np_)))
            host = np.zeros((np_.value, PAGE_SIZE), np.uint8)
            if np_.value:
                check(lib().cj_table_copy_column(self.handle, c, host.ctypes.data, host.nbytes))
            cols.append(Column(DataType(t), host))
        return ColumnarTable(self.num_rows, cols)

    def free(self):
        if getattr(self, "handle", None):
            if getattr(self, "_owned", True):
                lib().cj_table_free(self.handle)
            self.handle = None

    def __del__(self):
        if not _finalizing():
            self.free()


def read_cache_meta(path: str) -> dict:
    """Header of a `.tbl` cache file (TableMeta, include/data_access/
    table.h:30-35), checked against the file size."""
    m = _lib.CacheMetaC()
    check(lib().cj_cache_read_meta(os.fsencode(path), C.byref(m)))
    n = m.num_columns
    return {"num_rows": m.num_rows, "types": [DataType(m.types[i]) for i in range(n)],
            "num_pages": [m.num_pages[i] for i in range(n)]}


def write_cache(table: ColumnarTable, path: str) -> None:
    """Writes host pages as a `.tbl` cache file (DumpTable::dump,
    include/data_access/table.h:210-220)."""
    keep = []
    cols = (_lib.ColumnDesc * max(len(table.columns), 1))()
    for c, col in enumerate(table.columns):
        ptrs = col.page_pointers()
        keep.append(ptrs)
        cols[c].type = int(col.type)
        cols[c].num_pages = col.num_pages
        cols[c].pages = C.cast(ptrs, C.POINTER(C.c_void_p))
    td = _lib.TableDesc(table.num_rows, len(table.columns), cols)
    check(lib().cj_table_write_cache(C.byref(td), os.fsencode(path)))


class Catalog:
    """Resident tables by name (cj_catalog). load() reads a `.tbl` cache
    file into HBM once; catalog[name] is a ResidentTable for Plan.inputs."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = C.c_void_p()
        check(lib().cj_catalog_create(ctx.handle, C.byref(h)))
        self.handle = h.value
        self._meta = {}

    def load(self, name: str, path: str) -> None:
        meta = read_cache_meta(path)
        check(lib().cj_catalog_load(self.handle, name.encode(), os.fsencode(path)))
        self._meta[name] = meta

    def load_dir(self, directory: str) -> list:
        """Every `<name>.tbl` file of a directory, under its name."""
        names = []
        for f in sorted(os.listdir(directory)):
            if f.endswith(".tbl"):
                self.load(f[:-4], os.path.join(directory, f))
                names.append(f[:-4])
        return names

    def names(self) -> list:
        n = C.c_uint64()
        check(lib().cj_catalog_size(self.handle, C.byref(n)))
        out = []
        for i in range(n.value):
            p = C.c_char_p()
            check(lib().cj_catalog_name(self.handle, i, C.byref(p)))
            out.append(p.value.decode())
        return out

    def __getitem__(self, name: str) -> ResidentTable:
        h = C.c_void_p()
        check(lib().cj_catalog_get(self.handle, name.encode(), C.byref(h)))
        m = self._meta[name]
        return ResidentTable.from_handle(self.ctx, h.value, m["num_rows"], m["types"], owned=False)

    def close(self):
        if getattr(self, "handle", None):
            lib().cj_catalog_destroy(self.handle)
            self.handle = None

    def __del__(self):
        if not _finalizing():  # at exit the process releases everything
            self.close()


class Result:
    """A cj_result: the root output, pages on the host (pinned) or device."""

    def __init__(self, handle: int):
        self.handle = handle
        n = C.c_uint64()
        check(lib().cj_result_num_rows(handle, C.byref(n)))
        self.num_rows = n.value
        check(lib().cj_result_num_columns(handle, C.byref(n)))
        self.num_columns = n.value

    def column_info(self, c: int):
        t, np_, hp = C.c_int32(), C.c_uint64(), C.c_void_p()
        check(lib().cj_result_column(self.handle, c, C.byref(t), C.byref(np_), C.byref(hp)))
        return DataType(t.value), np_.value, hp.value

    def host_pages(self, c: int) -> np.ndarray:
        """Zero-copy view of column c's pinned host pages (valid until free)."""
        _, n, ptr = self.column_info(c)
        if not n:
            return np.zeros((0, PAGE_SIZE), dtype=np.uint8)
        if not ptr:
            raise ValueError("result kept on the device; use copy_column")
        buf = (C.c_uint8 * (n * PAGE_SIZE)).from_address(ptr)
        return np.frombuffer(buf, dtype=np.uint8).reshape(n, PAGE_SIZE)

    def copy_column(self, c: int) -> np.ndarray:
        _, n, _ = self.column_info(c)
        out = np.zeros((n, PAGE_SIZE), dtype=np.uint8)
        if n:
            check(lib().cj_result_copy_column(self.handle, c, out.ctypes.data, out.nbytes))
        return out

    def to_columnar(self) -> ColumnarTable:
        cols = []
        for c in range(self.num_columns):
            t, _, _ = self.column_info(c)
            cols.append(Column(t, self.copy_column(c)))
        return ColumnarTable(self.num_rows, cols)

    def free(self):
        if getattr(self, "handle", None):
            lib().cj_result_free(self.handle)
            self.handle = None

    def __del__(self):
        if not _finalizing():
            self.free()


def build_context(device: int = -1) -> Context:
    return Context(device)


def destroy_context(ctx: Context) -> None:
    ctx.close()


def execute_raw(plan: Plan, ctx: Context, flags: int = 0, desc: Optional[PlanDescriptor] = None):
    """Runs a plan; returns (Result, TimingStats)."""
    d = desc or PlanDescriptor(plan)
    h = C.c_void_p()
    ts, es = _lib.TimingStatsC(), _lib.ExecStatsC()
    check(lib().cj_execute(ctx.handle, C.byref(d.desc), int(flags), C.byref(h), C.byref(ts), C.byref(es)))
    stats = TimingStats(**{n: getattr(ts, n) for n, _ in _lib.TimingStatsC._fields_})
    stats.exec = {n: getattr(es, n) for n, _ in _lib.ExecStatsC._fields_}
    return Result(h.value), stats


def execute(plan: Plan, ctx: Context, stats_out: Optional[TimingStats] = None) -> ColumnarTable:
    """Contest::execute: runs the plan, returns the root's ColumnarTable."""
    res, st = execute_raw(plan, ctx)
    try:
        out = res.to_columnar()
    finally:
        res.free()
    if stats_out is not None:
        stats_out.__dict__.update(st.__dict__)
    return out


def execute_batch(plans, ctx: Context, flags: int = 0, descs=None):
    """Runs many plans together (cj_execute_batch). Returns (results,
    statuses, stats): results[i] is a Result or None when plans[i] failed
    validation (its status code in statuses[i])."""
    descs = descs or [p if isinstance(p, PlanDescriptor) else PlanDescriptor(p) for p in plans]
    n = len(descs)
    arr = (_lib.PlanDesc * max(n, 1))()
    for i, d in enumerate(descs):
        arr[i] = d.desc
    outs = (C.c_void_p * max(n, 1))()
    sts = (C.c_int32 * max(n, 1))()
    bs = _lib.BatchStatsC()
    check(lib().cj_execute_batch(ctx.handle, arr, n, int(flags), outs, sts, C.byref(bs)))
    results = [Result(outs[i]) if outs[i] else None for i in range(n)]
    return results, [sts[i] for i in range(n)], {k: getattr(bs, k) for k, _ in _lib.BatchStatsC._fields_}


class PreparedBatch:
    """A batch of plans over device-resident tables captured as one CUDA
    graph (cj_batch_prepare); run() replays it (cj_batch_run). The pages of
    a run's results are overwritten by the next run."""

    def __init__(self, plans, ctx: Context, flags: int = 0, descs=None):
        self.descs = descs or [p if isinstance(p, PlanDescriptor) else PlanDescriptor(p) for p in plans]
        self.n = len(self.descs)
        self._arr = (_lib.PlanDesc * max(self.n, 1))()
        for i, d in enumerate(self.descs):
            self._arr[i] = d.desc
        h = C.c_void_p()
        check(lib().cj_batch_prepare(ctx.handle, self._arr, self.n, int(flags), C.byref(h)))
        self.handle = h.value
        self.ctx = ctx

    def run(self):
        outs = (C.c_void_p * max(self.n, 1))()
        bs = _lib.BatchStatsC()
        check(lib().cj_batch_run(self.handle, outs, C.byref(bs)))
        return [Result(outs[i]) for i in range(self.n)], {k: getattr(bs, k) for k, _ in _lib.BatchStatsC._fields_}

    def close(self):
        if getattr(self, "handle", None):
            lib().cj_prepared_free(self.handle)
            self.handle = None

    def __del__(self):
        if not _finalizing():
            self.close()


class Server:
    """Serving front end (cj_server): plans submitted as they arrive run
    concurrently in `slots` worker streams under a device-memory budget; a
    worker that frees up takes up to `max_batch` queued plans that fit and
    runs them as one grouped execution (continuous batching). Host results
    are carved from `host_cache_bytes` of page-locked memory reserved at
    creation, when given; `device_reserve_bytes` pre-grows the server's
    device memory pool."""

    def __init__(self, device: int = -1, slots: int = 4, memory_budget: int = 0, flags: int = 0,
                 max_batch: int = 0, age_limit_us: int = 0, host_cache_bytes: int = 0,
                 device_reserve_bytes: int = 0):
        cfg = _lib.ServerConfigC(int(device), int(slots), int(memory_budget), int(flags), int(max_batch),
                                 int(age_limit_us), int(host_cache_bytes), int(device_reserve_bytes))
        h = C.c_void_p()
        check(lib().cj_server_create(C.byref(cfg), C.byref(h)))
        self.handle = h.value
        self._pending = {}

    def submit(self, plan) -> int:
        desc = plan if isinstance(plan, PlanDescriptor) else PlanDescriptor(plan)
        t = C.c_uint64()
        check(lib().cj_server_submit(self.handle, C.byref(desc.desc), C.byref(t)))
        self._pending[t.value] = desc  # pages must stay alive until wait()
        return t.value

    def wait(self, ticket: int, timeout_us: int = -1):
        h = C.c_void_p()
        es = _lib.ExecStatsC()
        rc = lib().cj_server_wait(self.handle, int(ticket), int(timeout_us), C.byref(h), C.byref(es))
        if rc != 10:  # CJ_ERR_TIMEOUT keeps the ticket pending
            self._pending.pop(ticket, None)
        check(rc)
        return Result(h.value), {n: getattr(es, n) for n, _ in _lib.ExecStatsC._fields_}

    def cancel(self, ticket: int):
        check(lib().cj_server_cancel(self.handle, int(ticket)))

    def stats(self, reset: bool = False) -> dict:
        st = _lib.ServerStatsC()
        check(lib().cj_server_get_stats(self.handle, C.byref(st), 1 if reset else 0))
        return {n: getattr(st, n) for n, _ in _lib.ServerStatsC._fields_}

    @staticmethod
    def estimate(plan) -> int:
        desc = plan if isinstance(plan, PlanDescriptor) else PlanDescriptor(plan)
        b = C.c_uint64()
        check(lib().cj_server_estimate(C.byref(desc.desc), C.byref(b)))
        return b.value

    def close(self):
        if getattr(self, "handle", None):
            lib().cj_server_destroy(self.handle)
            self.handle = None
            self._pending.clear()

    def __del__(self):
        if not _finalizing():  # at exit the process releases everything
            self.close()
