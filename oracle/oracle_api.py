"""ctypes access to the oracle (libcj_oracle.so) and to the reference's own
execute() (oracle/_ref/libcj_ref_t<N>.so). TEST INFRASTRUCTURE ONLY: used by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, as the
checker and the CPU baseline, never as the product path.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import re
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libcj_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
PAGE = 8192

_P = C.c_void_p
_oracle = None
_refs: dict = {}


def _pd_type():
    from calamarijoins_b200._lib import PlanDesc, TimingStatsC
    return PlanDesc, TimingStatsC


def oracle_lib() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            from . import build_oracle
            build_oracle.build_oracle()
        PlanDesc, _ = _pd_type()
        h = C.CDLL(ORACLE_SO)
        sigs = {
            "cjo_execute": (C.c_int, [C.POINTER(PlanDesc), C.POINTER(_P)]),
            "cjo_result_num_rows": (C.c_uint64, [_P]),
            "cjo_result_num_columns": (C.c_uint64, [_P]),
            "cjo_result_column": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_int32), C.POINTER(C.c_uint64),
                                            C.POINTER(_P)]),
            "cjo_result_free": (None, [_P]),
            "cjo_validate_column": (C.c_int, [C.c_int32, _P, C.c_uint64, C.c_uint64, C.c_char_p, C.c_uint64]),
            "cjo_encode_column": (C.c_int, [C.c_int32, _P, _P, _P, C.c_uint64, _P, C.c_uint64,
                                            C.POINTER(C.c_uint64)]),
            "cjo_paged_tables_equal": (C.c_int, [C.c_uint64, _P, C.c_uint64, _P, _P, C.c_uint64, _P, _P,
                                                 C.c_char_p, C.c_uint64]),
            "cjo_paged_table_fingerprint": (C.c_int, [C.c_uint64, _P, C.c_uint64, _P, _P,
                                                      C.POINTER(C.c_uint64)]),
            "cjo_filter": (C.c_int, [_P, _P, C.c_uint64, _P, C.POINTER(_P), _P]),
            "cjo_like": (C.c_int, [C.c_char_p, C.c_uint64, C.c_char_p, C.c_uint64]),
        }
        for n, (r, a) in sigs.items():
            f = getattr(h, n)
            f.restype, f.argtypes = r, a
        _oracle = h
    return _oracle


def ref_available() -> list[int]:
    """Thread counts of the reference builds present in oracle/_ref."""
    out = []
    for p in glob.glob(os.path.join(REF_DIR, "libcj_ref_t*.so")):
        m = re.search(r"_t(\d+)\.so$", p)
        if m:
            out.append(int(m.group(1)))
    return sorted(out)


def ref_lib(threads: int) -> C.CDLL:
    if threads not in _refs:
        path = os.path.join(REF_DIR, f"libcj_ref_t{threads}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        PlanDesc, TimingStatsC = _pd_type()
        h = C.CDLL(path)
        sigs = {
            "cjref_execute": (C.c_int, [C.POINTER(PlanDesc), C.POINTER(_P), C.POINTER(TimingStatsC),
                                        C.POINTER(C.c_double)]),
            "cjref_result_num_rows": (C.c_uint64, [_P]),
            "cjref_result_num_columns": (C.c_uint64, [_P]),
            "cjref_result_column": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_int32), C.POINTER(C.c_uint64),
                                              C.POINTER(_P)]),
            "cjref_result_free": (None, [_P]),
            "cjref_thread_count": (C.c_int, []),
        }
        for n, (r, a) in sigs.items():
            f = getattr(h, n)
            f.restype, f.argtypes = r, a
        _refs[threads] = h
    return _refs[threads]


class PagedResult:
    """A decoded-free copy of a paged result: types, row count, pages."""

    def __init__(self, num_rows: int, types: list, pages: list):
        self.num_rows = int(num_rows)
        self.types = list(types)
        self.pages = pages  # list of (n, 8192) uint8 arrays

    @staticmethod
    def from_result(res) -> "PagedResult":
        """From a calamarijoins_b200.Result."""
        types, pages = [], []
        for c in range(res.num_columns):
            t, _, _ = res.column_info(c)
            types.append(int(t))
            pages.append(res.copy_column(c))
        return PagedResult(res.num_rows, types, pages)

    @staticmethod
    def from_columnar(ct) -> "PagedResult":
        return PagedResult(ct.num_rows, [int(c.type) for c in ct.columns], [c.pages for c in ct.columns])


def _copy_paged(get_rows, get_ncols, get_col, h) -> PagedResult:
    n = get_rows(h)
    nc = get_ncols(h)
    types, pages = [], []
    for c in range(nc):
        t, np_, p = C.c_int32(), C.c_uint64(), C.c_void_p()
        get_col(h, c, C.byref(t), C.byref(np_), C.byref(p))
        types.append(t.value)
        if np_.value:
            buf = (C.c_uint8 * (np_.value * PAGE)).from_address(p.value)
            pages.append(np.frombuffer(buf, dtype=np.uint8).reshape(np_.value, PAGE).copy())
        else:
            pages.append(np.zeros((0, PAGE), np.uint8))
    return PagedResult(n, types, pages)


def oracle_execute(desc) -> PagedResult:
    """Runs the oracle on a calamarijoins_b200.PlanDescriptor."""
    L = oracle_lib()
    h = C.c_void_p()
    rc = L.cjo_execute(C.byref(desc.desc), C.byref(h))
    if rc != 0:
        raise RuntimeError(f"oracle failed with status {rc}")
    try:
        return _copy_paged(L.cjo_result_num_rows, L.cjo_result_num_columns, L.cjo_result_column, h.value)
    finally:
        L.cjo_result_free(h.value)


def ref_execute(desc, threads: Optional[int] = None):
    """Runs the reference's execute(); returns (PagedResult, wall ms, TimingStats)."""
    avail = ref_available()
    if not avail:
        raise FileNotFoundError("reference not built (oracle/build_oracle.py)")
    t = threads if threads in avail else avail[0]
    L = ref_lib(t)
    _, TimingStatsC = _pd_type()
    h, ts, ms = C.c_void_p(), TimingStatsC(), C.c_double()
    rc = L.cjref_execute(C.byref(desc.desc), C.byref(h), C.byref(ts), C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference failed with status {rc}")
    try:
        return (_copy_paged(L.cjref_result_num_rows, L.cjref_result_num_columns, L.cjref_result_column, h.value),
                ms.value, ts)
    finally:
        L.cjref_result_free(h.value)


def _ptr_array(arrays):
    arr = (C.c_void_p * max(len(arrays), 1))()
    for i, a in enumerate(arrays):
        arr[i] = a.ctypes.data if a.shape[0] else 0
    return arr


def tables_equal(a: PagedResult, b: PagedResult) -> tuple[bool, str]:
    """Row-multiset equality (values, NULLs, VARCHAR bytes, FP64 bitwise)."""
    if a.types != b.types:
        return False, f"types {a.types} vs {b.types}"
    L = oracle_lib()
    n = len(a.types)
    types = np.array(a.types, dtype=np.int32)
    npa = np.array([p.shape[0] for p in a.pages], dtype=np.uint64)
    npb = np.array([p.shape[0] for p in b.pages], dtype=np.uint64)
    pa, pb = _ptr_array(a.pages), _ptr_array(b.pages)
    msg = C.create_string_buffer(512)
    eq = L.cjo_paged_tables_equal(n, types.ctypes.data, a.num_rows, npa.ctypes.data, pa, b.num_rows,
                                  npb.ctypes.data, pb, msg, 512)
    return bool(eq), msg.value.decode()


def validate(r: PagedResult) -> tuple[bool, str]:
    """Structural validity of every column's pages."""
    L = oracle_lib()
    for c, (t, p) in enumerate(zip(r.types, r.pages)):
        msg = C.create_string_buffer(256)
        rc = L.cjo_validate_column(t, p.ctypes.data if p.shape[0] else None, p.shape[0], r.num_rows, msg, 256)
        if rc != 0:
            return False, f"column {c}: {msg.value.decode()}"
    return True, ""


def fingerprint(r: PagedResult) -> int:
    """Order-insensitive fingerprint of the row multiset."""
    L = oracle_lib()
    n = len(r.types)
    types = np.array(r.types, dtype=np.int32)
    nps = np.array([p.shape[0] for p in r.pages], dtype=np.uint64)
    ptrs = _ptr_array(r.pages)
    out = C.c_uint64()
    rc = L.cjo_paged_table_fingerprint(n, types.ctypes.data, r.num_rows, nps.ctypes.data, ptrs, C.byref(out))
    if rc != 0:
        raise RuntimeError(f"fingerprint failed with status {rc}")
    return out.value


def encode(dtype: int, values, valid=None, offsets=None) -> np.ndarray:
    """The oracle's ColumnInserter restatement (to cross-check the product's
    encoder). Fixed-width: values ndarray; VARCHAR: chars uint8 + offsets."""
    L = oracle_lib()
    vals = np.ascontiguousarray(values)
    v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint8)
    o = None if offsets is None else np.ascontiguousarray(offsets, dtype=np.uint64)
    n = (len(o) - 1) if o is not None else len(vals)
    cnt = C.c_uint64()
    vp = vals.ctypes.data if vals.size else None
    rc = L.cjo_encode_column(dtype, vp, o.ctypes.data if o is not None else None,
                             v.ctypes.data if v is not None else None, n, None, 0, C.byref(cnt))
    if rc:
        raise RuntimeError(f"encode failed {rc}")
    out = np.zeros((cnt.value, PAGE), np.uint8)
    if cnt.value:
        rc = L.cjo_encode_column(dtype, vp, o.ctypes.data if o is not None else None,
                                 v.ctypes.data if v is not None else None, n, out.ctypes.data, cnt.value,
                                 C.byref(cnt))
        if rc:
            raise RuntimeError(f"encode failed {rc}")
    return out


def _table_desc(table):
    """A cj_table_desc over a ColumnarTable's host pages (kept alive by the
    returned tuple)."""
    from calamarijoins_b200._lib import ColumnDesc, TableDesc
    keep = []
    cols = (ColumnDesc * max(len(table.columns), 1))()
    for c, col in enumerate(table.columns):
        ptrs = col.page_pointers()
        keep.append(ptrs)
        cols[c].type = int(col.type)
        cols[c].num_pages = col.num_pages
        cols[c].pages = C.cast(ptrs, C.POINTER(C.c_void_p))
    return TableDesc(table.num_rows, len(table.columns), cols), keep, cols


def oracle_filter(table, predicate, columns=None):
    """The oracle's scan filter (cjo_filter): (PagedResult of the selected
    rows projected to `columns`, selected flags as a bool array)."""
    from calamarijoins_b200.predicate import PredicateDesc
    L = oracle_lib()
    td, keep, cols_arr = _table_desc(table)
    cols = list(range(len(table.columns))) if columns is None else list(columns)
    ca = (C.c_uint64 * max(len(cols), 1))(*cols)
    pd = PredicateDesc(predicate) if predicate is not None else None
    sel = np.zeros(max(table.num_rows, 1), np.uint8)
    h = C.c_void_p()
    rc = L.cjo_filter(C.byref(td), C.byref(pd.desc) if pd else None, len(cols), ca, C.byref(h), sel.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle filter failed with status {rc}")
    try:
        res = _copy_paged(L.cjo_result_num_rows, L.cjo_result_num_columns, L.cjo_result_column, h.value)
    finally:
        L.cjo_result_free(h.value)
    return res, sel[:table.num_rows].astype(bool)


def oracle_like(s: bytes, pattern: bytes) -> bool:
    return oracle_lib().cjo_like(s, len(s), pattern, len(pattern)) == 1


REF_FILTER_SO = os.path.join(REF_DIR, "libcj_ref_filter.so")
_ref_filter = None


def ref_filter_available() -> bool:
    return os.path.exists(REF_FILTER_SO)


def ref_filter(table, predicate):
    """The reference's own column-wise Statement::eval (src/statement.cpp,
    compiled into oracle/_ref/libcj_ref_filter.so) on the table's rows:
    the selected flags as a bool array."""
    global _ref_filter
    from calamarijoins_b200 import DataType, decode_column
    from calamarijoins_b200._lib import PredicateC
    from calamarijoins_b200.predicate import PredicateDesc
    if _ref_filter is None:
        _ref_filter = C.CDLL(REF_FILTER_SO)
        _ref_filter.cjref_filter.restype = C.c_int
        _ref_filter.cjref_filter.argtypes = [C.c_uint64, _P, C.c_uint64, _P, _P, _P, C.POINTER(PredicateC), _P]
    n = table.num_rows
    keep = []
    nc = len(table.columns)
    types = np.array([int(c.type) for c in table.columns], np.int32)
    valid_p, values_p, offs_p = (C.c_void_p * max(nc, 1))(), (C.c_void_p * max(nc, 1))(), (C.c_void_p * max(nc, 1))()
    for c, col in enumerate(table.columns):
        vals, valid = decode_column(col)
        if col.type == DataType.VARCHAR:
            valid = np.array([v is not None for v in vals], np.uint8)
            parts = [v or b"" for v in vals]
            offs = np.zeros(n + 1, np.uint64)
            offs[1:] = np.cumsum([len(x) for x in parts])
            chars = np.frombuffer(b"".join(parts) or b"\0", np.uint8).copy()
            keep += [offs, chars]
            values_p[c], offs_p[c] = chars.ctypes.data, offs.ctypes.data
        else:
            vals = np.ascontiguousarray(vals)
            keep.append(vals)
            values_p[c] = vals.ctypes.data
        valid = np.ascontiguousarray(valid, np.uint8)
        keep.append(valid)
        valid_p[c] = valid.ctypes.data
    pd = PredicateDesc(predicate)
    sel = np.zeros(max(n, 1), np.uint8)
    rc = _ref_filter.cjref_filter(nc, types.ctypes.data, n, valid_p, values_p, offs_p, C.byref(pd.desc),
                                  sel.ctypes.data)
    if rc != 0:
        raise RuntimeError("reference filter failed")
    return sel[:n].astype(bool)
