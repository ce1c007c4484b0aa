"""Plan and paged-table types mirroring the reference's C++ API.

  DataType                 include/foundation/attribute.h:7-12
  Page / Column / ColumnarTable
                           include/data_model/plan.h:75-147
  Plan.new_scan_node / new_join_node / new_input
                           include/data_model/plan.h:149-185
  Table.to_columnar / from_columnar
                           src/build_table.cpp:520-659, 679-924 (the row <-> page
                           conversions the reference's tests use)

A column's pages are held as one C-contiguous uint8 array of shape
(num_pages, 8192), optionally in page-locked memory (`pinned=True`) so that
uploads run at full PCIe speed.
"""
from __future__ import annotations

import ctypes as C
from enum import IntEnum
from typing import Iterable, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import PAGE_SIZE, check, lib


class DataType(IntEnum):
    INT32 = 0
    INT64 = 1
    FP64 = 2
    VARCHAR = 3


_NP = {DataType.INT32: np.int32, DataType.INT64: np.int64, DataType.FP64: np.float64}


class PinnedBuffer:
    """Page-locked host memory from cj_host_alloc, exposed as a uint8 array."""

    def __init__(self, nbytes: int):
        p = C.c_void_p()
        check(lib().cj_host_alloc(max(int(nbytes), 1), C.byref(p)))
        self.ptr = p.value
        self.nbytes = int(nbytes)
        buf = (C.c_uint8 * max(self.nbytes, 1)).from_address(self.ptr)
        self.array = np.frombuffer(buf, dtype=np.uint8, count=self.nbytes)

    def __del__(self):
        if getattr(self, "ptr", None):
            try:
                lib().cj_host_free(self.ptr)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self.ptr = None


def page_array(num_pages: int, pinned: bool = False):
    """A zeroed (num_pages, 8192) uint8 array (and its owner when pinned)."""
    if pinned and num_pages:
        owner = PinnedBuffer(num_pages * PAGE_SIZE)
        arr = owner.array.reshape(num_pages, PAGE_SIZE)
        arr[:] = 0
        return arr, owner
    return np.zeros((num_pages, PAGE_SIZE), dtype=np.uint8), None


class Column:
    """Column (plan.h:82-142): a type and its 8 KiB pages."""

    def __init__(self, dtype: DataType, pages: Optional[np.ndarray] = None, owner=None):
        self.type = DataType(dtype)
        if pages is None:
            pages = np.zeros((0, PAGE_SIZE), dtype=np.uint8)
        pages = np.asarray(pages, dtype=np.uint8)
        if pages.ndim != 2 or pages.shape[1] != PAGE_SIZE or not pages.flags.c_contiguous:
            raise ValueError("pages must be a C-contiguous (n, 8192) uint8 array")
        self.pages = pages
        self._owner = owner

    @property
    def num_pages(self) -> int:
        return int(self.pages.shape[0])

    def page_pointers(self):
        n = self.num_pages
        arr = (C.c_void_p * max(n, 1))()
        if n:
            base = self.pages.ctypes.data
            for i in range(n):
                arr[i] = base + i * PAGE_SIZE
        return arr


class ColumnarTable:
    """ColumnarTable (plan.h:144-147)."""

    def __init__(self, num_rows: int = 0, columns: Optional[list] = None):
        self.num_rows = int(num_rows)
        self.columns: list[Column] = list(columns or [])


class ScanNode:
    def __init__(self, base_table_id: int):
        self.base_table_id = int(base_table_id)


class JoinNode:
    def __init__(self, build_left: bool, left: int, right: int, left_attr: int, right_attr: int):
        self.build_left = bool(build_left)
        self.left = int(left)
        self.right = int(right)
        self.left_attr = int(left_attr)
        self.right_attr = int(right_attr)


class PlanNode:
    def __init__(self, data, output_attrs: Sequence[tuple]):
        self.data = data
        self.output_attrs = [(int(i), DataType(t)) for i, t in output_attrs]


class Plan:
    """Plan (plan.h:149-185): nodes, inputs and the root index."""

    def __init__(self):
        self.nodes: list[PlanNode] = []
        self.inputs: list = []  # ColumnarTable or ResidentTable
        self.root = 0

    def new_join_node(self, build_left, left, right, left_attr, right_attr, output_attrs) -> int:
        self.nodes.append(PlanNode(JoinNode(build_left, left, right, left_attr, right_attr), output_attrs))
        return len(self.nodes) - 1

    def new_scan_node(self, base_table_id, output_attrs) -> int:
        self.nodes.append(PlanNode(ScanNode(base_table_id), output_attrs))
        return len(self.nodes) - 1

    def new_input(self, table) -> int:
        self.inputs.append(table)
        return len(self.inputs) - 1


class PlanDescriptor:
    """The POD cj_plan_desc for a Plan; keeps every referenced buffer alive."""

    def __init__(self, plan: Plan):
        from .engine import ResidentTable  # local import: engine imports plan

        self.plan = plan  # the pages the descriptor points at live in the plan
        self._keep = []
        n = len(plan.nodes)
        nodes = (_lib.PlanNodeDesc * max(n, 1))()
        for i, node in enumerate(plan.nodes):
            attrs = (_lib.Attr * max(len(node.output_attrs), 1))()
            for k, (idx, t) in enumerate(node.output_attrs):
                attrs[k].index = idx
                attrs[k].type = int(t)
            self._keep.append(attrs)
            d = nodes[i]
            d.num_output_attrs = len(node.output_attrs)
            d.output_attrs = attrs
            if isinstance(node.data, ScanNode):
                d.node_type = _lib.CJ_NODE_SCAN
                d.base_table_id = node.data.base_table_id
            else:
                j = node.data
                d.node_type = _lib.CJ_NODE_HASH_JOIN
                d.build_left = 1 if j.build_left else 0
                d.left, d.right = j.left, j.right
                d.left_attr, d.right_attr = j.left_attr, j.right_attr
        nt = len(plan.inputs)
        tables = (_lib.TableDesc * max(nt, 1))()
        resident = (C.c_void_p * max(nt, 1))()
        any_resident = False
        for t, tab in enumerate(plan.inputs):
            if isinstance(tab, ResidentTable):
                resident[t] = tab.handle
                tables[t].num_rows = tab.num_rows
                any_resident = True
                continue
            cols = (_lib.ColumnDesc * max(len(tab.columns), 1))()
            for c, col in enumerate(tab.columns):
                ptrs = col.page_pointers()
                self._keep.append(ptrs)
                cols[c].type = int(col.type)
                cols[c].num_pages = col.num_pages
                cols[c].pages = C.cast(ptrs, C.POINTER(C.c_void_p))
            self._keep.append(cols)
            tables[t].num_rows = tab.num_rows
            tables[t].num_columns = len(tab.columns)
            tables[t].columns = cols
        self._keep += [nodes, tables, resident]
        self.desc = _lib.PlanDesc()
        self.desc.num_nodes = n
        self.desc.nodes = nodes
        self.desc.num_inputs = nt
        self.desc.inputs = tables
        self.desc.resident_inputs = C.cast(resident, C.POINTER(C.c_void_p)) if any_resident else None
        self.desc.root = plan.root


# ---------------------------------------------------------------------------
# Page encoding (ColumnInserter<T>, plan.h:187-366) through the library's
# host encoder, and decoding back to Python values.
# ---------------------------------------------------------------------------
def _u8p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8)) if a is not None else None


def encode_column(dtype: DataType, values, valid=None, pinned: bool = False) -> Column:
    """Encodes one column into pages.

    Fixed-width types take a numpy array; VARCHAR takes a sequence of
    str/bytes (None = NULL) or a (chars uint8, offsets uint64[n+1]) pair.
    `valid` (bool/uint8 per row) marks present values; None = no NULLs.
    """
    dtype = DataType(dtype)
    offsets_p = None
    if dtype == DataType.VARCHAR:
        if isinstance(values, tuple):
            chars, offsets = values
            chars = np.ascontiguousarray(chars, dtype=np.uint8)
            offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
            n = len(offsets) - 1
        else:
            vals = list(values)
            n = len(vals)
            if valid is None and any(v is None for v in vals):
                valid = np.array([v is not None for v in vals], dtype=np.uint8)
            enc = [(v.encode() if isinstance(v, str) else (v or b"")) for v in vals]
            lens = np.array([len(e) for e in enc], dtype=np.uint64)
            offsets = np.zeros(n + 1, dtype=np.uint64)
            np.cumsum(lens, out=offsets[1:])
            chars = np.frombuffer(b"".join(enc), dtype=np.uint8) if n else np.zeros(0, np.uint8)
            chars = np.ascontiguousarray(chars)
        data = chars if len(chars) else np.zeros(1, np.uint8)
        offsets_p = offsets.ctypes.data_as(C.POINTER(C.c_uint64))
        keep = (chars, offsets)
    else:
        data = np.ascontiguousarray(values, dtype=_NP[dtype])
        n = len(data)
        keep = (data,)
        if n == 0:
            data = np.zeros(1, dtype=_NP[dtype])
    vmask = None
    if valid is not None:
        vmask = np.ascontiguousarray(valid, dtype=np.uint8)
        if len(vmask) != n:
            raise ValueError("valid has the wrong length")
    np_ = C.c_uint64()
    check(lib().cj_encode_num_pages(int(dtype), data.ctypes.data, offsets_p, _u8p(vmask), n, C.byref(np_)))
    pages, owner = page_array(np_.value, pinned)
    if np_.value:
        got = C.c_uint64()
        check(lib().cj_encode_column(int(dtype), data.ctypes.data, offsets_p, _u8p(vmask), n,
                                     pages.ctypes.data, np_.value, C.byref(got)))
    del keep
    return Column(dtype, pages, owner)


def decode_column(col: Column):
    """Decodes a column's pages (Table::from_columnar, build_table.cpp:520-659).

    Returns (values, valid): fixed-width values as a numpy array (0 where
    NULL); VARCHAR values as a list of bytes (None where NULL).
    """
    pages = col.pages
    if col.type != DataType.VARCHAR:
        w = 4 if col.type == DataType.INT32 else 8
        npd = _NP[col.type]
        vals_out, valid_out = [], []
        for p in range(pages.shape[0]):
            pg = pages[p]
            nr = int(pg[0]) | (int(pg[1]) << 8)
            nv = int(pg[2]) | (int(pg[3]) << 8)
            bm = np.unpackbits(pg[PAGE_SIZE - (nr + 7) // 8:], bitorder="little")[:nr].astype(bool)
            vals = np.zeros(nr, dtype=npd)
            vals[bm] = pg[w:w + nv * w].view(npd)[: int(bm.sum())]
            vals_out.append(vals)
            valid_out.append(bm)
        if not vals_out:
            return np.zeros(0, dtype=npd), np.zeros(0, dtype=bool)
        return np.concatenate(vals_out), np.concatenate(valid_out)
    out: list = []
    for p in range(pages.shape[0]):
        pg = pages[p]
        nr = int(pg[0]) | (int(pg[1]) << 8)
        nv = int(pg[2]) | (int(pg[3]) << 8)
        if nr == 0xFFFF:
            out.append(bytes(pg[4:4 + nv]))
        elif nr == 0xFFFE:
            out[-1] = out[-1] + bytes(pg[4:4 + nv])
        else:
            offs = pg[4:4 + 2 * nv].view(np.uint16)
            base = 4 + 2 * nv
            bm = np.unpackbits(pg[PAGE_SIZE - (nr + 7) // 8:], bitorder="little")[:nr]
            k, prev = 0, 0
            for i in range(nr):
                if bm[i]:
                    end = int(offs[k])
                    out.append(bytes(pg[base + prev: base + end]))
                    prev = end
                    k += 1
                else:
                    out.append(None)
    return out, np.array([v is not None for v in out], dtype=bool)


class Table:
    """Row-oriented table (the reference's Table, include/data_access/table.h)
    with conversions to and from the paged format. NULL is None."""

    def __init__(self, rows: Iterable[Sequence], types: Sequence[DataType]):
        self.types = [DataType(t) for t in types]
        self.rows = [list(r) for r in rows]

    def to_columnar(self, pinned: bool = False) -> ColumnarTable:
        cols = []
        for c, t in enumerate(self.types):
            vals = [r[c] for r in self.rows]
            if t == DataType.VARCHAR:
                cols.append(encode_column(t, vals, pinned=pinned))
            else:
                valid = np.array([v is not None for v in vals], dtype=np.uint8)
                arr = np.array([0 if v is None else v for v in vals], dtype=_NP[t])
                cols.append(encode_column(t, arr, valid, pinned=pinned))
        return ColumnarTable(len(self.rows), cols)

    @staticmethod
    def from_columnar(table: ColumnarTable) -> "Table":
        cols = []
        for col in table.columns:
            vals, valid = decode_column(col)
            if col.type == DataType.VARCHAR:
                cols.append([None if v is None else v.decode("utf-8", errors="surrogateescape") for v in vals])
            else:
                cols.append([v.item() if ok else None for v, ok in zip(vals, valid)])
        rows = [list(r) for r in zip(*cols)] if cols else [[] for _ in range(table.num_rows)]
        return Table(rows, [c.type for c in table.columns])

    def sorted_rows(self):
        def key(row):
            return tuple((0, 0) if v is None else (1, v) for v in row)
        return sorted(self.rows, key=key)
