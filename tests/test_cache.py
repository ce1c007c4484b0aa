"""The reference's `.tbl` table cache: cj_table_write_cache writes the
DumpTable format and cj_cache_read_meta checks it, without a GPU; on the
GPU, a cache file loaded into a resident table (directly or through a
catalog) gives the same join results as the host pages it came from.

The format is checked two ways. Against the reference's own code: its
Table::from_cache (src/build_table.cpp:140-197) reads the files the library
writes, and the library reads the files its DumpTable::dump
(include/data_access/table.h:136-221) writes (oracle/_ref/
libcj_ref_cache.so, compiled here with a std::ranges stand-in for range-v3).
And restated from the sources: TableMeta
(include/data_access/table.h:30-35) = u64 num_rows, u64 num_cols,
16 x 4-byte DataType, 16 x u64 page counts (208 bytes) at the start of an
8 KiB header page filled with zeros (FILLER_SIZE, table.h:37, 210-214),
then every column's pages in column order (table.h:215-219), read back
page by page in that order (src/build_table.cpp:183-193)."""
import os
import struct

import numpy as np
import pytest

from calamarijoins_b200 import (CJError, Catalog, ColumnarTable, DataType, Plan, ResidentTable, encode_column,
                                read_cache_meta, write_cache)
from calamarijoins_b200.datagen import join2, varchar_values

I, L, F, V = DataType.INT32, DataType.INT64, DataType.FP64, DataType.VARCHAR
META = struct.Struct("<QQ16i16Q")


def sample_table(seed=1, n=20_000):
    rng = np.random.default_rng(seed)
    valid = (rng.random(n) > 0.1).astype(np.uint8)
    return ColumnarTable(n, [encode_column(I, rng.integers(-100, 100, n).astype(np.int32), valid),
                             encode_column(L, rng.integers(0, 1 << 50, n)),
                             encode_column(F, rng.standard_normal(n), valid),
                             encode_column(V, varchar_values(n, rng, long_frac=0.002))])


def test_meta_layout():
    assert META.size == 208


def test_write_cache_is_the_dump_format(tmp_path):
    t = sample_table()
    path = str(tmp_path / "t.tbl")
    write_cache(t, path)
    data = open(path, "rb").read()
    rows, cols, *rest = META.unpack_from(data, 0)
    types, pages = rest[:16], rest[16:]
    assert rows == t.num_rows and cols == 4
    assert list(types[:4]) == [int(c.type) for c in t.columns] and not any(types[4:])
    assert list(pages[:4]) == [c.num_pages for c in t.columns] and not any(pages[4:])
    assert data[META.size:8192] == bytes(8192 - META.size)
    body = np.concatenate([c.pages.reshape(-1) for c in t.columns])
    assert len(data) == 8192 + body.size
    assert np.array_equal(np.frombuffer(data, np.uint8, offset=8192), body)
    m = read_cache_meta(path)
    assert m["num_rows"] == t.num_rows and m["types"] == [c.type for c in t.columns]
    assert m["num_pages"] == [c.num_pages for c in t.columns]


def test_empty_table(tmp_path):
    t = ColumnarTable(0, [encode_column(I, np.zeros(0, np.int32))])
    path = str(tmp_path / "e.tbl")
    write_cache(t, path)
    assert os.path.getsize(path) == 8192 + 8192 * t.columns[0].num_pages
    assert read_cache_meta(path)["num_rows"] == 0


def _write_raw(path, rows, cols, types, pages, body_pages):
    t = list(types) + [0] * (16 - len(types))
    p = list(pages) + [0] * (16 - len(pages))
    with open(path, "wb") as f:
        f.write(META.pack(rows, cols, *t, *p))
        f.write(bytes(8192 - META.size))
        f.write(bytes(8192 * body_pages))


@pytest.mark.parametrize("case", ["truncated", "too_long", "too_many_columns", "bad_type", "short"])
def test_malformed_files_are_rejected(tmp_path, case):
    path = str(tmp_path / "bad.tbl")
    if case == "truncated":
        _write_raw(path, 10, 1, [0], [3], 2)
    elif case == "too_long":
        _write_raw(path, 10, 1, [0], [1], 2)
    elif case == "too_many_columns":
        _write_raw(path, 10, 17, [0] * 16, [0] * 16, 0)
    elif case == "bad_type":
        _write_raw(path, 10, 1, [7], [1], 1)
    else:
        open(path, "wb").write(bytes(100))
    with pytest.raises(CJError) as e:
        read_cache_meta(path)
    assert e.value.status == 3  # CJ_ERR_MALFORMED_PAGE


def test_at_most_16_columns(tmp_path):
    t = ColumnarTable(5, [encode_column(I, np.arange(5, dtype=np.int32)) for _ in range(17)])
    with pytest.raises(CJError) as e:
        write_cache(t, str(tmp_path / "wide.tbl"))
    assert e.value.status == 7  # CJ_ERR_LIMIT


@pytest.mark.gpu
def test_cache_to_resident_tables_and_catalog(gpu_ctx, tmp_path):
    from tests.helpers import assert_same, run_oracle, run_product
    plan = join2(30_000, 300_000, seed=31, probe_null=0.05, build_payload=(L, V), probe_payload=(F,))
    for i, t in enumerate(plan.inputs):
        write_cache(t, str(tmp_path / f"t{i}.tbl"))
    want = run_oracle(plan)
    # one table at a time
    res_plan = Plan()
    res_plan.nodes, res_plan.root = plan.nodes, plan.root
    res_plan.inputs = [ResidentTable.from_cache(gpu_ctx, str(tmp_path / f"t{i}.tbl")) for i in range(2)]
    r, _ = run_product(res_plan, gpu_ctx)
    assert_same(r, want, "from_cache")
    for t in res_plan.inputs:
        t.free()
    # a catalog over the directory
    cat = Catalog(gpu_ctx)
    try:
        assert cat.load_dir(str(tmp_path)) == ["t0", "t1"]
        assert cat.names() == ["t0", "t1"]
        cat_plan = Plan()
        cat_plan.nodes, cat_plan.root = plan.nodes, plan.root
        cat_plan.inputs = [cat["t0"], cat["t1"]]
        r, _ = run_product(cat_plan, gpu_ctx)
        assert_same(r, want, "catalog")
        with pytest.raises(CJError):
            cat["missing"]
        with pytest.raises(CJError):
            cat.load("t0", str(tmp_path / "t0.tbl"))  # the name is taken
    finally:
        cat.close()


# ---- against the reference's own reader and writer ----

import ctypes as C

REF_CACHE_SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                            "libcj_ref_cache.so")
need_ref_cache = pytest.mark.skipif(not os.path.exists(REF_CACHE_SO), reason="reference cache code not compiled")


def ref_cache_lib():
    h = C.CDLL(REF_CACHE_SO)
    P = C.c_void_p
    from calamarijoins_b200._lib import TableDesc
    sigs = {"cjref_cache_read": (C.c_int, [C.c_char_p, C.POINTER(P)]), "cjref_cache_num_rows": (C.c_uint64, [P]),
            "cjref_cache_num_columns": (C.c_uint64, [P]),
            "cjref_cache_column": (C.c_int, [P, C.c_uint64, C.POINTER(C.c_int32), C.POINTER(C.c_uint64),
                                             C.POINTER(P), C.c_uint64]),
            "cjref_cache_free": (None, [P]), "cjref_cache_write": (C.c_int, [C.POINTER(TableDesc), C.c_char_p])}
    for n, (r, a) in sigs.items():
        f = getattr(h, n)
        f.restype, f.argtypes = r, a
    return h


def read_with_reference(path):
    """Table::from_cache(path) -> (num_rows, [(type, pages as (n, 8192) uint8)])."""
    L = ref_cache_lib()
    h = C.c_void_p()
    assert L.cjref_cache_read(path.encode(), C.byref(h)) == 0
    try:
        out = []
        for c in range(L.cjref_cache_num_columns(h)):
            t, n = C.c_int32(), C.c_uint64()
            L.cjref_cache_column(h, c, C.byref(t), C.byref(n), None, 0)
            ptrs = (C.c_void_p * max(n.value, 1))()
            L.cjref_cache_column(h, c, C.byref(t), C.byref(n), ptrs, n.value)
            pages = np.zeros((n.value, 8192), np.uint8)
            for k in range(n.value):
                pages[k] = np.frombuffer((C.c_uint8 * 8192).from_address(ptrs[k]), np.uint8)
            out.append((t.value, pages))
        return L.cjref_cache_num_rows(h), out
    finally:
        L.cjref_cache_free(h)


@need_ref_cache
@pytest.mark.parametrize("n", [0, 1, 20_000])
def test_reference_reads_what_the_library_writes(tmp_path, n):
    t = sample_table(n=max(n, 1)) if n else ColumnarTable(0, [encode_column(I, np.zeros(0, np.int32)),
                                                               encode_column(V, [])])
    path = str(tmp_path / "lib.tbl")
    write_cache(t, path)
    rows, cols = read_with_reference(path)
    assert rows == t.num_rows
    assert [c for c, _ in cols] == [int(c.type) for c in t.columns]
    for (_, pages), col in zip(cols, t.columns):
        assert np.array_equal(pages, col.pages.reshape(-1, 8192))


@need_ref_cache
def test_library_reads_what_the_reference_writes(tmp_path):
    from oracle.oracle_api import _table_desc
    t = sample_table(seed=3, n=30_000)
    path = str(tmp_path / "ref.tbl")
    td, keep, cols = _table_desc(t)
    assert ref_cache_lib().cjref_cache_write(C.byref(td), path.encode()) == 0
    m = read_cache_meta(path)
    assert m["num_rows"] == t.num_rows
    assert m["types"] == [c.type for c in t.columns]
    assert m["num_pages"] == [c.num_pages for c in t.columns]
    # and the library's writer produces the very same file
    mine = str(tmp_path / "lib.tbl")
    write_cache(t, mine)
    assert open(mine, "rb").read() == open(path, "rb").read()
