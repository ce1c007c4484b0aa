"""GPU: scan-side filters on resident tables (cj_table_filter) against the
oracle's filter: same selected rows, projected, in pages that are valid
and row-multiset-equal to the oracle's (the oracle is pinned against the
reference's own Statement::eval by tests/test_filter_oracle.py)."""
import numpy as np
import pytest

from calamarijoins_b200 import (CJError, ColumnarTable, Comparison, DataType, LogicalOperation, Plan,
                                ResidentTable, encode_column)
from calamarijoins_b200.datagen import config_c3
from oracle import oracle_api as oa
from tests.filter_cases import filter_table, rand_predicate
from tests.helpers import assert_same, run_oracle, run_product

pytestmark = pytest.mark.gpu
I, L, F, V = DataType.INT32, DataType.INT64, DataType.FP64, DataType.VARCHAR


def gpu_filter(ctx, table, pred, cols=None):
    rt = ResidentTable(ctx, table)
    try:
        out = rt.filter(pred, cols)
        try:
            host = out.download()
        finally:
            out.free()
    finally:
        rt.free()
    return oa.PagedResult.from_columnar(host)


@pytest.mark.parametrize("seed", range(4))
def test_random_predicates(gpu_ctx, seed):
    t = filter_table(20_000, seed, long_strings=(seed == 3))
    rng = np.random.default_rng(200 + seed)
    for k in range(12):
        pred = rand_predicate(rng)
        cols = [int(c) for c in rng.permutation(4)[: int(rng.integers(1, 5))]]
        want, sel = oa.oracle_filter(t, pred, cols)
        got = gpu_filter(gpu_ctx, t, pred, cols)
        assert got.num_rows == int(sel.sum())
        assert_same(got, want, f"seed {seed} predicate {k}")


def test_no_predicate_projects_all_rows(gpu_ctx):
    t = filter_table(7000, 9, long_strings=True)
    want, _ = oa.oracle_filter(t, None, [3, 1])
    assert_same(gpu_filter(gpu_ctx, t, None, [3, 1]), want)


def test_empty_selection_and_empty_table(gpu_ctx):
    t = filter_table(1000, 4)
    pred = Comparison(0, Comparison.GT, 1000)
    got = gpu_filter(gpu_ctx, t, pred)
    assert got.num_rows == 0
    e = ColumnarTable(0, [encode_column(I, np.zeros(0, np.int32))])
    assert gpu_filter(gpu_ctx, e, Comparison(0, Comparison.EQ, 1)).num_rows == 0


def test_large_table(gpu_ctx):
    """10,000,000 rows, full pages read in place: a range on INT32 and a
    LIKE on VARCHAR."""
    rng = np.random.default_rng(5)
    n = 10_000_000
    keys = rng.integers(0, 1 << 20, n).astype(np.int32)
    words = np.array([b"alpha", b"beta", b"gamma", b"delta", b"alphabet"], dtype=object)
    t = ColumnarTable(n, [encode_column(I, keys), encode_column(V, list(words[rng.integers(0, 5, n)]))])
    pred = LogicalOperation.makeAnd(Comparison(0, Comparison.LT, 1 << 18), Comparison(1, Comparison.LIKE, "%pha%"))
    want, sel = oa.oracle_filter(t, pred)
    got = gpu_filter(gpu_ctx, t, pred)
    assert got.num_rows == int(sel.sum()) > 0
    assert_same(got, want, "10M rows")


def test_filtered_tables_feed_a_plan(gpu_ctx):
    """The dimensions of a C3-shaped plan filtered on the GPU and joined as
    resident inputs give what the oracle gives on the oracle-filtered
    tables."""
    plan = config_c3(scale=0.02)
    preds = [Comparison(0, Comparison.GEQ, 0), LogicalOperation.makeNot(Comparison(1, Comparison.LIKE, "%a%")),
             Comparison(0, Comparison.NEQ, 3), Comparison(1, Comparison.IS_NOT_NULL), None]
    host = Plan()
    host.nodes, host.root = plan.nodes, plan.root
    host.inputs = [plan.inputs[0]]
    res = Plan()
    res.nodes, res.root = plan.nodes, plan.root
    keep = [ResidentTable(gpu_ctx, plan.inputs[0])]
    res.inputs = [keep[0]]
    for d, p in enumerate(preds):
        t = plan.inputs[1 + d]
        o, _ = oa.oracle_filter(t, p)
        from calamarijoins_b200 import Column
        host.inputs.append(ColumnarTable(o.num_rows, [Column(DataType(ty), pg) for ty, pg in zip(o.types, o.pages)]))
        rt = ResidentTable(gpu_ctx, t)
        keep.append(rt)
        f = rt.filter(p)
        keep.append(f)
        res.inputs.append(f)
    try:
        got, _ = run_product(res, gpu_ctx)
        assert_same(got, run_oracle(host), "filtered plan")
    finally:
        for t in keep:
            t.free()


def test_type_mismatch_rejected(gpu_ctx):
    t = filter_table(100, 1)
    rt = ResidentTable(gpu_ctx, t)
    try:
        for pred in (Comparison(3, Comparison.EQ, 5), Comparison(0, Comparison.LIKE, "a%"),
                     Comparison(1, Comparison.EQ, 2.5), Comparison(9, Comparison.EQ, 1)):
            with pytest.raises(CJError) as e:
                rt.filter(pred)
            assert e.value.status == 2  # CJ_ERR_INVALID_PLAN
    finally:
        rt.free()
