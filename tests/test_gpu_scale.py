"""GPU parity at the benchmarked sizes.

The product runs the workload configurations at (or near) the sizes the
benchmark measures them at, and every result is compared with the oracle
bit for bit (row multiset: values, NULLs, VARCHAR bytes, FP64 bit
patterns) plus a structural check of every output page. These sizes reach
paths that small cases never do: the probe storing keys into result pages
over tens of millions of rows, many thousands of output pages, long-string
pages at the C3 rate, heavy-hitter keys walking tens of thousands of build
tuples on one lane, and the direct-mapped table's 2^28 span limit.

The reference semantics checked are those of Contest::execute
(src/execute.cpp:207-300): inner equi-join, NULL never matches, output
columns = root output_attrs over (left ++ right)."""
import numpy as np
import pytest

from calamarijoins_b200 import (ColumnarTable, DataType, Plan, PlanDescriptor, ResidentTable, encode_column,
                                execute_batch, execute_raw)
from calamarijoins_b200 import _lib
from calamarijoins_b200.datagen import batch_plans, config_c2, config_c2s, config_c3
from oracle import oracle_api as oa
from tests.helpers import assert_same, run_oracle, run_product

pytestmark = pytest.mark.gpu
I, L, F, V = DataType.INT32, DataType.INT64, DataType.FP64, DataType.VARCHAR


def _resident_device_result(plan, ctx):
    """The bench's form of the call: inputs resident in HBM, result pages
    left on the device, then copied back for the comparison."""
    rp = Plan()
    rp.nodes, rp.root = plan.nodes, plan.root
    rp.inputs = [ResidentTable(ctx, t) for t in plan.inputs]
    try:
        res, st = execute_raw(rp, ctx, _lib.CJ_EXEC_RESULT_ON_DEVICE)
        try:
            return oa.PagedResult.from_result(res), st
        finally:
            res.free()
    finally:
        for t in rp.inputs:
            t.free()


def test_c2_full_size(gpu_ctx):
    """C2: 4,000,000 x 64,000,000, about 43.9M output rows; host pages in
    and out, and resident inputs with a device result."""
    plan = config_c2(seed=202, scale=1.0)
    want = run_oracle(plan)
    assert want.num_rows > 40_000_000
    got, st = run_product(plan, gpu_ctx)
    assert st.exec["num_direct_joins"] == 1
    assert_same(got, want, "c2 host")
    del got
    got, _ = _resident_device_result(plan, gpu_ctx)
    assert_same(got, want, "c2 resident")
    assert oa.fingerprint(got) == oa.fingerprint(want)


def test_c2s_full_size(gpu_ctx):
    """C2 with the build keys spread 500x: the open-addressing table."""
    plan = config_c2s(scale=1.0)
    want = run_oracle(plan)
    got, st = run_product(plan, gpu_ctx)
    assert st.exec["num_open_joins"] == 1
    assert_same(got, want, "c2s")


def test_c2_full_size_hash_table(gpu_ctx):
    """C2 forced onto the unchained hash table (radix-partitioned build,
    Bloom-tag probe) at full size."""
    gpu_ctx.set_option(_lib.CJ_OPT_DENSE_KEYS, 0)
    try:
        plan = config_c2(seed=202, scale=1.0)
        want = run_oracle(plan)
        got, st = run_product(plan, gpu_ctx)
        assert st.exec["num_direct_joins"] == 0 and st.exec["num_open_joins"] == 0
        assert_same(got, want, "c2 hash")
    finally:
        gpu_ctx.set_option(_lib.CJ_OPT_DENSE_KEYS, 8)


def test_c2h_full_size(gpu_ctx):
    """C2's shape with a non-unique build side (4M rows over 3M distinct
    keys): only the unchained hash table can serve it; about 59M output
    rows."""
    from calamarijoins_b200.datagen import config_c2h
    plan = config_c2h(scale=1.0)
    want = run_oracle(plan)
    assert want.num_rows > 50_000_000
    got, st = run_product(plan, gpu_ctx)
    assert st.exec["num_direct_joins"] == 0 and st.exec["num_open_joins"] == 0
    assert_same(got, want, "c2h")


@pytest.mark.parametrize("varchar_nulls", [False, True])
def test_c3_full_size(gpu_ctx, varchar_nulls):
    """C3 at full size: the 36M-row fact table through five joins into
    dimensions of 2,500 to 4,200,000 rows, VARCHAR outputs with 0.01 % long
    strings (several long-string pages in the result)."""
    plan = config_c3(scale=1.0, varchar_nulls=varchar_nulls)
    want = run_oracle(plan)
    got, _ = run_product(plan, gpu_ctx)
    assert_same(got, want, f"c3 nulls={varchar_nulls}")
    long_pages = sum(int(((p[:, 0] == 0xFF) & (p[:, 1] == 0xFF)).sum()) for t, p in zip(got.types, got.pages)
                     if t == int(V))
    assert long_pages > 0


def test_c4_all_plans_batched(gpu_ctx):
    """All 256 C4 plans at scale 0.1 through cj_execute_batch, each against
    the oracle."""
    plans = batch_plans(256, seed=404, scale=0.1)
    res, sts, st = execute_batch(plans, gpu_ctx)
    assert all(s == 0 for s in sts)
    assert st["num_nested_loop_joins"] > 0 and st["num_hash_joins"] > 0
    for i, (p, r) in enumerate(zip(plans, res)):
        got = oa.PagedResult.from_result(r)
        r.free()
        assert_same(got, run_oracle(p), f"c4 plan {i}")


def _heavy_hitter_plan(seed=12):
    """Many-to-many join: 200,000 build rows whose keys follow Zipf(1.2)
    over 50,000 values (the top key holds about 40,000 rows), 600,000
    probe rows spread evenly over the same values: the top key alone has
    several 10^5 matches, each of its probe rows tens of thousands."""
    from calamarijoins_b200.datagen import zipf_ranks
    rng = np.random.default_rng(seed)
    dom = 50_000
    perm = rng.permutation(dom).astype(np.int64)
    bk = perm[zipf_ranks(dom, 1.2, 200_000, rng) - 1]
    pk = perm[rng.integers(0, dom, 600_000)]
    pvalid = (rng.random(600_000) > 0.02).astype(np.uint8)
    plan = Plan()
    plan.inputs.append(ColumnarTable(len(bk), [encode_column(I, bk.astype(np.int32)),
                                               encode_column(L, rng.integers(-(1 << 40), 1 << 40, len(bk)))]))
    plan.inputs.append(ColumnarTable(len(pk), [encode_column(I, pk.astype(np.int32), pvalid),
                                               encode_column(I, rng.integers(0, 1 << 30, len(pk)).astype(np.int32))]))
    plan.new_scan_node(0, [(0, I), (1, L)])
    plan.new_scan_node(1, [(0, I), (1, I)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, I), (1, L), (3, I)])
    plan.root = 2
    top = np.bincount(bk).max()
    return plan, int(top)


def test_heavy_hitter_zipf_1_2(gpu_ctx):
    plan, top = _heavy_hitter_plan()
    assert top > 20_000
    want = run_oracle(plan)
    assert want.num_rows > 2_000_000
    got, st = run_product(plan, gpu_ctx)
    assert st.exec["num_direct_joins"] == 0
    assert_same(got, want, "heavy hitter")


def _span_plan(span_extra: int):
    """Unique build keys spanning 2^28 + span_extra values (2^25 rows, the
    fewest that allow the span at the default density 8), probed by a
    larger table (so that the keys build) of keys drawn from them and from
    outside their range."""
    rng = np.random.default_rng(28)
    nb = 1 << 25
    lo = -(1 << 27)
    span = (1 << 28) + span_extra
    inner = rng.choice(span - 2, size=nb - 2, replace=False) + 1
    keys = np.concatenate([[0, span - 1], inner]).astype(np.int64) + lo
    rng.shuffle(keys)
    npr = nb + 1_000_000
    pk = np.where(rng.random(npr) < 0.7, keys[rng.integers(0, nb, npr)], rng.integers(lo - 1000, lo + span + 1000, npr))
    plan = Plan()
    plan.inputs.append(ColumnarTable(nb, [encode_column(I, keys.astype(np.int32))]))
    plan.inputs.append(ColumnarTable(len(pk), [encode_column(I, pk.astype(np.int32))]))
    plan.new_scan_node(0, [(0, I)])
    plan.new_scan_node(1, [(0, I)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, I), (1, I)])
    plan.root = 2
    return plan


@pytest.mark.parametrize("span_extra,direct", [(0, True), (1, False)])
def test_direct_mapped_span_limit(gpu_ctx, span_extra, direct):
    """A key span of exactly 2^28 takes the direct-mapped table; one more
    value and the join goes to the open-addressing table. Same results."""
    plan = _span_plan(span_extra)
    want = run_oracle(plan)
    got, st = run_product(plan, gpu_ctx)
    assert st.exec["num_direct_joins"] == (1 if direct else 0)
    assert st.exec["num_open_joins"] == (0 if direct else 1)
    assert_same(got, want, f"span 2^28+{span_extra}")


def test_two_pass_radix_build(gpu_ctx):
    """A non-unique build side of 9,000,000 rows: 2^24 directory slots in
    2^13 partitions, more radix bits than one pass takes, so the build runs
    a second, per-partition radix pass."""
    from calamarijoins_b200.datagen import fk_column
    rng = np.random.default_rng(31)
    nb, npr = 9_000_000, 20_000_000
    distinct = rng.permutation(6_000_000).astype(np.int64) * 3 - 9_000_000
    bk = np.concatenate([distinct, distinct[:nb - len(distinct)]])
    rng.shuffle(bk)
    pk, pv = fk_column(distinct, npr, 0.9, 0.2, 0.02, rng)
    plan = Plan()
    plan.inputs.append(ColumnarTable(nb, [encode_column(I, bk.astype(np.int32)),
                                          encode_column(I, rng.integers(0, 1 << 30, nb).astype(np.int32))]))
    plan.inputs.append(ColumnarTable(npr, [encode_column(I, pk, pv)]))
    plan.new_scan_node(0, [(0, I), (1, I)])
    plan.new_scan_node(1, [(0, I)])
    plan.new_join_node(True, 0, 1, 0, 0, [(1, I), (2, I)])
    plan.root = 2
    want = run_oracle(plan)
    got, st = run_product(plan, gpu_ctx)
    assert st.exec["num_direct_joins"] == 0 and st.exec["num_open_joins"] == 0
    assert_same(got, want, "two-pass build")
