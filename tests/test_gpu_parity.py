"""GPU parity: the sm_100a path through the C ABI against the oracle and the
reference's known answers. Bit-exact: every output table must be the same
row multiset (values, NULLs, VARCHAR bytes, FP64 bit patterns) as the
oracle's, and every output page must be well formed."""
import numpy as np
import pytest

from calamarijoins_b200 import (CJError, ColumnarTable, DataType, Plan, PlanDescriptor, ResidentTable, Table,
                                encode_column, execute_raw)
from calamarijoins_b200 import _lib
from calamarijoins_b200.datagen import chain_plan, config_c1, config_c3, join2
from oracle import oracle_api as oa
from tests.helpers import assert_same, check_expect, load_unit_cases, plan_from_case, run_oracle, run_product

pytestmark = pytest.mark.gpu

I, L, F, V = DataType.INT32, DataType.INT64, DataType.FP64, DataType.VARCHAR
CASES = load_unit_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_unit_case(gpu_ctx, case):
    plan = plan_from_case(case)
    r, _ = run_product(plan, gpu_ctx)
    check_expect(r, case["expect"], case["name"])
    assert_same(r, run_oracle(plan), case["name"])


@pytest.mark.parametrize("nl_max", [0, 7, 64])
def test_unit_cases_any_threshold(gpu_ctx, nl_max):
    """Results do not depend on the nested-loop threshold."""
    gpu_ctx.set_option(_lib.CJ_OPT_NESTED_LOOP_MAX_BUILD, nl_max)
    try:
        for case in CASES:
            plan = plan_from_case(case)
            r, _ = run_product(plan, gpu_ctx)
            check_expect(r, case["expect"], case["name"])
    finally:
        gpu_ctx.set_option(_lib.CJ_OPT_NESTED_LOOP_MAX_BUILD, 64)


JOIN_CASES = [
    # n_build, n_probe, kwargs
    (1, 1000, dict()),
    (5, 3000, dict(build_null=0.2, probe_null=0.1)),
    (64, 20000, dict(zipf=1.2)),
    (65, 20000, dict(zipf=1.2)),
    (1000, 50000, dict(outside=0.3, probe_null=0.05)),
    (2047, 4096, dict(zipf=0.0)),
    (2049, 4096, dict(zipf=0.0)),
    (100_000, 1_000_000, dict(zipf=1.0, probe_null=0.05)),
    (300_000, 200_000, dict(zipf=0.8)),  # build larger than probe: sides swap
    (50_000, 400_000, dict(key_type=L, zipf=0.9, outside=0.2)),
    (20_000, 100_000, dict(unique_build=False, zipf=0.5)),  # many-to-many
    (3000, 30000, dict(build_payload=(I, L, F, V), probe_payload=(V, F), probe_null=0.1)),
]


@pytest.mark.parametrize("nb,npr,kw", JOIN_CASES, ids=[f"{a}x{b}-{i}" for i, (a, b, _) in enumerate(JOIN_CASES)])
@pytest.mark.parametrize("build_left", [True, False])
def test_join_parity(gpu_ctx, nb, npr, kw, build_left):
    plan = join2(nb, npr, seed=nb * 7 + npr, build_left=build_left, **kw)
    r, st = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), f"{nb}x{npr}")
    assert st.exec["kernel_launches"] > 0


@pytest.mark.parametrize("output", [[0], [3], [1, 2], [2, 0], []])
def test_projection_modes(gpu_ctx, output):
    """Build-only, probe-only and empty projections (collection modes,
    join_setup.h:146-173)."""
    plan = join2(5000, 40000, seed=11, zipf=1.0, build_payload=(I,), probe_payload=(F,), output=output,
                 probe_null=0.1)
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan))


def test_many_to_many_rerun(gpu_ctx):
    """Duplicate build keys: the first probe overflows its capacity guess and
    is re-run with the exact size."""
    plan = join2(4000, 6000, seed=5, unique_build=False, zipf=0.0)
    r, st = run_product(plan, gpu_ctx)
    assert st.exec["probe_reruns"] >= 1
    assert_same(r, run_oracle(plan))


def test_varchar_nulls_and_long_strings(gpu_ctx):
    plan = join2(4000, 30000, seed=9, build_payload=(V,), probe_payload=(V, I), probe_null=0.05,
                 varchar_kw=dict(long_frac=0.01))
    # NULLs inside the VARCHAR payloads too
    rng = np.random.default_rng(1)
    from calamarijoins_b200.datagen import varchar_values
    chars, offs = varchar_values(30000, rng, long_frac=0.005)
    valid = (rng.random(30000) > 0.3).astype(np.uint8)
    plan.inputs[1].columns[1] = encode_column(V, (chars, offs), valid)
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_chain_plans(gpu_ctx, seed):
    rng = np.random.default_rng(seed)
    ways = 2 + seed
    plan = chain_plan(ways, 20000, rng, max_build=50000, varchar_frac=0.5,
                      key_types=[I if (seed + d) % 2 else L for d in range(ways - 1)])
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), f"chain {seed}")


@pytest.mark.parametrize("varchar_nulls", [False, True])
def test_c3_pipeline_small(gpu_ctx, varchar_nulls):
    plan = config_c3(seed=33, scale=0.002, varchar_nulls=varchar_nulls, long_frac=0.002)
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), "c3")


def test_c1_full(gpu_ctx):
    plan = config_c1()
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), "c1")


def test_empty_inputs(gpu_ctx):
    plan = join2(10, 10, seed=1)
    plan.inputs[0] = ColumnarTable(0, [encode_column(I, np.zeros(0, np.int32)),
                                       encode_column(I, np.zeros(0, np.int32))])
    r, _ = run_product(plan, gpu_ctx)
    assert r.num_rows == 0 and r.types == [0, 0, 0, 1]
    assert all(p.shape[0] == 0 for p in r.pages)


def test_all_null_probe(gpu_ctx):
    plan = join2(100, 5000, seed=2, probe_null=1.0)
    r, _ = run_product(plan, gpu_ctx)
    assert r.num_rows == 0


def test_int32_min_through_intermediate(gpu_ctx):
    """INT32_MIN leaving a non-root join reads as NULL afterwards (value_t,
    intermediate.h:56-62): as an output value and as a key."""
    imin = -(2 ** 31)
    plan = Plan()
    a = Table([[1, imin], [2, 5], [3, imin]], [I, I]).to_columnar()
    b = Table([[1], [2], [3]], [I]).to_columnar()
    c = Table([[imin], [5], [7]], [I]).to_columnar()
    plan.inputs += [a, b, c]
    plan.new_scan_node(0, [(0, I), (1, I)])
    plan.new_scan_node(1, [(0, I)])
    plan.new_scan_node(2, [(0, I)])
    j = plan.new_join_node(True, 1, 0, 0, 0, [(0, I), (2, I)])  # (key, a.payload)
    plan.new_join_node(True, j, 2, 1, 0, [(0, I), (1, I), (2, I)])  # join on a.payload
    plan.root = 4
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan))
    assert r.num_rows == 1  # only payload 5 matches; INT32_MIN became NULL
    plan.root = j
    r2, _ = run_product(plan, gpu_ctx)
    assert_same(r2, run_oracle(plan))  # at the root it is still a value


def test_scan_root(gpu_ctx):
    plan = join2(1000, 10, seed=3, build_payload=(V, F))
    plan.root = 0
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan))
    assert r.num_rows == 1000


def test_resident_tables(gpu_ctx):
    plan = join2(20000, 100000, seed=4, build_payload=(L,), probe_payload=(V,), probe_null=0.1)
    want = run_oracle(plan)
    res_plan = Plan()
    res_plan.nodes = plan.nodes
    res_plan.root = plan.root
    res_plan.inputs = [ResidentTable(gpu_ctx, t) for t in plan.inputs]
    for _ in range(2):
        r, st = run_product(res_plan, gpu_ctx)
        assert_same(r, want)
        assert st.exec["h2d_bytes"] == 0


def test_result_on_device(gpu_ctx):
    plan = join2(5000, 20000, seed=6)
    res, _ = execute_raw(plan, gpu_ctx, _lib.CJ_EXEC_RESULT_ON_DEVICE)
    try:
        assert res.column_info(0)[2] is None  # no host copy
        r = oa.PagedResult.from_result(res)
    finally:
        res.free()
    assert_same(r, run_oracle(plan))


def test_malformed_pages_rejected(gpu_ctx):
    plan = join2(3000, 3000, seed=7)
    bad = plan.inputs[1].columns[0].pages.copy()
    bad[0, 2:4] = np.frombuffer(np.uint16(9000).tobytes(), np.uint8)  # n_values > n_rows
    plan.inputs[1].columns[0].pages = bad
    with pytest.raises(CJError) as e:
        run_product(plan, gpu_ctx)
    assert e.value.status == 3
    ok = join2(300, 3000, seed=8)  # context still usable
    r, _ = run_product(ok, gpu_ctx)
    assert_same(r, run_oracle(ok))


def test_row_count_mismatch_rejected(gpu_ctx):
    plan = join2(3000, 3000, seed=7)
    plan.inputs[1].num_rows = 2999
    with pytest.raises(CJError) as e:
        run_product(plan, gpu_ctx)
    assert e.value.status == 3


def test_invalid_plans(gpu_ctx):
    plan = join2(30, 30, seed=1)
    plan.nodes[2].output_attrs[0] = (0, DataType.FP64)  # wrong declared type
    with pytest.raises(CJError) as e:
        run_product(plan, gpu_ctx)
    assert e.value.status == 2
    plan = join2(30, 30, seed=1, build_payload=(F,), probe_payload=(F,))
    plan.nodes[2].data.left_attr = 1  # FP64 key
    with pytest.raises(CJError) as e:
        run_product(plan, gpu_ctx)
    assert e.value.status == 6


def test_memory_returns_to_pool(gpu_ctx):
    plan = join2(10000, 100000, seed=12, build_payload=(V,))
    run_product(plan, gpu_ctx)
    used1, _ = gpu_ctx.memory()
    for _ in range(3):
        run_product(plan, gpu_ctx)
    used2, _ = gpu_ctx.memory()
    assert used2 <= used1
