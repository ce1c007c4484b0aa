"""GPU: batched execution. Many plans of uneven size run level by level
with grouped launches; each result equals the plan run alone and the
oracle's."""
import numpy as np
import pytest

from calamarijoins_b200 import DataType, Plan, ResidentTable, execute_batch
from calamarijoins_b200.datagen import batch_plans, chain_plan, config_c3, join2
from oracle import oracle_api as oa
from tests.helpers import assert_same, load_unit_cases, plan_from_case, run_oracle, run_product

pytestmark = pytest.mark.gpu
I, L, V, F = DataType.INT32, DataType.INT64, DataType.VARCHAR, DataType.FP64


def collect(results):
    out = []
    for r in results:
        out.append(oa.PagedResult.from_result(r))
        r.free()
    return out


def test_batch_of_unit_cases(gpu_ctx):
    plans = [plan_from_case(c) for c in load_unit_cases()]
    res, sts, st = execute_batch(plans, gpu_ctx)
    assert all(s == 0 for s in sts)
    got = collect(res)
    for i, p in enumerate(plans):
        assert_same(got[i], run_oracle(p), f"case {i}")
    assert st["num_plans"] == len(plans)


def test_batch_mixed_equals_alone(gpu_ctx):
    rng = np.random.default_rng(9)
    plans = []
    for i in range(20):
        ways = int(rng.integers(2, 5))
        plans.append(chain_plan(ways, int(rng.integers(500, 50000)), rng, max_build=30000,
                                key_types=[I if rng.random() < 0.6 else L for _ in range(ways - 1)],
                                varchar_frac=0.3))
    plans.append(join2(3000, 20000, seed=2, build_payload=(F, V), probe_payload=(L,), probe_null=0.1,
                       varchar_kw=dict(long_frac=0.01)))
    plans.append(join2(2000, 3000, seed=3, unique_build=False))  # probe re-run inside the batch
    plans.append(config_c3(seed=4, scale=0.001, varchar_nulls=True, long_frac=0.002))
    alone = [run_product(p, gpu_ctx)[0] for p in plans]
    res, sts, st = execute_batch(plans, gpu_ctx)
    got = collect(res)
    for i in range(len(plans)):
        assert_same(got[i], alone[i], f"plan {i}")
    for i in (0, 20, 21, 22):
        assert_same(got[i], run_oracle(plans[i]), f"plan {i} vs oracle")
    assert st["probe_reruns"] >= 1
    assert st["syncs"] <= st["num_levels"] * 2 + 3


def test_batch_c4_shape_small(gpu_ctx):
    plans = batch_plans(64, seed=5, scale=0.01)
    res, sts, st = execute_batch(plans, gpu_ctx)
    got = collect(res)
    for i in range(0, 64, 9):
        assert_same(got[i], run_oracle(plans[i]), f"plan {i}")
    assert st["num_nested_loop_joins"] > 0 and st["num_hash_joins"] > 0


def test_batch_with_invalid_plan(gpu_ctx):
    good = join2(100, 1000, seed=1)
    bad = join2(100, 1000, seed=1)
    bad.root = 99
    res, sts, _ = execute_batch([good, bad, good], gpu_ctx)
    assert sts[1] != 0 and res[1] is None
    got = collect([res[0], res[2]])
    want = run_oracle(good)
    assert_same(got[0], want)
    assert_same(got[1], want)


def test_batch_resident_inputs(gpu_ctx):
    plan = join2(5000, 50000, seed=6, build_payload=(L,), probe_payload=(V,))
    rp = Plan()
    rp.nodes, rp.root = plan.nodes, plan.root
    rp.inputs = [ResidentTable(gpu_ctx, t) for t in plan.inputs]
    res, sts, st = execute_batch([rp] * 4, gpu_ctx)
    assert st["h2d_bytes"] == 0
    want = run_oracle(plan)
    for g in collect(res):
        assert_same(g, want)


def _resident(plans, ctx):
    out, tables = [], []
    for p in plans:
        rp = Plan()
        rp.nodes, rp.root = p.nodes, p.root
        rp.inputs = [ResidentTable(ctx, t) for t in p.inputs]
        tables.extend(rp.inputs)
        out.append(rp)
    return out, tables


@pytest.mark.parametrize("flags", [0, 1])  # host results, device results
def test_prepared_batch_replays(gpu_ctx, flags):
    """A batch captured as one CUDA graph: three replays in a row, each
    result equal to the oracle's (chain plans with nested-loop, direct and
    hash joins, INT64 keys, a many-to-many join)."""
    from calamarijoins_b200 import PreparedBatch
    rng = np.random.default_rng(14)
    plans = [chain_plan(int(rng.integers(2, 5)), int(rng.integers(1000, 80000)), rng, max_build=40000,
                        key_types=[I if rng.random() < 0.6 else L for _ in range(3)])
             for _ in range(12)]
    plans.append(join2(3000, 30000, seed=7, unique_build=False, build_payload=(L,), probe_payload=(F,)))
    plans.append(join2(40, 10000, seed=8))  # nested loop
    want = [run_oracle(p) for p in plans]
    rplans, tables = _resident(plans, gpu_ctx)
    pb = PreparedBatch(rplans, gpu_ctx, flags)
    try:
        for rep in range(3):
            res, st = pb.run()
            assert st["syncs"] == 1
            for i, r in enumerate(res):
                got = oa.PagedResult.from_result(r)
                r.free()
                assert_same(got, want[i], f"replay {rep} plan {i}")
    finally:
        pb.close()
        for t in tables:
            t.free()


def test_prepared_batch_needs_resident_inputs(gpu_ctx):
    from calamarijoins_b200 import CJError, PreparedBatch
    with pytest.raises(CJError) as e:
        PreparedBatch([join2(100, 1000, seed=1)], gpu_ctx)
    assert e.value.status == 6  # CJ_ERR_UNSUPPORTED


def test_prepared_batch_refuses_varchar_results(gpu_ctx):
    """A VARCHAR result's page count depends on the order of its rows,
    which differs between runs: a prepared batch refuses such plans."""
    from calamarijoins_b200 import CJError, PreparedBatch
    rplans, tables = _resident([join2(100, 1000, seed=1, build_payload=(V,))], gpu_ctx)
    try:
        with pytest.raises(CJError) as e:
            PreparedBatch(rplans, gpu_ctx)
        assert e.value.status == 6 and "VARCHAR" in str(e.value)
    finally:
        for t in tables:
            t.free()
