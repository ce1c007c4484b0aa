"""GPU: random plan trees through the product, against the oracle.

The plans are those of test_oracle_random_plans.py (where the oracle itself
is checked against the reference's execute()): 2-5 small tables, some
empty, INT32 keys over small domains with NULLs, INT32 and VARCHAR
payloads, and random join trees over scans of them: bushy or deep,
self-joins, keys anywhere in either side's outputs, output lists that
repeat or drop columns. Each plan runs through cj_execute with host and
with device results, and all of them together through one
cj_execute_batch; every result must equal the oracle's."""
import pytest

from calamarijoins_b200 import _lib, execute_batch
from oracle import oracle_api as oa
from tests.helpers import assert_same, run_oracle, run_product
from tests.test_oracle_random_plans import random_plan

pytestmark = pytest.mark.gpu

SEEDS = range(48)


def _plans():
    return [(s, p) for s in SEEDS for p in [random_plan(s)] if p is not None]


def test_random_plans_one_by_one(gpu_ctx):
    for seed, plan in _plans():
        want = run_oracle(plan)
        got, _ = run_product(plan, gpu_ctx)
        assert_same(got, want, f"seed {seed}")
        got, _ = run_product(plan, gpu_ctx, _lib.CJ_EXEC_RESULT_ON_DEVICE)
        assert_same(got, want, f"seed {seed}, result on the device")


def test_random_plans_batched(gpu_ctx):
    items = _plans()
    res, sts, _ = execute_batch([p for _, p in items], gpu_ctx)
    assert all(s == 0 for s in sts), sts
    for (seed, plan), r in zip(items, res):
        got = oa.PagedResult.from_result(r)
        r.free()
        assert_same(got, run_oracle(plan), f"seed {seed}, batched")
