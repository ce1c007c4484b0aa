"""GPU: serving. Plans submitted together run concurrently (several worker
streams, one memory pool, admission by estimated bytes) and each result is
the same as the plan run alone and as the oracle's."""
import numpy as np
import pytest

from calamarijoins_b200 import CJError, DataType, PlanDescriptor, Server
from calamarijoins_b200.datagen import chain_plan, join2
from oracle import oracle_api as oa
from tests.helpers import assert_same, run_oracle, run_product

pytestmark = pytest.mark.gpu
I, L, V = DataType.INT32, DataType.INT64, DataType.VARCHAR


def mixed_plans(n, seed=1):
    rng = np.random.default_rng(seed)
    plans = []
    for i in range(n):
        if i % 3 == 0:
            plans.append(join2(int(rng.integers(5, 5000)), int(rng.integers(1000, 60000)), seed=i,
                               build_payload=(L, V), probe_payload=(I,), probe_null=0.05))
        else:
            ways = int(rng.integers(2, 5))
            plans.append(chain_plan(ways, int(rng.integers(1000, 40000)), rng, max_build=20000,
                                    key_types=[I if rng.random() < 0.7 else L for _ in range(ways - 1)],
                                    varchar_frac=0.1))
    return plans


def test_alone_equals_in_the_mix(gpu_ctx):
    plans = mixed_plans(24)
    alone = [run_product(p, gpu_ctx)[0] for p in plans]
    srv = Server(slots=4)
    try:
        tickets = [srv.submit(p) for p in plans]
        mixed = []
        for t in tickets:
            res, _ = srv.wait(t)
            mixed.append(oa.PagedResult.from_result(res))
            res.free()
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == len(plans) and st["failed"] == 0
    assert st["p99_us"] >= st["p50_us"] > 0
    for i, (a, m) in enumerate(zip(alone, mixed)):
        assert_same(m, a, f"plan {i} alone vs mix")
    for i in (0, 1, 5):
        assert_same(mixed[i], run_oracle(plans[i]), f"plan {i} vs oracle")


def test_admission_budget_and_rejection():
    plans = mixed_plans(6, seed=2)
    est = [Server.estimate(p) for p in plans]
    srv = Server(slots=4, memory_budget=max(est) + 1)
    try:
        tickets = [srv.submit(p) for p in plans]
        for t in tickets:
            res, _ = srv.wait(t)
            res.free()
        st = srv.stats()
        assert st["peak_admitted_bytes"] <= st["memory_budget"]
        big = join2(2_000_000, 4_000_000, seed=3)
        with pytest.raises(CJError) as e:
            srv.submit(big)
        assert e.value.status == 9  # CJ_ERR_REJECTED
    finally:
        srv.close()


def test_failure_is_isolated():
    good = join2(1000, 5000, seed=4)
    bad = join2(1000, 5000, seed=5)
    bad.inputs[1].num_rows += 1  # pages hold one row fewer than declared
    srv = Server(slots=2)
    try:
        tb, tg = srv.submit(bad), srv.submit(good)
        with pytest.raises(CJError) as e:
            srv.wait(tb)
        assert e.value.status == 3
        res, _ = srv.wait(tg)
        r = oa.PagedResult.from_result(res)
        res.free()
        assert_same(r, run_oracle(good))
    finally:
        srv.close()


def test_continuous_batching_equals_alone(gpu_ctx):
    """One worker, many plans queued at once: the worker takes them in
    batches (one grouped execution each) and every result equals the plan
    run alone."""
    plans = mixed_plans(30, seed=6)
    alone = [run_product(p, gpu_ctx)[0] for p in plans]
    srv = Server(slots=1, max_batch=16)
    try:
        tickets = [srv.submit(p) for p in plans]
        got = []
        for t in tickets:
            res, _ = srv.wait(t)
            got.append(oa.PagedResult.from_result(res))
            res.free()
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == len(plans)
    assert st["mean_batch"] > 1.5, st
    for i, (a, g) in enumerate(zip(alone, got)):
        assert_same(g, a, f"plan {i} batched vs alone")


def test_admission_passes_over_a_plan_that_does_not_fit():
    """Two slots, a budget that holds one large plan and a few small ones:
    while the first large plan runs, a second large plan waits, and the
    small plans behind it are admitted ahead of it (it has not waited past
    the age limit); the second large plan runs once the first is done."""
    big = [join2(500_000, 12_000_000, seed=20 + i, probe_payload=(I,)) for i in range(2)]
    small = [join2(500, 5_000, seed=30 + i) for i in range(6)]
    eb = max(Server.estimate(p) for p in big)
    es = max(Server.estimate(p) for p in small)
    srv = Server(slots=2, memory_budget=eb + 3 * es, max_batch=1, age_limit_us=10_000_000)
    try:
        t_big = [srv.submit(p) for p in big]
        t_small = [srv.submit(p) for p in small]
        for t, p in zip(t_big + t_small, big + small):
            res, _ = srv.wait(t)
            r = oa.PagedResult.from_result(res)
            res.free()
            assert_same(r, run_oracle(p))
        st = srv.stats()
    finally:
        srv.close()
    assert st["skipped_ahead"] >= 1, st
    assert st["peak_admitted_bytes"] <= st["memory_budget"]


@pytest.mark.parametrize("cache_mb", [0, 64, 1024])
def test_reserved_host_cache(gpu_ctx, cache_mb):
    """Host results carved from a page-locked cache reserved at creation:
    results held at once, freed out of order and re-used by later plans of
    other sizes, each equal to the plan run alone. A cache too small for
    the results held at once (64 MB) falls back to allocating blocks; a
    large one (1 GB) serves them all without another allocation."""
    plans = mixed_plans(30, seed=9)
    alone = [run_product(p, gpu_ctx)[0] for p in plans]
    srv = Server(slots=4, max_batch=8, host_cache_bytes=cache_mb << 20)
    try:
        st0 = srv.stats(reset=True)
        assert st0["pinned_allocs"] == (1 if cache_mb else 0)  # the reservation itself
        for rnd in range(2):
            tickets = [srv.submit(p) for p in plans]
            results = [srv.wait(t)[0] for t in tickets]
            got = [oa.PagedResult.from_result(r) for r in results]
            for r in results[1::2] + results[0::2]:  # freed out of order
                r.free()
            for i, (g, a) in enumerate(zip(got, alone)):
                assert_same(g, a, f"round {rnd} plan {i} cache {cache_mb} MB")
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == 2 * len(plans) and st["failed"] == 0
    if cache_mb >= 1024:
        assert st["pinned_allocs"] == 0


def test_device_reserve(gpu_ctx):
    """A server whose pool takes 2 GB at creation holds at least that much
    from the start and runs plans as usual; the results equal the plans run
    alone."""
    plans = mixed_plans(8, seed=12)
    alone = [run_product(p, gpu_ctx)[0] for p in plans]
    srv = Server(slots=2, device_reserve_bytes=2 << 30)
    try:
        assert srv.stats()["pool_high_bytes"] >= 2 << 30
        tickets = [srv.submit(p) for p in plans]
        for i, (t, a) in enumerate(zip(tickets, alone)):
            r, _ = srv.wait(t)
            got = oa.PagedResult.from_result(r)
            r.free()
            assert_same(got, a, f"plan {i}")
    finally:
        srv.close()
