"""GPU: failure handling, with every failure made on the host.

Nothing here faults, traps or hangs the device. The failures are an
injected exhaustion of the device memory pool (CJ_OPT_FAIL_ALLOC_AT makes
the N-th allocation fail as cudaMallocFromPoolAsync would), and a request
cancelled while it waits in the server's queue. After each, the context (or
server) must keep working and give results equal to the oracle's, and the
memory of the failed call must come back to the pool."""
import numpy as np
import pytest

from calamarijoins_b200 import CJError, DataType, Server
from calamarijoins_b200 import _lib
from calamarijoins_b200.datagen import chain_plan, join2
from tests.helpers import assert_same, run_oracle, run_product

pytestmark = pytest.mark.gpu
I, L, V = DataType.INT32, DataType.INT64, DataType.VARCHAR


def _plan():
    rng = np.random.default_rng(77)
    return chain_plan(4, 200_000, rng, max_build=50_000, key_types=[I, L, I], varchar_frac=0.5)


def test_injected_allocation_failure_leaves_context_usable(gpu_ctx):
    plan = _plan()
    want = run_oracle(plan)
    gpu_ctx.set_option(_lib.CJ_OPT_BUFFER_CACHE_BYTES, 0)  # every buffer goes back to the pool at once
    try:
        got, _ = run_product(plan, gpu_ctx)
        assert_same(got, want, "before")
        used0, _ = gpu_ctx.memory()
        failures = 0
        for n in (1, 2, 3, 5, 8, 13, 21, 34, 55, 89):
            gpu_ctx.set_option(_lib.CJ_OPT_FAIL_ALLOC_AT, n)
            try:
                got, _ = run_product(plan, gpu_ctx)
                assert_same(got, want, f"allocation {n} never reached")
            except CJError as e:
                assert e.status == 4, e  # CJ_ERR_OUT_OF_MEMORY
                assert "injected" in str(e)
                failures += 1
            gpu_ctx.set_option(_lib.CJ_OPT_FAIL_ALLOC_AT, 0)
            got, _ = run_product(plan, gpu_ctx)
            assert_same(got, want, f"after a failure at allocation {n}")
            used, _ = gpu_ctx.memory()
            assert used == used0, f"allocation {n}: {used - used0} bytes not returned"
        assert failures >= 5
    finally:
        gpu_ctx.set_option(_lib.CJ_OPT_FAIL_ALLOC_AT, 0)
        gpu_ctx.set_option(_lib.CJ_OPT_BUFFER_CACHE_BYTES, 16 << 30)


def test_injected_failure_inside_a_batch(gpu_ctx):
    from calamarijoins_b200 import execute_batch
    from calamarijoins_b200.datagen import batch_plans
    plans = batch_plans(16, seed=8, scale=0.01)
    gpu_ctx.set_option(_lib.CJ_OPT_FAIL_ALLOC_AT, 40)
    try:
        with pytest.raises(CJError) as ei:
            execute_batch(plans, gpu_ctx)
        assert ei.value.status == 4
    finally:
        gpu_ctx.set_option(_lib.CJ_OPT_FAIL_ALLOC_AT, 0)
    res, sts, _ = execute_batch(plans, gpu_ctx)
    from oracle import oracle_api as oa
    for i, (p, r) in enumerate(zip(plans, res)):
        got = oa.PagedResult.from_result(r)
        r.free()
        assert_same(got, run_oracle(p), f"plan {i} after the failed batch")


def test_server_cancel_queued_request():
    """One slot: a large plan runs while three small ones queue; the third
    is cancelled before it starts. Its wait reports CJ_ERR_CANCELLED, the
    others complete with the oracle's results, and a plan that has already
    run can no longer be cancelled."""
    big = join2(1_000_000, 20_000_000, seed=3, probe_payload=(I,))
    small = [join2(1000, 50_000, seed=10 + i, build_payload=(L,), probe_payload=(V,)) for i in range(3)]
    srv = Server(slots=1)
    try:
        tb = srv.submit(big)
        ts = [srv.submit(p) for p in small]
        srv.cancel(ts[2])
        with pytest.raises(CJError) as ei:
            srv.wait(ts[2])
        assert ei.value.status == 11  # CJ_ERR_CANCELLED
        for t, p in zip([tb] + ts[:2], [big] + small[:2]):
            r, _ = srv.wait(t)
            from oracle import oracle_api as oa
            got = oa.PagedResult.from_result(r)
            r.free()
            assert_same(got, run_oracle(p))
        with pytest.raises(CJError):
            srv.cancel(tb)  # finished: nothing to cancel
        st = srv.stats()
        assert st["cancelled"] == 1 and st["completed"] == 3
    finally:
        srv.close()
