"""GPU: cj_hash_join_noalloc, the join entry point for callers that cannot
let a library allocate device memory (their own allocator or a fixed
budget owns the GPU). It must find exactly the (build row, probe row) pairs
that the regular allocating path (cj_execute) finds for the same two
tables, and keep doing so on a second call, which reuses the same fixed
device scratch array left over from the first.

Kept in a file of its own that pytest collects last."""
import ctypes as C

import numpy as np
import pytest
import torch

from calamarijoins_b200 import ColumnarTable, DataType, Plan, encode_column
from calamarijoins_b200 import _lib
from calamarijoins_b200.datagen import fk_column
from tests.helpers import run_oracle, run_product

pytestmark = pytest.mark.gpu
I = DataType.INT32


def make_tables(seed, nb, npr):
    rng = np.random.default_rng(seed)
    bkeys = rng.integers(0, nb // 2 + 1, size=nb).astype(np.int32)  # duplicates on the build side
    bvalid = (rng.random(nb) > 0.05).astype(np.uint8)
    pkeys, pvalid = fk_column(np.unique(bkeys).astype(np.int64), npr, 0.9, 0.25, 0.03, rng)
    pvalid = np.ones(npr, np.uint8) if pvalid is None else pvalid
    return bkeys, bvalid, pkeys.astype(np.int32), pvalid


def pairs_plan(bkeys, bvalid, pkeys, pvalid):
    """A 2-table plan whose outputs are the row numbers of the matching
    build and probe rows."""
    plan = Plan()
    nb, npr = len(bkeys), len(pkeys)
    plan.inputs.append(ColumnarTable(nb, [encode_column(I, bkeys, bvalid),
                                          encode_column(I, np.arange(nb, dtype=np.int32))]))
    plan.inputs.append(ColumnarTable(npr, [encode_column(I, pkeys, pvalid),
                                           encode_column(I, np.arange(npr, dtype=np.int32))]))
    plan.new_scan_node(0, [(0, I), (1, I)])
    plan.new_scan_node(1, [(0, I), (1, I)])
    plan.new_join_node(True, 0, 1, 0, 0, [(1, I), (3, I)])
    plan.root = 2
    return plan


def pairs_of(r):
    from calamarijoins_b200 import Column, decode_column
    b, _ = decode_column(Column(I, r.pages[0]))
    p, _ = decode_column(Column(I, r.pages[1]))
    return np.stack([b, p], axis=1).astype(np.int64)


def pairs_from_execute(ctx, bkeys, bvalid, pkeys, pvalid):
    """The regular, allocating entry point (cj_execute)."""
    r, _ = run_product(pairs_plan(bkeys, bvalid, pkeys, pvalid), ctx)
    return pairs_of(r)


def pairs_from_oracle(bkeys, bvalid, pkeys, pvalid):
    return pairs_of(run_oracle(pairs_plan(bkeys, bvalid, pkeys, pvalid)))


def bitmap(valid):
    n = len(valid)
    bits = np.packbits(valid.astype(np.uint8), bitorder="little")
    words = np.zeros(((n + 31) // 32) * 4, np.uint8)
    words[:len(bits)] = bits
    return torch.from_numpy(words.view(np.int32).copy()).cuda()


def pairs_from_noalloc(bkeys, bvalid, pkeys, pvalid, capacity, slack=0):
    """Calls the no-allocation entry point through the C ABI; returns the
    pairs written and the full match count. `slack` extra output entries
    past `capacity` are checked to stay untouched."""
    lib = _lib.lib()
    bk = torch.from_numpy(bkeys).cuda() if len(bkeys) else torch.zeros(1, dtype=torch.int32, device="cuda")
    pk = torch.from_numpy(pkeys).cuda() if len(pkeys) else torch.zeros(1, dtype=torch.int32, device="cuda")
    bv = bitmap(bvalid) if len(bvalid) else torch.zeros(1, dtype=torch.int32, device="cuda")
    pv = bitmap(pvalid) if len(pvalid) else torch.zeros(1, dtype=torch.int32, device="cuda")
    ob = torch.full((capacity + slack + 1,), -1, dtype=torch.int32, device="cuda")
    op = torch.full((capacity + slack + 1,), -1, dtype=torch.int32, device="cuda")
    dc = torch.zeros(1, dtype=torch.int64, device="cuda")
    hc = C.c_uint64(0)
    torch.cuda.synchronize()
    rc = lib.cj_hash_join_noalloc(bk.data_ptr(), bv.data_ptr(), len(bkeys), pk.data_ptr(), pv.data_ptr(),
                                  len(pkeys), ob.data_ptr(), op.data_ptr(), capacity, dc.data_ptr(), C.byref(hc),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.cj_last_error()
    total = hc.value
    assert total == int(dc.item())
    n = min(total, capacity)
    assert (ob[capacity:] == -1).all() and (op[capacity:] == -1).all(), "written past capacity"
    return np.stack([ob[:n].cpu().numpy(), op[:n].cpu().numpy()], axis=1).astype(np.int64), total


def sorted_pairs(a):
    return a[np.lexsort((a[:, 1], a[:, 0]))]


def test_noalloc_matches_execute_twice(gpu_ctx):
    # calls in a row, smaller, larger, then smaller again: the shared
    # scratch array keeps the previous call's directory and tuples, which
    # must not leak into the next result. Each result equals the regular
    # entry point's pairs and the oracle's.
    for seed, nb, npr in ((1, 5_000, 100_000), (2, 200_000, 400_000), (3, 3_000, 50_000)):
        bkeys, bvalid, pkeys, pvalid = make_tables(seed, nb, npr)
        want = sorted_pairs(pairs_from_execute(gpu_ctx, bkeys, bvalid, pkeys, pvalid))
        assert np.array_equal(want, sorted_pairs(pairs_from_oracle(bkeys, bvalid, pkeys, pvalid)))
        got, total = pairs_from_noalloc(bkeys, bvalid, pkeys, pvalid, capacity=len(want) + 1000)
        got = sorted_pairs(got)
        assert total == len(want)
        assert got.shape == want.shape
        assert np.array_equal(got, want)


def test_noalloc_capacity_below_count(gpu_ctx):
    """Fewer output slots than matches: the full count comes back, nothing is
    written past capacity, and what is written is a subset of the pairs."""
    bkeys, bvalid, pkeys, pvalid = make_tables(4, 20_000, 200_000)
    want = sorted_pairs(pairs_from_oracle(bkeys, bvalid, pkeys, pvalid))
    cap = len(want) // 3
    got, total = pairs_from_noalloc(bkeys, bvalid, pkeys, pvalid, capacity=cap, slack=4096)
    assert total == len(want)
    assert got.shape == (cap, 2)
    wset = set(map(tuple, want.tolist()))
    gl = list(map(tuple, got.tolist()))
    assert len(set(gl)) == cap and all(g in wset for g in gl)
    # and the next call with room for all of them gets all of them
    got, total = pairs_from_noalloc(bkeys, bvalid, pkeys, pvalid, capacity=total)
    assert np.array_equal(sorted_pairs(got), want)


@pytest.mark.parametrize("nb,npr", [(0, 1000), (1000, 0), (0, 0)])
def test_noalloc_empty_side(gpu_ctx, nb, npr):
    """An empty side joins to nothing: count 0, outputs untouched."""
    bkeys, bvalid, pkeys, pvalid = make_tables(5, max(nb, 2), max(npr, 2))
    bkeys, bvalid, pkeys, pvalid = bkeys[:nb], bvalid[:nb], pkeys[:npr], pvalid[:npr]
    got, total = pairs_from_noalloc(bkeys, bvalid, pkeys, pvalid, capacity=16, slack=16)
    assert total == 0 and got.shape == (0, 2)


def test_noalloc_rejects_oversized_build():
    lib = _lib.lib()
    dc = torch.zeros(1, dtype=torch.int64, device="cuda")
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = lib.cj_hash_join_noalloc(dummy.data_ptr(), dummy.data_ptr(), (1 << 18) + 1, dummy.data_ptr(),
                                  dummy.data_ptr(), 4, dummy.data_ptr(), dummy.data_ptr(), 4, dc.data_ptr(), None,
                                  None)
    assert rc == 7  # CJ_ERR_LIMIT
    assert b"262144" in lib.cj_last_error()
