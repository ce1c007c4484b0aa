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
from tests.helpers import run_product

pytestmark = pytest.mark.gpu
I = DataType.INT32


def make_tables(seed, nb, npr):
    rng = np.random.default_rng(seed)
    bkeys = rng.integers(0, nb // 2 + 1, size=nb).astype(np.int32)  # duplicates on the build side
    bvalid = (rng.random(nb) > 0.05).astype(np.uint8)
    pkeys, pvalid = fk_column(np.unique(bkeys).astype(np.int64), npr, 0.9, 0.25, 0.03, rng)
    pvalid = np.ones(npr, np.uint8) if pvalid is None else pvalid
    return bkeys, bvalid, pkeys.astype(np.int32), pvalid


def pairs_from_execute(ctx, bkeys, bvalid, pkeys, pvalid):
    """The regular entry point: a 2-table plan whose outputs are the row
    numbers of the matching build and probe rows."""
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
    r, _ = run_product(plan, ctx)
    from calamarijoins_b200 import Column, decode_column
    b, _ = decode_column(Column(I, r.pages[0]))
    p, _ = decode_column(Column(I, r.pages[1]))
    return np.stack([b, p], axis=1).astype(np.int64)


def bitmap(valid):
    n = len(valid)
    bits = np.packbits(valid.astype(np.uint8), bitorder="little")
    words = np.zeros(((n + 31) // 32) * 4, np.uint8)
    words[:len(bits)] = bits
    return torch.from_numpy(words.view(np.int32).copy()).cuda()


def pairs_from_noalloc(bkeys, bvalid, pkeys, pvalid, capacity):
    lib = _lib.lib()
    bk = torch.from_numpy(bkeys).cuda()
    pk = torch.from_numpy(pkeys).cuda()
    bv, pv = bitmap(bvalid), bitmap(pvalid)
    ob = torch.full((capacity,), -1, dtype=torch.int32, device="cuda")
    op = torch.full((capacity,), -1, dtype=torch.int32, device="cuda")
    dc = torch.zeros(1, dtype=torch.int64, device="cuda")
    hc = C.c_uint64(0)
    torch.cuda.synchronize()
    rc = lib.cj_hash_join_noalloc(bk.data_ptr(), bv.data_ptr(), len(bkeys), pk.data_ptr(), pv.data_ptr(),
                                  len(pkeys), ob.data_ptr(), op.data_ptr(), capacity, dc.data_ptr(), C.byref(hc),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.cj_last_error()
    n = hc.value
    assert n == int(dc.item())
    assert n <= capacity
    return np.stack([ob[:n].cpu().numpy(), op[:n].cpu().numpy()], axis=1).astype(np.int64)


def sorted_pairs(a):
    return a[np.lexsort((a[:, 1], a[:, 0]))]


def test_noalloc_matches_execute_twice(gpu_ctx):
    # two calls in a row, the second larger than the first: the shared
    # scratch array keeps the first call's contents and must not leak into
    # the second result
    for seed, nb, npr in ((1, 5_000, 100_000), (2, 200_000, 400_000)):
        bkeys, bvalid, pkeys, pvalid = make_tables(seed, nb, npr)
        want = sorted_pairs(pairs_from_execute(gpu_ctx, bkeys, bvalid, pkeys, pvalid))
        got = sorted_pairs(pairs_from_noalloc(bkeys, bvalid, pkeys, pvalid, capacity=len(want) + 1000))
        assert got.shape == want.shape
        assert np.array_equal(got, want)


def test_noalloc_rejects_oversized_build():
    lib = _lib.lib()
    dc = torch.zeros(1, dtype=torch.int64, device="cuda")
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = lib.cj_hash_join_noalloc(dummy.data_ptr(), dummy.data_ptr(), (1 << 18) + 1, dummy.data_ptr(),
                                  dummy.data_ptr(), 4, dummy.data_ptr(), dummy.data_ptr(), 4, dc.data_ptr(), None,
                                  None)
    assert rc == 7  # CJ_ERR_LIMIT
    assert b"262144" in lib.cj_last_error()
