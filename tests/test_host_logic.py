"""CPU: host-side logic that needs no GPU.

- The server's footprint estimate (cj_server_estimate), which admission
  compares with the memory budget: it covers the input pages of host
  tables, grows with the tables, counts resident tables' pages as already
  paid for, and rejects plans it cannot walk.
- The benchmark's bookkeeping: whole-job rates over ranks, the algorithmic
  bytes the roofline divides by, and the per-workload DRAM traffic table
  read from profiles/traffic.json."""
import json
import os

import numpy as np
import pytest

from calamarijoins_b200 import CJError, ColumnarTable, DataType, Plan, PlanDescriptor, Server, encode_column
from calamarijoins_b200.datagen import chain_plan, join2

import bench

I = DataType.INT32


def _pages_bytes(plan):
    return sum(c.num_pages * 8192 for t in plan.inputs for c in t.columns)


def test_estimate_covers_input_pages_and_grows():
    small = join2(1_000, 10_000, seed=1)
    big = join2(100_000, 1_000_000, seed=1)
    es, eb = Server.estimate(small), Server.estimate(big)
    assert es >= _pages_bytes(small) and eb >= _pages_bytes(big)
    assert eb > es


def test_estimate_of_deeper_plans_is_larger():
    rng = np.random.default_rng(3)
    two = chain_plan(2, 50_000, rng, max_build=20_000)
    rng = np.random.default_rng(3)
    five = chain_plan(5, 50_000, rng, max_build=20_000)
    assert Server.estimate(five) > Server.estimate(two)


def test_estimate_rejects_plans_it_cannot_walk():
    plan = Plan()
    plan.inputs.append(ColumnarTable(10, [encode_column(I, np.arange(10, dtype=np.int32))]))
    plan.new_scan_node(0, [(0, I)])
    plan.new_scan_node(0, [(0, I)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, I)])
    plan.root = 7  # no such node
    with pytest.raises(CJError):
        Server.estimate(PlanDescriptor(plan))


def test_whole_job_rate():
    assert bench.whole_job_rate(1000, 1, 2.0) == 500.0
    assert bench.whole_job_rate(1000, 4, 2.0) == 2000.0  # every rank processed its own units


def test_algorithmic_bytes_follow_the_workload():
    info = {"build_rows": 4_000_000, "probe_rows": 64_000_000, "slots": 1 << 22,
            "int32_pages": 1000, "int32_cols": 2}
    st = {"matches": 43_900_398, "num_direct_joins": 1}
    wl = bench.WL
    try:
        bench.WL = bench.WORKLOADS["c2"]
        probe = bench.algorithmic_bytes("probe_array", st, info)
        assert probe == pytest.approx(64e6 * (4 + 1 / 8) + 4e6 * 4 + 43_900_398 * 12)
        # a direct-mapped launch that found its table unusable did no work
        assert bench.algorithmic_bytes("probe_array", {**st, "num_direct_joins": 0}, info) is None
        pages = (43_900_398 + 1006) // 1007
        assert bench.algorithmic_bytes("write_pages_8byte", st, info) == pytest.approx(
            43_900_398 * (4 + 8 + 1 / 8) + pages * 8192)
        bench.WL = bench.WORKLOADS["c3"]
        assert bench.algorithmic_bytes("probe_array", st, info) is None  # multi-join: not derived
    finally:
        bench.WL = wl


def test_traffic_table_is_per_workload():
    with open(os.path.join(bench.ROOT, "profiles", "traffic.json")) as f:
        raw = json.load(f)
    for wl in ("c2", "c2h", "c2s"):
        assert bench.traffic_table(wl) == raw[wl]
        for kernel, entry in raw[wl].items():
            assert entry["bytes_per_launch"] > 0
            assert os.path.exists(os.path.join(bench.ROOT, "profiles", entry["source"].split()[0]))
    assert bench.traffic_table("no such workload") == {}
