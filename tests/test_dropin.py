"""The drop-in src/execute.cpp replacement (calamarijoins_b200/contest/
execute.cpp), compiled against the reference's own plan.h, runs plans
through Contest::build_context / execute / destroy_context on the GPU and
matches the oracle."""
import os
import struct
import subprocess
import tempfile

import numpy as np
import pytest

from calamarijoins_b200 import DataType, PlanDescriptor, ScanNode
from calamarijoins_b200.datagen import config_c3, join2
from oracle import oracle_api as oa
from tests.helpers import assert_same, load_unit_cases, plan_from_case, run_oracle

HARNESS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dropin", "dropin_harness")


def serialize(plan, path):
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", len(plan.nodes)))
        for n in plan.nodes:
            if isinstance(n.data, ScanNode):
                f.write(struct.pack("<ii5Q", 1, 0, n.data.base_table_id, 0, 0, 0, 0))
            else:
                j = n.data
                f.write(struct.pack("<ii5Q", 0, int(j.build_left), 0, j.left, j.right, j.left_attr, j.right_attr))
            f.write(struct.pack("<Q", len(n.output_attrs)))
            for idx, t in n.output_attrs:
                f.write(struct.pack("<Qi", idx, int(t)))
        f.write(struct.pack("<Q", len(plan.inputs)))
        for t in plan.inputs:
            f.write(struct.pack("<QQ", t.num_rows, len(t.columns)))
            for c in t.columns:
                f.write(struct.pack("<iQ", int(c.type), c.num_pages))
                f.write(c.pages.tobytes())
        f.write(struct.pack("<Q", plan.root))


def read_result(path) -> oa.PagedResult:
    data = open(path, "rb").read()
    rows, ncols = struct.unpack_from("<QQ", data, 0)
    off = 16
    types, pages = [], []
    for _ in range(ncols):
        t, n = struct.unpack_from("<iQ", data, off)
        off += 12
        pages.append(np.frombuffer(data, np.uint8, n * 8192, off).reshape(n, 8192).copy())
        off += n * 8192
        types.append(t)
    return oa.PagedResult(rows, types, pages)


def run_dropin(plan):
    with tempfile.TemporaryDirectory() as d:
        pin, pout = os.path.join(d, "plan.bin"), os.path.join(d, "out.bin")
        serialize(plan, pin)
        res = subprocess.run([HARNESS, pin, pout], capture_output=True, text=True, timeout=300)
        assert res.returncode == 0, res.stderr
        return read_result(pout)


needs_harness = pytest.mark.skipif(not os.path.exists(HARNESS),
                                   reason="drop-in harness not built (needs the reference's headers)")


@pytest.mark.gpu
@needs_harness
def test_dropin_unit_cases():
    for case in load_unit_cases():
        plan = plan_from_case(case)
        assert_same(run_dropin(plan), run_oracle(plan), case["name"])


@pytest.mark.gpu
@needs_harness
def test_dropin_mixed_types_and_pipeline():
    for plan in (join2(20000, 100000, seed=3, build_payload=(DataType.INT64, DataType.VARCHAR),
                       probe_payload=(DataType.FP64,), probe_null=0.1),
                 config_c3(seed=8, scale=0.001, varchar_nulls=True, long_frac=0.003)):
        assert_same(run_dropin(plan), run_oracle(plan))


@needs_harness
def test_dropin_harness_links_the_library():
    out = subprocess.run(["ldd", HARNESS], capture_output=True, text=True).stdout
    assert "libcj_b200.so" in out and "not found" not in out
