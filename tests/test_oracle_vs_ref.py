"""CPU: the oracle agrees with the reference's own execute() (compiled from
its sources into oracle/_ref) on seeded workloads inside the reference's
valid domain: INT32 keys, INT32 payloads with NULLs, VARCHAR payloads
without NULLs (long strings included), nested-loop and hash paths,
multi-level pipelines."""
import numpy as np
import pytest

from calamarijoins_b200 import DataType, PlanDescriptor
from calamarijoins_b200 import decode_column
from calamarijoins_b200.datagen import chain_plan, config_c2s, config_c3, join2
from oracle import oracle_api as oa

pytestmark = pytest.mark.skipif(not oa.ref_available(), reason="reference not compiled (oracle/build_oracle.py)")

I, V = DataType.INT32, DataType.VARCHAR


def agree(plan):
    d = PlanDescriptor(plan)
    r, _, _ = oa.ref_execute(d, oa.ref_available()[0])
    o = oa.oracle_execute(d)
    ok, msg = oa.tables_equal(o, r)
    assert ok, msg
    return o


@pytest.mark.parametrize("nb,npr,kw", [
    (1, 500, dict()),
    (7, 5000, dict(probe_null=0.2)),
    (8, 5000, dict(build_null=0.3)),
    (3000, 40000, dict(zipf=1.1, outside=0.3, probe_null=0.05)),
    (40000, 30000, dict(zipf=0.5)),
    (5000, 20000, dict(unique_build=False)),
    (2000, 20000, dict(build_payload=(V, I), probe_payload=(V,), varchar_kw=dict(long_frac=0.02))),
])
@pytest.mark.parametrize("build_left", [True, False])
def test_two_table(nb, npr, kw, build_left):
    kw = {"probe_payload": (I,), **kw}  # the reference cannot emit INT64 / FP64 columns
    agree(join2(nb, npr, seed=nb + npr, build_left=build_left, **kw))


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_chains(seed):
    rng = np.random.default_rng(seed)
    agree(chain_plan(2 + seed % 3, 30000, rng, max_build=20000, varchar_frac=0.5))


def test_c3_small():
    o = agree(config_c3(seed=5, scale=0.002, varchar_nulls=False, long_frac=0.002))
    assert o.num_rows > 0


def test_c2s_small():
    """C2s's spread build keys (unique multiples of 500 below 2^31, probe keys
    outside the domain above them) are inside the reference's domain."""
    plan = config_c2s(scale=0.005, int32_standin=True)
    keys, valid = decode_column(plan.inputs[0].columns[0])
    assert len(np.unique(keys)) == len(keys) and (keys % 500 == 0).all() and keys.max() < 2 ** 31
    o = agree(plan)
    assert 0 < o.num_rows < plan.inputs[1].num_rows
