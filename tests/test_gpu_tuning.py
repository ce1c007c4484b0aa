"""GPU: the autotuner. It times the hash build and probe per size class,
keeps the fastest launch parameters in the context and a file; a context
created with CJ_TUNING_FILE loads them; results stay those of the oracle
whatever was chosen."""
import os

import pytest

from calamarijoins_b200 import Context
from calamarijoins_b200.datagen import join2
from tests.helpers import assert_same, run_oracle, run_product

pytestmark = pytest.mark.gpu


def test_autotune_then_load(tmp_path):
    path = str(tmp_path / "tuning.txt")
    ctx = Context(0)
    try:
        assert ctx.tuning() == [(0, 0, 0)] * 6
        ctx.autotune(path, quick=True)
        table = ctx.tuning()
        assert all(spp in range(9, 14) and pc in (2, 4, 8) and qc in (2, 4, 6, 8) for spp, pc, qc in table), table
        assert os.path.exists(path)
        plans = [join2(nb, npr, seed=nb, unique_build=False, zipf=0.6, probe_null=0.03)
                 for nb, npr in ((3_000, 40_000), (40_000, 300_000), (300_000, 1_200_000))]
        for p in plans:
            got, _ = run_product(p, ctx)
            assert_same(got, run_oracle(p))
    finally:
        ctx.close()
    os.environ["CJ_TUNING_FILE"] = path
    try:
        ctx2 = Context(0)
        try:
            assert ctx2.tuning() == table
        finally:
            ctx2.close()
    finally:
        del os.environ["CJ_TUNING_FILE"]
