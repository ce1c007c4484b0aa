"""CPU: pins the oracle (and, where built, the reference's own execute())
against the 21 known-answer cases of the reference's unit tests, and
cross-checks the product's page encoder against the oracle's."""
import os
import re

import numpy as np
import pytest

from calamarijoins_b200 import DataType, PlanDescriptor, decode_column, encode_column
from oracle import oracle_api as oa
from tests.helpers import check_expect, load_unit_cases, plan_from_case

CASES = load_unit_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_unit_case(case):
    r = oa.oracle_execute(PlanDescriptor(plan_from_case(case)))
    check_expect(r, case["expect"], case["name"])


@pytest.mark.skipif(not oa.ref_available(), reason="reference not compiled (oracle/build_oracle.py)")
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_reference_unit_case(case):
    """The reference itself passes its own known answers through the bridge,
    and agrees with the oracle row for row."""
    d = PlanDescriptor(plan_from_case(case))
    r, _, _ = oa.ref_execute(d, oa.ref_available()[0])
    check_expect(r, case["expect"], case["name"])
    o = oa.oracle_execute(d)
    ok, msg = oa.tables_equal(o, r)
    assert ok, msg


def test_golden_fixture_is_current(tmp_path):
    """unit_cases.json is exactly what its generator writes today: run the
    generator into a scratch directory and compare the two files' data."""
    import json
    import shutil
    import subprocess
    import sys
    here = os.path.join(os.path.dirname(__file__), "golden")
    gen = tmp_path / "make_unit_cases.py"
    shutil.copy(os.path.join(here, "make_unit_cases.py"), gen)
    subprocess.run([sys.executable, str(gen)], check=True, capture_output=True, cwd=tmp_path)
    with open(tmp_path / "unit_cases.json") as f:
        fresh = json.load(f)
    with open(os.path.join(here, "unit_cases.json")) as f:
        current = json.load(f)
    assert len(current["cases"]) == 21
    assert fresh == current


@pytest.mark.parametrize("dtype", [DataType.INT32, DataType.INT64, DataType.FP64])
@pytest.mark.parametrize("null_frac", [0.0, 0.3, 1.0])
def test_encoder_matches_oracle_fixed(dtype, null_frac):
    rng = np.random.default_rng(7)
    n = 5000
    vals = {DataType.INT32: rng.integers(-100, 100, n, dtype=np.int32),
            DataType.INT64: rng.integers(-(2 ** 40), 2 ** 40, n, dtype=np.int64),
            DataType.FP64: rng.standard_normal(n)}[dtype]
    valid = (rng.random(n) >= null_frac).astype(np.uint8)
    prod = encode_column(dtype, vals, valid).pages
    ora = oa.encode(int(dtype), vals, valid)
    assert prod.shape == ora.shape  # same page breaks (ColumnInserter packing)
    r1 = oa.PagedResult(n, [int(dtype)], [prod])
    r2 = oa.PagedResult(n, [int(dtype)], [ora])
    assert oa.validate(r1)[0]
    assert oa.tables_equal(r1, r2)[0]
    dv, dm = decode_column(encode_column(dtype, vals, valid))
    assert np.array_equal(dm, valid.astype(bool))
    assert np.array_equal(dv[dm].view(np.uint8), vals[valid.astype(bool)].view(np.uint8))


@pytest.mark.parametrize("long_frac", [0.0, 0.05])
def test_encoder_matches_oracle_varchar(long_frac):
    from calamarijoins_b200.datagen import varchar_values
    rng = np.random.default_rng(3)
    n = 3000
    chars, offs = varchar_values(n, rng, long_frac=long_frac)
    valid = (rng.random(n) > 0.2).astype(np.uint8)
    prod = encode_column(DataType.VARCHAR, (chars, offs), valid).pages
    ora = oa.encode(int(DataType.VARCHAR), chars, valid, offs)
    assert prod.shape == ora.shape
    r1 = oa.PagedResult(n, [3], [prod])
    r2 = oa.PagedResult(n, [3], [ora])
    assert oa.validate(r1)[0]
    assert oa.tables_equal(r1, r2)[0]


def test_empty_and_edge_strings():
    vals = ["", "a", None, "x" * 8185, "y" * 8186, "", None, "z" * 20000]
    col = encode_column(DataType.VARCHAR, vals)
    dec, valid = decode_column(col)
    want = [None if v is None else v.encode() for v in vals]
    assert dec == want
    r = oa.PagedResult(len(vals), [3], [col.pages])
    assert oa.validate(r)[0]


def _ref_bloom():
    from oracle.build_oracle import reference_dir
    ref = reference_dir()
    return os.path.join(ref, "include", "join_execution", "bloom_tags.h") if ref else ""


REF_BLOOM = _ref_bloom()


@pytest.mark.skipif(not os.path.exists(REF_BLOOM), reason="reference tree not present")
def test_bloom_tags_regenerated():
    """The 2048 Bloom tags are the ascending 16-bit values with popcount 5
    (the rule the oracle and the library regenerate them by); read the
    reference's table as text and compare."""
    txt = open(REF_BLOOM).read()
    body = txt[txt.index("BLOOM_TAGS[2048]"):]
    vals = [int(x, 16) for x in re.findall(r"0x[0-9a-fA-F]{4}", body)][:2048]
    gen = [v for v in range(65536) if bin(v).count("1") == 5][:2048]
    assert vals == gen
