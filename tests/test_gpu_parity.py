"""GPU parity: the sm_100a path through the C ABI against the oracle and the
reference's known answers. Bit-exact: every output table must be the same
row multiset (values, NULLs, VARCHAR bytes, FP64 bit patterns) as the
oracle's, and every output page must be well formed."""
import numpy as np
import pytest

from calamarijoins_b200 import (CJError, Column, ColumnarTable, DataType, Plan, PlanDescriptor, ResidentTable, Table,
                                encode_column, execute_raw)
from calamarijoins_b200 import _lib
from calamarijoins_b200.datagen import chain_plan, config_c1, config_c3, join2
from oracle import oracle_api as oa
from tests.helpers import assert_same, check_expect, load_unit_cases, plan_from_case, run_oracle, run_product

pytestmark = pytest.mark.gpu

I, L, F, V = DataType.INT32, DataType.INT64, DataType.FP64, DataType.VARCHAR
CASES = load_unit_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_unit_case(gpu_ctx, case):
    plan = plan_from_case(case)
    r, _ = run_product(plan, gpu_ctx)
    check_expect(r, case["expect"], case["name"])
    assert_same(r, run_oracle(plan), case["name"])


@pytest.mark.parametrize("nl_max", [0, 7, 64])
def test_unit_cases_any_threshold(gpu_ctx, nl_max):
    """Results do not depend on the nested-loop threshold."""
    gpu_ctx.set_option(_lib.CJ_OPT_NESTED_LOOP_MAX_BUILD, nl_max)
    try:
        for case in CASES:
            plan = plan_from_case(case)
            r, _ = run_product(plan, gpu_ctx)
            check_expect(r, case["expect"], case["name"])
    finally:
        gpu_ctx.set_option(_lib.CJ_OPT_NESTED_LOOP_MAX_BUILD, 64)


JOIN_CASES = [
    # n_build, n_probe, kwargs
    (1, 1000, dict()),
    (5, 3000, dict(build_null=0.2, probe_null=0.1)),
    (64, 20000, dict(zipf=1.2)),
    (65, 20000, dict(zipf=1.2)),
    (1000, 50000, dict(outside=0.3, probe_null=0.05)),
    (2047, 4096, dict(zipf=0.0)),
    (2049, 4096, dict(zipf=0.0)),
    (100_000, 1_000_000, dict(zipf=1.0, probe_null=0.05)),
    (300_000, 200_000, dict(zipf=0.8)),  # build larger than probe: sides swap
    (50_000, 400_000, dict(key_type=L, zipf=0.9, outside=0.2)),
    (20_000, 100_000, dict(unique_build=False, zipf=0.5)),  # many-to-many
    (3000, 30000, dict(build_payload=(I, L, F, V), probe_payload=(V, F), probe_null=0.1)),
]


@pytest.mark.parametrize("nb,npr,kw", JOIN_CASES, ids=[f"{a}x{b}-{i}" for i, (a, b, _) in enumerate(JOIN_CASES)])
@pytest.mark.parametrize("build_left", [True, False])
def test_join_parity(gpu_ctx, nb, npr, kw, build_left):
    plan = join2(nb, npr, seed=nb * 7 + npr, build_left=build_left, **kw)
    r, st = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), f"{nb}x{npr}")
    assert st.exec["kernel_launches"] > 0


@pytest.mark.parametrize("output", [[0], [3], [1, 2], [2, 0], []])
def test_projection_modes(gpu_ctx, output):
    """Build-only, probe-only and empty projections (collection modes,
    join_setup.h:146-173)."""
    plan = join2(5000, 40000, seed=11, zipf=1.0, build_payload=(I,), probe_payload=(F,), output=output,
                 probe_null=0.1)
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan))


def test_many_to_many_rerun(gpu_ctx):
    """Duplicate build keys: the first probe overflows its capacity guess and
    is re-run with the exact size."""
    plan = join2(4000, 6000, seed=5, unique_build=False, zipf=0.0)
    r, st = run_product(plan, gpu_ctx)
    assert st.exec["probe_reruns"] >= 1
    assert_same(r, run_oracle(plan))


def test_varchar_nulls_and_long_strings(gpu_ctx):
    plan = join2(4000, 30000, seed=9, build_payload=(V,), probe_payload=(V, I), probe_null=0.05,
                 varchar_kw=dict(long_frac=0.01))
    # NULLs inside the VARCHAR payloads too
    rng = np.random.default_rng(1)
    from calamarijoins_b200.datagen import varchar_values
    chars, offs = varchar_values(30000, rng, long_frac=0.005)
    valid = (rng.random(30000) > 0.3).astype(np.uint8)
    plan.inputs[1].columns[1] = encode_column(V, (chars, offs), valid)
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_chain_plans(gpu_ctx, seed):
    rng = np.random.default_rng(seed)
    ways = 2 + seed
    plan = chain_plan(ways, 20000, rng, max_build=50000, varchar_frac=0.5,
                      key_types=[I if (seed + d) % 2 else L for d in range(ways - 1)])
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), f"chain {seed}")


@pytest.mark.parametrize("varchar_nulls", [False, True])
def test_c3_pipeline_small(gpu_ctx, varchar_nulls):
    plan = config_c3(seed=33, scale=0.002, varchar_nulls=varchar_nulls, long_frac=0.002)
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), "c3")


def test_c1_full(gpu_ctx):
    plan = config_c1()
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), "c1")


def test_empty_inputs(gpu_ctx):
    plan = join2(10, 10, seed=1)
    plan.inputs[0] = ColumnarTable(0, [encode_column(I, np.zeros(0, np.int32)),
                                       encode_column(I, np.zeros(0, np.int32))])
    r, _ = run_product(plan, gpu_ctx)
    assert r.num_rows == 0 and r.types == [0, 0, 0, 1]
    assert all(p.shape[0] == 0 for p in r.pages)


def test_all_null_probe(gpu_ctx):
    plan = join2(100, 5000, seed=2, probe_null=1.0)
    r, _ = run_product(plan, gpu_ctx)
    assert r.num_rows == 0


def test_int32_min_through_intermediate(gpu_ctx):
    """INT32_MIN leaving a non-root join reads as NULL afterwards (value_t,
    intermediate.h:56-62): as an output value and as a key."""
    imin = -(2 ** 31)
    plan = Plan()
    a = Table([[1, imin], [2, 5], [3, imin]], [I, I]).to_columnar()
    b = Table([[1], [2], [3]], [I]).to_columnar()
    c = Table([[imin], [5], [7]], [I]).to_columnar()
    plan.inputs += [a, b, c]
    plan.new_scan_node(0, [(0, I), (1, I)])
    plan.new_scan_node(1, [(0, I)])
    plan.new_scan_node(2, [(0, I)])
    j = plan.new_join_node(True, 1, 0, 0, 0, [(0, I), (2, I)])  # (key, a.payload)
    plan.new_join_node(True, j, 2, 1, 0, [(0, I), (1, I), (2, I)])  # join on a.payload
    plan.root = 4
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan))
    assert r.num_rows == 1  # only payload 5 matches; INT32_MIN became NULL
    plan.root = j
    r2, _ = run_product(plan, gpu_ctx)
    assert_same(r2, run_oracle(plan))  # at the root it is still a value


def test_build_key_output_read_from_probe_side(gpu_ctx):
    """An output of the build key is read through the probe side's row ids
    (the two keys are equal on every output row): at the root and below it,
    with NULL and INT32_MIN keys, with an intermediate probe side, and with a
    build side that contributes nothing but its key (no build row ids)."""
    imin = -(2 ** 31)
    rng = np.random.default_rng(11)
    nb, npr = 3000, 40000
    bk = rng.integers(-50, 2000, nb).astype(np.int32)
    bk[:7] = imin
    pk = rng.integers(-60, 2100, npr).astype(np.int32)
    pk[::97] = imin
    bv = (rng.random(nb) > 0.1).astype(np.uint8)
    pv = (rng.random(npr) > 0.1).astype(np.uint8)
    pay = rng.integers(0, 1 << 40, npr).astype(np.int64)
    plan = Plan()
    plan.inputs.append(ColumnarTable(nb, [encode_column(I, bk, bv), encode_column(F, rng.random(nb))]))
    plan.inputs.append(ColumnarTable(npr, [encode_column(I, pk, pv), encode_column(L, pay)]))
    plan.inputs.append(ColumnarTable(500, [encode_column(I, rng.integers(-60, 2100, 500).astype(np.int32))]))
    s0 = plan.new_scan_node(0, [(0, I), (1, F)])
    s1 = plan.new_scan_node(1, [(0, I), (1, L)])
    s2 = plan.new_scan_node(2, [(0, I)])
    # root projects only the build key and probe payload: no build row ids
    plan.new_join_node(True, s0, s1, 0, 0, [(0, I), (3, L)])
    plan.root = 3
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), "key only")
    # both keys and a build payload at the root
    plan.nodes[3].output_attrs = [(0, I), (1, F), (2, I), (3, L)]
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), "keys and payloads")
    # below the root: the projected build key feeds the next join's key and
    # the root's output; the next join's probe side is that intermediate
    j = plan.new_join_node(True, s0, s1, 0, 0, [(0, I), (3, L)])
    plan.new_join_node(True, s2, j, 0, 0, [(0, I), (1, I), (2, L)])
    plan.root = 5
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), "through an intermediate")


def _direct_case(kind, rng):
    """Build keys for the direct-mapped table cases."""
    if kind == "dense_i32":
        return rng.permutation(50_000).astype(np.int64) - 20_000, I
    if kind == "dense_i64":
        return rng.permutation(50_000).astype(np.int64) + (1 << 40), L
    if kind == "dense_dups":  # dense range, one key repeated: falls back to the hash table
        k = rng.permutation(50_000).astype(np.int64)
        k[123] = k[4567]
        return k, I
    if kind == "spread5":  # span about 5 x rows: direct at factor 8, hash at 2
        return rng.choice(250_000, 50_000, replace=False).astype(np.int64), I
    if kind == "sparse":  # span far above 8 x rows: hash table
        return rng.choice(1 << 30, 50_000, replace=False).astype(np.int64), I
    if kind == "extremes":  # INT32_MIN and INT32_MAX as keys: span 2^32
        k = rng.permutation(50_000).astype(np.int64)
        k[0], k[1] = -(2 ** 31), 2 ** 31 - 1
        return k, I
    raise ValueError(kind)


@pytest.mark.parametrize("kind,direct2,direct8,open2,open8", [
    ("dense_i32", 1, 1, 0, 0), ("dense_i64", 1, 1, 0, 0), ("dense_dups", 0, 0, 0, 0), ("spread5", 0, 1, 1, 0),
    ("sparse", 0, 0, 1, 1), ("extremes", 0, 0, 1, 1)])
def test_direct_mapped_build(gpu_ctx, kind, direct2, direct8, open2, open8):
    """Unique build keys spread over at most CJ_OPT_DENSE_KEYS times the
    build rows take a direct-mapped table; duplicates, wider spans and the
    option turned off take the hash table. Every path gives the oracle's
    result."""
    rng = np.random.default_rng(5)
    bkeys, kt = _direct_case(kind, rng)
    nb, npr = len(bkeys), 300_000
    pick = rng.integers(0, nb, npr)
    pkeys = bkeys[pick].copy()
    miss = rng.random(npr) < 0.3
    pkeys[miss] = rng.integers(bkeys.min() - 1000, bkeys.max() + 1000, int(miss.sum()))
    bv = (rng.random(nb) > 0.05).astype(np.uint8)
    bv[[0, 1, 123, 4567]] = 1  # the repeated and the extreme keys are not NULL
    pv = (rng.random(npr) > 0.02).astype(np.uint8)
    plan = Plan()
    npt = np.int32 if kt == I else np.int64
    if kt == I:
        pkeys = np.clip(pkeys, -(2 ** 31), 2 ** 31 - 1)
    plan.inputs.append(ColumnarTable(nb, [encode_column(kt, bkeys.astype(npt), bv),
                                          encode_column(L, rng.integers(0, 1 << 50, nb))]))
    plan.inputs.append(ColumnarTable(npr, [encode_column(kt, pkeys.astype(npt), pv),
                                           encode_column(F, rng.random(npr))]))
    plan.new_scan_node(0, [(0, kt), (1, L)])
    plan.new_scan_node(1, [(0, kt), (1, F)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, kt), (1, L), (2, kt), (3, F)])
    plan.root = 2
    want = run_oracle(plan)
    default = gpu_ctx.get_option(_lib.CJ_OPT_DENSE_KEYS)
    assert default == 8
    try:
        for opt, expect, expect_open in ((2, direct2, open2), (8, direct8, open8), (0, 0, 0)):
            gpu_ctx.set_option(_lib.CJ_OPT_DENSE_KEYS, opt)
            r, st = run_product(plan, gpu_ctx)
            assert_same(r, want, f"{kind} dense_keys={opt}")
            assert st.exec["num_direct_joins"] == expect
            assert st.exec["num_open_joins"] == expect_open
            assert st.exec["num_hash_joins"] == 1
    finally:
        gpu_ctx.set_option(_lib.CJ_OPT_DENSE_KEYS, default)


@pytest.mark.parametrize("case", ["unique", "dups", "nulls", "negative", "many_probe_misses", "int64_keys"])
def test_open_addressing_table(gpu_ctx, case):
    """Unique INT32 build keys spread far wider than the direct-mapped table
    allows take the open-addressing table; a repeated key, or INT64 build
    keys, go on to the hash table. Every case gives the oracle's result."""
    rng = np.random.default_rng(31)
    nb, npr = 200_000, 1_000_000
    kt = L if case == "int64_keys" else I
    if case == "negative":
        bkeys = -rng.choice(1 << 30, nb, replace=False).astype(np.int64)
    elif case == "int64_keys":
        bkeys = rng.choice(1 << 40, nb, replace=False).astype(np.int64) << 3
    else:
        bkeys = rng.choice(1 << 30, nb, replace=False).astype(np.int64) * 2
    if case == "dups":
        bkeys[rng.integers(0, nb, 50)] = bkeys[7]
    bv = (rng.random(nb) > 0.1).astype(np.uint8) if case == "nulls" else None
    pkeys = bkeys[rng.integers(0, nb, npr)]
    miss = rng.random(npr) < (0.9 if case == "many_probe_misses" else 0.25)
    pkeys[miss] = pkeys[miss] + 1  # odd (or shifted) keys: never a build key
    npt = np.int32 if kt == I else np.int64
    plan = Plan()
    plan.inputs.append(ColumnarTable(nb, [encode_column(kt, bkeys.astype(npt), bv),
                                          encode_column(I, rng.integers(0, 1000, nb).astype(np.int32))]))
    plan.inputs.append(ColumnarTable(npr, [encode_column(kt, pkeys.astype(npt), (rng.random(npr) > 0.02).astype(np.uint8)),
                                           encode_column(F, rng.random(npr))]))
    plan.new_scan_node(0, [(0, kt), (1, I)])
    plan.new_scan_node(1, [(0, kt), (1, F)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, kt), (1, I), (3, F)])
    plan.root = 2
    r, st = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan), case)
    assert st.exec["num_direct_joins"] == 0
    assert st.exec["num_open_joins"] == (0 if case in ("dups", "int64_keys") else 1)
    assert st.exec["num_hash_joins"] == 1


def test_direct_mapped_all_null_build(gpu_ctx):
    rng = np.random.default_rng(6)
    nb, npr = 1000, 20_000
    plan = Plan()
    plan.inputs.append(ColumnarTable(nb, [encode_column(I, np.arange(nb, dtype=np.int32), np.zeros(nb, np.uint8))]))
    plan.inputs.append(ColumnarTable(npr, [encode_column(I, rng.integers(0, nb, npr).astype(np.int32))]))
    plan.new_scan_node(0, [(0, I)])
    plan.new_scan_node(1, [(0, I)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, I), (1, I)])
    plan.root = 2
    r, st = run_product(plan, gpu_ctx)
    assert r.num_rows == 0
    assert_same(r, run_oracle(plan))
    assert st.exec["num_direct_joins"] == 1


def test_scan_root_pages_byte_identical(gpu_ctx):
    """A scan root writes its rows in order. For NULL-free columns (pages
    stored straight from registers) its pages are the input pages byte for
    byte: both hold 1984 / 1007 rows per page, ColumnInserter's fill. With
    NULLs the writer keeps that fixed fill (compacting each page's values in
    shared memory), where ColumnInserter packs more rows into a page; those
    columns must hold the same rows, in ceil(n / R) well-formed pages,
    including a column that mixes NULL-free pages with pages holding NULLs."""
    rng = np.random.default_rng(12)
    n = 50_000
    mixed = np.ones(n, np.uint8)
    mixed[20_000:21_000] = rng.random(1000) > 0.5  # NULLs on a few pages only
    cols = [
        encode_column(I, rng.integers(-(2 ** 31), 2 ** 31, n).astype(np.int32)),
        encode_column(L, rng.integers(-(1 << 62), 1 << 62, n)),
        encode_column(F, rng.standard_normal(n)),
        encode_column(I, rng.integers(0, 100, n).astype(np.int32), (rng.random(n) > 0.1).astype(np.uint8)),
        encode_column(F, rng.standard_normal(n), (rng.random(n) > 0.3).astype(np.uint8)),
        encode_column(L, rng.integers(0, 1 << 40, n), mixed),
    ]
    types = [I, L, F, I, F, L]
    plan = Plan()
    plan.inputs.append(ColumnarTable(n, cols))
    plan.new_scan_node(0, [(i, t) for i, t in enumerate(types)])
    plan.root = 0
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan))
    for c, col in enumerate(cols[:3]):
        assert r.pages[c].shape == col.pages.shape, c
        assert np.array_equal(r.pages[c], col.pages), f"column {c}: pages differ"
    for c in range(3, 6):
        R = 1984 if types[c] == I else 1007
        assert r.pages[c].shape[0] == (n + R - 1) // R


def test_scan_root(gpu_ctx):
    plan = join2(1000, 10, seed=3, build_payload=(V, F))
    plan.root = 0
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, run_oracle(plan))
    assert r.num_rows == 1000


def test_resident_tables(gpu_ctx):
    plan = join2(20000, 100000, seed=4, build_payload=(L,), probe_payload=(V,), probe_null=0.1)
    want = run_oracle(plan)
    res_plan = Plan()
    res_plan.nodes = plan.nodes
    res_plan.root = plan.root
    res_plan.inputs = [ResidentTable(gpu_ctx, t) for t in plan.inputs]
    for _ in range(2):
        r, st = run_product(res_plan, gpu_ctx)
        assert_same(r, want)
        assert st.exec["h2d_bytes"] == 0


def test_result_on_device(gpu_ctx):
    plan = join2(5000, 20000, seed=6)
    res, _ = execute_raw(plan, gpu_ctx, _lib.CJ_EXEC_RESULT_ON_DEVICE)
    try:
        assert res.column_info(0)[2] is None  # no host copy
        r = oa.PagedResult.from_result(res)
    finally:
        res.free()
    assert_same(r, run_oracle(plan))


@pytest.mark.parametrize("case", ["direct", "empty", "varchar", "dups", "probe_side_only"])
def test_device_counted_result(gpu_ctx, case):
    """A root over unique build keys whose result stays in HBM is written
    with the match count read on the device (result sized for the probe
    rows): one host synchronisation in the whole execution. A VARCHAR output
    or a table the device refuses (a repeated key) takes the counted path.
    Both give the oracle's result, with host and with device results."""
    kw = dict(build_payload=(L, F), probe_payload=(F, I), outside=0.3, probe_null=0.05)
    if case == "empty":
        kw["outside"] = 1.0
    if case == "varchar":
        kw["probe_payload"] = (F, V)
    if case == "dups":
        kw["unique_build"] = False
    if case == "probe_side_only":
        kw["output"] = [3, 4]  # probe key and probe FP64: no build row ids
    plan = join2(40_000, 250_000, seed=17, **kw)
    want = run_oracle(plan)
    if case == "empty":
        assert want.num_rows == 0
    for flags in (0, _lib.CJ_EXEC_RESULT_ON_DEVICE):
        got, st = run_product(plan, gpu_ctx, flags)
        assert_same(got, want, f"{case} flags={flags}")
        assert st.exec["output_rows"] == want.num_rows
        deferred = flags and case in ("direct", "empty", "probe_side_only")
        assert st.exec["num_direct_joins"] == (0 if case == "dups" else 1)
        if deferred:
            assert st.exec["host_syncs"] == 1
        else:
            assert st.exec["host_syncs"] >= 2


def test_malformed_pages_rejected(gpu_ctx):
    plan = join2(3000, 3000, seed=7)
    bad = plan.inputs[1].columns[0].pages.copy()
    bad[0, 2:4] = np.frombuffer(np.uint16(9000).tobytes(), np.uint8)  # n_values > n_rows
    plan.inputs[1].columns[0].pages = bad
    with pytest.raises(CJError) as e:
        run_product(plan, gpu_ctx)
    assert e.value.status == 3
    ok = join2(300, 3000, seed=8)  # context still usable
    r, _ = run_product(ok, gpu_ctx)
    assert_same(r, run_oracle(ok))


def test_row_count_mismatch_rejected(gpu_ctx):
    # fewer and more rows declared than the pages hold, on the probe side and
    # on the (NULL-free, full-page) build side, whose columns would otherwise
    # be read in place from their pages
    # (the 1.2M-row probe side has 605 INT32 pages: the page index spans
    # several blocks and the last one to finish checks the total)
    for side, delta, npr in ((1, -1, 5000), (1, 1, 5000), (0, 1, 5000), (0, 1000, 5000), (1, -1, 1_200_000),
                             (1, 1984, 1_200_000)):
        plan = join2(3000, npr, seed=7, build_payload=(L,), probe_payload=(F,))
        plan.inputs[side].num_rows += delta
        with pytest.raises(CJError) as e:
            run_product(plan, gpu_ctx)
        assert e.value.status == 3
    r, _ = run_product(join2(300, 500, seed=8), gpu_ctx)  # the context still works
    assert r.num_rows > 0


def _chunked(dtype, values, chunk):
    """A column written by a producer that starts a new page every `chunk`
    rows: every page but the last partial, unlike ColumnInserter's fill."""
    parts = [encode_column(dtype, values[i:i + chunk]) for i in range(0, len(values), chunk)]
    return Column(dtype, np.ascontiguousarray(np.concatenate([c.pages for c in parts])))


def test_partial_pages_are_decoded(gpu_ctx):
    """NULL-free fixed-width columns are read in place from their pages only
    when every page but the last holds the full 1984 / 1007 rows; columns of
    partial pages take the decode path. Both agree with the oracle."""
    rng = np.random.default_rng(9)
    nb, npr = 20_000, 200_000
    bk = rng.permutation(nb).astype(np.int32)
    pk = rng.integers(0, nb + 5000, npr).astype(np.int32)
    bp = rng.integers(-(1 << 60), 1 << 60, nb)
    pp = rng.random(npr)
    for chunk in (None, 1000, 1983):
        enc = (lambda t, v: encode_column(t, v)) if chunk is None else (lambda t, v, c=chunk: _chunked(t, v, c))
        plan = Plan()
        plan.inputs.append(ColumnarTable(nb, [enc(I, bk), enc(L, bp)]))
        plan.inputs.append(ColumnarTable(npr, [enc(I, pk), enc(F, pp)]))
        plan.new_scan_node(0, [(0, I), (1, L)])
        plan.new_scan_node(1, [(0, I), (1, F)])
        plan.new_join_node(True, 0, 1, 0, 0, [(0, I), (1, L), (2, I), (3, F)])
        plan.root = 2
        r, _ = run_product(plan, gpu_ctx)
        assert_same(r, run_oracle(plan), f"chunk={chunk}")


def test_invalid_plans(gpu_ctx):
    plan = join2(30, 30, seed=1)
    plan.nodes[2].output_attrs[0] = (0, DataType.FP64)  # wrong declared type
    with pytest.raises(CJError) as e:
        run_product(plan, gpu_ctx)
    assert e.value.status == 2
    plan = join2(30, 30, seed=1, build_payload=(F,), probe_payload=(F,))
    plan.nodes[2].data.left_attr = 1  # FP64 key
    with pytest.raises(CJError) as e:
        run_product(plan, gpu_ctx)
    assert e.value.status == 6


def test_buffer_cache_reuse_and_trim(gpu_ctx):
    """Buffers freed by one plan serve the next (no growth over repeated
    plans, same results); turning the cache off hands them back to the
    pool."""
    plan = join2(50_000, 400_000, seed=13, build_payload=(L, V), probe_payload=(F,))
    want = run_oracle(plan)
    r, _ = run_product(plan, gpu_ctx)
    assert_same(r, want)
    used1, _ = gpu_ctx.memory()
    for _ in range(3):
        r, _ = run_product(plan, gpu_ctx)
        assert_same(r, want)
    used2, _ = gpu_ctx.memory()
    assert used2 == used1
    default = gpu_ctx.get_option(_lib.CJ_OPT_BUFFER_CACHE_BYTES)
    try:
        gpu_ctx.set_option(_lib.CJ_OPT_BUFFER_CACHE_BYTES, 0)
        used3, _ = gpu_ctx.memory()
        assert used3 < used2
        r, _ = run_product(plan, gpu_ctx)
        assert_same(r, want)
        used4, _ = gpu_ctx.memory()
        assert used4 <= used3
    finally:
        gpu_ctx.set_option(_lib.CJ_OPT_BUFFER_CACHE_BYTES, default)


def test_memory_returns_to_pool(gpu_ctx):
    plan = join2(10000, 100000, seed=12, build_payload=(V,))
    run_product(plan, gpu_ctx)
    used1, _ = gpu_ctx.memory()
    for _ in range(3):
        run_product(plan, gpu_ctx)
    used2, _ = gpu_ctx.memory()
    assert used2 <= used1


@pytest.mark.parametrize("spp", [64, 2048, 16384])
def test_radix_passes_any_partition_size(gpu_ctx, spp):
    """Directory slots per partition 64 (2^13 partitions for 2^19 slots: two
    radix passes), 2048 (one pass) and 16384: the same results."""
    gpu_ctx.set_option(_lib.CJ_OPT_SLOTS_PER_PARTITION, spp)
    gpu_ctx.set_option(_lib.CJ_OPT_DENSE_KEYS, 0)
    try:
        for plan in (join2(300_000, 1_000_000, seed=41, unique_build=False, zipf=0.7, probe_null=0.05),
                     join2(300_000, 900_000, seed=42, key_type=L, zipf=0.9, outside=0.2)):
            r, st = run_product(plan, gpu_ctx)
            assert_same(r, run_oracle(plan), f"spp {spp}")
    finally:
        gpu_ctx.set_option(_lib.CJ_OPT_SLOTS_PER_PARTITION, 0)
        gpu_ctx.set_option(_lib.CJ_OPT_DENSE_KEYS, 8)


@pytest.mark.parametrize("key_type", [I, L])
def test_heavy_slots_written_by_the_warp(gpu_ctx, key_type):
    """Slots longer than 64 tuples are counted and written by the whole
    warp: a key repeated 5,000 times on the build side (and a second one 70
    times, just past the limit) against probe rows holding them, alone and
    inside a batch."""
    from calamarijoins_b200 import execute_batch
    rng = np.random.default_rng(66)
    nb, npr = 20_000, 60_000
    bk = rng.permutation(nb).astype(np.int64) + 100
    bk[:5000] = 7
    bk[5000:5070] = 8
    rng.shuffle(bk)
    pk = rng.integers(0, nb + 200, npr)
    pk[rng.choice(npr, 300, replace=False)] = 7
    pk[rng.choice(npr, 300, replace=False)] = 8
    npt = np.int32 if key_type == I else np.int64
    pvalid = (rng.random(npr) > 0.03).astype(np.uint8)
    plan = Plan()
    plan.inputs.append(ColumnarTable(nb, [encode_column(key_type, bk.astype(npt)),
                                          encode_column(I, rng.integers(0, 1 << 30, nb).astype(np.int32))]))
    plan.inputs.append(ColumnarTable(npr, [encode_column(key_type, pk.astype(npt), pvalid),
                                           encode_column(F, rng.standard_normal(npr))]))
    plan.new_scan_node(0, [(0, key_type), (1, I)])
    plan.new_scan_node(1, [(0, key_type), (1, F)])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, key_type), (1, I), (3, F)])
    plan.root = 2
    want = run_oracle(plan)
    assert want.num_rows > 1_000_000
    got, _ = run_product(plan, gpu_ctx)
    assert_same(got, want, "alone")
    res, sts, _ = execute_batch([plan, join2(100, 1000, seed=3)], gpu_ctx)
    got = oa.PagedResult.from_result(res[0])
    for r in res:
        r.free()
    assert_same(got, want, "batched")


@pytest.mark.parametrize("budget", [0, 1 << 40])
def test_hash_directory_layouts(budget):
    """INT32-key hash tables with 8-byte directory entries (budget 0) and
    with the slot's first tuple inline (16-byte entries): the same results."""
    import os
    from calamarijoins_b200 import Context
    os.environ["CJ_INLINE_DIR_MAX_BYTES"] = str(budget)
    try:
        ctx = Context(0)
    finally:
        del os.environ["CJ_INLINE_DIR_MAX_BYTES"]
    try:
        ctx.set_option(_lib.CJ_OPT_DENSE_KEYS, 0)
        for plan in (join2(200_000, 1_000_000, seed=51, unique_build=False, zipf=0.8, probe_null=0.05),
                     join2(300_000, 1_000_000, seed=52, zipf=0.9, outside=0.3),
                     join2(5_000, 100_000, seed=53, unique_build=False, zipf=1.2)):
            got, _ = run_product(plan, ctx)
            assert_same(got, run_oracle(plan), f"budget {budget}")
    finally:
        ctx.close()
