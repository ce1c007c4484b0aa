"""CPU: the oracle's scan filter (oracle/cj_oracle.c cjo_filter, cjo_like)
pinned against the reference's own column-wise Statement::eval
(src/statement.cpp, include/data_model/inner_column.h, compiled into
oracle/_ref/libcj_ref_filter.so; its RE2 is the shim's matcher for the
regex forms Comparison::like_match emits)."""
import numpy as np
import pytest

from calamarijoins_b200 import ColumnarTable, Comparison, DataType, LogicalOperation, decode_column, encode_column
from oracle import oracle_api as oa
from tests.filter_cases import filter_table, rand_predicate

V = DataType.VARCHAR
need_ref = pytest.mark.skipif(not oa.ref_filter_available(), reason="reference filter not compiled")

LIKE_CASES = [
    ("", "", True), ("", "%", True), ("", "_", False), ("a", "_", True), ("ab", "_", False), ("ab", "a%", True),
    ("ab", "%b", True), ("ab", "%c%", False), ("abcabc", "%b_a%", True), ("a\nb", "a%b", False),
    ("a\nb", "a_b", False), ("a\nb", "a\nb", True), ("a\nb", "a\n%", True), ("é", "_", True), ("é", "__", False),
    ("中文", "_文", True), ("中文", "%", True), ("x%y", "x%y", True), ("x.y", "x_y", True), ("x*y", "x*y", True),
    ("(a)", "(_)", True), ("a+b", "a+b", True), ("a\\b", "a\\b", True), ("aaa", "%a%a%a%", True),
    ("aa", "%a%a%a%", False), ("ab\ncd", "%\n%", True), ("ab\ncd", "%b\nc%", True), ("ab\ncd", "%b%c%", False),
]


@pytest.mark.parametrize("s,pat,want", LIKE_CASES)
def test_oracle_like_known_answers(s, pat, want):
    assert oa.oracle_like(s.encode(), pat.encode()) == want


@need_ref
def test_like_agrees_with_reference():
    """Each case as a one-column table under LIKE: the reference's
    like_match (through its RE2 pattern) agrees with the oracle."""
    strs = [s for s, _, _ in LIKE_CASES]
    t = ColumnarTable(len(strs), [encode_column(V, [s.encode() for s in strs])])
    for _, pat, _ in LIKE_CASES:
        got = oa.ref_filter(t, Comparison(0, Comparison.LIKE, pat))
        want = np.array([oa.oracle_like(s.encode(), pat.encode()) for s in strs])
        assert np.array_equal(got, want), pat


@need_ref
@pytest.mark.parametrize("seed", range(6))
def test_random_predicates_agree_with_reference(seed):
    t = filter_table(3000, seed)
    rng = np.random.default_rng(100 + seed)
    for k in range(25):
        pred = rand_predicate(rng)
        _, sel = oa.oracle_filter(t, pred)
        assert np.array_equal(sel, oa.ref_filter(t, pred)), f"predicate {k}"


def test_oracle_filter_pages_are_the_selected_rows():
    t = filter_table(5000, 7, long_strings=True)
    pred = LogicalOperation.makeOr(Comparison(0, Comparison.LT, 0), Comparison(3, Comparison.LIKE, "%ab%"))
    res, sel = oa.oracle_filter(t, pred, [3, 0, 2])
    ok, msg = oa.validate(res)
    assert ok, msg
    assert res.num_rows == int(sel.sum())
    from calamarijoins_b200 import Column
    got_s, _ = decode_column(Column(V, res.pages[0]))
    all_s, _ = decode_column(t.columns[3])
    assert got_s == [all_s[i] for i in np.flatnonzero(sel)]


def test_int32_literal_truncates_like_the_reference():
    """An INT32 column compares with the literal's low 32 bits
    (static_cast<int32_t>, src/statement.cpp:54)."""
    t = ColumnarTable(3, [encode_column(DataType.INT32, np.array([5, 6, 7], np.int32))])
    _, sel = oa.oracle_filter(t, Comparison(0, Comparison.EQ, (1 << 32) + 6))
    assert sel.tolist() == [False, True, False]
