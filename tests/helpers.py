"""Shared test helpers: golden-case loading, plan construction, running the
product / oracle / reference and comparing results."""
from __future__ import annotations

import json
import os

import numpy as np

from calamarijoins_b200 import (ColumnarTable, DataType, Plan, PlanDescriptor, Table, encode_column,
                                execute_raw)
from oracle import oracle_api as oa

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
T = {"INT32": DataType.INT32, "INT64": DataType.INT64, "FP64": DataType.FP64, "VARCHAR": DataType.VARCHAR}


def load_unit_cases():
    with open(os.path.join(GOLDEN, "unit_cases.json")) as f:
        return json.load(f)["cases"]


def expand_gen(g):
    kind = g["kind"]
    if kind == "range":
        return [[i] for i in range(g["start"], g["stop"], g.get("step", 1))]
    if kind == "const":
        return [[g["value"]] for _ in range(g["count"])]
    if kind == "mod":
        return [[(i % g["m"]) + 1] for i in range(g["count"])]
    if kind == "mod_null":
        return [[None if i % g["null_every"] == 0 else (i % g["m"]) + 1] for i in range(g["count"])]
    raise ValueError(kind)


def plan_from_case(case) -> Plan:
    plan = Plan()
    for n in case["nodes"]:
        attrs = [(a[0], T[a[1]]) for a in n["attrs"]]
        if n["kind"] == "scan":
            plan.new_scan_node(n["table"], attrs)
        else:
            plan.new_join_node(n["build_left"], n["left"], n["right"], n["left_attr"], n["right_attr"], attrs)
    for t in case["tables"]:
        rows = t["rows"] if "rows" in t else expand_gen(t["gen"])
        types = [T[x] for x in t["types"]]
        if not rows:
            plan.inputs.append(ColumnarTable(0, [encode_column(tt, [] if tt == DataType.VARCHAR
                                                               else np.zeros(0)) for tt in types]))
        else:
            plan.inputs.append(Table(rows, types).to_columnar())
    plan.root = case["root"]
    return plan


def paged_to_table(r: oa.PagedResult) -> Table:
    from calamarijoins_b200 import Column
    return Table.from_columnar(ColumnarTable(r.num_rows, [Column(DataType(t), p) for t, p in zip(r.types, r.pages)]))


def check_expect(r: oa.PagedResult, exp: dict, label: str = ""):
    ok, msg = oa.validate(r)
    assert ok, f"{label}: malformed output pages: {msg}"
    if "num_rows" in exp:
        assert r.num_rows == exp["num_rows"], f"{label}: rows {r.num_rows} != {exp['num_rows']}"
    if "derived_num_rows" in exp:
        assert r.num_rows == exp["derived_num_rows"], label
    if "min_rows" in exp:
        assert r.num_rows >= exp["min_rows"], label
    if "types" in exp:
        assert r.types == [int(T[t]) for t in exp["types"]], f"{label}: types {r.types}"
    need_rows = "rows" in exp or "check" in exp
    if not need_rows:
        return
    rows = paged_to_table(r).sorted_rows()
    if "rows" in exp:
        want = Table(exp["rows"], [T[t] for t in exp["types"]]).sorted_rows()
        assert rows == want, f"{label}: rows differ"
    chk = exp.get("check")
    if chk == "pairs_equal_1_to_n":
        assert all(row[0] == row[1] == i + 1 for i, row in enumerate(rows)), label
    elif chk == "triples_equal_1_to_n":
        assert all(row[0] == row[1] == row[2] == i + 1 for i, row in enumerate(rows)), label
    elif chk == "no_nulls":
        assert all(v is not None for row in rows for v in row), label
    elif chk == "pairs_equal_mod10_1":
        assert all(row[0] == row[1] and row[0] % 10 == 1 for row in rows), label


def run_product(plan: Plan, ctx, flags: int = 0):
    res, stats = execute_raw(plan, ctx, flags)
    try:
        return oa.PagedResult.from_result(res), stats
    finally:
        res.free()


def run_oracle(plan: Plan) -> oa.PagedResult:
    return oa.oracle_execute(PlanDescriptor(plan))


def assert_same(a: oa.PagedResult, b: oa.PagedResult, label: str = ""):
    ok, msg = oa.validate(a)
    assert ok, f"{label}: malformed pages: {msg}"
    ok, msg = oa.tables_equal(a, b)
    assert ok, f"{label}: results differ: {msg}"
