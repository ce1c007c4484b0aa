"""Writes tests/golden/unit_cases.json: the 21 known-answer join cases of the
reference's Catch2 suite (CalamariJoins tests/unit_tests.cpp), transcribed
as data: input tables, plan nodes, root, and the answer each case asserts.

Large inputs are stored as the loops that build them in the reference test
("gen" entries) instead of as literal rows. Where a case only asserts a
property ("> 0 rows, no NULLs"), the exact row count implied by its inputs
is added as `derived_num_rows`, computed here from those inputs.

Run: python tests/golden/make_unit_cases.py
"""
from __future__ import annotations

import json
import os
from collections import Counter

I, V = "INT32", "VARCHAR"


def scan(t, attrs):
    return {"kind": "scan", "table": t, "attrs": attrs}


def join(build_left, left, right, la, ra, attrs):
    return {"kind": "join", "build_left": build_left, "left": left, "right": right,
            "left_attr": la, "right_attr": ra, "attrs": attrs}


def tab(types, rows=None, gen=None):
    d = {"types": types}
    if rows is not None:
        d["rows"] = rows
    if gen is not None:
        d["gen"] = gen
    return d


def two_scan_join(attrs=((0, I), (1, I))):
    return [scan(0, [[0, I]]), scan(1, [[0, I]]), join(True, 0, 1, 0, 0, [list(a) for a in attrs])]


def expand(g):
    """Rows of a "gen" table (the reference test's loop)."""
    kind = g["kind"]
    if kind == "range":  # for (i = start; i < stop; i += step) push {i}
        return [[i] for i in range(g["start"], g["stop"], g.get("step", 1))]
    if kind == "const":
        return [[g["value"]] for _ in range(g["count"])]
    if kind == "mod":  # push {(i % m) + 1}
        return [[(i % g["m"]) + 1] for i in range(g["count"])]
    if kind == "mod_null":  # i % null_every == 0 ? NULL : (i % m) + 1
        return [[None if i % g["null_every"] == 0 else (i % g["m"]) + 1] for i in range(g["count"])]
    raise ValueError(kind)


def main():
    cases = []
    seq3 = [[1], [2], [3]]

    cases.append({"name": "Empty join", "line": "16-35", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], []), tab([I], [])],
                  "expect": {"num_rows": 0, "types": [I, I], "rows": []}})
    cases.append({"name": "One line join", "line": "37-70", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], [[1]]), tab([I], [[1]])],
                  "expect": {"num_rows": 1, "types": [I, I], "rows": [[1, 1]]}})
    cases.append({"name": "Simple join", "line": "72-120", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], seq3), tab([I], seq3)],
                  "expect": {"num_rows": 3, "types": [I, I], "rows": [[1, 1], [2, 2], [3, 3]]}})
    cases.append({"name": "Empty Result", "line": "122-165", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], seq3), tab([I], [[4], [5], [6]])],
                  "expect": {"num_rows": 0, "types": [I, I], "rows": []}})
    same = [[1], [1], [2], [3]]
    six = [[1, 1]] * 4 + [[2, 2], [3, 3]]
    cases.append({"name": "Multiple same keys", "line": "167-230", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], same), tab([I], same)],
                  "expect": {"num_rows": 6, "types": [I, I], "rows": six}})
    nk = [[1], [1], [None], [2], [3]]
    cases.append({"name": "NULL keys", "line": "232-298", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], nk), tab([I], nk)],
                  "expect": {"num_rows": 6, "types": [I, I], "rows": six}})
    mc = [[1, "xxx"], [1, "yyy"], [None, "zzz"], [2, "uuu"], [3, "vvv"]]
    mc_rows = [[1, 1, "xxx"], [1, 1, "xxx"], [1, 1, "yyy"], [1, 1, "yyy"], [2, 2, "uuu"], [3, 3, "vvv"]]
    for name, bl, line in (("Multiple columns", True, "300-352"), ("Build on right", False, "354-406")):
        cases.append({"name": name, "line": line, "root": 2,
                      "nodes": [scan(0, [[0, I]]), scan(1, [[1, V], [0, I]]),
                                join(bl, 0, 1, 0, 1, [[0, I], [2, I], [1, V]])],
                      "tables": [tab([I, V], mc), tab([I, V], mc)],
                      "expect": {"num_rows": 6, "types": [I, I, V], "rows": mc_rows}})
    cases.append({"name": "leftdeep 2-level join", "line": "408-466", "root": 4,
                  "nodes": [scan(0, [[0, I]]), scan(1, [[0, I]]), scan(2, [[0, I]]),
                            join(True, 0, 1, 0, 0, [[0, I], [1, I]]),
                            join(False, 3, 2, 0, 0, [[0, I], [1, I], [2, I]])],
                  "tables": [tab([I], seq3)] * 3,
                  "expect": {"num_rows": 3, "types": [I, I, I], "rows": [[1, 1, 1], [2, 2, 2], [3, 3, 3]]}})
    cases.append({"name": "3-way join", "line": "468-519", "root": 4,
                  "nodes": [scan(0, [[0, I], [1, V]]), scan(1, [[0, I], [1, V]]), scan(2, [[0, I], [1, V]]),
                            join(False, 0, 1, 0, 0, [[0, I], [1, V]]),
                            join(False, 3, 2, 0, 0, [[0, I], [1, V], [3, V]])],
                  "tables": [tab([I, V], [[1, "a"], [2, "b"], [3, "c"]]), tab([I, V], [[1, "x"], [2, "y"]]),
                             tab([I, V], [[1, "u"], [2, "v"], [3, "w"]])],
                  "expect": {"num_rows": 2, "types": [I, V, V], "rows": [[1, "a", "u"], [2, "b", "v"]]}})
    cases.append({"name": "Large Duplicate keys", "line": "521-546", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], gen={"kind": "const", "value": 1, "count": 100})] * 2,
                  "expect": {"num_rows": 10000}})
    cases.append({"name": "Sequential keys", "line": "547-568", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], gen={"kind": "range", "start": 1, "stop": 1001})] * 2,
                  "expect": {"num_rows": 1000}})
    cases.append({"name": "All NULL keys", "line": "570-592", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], [[None], [None], [None]])] * 2, "expect": {"num_rows": 0}})
    cases.append({"name": "All keys different", "line": "594-614", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], seq3), tab([I], [[4], [5], [6]])], "expect": {"num_rows": 0}})
    cases.append({"name": "Negative keys join", "line": "615-635", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], [[-1], [-2], [-3]]), tab([I], [[-2], [-3], [-4]])],
                  "expect": {"num_rows": 2}})
    cases.append({"name": "Heavy hash collisions", "line": "637-661", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], [[0], [1024], [2048], [3072]]), tab([I], [[0], [1024], [4096]])],
                  "expect": {"num_rows": 2}})
    cases.append({"name": "Threaded build large sequential keys", "line": "670-704", "nodes": two_scan_join(),
                  "root": 2, "tables": [tab([I], gen={"kind": "range", "start": 1, "stop": 15001})] * 2,
                  "expect": {"num_rows": 15000, "types": [I, I], "check": "pairs_equal_1_to_n"}})
    cases.append({"name": "Threaded build large duplicate keys", "line": "706-736", "nodes": two_scan_join(),
                  "root": 2, "tables": [tab([I], gen={"kind": "mod", "m": 10, "count": 1200})] * 2,
                  "expect": {"num_rows": 144000, "types": [I, I]}})
    cases.append({"name": "Threaded build multi-level join", "line": "738-780", "root": 4,
                  "nodes": [scan(0, [[0, I]]), scan(1, [[0, I]]), scan(2, [[0, I]]),
                            join(True, 0, 1, 0, 0, [[0, I], [1, I]]),
                            join(True, 3, 2, 0, 0, [[0, I], [1, I], [2, I]])],
                  "tables": [tab([I], gen={"kind": "range", "start": 1, "stop": 12001})] * 3,
                  "expect": {"num_rows": 12000, "types": [I, I, I], "check": "triples_equal_1_to_n"}})
    g1 = {"kind": "mod_null", "m": 100, "null_every": 7, "count": 15000}
    g2 = {"kind": "mod_null", "m": 100, "null_every": 11, "count": 15000}
    c1 = Counter(r[0] for r in expand(g1) if r[0] is not None)
    c2 = Counter(r[0] for r in expand(g2) if r[0] is not None)
    derived = sum(c1[k] * c2[k] for k in c1)
    cases.append({"name": "Threaded build with NULLs", "line": "782-826", "nodes": two_scan_join(), "root": 2,
                  "tables": [tab([I], gen=g1), tab([I], gen=g2)],
                  "expect": {"min_rows": 1, "types": [I, I], "check": "no_nulls",
                             "derived_num_rows": derived}})
    sp = {"kind": "range", "start": 1, "stop": 20001, "step": 10}
    cases.append({"name": "Threaded build sparse distribution", "line": "828-870", "nodes": two_scan_join(),
                  "root": 2, "tables": [tab([I], gen=sp)] * 2,
                  "expect": {"num_rows": 2000, "types": [I, I], "check": "pairs_equal_mod10_1"}})
    out = {"source": "CalamariJoins tests/unit_tests.cpp", "cases": cases}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "unit_cases.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(path, len(cases))


if __name__ == "__main__":
    main()
