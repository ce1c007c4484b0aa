"""CPU: the oracle agrees with the reference's own execute() on random plan
trees, not only the chains and two-table joins the workloads use.

Each example draws 2-5 small tables (some empty, INT32 key columns over
small domains with NULLs, INT32 payloads with NULLs, VARCHAR payloads
without NULLs: the reference's valid domain) and a random join tree over
scans of them: bushy or deep, a table scanned twice (self-join), join keys
anywhere in either side's outputs, output lists that repeat or drop
columns. The oracle's result must equal the reference's, row multiset for
row multiset. The oracle is the checker of every GPU parity test, so this
widens what its pin covers."""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

from calamarijoins_b200 import ColumnarTable, DataType, Plan, PlanDescriptor, encode_column
from oracle import oracle_api as oa

pytestmark = pytest.mark.skipif(not oa.ref_available(), reason="reference not compiled (oracle/build_oracle.py)")

I, V = DataType.INT32, DataType.VARCHAR


def random_table(rng):
    rows = int(rng.choice([0, 1, 5, 40, 150], p=[0.04, 0.08, 0.18, 0.35, 0.35]))
    cols, types = [], []
    for _ in range(int(rng.integers(1, 4))):
        dom = max(2, int(rng.integers(2, 60)))
        vals = rng.integers(-dom // 2, dom, size=rows).astype(np.int32)
        valid = (rng.random(rows) > rng.choice([0.0, 0.1, 0.5])).astype(np.uint8)
        cols.append(encode_column(I, vals, valid))
        types.append(I)
    if rng.random() < 0.5:
        strs = ["".join(chr(97 + int(c)) for c in rng.integers(0, 26, size=int(rng.integers(0, 12))))
                for _ in range(rows)]
        cols.append(encode_column(V, strs))
        types.append(V)
    return ColumnarTable(rows, cols), types


def random_plan(seed):
    """A random join tree over scans of 2-5 random tables; None when the
    draw leaves a join without an INT32 key on one side."""
    rng = np.random.default_rng(seed)
    plan = Plan()
    ttypes = []
    for _ in range(int(rng.integers(2, 6))):
        t, types = random_table(rng)
        plan.inputs.append(t)
        ttypes.append(types)
    # leaves: scans (a table may be scanned twice), each projecting a random
    # non-empty list of its columns
    nodes = []  # (node id, output types)
    for _ in range(int(rng.integers(2, 5))):
        tid = int(rng.integers(0, len(ttypes)))
        types = ttypes[tid]
        pick = [int(c) for c in rng.choice(len(types), size=int(rng.integers(1, len(types) + 1)), replace=False)]
        if I not in [types[c] for c in pick]:
            pick.append(types.index(I))
        nid = plan.new_scan_node(tid, [(c, types[c]) for c in pick])
        nodes.append((nid, [types[c] for c in pick]))
    # join random pairs until one tree is left (bushy or deep)
    while len(nodes) > 1:
        a, b = (int(x) for x in rng.choice(len(nodes), size=2, replace=False))
        (ln, lt), (rn, rt) = nodes[a], nodes[b]
        lk = [i for i, t in enumerate(lt) if t == I]
        rk = [i for i, t in enumerate(rt) if t == I]
        if not lk or not rk:
            return None
        both = lt + rt
        last = len(nodes) == 2
        n_out = int(rng.integers(1, len(both) + 2))
        outs = [int(x) for x in rng.integers(0, len(both), size=n_out)]  # repeats allowed
        if not last and I not in [both[i] for i in outs]:
            outs.append(int(rng.choice(lk)))
        nid = plan.new_join_node(bool(rng.random() < 0.5), ln, rn, int(rng.choice(lk)), int(rng.choice(rk)),
                                 [(i, both[i]) for i in outs])
        nodes = [n for k, n in enumerate(nodes) if k not in (a, b)] + [(nid, [both[i] for i in outs])]
    plan.root = nodes[0][0]
    return plan


@settings(max_examples=120, deadline=None, derandomize=True,
          suppress_health_check=[HealthCheck.too_slow, HealthCheck.filter_too_much])
@given(st.integers(min_value=0, max_value=2 ** 32 - 1))
def test_random_plan_trees(seed):
    plan = random_plan(seed)
    if plan is None:
        return
    d = PlanDescriptor(plan)
    r, _, _ = oa.ref_execute(d, oa.ref_available()[0])
    o = oa.oracle_execute(d)
    ok, msg = oa.tables_equal(o, r)
    assert ok, f"seed {seed}: {msg}"


def test_generator_reaches_the_shapes():
    """The draw covers what the test claims: bushy trees, self-joins,
    empty tables and repeated outputs."""
    from calamarijoins_b200 import _lib
    bushy = selfjoin = empty = repeated = 0
    for seed in range(300):
        plan = random_plan(seed)
        if plan is None:
            continue
        d = PlanDescriptor(plan).desc
        scans, children = [], []
        for k in range(d.num_nodes):
            nd = d.nodes[k]
            if nd.node_type == _lib.CJ_NODE_SCAN:
                scans.append(nd.base_table_id)
            else:
                children.append((nd.left, nd.right))
                idx = [nd.output_attrs[a].index for a in range(nd.num_output_attrs)]
                repeated += len(idx) != len(set(idx))
        is_join = {k for k in range(d.num_nodes) if d.nodes[k].node_type != _lib.CJ_NODE_SCAN}
        bushy += any(l in is_join and r in is_join for l, r in children)
        selfjoin += len(scans) != len(set(scans))
        empty += any(t.num_rows == 0 for t in plan.inputs)
    assert bushy > 0 and selfjoin > 0 and empty > 0 and repeated > 0, (bushy, selfjoin, empty, repeated)
