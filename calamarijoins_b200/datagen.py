"""Seeded synthetic workloads in the paged format.

The reference is benchmarked on the Join Order Benchmark over IMDB, which is
not available offline; these generators produce tables with the shapes,
sizes and value distributions of the benchmark configurations instead:

  config_c1  100,000-row build (unique shuffled INT32 keys + INT32 payload)
             joined with a 1,000,000-row probe (Zipf(1.0) foreign keys, 5%
             NULL, INT64 payload); 3 output columns
  config_c2  4,000,000 unique shuffled build keys joined with 64,000,000
             probe rows: Zipf(0.8) foreign keys, 30% outside the build
             domain, 2% NULL; outputs 2 INT32 + INT64 + FP64
  config_c2h C2's shape with a non-unique build side (4M rows over 3M
             distinct keys): the unchained hash table's workload
  config_c3  left-deep 6-way pipeline: 36,000,000-row fact table with five
             INT32 foreign keys (Zipf s in {0.5, 1.0, 1.2}) into dimensions of
             2,500 / 130,000 / 1,200,000 / 2,500,000 / 4,200,000 rows filtered
             to 0.1-40%, VARCHAR outputs with log-normal lengths (mean 20,
             max 200) and a 0.01% fraction of strings longer than 8,185 bytes
  batch_plans / serve_plans
             the 2-4-way and 2-16-way plan mixes of the batched and served
             modes

Every `scale` argument shrinks row counts proportionally (for tests).
INT32_MIN is never generated (the format's intermediate NULL sentinel).
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .plan import ColumnarTable, DataType, Plan, encode_column

INT32_MIN = -(2 ** 31)


def zipf_ranks(n: int, s: float, size: int, rng: np.random.Generator) -> np.ndarray:
    """`size` ranks in [1, n] with P(k) proportional to k^-s.

    Rejection-inversion sampling (W. Hormann, G. Derflinger, "Rejection-
    inversion to generate variates from monotone discrete distributions",
    ACM TOMACS 6(3), 1996), vectorised; s = 0 is uniform."""
    if size == 0:
        return np.zeros(0, dtype=np.int64)
    if s == 0:
        return rng.integers(1, n + 1, size=size, dtype=np.int64)

    def H(x):
        if abs(s - 1.0) < 1e-12:
            return np.log(x)
        return (np.power(x, 1.0 - s) - 1.0) / (1.0 - s)

    def Hinv(y):
        if abs(s - 1.0) < 1e-12:
            return np.exp(y)
        return np.power(1.0 + y * (1.0 - s), 1.0 / (1.0 - s))

    h = lambda x: np.power(x, -s)  # noqa: E731
    hx1 = H(1.5) - 1.0
    hn = H(n + 0.5)
    s_const = 2.0 - Hinv(H(2.5) - h(2.0))
    out = np.empty(size, dtype=np.int64)
    todo = np.arange(size)
    while todo.size:
        u = hn + rng.random(todo.size) * (hx1 - hn)
        x = Hinv(u)
        k = np.clip(np.floor(x + 0.5), 1, n)
        ok = (k - x <= s_const) | (u >= H(k + 0.5) - h(k))
        out[todo[ok]] = k[ok].astype(np.int64)
        todo = todo[~ok]
    return out


def varchar_values(n: int, rng: np.random.Generator, mean: float = 20.0, cap: int = 200,
                   long_frac: float = 0.0, long_range=(8186, 24000)):
    """(chars, offsets) of n strings with log-normal lengths (given mean,
    capped), plus a `long_frac` fraction of long strings."""
    sigma = 0.6
    mu = math.log(mean) - sigma * sigma / 2
    lens = np.clip(np.round(rng.lognormal(mu, sigma, n)), 0, cap).astype(np.int64)
    if long_frac > 0:
        m = rng.random(n) < long_frac
        lens[m] = rng.integers(long_range[0], long_range[1], size=int(m.sum()))
    offsets = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(lens, out=offsets[1:])
    total = int(offsets[-1])
    chars = rng.integers(97, 123, size=total, dtype=np.uint8)
    return chars, offsets


def _valid(n: int, null_frac: float, rng) -> Optional[np.ndarray]:
    if null_frac <= 0:
        return None
    return (rng.random(n) >= null_frac).astype(np.uint8)


def _payload(dtype: DataType, n: int, rng, null_frac: float = 0.0, pinned: bool = False, **vkw):
    valid = _valid(n, null_frac, rng)
    if dtype == DataType.INT32:
        vals = rng.integers(INT32_MIN + 1, 2 ** 31 - 1, size=n, dtype=np.int32)
    elif dtype == DataType.INT64:
        vals = rng.integers(-(2 ** 62), 2 ** 62, size=n, dtype=np.int64)
    elif dtype == DataType.FP64:
        vals = rng.standard_normal(n) * 1e6
    else:
        return encode_column(dtype, varchar_values(n, rng, **vkw), valid, pinned=pinned)
    return encode_column(dtype, vals, valid, pinned=pinned)


def fk_column(build_keys: np.ndarray, n: int, s: float, outside: float, null_frac: float, rng,
              dtype=DataType.INT32):
    """Foreign keys: Zipf(s) over the build keys (hot keys at random
    positions), an `outside` fraction drawn outside the build domain."""
    nb = len(build_keys)
    perm = rng.permutation(nb)
    ranks = zipf_ranks(nb, s, n, rng)
    keys = build_keys[perm[ranks - 1]].astype(np.int64)
    if outside > 0:
        m = rng.random(n) < outside
        hi = 2 ** 31 - 1 if dtype == DataType.INT32 else 2 ** 62
        lo = int(build_keys.max()) + 1 if nb else 0
        keys[m] = rng.integers(lo, hi, size=int(m.sum()))
    vals = keys.astype(np.int32 if dtype == DataType.INT32 else np.int64)
    return vals, _valid(n, null_frac, rng)


def join2(n_build: int, n_probe: int, *, seed: int = 1, zipf: float = 1.0, outside: float = 0.0,
          build_null: float = 0.0, probe_null: float = 0.0, key_type=DataType.INT32,
          build_payload=(DataType.INT32,), probe_payload=(DataType.INT64,), build_left: bool = True,
          output=None, pinned: bool = False, unique_build: bool = True, varchar_kw=None,
          key_scale: int = 1) -> Plan:
    """A 2-table equi-join plan: table 0 (build candidate) = key + build
    payloads, table 1 = foreign key + probe payloads. `output` lists
    (side, column) pairs over (left ++ right); default = every column.
    Unique build keys are a permutation of 0, key_scale, 2 key_scale, ..."""
    rng = np.random.default_rng(seed)
    vkw = varchar_kw or {}
    if unique_build:
        bkeys = rng.permutation(n_build).astype(np.int64) * key_scale
    else:
        bkeys = rng.integers(0, max(n_build // 4, 1), size=n_build).astype(np.int64)
    npt = np.int32 if key_type == DataType.INT32 else np.int64
    bcols = [encode_column(key_type, bkeys.astype(npt), _valid(n_build, build_null, rng), pinned=pinned)]
    for t in build_payload:
        bcols.append(_payload(t, n_build, rng, pinned=pinned, **vkw))
    fk, fv = fk_column(np.unique(bkeys) if not unique_build else bkeys, n_probe, zipf, outside, probe_null, rng,
                       key_type)
    pcols = [encode_column(key_type, fk, fv, pinned=pinned)]
    for t in probe_payload:
        pcols.append(_payload(t, n_probe, rng, pinned=pinned, **vkw))
    plan = Plan()
    plan.inputs.append(ColumnarTable(n_build, bcols))
    plan.inputs.append(ColumnarTable(n_probe, pcols))
    btypes = [key_type, *build_payload]
    ptypes = [key_type, *probe_payload]
    plan.new_scan_node(0, [(i, t) for i, t in enumerate(btypes)])
    plan.new_scan_node(1, [(i, t) for i, t in enumerate(ptypes)])
    allt = btypes + ptypes
    if output is None:
        output = list(range(len(allt)))
    plan.new_join_node(build_left, 0, 1, 0, 0, [(i, allt[i]) for i in output])
    plan.root = 2
    return plan


def config_c1(seed: int = 101, scale: float = 1.0, pinned: bool = False) -> Plan:
    nb, npr = max(int(100_000 * scale), 16), max(int(1_000_000 * scale), 16)
    # output: build key, build INT32 payload, probe INT64 payload
    return join2(nb, npr, seed=seed, zipf=1.0, probe_null=0.05, build_payload=(DataType.INT32,),
                 probe_payload=(DataType.INT64,), output=[0, 1, 3], pinned=pinned)


def config_c2(seed: int = 202, scale: float = 1.0, pinned: bool = False) -> Plan:
    nb, npr = max(int(4_000_000 * scale), 16), max(int(64_000_000 * scale), 16)
    # output: build key INT32, build INT64 payload, probe FK INT32, probe FP64 payload
    return join2(nb, npr, seed=seed, zipf=0.8, outside=0.30, probe_null=0.02,
                 build_payload=(DataType.INT64,), probe_payload=(DataType.FP64,), output=[0, 1, 2, 3],
                 pinned=pinned)


def config_c2s(seed: int = 212, scale: float = 1.0, pinned: bool = False, int32_standin: bool = False) -> Plan:
    """C2's shape with the build keys spread 500x (unique multiples of 500
    below 2^31): too wide for a direct-mapped table, so the join takes the
    open-addressing table."""
    nb, npr = max(int(4_000_000 * scale), 16), max(int(64_000_000 * scale), 16)
    payloads = (DataType.INT32,) if int32_standin else None
    return join2(nb, npr, seed=seed, zipf=0.8, outside=0.30, probe_null=0.02,
                 build_payload=payloads or (DataType.INT64,), probe_payload=payloads or (DataType.FP64,),
                 output=[0, 1, 2, 3], pinned=pinned, key_scale=500)


def config_c2h(seed: int = 222, scale: float = 1.0, pinned: bool = False, int32_standin: bool = False) -> Plan:
    """C2's shape with a non-unique build side, so that only the unchained
    hash table serves it: 4,000,000 build rows over 3,000,000 distinct keys
    (a third of them appear twice), INT64 payload; 64,000,000 probe rows,
    foreign keys Zipf(0.8) over the distinct keys, 30 % outside the build
    domain, 2 % NULL, FP64 payload. About 58.5M output rows."""
    rng = np.random.default_rng(seed)
    nb, npr = max(int(4_000_000 * scale), 16), max(int(64_000_000 * scale), 16)
    nd = max(nb * 3 // 4, 1)
    distinct = rng.permutation(nd).astype(np.int64)
    bkeys = np.concatenate([distinct, distinct[:nb - nd]])
    rng.shuffle(bkeys)
    I = DataType.INT32
    bp = (I,) if int32_standin else (DataType.INT64,)
    pp = (I,) if int32_standin else (DataType.FP64,)
    bcols = [encode_column(I, bkeys.astype(np.int32), pinned=pinned)] + [_payload(t, nb, rng, pinned=pinned)
                                                                         for t in bp]
    fk, fv = fk_column(distinct, npr, 0.8, 0.30, 0.02, rng)
    pcols = [encode_column(I, fk, fv, pinned=pinned)] + [_payload(t, npr, rng, pinned=pinned) for t in pp]
    plan = Plan()
    plan.inputs.append(ColumnarTable(nb, bcols))
    plan.inputs.append(ColumnarTable(npr, pcols))
    plan.new_scan_node(0, [(0, I), (1, bp[0])])
    plan.new_scan_node(1, [(0, I), (1, pp[0])])
    plan.new_join_node(True, 0, 1, 0, 0, [(0, I), (1, bp[0]), (2, I), (3, pp[0])])
    plan.root = 2
    return plan


C3_DIMS = (2_500, 130_000, 1_200_000, 2_500_000, 4_200_000)
C3_KEEP = (0.40, 0.40, 0.30, 0.20, 0.10)
C3_ZIPF = (0.5, 1.0, 1.2, 1.0, 0.5)


def config_c3(seed: int = 303, scale: float = 1.0, pinned: bool = False, varchar_nulls: bool = False,
              long_frac: float = 1e-4) -> Plan:
    """Left-deep 6-way: ((((fact x d0) x d1) x d2) x d3) x d4. Output: the
    fact row's first FK, a fact VARCHAR, and every dimension's VARCHAR."""
    rng = np.random.default_rng(seed)
    nf = max(int(36_000_000 * scale), 64)
    plan = Plan()
    vnull = 0.05 if varchar_nulls else 0.0
    fcols = []
    dim_tables = []
    for d, (nd, keep, s) in enumerate(zip(C3_DIMS, C3_KEEP, C3_ZIPF)):
        nd = max(int(nd * scale), 8)
        dom = rng.permutation(nd).astype(np.int64)
        kept = np.sort(rng.choice(nd, size=max(int(nd * keep), 1), replace=False))
        dkeys = dom[kept]
        fk, fv = fk_column(dom, nf, s, 0.0, 0.0, rng)
        fcols.append(encode_column(DataType.INT32, fk, fv, pinned=pinned))
        dv = encode_column(DataType.VARCHAR, varchar_values(len(dkeys), rng, long_frac=long_frac),
                           _valid(len(dkeys), vnull, rng), pinned=pinned)
        dk = encode_column(DataType.INT32, dkeys.astype(np.int32), pinned=pinned)
        dim_tables.append(ColumnarTable(len(dkeys), [dk, dv]))
    fcols.append(encode_column(DataType.VARCHAR, varchar_values(nf, rng, long_frac=long_frac),
                               _valid(nf, vnull, rng), pinned=pinned))
    I, V = DataType.INT32, DataType.VARCHAR
    plan.inputs.append(ColumnarTable(nf, fcols))
    for t in dim_tables:
        plan.inputs.append(t)
    fact = plan.new_scan_node(0, [(0, I), (1, I), (2, I), (3, I), (4, I), (5, V)])
    dims = [plan.new_scan_node(1 + d, [(0, I), (1, V)]) for d in range(5)]
    # running left output: [fk0..fk4, fact_v, dim varchars...]
    left = fact
    left_types = [I, I, I, I, I, V]
    for d in range(5):
        nl = len(left_types)
        out = [(i, t) for i, t in enumerate(left_types)] + [(nl + 1, V)]
        node = plan.new_join_node(False, left, dims[d], d, 0, out)
        left_types = left_types + [V]
        left = node
    plan.root = left
    return plan


def batch_plans(n_plans: int = 256, seed: int = 404, scale: float = 1.0, max_build: int = 1_000_000,
                max_probe: int = 10_000_000, pinned: bool = False) -> list:
    """2-4-way INT32 plans with builds log-uniform 10..max_build and probes
    log-uniform 1e3..max_probe (a fraction tiny enough for the nested loop)."""
    rng = np.random.default_rng(seed)
    plans = []
    for i in range(n_plans):
        ways = int(rng.integers(2, 5))
        nprobe = int(10 ** rng.uniform(3, math.log10(max(max_probe * scale, 1e3 + 1))))
        plans.append(chain_plan(ways, nprobe, rng, max_build=max(int(max_build * scale), 10), pinned=pinned))
    return plans


def chain_plan(ways: int, n_probe: int, rng, max_build: int = 1_000_000, key_types=None, zipf=None,
               varchar_frac: float = 0.0, pinned: bool = False) -> Plan:
    """Left-deep chain: a probe-side fact with ways-1 foreign keys, each
    joined to a dimension of log-uniform size 10..max_build."""
    I, V = DataType.INT32, DataType.VARCHAR
    nd = ways - 1
    kts = key_types or [I] * nd
    plan = Plan()
    dims = []
    fcols = []
    for d in range(nd):
        nb = int(10 ** rng.uniform(1, math.log10(max(max_build, 11))))
        kt = kts[d]
        s = float(rng.uniform(0, 1.2)) if zipf is None else zipf
        keys = rng.permutation(nb).astype(np.int64)
        fk, fv = fk_column(keys, n_probe, s, float(rng.uniform(0, 0.3)), 0.01, rng, kt)
        fcols.append(encode_column(kt, fk, fv, pinned=pinned))
        npt = np.int32 if kt == I else np.int64
        cols = [encode_column(kt, keys.astype(npt), pinned=pinned)]
        has_v = rng.random() < varchar_frac
        if has_v:
            cols.append(encode_column(V, varchar_values(nb, rng), pinned=pinned))
        else:
            cols.append(encode_column(I, rng.integers(0, 1 << 30, size=nb, dtype=np.int32), pinned=pinned))
        dims.append((ColumnarTable(nb, cols), kt, V if has_v else I))
    fcols.append(encode_column(I, rng.integers(0, 1 << 30, size=n_probe, dtype=np.int32), pinned=pinned))
    plan.inputs.append(ColumnarTable(n_probe, fcols))
    for t, _, _ in dims:
        plan.inputs.append(t)
    ftypes = [kts[d] for d in range(nd)] + [I]
    fact = plan.new_scan_node(0, [(i, t) for i, t in enumerate(ftypes)])
    dscans = [plan.new_scan_node(1 + d, [(0, dims[d][1]), (1, dims[d][2])]) for d in range(nd)]
    left, ltypes = fact, list(ftypes)
    for d in range(nd):
        n_l = len(ltypes)
        out = [(i, t) for i, t in enumerate(ltypes)] + [(n_l + 1, dims[d][2])]
        left = plan.new_join_node(True, left, dscans[d], d, 0, out)
        ltypes = ltypes + [dims[d][2]]
    plan.root = left
    return plan
