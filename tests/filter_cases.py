"""Seeded tables and predicate trees for the scan-filter tests (shared by
the CPU oracle-vs-reference tests and the GPU parity tests)."""
from __future__ import annotations

import numpy as np

from calamarijoins_b200 import ColumnarTable, Comparison, DataType, LogicalOperation, encode_column

I, L, F, V = DataType.INT32, DataType.INT64, DataType.FP64, DataType.VARCHAR
ALPHABET = ["a", "b", "c", "%", "_", "\n", "é", "中", " "]


def rand_string(rng, max_len=12):
    n = int(rng.integers(0, max_len + 1))
    return "".join(ALPHABET[int(k)] for k in rng.integers(0, len(ALPHABET), n))


def filter_table(n: int, seed: int, long_strings: bool = False) -> ColumnarTable:
    """INT32, INT64, FP64 and VARCHAR columns over small value domains (so
    that equality predicates hit), 10 % NULLs each; VARCHAR values drawn
    from a small alphabet with multi-byte characters and newlines."""
    rng = np.random.default_rng(seed)
    i32 = rng.integers(-50, 50, n).astype(np.int32)
    i64 = rng.integers(-(1 << 40), 1 << 40, n) // (1 << 34)
    f64 = np.round(rng.standard_normal(n) * 10, 1)
    f64[rng.random(n) < 0.01] = np.nan
    strs = [rand_string(rng) for _ in range(n)]
    if long_strings:
        for k in rng.choice(n, max(n // 500, 1), replace=False):
            strs[int(k)] = "ab" * int(rng.integers(4100, 9000)) + rand_string(rng)
    valid = [(rng.random(n) > 0.1).astype(np.uint8) for _ in range(4)]
    sv = [s.encode() if valid[3][k] else None for k, s in enumerate(strs)]
    return ColumnarTable(n, [encode_column(I, i32, valid[0]), encode_column(L, i64, valid[1]),
                             encode_column(F, f64, valid[2]), encode_column(V, sv)])


def rand_literal(rng, col):
    if col == 0:
        return int(rng.integers(-60, 60)) if rng.random() < 0.9 else int(rng.integers(-60, 60)) + (1 << 33)
    if col == 1:
        return int(rng.integers(-80, 80)) * (1 << 6) if rng.random() < 0.5 else int(rng.integers(-80, 80))
    if col == 2:
        return float(np.round(rng.standard_normal() * 10, 1))
    return rand_string(rng, 4)


def rand_pattern(rng):
    parts = []
    for _ in range(int(rng.integers(0, 5))):
        r = rng.random()
        parts.append("%" if r < 0.3 else ("_" if r < 0.5 else ALPHABET[int(rng.integers(0, len(ALPHABET)))]))
    return "".join(parts)


def rand_comparison(rng):
    col = int(rng.integers(0, 4))
    r = rng.random()
    if r < 0.1:
        return Comparison(col, Comparison.IS_NULL if rng.random() < 0.5 else Comparison.IS_NOT_NULL)
    if col == 3 and r < 0.55:
        return Comparison(col, Comparison.LIKE if rng.random() < 0.6 else Comparison.NOT_LIKE, rand_pattern(rng))
    return Comparison(col, int(rng.integers(0, 6)), rand_literal(rng, col))


def rand_predicate(rng, depth=0):
    r = rng.random()
    if depth >= 3 or r < 0.4:
        return rand_comparison(rng)
    if r < 0.65:
        return LogicalOperation.makeAnd(rand_predicate(rng, depth + 1), rand_predicate(rng, depth + 1))
    if r < 0.9:
        return LogicalOperation.makeOr(rand_predicate(rng, depth + 1), rand_predicate(rng, depth + 1))
    return LogicalOperation.makeNot(rand_predicate(rng, depth + 1))
