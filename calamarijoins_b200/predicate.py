"""Scan-side filter predicates, in the form of the reference's Statement
tree (include/data_model/statement.h): Comparison(column, op, value) and
LogicalOperation.makeAnd / makeOr / makeNot. A predicate is evaluated on
the GPU over a resident table by ResidentTable.filter (cj_table_filter),
with the reference's column-wise semantics (src/statement.cpp:47-241)."""
from __future__ import annotations

import ctypes as C
from typing import Union

from . import _lib
from .plan import DataType


class Statement:
    def flatten(self, nodes: list, keep: list) -> int:
        raise NotImplementedError


class Comparison(Statement):
    """Comparison::Op values (statement.h:57)."""
    EQ, NEQ, LT, GT, LEQ, GEQ, LIKE, NOT_LIKE, IS_NULL, IS_NOT_NULL = range(10)

    def __init__(self, column: int, op: int, value: Union[int, float, str, bytes, None] = None):
        self.column, self.op, self.value = int(column), int(op), value

    def flatten(self, nodes, keep) -> int:
        n = _lib.PredNodeC()
        n.kind, n.op, n.column = 0, self.op, self.column
        v = self.value
        if isinstance(v, bool) or v is None:
            n.literal_type = -1
        elif isinstance(v, int):
            n.literal_type, n.i64 = int(DataType.INT64), v
        elif isinstance(v, float):
            n.literal_type, n.f64 = int(DataType.FP64), v
        else:
            b = v.encode() if isinstance(v, str) else bytes(v)
            buf = C.create_string_buffer(b, len(b) + 1)
            keep.append(buf)
            n.literal_type, n.str, n.str_len = int(DataType.VARCHAR), C.cast(buf, C.c_char_p), len(b)
        nodes.append(n)
        return len(nodes) - 1


class LogicalOperation(Statement):
    AND, OR, NOT = 1, 2, 3

    def __init__(self, op: int, children):
        self.op, self.children = op, list(children)

    @staticmethod
    def makeAnd(left: Statement, right: Statement) -> "LogicalOperation":
        return LogicalOperation(LogicalOperation.AND, [left, right])

    @staticmethod
    def makeOr(left: Statement, right: Statement) -> "LogicalOperation":
        return LogicalOperation(LogicalOperation.OR, [left, right])

    @staticmethod
    def makeNot(child: Statement) -> "LogicalOperation":
        return LogicalOperation(LogicalOperation.NOT, [child])

    def flatten(self, nodes, keep) -> int:
        kids = [c.flatten(nodes, keep) for c in self.children]
        n = _lib.PredNodeC()
        n.kind = self.op
        n.left = kids[0]
        n.right = kids[1] if len(kids) > 1 else 0
        nodes.append(n)
        return len(nodes) - 1


class PredicateDesc:
    """The C description (cj_predicate) of a Statement tree; keeps the
    literal buffers alive."""

    def __init__(self, stmt: Statement):
        nodes, self._keep = [], []
        root = stmt.flatten(nodes, self._keep)
        self._arr = (_lib.PredNodeC * max(len(nodes), 1))(*nodes)
        self.desc = _lib.PredicateC(len(nodes), self._arr, root)
