"""calamarijoins_b200 — CalamariJoins' join pipeline on one NVIDIA B200.

Python mirror of the reference's plan / table API over libcj_b200.so (the
C ABI in include/cj_b200.h). The joins themselves run as sm_100a kernels.
"""
from ._lib import CJError, LIB_PATH, PAGE_SIZE
from .engine import (Catalog, Context, PreparedBatch, ResidentTable, Result, Server, TimingStats, build_context,
                     destroy_context, execute, execute_batch, execute_raw, read_cache_meta, write_cache)
from .predicate import Comparison, LogicalOperation
from .plan import (Column, ColumnarTable, DataType, JoinNode, PinnedBuffer, Plan, PlanDescriptor, PlanNode,
                   ScanNode, Table, decode_column, encode_column)

__all__ = [
    "Comparison", "LogicalOperation", "CJError", "LIB_PATH", "PAGE_SIZE", "Catalog", "read_cache_meta", "write_cache", "Context", "PreparedBatch", "ResidentTable", "Result", "Server", "TimingStats", "build_context",
    "destroy_context", "execute", "execute_batch", "execute_raw", "Column", "ColumnarTable", "DataType", "JoinNode",
    "PinnedBuffer", "Plan", "PlanDescriptor", "PlanNode", "ScanNode", "Table", "decode_column", "encode_column",
]
