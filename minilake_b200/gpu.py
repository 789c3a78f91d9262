"""Python face of the B200 execution core: a thin ctypes layer over
``libminilake_gpu.so`` (the C ABI in ``include/minilake_gpu.h``).

The classes mirror MiniLake's pipeline contract (crates/minilake-exec/src/pipeline.rs):
``FilterOperator`` / ``ProjectionOperator`` / ``HashJoinProbe`` are streaming
operators; ``HashAggregateSink`` / ``JoinBuildSink`` / ``SortSink`` are sinks with
``create_local()`` -> ``LocalSink.sink(batch)`` -> ``LocalSink.combine()`` ->
``finalize()``.  A sink may be given the streaming operators that precede it
(the "prologue"); its kernel then runs the whole pipeline per morsel.

There is no CPU fallback: importing this module fails loudly when the CUDA
library has not been built, and every call runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from .columns import HostColumn, Table

_LIB_PATH = os.path.join(os.path.dirname(__file__), "_lib", "libminilake_gpu.so")


class MiniLakeError(RuntimeError):
    """MiniLakeError (crates/minilake-core/src/error.rs); `code` is the C status."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class ResourcesExhausted(MiniLakeError):
    """ResourcesExhausted{operator, requested, used, limit} (memory.rs:114-128)."""

    def __init__(self, code, msg, operator, requested, used, limit):
        super().__init__(code, msg)
        self.operator, self.requested, self.used, self.limit = operator, requested, used, limit


class StalePlan(MiniLakeError):
    """A prepared query's data no longer fits its plan (ML_ERR_STALE_PLAN): prepare it again."""


def _load():
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} is missing: build the CUDA library first "
                          "(python -c 'import __graft_entry__ as g; g.build()')")
    lib = C.CDLL(_LIB_PATH)
    P, I32, I64, U64, VP = C.POINTER, C.c_int32, C.c_int64, C.c_uint64, C.c_void_p
    sigs = {
        "ml_gpu_last_error": ([], C.c_char_p),
        "ml_gpu_last_budget_error": ([C.c_char_p, C.c_size_t, P(U64), P(U64), P(U64)], C.c_int),
        "ml_gpu_ctx_create": ([C.c_int, U64, C.c_uint32, P(VP)], C.c_int),
        "ml_gpu_ctx_destroy": ([VP], C.c_int),
        "ml_gpu_pool_stats": ([VP, P(U64), P(U64), P(U64)], C.c_int),
        "ml_gpu_ctx_synchronize": ([VP], C.c_int),
        "ml_gpu_kernel_launches": ([VP, P(U64)], C.c_int),
        "ml_gpu_profile_read": ([VP, C.c_char_p, P(U64), P(C.c_double), I32], C.c_int),
        "ml_gpu_hashagg_rebind": ([VP, P(abi.MlPipeOp), I32, VP, I32, P(abi.MlExpr), I32, P(abi.MlAggSpec), I32],
                                  C.c_int),
        "ml_gpu_hashagg_reset": ([VP], C.c_int),
        "ml_gpu_hashagg_run_resident": ([VP, P(abi.MlColumn), I32, I64, I32], C.c_int),
        "ml_gpu_hashagg_graph_stats": ([VP, P(U64), P(U64)], C.c_int),
        "ml_gpu_card_features": ([VP, P(abi.MlColumn), I32, I64, VP, I64, I32, P(abi.MlExpr), I32, VP,
                                  P(C.c_double)], C.c_int),
        "ml_gpu_card_model_create": ([VP, U64, P(VP)], C.c_int),
        "ml_gpu_card_model_params": ([VP, VP, VP], C.c_int),
        "ml_gpu_card_model_step": ([VP, VP, VP, I32, C.c_float, P(C.c_float)], C.c_int),
        "ml_gpu_card_model_train": ([VP, VP, VP, I64, I32, I32, C.c_float, U64, P(C.c_float)], C.c_int),
        "ml_gpu_card_model_predict": ([VP, VP, I64, VP], C.c_int),
        "ml_gpu_card_model_destroy": ([VP], C.c_int),
        "ml_gpu_batch_upload": ([VP, P(abi.MlColumn), I32, I64, P(VP)], C.c_int),
        "ml_gpu_batch_num_rows": ([VP, P(I64)], C.c_int),
        "ml_gpu_batch_num_columns": ([VP, P(I32)], C.c_int),
        "ml_gpu_batch_columns": ([VP, P(abi.MlColumn), I32], C.c_int),
        "ml_gpu_batch_column_info": ([VP, I32, P(I32), P(I64), P(I32)], C.c_int),
        "ml_gpu_batch_fetch": ([VP, I32, VP, VP, VP], C.c_int),
        "ml_gpu_batch_destroy": ([VP], C.c_int),
        "ml_gpu_filter": ([VP, P(abi.MlExpr), P(abi.MlColumn), I32, I64, VP, I64, I32, VP, P(I64)], C.c_int),
        "ml_gpu_filter_static": ([VP, P(abi.MlExpr), P(abi.MlColumn), I32, I64, VP, I64, VP, P(I64)], C.c_int),
        "ml_gpu_project": ([VP, P(abi.MlExpr), P(abi.MlColumn), I32, I64, P(VP)], C.c_int),
        "ml_gpu_hash_columns": ([VP, P(abi.MlColumn), I32, I64, VP, I64, I32, VP], C.c_int),
        "ml_gpu_partition": ([VP, P(abi.MlColumn), I32, I64, VP, I32, I32, P(VP), VP], C.c_int),
        "ml_gpu_hashagg_create": ([VP, P(abi.MlPipeOp), I32, VP, I32, P(abi.MlExpr), I32, P(abi.MlAggSpec), I32,
                                   I64, P(VP)], C.c_int),
        "ml_gpu_hashagg_local_create": ([VP, P(VP)], C.c_int),
        "ml_gpu_hashagg_sink": ([VP, P(abi.MlColumn), I32, I64, VP, I64], C.c_int),
        "ml_gpu_hashagg_combine": ([VP], C.c_int),
        "ml_gpu_hashagg_finalize": ([VP, P(VP)], C.c_int),
        "ml_gpu_hashagg_stats": ([VP, P(I64), P(I64), P(I64)], C.c_int),
        "ml_gpu_hashagg_spill_stats": ([VP, P(I64), P(I64)], C.c_int),
        "ml_gpu_hashagg_destroy": ([VP], C.c_int),
        "ml_gpu_join_build_create": ([VP, P(abi.MlPipeOp), I32, VP, I32, P(abi.MlExpr), I32, P(VP)], C.c_int),
        "ml_gpu_join_build_local_create": ([VP, P(VP)], C.c_int),
        "ml_gpu_join_build_sink": ([VP, P(abi.MlColumn), I32, I64, VP, I64], C.c_int),
        "ml_gpu_join_build_combine": ([VP], C.c_int),
        "ml_gpu_join_build_finalize": ([VP, P(VP)], C.c_int),
        "ml_gpu_join_table_stats": ([VP, P(I64), P(I64), P(I64)], C.c_int),
        "ml_gpu_join_build_destroy": ([VP], C.c_int),
        "ml_gpu_join_probe": ([VP, VP, P(abi.MlExpr), I32, P(abi.MlColumn), I32, I64, VP, I64, I32, VP, VP, I64,
                               P(I64)], C.c_int),
        "ml_gpu_topn_create": ([VP, P(abi.MlPipeOp), I32, VP, I32, P(abi.MlSortKey), I32, I64, P(VP)], C.c_int),
        "ml_gpu_topn_local_create": ([VP, P(VP)], C.c_int),
        "ml_gpu_topn_sink": ([VP, P(abi.MlColumn), I32, I64, VP, I64], C.c_int),
        "ml_gpu_topn_combine": ([VP], C.c_int),
        "ml_gpu_topn_finalize": ([VP, P(VP)], C.c_int),
        "ml_gpu_topn_destroy": ([VP], C.c_int),
        "ml_gpu_parquet_decode": ([VP, VP, I64, I32, I32, I32, I32, I32, I64, I32, P(VP)], C.c_int),
        "ml_gpu_query_create": ([VP, P(VP)], C.c_int),
        "ml_gpu_query_add_build": ([VP, VP, P(abi.MlColumn), I32, I64, P(VP)], C.c_int),
        "ml_gpu_query_set_aggregate": ([VP, VP, P(abi.MlColumn), I32, I64], C.c_int),
        "ml_gpu_query_set_topn": ([VP, P(abi.MlSortKey), I32, I64], C.c_int),
        "ml_gpu_query_run": ([VP, P(VP)], C.c_int),
        "ml_gpu_query_run_host": ([VP, P(I64)], C.c_int),
        "ml_gpu_query_result": ([VP, I32, VP, VP, P(I32)], C.c_int),
        "ml_gpu_query_stats": ([VP, P(I64), P(I64), P(I32), C.c_char_p, I32], C.c_int),
        "ml_gpu_query_destroy": ([VP], C.c_int),
    }
    for name, (args, res) in sigs.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


LIB = _load()


def _check(status: int):
    if status == abi.OK:
        return
    msg = LIB.ml_gpu_last_error().decode(errors="replace")
    if status == abi.ERR_BUDGET:
        op = C.create_string_buffer(128)
        r, u, l = C.c_uint64(), C.c_uint64(), C.c_uint64()
        LIB.ml_gpu_last_budget_error(op, 128, C.byref(r), C.byref(u), C.byref(l))
        raise ResourcesExhausted(status, msg, op.value.decode(), r.value, u.value, l.value)
    if status == abi.ERR_STALE_PLAN:
        raise StalePlan(status, msg)
    raise MiniLakeError(status, msg)


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


SPILL = 8  # ML_CTX_SPILL
PROFILE = 2  # ML_CTX_PROFILE
INTERPRET = 4  # ML_CTX_INTERPRET: ahead-of-time interpreter kernels instead of specialized ones


class Context:
    """One device + the query-wide HBM budget (ExecConfig / MemoryPool)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, flags: int = 0):
        self.h = None
        self._children = weakref.WeakSet()  # batches and sinks that must go before the context
        h = C.c_void_p()
        _check(LIB.ml_gpu_ctx_create(device, hbm_budget, flags, C.byref(h)))
        self.h = h

    def _own(self, obj):
        self._children.add(obj)
        return obj

    def close(self):
        if self.h:
            for child in list(self._children):
                child.close()
            LIB.ml_gpu_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pool_stats(self):
        u, p, l = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(LIB.ml_gpu_pool_stats(self.h, C.byref(u), C.byref(p), C.byref(l)))
        return u.value, p.value, l.value

    def synchronize(self):
        _check(LIB.ml_gpu_ctx_synchronize(self.h))

    def kernel_launches(self) -> int:
        c = C.c_uint64()
        _check(LIB.ml_gpu_kernel_launches(self.h, C.byref(c)))
        return c.value

    def profile(self, kernel: str, reset: bool = False):
        """(launches, total device ms) of a kernel family; needs flags=PROFILE."""
        n, ms = C.c_uint64(), C.c_double()
        _check(LIB.ml_gpu_profile_read(self.h, kernel.encode(), C.byref(n), C.byref(ms), int(reset)))
        return n.value, ms.value

    def upload(self, cols: Sequence[HostColumn]) -> "DeviceBatch":
        keep = abi.Keep()
        arr = (abi.MlColumn * max(len(cols), 1))()
        for i, c in enumerate(cols):
            arr[i] = c.to_ml()
        n = len(cols[0]) if cols else 0
        h = C.c_void_p()
        _check(LIB.ml_gpu_batch_upload(self.h, arr, len(cols), n, C.byref(h)))
        del keep
        return DeviceBatch(self, h)

    def upload_table(self, table: Table) -> List["DeviceBatch"]:
        return [self.upload(rg) for rg in table.row_groups]


class DeviceBatch:
    """Columns resident in HBM (an uploaded table or a sink's output)."""

    def __init__(self, ctx: Context, h):
        self.ctx, self.h = ctx, h
        ctx._own(self)

    def close(self):
        if self.h:
            LIB.ml_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_rows(self) -> int:
        n = C.c_int64()
        _check(LIB.ml_gpu_batch_num_rows(self.h, C.byref(n)))
        return n.value

    @property
    def num_columns(self) -> int:
        n = C.c_int32()
        _check(LIB.ml_gpu_batch_num_columns(self.h, C.byref(n)))
        return n.value

    def ml_columns(self):
        n = self.num_columns
        arr = (abi.MlColumn * max(n, 1))()
        _check(LIB.ml_gpu_batch_columns(self.h, arr, n))
        return arr, n

    @property
    def types(self) -> List[int]:
        out = []
        for i in range(self.num_columns):
            t = C.c_int32()
            _check(LIB.ml_gpu_batch_column_info(self.h, i, C.byref(t), None, None))
            out.append(t.value)
        return out

    def fetch(self) -> List[HostColumn]:
        n = self.num_rows
        cols = []
        words = (n + 63) // 64
        for i in range(self.num_columns):
            t, sb, hv = C.c_int32(), C.c_int64(), C.c_int32()
            _check(LIB.ml_gpu_batch_column_info(self.h, i, C.byref(t), C.byref(sb), C.byref(hv)))
            valid = np.zeros(max(words, 1), dtype=np.uint64)
            if t.value == abi.UTF8:
                data = np.zeros(max(sb.value, 1), dtype=np.uint8)
                off = np.zeros(n + 1, dtype=np.uint32)
                _check(LIB.ml_gpu_batch_fetch(self.h, i, _ptr(data), _ptr(off), _ptr(valid)))
                col = HostColumn(abi.UTF8, data[:sb.value], offsets=off)
            else:
                data = np.zeros(max(n, 1), dtype=abi.NP_DTYPE[t.value])
                _check(LIB.ml_gpu_batch_fetch(self.h, i, _ptr(data), None, _ptr(valid)))
                col = HostColumn(t.value, data[:n])
            if hv.value:
                col.validity = valid[:words]
            cols.append(col)
        return cols


def parquet_decode(ctx: Context, chunk, physical_type: int, type_length: int, conversion: int, scale: int,
                   codec: int, num_rows: int, max_def: int) -> DeviceBatch:
    """One Parquet column chunk (its pages as stored in the file) decoded on the device into a
    one-column batch (read_column_chunk, parquet_reader.rs:215-294)."""
    buf = np.frombuffer(chunk, dtype=np.uint8) if not isinstance(chunk, np.ndarray) else chunk
    h = C.c_void_p()
    _check(LIB.ml_gpu_parquet_decode(ctx.h, buf.ctypes.data if len(buf) else None, len(buf), physical_type, type_length,
                                     conversion, scale, codec, num_rows, max_def, C.byref(h)))
    return DeviceBatch(ctx, h)


def partition(ctx: Context, cols, key_cols: Sequence[int], nparts: int):
    """Rows grouped by hash_columns(key columns) % nparts (stable): (DeviceBatch, counts)."""
    arr, nc, n, keep = _cols_arg(cols)
    keys = (C.c_int32 * max(len(key_cols), 1))(*key_cols)
    counts = np.zeros(max(nparts, 1), dtype=np.int64)
    h = C.c_void_p()
    _check(LIB.ml_gpu_partition(ctx.h, arr, nc, n, keys, len(key_cols), nparts, C.byref(h), _ptr(counts)))
    return DeviceBatch(ctx, h), counts[:nparts]


class _CudaArray:
    """__cuda_array_interface__ of a device buffer, so torch can view it without a copy."""

    _TYPESTR = {abi.BOOL: "|u1", abi.INT32: "<i4", abi.DATE: "<i4", abi.INT64: "<i8", abi.FLOAT64: "<f8"}

    def __init__(self, ptr: int, n: int, dtype: int, owner):
        self.owner = owner
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": self._TYPESTR[dtype], "data": (ptr, False),
                                         "version": 3, "strides": None}


def column_tensor(batch: "DeviceBatch", i: int):
    """Torch view (no copy) of fixed-width column i of a device batch; the batch must outlive it."""
    import torch
    arr, _ = batch.ml_columns()
    c = arr[i]
    if c.dtype not in _CudaArray._TYPESTR:
        raise TypeError("column_tensor: fixed-width columns only")
    n = batch.num_rows
    if n == 0:
        return torch.empty(0, dtype={abi.BOOL: torch.uint8, abi.INT32: torch.int32, abi.DATE: torch.int32,
                                     abi.INT64: torch.int64, abi.FLOAT64: torch.float64}[c.dtype], device="cuda")
    return torch.as_tensor(_CudaArray(c.data, n, c.dtype, batch), device="cuda")


def _cols_arg(cols, location=None):
    """HostColumn list / DeviceBatch / (MlColumn array, n) -> (MlColumn*, ncols, nrows, keep)."""
    if isinstance(cols, DeviceBatch):
        arr, n = cols.ml_columns()
        return arr, n, cols.num_rows, cols
    if isinstance(cols, tuple):
        arr, n, nrows = cols
        return arr, n, nrows, None
    arr = (abi.MlColumn * max(len(cols), 1))()
    for i, c in enumerate(cols):
        arr[i] = c.to_ml()
    return arr, len(cols), (len(cols[0]) if cols else 0), cols


def _sel_arg(sel):
    if sel is None:
        return None, 0, None
    s = np.ascontiguousarray(sel, dtype=np.uint32)
    return s.ctypes.data, len(s), s


# ---- streaming operators ---------------------------------------------------------------
class FilterOperator:
    """WHERE: refines the selection vector (operators/filter.rs:19-25)."""

    def __init__(self, ctx: Context, predicate: abi.Expr):
        self.ctx, self.pred = ctx, predicate

    def execute(self, cols, sel=None) -> np.ndarray:
        keep = abi.Keep()
        e = abi.encode_expr(self.pred, abi.BOOL, keep)
        arr, nc, n, _hold = _cols_arg(cols)
        sp, ns, _s = _sel_arg(sel)
        out = np.zeros(max(ns if sel is not None else n, 1), dtype=np.uint32)
        k = C.c_int64()
        _check(LIB.ml_gpu_filter(self.ctx.h, C.byref(e), arr, nc, n, sp, ns, abi.LOC_HOST, _ptr(out), C.byref(k)))
        return out[:k.value]


class ProjectionOperator:
    """SELECT expr: one output column over all physical rows (projection.rs:21-32)."""

    def __init__(self, ctx: Context, expr: abi.Expr, out_type: int):
        self.ctx, self.expr, self.out_type = ctx, expr, out_type

    def execute(self, cols) -> DeviceBatch:
        keep = abi.Keep()
        e = abi.encode_expr(self.expr, self.out_type, keep)
        arr, nc, n, _hold = _cols_arg(cols)
        h = C.c_void_p()
        _check(LIB.ml_gpu_project(self.ctx.h, C.byref(e), arr, nc, n, C.byref(h)))
        return DeviceBatch(self.ctx, h)


def hash_columns(ctx: Context, cols, sel=None) -> np.ndarray:
    """kernels/hash.rs:16-23 on the device."""
    arr, nc, n, _hold = _cols_arg(cols)
    sp, ns, _s = _sel_arg(sel)
    out = np.zeros(max(ns if sel is not None else n, 1), dtype=np.uint64)
    _check(LIB.ml_gpu_hash_columns(ctx.h, arr, nc, n, sp, ns, abi.LOC_HOST, _ptr(out)))
    return out[:(ns if sel is not None else n)]


class LocalSink:
    """The per-thread half of a sink (pipeline.rs:69-79); owns a CUDA stream."""

    def __init__(self, owner, h, fn_sink, fn_combine):
        self.owner, self.h, self._sink, self._combine = owner, h, fn_sink, fn_combine

    def sink(self, cols, sel=None):
        """LocalSink::sink: push one batch (HostColumns, a DeviceBatch, or an
        (MlColumn array, ncols, nrows) tuple) with an optional selection vector."""
        arr, nc, n, _hold = _cols_arg(cols)
        sp, ns, _s = _sel_arg(sel)
        _check(self._sink(self.h, arr, nc, n, sp, ns))

    def combine(self):
        """LocalSink::combine: merge into the global state (ends this handle)."""
        if self.h:
            _check(self._combine(self.h))
            self.h = None


def _local(sink, create, fn_sink, fn_combine) -> LocalSink:
    h = C.c_void_p()
    _check(create(sink.h, C.byref(h)))
    return LocalSink(sink, h, fn_sink, fn_combine)


# ---- sinks ------------------------------------------------------------------------------------
class HashAggregateSink:
    """GROUP BY (operators/aggregate/hash.rs:285-484); no GROUP BY = ungrouped (ungrouped.rs)."""

    def __init__(self, ctx: Context, input_types: Sequence[int], group_exprs: Sequence[tuple],
                 aggs: Sequence[abi.AggSpec], prologue: Sequence[abi.PipeOp] = (), size_hint: int = 0):
        self.ctx = ctx
        keep = abi.Keep()
        ops, nops = abi.encode_ops(prologue, keep)
        g, ng = abi.encode_exprs(group_exprs, keep)
        a, na = abi.encode_aggs(aggs, keep)
        types = np.asarray(input_types, dtype=np.int32)
        self.input_types = types
        h = C.c_void_p()
        _check(LIB.ml_gpu_hashagg_create(ctx.h, ops, nops, _ptr(types), len(types), g, ng, a, na, size_hint,
                                          C.byref(h)))
        self.h = h
        ctx._own(self)

    def create_local(self):
        return _local(self, LIB.ml_gpu_hashagg_local_create, LIB.ml_gpu_hashagg_sink, LIB.ml_gpu_hashagg_combine)

    # ---- resident use (serving): one query after another through the same device state ----
    def rebind(self, prologue: Sequence[abi.PipeOp], group_exprs: Sequence[tuple], aggs: Sequence[abi.AggSpec]):
        """New constants (same pipeline shape) for the next query."""
        keep = abi.Keep()
        ops, nops = abi.encode_ops(prologue, keep)
        g, ng = abi.encode_exprs(group_exprs, keep)
        a, na = abi.encode_aggs(aggs, keep)
        _check(LIB.ml_gpu_hashagg_rebind(self.h, ops, nops, _ptr(self.input_types), len(self.input_types), g, ng,
                                         a, na))

    def reset(self):
        _check(LIB.ml_gpu_hashagg_reset(self.h))

    def run_resident(self, cols, reset: bool = True):
        """Sink a device-resident batch (DeviceBatch or MlColumn tuple) as a replayed CUDA graph."""
        arr, nc, n, _hold = _cols_arg(cols)
        _check(LIB.ml_gpu_hashagg_run_resident(self.h, arr, nc, n, int(reset)))

    def graph_stats(self):
        b, r = C.c_uint64(), C.c_uint64()
        _check(LIB.ml_gpu_hashagg_graph_stats(self.h, C.byref(b), C.byref(r)))
        return {"built": b.value, "replayed": r.value}

    def finalize(self) -> DeviceBatch:
        h = C.c_void_p()
        _check(LIB.ml_gpu_hashagg_finalize(self.h, C.byref(h)))
        return DeviceBatch(self.ctx, h)

    def stats(self):
        g, c, r = C.c_int64(), C.c_int64(), C.c_int64()
        _check(LIB.ml_gpu_hashagg_stats(self.h, C.byref(g), C.byref(c), C.byref(r)))
        sp, sg = C.c_int64(), C.c_int64()
        _check(LIB.ml_gpu_hashagg_spill_stats(self.h, C.byref(sp), C.byref(sg)))
        return {"groups": g.value, "capacity": c.value, "resizes": r.value, "spills": sp.value,
                "spilled_groups": sg.value}

    def close(self):
        if self.h:
            LIB.ml_gpu_hashagg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class JoinBuildSink:
    """Build side of the hash join (operators/join.rs:72-242)."""

    def __init__(self, ctx: Context, input_types: Sequence[int], key_exprs: Sequence[tuple],
                 prologue: Sequence[abi.PipeOp] = ()):
        self.ctx = ctx
        keep = abi.Keep()
        ops, nops = abi.encode_ops(prologue, keep)
        k, nk = abi.encode_exprs(key_exprs, keep)
        types = np.asarray(input_types, dtype=np.int32)
        h = C.c_void_p()
        _check(LIB.ml_gpu_join_build_create(ctx.h, ops, nops, _ptr(types), len(types), k, nk, C.byref(h)))
        self.h = h
        self.table = None
        ctx._own(self)

    def create_local(self):
        return _local(self, LIB.ml_gpu_join_build_local_create, LIB.ml_gpu_join_build_sink,
                      LIB.ml_gpu_join_build_combine)

    def finalize(self):
        t = C.c_void_p()
        _check(LIB.ml_gpu_join_build_finalize(self.h, C.byref(t)))
        self.table = t.value
        return self.table

    @property
    def handle(self):
        """The finalized table (JoinTableRef) for a HashJoinProbe / Probe operator."""
        return self.table

    def stats(self):
        r, d, c = C.c_int64(), C.c_int64(), C.c_int64()
        _check(LIB.ml_gpu_join_table_stats(self.table, C.byref(r), C.byref(d), C.byref(c)))
        return {"build_rows": r.value, "distinct_keys": d.value, "capacity": c.value}

    def close(self):
        if self.h:
            LIB.ml_gpu_join_build_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HashJoinProbe:
    """Probe side of the hash join (operators/join.rs:244-337): (probe_row, build_row) pairs."""

    def __init__(self, ctx: Context, table, key_exprs: Sequence[tuple]):
        self.ctx, self.table, self.keys = ctx, table, key_exprs

    def execute(self, cols, sel=None, cap: Optional[int] = None):
        keep = abi.Keep()
        k, nk = abi.encode_exprs(self.keys, keep)
        arr, nc, n, _hold = _cols_arg(cols)
        sp, ns, _s = _sel_arg(sel)
        cap = cap if cap is not None else max(n, 16)
        while True:
            pi = np.zeros(max(cap, 1), dtype=np.uint32)
            bi = np.zeros(max(cap, 1), dtype=np.uint32)
            npairs = C.c_int64()
            st = LIB.ml_gpu_join_probe(self.ctx.h, self.table, k, nk, arr, nc, n, sp, ns, abi.LOC_HOST, _ptr(pi),
                                       _ptr(bi), cap, C.byref(npairs))
            if st == abi.ERR_INVALID and npairs.value > cap:
                cap = npairs.value
                continue
            _check(st)
            return pi[:npairs.value], bi[:npairs.value]


class SortSink:
    """ORDER BY ... [LIMIT n] (operators/sort.rs:85-267); limit None = every row."""

    def __init__(self, ctx: Context, input_types: Sequence[int], keys: Sequence[abi.SortKey], limit: Optional[int],
                 prologue: Sequence[abi.PipeOp] = ()):
        limit = -1 if limit is None else limit
        self.ctx = ctx
        keep = abi.Keep()
        ops, nops = abi.encode_ops(prologue, keep)
        k, nk = abi.encode_sort_keys(keys, keep)
        types = np.asarray(input_types, dtype=np.int32)
        h = C.c_void_p()
        _check(LIB.ml_gpu_topn_create(ctx.h, ops, nops, _ptr(types), len(types), k, nk, limit, C.byref(h)))
        self.h = h
        ctx._own(self)

    def create_local(self):
        return _local(self, LIB.ml_gpu_topn_local_create, LIB.ml_gpu_topn_sink, LIB.ml_gpu_topn_combine)

    def finalize(self) -> DeviceBatch:
        h = C.c_void_p()
        _check(LIB.ml_gpu_topn_finalize(self.h, C.byref(h)))
        return DeviceBatch(self.ctx, h)

    def close(self):
        if self.h:
            LIB.ml_gpu_topn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- learned cardinality estimator ----------------------------------------------------------
CARD_FEATURES, CARD_PARAMS = 72, 13057


def card_features(ctx: Context, cols, keys: Sequence[tuple], sel=None):
    """(72 FP32 features, HyperLogLog estimate) of the key expressions over a morsel's active
    rows; `cols` is a DeviceBatch, a list of HostColumns or an (MlColumn array, ncols, nrows)."""
    keep = abi.Keep()
    k, nk = abi.encode_exprs(keys, keep)
    arr, nc, n, _hold = _cols_arg(cols)
    sp, ns, _s = _sel_arg(sel)
    f = np.zeros(CARD_FEATURES, dtype=np.float32)
    est = C.c_double()
    _check(LIB.ml_gpu_card_features(ctx.h, arr, nc, n, sp, ns, abi.LOC_HOST, k, nk, _ptr(f), C.byref(est)))
    return f, est.value


class Query:
    """A prepared plan over device-resident batches (ml_gpu_query_*, executor.rs:270-288): join
    builds, one hash aggregate probing them, an optional top-N.  The first run() plans through
    the sink calls; later runs replay the whole plan as one CUDA graph.  StalePlan when the data
    no longer fits the plan; MiniLakeError(ERR_UNSUPPORTED) on a second run of a plan the graph
    cannot replay (stats()["why_not"] says why)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self._keep = []  # sinks and batches the plan reads
        h = C.c_void_p()
        _check(LIB.ml_gpu_query_create(ctx.h, C.byref(h)))
        self.h = h
        ctx._own(self)

    def add_build(self, sink: "JoinBuildSink", cols):
        """Run the build pipeline now; returns the table handle for Probe operators."""
        arr, nc, n, hold = _cols_arg(cols)
        t = C.c_void_p()
        _check(LIB.ml_gpu_query_add_build(self.h, sink.h, arr, nc, n, C.byref(t)))
        sink.table = t.value
        self._keep += [sink, cols, hold, arr]
        return t.value

    def set_aggregate(self, sink: "HashAggregateSink", cols):
        arr, nc, n, hold = _cols_arg(cols)
        _check(LIB.ml_gpu_query_set_aggregate(self.h, sink.h, arr, nc, n))
        self._keep += [sink, cols, hold, arr]

    def set_topn(self, keys: Sequence[abi.SortKey], limit: int):
        keep = abi.Keep()
        k, nk = abi.encode_sort_keys(keys, keep)
        _check(LIB.ml_gpu_query_set_topn(self.h, k, nk, limit))
        self._topn = True

    def run(self) -> DeviceBatch:
        out = C.c_void_p()
        _check(LIB.ml_gpu_query_run(self.h, C.byref(out)))
        return DeviceBatch(self.ctx, out)

    def run_host(self) -> List[HostColumn]:
        """One run with the result in host memory: replays of a top-N plan copy it inside the
        graph (ml_gpu_query_run_host); the planning run and other plans fetch a device batch."""
        if getattr(self, "_types", None) is None:
            b = self.run()
            cols = b.fetch()
            b.close()
            if getattr(self, "_topn", False) and self.stats()["why_not"] == "":
                self._types = [c.dtype for c in cols]
            return cols
        n = C.c_int64()
        _check(LIB.ml_gpu_query_run_host(self.h, C.byref(n)))
        k = n.value
        out = []
        for i, t in enumerate(self._types):
            vals = np.empty(max(k, 1), dtype=abi.NP_DTYPE[t])
            valid = np.zeros(max((k + 63) // 64, 1), dtype=np.uint64)
            hv = C.c_int32()
            _check(LIB.ml_gpu_query_result(self.h, i, _ptr(vals), _ptr(valid), C.byref(hv)))
            col = HostColumn(t, vals[:k])
            if hv.value:
                col.validity = valid[:(k + 63) // 64]
            out.append(col)
        return out

    def stats(self):
        r, p, k = C.c_int64(), C.c_int64(), C.c_int32()
        why = C.create_string_buffer(256)
        _check(LIB.ml_gpu_query_stats(self.h, C.byref(r), C.byref(p), C.byref(k), why, 256))
        return {"runs": r.value, "replays": p.value, "kernels": k.value, "why_not": why.value.decode()}

    def close(self):
        if self.h:
            LIB.ml_gpu_query_destroy(self.h)
            self.h = None
        self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CardinalityModel:
    """FP32 MLP 72-64-64-64-1 predicting log2(distinct keys), trained and run by the library's
    own CUDA kernels (forward, backward, Adam)."""

    def __init__(self, ctx: Context, seed: int = 0):
        self.ctx = ctx
        h = C.c_void_p()
        _check(LIB.ml_gpu_card_model_create(ctx.h, seed, C.byref(h)))
        self.h = h
        ctx._own(self)

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(CARD_PARAMS, dtype=np.float32)
        _check(LIB.ml_gpu_card_model_params(self.h, _ptr(out), None))
        return out

    @params.setter
    def params(self, values):
        v = np.ascontiguousarray(values, dtype=np.float32)
        assert v.shape == (CARD_PARAMS,)
        _check(LIB.ml_gpu_card_model_params(self.h, None, _ptr(v)))

    def step(self, x, y, lr: float = 1e-3) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        loss = C.c_float()
        _check(LIB.ml_gpu_card_model_step(self.h, _ptr(x), _ptr(y), len(y), lr, C.byref(loss)))
        return loss.value

    def train(self, x, y, epochs: int = 200, batch: int = 64, lr: float = 1e-3, seed: int = 0) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        loss = C.c_float()
        _check(LIB.ml_gpu_card_model_train(self.h, _ptr(x), _ptr(y), len(y), epochs, batch, lr, seed, C.byref(loss)))
        return loss.value

    def predict(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, CARD_FEATURES)
        out = np.zeros(len(x), dtype=np.float32)
        _check(LIB.ml_gpu_card_model_predict(self.h, _ptr(x), len(x), _ptr(out)))
        return out

    def close(self):
        if self.h:
            LIB.ml_gpu_card_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
