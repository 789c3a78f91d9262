"""TEST INFRASTRUCTURE — ctypes binding of the CPU oracle (``oracle/build/liborc.so``).

The oracle is a C++17 restatement of MiniLake's CPU hot path (the reference is
Rust; no toolchain here).  Only the tests, ``__graft_entry__.smoke()`` and
bench.py's CPU baseline / reference arm use it, as the checker and as the
timed CPU baseline; the product path never calls it.

``OracleEngine`` has the same interface as ``minilake_b200.engine.GpuEngine``
so one query plan runs on both.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import List, Sequence

import numpy as np

from minilake_b200 import abi
from minilake_b200.columns import HostColumn, Table

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liborc.so")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    P, I32, I64, U64, VP = C.POINTER, C.c_int32, C.c_int64, C.c_uint64, C.c_void_p
    sigs = {
        "orc_last_error": ([], C.c_char_p),
        "orc_last_budget_error": ([C.c_char_p, C.c_size_t, P(U64), P(U64), P(U64)], C.c_int),
        "orc_hash_u64": ([U64], U64),
        "orc_combine": ([U64, U64], U64),
        "orc_hash_bytes": ([C.c_char_p, C.c_size_t], U64),
        "orc_fold_mul": ([U64, U64], U64),
        "orc_swar_match_tag": ([U64, C.c_uint8], U64),
        "orc_swar_match_empty": ([U64], U64),
        "orc_swiss_batches": ([VP, VP, C.c_int, C.c_int, VP, P(I64), P(I64)], C.c_int),
        "orc_pool_script": ([U64, VP, C.c_int, VP, VP, VP], C.c_int),
        "orc_filter": ([P(abi.MlExpr), P(abi.MlColumn), C.c_int, I64, VP, I64, VP, P(I64)], C.c_int),
        "orc_project": ([P(abi.MlExpr), P(abi.MlColumn), C.c_int, I64, P(VP)], C.c_int),
        "orc_hash_columns": ([P(abi.MlColumn), C.c_int, I64, VP, I64, VP], C.c_int),
        "orc_hashagg_run": ([P(abi.MlColumn), C.c_int, C.c_int, VP, P(abi.MlPipeOp), C.c_int, P(abi.MlExpr), C.c_int,
                             P(abi.MlAggSpec), C.c_int, C.c_int, I64, U64, P(VP)], C.c_int),
        "orc_join_build_run": ([P(abi.MlColumn), C.c_int, C.c_int, VP, P(abi.MlPipeOp), C.c_int, P(abi.MlExpr),
                                C.c_int, C.c_int, I64, U64, P(VP)], C.c_int),
        "orc_join_destroy": ([VP], C.c_int),
        "orc_join_stats": ([VP, P(I64), P(I64), P(I64)], C.c_int),
        "orc_join_probe": ([VP, P(abi.MlExpr), C.c_int, P(abi.MlColumn), C.c_int, I64, VP, I64, VP, VP, I64, P(I64)],
                           C.c_int),
        "orc_topn_run": ([P(abi.MlColumn), C.c_int, C.c_int, VP, P(abi.MlPipeOp), C.c_int, P(abi.MlSortKey),
                          C.c_int, I64, C.c_int, I64, P(VP)], C.c_int),
        "orc_batch_num_rows": ([VP, P(I64)], C.c_int),
        "orc_batch_num_columns": ([VP, P(I32)], C.c_int),
        "orc_batch_column_info": ([VP, I32, P(I32), P(I64), P(I32)], C.c_int),
        "orc_batch_fetch": ([VP, I32, VP, VP, VP], C.c_int),
        "orc_batch_columns": ([VP, P(abi.MlColumn), I32], C.c_int),
        "orc_batch_destroy": ([VP], C.c_int),
    }
    for name, (args, res) in sigs.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


LIB = _load()


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class OracleBudgetError(OracleError):
    def __init__(self, code, msg, operator, requested, used, limit):
        super().__init__(code, msg)
        self.operator, self.requested, self.used, self.limit = operator, requested, used, limit


def check(st):
    if st == abi.OK:
        return
    msg = LIB.orc_last_error().decode(errors="replace")
    if st == abi.ERR_BUDGET:
        op = C.create_string_buffer(128)
        r, u, l = C.c_uint64(), C.c_uint64(), C.c_uint64()
        LIB.orc_last_budget_error(op, 128, C.byref(r), C.byref(u), C.byref(l))
        raise OracleBudgetError(st, msg, op.value.decode(), r.value, u.value, l.value)
    raise OracleError(st, msg)


class OBatch:
    """A result batch owned by the oracle."""

    def __init__(self, h):
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            LIB.orc_batch_destroy(self.h)
            self.h = None

    @property
    def num_rows(self):
        n = C.c_int64()
        check(LIB.orc_batch_num_rows(self.h, C.byref(n)))
        return n.value

    @property
    def num_columns(self):
        n = C.c_int32()
        check(LIB.orc_batch_num_columns(self.h, C.byref(n)))
        return n.value

    def fetch(self) -> List[HostColumn]:
        n = self.num_rows
        words = (n + 63) // 64
        out = []
        for i in range(self.num_columns):
            t, sb, hv = C.c_int32(), C.c_int64(), C.c_int32()
            check(LIB.orc_batch_column_info(self.h, i, C.byref(t), C.byref(sb), C.byref(hv)))
            valid = np.zeros(max(words, 1), dtype=np.uint64)
            if t.value == abi.UTF8:
                data = np.zeros(max(sb.value, 1), dtype=np.uint8)
                off = np.zeros(n + 1, dtype=np.uint32)
                check(LIB.orc_batch_fetch(self.h, i, data.ctypes.data, off.ctypes.data, valid.ctypes.data))
                col = HostColumn(abi.UTF8, data[:sb.value], offsets=off)
            else:
                data = np.zeros(max(n, 1), dtype=abi.NP_DTYPE[t.value])
                check(LIB.orc_batch_fetch(self.h, i, data.ctypes.data, None, valid.ctypes.data))
                col = HostColumn(t.value, data[:n])
            if hv.value:
                col.validity = valid[:words]
            out.append(col)
        return out

    def as_source(self):
        """One morsel holding this batch's columns (a BatchBuffer replay source)."""
        nc = self.num_columns
        arr = (abi.MlColumn * max(nc, 1))()
        check(LIB.orc_batch_columns(self.h, arr, nc))
        rows = np.array([self.num_rows], dtype=np.int64)
        return arr, 1, nc, rows, self


class OracleJoin:
    def __init__(self, h):
        self.h = h

    @property
    def handle(self):
        return self.h

    def stats(self):
        r, d, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(LIB.orc_join_stats(self.h, C.byref(r), C.byref(d), C.byref(c)))
        return {"build_rows": r.value, "distinct_keys": d.value, "capacity": c.value}

    def __del__(self):
        if getattr(self, "h", None):
            LIB.orc_join_destroy(self.h)
            self.h = None


def _source(src, keep):
    if isinstance(src, Table):
        return src.morsels(keep)
    if isinstance(src, OBatch):
        arr, nm, nc, rows, hold = src.as_source()
        keep.add(hold)
        keep.add(rows)
        return arr, nm, nc, rows
    if isinstance(src, list):  # a single batch of host columns
        t = Table("batch", [str(i) for i in range(len(src))], [src])
        return t.morsels(keep)
    raise TypeError(src)


class OracleEngine:
    """Runs plans on the CPU oracle with the reference's morsel-driven threading."""

    name = "oracle"

    def __init__(self, threads: int = 1, batch_size: int = 2048, memory_limit: int = 0):
        self.threads, self.batch_size, self.memory_limit = threads, batch_size, memory_limit

    def join_build(self, source, input_types, key_exprs, prologue=()):
        keep = abi.Keep()
        arr, nm, nc, rows = _source(source, keep)
        ops, nops = abi.encode_ops(prologue, keep)
        k, nk = abi.encode_exprs(key_exprs, keep)
        h = C.c_void_p()
        check(LIB.orc_join_build_run(arr, nm, nc, rows.ctypes.data, ops, nops, k, nk, self.threads,
                                     self.batch_size, self.memory_limit, C.byref(h)))
        return OracleJoin(h.value)

    def hashagg(self, source, input_types, group_exprs, aggs, prologue=(), size_hint=0):
        keep = abi.Keep()
        arr, nm, nc, rows = _source(source, keep)
        ops, nops = abi.encode_ops(prologue, keep)
        g, ng = abi.encode_exprs(group_exprs, keep)
        a, na = abi.encode_aggs(aggs, keep)
        h = C.c_void_p()
        check(LIB.orc_hashagg_run(arr, nm, nc, rows.ctypes.data, ops, nops, g, ng, a, na, self.threads,
                                  self.batch_size, self.memory_limit, C.byref(h)))
        return OBatch(h.value)

    def topn(self, source, input_types, keys, limit, prologue=()):
        keep = abi.Keep()
        arr, nm, nc, rows = _source(source, keep)
        ops, nops = abi.encode_ops(prologue, keep)
        k, nk = abi.encode_sort_keys(keys, keep)
        h = C.c_void_p()
        check(LIB.orc_topn_run(arr, nm, nc, rows.ctypes.data, ops, nops, k, nk, -1 if limit is None else limit,
                               self.threads,
                               self.batch_size, C.byref(h)))
        return OBatch(h.value)

    @staticmethod
    def fetch(batch) -> List[HostColumn]:
        return batch.fetch()

    @staticmethod
    def num_rows(batch) -> int:
        return batch.num_rows


# ---- single-batch helpers ------------------------------------------------------------------
def _cols(cols: Sequence[HostColumn]):
    arr = (abi.MlColumn * max(len(cols), 1))()
    for i, c in enumerate(cols):
        arr[i] = c.to_ml()
    return arr, len(cols), (len(cols[0]) if cols else 0)


def filter_rows(pred, cols, sel=None):
    keep = abi.Keep()
    e = abi.encode_expr(pred, abi.BOOL, keep)
    arr, nc, n = _cols(cols)
    s = None if sel is None else np.ascontiguousarray(sel, dtype=np.uint32)
    out = np.zeros(max(n if s is None else len(s), 1), dtype=np.uint32)
    k = C.c_int64()
    check(LIB.orc_filter(C.byref(e), arr, nc, n, None if s is None else s.ctypes.data,
                         0 if s is None else len(s), out.ctypes.data, C.byref(k)))
    return out[:k.value]


def project(expr, out_type, cols) -> List[HostColumn]:
    keep = abi.Keep()
    e = abi.encode_expr(expr, out_type, keep)
    arr, nc, n = _cols(cols)
    h = C.c_void_p()
    check(LIB.orc_project(C.byref(e), arr, nc, n, C.byref(h)))
    return OBatch(h.value).fetch()


def hash_columns(cols, sel=None):
    arr, nc, n = _cols(cols)
    s = None if sel is None else np.ascontiguousarray(sel, dtype=np.uint32)
    m = n if s is None else len(s)
    out = np.zeros(max(m, 1), dtype=np.uint64)
    check(LIB.orc_hash_columns(arr, nc, n, None if s is None else s.ctypes.data, 0 if s is None else len(s),
                               out.ctypes.data))
    return out[:m]


def join_probe(join: OracleJoin, key_exprs, cols, sel=None):
    keep = abi.Keep()
    k, nk = abi.encode_exprs(key_exprs, keep)
    arr, nc, n = _cols(cols)
    s = None if sel is None else np.ascontiguousarray(sel, dtype=np.uint32)
    cap = max(n, 16)
    while True:
        pi = np.zeros(cap, dtype=np.uint32)
        bi = np.zeros(cap, dtype=np.uint32)
        npairs = C.c_int64()
        st = LIB.orc_join_probe(join.h, k, nk, arr, nc, n, None if s is None else s.ctypes.data,
                                0 if s is None else len(s), pi.ctypes.data, bi.ctypes.data, cap, C.byref(npairs))
        if st == abi.ERR_INVALID and npairs.value > cap:
            cap = npairs.value
            continue
        check(st)
        return pi[:npairs.value], bi[:npairs.value]


def swiss_batches(batches: Sequence[Sequence[int]], hash_mode: int):
    keys = np.concatenate([np.asarray(b, dtype=np.uint64) for b in batches]) if batches else np.zeros(0, np.uint64)
    sizes = np.array([len(b) for b in batches], dtype=np.int64)
    out = np.zeros(max(len(keys), 1), dtype=np.uint32)
    ln, cap = C.c_int64(), C.c_int64()
    check(LIB.orc_swiss_batches(keys.ctypes.data if len(keys) else None, sizes.ctypes.data if len(sizes) else None,
                                len(batches), hash_mode, out.ctypes.data, C.byref(ln), C.byref(cap)))
    return out[:len(keys)], ln.value, cap.value


def pool_script(limit: int, ops):
    arr = np.asarray(ops, dtype=np.int64).reshape(-1)
    n = len(ops)
    res = np.zeros(max(n, 1), dtype=np.int32)
    used = np.zeros(max(n, 1), dtype=np.uint64)
    peak = np.zeros(max(n, 1), dtype=np.uint64)
    check(LIB.orc_pool_script(limit, arr.ctypes.data, n, res.ctypes.data, used.ctypes.data, peak.ctypes.data))
    return res[:n], used[:n], peak[:n]
