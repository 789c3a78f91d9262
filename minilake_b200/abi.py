"""ctypes mirror of ``include/minilake_gpu.h``.

The structs describe borrowed column views, prefix-serialized expression trees
(MiniLake's ``PhysicalExpr``, crates/minilake-exec/src/expr/mod.rs:109-173),
aggregate specs (``AggregateExpr``, operators/aggregate/mod.rs:22-31), sort
keys (``SortKey``, operators/sort.rs:25-32) and the streaming operators that can
be fused in front of a sink (Filter / Projection / HashJoinProbe).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, List, Optional, Sequence

import numpy as np

# status codes (crates/minilake-core/src/error.rs:8-48)
OK, ERR_INVALID, ERR_BUDGET, ERR_CUDA, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_INTERNAL, ERR_STALE_PLAN = range(8)

# data types (crates/minilake-core/src/types.rs:15-28)
BOOL, INT32, INT64, FLOAT64, DATE, UTF8, NULL = range(7)
TYPE_NAMES = {BOOL: "BOOLEAN", INT32: "INT32", INT64: "INT64", FLOAT64: "DOUBLE", DATE: "DATE",
              UTF8: "VARCHAR", NULL: "NULL"}
NP_DTYPE = {BOOL: np.uint8, INT32: np.int32, INT64: np.int64, FLOAT64: np.float64, DATE: np.int32}

ENC_PLAIN, ENC_DICT = 0, 1
LOC_HOST, LOC_DEVICE = 0, 1

# BinaryOp (expr/mod.rs:20-47)
(ADD, SUB, MUL, DIV, MOD, EQ, NOTEQ, LT, LTEQ, GT, GTEQ, AND, OR) = range(13)
# PhysicalExpr variants
(E_COLUMN, E_LITERAL, E_BINARY, E_NOT, E_NEGATE, E_IS_NULL, E_LIKE, E_IN_LIST, E_CASE,
 E_CAST) = range(10)
# AggregateFunction (accumulator.rs:25-38)
COUNT_STAR, COUNT, SUM, AVG, MIN, MAX = range(6)
# streaming operators
PIPE_FILTER, PIPE_PROJECT, PIPE_PROBE = range(3)


class MlColumn(C.Structure):
    _fields_ = [
        ("dtype", C.c_int32), ("encoding", C.c_int32), ("location", C.c_int32), ("_pad", C.c_int32),
        ("len", C.c_int64), ("data", C.c_void_p), ("offsets", C.c_void_p), ("validity", C.c_void_p),
        ("dict_len", C.c_int64), ("dict_offsets", C.c_void_p), ("dict_data", C.c_void_p),
    ]


class MlExprNode(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("op", C.c_int32), ("dtype", C.c_int32), ("nchild", C.c_int32),
        ("flag", C.c_int32), ("_pad", C.c_int32), ("i64", C.c_int64), ("f64", C.c_double),
        ("str", C.c_char_p), ("str_len", C.c_int64),
    ]


class MlExpr(C.Structure):
    _fields_ = [("nodes", C.POINTER(MlExprNode)), ("nnodes", C.c_int32), ("dtype", C.c_int32)]


class MlAggSpec(C.Structure):
    _fields_ = [("func", C.c_int32), ("arg_type", C.c_int32), ("arg", MlExpr)]


class MlSortKey(C.Structure):
    _fields_ = [("expr", MlExpr), ("asc", C.c_int32), ("nulls_first", C.c_int32)]


class MlPipeOp(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nexprs", C.c_int32), ("exprs", C.POINTER(MlExpr)),
                ("join", C.c_void_p), ("build_is_left", C.c_int32), ("_pad", C.c_int32)]


# ---------------------------------------------------------------------------------------
# Expression trees (PhysicalExpr) built in Python and serialized in prefix order.
# ---------------------------------------------------------------------------------------
@dataclass
class Expr:
    kind: int
    op: int = 0
    dtype: int = 0
    flag: int = 0
    i64: int = 0
    f64: float = 0.0
    s: Optional[bytes] = None
    kids: List["Expr"] = field(default_factory=list)

    # operator sugar -------------------------------------------------------------------
    def _bin(self, op, other):
        return Binary(op, self, _as_expr(other))

    def __add__(self, o): return self._bin(ADD, o)
    def __sub__(self, o): return self._bin(SUB, o)
    def __mul__(self, o): return self._bin(MUL, o)
    def __truediv__(self, o): return self._bin(DIV, o)
    def __mod__(self, o): return self._bin(MOD, o)
    def __rsub__(self, o): return Binary(SUB, _as_expr(o), self)
    def __rmul__(self, o): return Binary(MUL, _as_expr(o), self)
    def __radd__(self, o): return Binary(ADD, _as_expr(o), self)
    def eq(self, o): return self._bin(EQ, o)
    def ne(self, o): return self._bin(NOTEQ, o)
    def __lt__(self, o): return self._bin(LT, o)
    def __le__(self, o): return self._bin(LTEQ, o)
    def __gt__(self, o): return self._bin(GT, o)
    def __ge__(self, o): return self._bin(GTEQ, o)
    def __and__(self, o): return self._bin(AND, o)
    def __or__(self, o): return self._bin(OR, o)

    def nodes(self) -> List["Expr"]:
        out = [self]
        for k in self.kids:
            out.extend(k.nodes())
        return out


def Col(index: int) -> Expr:
    return Expr(E_COLUMN, i64=index)


def Lit(value: Any, dtype: Optional[int] = None) -> Expr:
    """A literal; Python ints default to INT64 and floats to FLOAT64 (the binder's
    literal types, scalar.rs)."""
    if value is None:
        return Expr(E_LITERAL, dtype=NULL)
    if dtype is None:
        if isinstance(value, bool):
            dtype = BOOL
        elif isinstance(value, int):
            dtype = INT64
        elif isinstance(value, float):
            dtype = FLOAT64
        elif isinstance(value, (str, bytes)):
            dtype = UTF8
        else:
            raise TypeError(value)
    if dtype == UTF8:
        b = value.encode() if isinstance(value, str) else bytes(value)
        return Expr(E_LITERAL, dtype=UTF8, s=b)
    if dtype == FLOAT64:
        return Expr(E_LITERAL, dtype=FLOAT64, f64=float(value))
    return Expr(E_LITERAL, dtype=dtype, i64=int(value))


def _as_expr(x) -> Expr:
    return x if isinstance(x, Expr) else Lit(x)


def Binary(op: int, left, right) -> Expr:
    return Expr(E_BINARY, op=op, kids=[_as_expr(left), _as_expr(right)])


def Not(e: Expr) -> Expr:
    return Expr(E_NOT, kids=[e])


def Negate(e: Expr) -> Expr:
    return Expr(E_NEGATE, kids=[e])


def IsNull(e: Expr, negated: bool = False) -> Expr:
    return Expr(E_IS_NULL, flag=int(negated), kids=[e])


def Like(e: Expr, pattern: str, negated: bool = False) -> Expr:
    return Expr(E_LIKE, flag=int(negated), s=pattern.encode(), kids=[e])


def InList(e: Expr, values: Sequence[Any], negated: bool = False) -> Expr:
    return Expr(E_IN_LIST, flag=int(negated), kids=[e] + [_as_expr(v) for v in values])


def Case(branches: Sequence[tuple], else_expr: Optional[Expr], dtype: int) -> Expr:
    kids: List[Expr] = []
    for c, v in branches:
        kids += [_as_expr(c), _as_expr(v)]
    if else_expr is not None:
        kids.append(_as_expr(else_expr))
    return Expr(E_CASE, dtype=dtype, flag=int(else_expr is not None), kids=kids)


def Cast(e: Expr, to: int) -> Expr:
    return Expr(E_CAST, dtype=to, kids=[e])


class Keep:
    """Holds ctypes buffers alive for the duration of a call."""

    def __init__(self):
        self.refs: List[Any] = []

    def add(self, x):
        self.refs.append(x)
        return x


def encode_expr(e: Expr, out_type: int, keep: Keep) -> MlExpr:
    ns = e.nodes()
    arr = keep.add((MlExprNode * max(len(ns), 1))())
    for i, n in enumerate(ns):
        a = arr[i]
        a.kind, a.op, a.dtype, a.nchild, a.flag = n.kind, n.op, n.dtype, len(n.kids), n.flag
        a.i64, a.f64 = n.i64, n.f64
        if n.s is not None:
            buf = keep.add(C.create_string_buffer(n.s, len(n.s) + 1))
            a.str = C.cast(buf, C.c_char_p)
            a.str_len = len(n.s)
    m = MlExpr()
    m.nodes = C.cast(arr, C.POINTER(MlExprNode))
    m.nnodes = len(ns)
    m.dtype = out_type
    return m


def encode_exprs(exprs: Sequence[tuple], keep: Keep):
    """exprs: sequence of (Expr, out_type) -> (MlExpr array, count)."""
    arr = keep.add((MlExpr * max(len(exprs), 1))())
    for i, (e, t) in enumerate(exprs):
        arr[i] = encode_expr(e, t, keep)
    return arr, len(exprs)


@dataclass
class AggSpec:
    func: int
    arg: Optional[Expr] = None
    arg_type: int = FLOAT64


def encode_aggs(aggs: Sequence[AggSpec], keep: Keep):
    arr = keep.add((MlAggSpec * max(len(aggs), 1))())
    for i, a in enumerate(aggs):
        arr[i].func = a.func
        arr[i].arg_type = a.arg_type
        if a.arg is not None:
            arr[i].arg = encode_expr(a.arg, a.arg_type, keep)
    return arr, len(aggs)


@dataclass
class SortKey:
    expr: Expr
    dtype: int
    asc: bool = True
    nulls_first: bool = False  # the binder's default is NULLS LAST (binder.rs:181)


def encode_sort_keys(keys: Sequence[SortKey], keep: Keep):
    arr = keep.add((MlSortKey * max(len(keys), 1))())
    for i, k in enumerate(keys):
        arr[i].expr = encode_expr(k.expr, k.dtype, keep)
        arr[i].asc = int(k.asc)
        arr[i].nulls_first = int(k.nulls_first)
    return arr, len(keys)


@dataclass
class PipeOp:
    """A streaming operator fused in front of a sink."""
    kind: int
    exprs: Sequence[tuple] = ()          # (Expr, type) pairs
    join: Any = None                     # join-table handle (c_void_p-compatible int)
    build_is_left: bool = False


def Filter(pred: Expr) -> PipeOp:
    return PipeOp(PIPE_FILTER, [(pred, BOOL)])


def Project(exprs: Sequence[tuple]) -> PipeOp:
    return PipeOp(PIPE_PROJECT, list(exprs))


def Probe(join_handle, keys: Sequence[tuple], build_is_left: bool = False) -> PipeOp:
    return PipeOp(PIPE_PROBE, list(keys), join_handle, build_is_left)


def encode_ops(ops: Sequence[PipeOp], keep: Keep):
    arr = keep.add((MlPipeOp * max(len(ops), 1))())
    for i, op in enumerate(ops):
        ex, n = encode_exprs(op.exprs, keep)
        arr[i].kind = op.kind
        arr[i].nexprs = n
        arr[i].exprs = C.cast(ex, C.POINTER(MlExpr))
        arr[i].join = op.join
        arr[i].build_is_left = int(op.build_is_left)
    return arr, len(ops)
