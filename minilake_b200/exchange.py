"""Multi-GPU form of the aggregate queries: one process per GPU, torch.distributed for the
collectives (NCCL between GPUs; the tests run the same plan between CPU processes over gloo).

The plan is MiniLake's distributed mode (minilake-dist/src/split.rs:54-127) with the merge
spread over the ranks:

  1. every rank scans its own share of the fact table's row groups (split.rs's workers scan
     their own files; the build sides are read whole by every rank) and runs the pipeline up to
     the topmost aggregate in Partial mode: group keys, then each accumulator's state
     (accumulator.rs:177-185, 382-405: COUNT and SUM their value, MIN/MAX theirs, AVG a sum and a
     count);
  2. the exchange step: each partial group goes to the rank that owns its key, partition =
     hash_columns(keys) % world (kernels/hash.rs:16-23), in one all-to-all per state column.
     A NULL state (a SUM/MIN/MAX whose group saw no valid input) travels with a validity byte;
  3. each rank merges the states it received in Final mode (accumulator.rs:407-497: counts and
     sums add, MIN/MAX fold, AVG = summed sum / summed count), so every group is finalized on
     exactly one rank;
  4. a top-N runs on each rank's groups and the ranks' lists are gathered; every rank merges
     them into the same answer (the global top N of disjoint groups is within the union of the
     local top Ns).

MiniLake's coordinator merges every worker's partials alone; spreading the merge keeps the
exchange at one pass over the partial states per rank, whatever the number of GPUs.  Group keys
must be fixed-width (integers, dates, booleans): the high-cardinality GROUP BY this step exists
for.  Low-cardinality string-keyed aggregates have a few dozen groups and are not exchanged.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from .abi import AVG, COUNT, COUNT_STAR, FLOAT64, INT64, MAX, MIN, SUM, AggSpec, Case, Cast, Col, Lit

FIXED_KEYS = (abi.BOOL, abi.INT32, abi.INT64, abi.DATE)


def split_row_groups(n_groups: int, rank: int, world: int) -> List[int]:
    """Row groups rank `rank` scans: every world-th one from `rank` (a file split)."""
    return list(range(rank, n_groups, world))


@dataclass
class PartialPlan:
    partial: List[AggSpec]  # the aggregates of the Partial-mode pipeline
    state_types: List[int]  # type of each partial state column
    finals: List[tuple]     # per output aggregate: ("state", j) or ("avg", j_sum, j_count)


def partial_plan(aggs: Sequence[AggSpec]) -> PartialPlan:
    """Partial-mode aggregates for `aggs` (AVG splits into a f64 SUM of its input, as
    Accumulator::prepare_input casts it, and a COUNT)."""
    partial, types, finals = [], [], []
    for a in aggs:
        if a.func == AVG:
            partial += [AggSpec(SUM, Cast(a.arg, FLOAT64), FLOAT64), AggSpec(COUNT, a.arg, a.arg_type)]
            types += [FLOAT64, INT64]
            finals.append(("avg", len(partial) - 2, len(partial) - 1))
            continue
        partial.append(a)
        if a.func in (COUNT_STAR, COUNT):
            types.append(INT64)
        elif a.func == SUM:
            types.append(FLOAT64 if a.arg_type == FLOAT64 else INT64)
        elif a.func in (MIN, MAX):
            types.append(a.arg_type)
        else:
            raise ValueError(f"aggregate {a.func} has no partial state")
        finals.append(("state", len(partial) - 1))
    return PartialPlan(partial, types, finals)


def _read(i: int, t: int, valid_col: Sequence[Optional[int]]):
    """Exchanged column i as an expression: through its validity byte when it carries one."""
    return Case([(Col(valid_col[i]), Col(i))], None, t) if valid_col[i] is not None else Col(i)


def merge_aggs(plan: PartialPlan, nkeys: int, valid_col: Sequence[Optional[int]]):
    """Final-mode aggregates over the exchanged columns [keys, states, validity bytes]: counts
    and sums add, MIN/MAX fold; a state that can be NULL is read through its validity byte."""
    out = []
    for j, (a, t) in enumerate(zip(plan.partial, plan.state_types)):
        func = MIN if a.func == MIN else MAX if a.func == MAX else SUM
        out.append(AggSpec(func, _read(nkeys + j, t, valid_col), t))
    return out


def final_projection(plan: PartialPlan, key_types: Sequence[int]):
    """Output columns after the Final merge: the keys, then each aggregate (AVG = sum / count,
    NULL when the count is 0, accumulator.rs:506-512), or None when no AVG needs computing."""
    if all(f[0] == "state" for f in plan.finals):
        return None
    nk = len(key_types)
    exprs = [(Col(i), t) for i, t in enumerate(key_types)]
    for f in plan.finals:
        if f[0] == "state":
            exprs.append((Col(nk + f[1]), plan.state_types[f[1]]))
        else:
            s, c = Col(nk + f[1]), Col(nk + f[2])
            exprs.append((Case([(c > Lit(0), s / Cast(c, FLOAT64))], None, FLOAT64), FLOAT64))
    return exprs


def _agree(flags: Sequence[bool], device) -> List[bool]:
    """The OR over the ranks of per-column flags (which columns carry validity bytes), so every
    rank makes the same exchange calls."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([int(f) for f in flags], dtype=torch.int32, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [bool(x) for x in t.cpu().tolist()]


def _recv_sizes(counts, world: int, device) -> List[int]:
    """Rows this rank receives from each rank (every rank's `counts` gathered)."""
    import torch
    import torch.distributed as dist
    send = torch.tensor([int(c) for c in counts], dtype=torch.int64, device=device)
    got = [torch.empty_like(send) for _ in range(world)]
    dist.all_gather(got, send)
    rank = dist.get_rank()
    return [int(g[rank].item()) for g in got]


def _all_to_all(t, counts, recv_sizes, device):
    """Exchange the row segments of tensor t (segment p, counts[p] rows, goes to rank p)."""
    import torch
    import torch.distributed as dist
    out = torch.empty(sum(recv_sizes), dtype=t.dtype, device=device)
    dist.all_to_all_single(out, t.contiguous(), output_split_sizes=list(recv_sizes),
                           input_split_sizes=[int(c) for c in counts])
    return out


class DeviceSide:
    """The exchange over device columns (GPU engine, NCCL): ml_gpu_partition groups the rows by
    destination rank on the device and each column segment crosses NVLink once."""

    device = "cuda"

    def __init__(self, engine):
        self.engine = engine
        self._keep = []

    def partition(self, batch, nkeys: int, world: int):
        from . import gpu
        ctx = self.engine.ctx
        types, nullable = [], []
        for i in range(batch.num_columns):
            import ctypes as C
            t, hv = C.c_int32(), C.c_int32()
            gpu._check(gpu.LIB.ml_gpu_batch_column_info(batch.h, i, C.byref(t), None, C.byref(hv)))
            if t.value not in FIXED_KEYS + (FLOAT64,):
                raise TypeError("the exchange carries fixed-width columns only")
            types.append(t.value)
            nullable.append(bool(hv.value))
        nullable = _agree(nullable, "cuda")
        # validity bytes of the nullable columns, computed on the device (IS NOT NULL)
        valid_batches = [gpu.ProjectionOperator(ctx, abi.IsNull(Col(i), negated=True), abi.BOOL).execute(batch)
                         for i, nb in enumerate(nullable) if nb]
        arr, nc = batch.ml_columns()
        views = [arr[i] for i in range(nc)]
        for vb in valid_batches:
            va, _ = vb.ml_columns()
            views.append(va[0])
        all_cols = (abi.MlColumn * len(views))(*views)
        part, counts = gpu.partition(ctx, (all_cols, len(views), batch.num_rows), list(range(nkeys)), world)
        self._keep += [part, valid_batches]
        tensors = [gpu.column_tensor(part, i) for i in range(len(views))]
        cols, v = [], nc
        for i in range(nc):
            valid = None
            if nullable[i]:
                valid = tensors[v]
                v += 1
            cols.append((types[i], tensors[i], valid))
        return cols, counts, None

    def exchange(self, cols, counts, world):
        sizes = _recv_sizes(counts, world, "cuda")
        got = []
        for dt, vals, valid in cols:
            r = _all_to_all(vals, counts, sizes, "cuda")
            rv = _all_to_all(valid, counts, sizes, "cuda") if valid is not None else None
            got.append((dt, r, rv))
        self._keep.append(got)
        return got

    def source(self, got, _fixed_fn):
        """A device morsel (ml_column views of the received tensors) for the Final merge."""
        n = int(got[0][1].numel()) if got else 0
        specs = [(dt, t) for dt, t, _ in got] + [(abi.BOOL, rv) for _, _, rv in got if rv is not None]
        arr = (abi.MlColumn * len(specs))()
        for i, (dt, t) in enumerate(specs):
            arr[i].dtype, arr[i].encoding, arr[i].location, arr[i].len = dt, abi.ENC_PLAIN, abi.LOC_DEVICE, n
            arr[i].data = t.data_ptr() if n else None
        self._keep.append(arr)
        return [(arr, len(specs), n)]


def distributed_hashagg(engine, side, source, input_types, group, aggs, prologue=(), world: int = 1):
    """The aggregate over this rank's share of `source`, merged across the ranks: returns
    (final batch, projection or None).  The final batch holds the groups this rank owns: keys,
    then the merged states (`projection`, when given, turns them into the aggregates' values).
    Collective: every rank calls it once, with the same plan."""
    key_types = [t for _, t in group]
    if any(t not in FIXED_KEYS for t in key_types):
        raise TypeError("the exchange step needs fixed-width group keys")
    plan = partial_plan(aggs)
    nk = len(group)
    partial = engine.hashagg(source, input_types, group, plan.partial, prologue)
    cols, counts, fixed_fn = side.partition(partial, nk, world)
    got = side.exchange(cols, counts, world)
    # the validity bytes follow the exchanged columns, in column order (keys included: a NULL
    # group key is its own group)
    valid_col, v = [], len(got)
    for _, _, rv in got:
        valid_col.append(v if rv is not None else None)
        v += 1 if rv is not None else 0
    merged_types = [dt for dt, _, _ in got] + [abi.BOOL] * (v - len(got))
    final = engine.hashagg(side.source(got, fixed_fn), merged_types,
                           [(_read(i, t, valid_col), t) for i, t in enumerate(key_types)],
                           merge_aggs(plan, nk, valid_col))
    return final, final_projection(plan, key_types)


def merge_topn(keys, sums, counts, limit: int):
    """Top `limit` rows by SUM DESC, key ASC of the concatenated candidates."""
    order = np.lexsort((keys, -sums))[:limit]
    return keys[order], sums[order], counts[order]


def exchange_topn(keys, sums, counts, limit: int, device="cpu"):
    """Gather every rank's local top-N (key i64, sum f64, count i64; at most `limit` rows) and
    return the merged global top N on every rank.  Collective: every rank calls it once."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size()
    n = len(keys)
    k = torch.full((limit,), np.iinfo(np.int64).max, dtype=torch.int64)
    s = torch.full((limit,), -np.inf, dtype=torch.float64)
    c = torch.zeros(limit, dtype=torch.int64)
    k[:n], s[:n], c[:n] = torch.as_tensor(keys), torch.as_tensor(sums), torch.as_tensor(counts)
    m = torch.tensor([n], dtype=torch.int64)
    parts = []
    for t in (m, k, s, c):
        t = t.to(device)
        out = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(out, t)
        parts.append([o.cpu().numpy() for o in out])
    ns, ks, ss, cs = parts
    keys_all = np.concatenate([ks[r][:ns[r][0]] for r in range(world)])
    sums_all = np.concatenate([ss[r][:ns[r][0]] for r in range(world)])
    counts_all = np.concatenate([cs[r][:ns[r][0]] for r in range(world)])
    return merge_topn(keys_all, sums_all, counts_all, limit)
