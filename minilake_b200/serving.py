"""Serving loop: a seeded Poisson stream of the three query shapes over HBM-resident tables.

* Tables: for each shape, `tables_per_shape` fact tables whose row counts are drawn
  log-uniform from [min_rows, max_rows], with the column distributions of the filter +
  GROUP BY, join + GROUP BY and star-join workloads; they are generated in HBM and stay there.
  The dimension tables are built into join tables once (the star join's filtered dimension A
  is rebuilt per query, its LIKE prefix being a query constant).
* Queries: arrivals are Poisson (rate `rate` queries/s, seed 46); each picks a shape, a table
  and constants uniform in their ranges (cutoffs in [0, 2557), a two-letter LIKE prefix).
* Continuous batching: `slots` worker threads, each with its own CUDA streams and its own
  resident hash-aggregate sinks (one per shape and table).  A query is admitted as soon as a
  slot is free and its memory estimate fits the HBM pool budget (160 GB); queries that arrive
  meanwhile wait in arrival order.  Admitted queries run concurrently on the device.
* Each query rebinds its slot's resident sink to the query's constants and runs the fused
  pipeline kernel as a replayed CUDA graph (captured the second time a slot runs the same
  table and join tables; a one-off combination runs without a graph), then finalizes and takes
  its top-N / ORDER BY on the device.
* Learned sizing on: each sink is presized with the cardinality model's prediction of the
  group count (from the table's scan features) and admission uses that estimate; off: no
  size hint (resize on overflow) and a fixed per-query estimate.

Latency = completion time - arrival time (wall clock, queueing included).

    python -m minilake_b200.serving --queries 20000 --rate 200 --learned both
"""
from __future__ import annotations

import argparse
import ctypes as C
import gc
import json
import math
import queue
import threading
import time
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

from . import abi, workloads
from .abi import FLOAT64, INT32, INT64, UTF8, Col, Filter, Like, Project, SortKey
from .columns import fixed, utf8_plain
from .datagen import F1_VALUES, F2_VALUES

SHAPES = ("filter_groupby", "join_groupby", "star_join")
BYTES_PER_ROW = {0: 36, 1: 20, 2: 4}  # columns every row reads (the star join's later stages see few rows)
POOL_BUDGET = 160 * 10**9


def _dict_arrays(values: List[bytes]):
    off = np.zeros(len(values) + 1, dtype=np.uint32)
    np.cumsum([len(v) for v in values], out=off[1:])
    return off, np.frombuffer(b"".join(values), dtype=np.uint8).copy()


class DeviceTable:
    """Fact-table columns in HBM (torch owns the memory) as an MlColumn array."""

    def __init__(self, cols: List[tuple]):
        # cols: (dtype, tensor, dictionary or None)
        self.keep = cols
        arr = (abi.MlColumn * len(cols))()
        self.dicts = []
        n = cols[0][1].numel()
        for i, (t, tensor, dictionary) in enumerate(cols):
            arr[i].dtype, arr[i].location, arr[i].len = t, abi.LOC_DEVICE, n
            arr[i].data = C.c_void_p(tensor.data_ptr())
            if dictionary is not None:
                off, data = _dict_arrays(dictionary)
                self.dicts.append((off, data))
                arr[i].encoding = abi.ENC_DICT
                arr[i].dict_len = len(dictionary)
                arr[i].dict_offsets = C.c_void_p(off.ctypes.data)
                arr[i].dict_data = C.c_void_p(data.ctypes.data)
        self.ml = (arr, len(cols), n)
        self.rows = n
        self.types = [t for t, _, _ in cols]
        self.nbytes = sum(int(x.numel() * x.element_size()) for _, x, _ in cols)


def star_dims(ctx):
    """The star join's dimension tables in HBM (seeded): A (150k keys, 18-character names),
    B (10k keys, region in [0, 25)), C (25 keys, labels); returns (A, B, C, names, A's keys)."""
    from .datagen import _random_words
    srng = np.random.Generator(np.random.PCG64(44))
    a_key = (srng.permutation(150_000) + 1).astype(np.int32)
    names = _random_words(srng, 150_000, 18)
    A = ctx.upload([fixed(INT32, a_key), utf8_plain(names)])
    b_key = (srng.permutation(10_000) + 1).astype(np.int32)
    region = srng.integers(0, 25, 10_000, dtype=np.int32)
    B = ctx.upload([fixed(INT32, b_key), fixed(INT32, region)])
    labels = _random_words(srng, 25, 10)
    C = ctx.upload([fixed(INT32, np.arange(25, dtype=np.int32)), utf8_plain(labels)])
    return A, B, C, names, a_key


def gen_fact(shape: int, rows: int, seed: int, dim_rows: int = 1_500_000, a_rows: int = 150_000,
             b_rows: int = 10_000) -> DeviceTable:
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    ri = lambda lo, hi, dt=torch.int32: torch.randint(lo, hi, (rows,), device="cuda", generator=g, dtype=dt)
    if shape == 0:
        d = ri(0, 2557)
        f1, f2 = ri(0, 3), ri(0, 2)
        qty = ri(1, 51, torch.int64).to(torch.float64)
        price = ri(90_000, 10_500_000, torch.int64).to(torch.float64) / 100.0
        disc = ri(0, 11, torch.int64).to(torch.float64) / 100.0
        return DeviceTable([(INT32, d, None), (UTF8, f1, F1_VALUES), (UTF8, f2, F2_VALUES),
                            (FLOAT64, qty, None), (FLOAT64, price, None), (FLOAT64, disc, None)])
    if shape == 1:
        fk = ri(1, dim_rows + 1, torch.int64)
        d = ri(0, 2557)
        v = torch.rand(rows, device="cuda", generator=g, dtype=torch.float64) * (105000.0 - 900.0) + 900.0
        return DeviceTable([(INT64, fk, None), (INT32, d, None), (FLOAT64, v, None)])
    # star join: k1 bounded Zipf(1.1) over the A keys (inverse CDF on the finite support)
    w = torch.arange(1, a_rows + 1, device="cuda", dtype=torch.float64) ** -1.1
    cdf = torch.cumsum(w, 0)
    cdf /= cdf[-1].clone()
    u = torch.rand(rows, device="cuda", generator=g, dtype=torch.float64)
    k1 = (torch.searchsorted(cdf, u, right=True) + 1).clamp(1, a_rows).to(torch.int32)
    k2 = ri(1, b_rows + 1)
    v = torch.rand(rows, device="cuda", generator=g, dtype=torch.float64) * 1e5
    wcol = torch.rand(rows, device="cuda", generator=g, dtype=torch.float64) * 0.1
    return DeviceTable([(INT32, k1, None), (INT32, k2, None), (FLOAT64, v, None), (FLOAT64, wcol, None)])


@dataclass
class Query:
    qid: int
    arrival: float        # seconds after the stream starts
    shape: int
    table: int
    const: object         # cutoff (shapes 0, 1) or LIKE prefix (shape 2)
    start: float = 0.0
    done: float = 0.0
    result: Optional[list] = None
    error: Optional[str] = None


def make_stream(n: int, rate: float, tables_per_shape: int, seed: int = 46) -> List[Query]:
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    for i in range(n):
        shape = int(rng.integers(3))
        const = int(rng.integers(0, 2557)) if shape < 2 else bytes(rng.integers(97, 123, 2, dtype=np.uint8)).decode()
        out.append(Query(i, float(t[i]), shape, int(rng.integers(tables_per_shape)), const))
    return out


class Server:
    def __init__(self, tables_per_shape: int = 4, min_rows: int = 1_000_000, max_rows: int = 200_000_000,
                 slots: int = 8, learned: bool = True, seed: int = 46, log=print, budget: int = POOL_BUDGET,
                 admit_limit: Optional[int] = None):
        from .gpu import Context, card_features
        self.log = log
        rng = np.random.default_rng(seed + 1)
        self.rows = [[int(round(math.exp(rng.uniform(math.log(min_rows), math.log(max_rows)))))
                      for _ in range(tables_per_shape)] for _ in SHAPES]
        self.tables = [[gen_fact(s, r, seed * 1000 + 10 * s + i) for i, r in enumerate(self.rows[s])]
                       for s in range(3)]
        table_bytes = sum(t.nbytes for ts in self.tables for t in ts)
        # the resident tables are held outside the library's pool: it gets the rest of the budget
        self.ctx = Context(0, hbm_budget=max(budget - table_bytes, 1 << 20))
        ctx = self.ctx
        # dimension tables (resident) and their join tables
        drng = np.random.Generator(np.random.PCG64(43))
        key = (drng.permutation(1_500_000) + 1).astype(np.int64)
        self.dim = ctx.upload([fixed(INT64, key)])
        self.dim_join = self._build(self.dim, [INT64], [(Col(0), INT64)])
        self.A, self.B, self.C, self.names, _ = star_dims(ctx)
        self.b_join = self._build(self.B, [INT32, INT32], [(Col(0), INT32)])
        self.c_join = self._build(self.C, [INT32, UTF8], [(Col(0), INT32)])
        # learned sizing: predicted group counts per (shape, table) from scan features
        self.learned = learned
        self.hint: Dict[tuple, int] = {}
        if learned:
            from .cardinality import train_model
            model = train_model(ctx, instances=200, seed=seed)
            for s in range(3):
                for i, t in enumerate(self.tables[s]):
                    keys = [(Col(1), UTF8), (Col(2), UTF8)] if s == 0 else [(Col(0), INT64 if s == 1 else INT32)]
                    f, _ = card_features(ctx, t.ml, keys)
                    groups = float(2.0 ** model.predict(f)[0])
                    self.hint[(s, i)] = int(groups * 1.25) + 16 if s != 2 else 64  # star join: 25 labels
            model.close()
        self.slots = slots
        self.budget_waits = 0
        self.budget_retries = 0
        self.admit_limit = admit_limit  # bytes of in-flight query state; default: what the pool has left
        self.mem_lock = threading.Condition()
        self.reserved = 0
        self.graphs = {"built": 0, "replayed": 0}

    def _build(self, batch, types, keys, prologue=()):
        from .gpu import JoinBuildSink
        j = JoinBuildSink(self.ctx, types, keys, prologue=prologue)
        loc = j.create_local()
        loc.sink(batch)
        loc.combine()
        j.finalize()
        return j

    # ---- one query --------------------------------------------------------------------------
    def estimate_bytes(self, q: Query) -> int:
        """Device bytes a query may add while it runs (hash state, outputs, top-N)."""
        if q.shape == 1:
            groups = 1_500_000
        elif self.learned:
            groups = self.hint.get((q.shape, q.table), 1024)
        else:
            groups = 1024
        return 64 * groups + (16 << 20)

    def plan(self, q: Query, a_join=None):
        if q.shape == 0:
            return workloads.filter_groupby_plan(q.const)
        if q.shape == 1:
            return workloads.join_groupby_plan(self.dim_join.handle, q.const)
        return workloads.star_join_plan(a_join, self.b_join, self.c_join)

    def execute(self, q: Query, sinks: dict):
        """Run one query on a slot (its resident sinks in `sinks`); returns the result columns."""
        from .gpu import HashAggregateSink, SortSink
        t = self.tables[q.shape][q.table]
        a_join = None
        if q.shape == 2:
            a_join = self._build(self.A, [INT32, UTF8], [(Col(0), INT32)],
                                 prologue=[Filter(Like(Col(1), q.const + "%")), Project([(Col(0), INT32)])])
        prologue, group, aggs = self.plan(q, a_join)
        key = (q.shape, q.table)
        sink = sinks.get(key)
        if sink is None:
            hint = self.hint.get(key, 0) if self.learned else 0
            sink = HashAggregateSink(self.ctx, t.types, group, aggs, prologue, size_hint=hint)
            sinks[key] = sink
        else:
            sink.rebind(prologue, group, aggs)
        sink.run_resident(t.ml, reset=True)
        agg = sink.finalize()
        n = agg.num_rows
        if q.shape == 0:
            out_types, keys, limit = workloads.FG_OUT_TYPES, [SortKey(Col(0), UTF8), SortKey(Col(1), UTF8)], max(n, 1)
        elif q.shape == 1:
            out_types, keys, limit = workloads.JG_OUT_TYPES, workloads.join_groupby_topn_keys(), 10
        else:
            out_types, keys, limit = workloads.SJ_OUT_TYPES, [SortKey(Col(1), FLOAT64, asc=False)], max(n, 1)
        ts = SortSink(self.ctx, out_types, keys, limit)
        loc = ts.create_local()
        loc.sink(agg)
        loc.combine()
        res = ts.finalize()
        cols = res.fetch()
        res.close()
        ts.close()
        agg.close()
        if a_join is not None:
            a_join.close()
        return [c.strings() if c.dtype == UTF8 else c.values.tolist() for c in cols]

    # ---- the loop -------------------------------------------------------------------------
    def serve(self, stream: List[Query], warmup: bool = True):
        """Run the stream in real time; returns the queries with their timings and results."""
        from .gpu import ResourcesExhausted
        pending: "queue.Queue[Optional[Query]]" = queue.Queue()
        # the slots' resident sinks (and their captured graphs) carry over from stream to stream
        if not hasattr(self, "sinks_per_slot"):
            self.sinks_per_slot = [dict() for _ in range(self.slots)]
        sinks_per_slot = self.sinks_per_slot
        if warmup:
            # the star join's filtered dimension is indexed directly or hashed depending on the
            # prefix: compile both kernel variants (the kernel cache is shared by all slots)
            for p in range(26 * 26):
                prefix = chr(97 + p // 26) + chr(97 + p % 26)
                self.execute(Query(-1, 0.0, 2, 0, prefix), sinks_per_slot[0])

            # every slot runs every shape and table, all slots at once: kernels compiled, graphs
            # captured, and the device allocator's cache grown to what concurrent queries hold
            def warm(k):
                for rep in range(2):
                    for s in range(3):
                        for i in range(len(self.tables[s])):
                            c = (600 + 1100 * rep) if s < 2 else ("ab", "qx")[rep]
                            self.execute(Query(-1, 0.0, s, i, c), sinks_per_slot[k])

            ws = [threading.Thread(target=warm, args=(k,)) for k in range(self.slots)]
            for th in ws:
                th.start()
            for th in ws:
                th.join()
        used, _, limit = self.ctx.pool_stats()
        room = self.admit_limit if self.admit_limit is not None else limit - used
        t0 = time.perf_counter() + 0.05

        def admit(q: Query) -> int:
            need = self.estimate_bytes(q)
            with self.mem_lock:
                waited = False
                while True:
                    if self.reserved + need <= room or self.reserved == 0:
                        self.reserved += need
                        if waited:
                            self.budget_waits += 1
                        return need
                    waited = True
                    self.mem_lock.wait(0.01)

        def release(need: int):
            with self.mem_lock:
                self.reserved -= need
                self.mem_lock.notify_all()

        def worker(k: int):
            sinks = sinks_per_slot[k]
            while True:
                q = pending.get()
                if q is None:
                    return
                need = admit(q)
                q.start = time.perf_counter() - t0
                for _ in range(100):
                    try:
                        q.result = self.execute(q, sinks)
                        q.error = None
                        break
                    except ResourcesExhausted as e:  # the pool is full right now: wait for a query to end
                        q.error = str(e)
                        with self.mem_lock:
                            self.budget_retries += 1
                            self.mem_lock.wait(0.05)
                    except Exception as e:  # a failed query is reported, the loop goes on
                        q.error = str(e)
                        break
                q.done = time.perf_counter() - t0
                release(need)

        # no garbage-collector pauses while queries are timed: the objects made so far are frozen
        # out of collection and collection waits until the stream is done
        gc.collect()
        gc.freeze()
        gc_was_enabled = gc.isenabled()
        gc.disable()
        threads = [threading.Thread(target=worker, args=(k,), daemon=True) for k in range(self.slots)]
        for th in threads:
            th.start()
        for q in stream:  # arrivals in real time
            delay = t0 + q.arrival - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            pending.put(q)
        for _ in threads:
            pending.put(None)
        for th in threads:
            th.join()
        if gc_was_enabled:
            gc.enable()
        gc.unfreeze()
        seen = self.__dict__.setdefault("graph_seen", {})
        for d in sinks_per_slot:
            for s in d.values():
                g = s.graph_stats()
                b0, r0 = seen.get(id(s), (0, 0))
                self.graphs["built"] += g["built"] - b0
                self.graphs["replayed"] += g["replayed"] - r0
                seen[id(s)] = (g["built"], g["replayed"])
        return stream

    def close(self):
        for d in getattr(self, "sinks_per_slot", []):
            for s in d.values():
                s.close()
        for j in (self.dim_join, self.b_join, self.c_join):
            j.close()
        for b in (self.dim, self.A, self.B, self.C):
            b.close()
        self.ctx.close()


def summarize(stream: List[Query], server: Server) -> dict:
    ok = [q for q in stream if q.error is None]
    lat = np.array([q.done - q.arrival for q in ok]) * 1e3
    span = max(q.done for q in ok) - min(q.arrival for q in ok)
    algo = sum(server.tables[q.shape][q.table].rows * BYTES_PER_ROW[q.shape] for q in ok)
    per_shape = {}
    for s, name in enumerate(SHAPES):
        l = np.array([q.done - q.arrival for q in ok if q.shape == s]) * 1e3
        if len(l):
            per_shape[name] = {"queries": int(len(l)), "p50_ms": float(np.percentile(l, 50)),
                               "p99_ms": float(np.percentile(l, 99))}
    # the slowest queries: when they arrived, how long they queued before a slot took them
    slow = sorted(ok, key=lambda q: q.arrival - q.done)[:12]
    slowest = [{"arrival_s": round(q.arrival, 4), "queued_ms": round((q.start - q.arrival) * 1e3, 3),
                "run_ms": round((q.done - q.start) * 1e3, 3), "shape": SHAPES[q.shape], "table": q.table}
               for q in slow]
    # host-side events that can stall every slot at once: device and pinned allocations, kernel
    # compilations, graph captures (count, total ms since the server started)
    ctx = getattr(server, "ctx", None)
    events = {k: [int(v) if i == 0 else round(v, 2) for i, v in enumerate(ctx.profile(k))]
              for k in ("device_alloc", "pinned_alloc", "jit_compile", "graph_capture")} if ctx else {}
    return {
        "slowest": slowest,
        "host_events": events,
        "queries": len(stream), "completed": len(ok), "failed": len(stream) - len(ok),
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "p999_ms": float(np.percentile(lat, 99.9)), "max_ms": float(lat.max()),
        "queries_per_s": len(ok) / span, "algorithmic_GB_per_s": algo / span / 1e9,
        "budget_waits": server.budget_waits, "budget_retries": server.budget_retries, "per_shape": per_shape,
        "graphs_captured": server.graphs["built"], "graph_replays": server.graphs["replayed"],
        "table_rows": server.rows, "learned_sizing": server.learned, "slots": server.slots,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--queries", type=int, default=20000)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--tables-per-shape", type=int, default=4)
    ap.add_argument("--min-rows", type=int, default=1_000_000)
    ap.add_argument("--max-rows", type=int, default=200_000_000)
    ap.add_argument("--learned", choices=["on", "off", "both"], default="both")
    ap.add_argument("--seed", type=int, default=46)
    ap.add_argument("--sweep", default="", help="comma-separated arrival rates (q/s): a load sweep, "
                                                  "--queries queries at each rate over the same tables")
    a = ap.parse_args()
    import sys
    log = lambda *m: print(*m, file=sys.stderr, flush=True)
    out = {}
    if a.sweep:
        rates = [float(r) for r in a.sweep.split(",")]
        for mode in (["on", "off"] if a.learned == "both" else [a.learned]):
            server = Server(a.tables_per_shape, a.min_rows, a.max_rows, a.slots, mode == "on", a.seed, log)
            rows = []
            for i, rate in enumerate(rates):
                stream = make_stream(a.queries, rate, a.tables_per_shape, a.seed + i)
                server.serve(stream, warmup=i == 0)
                r = summarize(stream, server)
                rows.append({"rate": rate, **{k: r[k] for k in ("completed", "failed", "p50_ms", "p99_ms", "p999_ms",
                                                                 "max_ms", "queries_per_s", "algorithmic_GB_per_s")}})
                log(f"learned {mode} rate {rate}: {json.dumps(rows[-1])}")
            out["sweep_learned_" + mode] = rows
            server.close()
        print(json.dumps(out), flush=True)
        return
    for mode in (["on", "off"] if a.learned == "both" else [a.learned]):
        server = Server(a.tables_per_shape, a.min_rows, a.max_rows, a.slots, mode == "on", a.seed, log)
        stream = make_stream(a.queries, a.rate, a.tables_per_shape, a.seed)
        log(f"learned sizing {mode}: serving {a.queries} queries at {a.rate}/s")
        server.serve(stream)
        out["learned_" + mode] = summarize(stream, server)
        log(json.dumps(out["learned_" + mode]))
        server.close()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
