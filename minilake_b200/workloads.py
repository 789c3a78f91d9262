"""The physical plans of the three plain-GPU workloads, engine-agnostic.

Each plan is what MiniLake's binder and physical planner produce for the query
(binder.rs:444-476 left-deep joins in FROM order, physical_planner.rs:127-129
build side = smaller estimate, :150-171 ORDER BY + LIMIT -> top-N), expressed as
pipelines of Filter / Projection / HashJoinProbe operators ending in a sink.
The same function runs on the GPU engine and on the CPU oracle.
"""
from __future__ import annotations

from . import abi
from .abi import (AVG, BOOL, COUNT_STAR, FLOAT64, INT32, INT64, SUM, UTF8, AggSpec, Col, Filter, Like, Lit,
                  Probe, Project, SortKey)

# filter + low-cardinality GROUP BY ----------------------------------------------------------
# SELECT f1, f2, sum(qty), sum(price*(1-disc)), avg(disc), count(*) FROM t
#   WHERE d <= 2467 GROUP BY f1, f2 ORDER BY f1, f2
FG_SCAN = ["d", "f1", "f2", "qty", "price", "disc"]  # projection pushdown: tax is not read


def filter_groupby_plan(cutoff: int = 2467):
    prologue = [Filter(Col(0) <= Lit(cutoff))]
    group = [(Col(1), UTF8), (Col(2), UTF8)]
    aggs = [AggSpec(SUM, Col(3), FLOAT64),
            AggSpec(SUM, Col(4) * (Lit(1) - Col(5)), FLOAT64),
            AggSpec(AVG, Col(5), FLOAT64),
            AggSpec(COUNT_STAR)]
    return prologue, group, aggs


FG_OUT_TYPES = [UTF8, UTF8, FLOAT64, FLOAT64, FLOAT64, INT64]


def run_filter_groupby(engine, table, cutoff: int = 2467, size_hint: int = 0):
    src = table.project(FG_SCAN) if hasattr(table, "project") else table
    prologue, group, aggs = filter_groupby_plan(cutoff)
    agg = engine.hashagg(src, [INT32, UTF8, UTF8, FLOAT64, FLOAT64, FLOAT64], group, aggs, prologue, size_hint)
    n = engine.num_rows(agg)
    keys = [SortKey(Col(0), UTF8), SortKey(Col(1), UTF8)]
    res = engine.topn(agg, FG_OUT_TYPES, keys, max(n, 1))
    return engine.fetch(res)


# join + high-cardinality GROUP BY + top-10 -------------------------------------------------------
# SELECT fk, sum(v), count(*) FROM dim, fact WHERE fk = key AND d > 1200
#   GROUP BY fk ORDER BY sum(v) DESC, fk ASC LIMIT 10
JG_OUT_TYPES = [INT64, FLOAT64, INT64]


def join_groupby_build(engine, dim):
    d = dim.project(["key"]) if hasattr(dim, "project") else dim
    return engine.join_build(d, [INT64], [(Col(0), INT64)])


def join_groupby_plan(join_handle, cutoff: int = 1200):
    # fact scan [fk, d, v]; the build side (dim) is on the left: [key, fk, d, v] after the probe
    prologue = [Filter(Col(1) > Lit(cutoff)), Probe(join_handle, [(Col(0), INT64)], build_is_left=True)]
    group = [(Col(1), INT64)]
    aggs = [AggSpec(SUM, Col(3), FLOAT64), AggSpec(COUNT_STAR)]
    return prologue, group, aggs


def join_groupby_topn_keys():
    return [SortKey(Col(1), FLOAT64, asc=False), SortKey(Col(0), INT64, asc=True)]


def run_join_groupby(engine, dim, fact, cutoff: int = 1200, limit: int = 10, size_hint: int = 0, join=None):
    j = join if join is not None else join_groupby_build(engine, dim)
    f = fact.project(["fk", "d", "v"]) if hasattr(fact, "project") else fact
    prologue, group, aggs = join_groupby_plan(j.handle, cutoff)
    agg = engine.hashagg(f, [INT64, INT32, FLOAT64], group, aggs, prologue, size_hint)
    res = engine.topn(agg, JG_OUT_TYPES, join_groupby_topn_keys(), limit)
    return engine.fetch(res)


# star join with skew + string filter --------------------------------------------------------------
# SELECT label, sum(v*(1-w)) AS s FROM fact, a, b, c WHERE name LIKE 'ab%' AND k1 = a.key
#   AND k2 = b.key AND region = c.key GROUP BY label ORDER BY s DESC
SJ_OUT_TYPES = [UTF8, FLOAT64]


def star_join_builds(engine, A, B, C, pattern: str = "ab%"):
    a = engine.join_build(A, [INT32, UTF8], [(Col(0), INT32)],
                          prologue=[Filter(Like(Col(1), pattern)), Project([(Col(0), INT32)])])
    b = engine.join_build(B, [INT32, INT32], [(Col(0), INT32)])
    c = engine.join_build(C, [INT32, UTF8], [(Col(0), INT32)])
    return a, b, c


def star_join_plan(a, b, c):
    # fact scan [k1, k2, v, w] -> probe a -> [.., a.key] -> probe b -> [.., b.key, b.region]
    # -> probe c -> [.., c.key, c.label]
    prologue = [Probe(a.handle, [(Col(0), INT32)]),
                Probe(b.handle, [(Col(1), INT32)]),
                Probe(c.handle, [(Col(6), INT32)])]
    group = [(Col(8), UTF8)]
    aggs = [AggSpec(SUM, Col(2) * (Lit(1) - Col(3)), FLOAT64)]
    return prologue, group, aggs


def run_star_join(engine, fact, A, B, C, builds=None, size_hint: int = 0):
    a, b, c = builds if builds is not None else star_join_builds(engine, A, B, C)
    f = fact.project(["k1", "k2", "v", "w"]) if hasattr(fact, "project") else fact
    prologue, group, aggs = star_join_plan(a, b, c)
    agg = engine.hashagg(f, [INT32, INT32, FLOAT64, FLOAT64], group, aggs, prologue, size_hint)
    n = engine.num_rows(agg)
    res = engine.topn(agg, SJ_OUT_TYPES, [SortKey(Col(1), FLOAT64, asc=False)], max(n, 1))
    return engine.fetch(res)
