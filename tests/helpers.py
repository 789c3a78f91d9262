"""Shared fixtures for the tests: MiniLake's end-to-end test tables
(crates/minilake-sql/tests/end_to_end.rs:21-181) as host row groups, and the
physical plans of its SQL tests, runnable on the GPU engine and the oracle."""
import json
import os

import numpy as np

from minilake_b200 import abi
from minilake_b200.abi import (AVG, BOOL, COUNT, COUNT_STAR, DATE, FLOAT64, INT32, INT64, MIN, SUM, UTF8, AggSpec,
                               Case, Col, Filter, InList, Like, Lit, Probe, SortKey)
from minilake_b200.columns import Table, encode_strings, fixed

HERE = os.path.dirname(os.path.abspath(__file__))


def golden():
    with open(os.path.join(HERE, "golden", "known_answers.json")) as f:
        return json.load(f)


def _days(s):
    from datetime import date
    y, m, d = map(int, s.split("-"))
    return (date(y, m, d) - date(1970, 1, 1)).days


FLAGS = [b"A", b"N", b"R"]
PRIOS = [b"1-URGENT", b"2-HIGH", b"3-MEDIUM"]


def e2e_tables():
    """lineitem: 10,000 rows in 4 row groups; orders: 1,000 rows in 10 row groups."""
    n_line, n_ord = 10_000, 1_000
    day0 = _days("1995-01-01")
    i = np.arange(n_line)
    orderkey = (i % n_ord).astype(np.int64)
    qty_valid = (i % 13) != 0
    qty = np.where(qty_valid, (i % 50).astype(np.float64), 0.0)
    price = (i % 97).astype(np.float64) + 0.5
    flag = i % 3
    ship = (day0 + i % 30).astype(np.int32)
    rgs = []
    for c in np.array_split(np.arange(n_line), 4):
        a, b = c[0], c[-1] + 1
        rgs.append([fixed(INT64, orderkey[a:b]), fixed(FLOAT64, qty[a:b], qty_valid[a:b]),
                    fixed(FLOAT64, price[a:b]), encode_strings(FLAGS, flag[a:b]), fixed(DATE, ship[a:b])])
    lineitem = Table("lineitem", ["l_orderkey", "l_qty", "l_price", "l_flag", "l_shipdate"], rgs)
    j = np.arange(n_ord)
    odate = (day0 + j // 100).astype(np.int32)
    orgs = []
    for c in np.array_split(j, 10):
        a, b = c[0], c[-1] + 1
        orgs.append([fixed(INT64, j[a:b]), fixed(DATE, odate[a:b]), encode_strings(PRIOS, j[a:b] % 3)])
    orders = Table("orders", ["o_orderkey", "o_orderdate", "o_orderpriority"], orgs)
    return lineitem, orders


def q_count(engine, lineitem):
    t = lineitem.project(["l_qty"])
    out = engine.hashagg(t, [FLOAT64], [], [AggSpec(COUNT_STAR), AggSpec(COUNT, Col(0), FLOAT64)])
    return engine.fetch(out)


def q_group_by(engine, lineitem, cutoff):
    t = lineitem.project(["l_qty", "l_price", "l_flag", "l_shipdate"])
    agg = engine.hashagg(t, [FLOAT64, FLOAT64, UTF8, DATE], [(Col(2), UTF8)],
                         [AggSpec(SUM, Col(1), FLOAT64), AggSpec(COUNT_STAR), AggSpec(AVG, Col(0), FLOAT64),
                          AggSpec(MIN, Col(3), DATE)],
                         prologue=[Filter(Col(3) < Lit(cutoff, DATE))])
    n = engine.num_rows(agg)
    res = engine.topn(agg, [UTF8, FLOAT64, INT64, FLOAT64, DATE], [SortKey(Col(0), UTF8)], max(n, 1))
    return engine.fetch(res)


def q_join_top_n(engine, lineitem, orders, cutoff):
    o = orders.project(["o_orderkey", "o_orderdate", "o_orderpriority"])
    j = engine.join_build(o, [INT64, DATE, UTF8], [(Col(0), INT64)],
                          prologue=[Filter(Col(1) >= Lit(cutoff, DATE))])
    l = lineitem.project(["l_orderkey", "l_price"])
    # build (orders) on the left: [o_orderkey, o_orderdate, o_orderpriority, l_orderkey, l_price]
    agg = engine.hashagg(l, [INT64, FLOAT64], [(Col(2), UTF8)], [AggSpec(SUM, Col(4), FLOAT64)],
                         prologue=[Probe(j.handle, [(Col(0), INT64)], build_is_left=True)])
    res = engine.topn(agg, [UTF8, FLOAT64], [SortKey(Col(1), FLOAT64, asc=False)], 2)
    return engine.fetch(res), j


def q_case_in_like_between(engine, lineitem):
    t = lineitem.project(["l_price", "l_flag"])
    pred = ((Col(0) >= Lit(10)) & (Col(0) <= Lit(20))) & Like(Col(1), "%")
    case = Case([(InList(Col(1), ["A", "R"]), Lit(1))], Lit(0), INT64)
    out = engine.hashagg(t, [FLOAT64, UTF8], [], [AggSpec(SUM, case, INT64), AggSpec(COUNT_STAR)],
                         prologue=[Filter(pred)])
    return engine.fetch(out)


def valid_mask(col):
    return col.valid_mask()


def rel_err(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
