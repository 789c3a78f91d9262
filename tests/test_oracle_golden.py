"""The CPU oracle against the known answers of MiniLake's own tests (golden vectors,
tests/golden/known_answers.json).  CPU only."""
import math

import numpy as np
import pytest

from helpers import (e2e_tables, golden, q_case_in_like_between, q_count, q_group_by, q_join_top_n, rel_err)
from minilake_b200 import abi
from minilake_b200.abi import (AND, BOOL, DIV, FLOAT64, INT64, MUL, OR, Binary, Case, Col, InList, IsNull, Like, Lit,
                               Not)
from minilake_b200.columns import fixed, utf8_plain
from oracle import orc

G = golden()


def test_compare_scalar_and_select():  # cmp.rs:124-133
    g = G["compare_scalar_and_select"]
    cols = [fixed(INT64, g["values"])]
    assert list(orc.filter_rows(Col(0) < Lit(g["lt"]), cols)) == g["selection"]
    assert list(orc.filter_rows(Col(0) < Lit(g["lt"]), cols, g["selection_with_input"]["input"])) == \
        g["selection_with_input"]["out"]
    v = [fixed(INT64, g["values"], np.array(g["selection_with_validity"]["valid"]))]
    assert list(orc.filter_rows(Col(0) < Lit(g["lt"]), v)) == g["selection_with_validity"]["out"]
    m = orc.project(Col(0) < Lit(g["lt"]), BOOL, cols)[0]
    assert [bool(x) for x in m.values] == g["mask"]


def test_empty_and_all():  # cmp.rs:135-140
    assert list(orc.filter_rows(Lit(True), [fixed(INT64, [0, 0, 0])])) == G["empty_and_all"]["all_true3"]
    assert list(orc.filter_rows(Col(0) > Lit(5), [fixed(INT64, [0, 0, 0])])) == []
    assert list(orc.filter_rows(Col(0) > Lit(5), [fixed(INT64, [])])) == []


def test_kleene():  # boolean.rs:69-84
    g = G["kleene"]
    cols = [fixed(BOOL, g["a"], np.array(g["a_valid"])), fixed(BOOL, g["b"])]
    for op, key in ((AND, "and"), (OR, "or")):
        r = orc.project(Binary(op, Col(0), Col(1)), BOOL, cols)[0]
        assert [bool(x) for x in r.valid_mask()] == g[key + "_valid"]
        for v, want, ok in zip(r.values, g[key + "_value"], g[key + "_valid"]):
            if ok:
                assert bool(v) == want
    sk = G["scalar_kleene"]  # scalar_ops.rs:158-164
    r = orc.project(Binary(AND, Lit(None), Lit(False)), BOOL, [fixed(INT64, [1])])[0]
    assert r.valid_mask()[0] and not r.values[0] and sk["null_and_false"] is False
    r = orc.project(Binary(OR, Lit(None), Lit(False)), BOOL, [fixed(INT64, [1])])[0]
    assert not r.valid_mask()[0] and sk["null_or_false"] is None


def test_arith():  # arith.rs:136-153
    g = G["arith_ops"]
    cols = [fixed(INT64, g["a"]), fixed(INT64, g["b"])]
    assert list(orc.project(Col(0) + Col(1), INT64, cols)[0].values) == g["add"]
    assert list(orc.project(Lit(100) - Col(1), INT64, cols)[0].values) == g["sub_from_100"]
    r = orc.project(Col(1) % Lit(0), INT64, cols)[0]
    assert list(r.values) == g["mod_zero_values"] and not r.valid_mask().any()
    m = g["mul_one_minus"]
    r = orc.project(Col(0) * (Lit(1) - Col(1)), FLOAT64, [fixed(FLOAT64, [m["a"]]), fixed(FLOAT64, [m["b"]])])[0]
    assert r.values[0] == m["out"]


def test_like():  # like.rs:134-166, string.rs:37-49
    for pat, s, want in G["like_matching"]:
        r = orc.project(Like(Col(0), pat), BOOL, [utf8_plain([s.encode()])])[0]
        assert bool(r.values[0]) == want, (pat, s)
    g = G["like_on_plain_strings"]
    col = [utf8_plain([v.encode() for v in g["values"]])]
    assert [bool(x) for x in orc.project(Like(Col(0), "PROMO%"), BOOL, col)[0].values] == g["like"]
    assert [bool(x) for x in orc.project(InList(Col(0), ["STD"]), BOOL, col)[0].values] == g["in_std"]


def test_eval():  # eval.rs:548-612
    g = G["eval"]
    cols = [fixed(INT64, g["a"]), fixed(FLOAT64, g["b"])]
    pred = (Col(0) >= Lit(5)) & (Col(1) < Lit(3.0))
    assert list(orc.filter_rows(pred, cols)) == g["select_a_ge5_and_b_lt3"]
    assert orc.project(Col(0) * Col(1), FLOAT64, cols)[0].values[3] == g["a_times_b_row3"]
    r = orc.project(Col(1) / Lit(0), FLOAT64, cols)[0]
    assert int((~r.valid_mask()).sum()) == g["b_div_zero_null_count"]
    c = Case([(Col(0) > Lit(5), Lit(1))], Lit(0), INT64)
    assert list(orc.project(c, INT64, cols)[0].values) == g["case_a_gt5_then1_else0"]


def test_accumulator_grouped_sum_avg():  # accumulator.rs:600-623
    from minilake_b200.abi import AVG, SUM, AggSpec
    g = G["accumulator"]
    cols = [fixed(INT64, g["gids"]), fixed(FLOAT64, g["values"], np.array(g["valid"]))]
    eng = orc.OracleEngine(threads=1)
    out = eng.fetch(eng.hashagg([cols[0], cols[1]], [INT64, FLOAT64], [(Col(0), INT64)],
                                [AggSpec(SUM, Col(1), FLOAT64), AggSpec(AVG, Col(1), FLOAT64)]))
    order = np.argsort(out[0].values)
    assert list(out[1].values[order]) == g["sum"]
    assert out[2].values[order][1] == g["avg_group1"]


def test_hash_and_swar():  # hash.rs:60-68, swiss.rs:308-316
    g = G["hash"]
    hs = {orc.LIB.orc_hash_u64(i) for i in range(g["distinct_u64"])}
    assert len(hs) == g["distinct_u64"]
    for a, b in g["bytes_differ"]:
        assert orc.LIB.orc_hash_bytes(a.encode(), len(a.encode())) != orc.LIB.orc_hash_bytes(b.encode(), len(b.encode()))
    s = G["swiss"]
    group = int.from_bytes(bytes(s["swar_group"]), "little")
    m = orc.LIB.orc_swar_match_tag(group, s["swar_tag"])
    hits = [i for i in range(8) if m & (0x80 << (i * 8))]
    assert all(h in hits for h in s["swar_hits_include"])
    assert orc.LIB.orc_swar_match_empty(group) == s["match_empty"]


def test_swiss_growth_and_collisions():  # swiss.rs:317-350, proptest_tables.rs:14-79
    s = G["swiss"]
    keys = list(range(s["grow_keys"]))
    out, n, cap = orc.swiss_batches([keys], 0)
    assert n == s["grow_keys"] and list(out) == keys and cap >= n
    out, n, _ = orc.swiss_batches([list(range(s["full_collision_keys"]))], 2)
    assert n == s["full_collision_keys"] and list(out) == list(range(n))
    rng = np.random.default_rng(7)
    for mode, hi in ((0, 500), (1, 200)):
        for _ in range(20):
            batches = [list(rng.integers(0, hi, rng.integers(0, 300))) for _ in range(rng.integers(0, 20))]
            out, n, _ = orc.swiss_batches(batches, mode)
            ref, exp = {}, []
            for b in batches:
                for k in b:
                    exp.append(ref.setdefault(int(k), len(ref)))
            assert list(out) == exp and n == len(ref)


def test_memory_pool():  # memory.rs:163-180
    g = G["memory_pool"]
    res, used, peak = orc.pool_script(g["limit"], g["script"])
    names = {abi.OK: "ok", abi.ERR_BUDGET: "budget"}
    assert [names[int(r)] for r in res] == g["status"]
    assert list(used) == g["used_after"] and peak[-1] == g["peak_end"]


def test_end_to_end_queries():  # end_to_end.rs:218-339 (1 and 4 threads)
    e = G["end_to_end"]
    lineitem, orders = e2e_tables()
    for threads in (1, 4):
        eng = orc.OracleEngine(threads=threads, batch_size=1000)
        r = q_count(eng, lineitem)
        assert [int(r[0].values[0]), int(r[1].values[0])] == [e["count_star_and_nulls"]["count_star"],
                                                            e["count_star_and_nulls"]["count_qty"]]
        g = e["group_by_order_by"]
        r = q_group_by(eng, lineitem, g["cutoff"])
        assert [s.decode() for s in r[0].strings()] == [row[0] for row in g["rows"]]
        assert rel_err(r[1].values, [row[1] for row in g["rows"]]).max() <= 1e-9
        assert list(r[2].values) == [row[2] for row in g["rows"]]
        assert rel_err(r[3].values, [row[3] for row in g["rows"]]).max() <= 1e-9
        assert list(r[4].values) == [row[4] for row in g["rows"]]
        j = e["join_top_n"]
        r, _ = q_join_top_n(eng, lineitem, orders, j["cutoff"])
        assert [s.decode() for s in r[0].strings()] == [row[0] for row in j["rows"]]
        assert rel_err(r[1].values, [row[1] for row in j["rows"]]).max() <= 1e-9
        c = e["case_in_like_between"]
        r = q_case_in_like_between(eng, lineitem)
        assert [int(r[0].values[0]), int(r[1].values[0])] == [c["sum_case"], c["count"]]


def test_memory_limit_refusal():  # memory_limit.rs:47-68
    from minilake_b200.abi import SUM, AggSpec
    g = G["memory_limit"]
    groups = g["groups"]
    rgs = []
    for b in range(g["batches"]):
        k = (np.arange(groups) * 7 + b) % groups
        rgs.append([fixed(INT64, k), fixed(INT64, np.ones(groups, dtype=np.int64))])
    from minilake_b200.columns import Table
    t = Table("t", ["k", "v"], rgs)
    eng = orc.OracleEngine(threads=1, memory_limit=g["budget"])
    with pytest.raises(orc.OracleBudgetError) as ei:
        eng.hashagg(t, [INT64, INT64], [(Col(0), INT64)], [AggSpec(SUM, Col(1), INT64)])
    assert ei.value.operator == "HashAggregate"
    ok = orc.OracleEngine(threads=2).fetch(orc.OracleEngine(threads=2).hashagg(
        t, [INT64, INT64], [(Col(0), INT64)], [AggSpec(SUM, Col(1), INT64)]))
    assert len(ok[0].values) == groups and (ok[1].values == g["batches"]).all()
