"""Writes tests/golden/known_answers.json: the known-answer cases of MiniLake's own
test suite for the hot path, transcribed from the reference test files (cited per
case), plus the expected results of its end-to-end SQL tests, recomputed here the
way those tests compute their references (plain iterators over the same
deterministic fixture rows, crates/minilake-sql/tests/end_to_end.rs:44-68,
218-339).

MiniLake is Rust and cannot be built or run in this environment, so these
asserted values are the golden vectors that pin the CPU oracle.

    python tests/golden/make_golden.py
"""
import json
import os
from datetime import date

HERE = os.path.dirname(os.path.abspath(__file__))


def days(s):  # days since 1970-01-01
    y, m, d = map(int, s.split("-"))
    return (date(y, m, d) - date(1970, 1, 1)).days


def end_to_end():
    """end_to_end.rs:21-68 fixture rows and the references of its tests."""
    n_line, n_ord = 10_000, 1_000
    flags = ["A", "N", "R"]
    prios = ["1-URGENT", "2-HIGH", "3-MEDIUM"]
    day0 = days("1995-01-01")
    lines = [dict(orderkey=i % n_ord, qty=None if i % 13 == 0 else float(i % 50), price=(i % 97) + 0.5,
                  flag=flags[i % 3], shipdate=day0 + i % 30) for i in range(n_line)]
    orders = [dict(orderkey=j, date=day0 + j // 100, prio=prios[j % 3]) for j in range(n_ord)]
    out = {}
    # count_star_and_nulls (end_to_end.rs:218-231)
    nulls = sum(1 for l in lines if l["qty"] is None)
    out["count_star_and_nulls"] = {"count_star": n_line, "count_qty": n_line - nulls}
    # group_by_order_by_matches_reference (end_to_end.rs:233-267)
    cutoff = days("1995-01-10")
    ref = {}
    for l in lines:
        if l["shipdate"] < cutoff:
            e = ref.setdefault(l["flag"], [0.0, 0, 0.0, 0, 2**31 - 1])
            e[0] += l["price"]
            e[1] += 1
            if l["qty"] is not None:
                e[2] += l["qty"]
                e[3] += 1
            e[4] = min(e[4], l["shipdate"])
    out["group_by_order_by"] = {
        "cutoff": cutoff,
        "rows": [[f, e[0], e[1], e[2] / e[3], e[4]] for f, e in sorted(ref.items())],
    }
    # join_top_n_matches_reference (end_to_end.rs:269-298)
    cut = days("1995-01-05")
    rev = {}
    for l in lines:
        o = orders[l["orderkey"]]
        if o["date"] >= cut:
            rev[o["prio"]] = rev.get(o["prio"], 0.0) + l["price"]
    exp = sorted(rev.items(), key=lambda kv: -kv[1])[:2]
    out["join_top_n"] = {"cutoff": cut, "rows": [[p, v] for p, v in exp]}
    # case_in_like_between (end_to_end.rs:319-339)
    sel = [l for l in lines if 10.0 <= l["price"] <= 20.0]
    ar = sum(1 for l in sel if l["flag"] in ("A", "R"))
    out["case_in_like_between"] = {"sum_case": ar, "count": len(sel)}
    return out


def known_answers():
    EMPTY = 0x80
    group = bytes([5, EMPTY, 7, 5, 0, 1, 2, 3])
    return {
        # kernels/cmp.rs:124-140
        "compare_scalar_and_select": {
            "values": [5, 1, 7, 3], "lt": 4, "mask": [False, True, False, True],
            "selection": [1, 3], "selection_with_input": {"input": [0, 3], "out": [3]},
            "selection_with_validity": {"valid": [True, False, True, True], "out": [3]},
        },
        "empty_and_all": {"all_true3": [0, 1, 2], "all_false3": [], "empty": []},
        # kernels/boolean.rs:69-84: rows (NULL,F) (NULL,T) (T,T)
        "kleene": {
            "a": [True, True, True], "a_valid": [False, False, True], "b": [False, True, True],
            "and_valid": [True, False, True], "and_value": [False, None, True],
            "or_valid": [False, True, True], "or_value": [None, True, True],
        },
        # kernels/arith.rs:136-153
        "arith_ops": {
            "a": [1, 2, 3], "b": [10, 20, 30], "add": [11, 22, 33], "sub_from_100": [90, 80, 70],
            "mod_zero_values": [0, 0, 0], "mul_one_minus": {"a": 10.0, "b": 0.1, "out": 9.0},
        },
        # expr/like.rs:134-166
        "like_shapes": {"PROMO%": ["prefix", "PROMO"], "%BRASS": ["suffix", "BRASS"],
                        "%green%": ["contains", "green"], "%a%b%": ["general", "%a%b%"]},
        "like_matching": [
            ["PROMO%", "PROMO BRUSHED", True], ["PROMO%", "STANDARD", False], ["%BRASS", "LARGE BRASS", True],
            ["%green%", "forest green metallic", True], ["%special%requests%", "a special big requests x", True],
            ["%special%requests%", "requests special", False], ["a_c", "abc", True], ["a_c", "abbc", False],
            ["%", "", True],
        ],
        # kernels/string.rs:37-49
        "like_on_plain_strings": {"values": ["PROMO A", "STD", "PROMO B"], "like": [True, False, True],
                                  "in_std": [False, True, False]},
        # expr/eval.rs:548-612: a = [1, 5, 10, 20] (INT64), b = [0.5, 1.5, 2.5, 3.5]
        "eval": {
            "a": [1, 5, 10, 20], "b": [0.5, 1.5, 2.5, 3.5],
            "select_a_ge5_and_b_lt3": [1, 2], "a_times_b_row3": 70.0,
            "b_div_zero_null_count": 4, "case_a_gt5_then1_else0": [0, 0, 1, 1],
        },
        # operators/aggregate/accumulator.rs:600-633
        "accumulator": {
            "values": [1.0, 2.0, 3.0, 4.0], "valid": [True, True, False, True], "gids": [0, 1, 0, 1],
            "sum": [1.0, 6.0], "avg_group1": 3.0,
        },
        # minilake-hashtable/src/swiss.rs:308-350
        "swiss": {
            "swar_group": list(group), "swar_tag": 5, "swar_hits_include": [0, 3], "match_empty": EMPTY << 8,
            "grow_keys": 10_000, "absent_key": 99_999, "full_collision_keys": 100,
        },
        # minilake-hashtable/src/hash.rs:60-68
        "hash": {"distinct_u64": 10_000, "bytes_differ": [["abc", "abd"], ["", "\u0000"]]},
        # kernels/scalar_ops.rs:158-164
        "scalar_kleene": {"null_and_false": False, "null_or_false": None},
        # minilake-exec/src/memory.rs:163-180: (reservation, op, bytes) with op 0 grow, 1 resize, 2 drop
        "memory_pool": {
            "limit": 100,
            "script": [[0, 0, 60], [1, 0, 50], [1, 0, 40], [0, 2, 0], [1, 1, 10]],
            "status": ["ok", "budget", "ok", "ok", "ok"],
            "used_after": [60, 60, 100, 40, 10], "peak_end": 100, "budget_used_observed": 60,
        },
        # minilake-exec/tests/memory_limit.rs:14-68
        "memory_limit": {"groups": 50_000, "batches": 10, "budget": 64 * 1024},
        # minilake-sql/tests/end_to_end.rs
        "end_to_end": end_to_end(),
    }


if __name__ == "__main__":
    path = os.path.join(HERE, "known_answers.json")
    with open(path, "w") as f:
        json.dump(known_answers(), f, indent=1, sort_keys=True)
    print("wrote", path)
