"""The serving loop: every query's result is the same alone and in the concurrent mix
(integers and strings exact, float64 within relative 1e-12), admission waits for memory
instead of failing, and latency / throughput are reported."""
import math

import pytest

pytestmark = pytest.mark.gpu
F64_TOL = 1e-12


def _same(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert len(x) == len(y)
        for u, v in zip(x, y):
            if isinstance(u, float):
                assert abs(u - v) <= F64_TOL * max(abs(v), 1e-300) or (math.isnan(u) and math.isnan(v)), (u, v)
            else:
                assert u == v


def test_results_alone_equal_results_in_the_mix():
    from minilake_b200 import serving
    srv = serving.Server(tables_per_shape=2, min_rows=200_000, max_rows=2_000_000, slots=4, learned=True, seed=46,
                         log=lambda *a: None)
    stream = serving.make_stream(90, 500.0, 2, seed=47)
    srv.serve(stream)
    assert all(q.error is None for q in stream), [q.error for q in stream if q.error][:3]
    for q in stream:  # alone: a fresh slot, one query at a time
        alone = srv.execute(serving.Query(q.qid, 0.0, q.shape, q.table, q.const), {})
        _same(alone, q.result)
    summary = serving.summarize(stream, srv)
    assert summary["completed"] == 90 and summary["p99_ms"] >= summary["p50_ms"] > 0
    assert summary["graph_replays"] > 0
    srv.close()


def test_admission_waits_for_memory_under_a_tight_budget():
    """With room for about one query's state at a time, queries wait to be admitted instead
    of failing, and all of them complete."""
    from minilake_b200 import serving
    srv = serving.Server(tables_per_shape=1, min_rows=200_000, max_rows=400_000, slots=4, learned=False, seed=48,
                         log=lambda *a: None, admit_limit=(16 << 20) + 64 * 1_500_000)
    stream = serving.make_stream(60, 2000.0, 1, seed=49)
    srv.serve(stream)
    assert all(q.error is None for q in stream)
    assert srv.budget_waits > 0
    srv.close()
