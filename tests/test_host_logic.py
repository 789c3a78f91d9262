"""Host-side logic of the measurement and serving drivers (CPU, no device): the Poisson query
stream, the latency summary, the learned-sizing instance generator and q-error, and the
per-operator throughput arithmetic."""
import math
from types import SimpleNamespace

import numpy as np

from minilake_b200 import cardinality, opbench, serving


def test_query_stream_is_seeded_poisson_over_the_three_shapes():
    a = serving.make_stream(5000, 200.0, 4, seed=46)
    b = serving.make_stream(5000, 200.0, 4, seed=46)
    assert [(q.arrival, q.shape, q.table, q.const) for q in a] == [(q.arrival, q.shape, q.table, q.const) for q in b]
    gaps = np.diff([0.0] + [q.arrival for q in a])
    assert np.all(gaps > 0)
    assert abs(gaps.mean() - 1 / 200.0) < 0.1 / 200.0  # exponential inter-arrivals at the rate
    shapes = np.bincount([q.shape for q in a], minlength=3)
    assert shapes.min() > 1500  # each shape about a third
    for q in a:
        assert 0 <= q.table < 4
        if q.shape < 2:
            assert isinstance(q.const, int) and 0 <= q.const < 2557  # a cutoff
        else:
            assert isinstance(q.const, str) and len(q.const) == 2 and q.const.isalpha()  # a LIKE prefix


def test_latency_summary_percentiles_and_rates():
    stream = []
    for i in range(100):  # latencies 1..100 ms, arrivals every 10 ms
        q = serving.Query(i, i * 0.01, i % 3, 0, 5)
        q.done, q.error = q.arrival + (i + 1) * 1e-3, None
        stream.append(q)
    failed = serving.Query(100, 1.0, 0, 0, 5)
    failed.error = "refused"
    stream.append(failed)
    table = SimpleNamespace(rows=1_000_000)
    server = SimpleNamespace(tables=[[table]] * 3, budget_waits=0, budget_retries=0,
                             graphs={"built": 1, "replayed": 2}, rows=[[1]], learned=False, slots=8)
    s = serving.summarize(stream, server)
    lat = np.arange(1, 101, dtype=float)
    assert s["completed"] == 100 and s["failed"] == 1 and s["queries"] == 101
    assert math.isclose(s["p50_ms"], np.percentile(lat, 50)) and math.isclose(s["p99_ms"], np.percentile(lat, 99))
    assert math.isclose(s["max_ms"], 100.0)
    span = stream[99].done - stream[0].arrival
    assert math.isclose(s["queries_per_s"], 100 / span)
    algo = sum(1_000_000 * serving.BYTES_PER_ROW[q.shape] for q in stream[:100])
    assert math.isclose(s["algorithmic_GB_per_s"], algo / span / 1e9)
    assert set(s["per_shape"]) == set(serving.SHAPES)


def test_learned_sizing_instances_and_q_error():
    insts = cardinality.make_instances(400, seed=45, min_rows=1_000_000, max_rows=100_000_000)
    assert insts == cardinality.make_instances(400, seed=45, min_rows=1_000_000, max_rows=100_000_000)
    for inst in insts:
        assert 1_000_000 <= inst.rows <= 100_000_000
        assert 1 <= inst.distinct <= min(inst.rows, 1 << 26)
        assert inst.key_type in cardinality.KEY_TYPES and inst.dist in cardinality.DISTS
        assert 0.5 <= inst.s <= 1.5 and 0.0 <= inst.null_frac <= 0.1
    assert {i.key_type for i in insts} == set(cardinality.KEY_TYPES)
    q = cardinality.q_error(np.array([10.0, 40.0, 0.5]), np.array([20.0, 20.0, 1.0]))
    assert np.allclose(q, [2.0, 2.0, 1.0])  # symmetric; estimates below 1 count as 1


def test_operator_line_arithmetic():
    line = opbench._line(100_000_000, 0.5, 3_600_000_000, 6650.0)
    assert math.isclose(line["gbs"], 7200.0)  # 3.6 GB in 0.5 ms
    assert math.isclose(line["rows_per_s"], 2e11)
    assert math.isclose(line["frac_of_hbm_peak"], round(7200.0 / 6650.0, 3))
    peak, kind = opbench.hbm_peak()
    assert peak > 0 and kind in ("measured", "fallback")


def test_bench_data_shards_and_traffic_record():
    """bench.py: every rank's share of the fact table references keys over all of 1..1.5M (a
    split by row group, so the ranks' partial aggregates overlap and need the exchange), the
    dimension keys are a permutation of 1..1.5M, and the DRAM bytes per launch carried for the
    bench line's `roofline.traffic` cover at least the algorithmic bytes."""
    import bench
    for world in (1, 2, 4):
        for rank in range(world):
            key, fk, d, v = bench.make_data(rank, world, fact_rows=20_000)
            assert np.array_equal(np.sort(key), np.arange(1, bench.DIM_ROWS + 1))
            assert fk.min() >= 1 and fk.max() <= bench.DIM_ROWS
            assert len(np.unique(fk % 4)) == 4
            assert d.min() >= 0 and d.max() < 2557 and v.min() >= 900.0 and v.max() < 105000.0
    assert bench.NCU_DRAM_BYTES_PER_LAUNCH >= bench.FACT_ROWS * bench.BYTES_PER_ROW
    peak, kind = bench.measured_peak()
    assert peak > 0 and kind in ("measured", "fallback")
