"""Prepared queries (ml_gpu_query_*): the first run plans through the sink calls, later runs
replay the whole plan (join build, fused aggregate, final values, top-N) as one CUDA graph.
Every run's result must equal the CPU oracle's on the batches' current contents (keys, counts
and row order bit-exact; f64 sums within 1e-12), including after the batches were rewritten in
place between runs; data that no longer fits the recorded plan must give StalePlan, not a wrong
answer; plans the graph cannot replay must say why and refuse a second run."""
import numpy as np
import pytest

from minilake_b200 import abi, workloads
from minilake_b200.abi import COUNT_STAR, FLOAT64, INT32, INT64, SUM, UTF8, AggSpec, Col, Filter, Lit, SortKey
from minilake_b200.columns import Table, encode_strings, fixed
from oracle import orc
from test_gpu_parity import F64_TOL, assert_same_rows

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from minilake_b200.gpu import Context
    c = Context(0)
    yield c
    c.close()


def _data(seed, nd=50_000, nf=1_000_000, sparse=False):
    rng = np.random.default_rng(seed)
    key = rng.permutation(nd).astype(np.int64) * (1_000_003 if sparse else 1) + 7
    fk = key[rng.integers(0, nd, nf)]
    miss = rng.random(nf) < 0.05
    fk[miss] = 10**12 + rng.integers(0, 1000, miss.sum())  # no build row
    d = rng.integers(0, 2500, nf, dtype=np.int32)
    v = np.round(rng.random(nf) * 100, 2)
    return key, fk, d, v


def _oracle_top(key, fk, d, v, limit=10):
    eng = orc.OracleEngine(threads=4)
    dim = Table("dim", ["key"], [[fixed(INT64, key)]])
    fact = Table("fact", ["fk", "d", "v"], [[fixed(INT64, fk), fixed(INT32, d), fixed(FLOAT64, v)]])
    return workloads.run_join_groupby(eng, dim, fact, limit=limit)


def _torch_table(cols):
    import torch
    from minilake_b200.serving import DeviceTable
    ts = [(t, torch.from_numpy(np.ascontiguousarray(a)).cuda(), None) for t, a in cols]
    return DeviceTable(ts), [x for _, x, _ in ts]


def _prepare(ctx, dim_ml, fact_ml, limit=10):
    from minilake_b200.gpu import HashAggregateSink, JoinBuildSink, Query
    q = Query(ctx)
    jt = q.add_build(JoinBuildSink(ctx, [INT64], [(Col(0), INT64)]), dim_ml)
    prologue, group, aggs = workloads.join_groupby_plan(jt)
    q.set_aggregate(HashAggregateSink(ctx, [INT64, INT32, FLOAT64], group, aggs, prologue), fact_ml)
    if limit:
        q.set_topn(workloads.join_groupby_topn_keys(), limit)
    return q


def _same_top(got, want):
    # (fk, sum, count) in order: keys and counts exact, sums within the tolerance
    assert len(got[0]) == len(want[0])
    assert np.array_equal(got[0].values, want[0].values)
    assert np.array_equal(got[2].values, want[2].values)
    np.testing.assert_allclose(got[1].values, want[1].values, rtol=F64_TOL, atol=0)


@pytest.mark.parametrize("sparse", [False, True])
def test_replays_match_the_oracle_and_follow_the_data(ctx, sparse):
    key, fk, d, v = _data(1 + sparse, sparse=sparse)
    dim, dim_t = _torch_table([(INT64, key)])
    fact, fact_t = _torch_table([(INT64, fk), (INT32, d), (FLOAT64, v)])
    q = _prepare(ctx, dim.ml, fact.ml)
    want = _oracle_top(key, fk, d, v)
    for _ in range(3):
        _same_top(q.run().fetch(), want)
    st = q.stats()
    assert st["why_not"] == "" and st["runs"] == 3 and st["replays"] == 2 and st["kernels"] > 5
    for _ in range(2):  # the result read back inside the graph
        _same_top(q.run_host(), want)
    assert q.stats()["replays"] == 4
    # new contents, same buffers: the replay recomputes everything from them
    rng = np.random.default_rng(9)
    v2 = np.round(rng.random(len(v)) * 100, 2)
    d2 = rng.integers(0, 2500, len(d), dtype=np.int32)
    key2 = key[rng.permutation(len(key))]  # the same keys in another order: the index is rebuilt
    import torch
    fact_t[1].copy_(torch.from_numpy(d2))
    fact_t[2].copy_(torch.from_numpy(v2))
    dim_t[0].copy_(torch.from_numpy(key2))
    _same_top(q.run_host(), _oracle_top(key2, fk, d2, v2))
    assert q.stats()["replays"] == 5
    q.close()


def test_a_build_key_outside_the_index_is_a_stale_plan(ctx):
    from minilake_b200.gpu import StalePlan
    key, fk, d, v = _data(3)
    dim, dim_t = _torch_table([(INT64, key)])
    fact, _ = _torch_table([(INT64, fk), (INT32, d), (FLOAT64, v)])
    q = _prepare(ctx, dim.ml, fact.ml)
    q.run()
    _same_top(q.run().fetch(), _oracle_top(key, fk, d, v))
    key2 = key.copy()
    key2[5] = key.max() + 10**6  # past the dense index's range
    import torch
    dim_t[0].copy_(torch.from_numpy(key2))
    with pytest.raises(StalePlan, match="dense index"):
        q.run()
    with pytest.raises(StalePlan):
        q.run()
    q.close()
    # a new plan over the changed data is right again
    q = _prepare(ctx, dim.ml, fact.ml)
    _same_top(q.run().fetch(), _oracle_top(key2, fk, d, v))
    _same_top(q.run().fetch(), _oracle_top(key2, fk, d, v))
    q.close()


def test_duplicate_build_keys_appearing_is_a_stale_plan(ctx):
    from minilake_b200.gpu import StalePlan
    key, fk, d, v = _data(4)
    dim, dim_t = _torch_table([(INT64, key)])
    fact, _ = _torch_table([(INT64, fk), (INT32, d), (FLOAT64, v)])
    q = _prepare(ctx, dim.ml, fact.ml)
    q.run()
    key2 = key.copy()
    key2[1] = key2[0]
    import torch
    dim_t[0].copy_(torch.from_numpy(key2))
    with pytest.raises(StalePlan, match="duplicates"):
        q.run()
    q.close()


def _grouped_plan(ctx, fact_ml, size_hint, limit):
    # GROUP BY a fact column (hashed groups), no join: SUM(v), COUNT(*) by g, top-N by sum
    from minilake_b200.gpu import HashAggregateSink, Query
    q = Query(ctx)
    q.set_aggregate(HashAggregateSink(ctx, [INT64, FLOAT64], [(Col(0), INT64)],
                                      [AggSpec(SUM, Col(1), FLOAT64), AggSpec(COUNT_STAR)],
                                      [Filter(Col(1) > Lit(1.0))], size_hint), fact_ml)
    if limit:
        q.set_topn([SortKey(Col(1), FLOAT64, asc=False), SortKey(Col(0), INT64)], limit)
    return q


def _oracle_grouped(g, v, limit):
    eng = orc.OracleEngine(threads=4)
    t = Table("t", ["g", "v"], [[fixed(INT64, g), fixed(FLOAT64, v)]])
    out = eng.hashagg(t, [INT64, FLOAT64], [(Col(0), INT64)], [AggSpec(SUM, Col(1), FLOAT64), AggSpec(COUNT_STAR)],
                      [Filter(Col(1) > Lit(1.0))])
    if limit:
        out = eng.topn(out, [INT64, FLOAT64, INT64], [SortKey(Col(1), FLOAT64, asc=False), SortKey(Col(0), INT64)],
                       limit)
    return eng.fetch(out)


def test_hashed_groups_without_a_top_n_and_overflow(ctx):
    from minilake_b200.gpu import StalePlan
    rng = np.random.default_rng(5)
    n = 800_000
    g = rng.integers(0, 20_000, n).astype(np.int64) * 7919
    v = np.round(rng.random(n) * 10, 3)
    fact, fact_t = _torch_table([(INT64, g), (FLOAT64, v)])
    q = _grouped_plan(ctx, fact.ml, 40_000, None)  # sized for 20k groups: no resize in the planning run
    want = _oracle_grouped(g, v, None)
    for _ in range(3):
        assert_same_rows(q.run().fetch(), want, 1, {1})
    assert q.stats()["replays"] == 2
    # many more groups than the recorded table holds: the overflow check stops the replay
    import torch
    g2 = rng.integers(0, 600_000, n).astype(np.int64)
    fact_t[0].copy_(torch.from_numpy(g2))
    with pytest.raises(StalePlan, match="overflowed"):
        q.run()
    q.close()


@pytest.mark.parametrize("limit", [1, 7, 32])
def test_hashed_groups_top_n(ctx, limit):
    rng = np.random.default_rng(6 + limit)
    n = 500_000
    g = rng.integers(0, 50_000, n).astype(np.int64) - 25_000
    v = np.round(rng.random(n) * 10, 3)
    fact, _ = _torch_table([(INT64, g), (FLOAT64, v)])
    q = _grouped_plan(ctx, fact.ml, 0, limit)
    want = _oracle_grouped(g, v, limit)
    for _ in range(3):
        got = q.run().fetch()
        assert np.array_equal(got[0].values, want[0].values) and np.array_equal(got[2].values, want[2].values)
        np.testing.assert_allclose(got[1].values, want[1].values, rtol=F64_TOL, atol=0)
    q.close()


def test_fewer_groups_than_the_limit(ctx):
    from minilake_b200.gpu import StalePlan
    g = np.repeat(np.arange(5, dtype=np.int64), 1000)
    v = np.full(len(g), 2.0)
    fact, fact_t = _torch_table([(INT64, g), (FLOAT64, v)])
    q = _grouped_plan(ctx, fact.ml, 0, 10)
    for _ in range(2):
        got = q.run().fetch()
        assert got[0].values.tolist() == [0, 1, 2, 3, 4]
    # a sixth group would change the result's row count: the planned rows no longer hold
    import torch
    g2 = g.copy()
    g2[0] = 99
    fact_t[0].copy_(torch.from_numpy(g2))
    with pytest.raises(StalePlan, match="result rows"):
        q.run()
    q.close()


def test_a_plan_the_graph_cannot_replay_runs_once(ctx):
    from minilake_b200.gpu import HashAggregateSink, MiniLakeError, Query
    rng = np.random.default_rng(8)
    n = 10_000
    words = [b"a", b"bb", b"ccc"]
    cols = [encode_strings(words, rng.integers(0, 3, n)), fixed(FLOAT64, rng.random(n))]
    batch = ctx.upload(cols)
    q = Query(ctx)
    q.set_aggregate(HashAggregateSink(ctx, [UTF8, FLOAT64], [(Col(0), UTF8)], [AggSpec(SUM, Col(1), FLOAT64)]),
                    batch)
    got = q.run().fetch()
    assert sorted(got[0].strings()) == words
    assert "string" in q.stats()["why_not"]
    with pytest.raises(MiniLakeError) as ei:
        q.run()
    assert ei.value.code == abi.ERR_UNSUPPORTED
    q.close()


def test_nullable_inputs_through_a_replay(ctx):
    # NULL fact values and NULL build keys: the replay keeps the seen-counts and skips NULL keys
    from minilake_b200.gpu import HashAggregateSink, JoinBuildSink, Query
    rng = np.random.default_rng(10)
    nd, nf = 20_000, 300_000
    key = rng.permutation(nd).astype(np.int64)
    kvalid = rng.random(nd) > 0.02
    fk = rng.integers(0, nd, nf).astype(np.int64)
    d = rng.integers(0, 2500, nf, dtype=np.int32)
    v = rng.random(nf)
    vvalid = rng.random(nf) > 0.1
    dim_cols = [fixed(INT64, key, kvalid)]
    fact_cols = [fixed(INT64, fk), fixed(INT32, d), fixed(FLOAT64, v, vvalid)]
    dim_b, fact_b = ctx.upload(dim_cols), ctx.upload(fact_cols)
    q = Query(ctx)
    jt = q.add_build(JoinBuildSink(ctx, [INT64], [(Col(0), INT64)]), dim_b)
    prologue, group, aggs = workloads.join_groupby_plan(jt)
    q.set_aggregate(HashAggregateSink(ctx, [INT64, INT32, FLOAT64], group, aggs, prologue), fact_b)
    q.set_topn(workloads.join_groupby_topn_keys(), 10)
    eng = orc.OracleEngine(threads=4)
    want = workloads.run_join_groupby(eng, Table("dim", ["key"], [dim_cols]), Table("fact", ["fk", "d", "v"], [fact_cols]))
    for _ in range(3):
        _same_top(q.run().fetch(), want)
    assert q.stats()["replays"] == 2
    q.close()
