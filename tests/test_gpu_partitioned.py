"""The radix-partitioned aggregation against the CPU oracle.

It runs when the GROUP BY key is the join key of a probe (the group id is the probe's match),
the group space is larger than shared memory holds, and a launch has at least 2^20 rows.  Every
group's key and COUNT must match bit-exact, MIN/MAX bit-exact, f64 SUM/AVG within 1e-12
relative.  Cases: the join + GROUP BY of the benchmark with one launch spanning several phase
A/B rounds (8,388,608 rows each); skewed keys that fill one partition's shared-memory buffer
and its regions (the records past them take the direct path); a hashed (not dense) build side
with every accumulator kind.
"""
import numpy as np
import pytest

from helpers import rel_err
from minilake_b200.abi import AVG, COUNT, COUNT_STAR, FLOAT64, INT32, INT64, MAX, MIN, SUM, AggSpec, Col, Filter, Lit, Probe
from minilake_b200.columns import Table, fixed
from oracle import orc

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    from minilake_b200.gpu import PROFILE, Context
    c = Context(0, flags=PROFILE)
    yield c
    c.close()


def _tables(key, fk, d, v, groups=8):
    dim = Table("dim", ["key"], [[fixed(INT64, c)] for c in np.array_split(key, 2)])
    fact = Table("fact", ["fk", "d", "v"],
                 [[fixed(INT64, a), fixed(INT32, b), fixed(FLOAT64, c)]
                  for a, b, c in zip(np.array_split(fk, groups), np.array_split(d, groups), np.array_split(v, groups))])
    return dim, fact


def _gpu_agg(ctx, key, fk, d, v, group, aggs, prologue_fn):
    """One launch over the whole fact table (one device-resident morsel), like the benchmark."""
    from minilake_b200.engine import GpuEngine
    eng = GpuEngine(ctx)
    dim_dev = ctx.upload([fixed(INT64, key)])
    fact_dev = ctx.upload([fixed(INT64, fk), fixed(INT32, d), fixed(FLOAT64, v)])
    j = eng.join_build([dim_dev], [INT64], [(Col(0), INT64)])
    ctx.profile("part_scatter", reset=True)
    out = eng.hashagg([fact_dev], [INT64, INT32, FLOAT64], group, aggs, prologue_fn(j.handle))
    launches, _ = ctx.profile("part_scatter", reset=True)
    cols = out.fetch()
    out.close()
    j.close()
    return cols, launches


def _oracle_agg(key, fk, d, v, group, aggs, prologue_fn):
    eng = orc.OracleEngine(threads=8)
    dim, fact = _tables(key, fk, d, v)
    j = eng.join_build(dim, [INT64], [(Col(0), INT64)])
    return eng.fetch(eng.hashagg(fact, [INT64, INT32, FLOAT64], group, aggs, prologue_fn(j.handle)))


def _by_key(cols):
    order = np.argsort(cols[0].values, kind="stable")
    return [c.values[order] for c in cols], [c.valid_mask()[order] for c in cols]


def _join_plan(cutoff):
    return lambda h: [Filter(Col(1) > Lit(cutoff)), Probe(h, [(Col(0), INT64)], build_is_left=True)]


def _check_join_groupby(ctx, key, fk, d, v, cutoff=1200):
    group = [(Col(1), INT64)]
    aggs = [AggSpec(SUM, Col(3), FLOAT64), AggSpec(COUNT_STAR)]
    got, launches = _gpu_agg(ctx, key, fk, d, v, group, aggs, _join_plan(cutoff))
    want = _oracle_agg(key, fk, d, v, group, aggs, _join_plan(cutoff))
    (gk, gs, gc), _ = _by_key(got)
    (wk, ws, wc), _ = _by_key(want)
    assert np.array_equal(gk, wk), "group keys differ"
    assert np.array_equal(gc, wc), "COUNT(*) differs"
    assert rel_err(gs, ws).max() <= TOL
    return launches


def test_dense_groups_several_rounds(ctx):
    rng = np.random.Generator(np.random.PCG64(7))
    dim_rows, rows = 1_500_000, 20_000_000
    key = (rng.permutation(dim_rows) + 1).astype(np.int64)
    fk = rng.integers(1, dim_rows + 1, rows, dtype=np.int64)
    d = rng.integers(0, 2557, rows, dtype=np.int32)
    v = rng.uniform(900.0, 105000.0, rows)
    launches = _check_join_groupby(ctx, key, fk, d, v)
    assert launches == 3, f"expected three phase A rounds of 8,388,608 rows, got {launches}"


def test_skewed_keys_take_the_direct_path(ctx):
    rng = np.random.Generator(np.random.PCG64(8))
    dim_rows, rows = 1_500_000, 6_000_000
    key = (rng.permutation(dim_rows) + 1).astype(np.int64)
    fk = rng.integers(1, dim_rows + 1, rows, dtype=np.int64)
    hot = rng.random(rows) < 0.6
    fk[hot] = 777_777  # one key: its partition's buffers and regions overflow
    near = rng.random(rows) < 0.2
    fk[near] = rng.integers(1, 9_000, int(near.sum()), dtype=np.int64)  # one key range
    d = rng.integers(0, 2557, rows, dtype=np.int32)
    v = rng.uniform(900.0, 105000.0, rows)
    assert _check_join_groupby(ctx, key, fk, d, v, cutoff=100) == 1


def test_hashed_build_every_accumulator(ctx):
    rng = np.random.Generator(np.random.PCG64(9))
    dim_rows, rows = 300_000, 6_000_000
    key = rng.choice(1 << 40, dim_rows, replace=False).astype(np.int64)  # sparse: a hash table
    fk = key[rng.integers(0, dim_rows, rows)]
    miss = rng.random(rows) < 0.1
    fk[miss] = -fk[miss] - 1  # no match
    d = rng.integers(-5000, 5000, rows, dtype=np.int32)
    v = rng.normal(0.0, 1e4, rows)
    group = [(Col(1), INT64)]
    aggs = [AggSpec(SUM, Col(3), FLOAT64), AggSpec(AVG, Col(3), FLOAT64), AggSpec(MIN, Col(3), FLOAT64),
            AggSpec(MAX, Col(2), INT32), AggSpec(COUNT, Col(3), FLOAT64), AggSpec(COUNT_STAR)]

    def plan(h):
        return [Probe(h, [(Col(0), INT64)], build_is_left=True)]

    got, launches = _gpu_agg(ctx, key, fk, d, v, group, aggs, plan)
    assert launches == 1
    want = _oracle_agg(key, fk, d, v, group, aggs, plan)
    g, gv = _by_key(got)
    w, wv = _by_key(want)
    assert np.array_equal(g[0], w[0])
    for k in (3, 4, 5, 6):  # MIN, MAX, COUNT(v), COUNT(*)
        assert np.array_equal(g[k], w[k]), f"column {k} differs"
    # SUM and AVG of signed values: the tolerance scales with the summed magnitudes
    scale = np.bincount(np.searchsorted(w[0], fk[~miss]), weights=np.abs(v[~miss]), minlength=len(w[0]))
    assert (np.abs(g[1] - w[1]) <= TOL * scale).all(), "SUM differs"
    assert (np.abs(g[2] - w[2]) <= TOL * scale / w[6]).all(), "AVG differs"
    for k in range(7):
        assert np.array_equal(gv[k], wv[k])


def test_small_launches_keep_the_plain_kernel(ctx):
    rng = np.random.Generator(np.random.PCG64(10))
    dim_rows, rows = 200_000, 600_000
    key = (rng.permutation(dim_rows) + 1).astype(np.int64)
    fk = rng.integers(1, dim_rows + 1, rows, dtype=np.int64)
    d = rng.integers(0, 2557, rows, dtype=np.int32)
    v = rng.uniform(900.0, 105000.0, rows)
    assert _check_join_groupby(ctx, key, fk, d, v) == 0
