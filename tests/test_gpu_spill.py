"""Out-of-HBM aggregation (aggregate/hash.rs:189-281, 330-425; memory_limit.rs:70-101): with
ML_CTX_SPILL, a GROUP BY whose table outgrows the HBM budget moves its partial states to host
memory in 16 hash partitions and merges them one partition at a time at finalize.  The result must
equal the oracle's (keys, counts, integer sums, MIN/MAX bit-exact; f64 SUM/AVG within 1e-12),
the pool's peak must stay within the budget, and without spilling the same budget must refuse
the query with ResourcesExhausted and release everything."""
import numpy as np
import pytest

from minilake_b200.abi import AVG, COUNT_STAR, FLOAT64, INT64, MAX, MIN, SUM, AggSpec, Col
from minilake_b200.columns import Table, fixed
from oracle import orc
from test_gpu_parity import assert_same_rows

pytestmark = pytest.mark.gpu

GROUPS, BATCHES = 500_000, 8
BUDGET = 48 << 20  # holds half the table, or the output and one partition's table
AGGS = [AggSpec(SUM, Col(1), INT64), AggSpec(SUM, Col(2), FLOAT64), AggSpec(COUNT_STAR), AggSpec(MIN, Col(2), FLOAT64),
        AggSpec(MAX, Col(1), INT64), AggSpec(AVG, Col(2), FLOAT64)]


def _table():
    rng = np.random.default_rng(3)
    perm = rng.permutation(GROUPS).astype(np.int64) * 1_000_003 + 17
    rgs = []
    for b in range(BATCHES):
        k = perm[(np.arange(GROUPS) * 7 + b * 13) % GROUPS]  # every batch holds every group
        v = rng.integers(-1000, 1000, GROUPS)
        x = rng.uniform(1.0, 1e3, GROUPS)  # positive: sums do not cancel
        xv = rng.random(GROUPS) > 0.1
        if b == 0:
            xv[:] = True  # the first morsel has no NULL: counting valid inputs starts mid-query
        rgs.append([fixed(INT64, k), fixed(INT64, v), fixed(FLOAT64, x, xv)])
    return Table("t", ["k", "v", "x"], rgs)


@pytest.mark.parametrize("threads", [1, 2])
def test_spilled_aggregate_matches_oracle_within_budget(threads):
    from minilake_b200.engine import GpuEngine
    from minilake_b200.gpu import SPILL, Context, HashAggregateSink
    t = _table()
    ctx = Context(0, hbm_budget=BUDGET, flags=SPILL)
    eng = GpuEngine(ctx, threads=threads)
    sink = HashAggregateSink(ctx, [INT64, INT64, FLOAT64], [(Col(0), INT64)], AGGS)
    eng.drive(sink, t)
    out = sink.finalize()
    stats = sink.stats()
    got = out.fetch()
    out.close()
    sink.close()
    used, peak, limit = ctx.pool_stats()
    assert stats["spills"] > 0 and stats["groups"] == GROUPS
    assert peak <= BUDGET, f"peak {peak} above the budget"
    assert used == 0
    want = orc.OracleEngine(threads=8).fetch(
        orc.OracleEngine(threads=8).hashagg(t, [INT64, INT64, FLOAT64], [(Col(0), INT64)], AGGS))
    assert_same_rows(got, want, 1, {2, 6})
    ctx.close()


def test_without_spilling_the_budget_refuses():
    from minilake_b200.engine import GpuEngine
    from minilake_b200.gpu import Context, ResourcesExhausted
    ctx = Context(0, hbm_budget=BUDGET)
    with pytest.raises(ResourcesExhausted) as ei:
        GpuEngine(ctx).hashagg(_table(), [INT64, INT64, FLOAT64], [(Col(0), INT64)], AGGS)
    assert ei.value.operator.startswith("HashAggregate")
    assert ctx.pool_stats()[0] == 0
    ctx.close()
