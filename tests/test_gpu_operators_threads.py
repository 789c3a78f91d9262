"""Standalone operators called from many threads at once, as MiniLake's workers call
Operator::execute on one shared operator (pipeline.rs:52-57): each call runs on its own pooled
stream, and every thread's result must equal the same call made alone (selections, probe pairs
and hashes are index work: identical)."""
import threading

import numpy as np
import pytest

from minilake_b200.abi import FLOAT64, INT64, Col, Lit
from minilake_b200.columns import fixed

pytestmark = pytest.mark.gpu


def test_filter_probe_and_hash_from_eight_threads():
    from minilake_b200.gpu import Context, FilterOperator, HashJoinProbe, JoinBuildSink, hash_columns
    ctx = Context(0)
    rng = np.random.default_rng(11)
    j = JoinBuildSink(ctx, [INT64], [(Col(0), INT64)])
    loc = j.create_local()
    loc.sink([fixed(INT64, rng.permutation(200_000).astype(np.int64) * 2)])
    loc.combine()
    j.finalize()
    batches = []
    for t in range(8):
        n = 300_000 + 1000 * t
        batches.append([fixed(INT64, rng.integers(0, 400_000, n)), fixed(FLOAT64, rng.random(n))])
    filt = FilterOperator(ctx, Col(1) > Lit(0.3))
    probe = HashJoinProbe(ctx, j.table, [(Col(0), INT64)])

    def work(cols):
        sel = filt.execute(cols)
        pi, bi = probe.execute(cols, sel)
        h = hash_columns(ctx, cols, sel)
        return sel, pi, bi, h

    alone = [work(b) for b in batches]
    got = [None] * len(batches)
    errors = []

    def run(i):
        try:
            for _ in range(3):
                got[i] = work(batches[i])
        except BaseException as e:  # reported below
            errors.append(e)

    ts = [threading.Thread(target=run, args=(i,)) for i in range(len(batches))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors
    for a, g in zip(alone, got):
        for x, y in zip(a, g):
            assert np.array_equal(x, y)
    j.close()
    ctx.close()
