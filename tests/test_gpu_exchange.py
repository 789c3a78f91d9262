"""The device side of the multi-GPU exchange on one B200.

ml_gpu_partition must group rows by hash_columns(keys) % nparts exactly as the oracle's hash
assigns them, keep input order within each partition, and carry every column (validity
included).  The whole device path (Partial aggregate, partitioning, torch views of the device
columns, NCCL all-to-all, Final merge from the received tensors) runs in a one-rank NCCL group
and must match the oracle's single-process aggregate; the partitioning across several ranks is
covered by the gloo test on CPU.
"""
import os
import socket

import numpy as np
import pytest

from minilake_b200.abi import AVG, COUNT, COUNT_STAR, FLOAT64, INT32, INT64, MAX, MIN, SUM, AggSpec, Col, Filter, Lit
from minilake_b200.columns import fixed
from oracle import orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from minilake_b200.gpu import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("nparts", [1, 3, 7, 64])
def test_partition_groups_rows_by_key_hash(ctx, nparts):
    from minilake_b200.gpu import partition
    rng = np.random.default_rng(nparts)
    n = 300_001
    k = rng.integers(-(1 << 40), 1 << 40, n)
    d = rng.integers(0, 1000, n, dtype=np.int32)
    v = rng.normal(size=n)
    valid = rng.random(n) > 0.3
    cols = [fixed(INT64, k), fixed(INT32, d), fixed(FLOAT64, v, valid)]
    out, counts = partition(ctx, cols, [0, 1], nparts)
    h = orc.hash_columns(cols[:2])
    dest = (h % np.uint64(nparts)).astype(np.int64)
    order = np.argsort(dest, kind="stable")
    assert counts.tolist() == np.bincount(dest, minlength=nparts).tolist()
    got = out.fetch()
    assert np.array_equal(got[0].values, k[order])
    assert np.array_equal(got[1].values, d[order])
    assert np.array_equal(got[2].valid_mask(), valid[order])
    assert np.array_equal(got[2].values[valid[order]], v[order][valid[order]])
    out.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_device_exchange_path_in_one_rank_group(ctx):
    import torch
    import torch.distributed as dist
    from minilake_b200 import exchange
    from minilake_b200.abi import Probe
    from minilake_b200.engine import GpuEngine
    from minilake_b200.gpu import ProjectionOperator
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    from datetime import timedelta
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        rng = np.random.default_rng(3)
        dim_rows, n = 200_000, 3_000_000
        key = (rng.permutation(dim_rows) + 1).astype(np.int64)
        fk = rng.integers(1, dim_rows + 1, n, dtype=np.int64)
        d = rng.integers(0, 2557, n, dtype=np.int32)
        x = rng.normal(0.0, 100.0, n)
        xv = (rng.random(n) > 0.2) & (d % 97 != 5)
        fact = [fixed(INT64, fk), fixed(INT32, d), fixed(FLOAT64, x, xv)]
        eng = GpuEngine(ctx)
        dim_dev = ctx.upload([fixed(INT64, key)])
        fact_dev = ctx.upload(fact)
        j = eng.join_build([dim_dev], [INT64], [(Col(0), INT64)])
        # after the probe: [key, fk, d, x]
        prologue = [Filter(Col(1) > Lit(100)), Probe(j.handle, [(Col(0), INT64)], build_is_left=True)]
        group = [(Col(2), INT32)]
        aggs = [AggSpec(SUM, Col(3), FLOAT64), AggSpec(AVG, Col(3), FLOAT64), AggSpec(MIN, Col(3), FLOAT64),
                AggSpec(MAX, Col(3), FLOAT64), AggSpec(COUNT, Col(3), FLOAT64), AggSpec(COUNT_STAR)]
        final, proj = exchange.distributed_hashagg(eng, exchange.DeviceSide(eng), [fact_dev],
                                                   [INT64, INT32, FLOAT64], group, aggs, prologue, 1)
        got = [ProjectionOperator(ctx, e, t).execute(final).fetch()[0] for e, t in proj]
        oeng = orc.OracleEngine(threads=8)
        oj = oeng.join_build([fixed(INT64, key)], [INT64], [(Col(0), INT64)])
        oprologue = [Filter(Col(1) > Lit(100)), Probe(oj.handle, [(Col(0), INT64)], build_is_left=True)]
        want = oeng.fetch(oeng.hashagg(fact, [INT64, INT32, FLOAT64], group, aggs, oprologue))
        go, wo = np.argsort(got[0].values), np.argsort(want[0].values)
        assert np.array_equal(got[0].values[go], want[0].values[wo])
        for c in range(1, len(want)):
            gm, wm = got[c].valid_mask()[go], want[c].valid_mask()[wo]
            assert np.array_equal(gm, wm), f"column {c}: NULLs differ"
            gv, wv = got[c].values[go][wm], want[c].values[wo][wm]
            if want[c].dtype == FLOAT64:
                np.testing.assert_allclose(gv, wv, rtol=1e-12, atol=1e-9, err_msg=f"column {c}")
            else:
                assert np.array_equal(gv, wv), f"column {c} differs"
        assert (~want[1].valid_mask()).any(), "some groups see no valid input (NULL states)"
        final.close()
        j.close()
    finally:
        dist.destroy_process_group()
