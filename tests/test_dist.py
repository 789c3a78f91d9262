"""The multi-GPU path on CPU: world_size 2 gloo processes run the join + GROUP BY + top-10 query
on their shards of the fact table (partitioned on the join key, dimension replicated) with the
oracle engine, exchange their local top-10s, and must get the single-process answer."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROWS = 120_000


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    from minilake_b200 import workloads
    from minilake_b200.exchange import exchange_topn
    from oracle import orc
    key, fk, d, v = bench.make_data(rank, world, ROWS)
    dim, fact = bench.oracle_tables(key, fk, d, v)
    top = workloads.run_join_groupby(orc.OracleEngine(threads=2), dim, fact)
    mk, ms, mc = exchange_topn(top[0].values, top[1].values, top[2].values, 10)
    out.put((rank, set(np.unique(fk).tolist()) if rank == 0 else None, fk.copy(), d.copy(), v.copy(),
             mk.tolist(), ms.tolist(), mc.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_exchange_matches_single_process():
    import bench
    from minilake_b200 import workloads
    from oracle import orc
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # the shards hold disjoint keys (k % 2 == rank)
    assert all(k % 2 == 0 for k in np.unique(res[0][2])) and all(k % 2 == 1 for k in np.unique(res[1][2]))
    assert res[0][5:] == res[1][5:], "every rank gets the same merged answer"
    # the single-process query over both shards
    key = bench.make_data(0, 1, 1)[0]
    fk = np.concatenate([res[0][2], res[1][2]])
    d = np.concatenate([res[0][3], res[1][3]])
    v = np.concatenate([res[0][4], res[1][4]])
    dim, fact = bench.oracle_tables(key, fk, d, v)
    want = workloads.run_join_groupby(orc.OracleEngine(threads=2), dim, fact)
    assert res[0][5] == want[0].values.tolist()
    assert res[0][7] == want[2].values.tolist()
    np.testing.assert_allclose(res[0][6], want[1].values, rtol=1e-12)
