"""The multi-GPU plan on CPU: world-size-2 gloo processes split one fact table by row group (not
by key), aggregate their shares in Partial mode with the oracle engine, exchange the partial
states by key hash (all-to-all), merge the groups they own in Final mode, and gather the
top-10.  Together they must give the single-process answer: every group of the aggregate
(keys and counts bit-exact, sums within 1e-12), disjoint group ownership by hash, and the same
merged top-10 on every rank.  A second query has NULL inputs, groups whose states are NULL,
AVG, MIN and MAX."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from minilake_b200 import abi, exchange

ROWS, DIM, GROUPS = 120_000, 40_000, 12


class HostSide:
    """The exchange step over host columns for the CPU engine (gloo): the counterpart of
    minilake_b200.exchange.DeviceSide, partitioning with the oracle's hash_columns."""

    device = "cpu"

    def __init__(self, engine):
        self.engine = engine

    def partition(self, batch, nkeys: int, world: int):
        """([(dtype, values, valid-or-None)], counts): the batch's columns with their rows grouped
        by destination rank."""
        from oracle import orc

        from minilake_b200.columns import fixed
        cols = self.engine.fetch(batch)
        n = len(cols[0]) if cols else 0
        h = orc.hash_columns(cols[:nkeys]) if n else np.zeros(0, np.uint64)
        dest = (np.asarray(h, dtype=np.uint64) % np.uint64(world)).astype(np.int64)
        order = np.argsort(dest, kind="stable")
        counts = np.bincount(dest, minlength=world)
        if any(c.dtype not in exchange.FIXED_KEYS + (abi.FLOAT64,) for c in cols):
            raise TypeError("the exchange carries fixed-width columns only")
        carry = exchange._agree([c.validity is not None for c in cols], "cpu")
        out = []
        for c, cv in zip(cols, carry):
            valid = c.valid_mask()[order] if cv else None
            out.append((c.dtype, np.ascontiguousarray(c.values[order]), valid))
        return out, counts, fixed

    def exchange(self, cols, counts, world):
        import torch
        sizes = exchange._recv_sizes(counts, world, "cpu")
        got = []
        for dt, vals, valid in cols:
            r = exchange._all_to_all(torch.from_numpy(vals), counts, sizes, "cpu").numpy()
            rv = None
            if valid is not None:
                rv = exchange._all_to_all(torch.from_numpy(valid.astype(np.uint8)), counts, sizes, "cpu").numpy()
            got.append((dt, r, rv))
        return got

    def source(self, got, fixed_fn):
        """Host columns [values..., validity bytes of the nullable ones] for the Final merge."""
        cols = [fixed_fn(dt, v) for dt, v, _ in got]
        cols += [fixed_fn(abi.BOOL, rv) for _, _, rv in got if rv is not None]
        return cols


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _data():
    rng = np.random.Generator(np.random.PCG64(11))
    key = (rng.permutation(DIM) + 1).astype(np.int64)
    fk = rng.integers(1, DIM + 1, ROWS, dtype=np.int64)
    d = rng.integers(0, 2557, ROWS, dtype=np.int32)
    v = rng.uniform(900.0, 105000.0, ROWS)
    x = rng.normal(0.0, 100.0, ROWS)
    x_valid = (rng.random(ROWS) > 0.2) & (d % 97 != 5)  # groups d = 5 (mod 97) see no valid x
    return key, fk, d, v, x, x_valid


def _tables(rank=None, world=1):
    from minilake_b200.abi import FLOAT64, INT32, INT64
    from minilake_b200.columns import Table, fixed
    from minilake_b200.exchange import split_row_groups
    key, fk, d, v, x, xv = _data()
    idx = np.array_split(np.arange(ROWS), GROUPS)
    take = range(GROUPS) if rank is None else split_row_groups(GROUPS, rank, world)
    rgs = [[fixed(INT64, fk[idx[i]]), fixed(INT32, d[idx[i]]), fixed(FLOAT64, v[idx[i]]),
            fixed(FLOAT64, x[idx[i]], xv[idx[i]])] for i in take]
    fact = Table("fact", ["fk", "d", "v", "x"], rgs)
    dim = Table("dim", ["key"], [[fixed(INT64, key)]])
    return dim, fact


def _queries(j):
    from minilake_b200.abi import (AVG, COUNT, COUNT_STAR, FLOAT64, INT32, INT64, MAX, MIN, SUM, AggSpec, Col, Filter,
                                   Lit, Probe)
    join_groupby = ([Filter(Col(1) > Lit(1200)), Probe(j.handle, [(Col(0), INT64)], build_is_left=True)],
                    [(Col(1), INT64)], [AggSpec(SUM, Col(3), FLOAT64), AggSpec(COUNT_STAR)])
    # after the probe: [key, fk, d, v, x]
    nullable = ([Probe(j.handle, [(Col(0), INT64)], build_is_left=True)], [(Col(2), INT32)],
                [AggSpec(SUM, Col(4), FLOAT64), AggSpec(AVG, Col(4), FLOAT64), AggSpec(MIN, Col(4), FLOAT64),
                 AggSpec(MAX, Col(3), FLOAT64), AggSpec(COUNT, Col(4), FLOAT64), AggSpec(COUNT_STAR)])
    return [join_groupby, nullable]


def _final_rows(eng, batch, proj):
    """A final batch as (values, valid) per column, with AVG computed (sum / count, NULL when the
    count is 0) by the oracle's expressions when the plan has a projection."""
    from oracle import orc
    cols = eng.fetch(batch)
    if proj is None:
        return [(c.values, c.valid_mask()) for c in cols]
    return [(c.values, c.valid_mask()) for c in (orc.project(e, t, cols)[0] for e, t in proj)]


def _rank(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from minilake_b200.abi import FLOAT64, INT32, INT64, Col
    from oracle import orc
    eng = orc.OracleEngine(threads=2)
    dim, fact = _tables(rank, world)
    j = eng.join_build(dim, [INT64], [(Col(0), INT64)])
    results = []
    for prologue, group, aggs in _queries(j):
        final, proj = exchange.distributed_hashagg(eng, HostSide(eng), fact,
                                                   [INT64, INT32, FLOAT64, FLOAT64], group, aggs, prologue, world)
        results.append(_final_rows(eng, final, proj))
    # the benchmark query's top 10: each rank's top 10 of the groups it owns, gathered and merged
    keys, sums, counts = results[0][0][0], results[0][1][0], results[0][2][0]
    order = np.lexsort((keys, -sums))[:10]
    mk, ms, mc = exchange.exchange_topn(keys[order], sums[order], counts[order], 10)
    out.put((rank, [[(v.tolist(), m.tolist()) for v, m in r] for r in results], mk.tolist(), ms.tolist(), mc.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_partial_exchange_final_match_single_process():
    from minilake_b200.abi import FLOAT64, INT32, INT64, Col
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
    assert res[0][2:] == res[1][2:], "every rank gets the same merged top-10"
    # the single-process plan over the whole table
    eng = orc.OracleEngine(threads=2)
    dim, fact = _tables()
    j = eng.join_build(dim, [INT64], [(Col(0), INT64)])
    for qi, (prologue, group, aggs) in enumerate(_queries(j)):
        want = eng.fetch(eng.hashagg(fact, [INT64, INT32, FLOAT64, FLOAT64], group, aggs, prologue))
        order = np.argsort(want[0].values, kind="stable")
        got_cols = []
        owners = []
        for r in range(2):
            cols = res[r][1][qi]
            got_cols.append([(np.asarray(v), np.asarray(m, dtype=bool)) for v, m in cols])
            owners.append(np.asarray(cols[0][0]))
        # each group is finalized on exactly one rank: the owner of its key hash
        assert len(np.intersect1d(owners[0], owners[1])) == 0
        for r in range(2):
            if len(owners[r]):
                from minilake_b200.columns import fixed
                h = orc.hash_columns([fixed(group[0][1], owners[r])])
                assert np.all(h % np.uint64(2) == np.uint64(r))
        merged = [(np.concatenate([g[c][0] for g in got_cols]), np.concatenate([g[c][1] for g in got_cols]))
                  for c in range(len(want))]
        morder = np.argsort(merged[0][0], kind="stable")
        assert np.array_equal(merged[0][0][morder], want[0].values[order]), "group keys differ"
        for c in range(1, len(want)):
            gv, gm = merged[c][0][morder], merged[c][1][morder]
            wv, wm = want[c].values[order], want[c].valid_mask()[order]
            assert np.array_equal(gm, wm), f"query {qi} column {c}: NULLs differ"
            if want[c].dtype == FLOAT64:  # sums of signed values (query 1) may cancel: 1e-9 absolute
                np.testing.assert_allclose(gv[wm], wv[wm], rtol=1e-12, atol=1e-9 if qi == 1 else 0.0,
                                           err_msg=f"query {qi} column {c}")
            else:
                assert np.array_equal(gv[wm], wv[wm]), f"query {qi} column {c} differs"
    # the merged top-10 equals the single-process top-10
    from minilake_b200 import workloads
    top = workloads.run_join_groupby(eng, dim, fact)
    assert res[0][2] == top[0].values.tolist()
    assert res[0][4] == top[2].values.tolist()
    np.testing.assert_allclose(res[0][3], top[1].values, rtol=1e-12)
    assert exchange.split_row_groups(12, 1, 2) == list(range(1, 12, 2))
