"""Multi-GPU form of the join + GROUP BY + top-N query (one process per GPU).

The fact table is partitioned on the join key: rank r holds the fact rows whose key k satisfies
k % world == r (the dimension table is replicated).  Every group then lives on exactly one rank,
each rank aggregates its own groups with no data-path collective, and the only exchange is the
final one: the ranks' local top-N lists are gathered and merged (the global top N of disjoint
groups is inside the union of the local top Ns), as MiniLake's distributed mode merges partial
results on its coordinator (minilake-dist/src/split.rs:54-127).
"""
from __future__ import annotations

import numpy as np


def shard_keys(rank: int, world: int, dim_rows: int):
    """(first, count): rank `rank` owns the keys first, first + world, ... (count of them) of
    1..dim_rows, i.e. those with k % world == rank."""
    first = rank if rank > 0 else world
    count = (dim_rows - first) // world + 1 if first <= dim_rows else 0
    return first, count


def merge_topn(keys, sums, counts, limit: int):
    """Top `limit` rows by SUM DESC, key ASC of the concatenated candidates."""
    order = np.lexsort((keys, -sums))[:limit]
    return keys[order], sums[order], counts[order]


def exchange_topn(keys, sums, counts, limit: int, device="cpu"):
    """Gather every rank's local top-N (key i64, sum f64, count i64; at most `limit` rows) and
    return the merged global top N on every rank.  Collective: every rank calls it once."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size()
    n = len(keys)
    k = torch.full((limit,), np.iinfo(np.int64).max, dtype=torch.int64)
    s = torch.full((limit,), -np.inf, dtype=torch.float64)
    c = torch.zeros(limit, dtype=torch.int64)
    k[:n], s[:n], c[:n] = torch.as_tensor(keys), torch.as_tensor(sums), torch.as_tensor(counts)
    m = torch.tensor([n], dtype=torch.int64)
    parts = []
    for t in (m, k, s, c):
        t = t.to(device)
        out = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(out, t)
        parts.append([o.cpu().numpy() for o in out])
    ns, ks, ss, cs = parts
    keys_all = np.concatenate([ks[r][:ns[r][0]] for r in range(world)])
    sums_all = np.concatenate([ss[r][:ns[r][0]] for r in range(world)])
    counts_all = np.concatenate([cs[r][:ns[r][0]] for r in range(world)])
    return merge_topn(keys_all, sums_all, counts_all, limit)
