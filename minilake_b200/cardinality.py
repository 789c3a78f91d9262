"""Learned sizing of GROUP BY hash tables: the cardinality-estimator sweep.

Seeded synthetic GROUP BY instances (rows log-uniform in [min_rows, max_rows], distinct keys
log-uniform in [1, 2^26] capped at the rows, keys int32 / int64 / two int32 columns, uniform,
sequential or Zipf(s in [0.5, 1.5]) key frequencies, NULL fraction uniform in [0, 0.1]) are
generated directly in HBM.  For each the library computes the scan features
(`ml_gpu_card_features`: HyperLogLog register histogram and scan statistics) and the plain
engine computes the true number of groups.  The MLP is trained on the first instances and
tested on the rest, where each query runs four ways: with the plain resize-on-overflow table
(no size hint), presized from MiniLake's planner estimate (a tenth of the input rows), presized
from the HyperLogLog estimate, and presized from the MLP's prediction; the last two are timed
with the features scan (and the MLP's inference) they need.  All four must give identical
results.  The size hint also decides shared-memory pre-aggregation (a table of at most 65,536
groups is pre-aggregated per CTA in shared memory, a larger one is updated in L2).

Zipf keys are drawn by inverse-CDF sampling of the bounded continuous power law on [1, D+1)
(rank = floor(x) - 1), the usual stand-in for a finite Zipf law.

    python -m minilake_b200.cardinality --instances 2000 --train 1500
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time
from dataclasses import dataclass

import numpy as np

from . import abi
from .abi import AggSpec, Col, COUNT_STAR, INT32, INT64

KEY_TYPES = ("int32", "int64", "int32x2")
DISTS = ("uniform", "sequential", "zipf")


@dataclass
class Instance:
    rows: int
    distinct: int   # key values drawn from (before NULLs)
    key_type: str
    dist: str
    s: float        # Zipf exponent
    null_frac: float
    seed: int


def make_instances(n: int, seed: int = 45, min_rows: int = 1_000_000, max_rows: int = 100_000_000,
                   max_distinct: int = 1 << 26):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        rows = int(round(math.exp(rng.uniform(math.log(min_rows), math.log(max_rows)))))
        distinct = int(round(math.exp(rng.uniform(0.0, math.log(max_distinct)))))
        out.append(Instance(rows=rows, distinct=max(1, min(distinct, rows)), key_type=KEY_TYPES[rng.integers(3)],
                            dist=DISTS[rng.integers(3)], s=float(rng.uniform(0.5, 1.5)),
                            null_frac=float(rng.uniform(0.0, 0.1)), seed=int(rng.integers(1 << 62))))
    return out


def _pack_validity(valid):
    """bool tensor -> u64 words, LSB first (int64 storage)."""
    import torch
    n = valid.numel()
    pad = (-n) % 64
    v = torch.nn.functional.pad(valid.to(torch.int64), (0, pad)).view(-1, 64)
    weights = torch.ones(64, dtype=torch.int64, device=valid.device) << torch.arange(64, device=valid.device)
    return (v * weights).sum(dim=1)


class DeviceInstance:
    """The key columns of one instance in HBM (torch owns the memory)."""

    def __init__(self, inst: Instance, device="cuda"):
        import torch
        g = torch.Generator(device=device)
        g.manual_seed(inst.seed)
        n, d = inst.rows, inst.distinct
        if inst.dist == "uniform":
            ids = torch.randint(0, d, (n,), device=device, generator=g, dtype=torch.int64)
        elif inst.dist == "sequential":
            ids = torch.arange(n, device=device, dtype=torch.int64) % d
        else:
            u = torch.rand(n, device=device, generator=g, dtype=torch.float64)
            if abs(inst.s - 1.0) < 1e-9:
                x = torch.pow(float(d + 1), u)
            else:
                a = 1.0 - inst.s
                x = torch.pow(1.0 + u * ((d + 1.0) ** a - 1.0), 1.0 / a)
            ids = torch.clamp(torch.floor(x).to(torch.int64) - 1, 0, d - 1)
        valid = torch.rand(n, device=device, generator=g) >= inst.null_frac
        if inst.key_type == "int32":
            self.cols = [ids.to(torch.int32)]
            self.types = [INT32]
        elif inst.key_type == "int64":
            self.cols = [ids * 0x9E3779B1 + 12345]
            self.types = [INT64]
        else:
            self.cols = [(ids % 4096).to(torch.int32), (ids // 4096).to(torch.int32)]
            self.types = [INT32, INT32]
        self.validity = _pack_validity(valid)
        self.rows = n
        self.ids, self.valid = ids, valid
        arr = (abi.MlColumn * len(self.cols))()
        for i, (c, t) in enumerate(zip(self.cols, self.types)):
            arr[i].dtype, arr[i].encoding, arr[i].location, arr[i].len = t, abi.ENC_PLAIN, abi.LOC_DEVICE, n
            arr[i].data = C.c_void_p(c.data_ptr())
            arr[i].validity = C.c_void_p(self.validity.data_ptr())
        self.ml = (arr, len(self.cols), n)
        self.keys = [(Col(i), t) for i, t in enumerate(self.types)]

    def unique_groups(self) -> int:
        """Distinct non-NULL keys + 1 if any key is NULL (GROUP BY semantics), counted with
        torch.unique: a cross-check of the engine's count in tests."""
        import torch
        nn = self.ids[self.valid]
        distinct = int(torch.unique(nn).numel()) if nn.numel() else 0
        return distinct + (1 if bool((~self.valid).any()) else 0)


def aggregate(ctx, di: DeviceInstance, size_hint: int, fetch: bool = True):
    """GROUP BY the key with COUNT(*): (sink + finalize ms, groups, resizes, result checksum)."""
    from .gpu import HashAggregateSink
    ctx.synchronize()
    t0 = time.perf_counter()
    sink = HashAggregateSink(ctx, di.types, di.keys, [AggSpec(COUNT_STAR)], size_hint=size_hint)
    loc = sink.create_local()
    loc.sink(di.ml)
    loc.combine()
    out = sink.finalize()
    ctx.synchronize()
    ms = (time.perf_counter() - t0) * 1e3
    st = sink.stats()
    digest = _checksum(out.fetch()) if fetch else None
    sink.close()
    out.close()
    return ms, st["groups"], st["resizes"], digest


def _checksum(cols):
    """Order-independent digest of (key..., count) rows; NULL keys digest as a sentinel."""
    k1, k2 = np.uint64(0x9E3779B97F4A7C15), np.uint64(0xBF58476D1CE4E5B9)
    h = np.zeros(len(cols[-1].values), dtype=np.uint64)
    for c in cols[:-1]:
        v = c.values.astype(np.int64).view(np.uint64)
        v = np.where(c.valid_mask(), v, np.uint64(0xFFFF_FFFF_FFFF_FFF1))
        h = (h ^ v) * k1
    h ^= cols[-1].values.astype(np.uint64) * k2
    with np.errstate(over="ignore"):
        return int(h.sum(dtype=np.uint64)), int(cols[-1].values.sum())


def q_error(pred, true):
    pred, true = np.maximum(pred, 1.0), np.maximum(true, 1.0)
    return np.maximum(pred / true, true / pred)


def train_model(ctx, instances: int = 200, seed: int = 45, min_rows: int = 1_000_000, max_rows: int = 20_000_000,
                epochs: int = 200):
    """A cardinality model trained on a fresh sweep of `instances` (all used for training)."""
    from .gpu import CardinalityModel, card_features
    feats = np.zeros((instances, 72), dtype=np.float32)
    truth = np.zeros(instances)
    for i, inst in enumerate(make_instances(instances, seed, min_rows, max_rows)):
        di = DeviceInstance(inst)
        feats[i], est = card_features(ctx, di.ml, di.keys)
        truth[i] = aggregate(ctx, di, int(est * 1.5) + 16, fetch=False)[1]
        del di
    model = CardinalityModel(ctx, seed=seed)
    model.train(feats, np.log2(truth).astype(np.float32), epochs=epochs, batch=64, lr=1e-3, seed=seed)
    return model


def run(instances: int = 2000, train: int = 1500, seed: int = 45, min_rows: int = 1_000_000,
        max_rows: int = 100_000_000, epochs: int = 400, log=print):
    from .gpu import CardinalityModel, Context, card_features
    ctx = Context(0)
    insts = make_instances(instances, seed, min_rows, max_rows)
    feats = np.zeros((instances, 72), dtype=np.float32)
    hll = np.zeros(instances)
    truth = np.zeros(instances)
    t0 = time.perf_counter()
    for i, inst in enumerate(insts):
        di = DeviceInstance(inst)
        feats[i], hll[i] = card_features(ctx, di.ml, di.keys)
        truth[i] = aggregate(ctx, di, int(hll[i] * 1.5) + 16, fetch=False)[1]  # the plain engine's count
        del di
        if i % 200 == 199:
            log(f"features {i + 1}/{instances} ({time.perf_counter() - t0:.1f} s)")
    y = np.log2(truth).astype(np.float32)
    model = CardinalityModel(ctx, seed=seed)
    t1 = time.perf_counter()
    loss = model.train(feats[:train], y[:train], epochs=epochs, batch=64, lr=1e-3, seed=seed)
    train_s = time.perf_counter() - t1
    pred = np.exp2(model.predict(feats[train:]).astype(np.float64))
    q_mlp = q_error(pred, truth[train:])
    q_hll = q_error(hll[train:], truth[train:])
    # compile every kernel shape the timed runs use (key type x table size x resume) first
    for kt in KEY_TYPES:
        for d in (100, 200_000):
            di = DeviceInstance(Instance(rows=300_000, distinct=d, key_type=kt, dist="uniform", s=1.0,
                                         null_frac=0.05, seed=1))
            aggregate(ctx, di, 0, fetch=False)
            aggregate(ctx, di, 2 * d, fetch=False)
            del di
    # Four arms per test instance, each timed with everything it needs before the GROUP BY:
    #   plain    no size hint: the table starts small and grows on overflow (swiss.rs:219-232);
    #   planner  MiniLake's own estimate, a tenth of the input rows (physical_planner.rs:251-295);
    #   hll      the features scan, then the HyperLogLog estimate x 1.25;
    #   learned  the features scan and the MLP's inference, then its prediction x 1.25.
    arms = ("plain", "planner", "hll", "learned")
    ms = {a: [] for a in arms}
    resizes = {a: [] for a in arms}
    feat_ms, infer_ms, identical = [], [], True
    for j, inst in enumerate(insts[train:]):
        di = DeviceInstance(inst)
        res = {"plain": aggregate(ctx, di, 0), "planner": aggregate(ctx, di, max(inst.rows // 10, 1))}
        ctx.synchronize()
        t0 = time.perf_counter()
        _, est = card_features(ctx, di.ml, di.keys)
        t_feat = (time.perf_counter() - t0) * 1e3
        res["hll"] = aggregate(ctx, di, int(est * 1.25) + 16)
        ctx.synchronize()
        t0 = time.perf_counter()
        f, _ = card_features(ctx, di.ml, di.keys)
        t1 = time.perf_counter()
        p1 = float(np.exp2(model.predict(f[None, :])[0]))
        t2 = time.perf_counter()
        res["learned"] = aggregate(ctx, di, int(p1 * 1.25) + 16)
        feat_ms.append((t1 - t0) * 1e3)
        infer_ms.append((t2 - t1) * 1e3)
        extra = {"plain": 0.0, "planner": 0.0, "hll": t_feat, "learned": (t2 - t0) * 1e3}
        for a in arms:
            ms[a].append(res[a][0] + extra[a])
            resizes[a].append(res[a][2])
            identical &= res[a][1] == truth[train + j] and res[a][3] == res["plain"][3]
        del di
    model.close()
    ctx.close()
    pct = lambda a, p: float(np.percentile(a, p))
    tot = {a: float(np.sum(ms[a])) for a in arms}
    return {
        "instances": instances, "train": train, "test": instances - train, "seed": seed,
        "rows": [min_rows, max_rows], "train_seconds": train_s, "final_train_loss": loss,
        "q_error_mlp": {"median": pct(q_mlp, 50), "p90": pct(q_mlp, 90), "p99": pct(q_mlp, 99), "max": float(q_mlp.max())},
        "q_error_hll": {"median": pct(q_hll, 50), "p90": pct(q_hll, 90), "p99": pct(q_hll, 99), "max": float(q_hll.max())},
        "total_ms": tot,
        "median_ms": {a: float(np.median(ms[a])) for a in arms},
        "resizes_mean": {a: float(np.mean(resizes[a])) for a in arms},
        "features_ms_total": float(np.sum(feat_ms)), "inference_ms_total": float(np.sum(infer_ms)),
        "learned_vs_plain": tot["plain"] / max(tot["learned"], 1e-9),
        "learned_vs_hll": tot["hll"] / max(tot["learned"], 1e-9),
        "learned_vs_planner": tot["planner"] / max(tot["learned"], 1e-9),
        "identical_results": bool(identical),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=2000)
    ap.add_argument("--train", type=int, default=1500)
    ap.add_argument("--min-rows", type=int, default=1_000_000)
    ap.add_argument("--max-rows", type=int, default=100_000_000)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--seed", type=int, default=45)
    a = ap.parse_args()
    import sys
    res = run(a.instances, a.train, a.seed, a.min_rows, a.max_rows, a.epochs,
              log=lambda *m: print(*m, file=sys.stderr, flush=True))
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
