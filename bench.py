"""Benchmark: the join + high-cardinality GROUP BY + top-10 workload on B200.

Workload (one step = one full query): dimension 1,500,000 rows (key i64), fact
60,000,000 rows (fk i64, d i32, v f64); WHERE d > 1200, JOIN fk = key, GROUP BY fk
with SUM(v) and COUNT(*), ORDER BY SUM(v) DESC, fk LIMIT 10.  Seeded synthetic data.

* value   rows/s of the fact table with the tables already resident in HBM
          (join build + fused filter/probe/aggregate + top-N, per step)
* e2e     the same query through the C ABI with pinned host buffers: the host->device
          copy of both tables and the device->host read of the 10 result rows are inside
          every step (morsels pushed from several host threads, one stream each)
* roofline  the fused pipeline-aggregate kernel: algorithmic bytes (20 B per fact
          row: fk 8 + d 4 + v 8) / its CUDA-event time, vs the measured HBM copy peak
* cpu_baseline  the CPU oracle (a C++ restatement of MiniLake's engine) on this
          host's cores, the full workload

Multi-GPU (torchrun, N ranks): weak scaling; rank r scans its own 60M-row share of the fact
table (fk uniform over every key, as a split by row group gives), the dimension table is
replicated, every rank aggregates its share in Partial mode, the exchange step sends each
partial group to the rank that owns its key hash (one NCCL all-to-all per state column), the
owners merge, and the ranks' top-10 lists are gathered and merged on every rank.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FACT_ROWS = 60_000_000
DIM_ROWS = 1_500_000
ROW_GROUPS = 128
BYTES_PER_ROW = 20  # fk 8 + d 4 + v 8 (the kernel's algorithmic bytes)
METRIC = "rows/s & HBM GB/s per op; learned vs plain sizing on B200; p50/p99 latency"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def make_data(rank: int, world: int, fact_rows: int = FACT_ROWS):
    """Dimension table (replicated) and this rank's share of the fact table, as flat arrays.
    Every rank's fact rows reference keys uniform over all of 1..DIM_ROWS (a split by row
    group, not by key), so the ranks' partial aggregates overlap in nearly every group."""
    rng = np.random.Generator(np.random.PCG64(43))
    key = (rng.permutation(DIM_ROWS) + 1).astype(np.int64)
    frng = np.random.Generator(np.random.PCG64(43 + 1000 * rank))
    fk = frng.integers(1, DIM_ROWS + 1, fact_rows, dtype=np.int64)
    d = frng.integers(0, 2557, fact_rows, dtype=np.int32)
    v = frng.uniform(900.0, 105000.0, fact_rows)
    return key, fk, d, v


class ClockSampler:
    """SM clock and clock-event reasons of this rank's GPU, sampled through NVML every
    2 ms from a thread while the timed region runs (reads only; changes no setting)."""


    def __init__(self, device_index: int):
        self.samples, self.reasons, self.max_mhz = [], set(), 0.0
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            try:
                uuid = str(torch.cuda.get_device_properties(device_index).uuid)
                h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self._reasons_fn = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
            self._bits = {"hw_slowdown": pynvml.nvmlClocksThrottleReasonHwSlowdown,
                          "hw_thermal_slowdown": pynvml.nvmlClocksThrottleReasonHwThermalSlowdown,
                          "sw_thermal_slowdown": pynvml.nvmlClocksThrottleReasonSwThermalSlowdown,
                          "sw_power_cap": pynvml.nvmlClocksThrottleReasonSwPowerCap}
            self._nvml, self._h = pynvml, h
        except Exception:
            self._nvml = None

    def __enter__(self):
        if self._nvml is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def _run(self):
        n, h = self._nvml, self._h
        while not self._stop.is_set():
            try:
                self.samples.append(float(n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM)))
                bits = self._reasons_fn(h)
                for name, bit in self._bits.items():
                    if bits & bit:
                        self.reasons.add(name)
            except Exception:
                return
            time.sleep(0.002)

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread is not None:
            self._thread.join()

    def summary(self):
        if not self.samples:
            return None
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples), "source": "NVML, 2 ms period, during the timed steps"}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# DRAM bytes (read + write) of one launch of the fused aggregate kernel on the full 60M-row
# workload, from one ncu capture of it (`ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum
# --clock-control none -k regex:ml_pipeline_aggregate -s 3 -c 1 python bench.py --steps 3
# --warmup 3 --skip-cpu --skip-ops`; those two metrics take one pass).  A device counter cannot be
# read from inside the timed run, so the figure is carried here and labelled as such.
NCU_DRAM_BYTES_PER_LAUNCH = 1_228_317_184


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


# ---------------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------------
class GpuQuery:
    def __init__(self, ctx, key, fk, d, v):
        from minilake_b200 import abi
        from minilake_b200.columns import fixed
        self.ctx = ctx
        self.abi = abi
        self.dim_cols = [fixed(abi.INT64, key)]
        self.fact_cols = [fixed(abi.INT64, fk), fixed(abi.INT32, d), fixed(abi.FLOAT64, v)]
        self.dim_dev = ctx.upload(self.dim_cols)
        self.fact_dev = ctx.upload(self.fact_cols)

    def run(self, dim_source, fact_sources, threads=1, size_hint=1_500_000):
        """One query; fact_sources: list of morsels (DeviceBatch or host column lists)."""
        from minilake_b200 import workloads
        from minilake_b200.engine import GpuEngine
        eng = GpuEngine(self.ctx, threads=threads)
        j = workloads.join_groupby_build(eng, [dim_source] if not isinstance(dim_source, list) else dim_source)
        prologue, group, aggs = workloads.join_groupby_plan(j.handle)
        agg = eng.hashagg(fact_sources, [self.abi.INT64, self.abi.INT32, self.abi.FLOAT64], group, aggs, prologue,
                          size_hint=size_hint)
        res = eng.topn(agg, workloads.JG_OUT_TYPES, workloads.join_groupby_topn_keys(), 10)
        out = res.fetch()
        j.close()
        return out


    def prepared(self, size_hint=1_500_000):
        """The same query over the HBM-resident tables as a prepared plan (gpu.Query): the first
        run plans through the sink calls, every later run replays the whole plan -- the join
        build, the fused filter + probe + aggregate, the groups' final values, the top 10 -- as
        one CUDA graph launch over the current contents of the tables."""
        from minilake_b200 import gpu, workloads
        q = gpu.Query(self.ctx)
        jt = q.add_build(gpu.JoinBuildSink(self.ctx, [self.abi.INT64], [(self.abi.Col(0), self.abi.INT64)]),
                         self.dim_dev)
        prologue, group, aggs = workloads.join_groupby_plan(jt)
        q.set_aggregate(gpu.HashAggregateSink(self.ctx, [self.abi.INT64, self.abi.INT32, self.abi.FLOAT64], group,
                                              aggs, prologue, size_hint), self.fact_dev)
        q.set_topn(workloads.join_groupby_topn_keys(), 10)
        return q

    def run_distributed(self, world: int, dim_source, fact_sources, threads=1):
        """The query over this rank's share, merged across the ranks (minilake_b200.exchange):
        the merged global top 10 as (fk, sum, count) arrays on every rank."""
        from minilake_b200 import exchange, workloads
        from minilake_b200.engine import GpuEngine
        eng = GpuEngine(self.ctx, threads=threads)
        j = workloads.join_groupby_build(eng, [dim_source] if not isinstance(dim_source, list) else dim_source)
        prologue, group, aggs = workloads.join_groupby_plan(j.handle)
        side = exchange.DeviceSide(eng)
        final, proj = exchange.distributed_hashagg(eng, side, fact_sources,
                                                   [self.abi.INT64, self.abi.INT32, self.abi.FLOAT64], group, aggs,
                                                   prologue, world)
        res = eng.topn(final, workloads.JG_OUT_TYPES, workloads.join_groupby_topn_keys(), 10)
        top = res.fetch()
        out = exchange.exchange_topn(top[0].values, top[1].values, top[2].values, 10, device="cuda")
        j.close()
        return out


def pinned_like(a: np.ndarray):
    import torch
    t = torch.empty(a.shape, dtype={np.int64: torch.int64, np.int32: torch.int32,
                                    np.float64: torch.float64}[a.dtype.type], pin_memory=True)
    arr = t.numpy()
    arr[...] = a
    return arr, t


def gpu_arm(args):
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    from minilake_b200.columns import fixed
    from minilake_b200.gpu import PROFILE, Context
    log(f"[rank {rank}] generating data")
    key, fk, d, v = make_data(rank, world, args.fact_rows)
    rows = args.fact_rows
    ctx = Context(local, flags=PROFILE)
    log(f"[rank {rank}] uploading tables")
    q = GpuQuery(ctx, key, fk, d, v)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def step(dim_source, fact_sources, threads=1):
        """One query: (fk, sum, count) of the top 10; with N ranks, merged across them."""
        if world > 1:
            return q.run_distributed(world, dim_source, fact_sources, threads)
        top = q.run(dim_source, fact_sources, threads)
        return top[0].values, top[1].values, top[2].values

    # ---- value: HBM-resident tables, one launch over the whole fact table -------------
    # One GPU: the prepared plan (one CUDA graph per step after the planning run, which is the
    # first warm-up step).  N GPUs: the operator calls and the exchange of partial aggregates.
    pq = q.prepared() if world == 1 else None

    def resident_step():
        if pq is None:
            return step(q.dim_dev, [q.fact_dev])
        top = pq.run_host()
        return top[0].values, top[1].values, top[2].values

    log(f"[rank {rank}] warm-up")
    for _ in range(args.warmup):
        resident_step()
    ctx.profile("pipeline_aggregate", reset=True)
    l0 = ctx.kernel_launches()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record()
        top = None
        for _ in range(args.steps):
            top = resident_step()
        e1.record()
        barrier()
    ms = e0.elapsed_time(e1)
    clocks = clk.summary()
    launches = ctx.kernel_launches() - l0
    n_agg, agg_ms = ctx.profile("pipeline_aggregate", reset=True)
    query_stats = pq.stats() if pq is not None else None
    # the same steps through the operator calls (one call per sink, host work between kernels)
    op_ms = None
    if world == 1:
        top_op = step(q.dim_dev, [q.fact_dev])
        assert np.array_equal(top_op[0], top[0]), "operator-call and prepared-plan results differ"
        torch.cuda.synchronize()
        o0, o1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        o0.record()
        for _ in range(5):
            step(q.dim_dev, [q.fact_dev])
        o1.record()
        torch.cuda.synchronize()
        op_ms = o0.elapsed_time(o1) / 5
        if n_agg == 0:  # no kernel timing inside the graph: the fused kernel's own launches
            n_agg, agg_ms = ctx.profile("pipeline_aggregate", reset=True)
        pq.close()
    ms_t = torch.tensor([ms], device="cuda")
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(ms_t.item())

    # ---- e2e: pinned host tables; copies inside every step ---------------------------
    log(f"[rank {rank}] device-resident: {ms_max / args.steps:.3f} ms/step; end-to-end next")
    pinned, keep = [], []
    for a in (fk, d, v):
        p, t = pinned_like(a)
        pinned.append(p)
        keep.append(t)
    pkey, tkey = pinned_like(key)
    keep.append(tkey)
    from minilake_b200 import abi
    nmorsel = 16
    bounds = np.linspace(0, rows, nmorsel + 1).astype(np.int64)
    morsels = [[fixed(abi.INT64, pinned[0][bounds[i]:bounds[i + 1]]), fixed(abi.INT32, pinned[1][bounds[i]:bounds[i + 1]]),
                fixed(abi.FLOAT64, pinned[2][bounds[i]:bounds[i + 1]])] for i in range(nmorsel)]
    dim_host = [fixed(abi.INT64, pkey)]
    for _ in range(max(1, args.warmup // 2)):
        step(dim_host, morsels, threads=4)
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(args.steps):
        top_e2e = step(dim_host, morsels, threads=4)
    f1.record()
    barrier()
    e2e_ms = f0.elapsed_time(f1)
    et = torch.tensor([e2e_ms], device="cuda")
    if world > 1:
        torch.distributed.all_reduce(et, op=torch.distributed.ReduceOp.MAX)
    e2e_ms = float(et.item())
    assert np.array_equal(top_e2e[0], top[0]), "e2e and HBM-resident results differ"

    if rank == 0:
        rows_total = rows * world
        value = rows_total / (ms_max / 1e3 / args.steps)
        e2e = rows_total / (e2e_ms / 1e3 / args.steps)
        peak, peak_kind = measured_peak()
        per_launch_ms = agg_ms / max(n_agg, 1)
        achieved = rows * BYTES_PER_ROW / (per_launch_ms / 1e3) / 1e9
        log("CPU baseline")
        cpu = cpu_baseline(key, fk, d, v) if world == 1 and not args.skip_cpu else None
        ops = None
        if world == 1 and not args.skip_ops:
            log("per-operator throughput")
            from minilake_b200 import opbench
            ops = opbench.run(iters=5, log=log)  # {"peak_gbs", "peak_kind", "ops": {...}}
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "rows/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded numpy PCG64 with the workload's shapes and value distributions)",
            "config": {"workload": "join + high-cardinality GROUP BY + top-10: dim 1.5M rows (key i64), "
                                   f"fact {rows / 1e6:g}M rows per GPU (fk i64, d i32, v f64), d > 1200, GROUP BY fk, "
                                   "SUM(v), COUNT(*), ORDER BY SUM(v) DESC, fk LIMIT 10",
                       "fact_rows_per_gpu": rows, "dim_rows": DIM_ROWS,
                       "l2": "inputs larger than L2 (1.2 GB fact table per step)",
                       "parallelism": f"weak, fact split by row group over {world} GPU(s); partial aggregates "
                                      "exchanged by key hash (NCCL all-to-all), merged by their owners"},
            "e2e": {"value": e2e, "unit": "rows/s",
                    "h2d_bytes_per_step": int(rows * BYTES_PER_ROW + DIM_ROWS * 8),
                    "d2h_bytes_per_step": int(10 * 24),
                    "ms_per_step": e2e_ms / args.steps},
            "gpu_launches": int(launches),
            "step": ("prepared plan: after the planning run each step is one CUDA graph launch (join build, "
                     "fused filter + probe + aggregate, final values, top 10, and the 240-byte read-back of the result)"
                     if world == 1 else "operator calls per sink, partial aggregates exchanged by key hash"),
            "prepared_query": query_stats,
            "operator_calls_ms_per_step": op_ms,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "kernel": "ml_pipeline_aggregate (runtime-specialized fused filter + join probe + "
                                   "hash aggregate)",
                         "kernel_ms_per_launch": per_launch_ms,
                         "algorithmic_bytes_per_launch": rows * BYTES_PER_ROW,
                         "traffic": NCU_DRAM_BYTES_PER_LAUNCH if rows == FACT_ROWS else None,
                         "traffic_source": "ncu capture of one full-size launch (dram__bytes_read.sum + "
                                           "dram__bytes_write.sum), carried as a constant"},
            "cpu_baseline": cpu,
            "ops": ops,
            "clocks": clocks,
            "top10_fk": [int(x) for x in top[0]],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    ctx.close()


# ---------------------------------------------------------------------------------------------
# CPU baseline / reference arm: the oracle (C++ restatement of MiniLake's engine)
# ---------------------------------------------------------------------------------------------
def oracle_tables(key, fk, d, v):
    from minilake_b200 import abi
    from minilake_b200.columns import Table, fixed
    dim = Table("dim", ["key"], [[fixed(abi.INT64, c)] for c in np.array_split(key, 4)])
    idx = np.linspace(0, len(fk), ROW_GROUPS + 1).astype(np.int64)
    fact = Table("fact", ["fk", "d", "v"],
                 [[fixed(abi.INT64, fk[idx[i]:idx[i + 1]]), fixed(abi.INT32, d[idx[i]:idx[i + 1]]),
                   fixed(abi.FLOAT64, v[idx[i]:idx[i + 1]])] for i in range(ROW_GROUPS)])
    return dim, fact


def oracle_step(eng, dim, fact):
    from minilake_b200 import workloads
    return workloads.run_join_groupby(eng, dim, fact)


def _time_oracle(dim, fact, threads, runs):
    from oracle import orc
    eng = orc.OracleEngine(threads=threads)
    oracle_step(eng, dim, fact)
    times = []
    for _ in range(runs):
        t0 = time.perf_counter()
        oracle_step(eng, dim, fact)
        times.append(time.perf_counter() - t0)
    return float(np.median(times)), float(min(times)), float(max(times))


def cpu_baseline(key, fk, d, v, runs=3):
    """The oracle on this host: all cores (the line's value) and 8 threads (the configuration's
    `--threads 8`), median of `runs` after one warm-up, like MiniLake's `bench` command."""
    threads = os.cpu_count() or 1
    dim, fact = oracle_tables(key, fk, d, v)
    med, lo, hi = _time_oracle(dim, fact, threads, runs)
    med8, lo8, hi8 = _time_oracle(dim, fact, 8, runs)
    return {"value": len(fk) / med, "unit": "rows/s", "cores": threads, "kind": "port",
            "sample": f"the full workload ({len(fk):,} fact rows), median of {runs} runs after 1 warm-up, "
                      f"pre-decoded in-memory columns, {threads} threads",
            "ms": {"median": med * 1e3, "min": lo * 1e3, "max": hi * 1e3},
            "threads_8": {"value": len(fk) / med8, "unit": "rows/s", "cores": 8,
                          "ms": {"median": med8 * 1e3, "min": lo8 * 1e3, "max": hi8 * 1e3}},
            "cpu_model": cpu_model(), "host_threads": threads}


def reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import orc
    key, fk, d, v = make_data(0, 1)
    dim, fact = oracle_tables(key, fk, d, v)
    threads = os.cpu_count() or 1
    eng = orc.OracleEngine(threads=threads)
    for _ in range(args.warmup):
        oracle_step(eng, dim, fact)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle_step(eng, dim, fact)
    dt = time.perf_counter() - t0
    value = FACT_ROWS / (dt / args.steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded numpy PCG64 with the workload's shapes and value distributions)",
        "config": {"workload": "join + high-cardinality GROUP BY + top-10: dim 1.5M rows (key i64), "
                               "fact 60M rows (fk i64, d i32, v f64), d > 1200, GROUP BY fk, SUM(v), COUNT(*), "
                               "ORDER BY SUM(v) DESC, fk LIMIT 10",
                   "engine": "C++ restatement of MiniLake's CPU engine (the Rust reference cannot be built here)"},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                         "sample": f"the full workload per step ({FACT_ROWS:,} fact rows), {threads} threads",
                         "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-ops", action="store_true", help="leave out the per-operator throughput lines")
    ap.add_argument("--fact-rows", type=int, default=FACT_ROWS,
                    help="fact rows per GPU (smaller cases are for profiling; the benchmark is 60M)")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
