"""Per-operator device throughput: rows/s and HBM GB/s of each hot operator, on tables in HBM.

Each operator runs on seeded synthetic tables generated on the device (the shapes of the
benchmark queries), twice untimed, then `--iters` times with its kernels timed by CUDA events
on the launching stream (the library's profile counters).  GB/s counts ALGORITHMIC bytes: the
bytes an operator must move per row, stated with each operator below; a value near the HBM
copy bandwidth (measured on these GPUs, or the fallback figure; `peak_kind` says which) means
the kernel is at the HBM roofline.

    filter           WHERE d <= 2467 over 100M rows -> selection vector.  Flags pass: 4 B/row read
                     (d) + 1 bit/row written; compaction: 1 bit/row read + 4 B per selected row.
    filter_groupby   WHERE d <= 2467 GROUP BY two dictionary strings, SUM, SUM(x*(1-y)), AVG,
                     COUNT(*) over 100M rows: 36 B/row (d 4, two dict codes 4+4, three f64 24).
    join_groupby     d > 1200, probe of the dense join index on fk (1.5M distinct keys),
                     GROUP BY fk SUM(v) COUNT(*) over 60M rows: 20 B/row (fk 8, d 4, v 8).
    join_build       1.5M distinct i64 keys -> dense join index: 8 B/row read + 4 B/row index.
    star_join        name LIKE 'ab%' on A (150k plain strings) -> probe A on k1 (Zipf 1.1), B on k2,
                     C on region, GROUP BY label SUM(v*(1-w)) over 60M rows: 4 B/row (k1) + 20 B
                     per row that survives the A probe (k2 4, v 8, w 8).
    topn             ORDER BY v DESC LIMIT 10 over 60M f64 values: 8 B/row.
    card_features    HyperLogLog scan of a 60M-row i64 key column: 8 B/row.

    python -m minilake_b200.opbench [--iters 5] [--rows-filter 100000000] [--rows-join 60000000]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os

import numpy as np

from . import abi
from .abi import AggSpec, Col, COUNT_STAR, FLOAT64, INT32, INT64, Lit, SortKey, SUM


def hbm_peak():
    """(GB/s, kind): the measured HBM copy bandwidth of this machine's GPUs ("measured", from
    MEASURED_PEAKS.json), else the earlier measurement on the same kind of B200 ("fallback")."""
    p = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _timed(ctx, keys, fn, iters):
    """Run fn twice untimed, then `iters` times; mean device ms per run of the kernels in `keys`."""
    for _ in range(2):
        fn()
    for k in keys:
        ctx.profile(k, reset=True)
    out = None
    for _ in range(iters):
        out = fn()
    ms = {k: ctx.profile(k, reset=True)[1] / iters for k in keys}
    return ms, out


def _line(rows, ms, nbytes, peak):
    gbs = nbytes / (ms * 1e6) if ms > 0 else 0.0
    return {"rows": int(rows), "ms": round(ms, 4), "rows_per_s": rows / (ms * 1e-3) if ms > 0 else 0.0,
            "algorithmic_bytes": int(nbytes), "gbs": round(gbs, 1), "frac_of_hbm_peak": round(gbs / peak, 3)}


def run(iters: int = 5, rows_filter: int = 100_000_000, rows_join: int = 60_000_000, dim_rows: int = 1_500_000,
        seed: int = 1234, log=print):
    import torch

    from . import serving, workloads
    from .engine import GpuEngine
    from .gpu import LIB, PROFILE, Context, HashAggregateSink, JoinBuildSink, SortSink, _check, card_features

    ctx = Context(0, flags=PROFILE)
    peak, peak_kind = hbm_peak()
    res = {}

    # ---- filter and filter + low-cardinality GROUP BY ------------------------------------
    t0 = serving.gen_fact(0, rows_filter, seed)
    keep = abi.Keep()
    pred = abi.encode_expr(Col(0) <= Lit(2467), abi.BOOL, keep)
    arr, nc, n = t0.ml
    sel = torch.empty(n, dtype=torch.int32, device="cuda")
    k = C.c_int64()

    def filt():
        _check(LIB.ml_gpu_filter(ctx.h, C.byref(pred), arr, nc, n, None, 0, abi.LOC_DEVICE,
                                 C.c_void_p(sel.data_ptr()), C.byref(k)))
        return k.value

    ms, nsel = _timed(ctx, ("select", "select_write"), filt, iters)
    tot = ms["select"] + ms["select_write"]
    res["filter"] = _line(n, tot, 4 * n + n / 8 + n / 8 + 4 * nsel, peak)
    res["filter"]["selected"] = int(nsel)
    res["filter"]["flags_ms"], res["filter"]["compact_ms"] = round(ms["select"], 4), round(ms["select_write"], 4)
    log(f"filter: {res['filter']}")

    prologue, group, aggs = workloads.filter_groupby_plan(2467)

    def fg():
        sink = HashAggregateSink(ctx, t0.types, group, aggs, prologue)
        loc = sink.create_local()
        loc.sink(t0.ml)
        loc.combine()
        out = sink.finalize()
        g = out.num_rows
        out.close()
        sink.close()
        return g

    ms, groups = _timed(ctx, ("pipeline_aggregate",), fg, iters)
    res["filter_groupby"] = _line(n, ms["pipeline_aggregate"], 36 * n, peak)
    res["filter_groupby"]["groups"] = int(groups)
    log(f"filter_groupby: {res['filter_groupby']}")
    del t0, sel
    torch.cuda.empty_cache()

    # ---- join build, join + high-cardinality GROUP BY, top-N, cardinality features ----------
    t1 = serving.gen_fact(1, rows_join, seed + 1, dim_rows=dim_rows)
    dim = serving.DeviceTable([(INT64, torch.arange(1, dim_rows + 1, device="cuda", dtype=torch.int64), None)])

    def build():
        j = JoinBuildSink(ctx, [INT64], [(Col(0), INT64)])
        loc = j.create_local()
        loc.sink(dim.ml)
        loc.combine()
        j.finalize()
        return j

    joins = []
    ms, _ = _timed(ctx, ("join_insert",), lambda: joins.append(build()), iters)
    res["join_build"] = _line(dim_rows, ms["join_insert"], 12 * dim_rows, peak)
    log(f"join_build: {res['join_build']}")
    j = joins[-1]
    for other in joins[:-1]:
        other.close()

    jp, jg, ja = workloads.join_groupby_plan(j.handle, 1200)

    def jgb():
        sink = HashAggregateSink(ctx, t1.types, jg, ja, jp, size_hint=dim_rows)
        loc = sink.create_local()
        loc.sink(t1.ml)
        loc.combine()
        out = sink.finalize()
        g = out.num_rows
        out.close()
        sink.close()
        return g

    ms, groups = _timed(ctx, ("pipeline_aggregate",), jgb, iters)
    res["join_groupby"] = _line(rows_join, ms["pipeline_aggregate"], 20 * rows_join, peak)
    res["join_groupby"]["groups"] = int(groups)
    log(f"join_groupby: {res['join_groupby']}")
    j.close()

    # ---- star join (fact shape 2) ------------------------------------------------------------
    t2 = serving.gen_fact(2, rows_join, seed + 2)
    dim_a, dim_b, dim_c, names, a_key = serving.star_dims(ctx)
    eng = GpuEngine(ctx)
    a, b, c = workloads.star_join_builds(eng, dim_a, dim_b, dim_c)
    sp, sg, sa = workloads.star_join_plan(a, b, c)
    # fact rows whose k1 is the key of a name starting with "ab" (the rows the later stages read)
    match = torch.from_numpy(a_key[[i for i, nm in enumerate(names) if nm.startswith(b"ab")]]).to("cuda")
    survivors = int(torch.isin(t2.keep[0][1], match).sum().item())

    def star():
        sink = HashAggregateSink(ctx, t2.types, sg, sa, sp)
        loc = sink.create_local()
        loc.sink(t2.ml)
        loc.combine()
        out = sink.finalize()
        g = out.num_rows
        out.close()
        sink.close()
        return g

    ms, groups = _timed(ctx, ("pipeline_aggregate",), star, iters)
    res["star_join"] = _line(rows_join, ms["pipeline_aggregate"], 4 * rows_join + 20 * survivors, peak)
    res["star_join"]["groups"], res["star_join"]["rows_after_a_probe"] = int(groups), survivors
    log(f"star_join: {res['star_join']}")
    for j in (a, b, c):
        j.close()
    del t2
    torch.cuda.empty_cache()

    v_only = serving.DeviceTable([(FLOAT64, t1.keep[2][1], None)])

    def topn():
        ts = SortSink(ctx, [FLOAT64], [SortKey(Col(0), FLOAT64, asc=False)], 10)
        loc = ts.create_local()
        loc.sink(v_only.ml)
        loc.combine()
        out = ts.finalize()
        m = out.num_rows
        out.close()
        ts.close()
        return m

    ms, _ = _timed(ctx, ("topn",), topn, iters)
    res["topn"] = _line(rows_join, ms["topn"], 8 * rows_join, peak)
    log(f"topn: {res['topn']}")

    ms, (_, est) = _timed(ctx, ("card_hll",), lambda: card_features(ctx, t1.ml, [(Col(0), INT64)]), iters)
    res["card_features"] = _line(rows_join, ms["card_hll"], 8 * rows_join, peak)
    res["card_features"]["hll_estimate"] = round(float(est))
    log(f"card_features: {res['card_features']}")
    ctx.close()
    return {"peak_gbs": peak, "peak_kind": peak_kind, "ops": res}


def parquet_column_chunk(column: str = "price", rows: int = 250_000, row_groups: int = 2, iters: int = 4,
                         log=print) -> dict:
    """One column chunk decoded alone: row group 0's chunk of `column` from configuration 0's table
    as a seeded Snappy Parquet file (rows / row_groups rows per row group), `iters` calls of
    ml_gpu_parquet_decode one after another; wall-clock milliseconds per call (the first call
    includes the context's first use of each kernel)."""
    import tempfile

    import pyarrow.parquet as pq

    from . import datagen, gpu, parquet
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "cfg0.parquet")
        datagen.filter_groupby_parquet(path, rows=rows, row_groups=row_groups)
        pf = pq.ParquetFile(path)
        names = [pf.schema.column(i).name for i in range(len(pf.schema))]
        md = pf.metadata.row_group(0)
        ci = names.index(column)
        sch, meta = pf.schema.column(ci), md.column(ci)
        conv, scale = parquet.conversion(sch)
        data = parquet.chunk_bytes(path, meta)
        args = (data, parquet.PHYSICAL[sch.physical_type], sch.length or 0, conv, scale,
                parquet.CODECS[meta.compression], md.num_rows, sch.max_definition_level)
    ctx = gpu.Context(0)
    times = []
    for _ in range(iters):
        times.append(_wall(lambda: gpu.parquet_decode(ctx, *args).close()))
    ctx.close()
    out = {"column": column, "rows": md.num_rows, "chunk_bytes": len(data), "ms": [round(t * 1e3, 2) for t in times]}
    log(f"parquet_column_chunk: {out}")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", type=int, default=5)
    ap.add_argument("--rows-filter", type=int, default=100_000_000)
    ap.add_argument("--rows-join", type=int, default=60_000_000)
    ap.add_argument("--parquet", action="store_true", help="only the Parquet decode comparison")
    ap.add_argument("--parquet-threads", type=int, default=16, help="host threads calling the decoder at once")
    ap.add_argument("--parquet-column", help="only one column chunk of a small file, decoded alone (e.g. price)")
    a = ap.parse_args()
    if a.parquet_column:
        print(json.dumps(parquet_column_chunk(a.parquet_column)), flush=True)
        return
    if a.parquet:
        import sys
        # one hardware work queue per calling thread (up to 32): calls on different streams do not
        # wait behind each other's long Snappy kernels (read when the CUDA context is created)
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", str(min(max(a.parquet_threads, 8), 32)))
        lg = lambda *m: print(*m, file=sys.stderr, flush=True)  # noqa: E731
        print(json.dumps([parquet_decode(log=lg, compression=c, threads=a.parquet_threads) for c in ("snappy", "none")]),
              flush=True)
        return
    import sys
    out = run(a.iters, a.rows_filter, a.rows_join, log=lambda *m: print(*m, file=sys.stderr, flush=True))
    print(json.dumps(out), flush=True)



def parquet_decode(rows: int = 20_000_000, row_groups: int = 160, threads: int = 16, iters: int = 3, log=print,
                   compression: str = "snappy"):
    """Configuration 0's table as a seeded Snappy Parquet file (rows / row_groups rows per row
    group), its six scanned columns decoded on the GPU (ml_gpu_parquet_decode per column chunk,
    `threads` host threads calling it at once, each call on its own stream) against pyarrow's
    multi-threaded CPU decode of the same columns.  Wall-clock time from file bytes in host
    memory to decoded columns (GPU: in HBM), best of `iters`; the file is read once beforehand."""
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    import pyarrow.parquet as pq

    from . import datagen, gpu, parquet, workloads
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "cfg0.parquet")
        datagen.filter_groupby_parquet(path, rows=rows, row_groups=row_groups, compression=compression)
        pf = pq.ParquetFile(path)
        names = [pf.schema.column(i).name for i in range(len(pf.schema))]
        cols = [names.index(c) for c in workloads.FG_SCAN]
        jobs, compressed = [], 0
        for rg in range(pf.metadata.num_row_groups):
            md = pf.metadata.row_group(rg)
            for ci in cols:
                meta, sch = md.column(ci), pf.schema.column(ci)
                conv, scale = parquet.conversion(sch)
                data = parquet.chunk_bytes(path, meta)
                compressed += len(data)
                jobs.append((data, parquet.PHYSICAL[sch.physical_type], sch.length or 0, conv, scale,
                             parquet.CODECS[meta.compression], md.num_rows, sch.max_definition_level))
        ctx = gpu.Context(0)

        def one(j):
            gpu.parquet_decode(ctx, *j).close()

        def gpu_run():
            with ThreadPoolExecutor(threads) as ex:
                list(ex.map(one, jobs))
        gpu_run()
        best_gpu = min(_wall(gpu_run) for _ in range(iters))
        cpu_threads = os.cpu_count() or 1
        pq.read_table(path, columns=workloads.FG_SCAN, use_threads=True)
        best_cpu = min(_wall(lambda: pq.read_table(path, columns=workloads.FG_SCAN, use_threads=True))
                       for _ in range(iters))
        ctx.close()
    out = {"compression": compression, "rows": rows, "row_groups": row_groups, "column_chunks": len(jobs),
           "compressed_bytes": compressed,
           "gpu_ms": round(best_gpu * 1e3, 2), "gpu_rows_per_s": rows / best_gpu,
           "gpu_compressed_gbs": round(compressed / best_gpu / 1e9, 3), "gpu_host_threads": threads,
           "cpu_pyarrow_ms": round(best_cpu * 1e3, 2), "cpu_rows_per_s": rows / best_cpu, "cpu_threads": cpu_threads}
    log(f"parquet_decode: {out}")
    return out


def _wall(fn):
    import time
    t0 = time.perf_counter()
    fn()
    return time.perf_counter() - t0


if __name__ == "__main__":
    main()
