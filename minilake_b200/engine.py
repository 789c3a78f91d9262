"""Drives sinks the way MiniLake's executor does (pipeline.rs:109-136,
scheduler.rs:102-144): worker threads take morsels from a shared counter, each
with its own local sink (here: its own CUDA stream), then combine once.

Sources are a host ``Table`` (each row group is copied to HBM inside the sink
call), a list of ``DeviceBatch`` (HBM-resident row groups), or a single
``DeviceBatch`` (e.g. the output of an earlier sink: a BatchBuffer replay).
"""
from __future__ import annotations

import threading
from typing import List, Sequence

from . import abi
from .columns import HostColumn, Table
from .gpu import Context, DeviceBatch, HashAggregateSink, JoinBuildSink, SortSink


class GpuEngine:
    name = "gpu"

    def __init__(self, ctx: Context, threads: int = 1):
        self.ctx, self.threads = ctx, max(1, threads)

    def _morsels(self, source) -> list:
        if isinstance(source, Table):
            return list(source.row_groups)
        if isinstance(source, DeviceBatch):
            return [source]
        if isinstance(source, (list, tuple)):
            if source and isinstance(source[0], HostColumn):
                return [list(source)]
            return list(source)
        raise TypeError(source)

    def drive(self, sink, source):
        morsels = self._morsels(source)
        nthreads = min(self.threads, max(1, len(morsels)))
        if nthreads == 1:
            local = sink.create_local()
            for m in morsels:
                local.sink(m)
            local.combine()
            return
        lock = threading.Lock()
        nxt = [0]
        errors: List[BaseException] = []

        def worker():
            try:
                local = sink.create_local()
                while True:
                    with lock:
                        i = nxt[0]
                        nxt[0] += 1
                    if i >= len(morsels) or errors:
                        break
                    local.sink(morsels[i])
                local.combine()
            except BaseException as e:  # first error wins, the others stop early
                errors.append(e)

        ts = [threading.Thread(target=worker) for _ in range(nthreads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        if errors:
            raise errors[0]

    def join_build(self, source, input_types, key_exprs, prologue=()):
        sink = JoinBuildSink(self.ctx, input_types, key_exprs, prologue)
        try:
            self.drive(sink, source)
            sink.finalize()
        except BaseException:
            sink.close()  # a failed operator releases everything it reserved
            raise
        return sink

    def hashagg(self, source, input_types, group_exprs, aggs, prologue=(), size_hint=0):
        sink = HashAggregateSink(self.ctx, input_types, group_exprs, aggs, prologue, size_hint)
        try:
            self.drive(sink, source)
            out = sink.finalize()
            out.sink_stats = sink.stats()
        finally:
            sink.close()
        return out

    def topn(self, source, input_types, keys, limit, prologue=()):
        sink = SortSink(self.ctx, input_types, keys, limit, prologue)
        try:
            self.drive(sink, source)
            out = sink.finalize()
        finally:
            sink.close()
        return out

    @staticmethod
    def fetch(batch) -> List[HostColumn]:
        return batch.fetch()

    @staticmethod
    def num_rows(batch) -> int:
        return batch.num_rows
