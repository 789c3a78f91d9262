"""Device-resident selection vectors are checked by the kernels: a selected row id at or past
the batch's rows (operators/filter.rs:19-25 and join.rs:263-315 take a SelectionVector whose
ids index the batch) is skipped on the device and the call fails with ML_ERR_INVALID instead of
reading past the columns; the context stays usable and the next call's result is exact.  Host
selections were already checked on the host.  Both kernel forms run (the `ctx` fixture)."""
import ctypes as C

import numpy as np
import pytest

from minilake_b200 import abi
from minilake_b200.abi import INT64, Col, Lit
from minilake_b200.columns import fixed
from test_gpu_parity import ctx  # noqa: F401  (fixture: specialized and interpreter kernels)

pytestmark = pytest.mark.gpu

N = 50_000


def _setup(ctx):
    import torch
    rng = np.random.default_rng(3)
    x = rng.integers(-1000, 1000, N).astype(np.int64)
    batch = ctx.upload([fixed(INT64, x)])
    good = np.sort(rng.choice(N, 4000, replace=False)).astype(np.uint32)
    bad = good.copy()
    bad[1234] = N + 17  # one id past the batch
    dev = lambda a: torch.from_numpy(a.view(np.int32).copy()).cuda()  # noqa: E731
    return x, batch, good, dev(good), dev(bad)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_filter_with_a_bad_device_selection(ctx):
    import torch
    from minilake_b200.gpu import LIB, MiniLakeError, _check
    x, batch, good, dgood, dbad = _setup(ctx)
    arr, nc = batch.ml_columns()
    keep = abi.Keep()
    e = abi.encode_expr(Col(0) > Lit(0), abi.BOOL, keep)
    out = torch.zeros(len(good), dtype=torch.int32, device="cuda")
    k = C.c_int64()
    for static in (False, True):
        call = (lambda s: LIB.ml_gpu_filter_static(ctx.h, C.byref(e), arr, nc, N, _ptr(s), len(good), _ptr(out),
                                                   C.byref(k))) if static else \
               (lambda s: LIB.ml_gpu_filter(ctx.h, C.byref(e), arr, nc, N, _ptr(s), len(good), abi.LOC_DEVICE,
                                            _ptr(out), C.byref(k)))
        with pytest.raises(MiniLakeError, match="past the batch") as ei:
            _check(call(dbad))
        assert ei.value.code == abi.ERR_INVALID
        _check(call(dgood))
        want = good[x[good] > 0]
        assert np.array_equal(out[:k.value].cpu().numpy().view(np.uint32), want)


def test_hash_columns_with_a_bad_device_selection(ctx):
    import torch
    from minilake_b200.gpu import LIB, MiniLakeError, _check
    x, batch, good, dgood, dbad = _setup(ctx)
    arr, nc = batch.ml_columns()
    out = torch.zeros(len(good), dtype=torch.int64, device="cuda")
    with pytest.raises(MiniLakeError, match="past the batch"):
        _check(LIB.ml_gpu_hash_columns(ctx.h, arr, nc, N, _ptr(dbad), len(good), abi.LOC_DEVICE, _ptr(out)))
    _check(LIB.ml_gpu_hash_columns(ctx.h, arr, nc, N, _ptr(dgood), len(good), abi.LOC_DEVICE, _ptr(out)))
    host = np.zeros(len(good), dtype=np.uint64)
    _check(LIB.ml_gpu_hash_columns(ctx.h, arr, nc, N, good.ctypes.data, len(good), abi.LOC_HOST, host.ctypes.data))
    assert np.array_equal(out.cpu().numpy().view(np.uint64), host)


def test_join_probe_with_a_bad_device_selection(ctx):
    import torch
    from minilake_b200.gpu import LIB, JoinBuildSink, MiniLakeError, _check
    x, batch, good, dgood, dbad = _setup(ctx)
    arr, nc = batch.ml_columns()
    j = JoinBuildSink(ctx, [INT64], [(Col(0), INT64)])
    loc = j.create_local()
    loc.sink([fixed(INT64, np.arange(0, 1000, 3, dtype=np.int64))])
    loc.combine()
    j.finalize()
    keep = abi.Keep()
    kx, nk = abi.encode_exprs([(Col(0), INT64)], keep)
    cap = len(good)
    pi = torch.zeros(cap, dtype=torch.int32, device="cuda")
    bi = torch.zeros(cap, dtype=torch.int32, device="cuda")
    npairs = C.c_int64()
    with pytest.raises(MiniLakeError, match="past the batch"):
        _check(LIB.ml_gpu_join_probe(ctx.h, j.table, kx, nk, arr, nc, N, _ptr(dbad), len(good), abi.LOC_DEVICE,
                                     _ptr(pi), _ptr(bi), cap, C.byref(npairs)))
    _check(LIB.ml_gpu_join_probe(ctx.h, j.table, kx, nk, arr, nc, N, _ptr(dgood), len(good), abi.LOC_DEVICE,
                                 _ptr(pi), _ptr(bi), cap, C.byref(npairs)))
    m = npairs.value
    got = pi[:m].cpu().numpy().view(np.uint32)  # probe rows are the batch's row ids
    want = good[(x[good] >= 0) & (x[good] < 1000) & (x[good] % 3 == 0)]
    assert np.array_equal(np.sort(got), np.sort(want))
    j.close()
