"""ml_gpu_filter_static — the filter whose temporaries live in a static device array —
against ml_gpu_filter on the same device-resident inputs, through the C ABI.  Selections
are index work: they must be identical."""
import ctypes as C

import numpy as np
import pytest

from minilake_b200 import abi
from minilake_b200.abi import FLOAT64, INT32, IsNull, Like, Col, Lit
from minilake_b200.columns import encode_strings, fixed, utf8_dict, utf8_plain

pytestmark = pytest.mark.gpu

WORDS = [b"apple", b"abricot", b"banana", b"ab", b"", b"zeta"]


def _device_u32(n):
    import torch
    return torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")


def _filter(lib, ctx, pred, cols, nc, nrows, sel, nsel, out, static):
    keep = abi.Keep()
    e = abi.encode_expr(pred, abi.BOOL, keep)
    k = C.c_int64()
    sp = C.c_void_p(sel.data_ptr()) if sel is not None else None
    if static:
        st = lib.ml_gpu_filter_static(ctx.h, C.byref(e), cols, nc, nrows, sp, nsel, C.c_void_p(out.data_ptr()),
                                      C.byref(k))
    else:
        st = lib.ml_gpu_filter(ctx.h, C.byref(e), cols, nc, nrows, sp, nsel, abi.LOC_DEVICE,
                               C.c_void_p(out.data_ptr()), C.byref(k))
    return st, k.value


def test_static_filter_matches_filter_on_two_calls_in_a_row():
    import torch
    from minilake_b200.gpu import LIB, Context
    ctx = Context(0)
    rng = np.random.default_rng(31)
    n = 250_000
    valid = rng.random(n) > 0.1
    batch = ctx.upload([fixed(INT32, rng.integers(-100, 100, n, dtype=np.int32), valid),
                        fixed(FLOAT64, rng.random(n)),
                        encode_strings(WORDS, rng.integers(0, len(WORDS), n), rng.random(n) > 0.05),
                        utf8_plain([WORDS[i] for i in rng.integers(0, len(WORDS), n)])])
    cols, nc = batch.ml_columns()
    sel = torch.from_numpy(np.sort(rng.choice(n, n // 3, replace=False)).astype(np.int32)).cuda()
    calls = [((Col(0) > Lit(10)) & Like(Col(2), "ab%"), None, 0),
             ((Col(1) < Lit(0.25)) | IsNull(Col(0)) | Like(Col(3), "%an%"), sel, len(sel))]
    free_after = []
    for pred, s, ns in calls:
        ref, got = _device_u32(n), _device_u32(n)
        st, k_ref = _filter(LIB, ctx, pred, cols, nc, n, s, ns, ref, static=False)
        assert st == 0
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info()[0]
        st, k = _filter(LIB, ctx, pred, cols, nc, n, s, ns, got, static=True)
        assert st == 0, LIB.ml_gpu_last_error()
        free_after.append((before, torch.cuda.mem_get_info()[0]))
        assert k == k_ref and k > 0
        assert torch.equal(got[:k], ref[:k])
    # the second call finds its scratch in place: the device's free memory does not move
    assert free_after[1][0] == free_after[1][1]
    batch.close()
    ctx.close()


def test_static_filter_rejects_calls_over_its_limit():
    import torch
    from minilake_b200.gpu import LIB, Context
    ctx = Context(0)
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    rows = (1 << 24) + 1
    col = (abi.MlColumn * 1)()
    col[0].dtype, col[0].encoding, col[0].location, col[0].len = INT32, abi.ENC_PLAIN, abi.LOC_DEVICE, rows
    col[0].data = C.c_void_p(dummy.data_ptr())
    keep = abi.Keep()
    e = abi.encode_expr(Col(0) > Lit(0), abi.BOOL, keep)
    k = C.c_int64()
    st = LIB.ml_gpu_filter_static(ctx.h, C.byref(e), col, 1, rows, None, 0, C.c_void_p(dummy.data_ptr()), C.byref(k))
    assert st == abi.ERR_INVALID
    assert b"16777216 rows" in LIB.ml_gpu_last_error()
    ctx.close()


def _rows_batch(ctx, n, seed):
    rng = np.random.default_rng(seed)
    return ctx.upload([fixed(INT32, rng.integers(-100, 100, n, dtype=np.int32)), fixed(FLOAT64, rng.random(n)),
                       encode_strings(WORDS, rng.integers(0, len(WORDS), n)),
                       utf8_plain([WORDS[i] for i in rng.integers(0, len(WORDS), n)])])


def test_static_filter_runs_when_the_budget_is_spent():
    """The use the entry point exists for: a query whose HBM budget has no room left."""
    import torch
    from minilake_b200.gpu import LIB, Context
    free_ctx, tight = Context(0), Context(0, hbm_budget=4096)
    n = 200_000
    batch = _rows_batch(free_ctx, n, 5)  # device columns any context on the device can read
    cols, nc = batch.ml_columns()
    pred = (Col(0) > Lit(-20)) & Like(Col(3), "%an%")
    ref, got, spent = _device_u32(n), _device_u32(n), _device_u32(n)
    st, k_ref = _filter(LIB, free_ctx, pred, cols, nc, n, None, 0, ref, static=False)
    assert st == 0
    st, _ = _filter(LIB, tight, pred, cols, nc, n, None, 0, spent, static=False)
    assert st == abi.ERR_BUDGET, "ml_gpu_filter's temporaries are charged to the budget"
    st, k = _filter(LIB, tight, pred, cols, nc, n, None, 0, got, static=True)
    assert st == 0, LIB.ml_gpu_last_error()
    assert k == k_ref and torch.equal(got[:k], ref[:k])
    batch.close()
    tight.close()
    free_ctx.close()


def test_static_filter_limits_and_recovery():
    """Each documented limit fails with ML_ERR_INVALID and names itself; a normal call after
    them still matches ml_gpu_filter; an empty batch selects nothing."""
    import torch
    from minilake_b200.abi import InList
    from minilake_b200.gpu import LIB, Context
    ctx = Context(0)
    n = 50_000
    batch = _rows_batch(ctx, n, 6)
    cols, nc = batch.ml_columns()
    out = _device_u32(n)
    # 64 KiB of literals: an IN list of long strings over the plain string column
    long_words = [bytes([97 + i % 26]) * 400 + str(i).encode() for i in range(200)]
    st, _ = _filter(LIB, ctx, InList(Col(3), long_words), cols, nc, n, None, 0, out, static=True)
    assert st == abi.ERR_INVALID and b"bytes of literals" in LIB.ml_gpu_last_error()
    # 512 KiB of dictionary tables: a dictionary of 65,536 entries needs about 1 MB of them
    pool = [b"w%06d" % i for i in range(65_536)]
    big = ctx.upload([utf8_dict(pool, (np.arange(n) % len(pool)).astype(np.uint32))])
    bcols, bnc = big.ml_columns()
    st, _ = _filter(LIB, ctx, Like(Col(0), "w00%"), bcols, bnc, n, None, 0, out, static=True)
    assert st == abi.ERR_INVALID and b"dictionary tables" in LIB.ml_gpu_last_error()
    # the array is still usable
    pred = (Col(1) < Lit(0.5)) & Like(Col(2), "ab%")
    ref, got = _device_u32(n), _device_u32(n)
    assert _filter(LIB, ctx, pred, cols, nc, n, None, 0, ref, static=False)[0] == 0
    st, k = _filter(LIB, ctx, pred, cols, nc, n, None, 0, got, static=True)
    assert st == 0 and torch.equal(got[:k], ref[:k])
    # no rows: nothing selected
    empty = (abi.MlColumn * nc)(*[cols[i] for i in range(nc)])
    for i in range(nc):
        empty[i].len = 0
    st, k = _filter(LIB, ctx, pred, empty, nc, 0, None, 0, got, static=True)
    assert st == 0 and k == 0, LIB.ml_gpu_last_error()
    big.close()
    batch.close()
    ctx.close()


def test_static_filter_two_threads_at_once():
    """Calls from two threads (two contexts on one device) take turns on the shared array."""
    import threading

    import torch
    from minilake_b200.gpu import LIB, Context
    ctxs = [Context(0), Context(0)]
    n = 120_000
    batches = [_rows_batch(c, n, 40 + i) for i, c in enumerate(ctxs)]
    preds = [(Col(0) > Lit(0)) & Like(Col(3), "%a%"), (Col(1) < Lit(0.3)) | Like(Col(2), "b%")]
    refs = []
    for c, b, p in zip(ctxs, batches, preds):
        cols, nc = b.ml_columns()
        r = _device_u32(n)
        st, k = _filter(LIB, c, p, cols, nc, n, None, 0, r, static=False)
        assert st == 0
        refs.append(r[:k].clone())
    torch.cuda.synchronize()
    errors = []

    def work(i):
        try:
            cols, nc = batches[i].ml_columns()
            for _ in range(20):
                got = _device_u32(n)
                st, k = _filter(LIB, ctxs[i], preds[i], cols, nc, n, None, 0, got, static=True)
                torch.cuda.synchronize()
                if st != 0 or not torch.equal(got[:k], refs[i]):
                    errors.append((i, st, LIB.ml_gpu_last_error()))
        except BaseException as e:  # reported below
            errors.append((i, repr(e)))

    ts = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors
    for b in batches:
        b.close()
    for c in ctxs:
        c.close()
