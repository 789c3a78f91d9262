"""ORDER BY without a limit, limits above the per-warp top-N, and dictionary sort keys: the GPU's
stable radix sort against the CPU oracle's stable sort (sort.rs:85-132).  Row order is index
work: every output column must match exactly, NULLs included.  Keys mix ties, NULLs first and
last, f64 specials (NaN, +-inf, -0.0 against +0.0), plain strings of every length around the
8-byte word boundaries, dictionary strings, booleans and dates, ascending and descending."""
import numpy as np
import pytest

from minilake_b200.abi import BOOL, DATE, FLOAT64, INT32, INT64, UTF8, Col, SortKey
from minilake_b200.columns import Table, encode_strings, fixed, utf8_plain
from oracle import orc

pytestmark = pytest.mark.gpu

WORDS = [b"", b"a", b"ab", b"abcdefg", b"abcdefgh", b"abcdefghi", b"abcdefgh\x00", b"zz", b"b" * 17, b"b" * 16,
         b"\xff\xfe", b"mid", b"abcdefgz", b"b" * 15]
TYPES = [INT32, FLOAT64, UTF8, UTF8, INT64, BOOL, DATE]


@pytest.fixture(scope="module")
def engine():
    from minilake_b200.engine import GpuEngine
    from minilake_b200.gpu import Context
    ctx = Context(0)
    yield GpuEngine(ctx)
    ctx.close()


def _table(n=200_000, groups=6, seed=5):
    rng = np.random.default_rng(seed)
    a = rng.integers(-3, 4, n, dtype=np.int32)
    f = rng.normal(size=n)
    special = rng.random(n)
    f[special < 0.02] = np.nan
    f[(special >= 0.02) & (special < 0.04)] = np.inf
    f[(special >= 0.04) & (special < 0.06)] = -np.inf
    f[(special >= 0.06) & (special < 0.09)] = 0.0
    f[(special >= 0.09) & (special < 0.12)] = -0.0
    f_valid = rng.random(n) > 0.1
    s_idx = rng.integers(0, len(WORDS), n)
    s_valid = rng.random(n) > 0.05
    d_idx = rng.integers(0, len(WORDS), n)
    i64 = rng.integers(-(1 << 62), 1 << 62, n)
    b = (rng.random(n) > 0.5).astype(np.uint8)
    dt = rng.integers(-400, 20000, n, dtype=np.int32)
    rgs = []
    for c in np.array_split(np.arange(n), groups):
        rgs.append([fixed(INT32, a[c]), fixed(FLOAT64, f[c], f_valid[c]),
                    utf8_plain([WORDS[i] for i in s_idx[c]], s_valid[c]),
                    encode_strings(WORDS, d_idx[c]), fixed(INT64, i64[c]), fixed(BOOL, b[c]), fixed(DATE, dt[c])])
    return Table("t", ["a", "f", "s", "d", "i", "b", "dt"], rgs)


KEYSETS = [
    [SortKey(Col(0), INT32), SortKey(Col(1), FLOAT64, asc=False, nulls_first=True)],
    [SortKey(Col(2), UTF8), SortKey(Col(0), INT32, asc=False)],
    [SortKey(Col(3), UTF8, asc=False), SortKey(Col(1), FLOAT64)],
    [SortKey(Col(5), BOOL, asc=False), SortKey(Col(6), DATE), SortKey(Col(2), UTF8, asc=False, nulls_first=True)],
    [SortKey(Col(1), FLOAT64, nulls_first=True)],
]


def _same(got, want):
    assert len(got) == len(want)
    for c, (g, w) in enumerate(zip(got, want)):
        assert len(g) == len(w), f"column {c}: {len(g)} rows, want {len(w)}"
        gm, wm = g.valid_mask(), w.valid_mask()
        assert np.array_equal(gm, wm), f"column {c}: NULLs differ"
        if g.dtype == UTF8:
            gs, ws = g.strings(), w.strings()
            assert [x for x, m in zip(gs, gm) if m] == [x for x, m in zip(ws, wm) if m], f"column {c} differs"
        elif g.dtype == FLOAT64:  # bit patterns: -0.0 and NaN included
            assert np.array_equal(g.values.view(np.uint64)[gm], w.values.view(np.uint64)[wm]), f"column {c} differs"
        else:
            assert np.array_equal(g.values[gm], w.values[wm]), f"column {c} differs"


@pytest.mark.parametrize("k", range(len(KEYSETS)))
def test_order_by_matches_oracle(engine, k):
    t = _table()
    got = engine.fetch(engine.topn(t, TYPES, KEYSETS[k], None))
    want = orc.OracleEngine(threads=1).fetch(orc.OracleEngine(threads=1).topn(t, TYPES, KEYSETS[k], None))
    _same(got, want)


def test_limit_above_the_warp_top_n(engine):
    t = _table(n=400_000, seed=7)
    keys = [SortKey(Col(4), INT64, asc=False)]  # distinct keys: no ties at the limit
    for limit in (2049, 5000, 399_999, 1 << 40):
        got = engine.fetch(engine.topn(t, TYPES, keys, limit))
        want = orc.OracleEngine(threads=4).fetch(orc.OracleEngine(threads=4).topn(t, TYPES, keys, limit))
        _same(got, want)


def test_dictionary_key_with_a_small_limit(engine):
    t = _table(n=50_000, seed=9)
    keys = [SortKey(Col(3), UTF8), SortKey(Col(4), INT64)]
    got = engine.fetch(engine.topn(t, TYPES, keys, 100))
    want = orc.OracleEngine(threads=1).fetch(orc.OracleEngine(threads=1).topn(t, TYPES, keys, 100))
    _same(got, want)


def test_empty_and_multi_threaded_sorts(engine):
    from minilake_b200.engine import GpuEngine
    empty = Table("e", ["a"], [[fixed(INT64, np.zeros(0, np.int64))]])
    assert engine.num_rows(engine.topn(empty, [INT64], [SortKey(Col(0), INT64)], None)) == 0
    # four local sinks; a unique last key makes the order independent of morsel arrival
    t = _table(n=300_000, groups=16, seed=11)
    keys = [SortKey(Col(0), INT32), SortKey(Col(4), INT64)]
    got = GpuEngine(engine.ctx, threads=4).fetch(GpuEngine(engine.ctx, threads=4).topn(t, TYPES, keys, None))
    want = orc.OracleEngine(threads=1).fetch(orc.OracleEngine(threads=1).topn(t, TYPES, keys, None))
    _same(got, want)


def test_sort_of_20m_rows_is_a_sorted_permutation(engine):
    import torch
    from minilake_b200.serving import DeviceTable
    n = 20_000_000
    v = torch.rand(n, dtype=torch.float64, device="cuda") * 1e5
    src = DeviceTable([(FLOAT64, v, None)])
    out = engine.topn([src.ml], [FLOAT64], [SortKey(Col(0), FLOAT64, asc=False)], None)
    got = out.fetch()[0].values
    ref = np.sort(v.cpu().numpy())[::-1]
    assert np.array_equal(got, ref)


def _stable_top(cols, keys, k):
    """Row ids of the first k rows of a stable sort by `keys` (numpy): for each key its NULL
    placement, then its value (negated when descending), the row id last: the GPU's documented
    tie rule, the earlier row first."""
    n = len(cols[0][0])
    lex = [np.arange(n)]
    for key in reversed(keys):
        vals, valid = cols[key.expr.i64]
        v = np.where(valid, vals.astype(np.float64), 0.0)
        lex.append(-v if not key.asc else v)
        lex.append(np.where(valid, 1, 0) if key.nulls_first else np.where(valid, 0, 1))
    return np.lexsort(lex)[:k]


def test_limits_over_heavy_ties_keep_the_earlier_rows(engine):
    """Top-N with k <= 32 over 2M rows (the multi-CTA scan with its shared threshold and final
    merge) on keys where thousands of rows tie at the limit, with NULLs first and last: the rows
    kept and their order are those of a stable sort (the row id breaks the last tie)."""
    rng = np.random.default_rng(17)
    n = 2_000_000
    c0 = rng.integers(0, 100, n).astype(np.int32)
    c1 = rng.integers(0, 50, n).astype(np.float64)
    v1 = rng.random(n) > 0.1
    c2 = rng.permutation(n).astype(np.int64)
    c3 = (rng.random(n) > 0.5).astype(np.uint8)
    c4 = rng.integers(0, 10, n).astype(np.int32)
    ones = np.ones(n, bool)
    cols = [(c0, ones), (c1, v1), (c2, ones), (c3, ones), (c4, ones)]
    types = [INT32, FLOAT64, INT64, BOOL, DATE]
    t = Table("t", ["c0", "c1", "c2", "c3", "c4"],
              [[fixed(INT32, c0), fixed(FLOAT64, c1, v1), fixed(INT64, c2), fixed(BOOL, c3), fixed(DATE, c4)]])
    cases = [([SortKey(Col(0), INT32, asc=False)], 32),
             ([SortKey(Col(1), FLOAT64, nulls_first=True)], 10),
             ([SortKey(Col(1), FLOAT64, asc=False), SortKey(Col(0), INT32)], 17),
             ([SortKey(Col(3), BOOL, asc=False)], 7),
             ([SortKey(Col(4), DATE), SortKey(Col(2), INT64, asc=False)], 1),
             ([SortKey(Col(1), FLOAT64)], 32)]
    for keys, k in cases:
        got = engine.fetch(engine.topn(t, types, keys, k))
        rows = _stable_top(cols, keys, k)
        assert len(got[0]) == k, keys
        for c, (vals, valid) in enumerate(cols):
            assert np.array_equal(got[c].valid_mask(), valid[rows]), (keys, c)
            assert np.array_equal(got[c].values[valid[rows]], vals[rows][valid[rows]]), (keys, c)
