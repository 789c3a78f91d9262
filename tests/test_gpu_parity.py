"""Parity of the CUDA path (through the C ABI) with the CPU oracle on the same seeded
inputs.  Integer/byte/index results must be bit-exact; float64 sums within 1e-12
relative (summation order differs); everything else bit-exact."""
import numpy as np
import pytest

from helpers import (e2e_tables, golden, q_case_in_like_between, q_count, q_group_by, q_join_top_n, rel_err)
from minilake_b200 import abi
from minilake_b200.abi import (AND, AVG, BOOL, COUNT, COUNT_STAR, DATE, DIV, FLOAT64, INT32, INT64, MAX, MIN, MOD,
                               OR, SUM, UTF8, AggSpec, Binary, Case, Cast, Col, Filter, InList, IsNull, Like, Lit,
                               Negate, Not, Probe, Project, SortKey)
from minilake_b200.columns import Table, encode_strings, fixed, utf8_dict, utf8_plain
from oracle import orc

pytestmark = pytest.mark.gpu
F64_TOL = 1e-12


@pytest.fixture(scope="module", params=["specialized", "interpreter"])
def ctx(request):
    """Every parity test runs twice: with the runtime-specialized pipeline kernels (the
    default) and with the ahead-of-time interpreter kernels (ML_CTX_INTERPRET)."""
    from minilake_b200.gpu import INTERPRET, Context
    c = Context(0, flags=INTERPRET if request.param == "interpreter" else 0)
    c.mode = request.param
    yield c
    c.close()


@pytest.fixture(scope="module")
def gpu_engine(ctx):
    from minilake_b200.engine import GpuEngine
    return GpuEngine(ctx)


WORDS = [b"apple", b"banana", b"cherry", b"abricot", b"", b"ab", b"zeta", b"apricot pie", b"BANANA"]


def random_batch(rng, n, null_frac=0.1, dict_strings=True):
    """[i32, i64, f64, date, bool, utf8 (dict or plain), utf8 plain] with NULLs."""
    def nulls():
        return rng.random(n) >= null_frac

    i32 = rng.integers(-50, 50, n, dtype=np.int32)
    i64 = rng.integers(-1000, 1000, n, dtype=np.int64)
    f64 = np.round(rng.normal(0, 100, n), 3)
    f64[rng.random(n) < 0.05] = -0.0
    f64[rng.random(n) < 0.05] = 0.0
    dt = rng.integers(9000, 9100, n, dtype=np.int32)
    b = rng.random(n) < 0.5
    idx = rng.integers(0, len(WORDS), n)
    s1 = encode_strings(WORDS, idx, nulls()) if dict_strings else utf8_plain([WORDS[i] for i in idx], nulls())
    s2 = utf8_plain([WORDS[i] for i in rng.integers(0, len(WORDS), n)], nulls())
    return [fixed(INT32, i32, nulls()), fixed(INT64, i64, nulls()), fixed(FLOAT64, f64, nulls()),
            fixed(DATE, dt, nulls()), fixed(abi.BOOL, b, nulls()), s1, s2]


TYPES = [INT32, INT64, FLOAT64, DATE, BOOL, UTF8, UTF8]

PREDICATES = [
    Col(0) < Lit(3),
    Col(1) >= Lit(-10),
    (Col(2) > Lit(0.5)) & (Col(0) <= Lit(20)),
    (Col(2) > Lit(0.5)) | Not(Col(4)),
    Col(3).eq(Lit(9050, DATE)),
    Col(5).eq(Lit("apple")),
    Col(5) > Lit("b"),
    Lit("banana").ne(Col(6)),
    Like(Col(5), "ab%"), Like(Col(6), "%an%"), Like(Col(5), "%e"), Like(Col(6), "a_r%"), Like(Col(5), "zeta"),
    Like(Col(6), "ap%", negated=True),
    InList(Col(0), [1, 2, 3, -7]), InList(Col(5), ["cherry", "zeta", ""]), InList(Col(6), ["ab"], negated=True),
    IsNull(Col(2)), IsNull(Col(5), negated=True),
    (Col(1) % Lit(7)).eq(Lit(0)),
    (Col(1) / Col(0)) > Lit(2.0),
    Binary(abi.GT, Col(0) + Col(1), Col(1) * Lit(2)),
    Case([(Col(0) > Lit(0), Col(4)), (Col(1) < Lit(0), Lit(True))], Lit(False), BOOL),
    Cast(Col(2), INT64) > Lit(10),
    Col(5).eq(Col(6)),
    Negate(Col(0)) > Lit(10),
    Lit(True),
    Col(0) > Lit(None, INT64),
]


def test_filter_matches_oracle(ctx):
    from minilake_b200.gpu import FilterOperator
    rng = np.random.default_rng(1)
    for n in (0, 1, 31, 1000, 70_001):
        for dict_strings in (True, False):
            cols = random_batch(rng, n, dict_strings=dict_strings)
            sel = np.sort(rng.choice(n, n // 3, replace=False)).astype(np.uint32) if n else None
            for k, p in enumerate(PREDICATES):
                want = orc.filter_rows(p, cols)
                got = FilterOperator(ctx, p).execute(cols)
                assert np.array_equal(got, want), (n, k)
                if sel is not None:
                    want = orc.filter_rows(p, cols, sel)
                    got = FilterOperator(ctx, p).execute(cols, sel)
                    assert np.array_equal(got, want), ("sel", n, k)


EXPRS = [
    (Col(2) * (Lit(1) - Col(2)), FLOAT64),
    (Col(0) + Col(1), INT64),
    (Col(0) * Lit(1_000_000_007), INT64),
    (Col(2) / Col(1), FLOAT64),
    (Col(1) % Col(0), INT64),
    (Col(0) % Lit(-1), INT32),
    (Cast(Col(2), INT32), INT32),
    (Cast(Col(1), FLOAT64), FLOAT64),
    (Col(3) + Lit(30), DATE),
    (Case([(Col(0) > Lit(0), Col(2)), (IsNull(Col(2)), Lit(-1.5))], None, FLOAT64), FLOAT64),
    (Negate(Col(2)), FLOAT64),
    (Col(2) + Col(2) * Col(2), FLOAT64),
    (Lit(7), INT64),
]


def test_project_matches_oracle_bit_exact(ctx):
    from minilake_b200.gpu import ProjectionOperator
    rng = np.random.default_rng(2)
    for n in (1, 257, 50_000):
        cols = random_batch(rng, n)
        for k, (e, t) in enumerate(EXPRS):
            want = orc.project(e, t, cols)[0]
            got = ProjectionOperator(ctx, e, t).execute(cols).fetch()[0]
            vm = want.valid_mask()
            assert np.array_equal(got.valid_mask(), vm), (n, k)
            a, b = got.values[vm], want.values[vm]
            if t == FLOAT64:
                assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (n, k)
            else:
                assert np.array_equal(a, b), (n, k)


def test_hash_columns_bit_exact(ctx):
    from minilake_b200.gpu import hash_columns
    rng = np.random.default_rng(3)
    for n in (0, 5, 10_000):
        cols = random_batch(rng, n)
        for subset in ([0], [1, 2], [3, 4], [5], [6], [0, 1, 2, 3, 4, 5, 6]):
            cs = [cols[i] for i in subset]
            assert np.array_equal(hash_columns(ctx, cs), orc.hash_columns(cs)), (n, subset)
        if n:
            sel = np.arange(0, n, 3, dtype=np.uint32)
            assert np.array_equal(hash_columns(ctx, cols, sel), orc.hash_columns(cols, sel))


def _rows(cols, key_idx):
    """Result rows as python tuples (None for NULL), sorted by the key columns."""
    out = []
    n = len(cols[0])
    vals = []
    for c in cols:
        vm = c.valid_mask()
        if c.dtype == UTF8:
            s = c.strings()
            vals.append([s[i] if vm[i] else None for i in range(n)])
        else:
            vals.append([c.values[i].item() if vm[i] else None for i in range(n)])
    for i in range(n):
        out.append(tuple(v[i] for v in vals))
    return sorted(out, key=lambda r: tuple((x is None, x if x is not None else 0) for x in (r[k] for k in key_idx)))


def assert_same_rows(got, want, nkeys, float_cols=()):
    g = _rows(got, list(range(nkeys)))
    w = _rows(want, list(range(nkeys)))
    assert len(g) == len(w)
    for a, b in zip(g, w):
        for k, (x, y) in enumerate(zip(a, b)):
            if k in float_cols and x is not None and y is not None:
                assert abs(x - y) <= F64_TOL * max(abs(y), 1e-300) or x == y, (a, b)
            else:
                assert x == y or (isinstance(x, float) and np.isnan(x) and np.isnan(y)), (a, b)


AGGS = [AggSpec(COUNT_STAR), AggSpec(COUNT, Col(2), FLOAT64), AggSpec(SUM, Col(2), FLOAT64),
        AggSpec(SUM, Col(0), INT32), AggSpec(AVG, Col(1), INT64), AggSpec(MIN, Col(3), DATE),
        AggSpec(MAX, Col(2), FLOAT64), AggSpec(MAX, Col(1), INT64)]
AGG_FLOAT_COLS = (2, 4, 6)  # offsets after the keys: SUM f64, AVG, MAX f64 (MAX compares exactly)


@pytest.mark.parametrize("keys", [[(Col(0), INT32)], [(Col(5), UTF8)], [(Col(4), BOOL), (Col(3), DATE)],
                                  [(Col(5), UTF8), (Col(4), BOOL)],
                                  [(Col(1), INT64), (Col(0), INT32)], [(Cast(Col(2), INT64), INT64)], []])
def test_hashagg_matches_oracle(gpu_engine, keys):
    rng = np.random.default_rng(4)
    rgs = [random_batch(rng, n) for n in (5000, 1, 0, 12_345)]
    t = Table("t", [str(i) for i in range(7)], rgs)
    pro = [Filter(Col(1) > Lit(-900))]
    for size_hint in (0, 100_000):
        got = gpu_engine.fetch(gpu_engine.hashagg(t, TYPES, keys, AGGS, pro, size_hint=size_hint))
        want = orc.OracleEngine(threads=3).fetch(orc.OracleEngine(threads=3).hashagg(t, TYPES, keys, AGGS, pro))
        nk = len(keys)
        fl = {nk + 2, nk + 4}
        assert_same_rows(got, want, nk, fl)


def test_predicates_in_fused_aggregate(ctx, gpu_engine):
    """Every expression form as the filter of a fused aggregate (the pipeline kernel
    evaluates it per row), against the oracle."""
    rng = np.random.default_rng(9)
    t = Table("t", [str(i) for i in range(7)], [random_batch(rng, n) for n in (7000, 3000)])
    aggs = [AggSpec(COUNT_STAR), AggSpec(SUM, Col(2), FLOAT64), AggSpec(MIN, Col(1), INT64)]
    oracle = orc.OracleEngine(threads=2)
    before = ctx.profile("jit_launch")[0]
    for pred in PREDICATES:
        got = gpu_engine.fetch(gpu_engine.hashagg(t, TYPES, [(Col(0), INT32)], aggs, [Filter(pred)]))
        want = oracle.fetch(oracle.hashagg(t, TYPES, [(Col(0), INT32)], aggs, [Filter(pred)]))
        assert_same_rows(got, want, 1, {2})
    launched = ctx.profile("jit_launch")[0] - before
    assert launched > 0 if ctx.mode == "specialized" else launched == 0


def test_hashagg_resize_on_overflow_is_exact(gpu_engine):
    rng = np.random.default_rng(5)
    n = 300_000
    keys = rng.integers(0, 120_000, n).astype(np.int64)
    v = rng.random(n)
    t = Table("t", ["k", "v"], [[fixed(INT64, keys[i::3]), fixed(FLOAT64, v[i::3])] for i in range(3)])
    aggs = [AggSpec(SUM, Col(1), FLOAT64), AggSpec(COUNT_STAR)]
    plain = gpu_engine.hashagg(t, [INT64, FLOAT64], [(Col(0), INT64)], aggs, size_hint=0)
    assert plain.sink_stats["resizes"] > 0
    sized = gpu_engine.hashagg(t, [INT64, FLOAT64], [(Col(0), INT64)], aggs, size_hint=120_000)
    assert sized.sink_stats["resizes"] == 0
    a, b = plain.fetch(), sized.fetch()
    assert_same_rows(a, b, 1, {1})
    k, cnt = np.unique(keys, return_counts=True)
    r = _rows(a, [0])
    assert [x[0] for x in r] == list(k) and [x[2] for x in r] == list(cnt)


def test_join_probe_pairs_match_oracle(ctx, gpu_engine):
    from minilake_b200.gpu import HashJoinProbe
    rng = np.random.default_rng(6)
    nb = 5000
    bkey = rng.integers(0, 2000, nb).astype(np.int64)  # duplicates
    bvalid = rng.random(nb) > 0.05                       # NULL keys never match
    build = Table("b", ["k", "x"], [[fixed(INT64, bkey[:2500], bvalid[:2500]), fixed(INT32, np.arange(2500))],
                                    [fixed(INT64, bkey[2500:], bvalid[2500:]), fixed(INT32, np.arange(2500, nb))]])
    g = gpu_engine.join_build(build, [INT64, INT32], [(Col(0), INT64)])
    # one oracle thread: its build batch keeps the row groups in order, as the single-threaded
    # GPU engine's does, so build row ids of both sides index `bkey` the same way
    o = orc.OracleEngine(threads=1).join_build(build, [INT64, INT32], [(Col(0), INT64)])
    assert g.stats()["build_rows"] == o.stats()["build_rows"] == nb
    assert g.stats()["distinct_keys"] == o.stats()["distinct_keys"]
    pk = rng.integers(-5, 2100, 20_000).astype(np.int64)
    cols = [fixed(INT64, pk, rng.random(20_000) > 0.1)]
    gp, gb = HashJoinProbe(ctx, g.handle, [(Col(0), INT64)]).execute(cols)
    op, ob = orc.join_probe(o, [(Col(0), INT64)], cols)
    assert np.array_equal(gp, np.sort(gp, kind="stable")), "pairs ordered by probe row"
    # build row ids index each side's own build batch: compare the build keys and x payloads
    gx = np.concatenate([np.arange(2500), np.arange(2500, nb)])
    assert sorted(zip(gp.tolist(), bkey[gx[gb]].tolist())) == sorted(zip(op.tolist(), bkey[ob].tolist()))
    assert len(gp) == len(op)


def test_join_chains_through_fused_aggregate(gpu_engine):
    rng = np.random.default_rng(7)
    dim = Table("d", ["k", "g"], [[fixed(INT64, rng.integers(0, 300, 2000)), fixed(INT32, rng.integers(0, 9, 2000))]])
    fact = Table("f", ["fk", "v"], [[fixed(INT64, rng.integers(0, 320, 30_000)), fixed(FLOAT64, rng.random(30_000))]
                                    for _ in range(3)])
    for eng in (gpu_engine, orc.OracleEngine(threads=2)):
        j = eng.join_build(dim, [INT64, INT32], [(Col(0), INT64)])
        out = eng.hashagg(fact, [INT64, FLOAT64], [(Col(3), INT32)],
                          [AggSpec(SUM, Col(1), FLOAT64), AggSpec(COUNT_STAR)],
                          prologue=[Probe(j.handle, [(Col(0), INT64)])])
        if eng is gpu_engine:
            got = eng.fetch(out)
        else:
            want = eng.fetch(out)
    assert_same_rows(got, want, 1, {1})


def test_topn_matches_oracle(gpu_engine):
    rng = np.random.default_rng(8)
    n = 40_000
    a = rng.permutation(n).astype(np.int64)
    f = rng.normal(0, 1, n)
    f[::97] = -0.0
    valid = rng.random(n) > 0.02
    s = [b"%06d" % x for x in rng.permutation(n)]
    t = Table("t", ["a", "f", "s"], [[fixed(INT64, a[:n // 2]), fixed(FLOAT64, f[:n // 2], valid[:n // 2]),
                                     utf8_plain(s[:n // 2])],
                                    [fixed(INT64, a[n // 2:]), fixed(FLOAT64, f[n // 2:], valid[n // 2:]),
                                     utf8_plain(s[n // 2:])]])
    cases = [([SortKey(Col(1), FLOAT64, asc=False), SortKey(Col(0), INT64)], 10),
             ([SortKey(Col(1), FLOAT64, asc=True, nulls_first=True), SortKey(Col(0), INT64)], 100),
             ([SortKey(Col(2), UTF8, asc=False)], 2048),
             ([SortKey(Col(0), INT64)], 1)]
    for keys, k in cases:
        got = gpu_engine.fetch(gpu_engine.topn(t, [INT64, FLOAT64, UTF8], keys, k))
        want = orc.OracleEngine(threads=2).fetch(orc.OracleEngine(threads=2).topn(t, [INT64, FLOAT64, UTF8], keys, k))
        assert np.array_equal(got[0].values, want[0].values), keys
        assert got[2].strings() == want[2].strings()


def test_end_to_end_known_answers(gpu_engine):
    e = golden()["end_to_end"]
    lineitem, orders = e2e_tables()
    r = q_count(gpu_engine, lineitem)
    assert [int(r[0].values[0]), int(r[1].values[0])] == [e["count_star_and_nulls"]["count_star"],
                                                        e["count_star_and_nulls"]["count_qty"]]
    g = e["group_by_order_by"]
    r = q_group_by(gpu_engine, lineitem, g["cutoff"])
    assert [s.decode() for s in r[0].strings()] == [row[0] for row in g["rows"]]
    assert rel_err(r[1].values, [row[1] for row in g["rows"]]).max() <= 1e-9
    assert list(r[2].values) == [row[2] for row in g["rows"]]
    assert rel_err(r[3].values, [row[3] for row in g["rows"]]).max() <= 1e-9
    assert list(r[4].values) == [row[4] for row in g["rows"]]
    j = e["join_top_n"]
    r, _ = q_join_top_n(gpu_engine, lineitem, orders, j["cutoff"])
    assert [s.decode() for s in r[0].strings()] == [row[0] for row in j["rows"]]
    assert rel_err(r[1].values, [row[1] for row in j["rows"]]).max() <= 1e-9
    c = e["case_in_like_between"]
    r = q_case_in_like_between(gpu_engine, lineitem)
    assert [int(r[0].values[0]), int(r[1].values[0])] == [c["sum_case"], c["count"]]


def test_hbm_budget_refusal_and_release():  # memory_limit.rs:47-68, end_to_end.rs:341-359
    from minilake_b200.engine import GpuEngine
    from minilake_b200.gpu import Context, ResourcesExhausted
    g = golden()["memory_limit"]
    groups = g["groups"]
    rgs = [[fixed(INT64, (np.arange(groups) * 7 + b) % groups), fixed(INT64, np.ones(groups, dtype=np.int64))]
           for b in range(g["batches"])]
    t = Table("t", ["k", "v"], rgs)
    ctx = Context(0, hbm_budget=g["budget"])
    with pytest.raises(ResourcesExhausted) as ei:
        GpuEngine(ctx).hashagg(t, [INT64, INT64], [(Col(0), INT64)], [AggSpec(SUM, Col(1), INT64)])
    assert ei.value.operator.startswith("HashAggregate")
    assert ctx.pool_stats()[0] == 0, "everything reserved by the failed operator is released"
    lineitem, orders = e2e_tables()
    small = Context(0, hbm_budget=1024)
    with pytest.raises(ResourcesExhausted):
        q_join_top_n(GpuEngine(small), lineitem, orders, 0)
    ok = Context(0)
    out = GpuEngine(ok).hashagg(t, [INT64, INT64], [(Col(0), INT64)], [AggSpec(SUM, Col(1), INT64)]).fetch()
    assert len(out[0].values) == groups and (out[1].values == g["batches"]).all()
    small.close()
    ctx.close()
    ok.close()


def test_multithreaded_local_sinks_share_one_table(ctx):
    from minilake_b200.engine import GpuEngine
    from minilake_b200 import datagen, workloads
    t = datagen.filter_groupby(rows=400_000, row_groups=16)
    got = workloads.run_filter_groupby(GpuEngine(ctx, threads=4), t)
    want = workloads.run_filter_groupby(orc.OracleEngine(threads=4), t)
    assert got[0].strings() == want[0].strings() and got[1].strings() == want[1].strings()
    assert np.array_equal(got[5].values, want[5].values) and np.array_equal(got[2].values, want[2].values)
    assert rel_err(got[3].values, want[3].values).max() <= F64_TOL


@pytest.mark.parametrize("by_build_column", [False, True])
def test_group_by_join_key_with_duplicate_and_null_build_keys(gpu_engine, by_build_column):
    rng = np.random.default_rng(11)
    nd = 3000
    dk = rng.integers(0, 500, nd).astype(np.int64)  # duplicate keys: chains
    dim = Table("d", ["k", "x"], [[fixed(INT64, dk, rng.random(nd) > 0.02), fixed(INT32, rng.integers(0, 9, nd))]])
    fact = Table("f", ["fk", "d", "v"], [[fixed(INT64, rng.integers(-5, 520, 40_000)),
                                          fixed(INT32, rng.integers(0, 100, 40_000)),
                                          fixed(FLOAT64, rng.random(40_000), rng.random(40_000) > 0.03)]
                                         for _ in range(2)])
    # the build (dim) is on the right: [fk, d, v, k, x]
    key = Col(3) if by_build_column else Col(0)
    aggs = [AggSpec(SUM, Col(2), FLOAT64), AggSpec(COUNT_STAR), AggSpec(MIN, Col(1), INT32), AggSpec(COUNT, Col(2), FLOAT64)]
    res = {}
    for name, eng in (("gpu", gpu_engine), ("oracle", orc.OracleEngine(threads=2))):
        j = eng.join_build(dim, [INT64, INT32], [(Col(0), INT64)])
        out = eng.hashagg(fact, [INT64, INT32, FLOAT64], [(key, INT64)], aggs,
                          prologue=[Filter(Col(1) < Lit(90)), Probe(j.handle, [(Col(0), INT64)])])
        if name == "gpu":
            assert out.sink_stats["capacity"] == 0, "expected the join-key group mode (no aggregate table)"
        res[name] = eng.fetch(out)
    assert_same_rows(res["gpu"], res["oracle"], 1, {1})


@pytest.mark.parametrize("kind", ["dense", "small_wide", "sparse", "negative_i32", "compound", "utf8"])
def test_join_index_kinds_match_oracle(gpu_engine, kind):
    """Dense integer keys use the direct index, all other keys (string keys by their global
    string ids) the hash table; both must give the oracle's matches (through the fused
    aggregate) and distinct-key counts."""
    rng = np.random.default_rng(12)
    nd, nf = 4000, 30_000
    valid = rng.random(nd) > 0.03
    if kind == "dense":
        pool = np.arange(100, 2100, dtype=np.int64)
        types, mk = [INT64], lambda v, m=None: [fixed(INT64, v, m)]
    elif kind == "small_wide":  # few keys spread over a range that still fits a 4 MB index
        pool = np.sort(rng.choice(500_000, 300, replace=False)).astype(np.int64) + 7
        types, mk = [INT64], lambda v, m=None: [fixed(INT64, v, m)]
    elif kind == "sparse":
        pool = rng.integers(-2**62, 2**62, 1500, dtype=np.int64)
        types, mk = [INT64], lambda v, m=None: [fixed(INT64, v, m)]
    elif kind == "negative_i32":
        pool = np.arange(-1000, 1000, dtype=np.int32)
        types, mk = [INT32], lambda v, m=None: [fixed(INT32, v, m)]
    elif kind == "compound":
        pool = np.arange(3000, dtype=np.int64)
        types = [INT32, INT32]
        mk = lambda v, m=None: [fixed(INT32, (v % 50).astype(np.int32), m), fixed(INT32, (v // 50).astype(np.int32))]
    else:
        pool = np.array([b"k%05d" % i for i in range(1200)], dtype=object)
        types = [UTF8]
        mk = lambda v, m=None: [utf8_plain(list(v), m)]
    dk = pool[rng.integers(0, len(pool), nd)]
    # fact keys: mostly from the pool, some misses
    fk = pool[rng.integers(0, len(pool), nf)]
    if kind == "dense":  # probe keys below, inside and above the indexed range
        fk = rng.integers(0, 2300, nf).astype(np.int64)
    nkey = len(types)
    dim = Table("d", [f"k{i}" for i in range(nkey)] + ["x"], [mk(dk, valid) + [fixed(INT32, rng.integers(0, 13, nd))]])
    fact = Table("f", [f"f{i}" for i in range(nkey)] + ["v"], [mk(fk) + [fixed(FLOAT64, rng.random(nf))]])
    keys = [(Col(i), t) for i, t in enumerate(types)]
    # fact columns [f.., v] then build columns [k.., x]: x is column 2 * nkey + 1
    group = [(Col(2 * nkey + 1), INT32)]
    aggs = [AggSpec(SUM, Col(nkey), FLOAT64), AggSpec(COUNT_STAR)]
    res, stats = {}, {}
    for name, eng in (("gpu", gpu_engine), ("oracle", orc.OracleEngine(threads=2))):
        j = eng.join_build(dim, types + [INT32], keys)
        stats[name] = j.stats()
        out = eng.hashagg(fact, types + [FLOAT64], group, aggs, prologue=[Probe(j.handle, keys)])
        res[name] = eng.fetch(out)
    assert stats["gpu"]["distinct_keys"] == stats["oracle"]["distinct_keys"]
    if kind == "dense":
        assert stats["gpu"]["capacity"] == 2000  # value range 100..2099: direct index
    elif kind == "small_wide":
        lo, hi = dk[valid].min(), dk[valid].max()
        assert stats["gpu"]["capacity"] == hi - lo + 1  # direct index over the valid keys' range
    else:
        cap = stats["gpu"]["capacity"]
        assert cap & (cap - 1) == 0, "hash table capacity is a power of two"
    assert_same_rows(res["gpu"], res["oracle"], 1, {1})


def test_group_by_dense_join_key_checks_membership_per_group(ctx, gpu_engine):
    """GROUP BY a dense, distinct join key at the end of the pipeline: rows aggregate by the
    key's index position and only keys present in the build side are emitted (fact keys that
    are in the key range but not in the dimension, outside it, or NULL never appear)."""
    rng = np.random.default_rng(13)
    dk = np.sort(rng.choice(4000, 3000, replace=False)).astype(np.int64) + 100
    dim = Table("d", ["k"], [[fixed(INT64, rng.permutation(dk))]])
    n = 50_000
    fact = Table("f", ["fk", "d", "v"], [[fixed(INT64, rng.integers(-20, 4200, n).astype(np.int64), rng.random(n) > 0.02),
                                          fixed(INT32, rng.integers(0, 100, n)), fixed(FLOAT64, rng.random(n))]
                                         for _ in range(2)])
    aggs = [AggSpec(SUM, Col(2), FLOAT64), AggSpec(COUNT_STAR), AggSpec(MIN, Col(1), INT32), AggSpec(AVG, Col(2), FLOAT64)]
    res = {}
    for name, eng in (("gpu", gpu_engine), ("oracle", orc.OracleEngine(threads=2))):
        j = eng.join_build(dim, [INT64], [(Col(0), INT64)])
        out = eng.hashagg(fact, [INT64, INT32, FLOAT64], [(Col(0), INT64)], aggs,
                          prologue=[Filter(Col(1) < Lit(80)), Probe(j.handle, [(Col(0), INT64)])])
        if name == "gpu":
            assert j.stats()["capacity"] <= 4000  # the direct (dense) index
        res[name] = eng.fetch(out)
    assert_same_rows(res["gpu"], res["oracle"], 1, {1, 4})


@pytest.mark.parametrize("groups", [3, 20])
def test_low_cardinality_group_by_every_aggregate(gpu_engine, groups):
    """Few groups and no NULLs: the first groups take per-thread accumulators in the
    specialized kernel (the rest shared-memory atomics); every aggregate kind against the oracle."""
    rng = np.random.default_rng(14 + groups)
    n = 60_000
    cols = lambda: [fixed(INT32, rng.integers(0, groups, n).astype(np.int32)), fixed(INT64, rng.integers(-10**6, 10**6, n)),
                    fixed(FLOAT64, np.round(rng.normal(0, 50, n), 2)), fixed(DATE, rng.integers(9000, 9500, n).astype(np.int32))]
    t = Table("t", ["g", "i", "f", "d"], [cols() for _ in range(3)])
    types = [INT32, INT64, FLOAT64, DATE]
    pro = [Filter(Col(1) > Lit(-900_000))]
    oracle = orc.OracleEngine(threads=2)
    for aggs in ([AggSpec(COUNT_STAR), AggSpec(COUNT, Col(2), FLOAT64), AggSpec(SUM, Col(1), INT64),
                  AggSpec(SUM, Col(2), FLOAT64), AggSpec(AVG, Col(2), FLOAT64), AggSpec(MIN, Col(1), INT64),
                  AggSpec(MAX, Col(1), INT64)],
                 [AggSpec(MIN, Col(2), FLOAT64), AggSpec(MAX, Col(2), FLOAT64), AggSpec(MIN, Col(3), DATE),
                  AggSpec(MAX, Col(3), DATE), AggSpec(COUNT_STAR)]):
        got = gpu_engine.fetch(gpu_engine.hashagg(t, types, [(Col(0), INT32)], aggs, pro))
        want = oracle.fetch(oracle.hashagg(t, types, [(Col(0), INT32)], aggs, pro))
        assert_same_rows(got, want, 1, {4, 5} if len(aggs) == 7 else set())


@pytest.mark.parametrize("dups", [False, True])
def test_semi_join_probe_matches_oracle(gpu_engine, dups):
    """A probe whose build rows nothing reads (GROUP BY and aggregates over fact columns only)
    tests membership in the dense index's bitmap when the build keys are distinct; with
    duplicate build keys every match still counts once per build row."""
    rng = np.random.default_rng(21)
    nd, nf = 3000, 50_000
    dk = rng.choice(200_000, nd, replace=False).astype(np.int64) + 11
    if dups:
        dk[: nd // 3] = dk[nd // 3: 2 * (nd // 3)]
    valid = rng.random(nd) > 0.02
    dim = Table("d", ["k", "x"], [[fixed(INT64, dk, valid), fixed(INT32, rng.integers(0, 9, nd).astype(np.int32))]])
    fk = np.where(rng.random(nf) < 0.5, dk[rng.integers(0, nd, nf)], rng.integers(0, 200_020, nf)).astype(np.int64)
    g = rng.integers(0, 40, nf).astype(np.int32)
    fact = Table("f", ["fk", "g", "v"], [[fixed(INT64, fk[:20_000]), fixed(INT32, g[:20_000]), fixed(FLOAT64, rng.random(20_000))],
                                        [fixed(INT64, fk[20_000:]), fixed(INT32, g[20_000:]), fixed(FLOAT64, rng.random(nf - 20_000))]])
    keys = [(Col(0), INT64)]
    aggs = [AggSpec(SUM, Col(2), FLOAT64), AggSpec(COUNT_STAR)]
    res = {}
    for name, eng in (("gpu", gpu_engine), ("oracle", orc.OracleEngine(threads=1))):
        j = eng.join_build(dim, [INT64, INT32], keys)
        out = eng.hashagg(fact, [INT64, INT32, FLOAT64], [(Col(1), INT32)], aggs, prologue=[Probe(j.handle, keys)])
        res[name] = eng.fetch(out)
    assert_same_rows(res["gpu"], res["oracle"], 1, {1})


def test_resident_runs_match_a_local_sink(ctx, gpu_engine):
    """ml_gpu_hashagg_run_resident: the first run of a launch shape goes without a graph, the
    second is captured, later ones replay; every run (with reset) gives the local sink's result,
    also after new constants are bound."""
    from minilake_b200.gpu import HashAggregateSink
    rng = np.random.default_rng(33)
    n = 70_000
    cols = [fixed(INT32, rng.integers(0, 50, n).astype(np.int32)), fixed(INT64, rng.integers(-500, 500, n)),
            fixed(FLOAT64, np.round(rng.normal(0, 10, n), 3))]
    dev = ctx.upload(cols)
    types = [INT32, INT64, FLOAT64]
    group = [(Col(0), INT32)]
    aggs = [AggSpec(SUM, Col(2), FLOAT64), AggSpec(MAX, Col(1), INT64), AggSpec(COUNT_STAR)]
    t = Table("t", ["g", "i", "f"], [cols])
    sink = HashAggregateSink(ctx, types, group, aggs, [Filter(Col(1) > Lit(-400))], size_hint=128)
    for cutoff in (-400, 100):
        if cutoff != -400:
            sink.rebind([Filter(Col(1) > Lit(cutoff))], group, aggs)
        want = gpu_engine.fetch(gpu_engine.hashagg(t, types, group, aggs, [Filter(Col(1) > Lit(cutoff))]))
        for _ in range(3):
            sink.run_resident(dev, reset=True)
            out = sink.finalize()
            assert_same_rows(gpu_engine.fetch(out), want, 1, {1})
            out.close()
    st = sink.graph_stats()
    assert st["built"] >= 1 and st["replayed"] >= 1, st
    sink.close()
