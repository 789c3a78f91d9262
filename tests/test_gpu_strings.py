"""String keys against the CPU oracle: GROUP BY a plain (not dictionary-encoded) source string
column, and joins on string keys (group_keys.rs:88-92, join.rs:160-203 with kernels/hash.rs:55-77).

Row groups of one column may be plain or dictionary-encoded (encode_strings picks per row group,
as the Parquet reader does), the same strings recur across row groups, NULL keys form their own
group (GROUP BY) and never match (joins), build sides hold duplicate keys.  Group keys, counts,
join pairs: bit-exact; f64 sums within 1e-12.  Both kernel forms run (the `ctx` fixture)."""
import numpy as np
import pytest

from minilake_b200.abi import COUNT_STAR, FLOAT64, INT32, INT64, SUM, UTF8, AggSpec, Col, Filter, Lit, Probe
from minilake_b200.columns import Table, encode_strings, fixed, utf8_plain
from oracle import orc
from test_gpu_parity import assert_same_rows, ctx, gpu_engine  # noqa: F401  (fixtures)

pytestmark = pytest.mark.gpu

POOL = [b"w%05d-%s" % (i, b"x" * (i % 23)) for i in range(3000)] + [b"", b"a", b"ab"]


def _string_col(rng, idx, valid, plain):
    if plain:
        return utf8_plain([POOL[i] for i in idx], valid)
    return encode_strings(POOL, idx, valid)


def _fact(rng, n, groups, distinct):
    rgs = []
    for g in range(groups):
        idx = rng.integers(0, distinct, n)
        valid = rng.random(n) > 0.05
        # alternate plain and dictionary row groups of the same column
        rgs.append([_string_col(rng, idx, valid, plain=g % 2 == 0), fixed(FLOAT64, rng.random(n)),
                    fixed(INT32, rng.integers(0, 100, n, dtype=np.int32))])
    return Table("f", ["s", "v", "d"], rgs)


@pytest.mark.parametrize("distinct", [40, 3000])
def test_group_by_plain_source_string(gpu_engine, distinct):
    from minilake_b200.engine import GpuEngine
    rng = np.random.default_rng(distinct)
    fact = _fact(rng, 20_000, 6, distinct)
    aggs = [AggSpec(SUM, Col(1), FLOAT64), AggSpec(COUNT_STAR)]
    group = [(Col(0), UTF8), (Col(2), INT32)] if distinct == 40 else [(Col(0), UTF8)]
    prologue = [Filter(Col(2) < Lit(80))]
    want = orc.OracleEngine(threads=2).fetch(
        orc.OracleEngine(threads=2).hashagg(fact, [UTF8, FLOAT64, INT32], group, aggs, prologue))
    for eng in (gpu_engine, GpuEngine(gpu_engine.ctx, threads=3)):
        got = eng.fetch(eng.hashagg(fact, [UTF8, FLOAT64, INT32], group, aggs, prologue))
        assert_same_rows(got, want, len(group), {len(group)})


def _dim(rng, nd, plain):
    idx = rng.integers(0, 2500, nd)  # duplicate build keys
    valid = rng.random(nd) > 0.03     # NULL build keys never match
    return Table("d", ["s", "x"], [[_string_col(rng, idx, valid, plain), fixed(INT32, np.arange(nd, dtype=np.int32))]])


@pytest.mark.parametrize("build_plain", [True, False])
def test_string_join_keys_through_the_fused_aggregate(gpu_engine, build_plain):
    rng = np.random.default_rng(17 + build_plain)
    dim = _dim(rng, 4000, build_plain)
    fact = _fact(rng, 15_000, 4, 3003)
    keys = [(Col(0), UTF8)]
    res = {}
    for name, eng in (("gpu", gpu_engine), ("oracle", orc.OracleEngine(threads=1))):
        j = eng.join_build(dim, [UTF8, INT32], keys)
        # [s_build, x, s, v, d] (build on the left): GROUP BY the build-side payload
        out = eng.hashagg(fact, [UTF8, FLOAT64, INT32], [(Col(1), INT32)],
                          [AggSpec(SUM, Col(3), FLOAT64), AggSpec(COUNT_STAR)],
                          prologue=[Probe(j.handle, keys, build_is_left=True)])
        res[name] = eng.fetch(out)
    assert_same_rows(res["gpu"], res["oracle"], 1, {1})


def test_string_join_probe_pairs(ctx, gpu_engine):
    from minilake_b200.gpu import HashJoinProbe
    rng = np.random.default_rng(23)
    dim = _dim(rng, 3000, True)
    g = gpu_engine.join_build(dim, [UTF8, INT32], [(Col(0), UTF8)])
    o = orc.OracleEngine(threads=1).join_build(dim, [UTF8, INT32], [(Col(0), UTF8)])
    assert g.stats()["distinct_keys"] == o.stats()["distinct_keys"]
    n = 12_000
    idx = rng.integers(0, len(POOL), n)
    for plain in (True, False):
        cols = [_string_col(rng, idx, rng.random(n) > 0.1, plain)]
        gp, gb = HashJoinProbe(ctx, g.handle, [(Col(0), UTF8)]).execute(cols)
        op, ob = orc.join_probe(o, [(Col(0), UTF8)], cols)
        # one build batch in row-group order on both sides: build rows index the same rows
        assert sorted(zip(gp.tolist(), gb.tolist())) == sorted(zip(op.tolist(), ob.tolist()))
        assert np.array_equal(gp, np.sort(gp, kind="stable")), "pairs ordered by probe row"


# MIN/MAX over strings (accumulator.rs:156-160): byte order (bytes >= 0x80 after ASCII), a
# prefix before its extensions, the empty string first; later batches bring strings the earlier
# ones did not have (the group states' ranks are renumbered); NULL inputs skipped, a group with
# only NULLs gives NULL.
MM_POOL = [b"", b"a", b"ab", b"abc", b"abd", b"b", b"\xc3\xa9t\xc3\xa9", b"zz", b"Zz", b"a\x00b", b"a\x00"] + \
          [b"s%04d" % i for i in range(400)]


def _mm_table(rng, groups, plain_first):
    rgs = []
    for g in range(groups):
        n = 6000
        hi = 60 + g * 60  # each row group reaches further into the pool: new strings arrive late
        idx = rng.integers(0, min(hi, len(MM_POOL)), n)
        valid = rng.random(n) > 0.1
        k = rng.integers(0, 50, n).astype(np.int64)
        k[k == 49] = 1000 + g  # groups seen in one row group only
        s = utf8_plain([MM_POOL[i] for i in idx], valid) if (g % 2 == 0) == plain_first \
            else encode_strings(MM_POOL, idx, valid)
        rgs.append([fixed(INT64, k), s, fixed(FLOAT64, rng.random(n))])
    only_nulls = [fixed(INT64, np.full(5, 7777, dtype=np.int64)), utf8_plain([b"x"] * 5, np.zeros(5, bool)),
                  fixed(FLOAT64, np.ones(5))]
    rgs.append(only_nulls)
    return Table("t", ["k", "s", "v"], rgs)


@pytest.mark.parametrize("plain_first", [True, False])
def test_min_max_of_strings(gpu_engine, plain_first):
    from minilake_b200.abi import MAX, MIN
    from minilake_b200.engine import GpuEngine
    rng = np.random.default_rng(31 + plain_first)
    t = _mm_table(rng, 6, plain_first)
    types = [INT64, UTF8, FLOAT64]
    aggs = [AggSpec(MIN, Col(1), UTF8), AggSpec(MAX, Col(1), UTF8), AggSpec(COUNT_STAR), AggSpec(SUM, Col(2), FLOAT64)]
    for group in ([(Col(0), INT64)], []):
        want = orc.OracleEngine(threads=1).fetch(orc.OracleEngine(threads=1).hashagg(t, types, group, aggs))
        for eng in (gpu_engine, GpuEngine(gpu_engine.ctx, threads=3)):
            got = eng.fetch(eng.hashagg(t, types, group, aggs))
            assert_same_rows(got, want, len(group), {len(group) + 3})


def test_min_max_of_strings_grouped_by_a_string(gpu_engine):
    from minilake_b200.abi import MAX, MIN
    rng = np.random.default_rng(37)
    fact = _fact(rng, 20_000, 4, 300)  # [s, v, d]
    # GROUP BY d % 7 as an int, MIN/MAX of the string; and GROUP BY the string, MIN of itself
    types = [UTF8, FLOAT64, INT32]
    for group, aggs in (([(Col(2), INT32)], [AggSpec(MIN, Col(0), UTF8), AggSpec(MAX, Col(0), UTF8)]),
                        ([(Col(0), UTF8)], [AggSpec(MIN, Col(0), UTF8), AggSpec(COUNT_STAR)])):
        want = orc.OracleEngine(threads=2).fetch(orc.OracleEngine(threads=2).hashagg(fact, types, group, aggs))
        got = gpu_engine.fetch(gpu_engine.hashagg(fact, types, group, aggs))
        assert_same_rows(got, want, 1)
