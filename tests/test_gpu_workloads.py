"""The three plain-GPU workloads on the B200 against the CPU oracle (reduced sizes) and,
at the full sizes, against independent numpy computations of size-independent facts
(group counts, totals, the top-N ranking).  Float64 sums: 1e-12 relative."""
import math

import numpy as np
import pytest

from helpers import rel_err
from minilake_b200 import datagen, workloads
from oracle import orc

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def engine():
    from minilake_b200.engine import GpuEngine
    from minilake_b200.gpu import Context
    ctx = Context(0)
    yield GpuEngine(ctx)
    ctx.close()


def test_filter_groupby_matches_oracle(engine):
    t = datagen.filter_groupby(rows=1_000_000, row_groups=8)
    got = workloads.run_filter_groupby(engine, t)
    want = workloads.run_filter_groupby(orc.OracleEngine(threads=8), t)
    assert got[0].strings() == want[0].strings() and got[1].strings() == want[1].strings()
    assert np.array_equal(got[5].values, want[5].values)  # COUNT(*)
    assert np.array_equal(got[2].values, want[2].values)  # SUM(qty): integer-valued, exact
    for k in (3, 4):
        assert rel_err(got[k].values, want[k].values).max() <= TOL
    # both engines against exactly rounded sums (math.fsum) per group
    rgs = t.row_groups
    d = np.concatenate([rg[0].values for rg in rgs])
    f1 = np.concatenate([np.array(rg[1].strings()) for rg in rgs])
    f2 = np.concatenate([np.array(rg[2].strings()) for rg in rgs])
    price = np.concatenate([rg[4].values for rg in rgs])
    disc = np.concatenate([rg[5].values for rg in rgs])
    m = d <= 2467
    for i, (a, b) in enumerate(zip(got[0].strings(), got[1].strings())):
        sel = m & (f1 == a) & (f2 == b)
        exact = math.fsum(price[sel] * (1.0 - disc[sel]))
        assert abs(got[3].values[i] - exact) <= TOL * exact
        assert abs(want[3].values[i] - exact) <= TOL * exact


def test_join_groupby_matches_oracle_reduced(engine):
    dim, fact = datagen.join_groupby(fact_rows=4_000_000, row_groups=16, dim_rows=100_000)
    got = workloads.run_join_groupby(engine, dim, fact)
    want = workloads.run_join_groupby(orc.OracleEngine(threads=8), dim, fact)
    assert np.array_equal(got[0].values, want[0].values)
    assert np.array_equal(got[2].values, want[2].values)
    assert rel_err(got[1].values, want[1].values).max() <= TOL


def test_join_groupby_full_size(engine):
    dim, fact = datagen.join_groupby()
    got = workloads.run_join_groupby(engine, dim, fact)
    fk = np.concatenate([rg[0].values for rg in fact.row_groups])
    d = np.concatenate([rg[1].values for rg in fact.row_groups])
    v = np.concatenate([rg[2].values for rg in fact.row_groups])
    m = d > 1200
    sums = np.bincount(fk[m], weights=v[m], minlength=1_500_001)
    counts = np.bincount(fk[m], minlength=1_500_001)
    order = np.lexsort((np.arange(len(sums)), -sums))[:11]
    gaps = -np.diff(sums[order])
    assert gaps[:10].min() > 1e-6 * sums[order[0]], "top-11 sums too close to rank bit-exactly"
    assert list(got[0].values) == list(order[:10])
    assert list(got[2].values) == list(counts[order[:10]])
    assert rel_err(got[1].values, sums[order[:10]]).max() <= 1e-11  # bincount's own order differs


def test_star_join_matches_oracle(engine):
    fact, A, B, C = datagen.star_join(fact_rows=6_000_000, row_groups=12)
    got = workloads.run_star_join(engine, fact, A, B, C)
    want = workloads.run_star_join(orc.OracleEngine(threads=8), fact, A, B, C)
    assert got[0].strings() == want[0].strings()
    assert rel_err(got[1].values, want[1].values).max() <= TOL


def test_star_join_full_size_totals(engine):
    fact, A, B, C = datagen.star_join()
    got = workloads.run_star_join(engine, fact, A, B, C)
    names = A.row_groups[0][1].strings()
    akeys = A.row_groups[0][0].values
    keep = np.zeros(150_001, dtype=bool)
    keep[akeys[[n.startswith(b"ab") for n in names]]] = True
    bregion = np.zeros(10_001, dtype=np.int64)
    bregion[B.row_groups[0][0].values] = B.row_groups[0][1].values
    labels = C.row_groups[0][1].strings()
    k1 = np.concatenate([rg[0].values for rg in fact.row_groups])
    k2 = np.concatenate([rg[1].values for rg in fact.row_groups])
    v = np.concatenate([rg[3].values for rg in fact.row_groups])
    w = np.concatenate([rg[4].values for rg in fact.row_groups])
    m = keep[k1]
    reg = bregion[k2[m]]
    val = v[m] * (1.0 - w[m])
    exp = {labels[r]: math.fsum(val[reg == r]) for r in np.unique(reg)}
    assert sorted(got[0].strings()) == sorted(exp)
    for lab, s in zip(got[0].strings(), got[1].values):
        assert abs(s - exp[lab]) <= TOL * abs(exp[lab])
    assert list(got[1].values) == sorted(got[1].values, reverse=True)
