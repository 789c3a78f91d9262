"""Seeded synthetic tables with the shapes of the three plain-GPU workloads.

Every table is generated with numpy's PCG64 from a fixed seed and cut into row
groups (morsels).  String columns follow MiniLake's reader: dictionary-encoded
per row group only when a row group has at most n/8 distinct values
(minilake-storage/src/parquet_reader.rs:173-212), else plain UTF8.

* filter + low-cardinality GROUP BY (seed 42): 1,000,000 rows in 8 row groups
  d i32 U[0,2557), f1 in 3 strings, f2 in 2 strings, qty f64 integer U{1..50},
  price f64 U[900,105000) in cents, disc {0.00..0.10}, tax {0.00..0.08}
* join + high-cardinality GROUP BY (seed 43): dim 1,500,000 rows (key i64 =
  permutation of 1..1.5M, g i32 U[0,5)); fact 60,000,000 rows in 128 row groups
  (fk i64 uniform over the dim keys, d i32 U[0,2557), v f64 U[900,105000))
* star join with skew (seed 44): fact 60,000,000 rows (k1 i32 Zipf(1.1) over
  150,000 keys, k2 i32 U over 10,000 keys, a i64 row index, v f64 U[0,1e5),
  w f64 U[0,0.1]); A 150,000 rows (key i32, name: 18-char distinct lowercase);
  B 10,000 rows (key i32, region i32 U[0,25)); C 25 rows (key i32, label: 25
  distinct strings)
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from . import abi
from .columns import HostColumn, Table, encode_strings, fixed

F1_VALUES = [b"A", b"N", b"R"]
F2_VALUES = [b"F", b"O"]


def _split(n: int, groups: int) -> List[Tuple[int, int]]:
    base, extra = divmod(n, groups)
    out, s = [], 0
    for g in range(groups):
        k = base + (1 if g < extra else 0)
        out.append((s, s + k))
        s += k
    return out


def _rg_table(name, names, arrays, groups, string_pools=None) -> Table:
    """arrays: list of (dtype, ndarray); for UTF8 the ndarray holds indices into
    string_pools[name]."""
    n = len(arrays[0][1])
    rgs = []
    for (a, b) in _split(n, groups):
        cols: List[HostColumn] = []
        for nm, (dt, arr) in zip(names, arrays):
            if dt == abi.UTF8:
                cols.append(encode_strings(string_pools[nm], arr[a:b]))
            else:
                cols.append(fixed(dt, arr[a:b]))
        rgs.append(cols)
    return Table(name, names, rgs)


def filter_groupby(rows: int = 1_000_000, row_groups: int = 8, seed: int = 42) -> Table:
    rng = np.random.Generator(np.random.PCG64(seed))
    d = rng.integers(0, 2557, rows, dtype=np.int32)
    f1 = rng.integers(0, 3, rows)
    f2 = rng.integers(0, 2, rows)
    qty = rng.integers(1, 51, rows).astype(np.float64)
    price = rng.integers(90_000, 10_500_000, rows) / 100.0
    disc = rng.integers(0, 11, rows) / 100.0
    tax = rng.integers(0, 9, rows) / 100.0
    names = ["d", "f1", "f2", "qty", "price", "disc", "tax"]
    arrays = [(abi.INT32, d), (abi.UTF8, f1), (abi.UTF8, f2), (abi.FLOAT64, qty),
              (abi.FLOAT64, price), (abi.FLOAT64, disc), (abi.FLOAT64, tax)]
    return _rg_table("t", names, arrays, row_groups, {"f1": F1_VALUES, "f2": F2_VALUES})


def join_groupby(fact_rows: int = 60_000_000, row_groups: int = 128,
                 dim_rows: int = 1_500_000, seed: int = 43,
                 dim_row_groups: int = 4) -> Tuple[Table, Table]:
    rng = np.random.Generator(np.random.PCG64(seed))
    key = (rng.permutation(dim_rows) + 1).astype(np.int64)
    g = rng.integers(0, 5, dim_rows, dtype=np.int32)
    dim = _rg_table("dim", ["key", "g"], [(abi.INT64, key), (abi.INT32, g)], dim_row_groups)
    fk = rng.integers(1, dim_rows + 1, fact_rows, dtype=np.int64)
    d = rng.integers(0, 2557, fact_rows, dtype=np.int32)
    v = rng.uniform(900.0, 105000.0, fact_rows)
    fact = _rg_table("fact", ["fk", "d", "v"],
                     [(abi.INT64, fk), (abi.INT32, d), (abi.FLOAT64, v)], row_groups)
    return dim, fact


def _random_words(rng, n: int, length: int) -> List[bytes]:
    out: List[bytes] = []
    seen = set()
    while len(out) < n:
        m = n - len(out)
        raw = rng.integers(97, 123, (m, length), dtype=np.uint8)
        for row in raw:
            w = row.tobytes()
            if w not in seen:
                seen.add(w)
                out.append(w)
    return out


def zipf_keys(rng, n: int, keys: int, s: float) -> np.ndarray:
    """Bounded Zipf(s) over ranks 1..keys by inverse-CDF sampling on the finite support."""
    w = np.arange(1, keys + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    u = rng.random(n)
    return (np.searchsorted(cdf, u, side="right") + 1).clip(1, keys).astype(np.int32)


def star_join(fact_rows: int = 60_000_000, row_groups: int = 128, a_rows: int = 150_000,
              b_rows: int = 10_000, c_rows: int = 25, seed: int = 44):
    rng = np.random.Generator(np.random.PCG64(seed))
    a_key = (rng.permutation(a_rows) + 1).astype(np.int32)
    names = _random_words(rng, a_rows, 18)
    A = _rg_table("a", ["key", "name"], [(abi.INT32, a_key), (abi.UTF8, np.arange(a_rows))], 1,
                  {"name": names})
    b_key = (rng.permutation(b_rows) + 1).astype(np.int32)
    region = rng.integers(0, 25, b_rows, dtype=np.int32)
    B = _rg_table("b", ["key", "region"], [(abi.INT32, b_key), (abi.INT32, region)], 1)
    labels = _random_words(rng, c_rows, 10)
    C = _rg_table("c", ["key", "label"],
                  [(abi.INT32, np.arange(c_rows, dtype=np.int32)), (abi.UTF8, np.arange(c_rows))], 1,
                  {"label": labels})
    k1 = zipf_keys(rng, fact_rows, a_rows, 1.1)
    k2 = rng.integers(1, b_rows + 1, fact_rows, dtype=np.int32)
    a = np.arange(fact_rows, dtype=np.int64)
    v = rng.uniform(0.0, 1e5, fact_rows)
    w = rng.uniform(0.0, 0.1, fact_rows)
    fact = _rg_table("fact", ["k1", "k2", "a", "v", "w"],
                     [(abi.INT32, k1), (abi.INT32, k2), (abi.INT64, a), (abi.FLOAT64, v),
                      (abi.FLOAT64, w)], row_groups)
    return fact, A, B, C


def filter_groupby_parquet(path: str, rows: int = 1_000_000, row_groups: int = 8, seed: int = 42,
                           compression: str = "snappy") -> None:
    """The filter + GROUP BY table (the same seeded values as filter_groupby) written as a Parquet
    file with `row_groups` row groups: d int32, f1 and f2 strings, qty / price / disc / tax double."""
    import pyarrow as pa
    import pyarrow.parquet as pq
    rng = np.random.Generator(np.random.PCG64(seed))
    d = rng.integers(0, 2557, rows, dtype=np.int32)
    f1 = rng.integers(0, 3, rows)
    f2 = rng.integers(0, 2, rows)
    qty = rng.integers(1, 51, rows).astype(np.float64)
    price = rng.integers(90_000, 10_500_000, rows) / 100.0
    disc = rng.integers(0, 11, rows) / 100.0
    tax = rng.integers(0, 9, rows) / 100.0
    strings = lambda pool, idx: pa.DictionaryArray.from_arrays(pa.array(idx, pa.int32()),  # noqa: E731
                                                               pa.array([s.decode() for s in pool])).cast(pa.string())
    t = pa.table({"d": d, "f1": strings(F1_VALUES, f1), "f2": strings(F2_VALUES, f2), "qty": qty, "price": price,
                  "disc": disc, "tax": tax})
    per = -(-rows // row_groups)
    pq.write_table(t, path, row_group_size=per, compression=compression)
