"""Parquet column chunks decoded on the device (ml_gpu_parquet_decode) against the CPU
restatement of read_column_chunk and encode_strings (parquet_reader.rs:104-294) over pyarrow's
decode of the same files.  Values, NULL slots and validity are compared bit for bit (floats by
their bit patterns), string dictionaries entry by entry and code by code (first-occurrence order,
per row group), plain strings byte for byte.  The files cover Snappy and uncompressed pages, v1
and v2 data pages, dictionary and PLAIN encodings (and a dictionary that overflows into PLAIN
pages mid-chunk), many small pages, NULL-only and NULL-free columns, and every conversion."""
import ctypes as C
import datetime
import decimal

import numpy as np
import pytest

from minilake_b200 import abi
from oracle.parquet_ref import expected_column

pytestmark = pytest.mark.gpu

WORDS = ["", "a", "ab", "abc", "été", "zz", "Zz", "x" * 40]


def _table(rng, n):
    import pyarrow as pa
    valid = rng.random(n) > 0.1
    def nulls(a):
        return [x if ok else None for x, ok in zip(a, valid)]
    dt0 = datetime.date(1990, 1, 1)
    f64 = rng.normal(size=n) * 1e6
    f64[rng.random(n) < 0.02] = np.nan
    f64[rng.random(n) < 0.02] = -0.0
    f64[rng.random(n) < 0.01] = np.inf
    big = [int(x) * 10**12 + int(y) for x, y in zip(rng.integers(-10**17, 10**17, n), rng.integers(0, 10**12, n))]
    return pa.table({
        "i32": pa.array(nulls(rng.integers(-2**31, 2**31 - 1, n).tolist()), pa.int32()),
        "dt": pa.array(nulls([dt0 + datetime.timedelta(days=int(d)) for d in rng.integers(0, 20000, n)]), pa.date32()),
        "i64": pa.array(rng.integers(-2**62, 2**62, n), pa.int64()),
        "f32": pa.array(nulls(rng.normal(size=n).astype(np.float32).tolist()), pa.float32()),
        "f64": pa.array(nulls(f64.tolist()), pa.float64()),
        "b": pa.array(nulls((rng.random(n) > 0.5).tolist()), pa.bool_()),
        "lo": pa.array(nulls([WORDS[i] for i in rng.integers(0, len(WORDS), n)]), pa.string()),
        "hi": pa.array(nulls([f"v{i}-{'q' * (i % 13)}" for i in rng.integers(0, 10**9, n)]), pa.string()),
        "dec9": pa.array(nulls([decimal.Decimal(int(x)).scaleb(-2) for x in rng.integers(-10**8, 10**8, n)]),
                         pa.decimal128(9, 2)),
        "dec18": pa.array(nulls([decimal.Decimal(int(x)).scaleb(-4) for x in rng.integers(-10**17, 10**17, n)]),
                          pa.decimal128(18, 4)),
        "dec30": pa.array(nulls([decimal.Decimal(x).scaleb(-6) for x in big]), pa.decimal128(30, 6)),
        "allnull": pa.array([None] * n, pa.int64()),
    })


def _write(path, table, **kw):
    import pyarrow.parquet as pq
    pq.write_table(table, path, row_group_size=kw.pop("row_group_size", 7000), **kw)


def _check_file(ctx, path):
    import pyarrow.parquet as pq
    import torch
    from minilake_b200 import gpu, parquet
    pf = pq.ParquetFile(path)
    names = [pf.schema.column(i).name for i in range(len(pf.schema))]
    for rg in range(pf.metadata.num_row_groups):
        got = parquet.read_row_group(ctx, path, rg)
        arrow = pf.read_row_group(rg)
        for name, batch in zip(names, got):
            conv, scale = parquet.conversion(pf.schema.column(names.index(name)))
            want = expected_column(arrow.column(name), conv, scale)
            n = arrow.num_rows
            assert batch.num_rows == n
            arr, _ = batch.ml_columns()
            c = arr[0]
            if want["validity"] is None:
                assert not c.validity, (name, rg, "a validity bitmap without NULLs")
            else:
                words = np.zeros((n + 63) // 64, dtype=np.uint64)
                h = batch.fetch()[0]
                assert h.validity is not None, (name, rg)
                assert np.array_equal(h.valid_mask(), want["validity"]), (name, rg)
            if "strings" in want:
                kind = want["strings"][0]
                if kind == "dict":
                    _, entries, codes = want["strings"]
                    assert c.encoding == abi.ENC_DICT, (name, rg, "expected a dictionary column")
                    offs = np.ctypeslib.as_array(C.cast(c.dict_offsets, C.POINTER(C.c_uint32)), (c.dict_len + 1,))
                    data = C.string_at(c.dict_data, int(offs[-1])) if offs[-1] else b""
                    got_entries = [data[offs[i]:offs[i + 1]] for i in range(c.dict_len)]
                    assert got_entries == entries, (name, rg)
                    got_codes = torch.as_tensor(gpu._CudaArray(c.data, n, abi.INT32, batch), device="cuda").cpu().numpy()
                    assert np.array_equal(got_codes.view(np.uint32), codes), (name, rg)
                else:
                    assert c.encoding == abi.ENC_PLAIN, (name, rg, "expected a plain column")
                    assert batch.fetch()[0].strings() == want["strings"][1], (name, rg)
            else:
                h = batch.fetch()[0]
                g, w = h.values, want["values"]
                assert g.dtype.itemsize == w.dtype.itemsize, (name, g.dtype, w.dtype)
                assert np.array_equal(g.view(f"u{g.dtype.itemsize}"), w.view(f"u{w.dtype.itemsize}")), (name, rg)
            batch.close()


@pytest.fixture(scope="module")
def ctx():
    from minilake_b200.gpu import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("compression", ["NONE", "SNAPPY"])
@pytest.mark.parametrize("version", ["1.0", "2.0"])
def test_pages_of_every_kind(ctx, tmp_path, compression, version):
    rng = np.random.default_rng(1 + (compression == "SNAPPY") + 2 * (version == "2.0"))
    path = str(tmp_path / "t.parquet")
    _write(path, _table(rng, 20_000), compression=compression, data_page_version=version, data_page_size=8 << 10)
    _check_file(ctx, path)


def test_plain_pages_and_a_dictionary_that_overflows(ctx, tmp_path):
    rng = np.random.default_rng(7)
    t = _table(rng, 30_000)
    p1 = str(tmp_path / "plain.parquet")
    _write(p1, t, use_dictionary=False, compression="SNAPPY")
    _check_file(ctx, p1)
    p2 = str(tmp_path / "overflow.parquet")  # dictionary pages cut at 2 KB: later pages fall back to PLAIN
    _write(p2, t, dictionary_pagesize_limit=2048, data_page_size=4096, row_group_size=30_000, compression="SNAPPY")
    _check_file(ctx, p2)


def test_decimals_stored_as_integers_and_required_columns(ctx, tmp_path):
    import pyarrow as pa
    rng = np.random.default_rng(9)
    n = 12_345
    t = pa.table({
        "d9": pa.array([decimal.Decimal(int(x)).scaleb(-3) for x in rng.integers(-10**8, 10**8, n)], pa.decimal128(9, 3)),
        "d18": pa.array([decimal.Decimal(int(x)).scaleb(-7) for x in rng.integers(-10**17, 10**17, n)],
                        pa.decimal128(18, 7)),
        "req": pa.array(rng.integers(0, 100, n), pa.int64()),
        "lo": pa.array([WORDS[i] for i in rng.integers(0, 3, n)], pa.string()),
    })
    schema = pa.schema([pa.field("d9", pa.decimal128(9, 3), nullable=False), pa.field("d18", pa.decimal128(18, 7)),
                        pa.field("req", pa.int64(), nullable=False), pa.field("lo", pa.string(), nullable=False)])
    path = str(tmp_path / "dec.parquet")
    _write(path, t.cast(schema), store_decimal_as_integer=True, compression="SNAPPY", row_group_size=5000)
    import pyarrow.parquet as pq
    pf = pq.ParquetFile(path)
    assert pf.schema.column(0).physical_type == "INT32" and pf.schema.column(1).physical_type == "INT64"
    assert pf.schema.column(2).max_definition_level == 0
    _check_file(ctx, path)


def test_a_truncated_chunk_is_refused(ctx, tmp_path):
    import pyarrow.parquet as pq
    from minilake_b200 import gpu, parquet
    rng = np.random.default_rng(11)
    path = str(tmp_path / "t.parquet")
    _write(path, _table(rng, 5000), compression="SNAPPY")
    pf = pq.ParquetFile(path)
    meta = pf.metadata.row_group(0).column(0)
    chunk = parquet.chunk_bytes(path, meta)
    conv, scale = parquet.conversion(pf.schema.column(0))
    for cut in (len(chunk) - 1, len(chunk) // 2, 3):
        with pytest.raises(gpu.MiniLakeError) as ei:
            gpu.parquet_decode(ctx, chunk[:cut], parquet.PHYSICAL["INT32"], 0, conv, scale, 1,
                               pf.metadata.row_group(0).num_rows, 1)
        assert ei.value.code == abi.ERR_INVALID
    # the context is still usable
    got = parquet.read_row_group(ctx, path, 0, ["i32"])[0]
    assert got.num_rows == pf.metadata.row_group(0).num_rows


def test_filter_groupby_from_a_parquet_file(ctx, tmp_path):
    """Configuration 0 as MiniLake runs it: the seeded Parquet file's row groups decoded on the
    device are the scan's morsels; the result equals the oracle's over the same values."""
    from minilake_b200 import datagen, parquet, workloads
    from minilake_b200.engine import GpuEngine
    from oracle import orc
    from test_gpu_parity import assert_same_rows
    path = str(tmp_path / "cfg0.parquet")
    datagen.filter_groupby_parquet(path, rows=1_000_000, row_groups=8)
    morsels = parquet.read_table(ctx, path, workloads.FG_SCAN)
    assert len(morsels) == 8
    got = workloads.run_filter_groupby(GpuEngine(ctx, threads=3), [m.ml for m in morsels])
    want = workloads.run_filter_groupby(orc.OracleEngine(threads=2), datagen.filter_groupby(1_000_000, 8))
    assert_same_rows(got, want, 2, {2, 3, 4})
    # f1 / f2 came back dictionary-encoded per row group (3 and 2 values)
    arr, _ = morsels[0].batches[1].ml_columns()
    assert arr[0].encoding == abi.ENC_DICT and arr[0].dict_len == 3
    for m in morsels:
        m.close()


def test_pages_of_many_fragments(ctx, tmp_path):
    """1 MB pages (16 fragments of Snappy output each): incompressible values (64 KB literals),
    long runs (copies overlapping themselves, each depending on the one before), dictionary pages
    of 100k+ distinct doubles, and strings of random letters (short literals and copies)."""
    import pyarrow as pa
    rng = np.random.default_rng(21)
    n = 400_000
    valid = rng.random(n) > 0.05
    letters = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz", dtype=np.uint8)
    txt = [bytes(letters[rng.integers(0, 26, k)]).decode() if ok else None
           for k, ok in zip(rng.integers(0, 40, n), valid)]
    t = pa.table({
        "rnd": pa.array(rng.integers(-2**63, 2**63 - 1, n, dtype=np.int64)),
        "runs": pa.array(np.repeat(rng.integers(0, 1 << 40, n // 2000), 2000).astype(np.int64)),
        "price": pa.array(rng.integers(90_000, 10_500_000, n) / 100.0),
        "txt": pa.array(txt, pa.string()),
    })
    p1 = str(tmp_path / "plain.parquet")
    _write(p1, t, use_dictionary=False, compression="SNAPPY", data_page_size=1 << 20, row_group_size=n)
    _check_file(ctx, p1)
    p2 = str(tmp_path / "dict.parquet")
    _write(p2, t, compression="SNAPPY", data_page_size=1 << 20, row_group_size=n // 2)
    _check_file(ctx, p2)


@pytest.mark.parametrize("shape", ["compressor", "literal_only", "crossing", "reaching_back", "short_literals"])
def test_snappy_streams_of_every_shape(ctx, tmp_path, shape):
    """The same column chunk re-compressed as Snappy streams the fragment decode cannot split
    (elements crossing 64 KB boundaries, copies reaching into an earlier fragment), which the serial
    pass decodes, and ones it can: every one decodes to pyarrow's values."""
    import pyarrow as pa
    import pyarrow.parquet as pq
    import snappy_streams as ss
    from minilake_b200 import gpu, parquet
    rng = np.random.default_rng(33)
    n = 60_000
    v = np.where(rng.random(n) < 0.5, rng.integers(0, 50, n), rng.integers(0, 1 << 40, n)).astype(np.int64)
    v[10_000:20_000] = 7
    path = str(tmp_path / "u.parquet")
    pq.write_table(pa.table({"v": pa.array(v, mask=rng.random(n) < 0.1)}), path, compression="NONE",
                   use_dictionary=False, data_page_size=1 << 22)
    pf = pq.ParquetFile(path)
    meta = pf.metadata.row_group(0).column(0)
    kw = {"compressor": {}, "literal_only": {"block": None, "matches": False}, "crossing": {"block": None},
          "reaching_back": {"reach": 65535}, "short_literals": {"max_literal": 7}}[shape]
    chunk = ss.recompress_chunk(parquet.chunk_bytes(path, meta), lambda b: ss.encode(b, **kw))
    conv, scale = parquet.conversion(pf.schema.column(0))
    got = gpu.parquet_decode(ctx, chunk, parquet.PHYSICAL["INT64"], 0, conv, scale, parquet.CODECS["SNAPPY"], n, 1)
    want = expected_column(pf.read_row_group(0).column("v"), conv, scale)
    h = got.fetch()[0]
    assert np.array_equal(h.valid_mask(), want["validity"])
    assert np.array_equal(h.values.view(np.uint64), want["values"].view(np.uint64))
    got.close()


def test_a_snappy_stream_of_the_wrong_length_is_refused(ctx, tmp_path):
    import pyarrow as pa
    import pyarrow.parquet as pq
    import snappy_streams as ss
    from minilake_b200 import gpu, parquet
    n = 40_000
    path = str(tmp_path / "u.parquet")
    pq.write_table(pa.table({"v": np.arange(n, dtype=np.int64)}), path, compression="NONE", use_dictionary=False,
                   data_page_size=1 << 22)
    pf = pq.ParquetFile(path)
    chunk = parquet.chunk_bytes(path, pf.metadata.row_group(0).column(0))
    conv, scale = parquet.conversion(pf.schema.column(0))
    max_def = pf.schema.column(0).max_definition_level
    bad = [lambda b: ss.varint(len(b) + 1) + ss.encode(b)[len(ss.varint(len(b))):],   # declares a byte more
           lambda b: ss.varint(len(b)) + ss.encode(b[:-8])[len(ss.varint(len(b) - 8)):]
           + ss.copy(len(b), 8)]                                                     # a copy before the output
    for f in bad:
        with pytest.raises(gpu.MiniLakeError) as ei:
            gpu.parquet_decode(ctx, ss.recompress_chunk(chunk, f), parquet.PHYSICAL["INT64"], 0, conv, scale,
                               parquet.CODECS["SNAPPY"], n, max_def)
        assert ei.value.code == abi.ERR_INVALID
    ok = gpu.parquet_decode(ctx, ss.recompress_chunk(chunk, ss.encode), parquet.PHYSICAL["INT64"], 0, conv, scale,
                            parquet.CODECS["SNAPPY"], n, max_def)
    assert np.array_equal(ok.fetch()[0].values, np.arange(n, dtype=np.int64))
    ok.close()
