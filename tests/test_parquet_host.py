"""The host side of the Parquet path, on the CPU: the oracle's string encoding and big-endian
decimal rule against the reference's own tests (parquet_reader.rs:364-381), the oracle's decimal
values against the bytes the file stores, the Conversion mapping (parquet_reader.rs:58-80) and the
column-chunk bytes handed to the device."""
import datetime
import decimal

import numpy as np

import snappy_streams as ss
from oracle.parquet_ref import _unscaled, be_i128, encode_strings, expected_column


def test_encode_strings_known_answers():
    """dictionary_encoding_kicks_in (parquet_reader.rs:372-381)."""
    kind, entries, codes = encode_strings([b"A" if i % 2 == 0 else b"B" for i in range(1000)])
    assert kind == "dict" and entries == [b"A", b"B"]
    assert np.array_equal(codes, np.arange(1000, dtype=np.uint32) % 2)
    uniq = [f"v{i}".encode() for i in range(100)]
    assert encode_strings(uniq) == ("plain", uniq)
    # the limit itself: rows / 8 distinct values stay a dictionary, one more does not
    rows = [str(i % 12).encode() for i in range(96)]
    assert encode_strings(rows)[0] == "dict"
    assert encode_strings(rows[:95] + [b"x"])[0] == "plain"


def test_be_i128_known_answers():
    """decimal_bytes (parquet_reader.rs:364-370), and the 16-byte cut and wrap."""
    assert be_i128(bytes([0x01, 0x00])) == 256
    assert be_i128(bytes([0xFF, 0xFF])) == -1
    assert be_i128(bytes([0xFF, 0x00])) == -256
    assert be_i128(b"") == 0
    assert be_i128(bytes([0x80] + [0] * 15)) == -(1 << 127)
    # only the first 16 bytes are shifted in
    assert be_i128(bytes([0x00] + [0xFF] * 16)) == (1 << 120) - 1
    assert be_i128(bytes([0xFF] * 17 + [0x00])) == -1


def _write(path, table, **kw):
    import pyarrow.parquet as pq
    pq.write_table(table, path, compression="NONE", use_dictionary=False, data_page_size=1 << 24, **kw)


def test_decimal_values_match_the_stored_bytes(tmp_path):
    """The oracle's decimals (pyarrow's unscaled integers) are what be_i128 gives for the bytes the
    file stores (FIXED_LEN_BYTE_ARRAY, big-endian): the two paths agree on the same file."""
    import pyarrow as pa
    import pyarrow.parquet as pq
    from minilake_b200 import parquet
    rng = np.random.default_rng(5)
    n = 3000
    big = [int(x) * 10**12 + int(y) for x, y in zip(rng.integers(-10**17, 10**17, n), rng.integers(0, 10**12, n))]
    valid = rng.random(n) > 0.2
    arr = pa.array([decimal.Decimal(v).scaleb(-6) if ok else None for v, ok in zip(big, valid)], pa.decimal128(30, 6))
    path = str(tmp_path / "d.parquet")
    _write(path, pa.table({"d": arr}))
    pf = pq.ParquetFile(path)
    col, meta = pf.schema.column(0), pf.metadata.row_group(0).column(0)
    assert col.physical_type == "FIXED_LEN_BYTE_ARRAY" and parquet.conversion(col) == (parquet.CONV_DECIMAL_BYTES, 6)
    (hdr, ptype, payload), = ss.pages(parquet.chunk_bytes(path, meta))
    assert ptype == 0  # one v1 data page: definition levels (4-byte length, RLE), then the values
    lv = int.from_bytes(payload[:4], "little")
    values = payload[4 + lv:]
    w = col.length
    assert len(values) == w * int(valid.sum())
    stored = [be_i128(values[i:i + w]) for i in range(0, len(values), w)]
    read = pf.read_row_group(0).column("d").combine_chunks()
    assert stored == [v for v, ok in zip(_unscaled(read), valid) if ok]
    want = expected_column(read, parquet.CONV_DECIMAL_BYTES, 6)["values"]
    assert np.array_equal(want[valid], np.array([float(v) / 1e6 for v in stored]))


def test_conversion_for_each_column_type(tmp_path):
    import pyarrow as pa
    import pyarrow.parquet as pq
    from minilake_b200 import parquet
    n = 10
    t = pa.table({
        "b": pa.array([True] * n), "i32": pa.array(np.arange(n, dtype=np.int32)),
        "dt": pa.array([datetime.date(2000, 1, 1)] * n), "i64": pa.array(np.arange(n, dtype=np.int64)),
        "f32": pa.array(np.ones(n, np.float32)), "f64": pa.array(np.ones(n)), "s": pa.array(["x"] * n),
        "d9": pa.array([decimal.Decimal("1.25")] * n, pa.decimal128(9, 2)),
        "d30": pa.array([decimal.Decimal("1.250")] * n, pa.decimal128(30, 3)),
    })
    p1 = str(tmp_path / "a.parquet")
    _write(p1, t)
    sch = pq.ParquetFile(p1).schema
    got = {sch.column(i).name: parquet.conversion(sch.column(i)) for i in range(len(sch))}
    assert got == {"b": (parquet.CONV_BOOL, 0), "i32": (parquet.CONV_INT32, 0), "dt": (parquet.CONV_DATE, 0),
                   "i64": (parquet.CONV_INT64, 0), "f32": (parquet.CONV_FLOAT, 0), "f64": (parquet.CONV_DOUBLE, 0),
                   "s": (parquet.CONV_UTF8, 0), "d9": (parquet.CONV_DECIMAL_BYTES, 2),
                   "d30": (parquet.CONV_DECIMAL_BYTES, 3)}
    p2 = str(tmp_path / "b.parquet")
    _write(p2, t.select(["d9"]).append_column("d18", pa.array([decimal.Decimal("1.5")] * n, pa.decimal128(18, 1))),
           store_decimal_as_integer=True)
    sch = pq.ParquetFile(p2).schema
    assert parquet.conversion(sch.column(0)) == (parquet.CONV_DECIMAL_I32, 2)
    assert parquet.conversion(sch.column(1)) == (parquet.CONV_DECIMAL_I64, 1)


def test_chunk_bytes_are_the_chunks_pages(tmp_path):
    """chunk_bytes gives the device exactly the chunk's pages: the dictionary page first when the
    chunk has one, and page headers plus payloads that add up to its compressed size."""
    import pyarrow as pa
    import pyarrow.parquet as pq
    from minilake_b200 import parquet
    rng = np.random.default_rng(2)
    t = pa.table({"k": pa.array(rng.integers(0, 50, 40_000)), "v": pa.array(rng.normal(size=40_000))})
    path = str(tmp_path / "c.parquet")
    pq.write_table(t, path, compression="SNAPPY", data_page_size=16 << 10, row_group_size=20_000)
    pf = pq.ParquetFile(path)
    for rg in range(pf.metadata.num_row_groups):
        for ci in range(2):
            meta = pf.metadata.row_group(rg).column(ci)
            chunk = parquet.chunk_bytes(path, meta)
            assert len(chunk) == meta.total_compressed_size
            pages = ss.pages(chunk)
            assert sum(len(h) + len(p) for h, _, p in pages) == len(chunk)
            assert (pages[0][1] == 2) == bool(meta.has_dictionary_page)  # 2: DICTIONARY_PAGE
            assert all(t in (0, 2, 3) for _, t, _ in pages) and len(pages) > 1


def test_the_per_chunk_command_finds_its_chunk(monkeypatch):
    """`opbench --parquet-column price` (the command behind the per-chunk figures) builds its
    file and hands the decoder row group 0's price chunk; the device calls are stubbed."""
    from minilake_b200 import gpu, opbench, parquet
    calls = []

    class Ctx:
        def __init__(self, device):
            pass

        def close(self):
            pass

    class Batch:
        def close(self):
            pass

    monkeypatch.setattr(gpu, "Context", Ctx)
    monkeypatch.setattr(gpu, "parquet_decode", lambda ctx, *a: calls.append(a) or Batch())
    out = opbench.parquet_column_chunk("price", iters=2, log=lambda *m: None)
    assert out["rows"] == 125_000 and len(out["ms"]) == 2 and len(calls) == 2
    chunk, physical, _, conv, _, codec, rows, max_def = calls[0]
    assert len(chunk) == out["chunk_bytes"] and physical == parquet.PHYSICAL["DOUBLE"]
    assert conv == parquet.CONV_DOUBLE and codec == parquet.CODECS["SNAPPY"] and rows == 125_000
    assert ss.pages(chunk)[0][1] == 2  # its dictionary page first
