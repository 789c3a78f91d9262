"""CPU restatement of MiniLake's column-chunk conversions and string encoding
(crates/minilake-storage/src/parquet_reader.rs:104-294, encode_strings :176-212) over
pyarrow's decode of the same row group: the checker of ml_gpu_parquet_decode.

This is test infrastructure: only tests import it.  In the reference the pages are decoded by the
third-party `parquet` crate 60.0.0 (not vendored; absent here); here pyarrow 24 decodes the same
file, and parity at that boundary is that both give the values the generator wrote.  What the
reference adds on top is restated below: one slot per row with the type's default for NULL rows
(`spread`, :137-151), a validity bitmap only when some value is NULL (`read_all`, :129-131),
FLOAT -> f64, DECIMAL -> (unscaled as f64) / 10f64.powi(scale) (:217-262, `be_i128` :154-166),
and strings dictionary-encoded in order of first occurrence (NULL rows as "") when they hold at
most clamp(rows / 8, 1, 65,536) distinct values (:176-212)."""
from __future__ import annotations

import numpy as np

MAX_DICT = 1 << 16  # parquet_reader.rs:173


def powi(a: float, b: int) -> float:
    """10f64.powi(b): binary exponentiation (compiler-rt __powidf2, what powi lowers to)."""
    recip = b < 0
    r = 1.0
    while True:
        if b & 1:
            r *= a
        b = int(b / 2)
        if b == 0:
            break
        a *= a
    return 1.0 / r if recip else r


def be_i128(b: bytes) -> int:
    """be_i128 (parquet_reader.rs:158-168): the sign from the first byte, then the first 16 bytes
    shifted in, the shifts wrapping at 128 bits as i128 shifts do."""
    v = -1 if b and b[0] & 0x80 else 0
    for x in b[:16]:
        v = (((v << 8) | x) + (1 << 127)) % (1 << 128) - (1 << 127)
    return v


def encode_strings(rows):
    """encode_strings (parquet_reader.rs:176-212): ("dict", entries, codes) or ("plain", rows)."""
    n = len(rows)
    limit = min(max(n // 8, 1), MAX_DICT)
    index, entries, codes = {}, [], []
    for v in rows:
        c = index.get(v)
        if c is None:
            c = index[v] = len(entries)
            entries.append(v)
            if len(index) > limit:
                return "plain", list(rows)
        codes.append(c)
    return "dict", entries, np.asarray(codes, dtype=np.uint32)


def _unscaled(arr):
    """The unscaled integers of a pyarrow decimal array (16-byte little-endian two's complement)."""
    raw = np.frombuffer(arr.buffers()[1], dtype=np.uint8)[arr.offset * 16:(arr.offset + len(arr)) * 16]
    return [int.from_bytes(bytes(raw[i * 16:(i + 1) * 16]), "little", signed=True) for i in range(len(arr))]


def expected_column(arr, conv: int, scale: int) -> dict:
    """The column read_column_chunk returns for pyarrow array `arr` (one row group's column).
    conv: the Conversion code (minilake_b200.parquet.CONV_*)."""
    import pyarrow as pa
    if isinstance(arr, pa.ChunkedArray):
        arr = arr.combine_chunks()
    n = len(arr)
    valid = np.asarray(arr.is_valid().to_numpy(zero_copy_only=False), dtype=bool) if n else np.zeros(0, bool)
    out = {"validity": valid if not valid.all() else None}
    if conv == 6:  # UTF8
        vals = arr.to_pylist()
        rows = [v.encode() if isinstance(v, str) else (v if v is not None else b"") for v in vals]
        out["strings"] = encode_strings(rows)
        return out
    if conv in (7, 8, 9):  # decimals
        d = powi(10.0, scale)
        ints = _unscaled(arr)
        vals = np.array([float(x) / d if ok else 0.0 for x, ok in zip(ints, valid)], dtype=np.float64)
    elif conv == 4:  # FLOAT -> f64
        vals = np.where(valid, arr.fill_null(0).to_numpy(zero_copy_only=False).astype(np.float64), 0.0)
    else:
        np_type = {0: np.uint8, 1: np.int32, 2: np.int32, 3: np.int64, 5: np.float64}[conv]
        filled = arr.fill_null(False if conv == 0 else 0)
        if conv == 2:  # date32 -> days
            filled = filled.cast("int32")
        vals = filled.to_numpy(zero_copy_only=False).astype(np_type)
    out["values"] = vals
    return out
