"""Parquet row groups decoded on the GPU: the storage layer's Table::read_row_group
(crates/minilake-storage/src/table.rs:204-240) with read_column_chunk
(parquet_reader.rs:215-294) running on the device through ml_gpu_parquet_decode.

The file's footer is read with pyarrow, for metadata only: where each column chunk lies, its
physical and logical types, its codec and its maximum definition level (what MiniLake takes from
the parquet crate's metadata).  The chunk's pages, headers included, go to the device as stored."""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np

from . import gpu

PHYSICAL = {"BOOLEAN": 0, "INT32": 1, "INT64": 2, "FLOAT": 4, "DOUBLE": 5, "BYTE_ARRAY": 6, "FIXED_LEN_BYTE_ARRAY": 7}
CODECS = {"UNCOMPRESSED": 0, "SNAPPY": 1}
(CONV_BOOL, CONV_INT32, CONV_DATE, CONV_INT64, CONV_FLOAT, CONV_DOUBLE, CONV_UTF8, CONV_DECIMAL_I32, CONV_DECIMAL_I64,
 CONV_DECIMAL_BYTES) = range(10)


def conversion(col) -> tuple:
    """Conversion::for_column (parquet_reader.rs:58-80) of a pyarrow ColumnSchema: (conv, scale)."""
    pt, ct = col.physical_type, col.converted_type
    if pt == "BOOLEAN":
        return CONV_BOOL, 0
    if pt == "INT32":
        if ct == "DATE":
            return CONV_DATE, 0
        return (CONV_DECIMAL_I32, col.scale) if ct == "DECIMAL" else (CONV_INT32, 0)
    if pt == "INT64":
        return (CONV_DECIMAL_I64, col.scale) if ct == "DECIMAL" else (CONV_INT64, 0)
    if pt == "FLOAT":
        return CONV_FLOAT, 0
    if pt == "DOUBLE":
        return CONV_DOUBLE, 0
    if pt in ("BYTE_ARRAY", "FIXED_LEN_BYTE_ARRAY") and ct == "DECIMAL":
        return CONV_DECIMAL_BYTES, col.scale
    if pt == "BYTE_ARRAY":
        return CONV_UTF8, 0
    raise gpu.MiniLakeError(5, f"parquet column '{col.name}' has type {pt}/{ct}")


def chunk_bytes(path: str, meta) -> bytes:
    """The bytes of one column chunk (its dictionary page, if any, then its data pages)."""
    start = meta.dictionary_page_offset if meta.has_dictionary_page and meta.dictionary_page_offset else \
        meta.data_page_offset
    with open(path, "rb") as f:
        f.seek(start)
        return f.read(meta.total_compressed_size)


def read_row_group(ctx: gpu.Context, path: str, row_group: int,
                   columns: Optional[Sequence[str]] = None) -> List[gpu.DeviceBatch]:
    """Every requested column of one row group, decoded on the device: one single-column
    DeviceBatch per column, in the requested order."""
    import pyarrow.parquet as pq
    pf = pq.ParquetFile(path)
    md = pf.metadata.row_group(row_group)
    names = [pf.schema.column(i).name for i in range(len(pf.schema))]
    want = list(columns) if columns is not None else names
    out = []
    for name in want:
        ci = names.index(name)
        col = pf.schema.column(ci)
        if col.max_repetition_level:
            raise gpu.MiniLakeError(5, f"parquet column '{name}' is repeated")
        meta = md.column(ci)
        if meta.compression not in CODECS:
            raise gpu.MiniLakeError(5, f"parquet column '{name}' uses codec {meta.compression}")
        conv, scale = conversion(col)
        out.append(gpu.parquet_decode(ctx, chunk_bytes(path, meta), PHYSICAL[col.physical_type], col.length or 0, conv,
                                      scale, CODECS[meta.compression], md.num_rows, col.max_definition_level))
    return out


class Morsel:
    """One row group's decoded columns as a morsel for the sinks and operators (the MlColumn
    array they take); it keeps the single-column batches alive."""

    def __init__(self, batches: List[gpu.DeviceBatch]):
        from . import abi
        self.batches = batches
        arr = (abi.MlColumn * max(len(batches), 1))()
        for i, b in enumerate(batches):
            cols, _ = b.ml_columns()
            arr[i] = cols[0]
        self.ml = (arr, len(batches), batches[0].num_rows if batches else 0)

    def close(self):
        for b in self.batches:
            b.close()
        self.batches = []


def read_table(ctx: gpu.Context, path: str, columns: Optional[Sequence[str]] = None) -> List[Morsel]:
    """Every row group of a file decoded on the device, one morsel per row group (the scan's
    morsels, scheduler.rs:44-144)."""
    import pyarrow.parquet as pq
    n = pq.ParquetFile(path).metadata.num_row_groups
    return [Morsel(read_row_group(ctx, path, rg, columns)) for rg in range(n)]
