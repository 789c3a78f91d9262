"""Host-side columns and tables in MiniLake's layout (crates/minilake-core).

* fixed width: numpy values (bool as u8, i32, i64, f64, date as i32)
* UTF8 plain: u32 offsets (n+1) + bytes (``StringVec``, column.rs:14-22)
* UTF8 dict: u32 codes + dictionary offsets/bytes (``DictVec``, column.rs:126-131)
* validity: optional u64 words, bit i = row i valid, LSB first (bitmap.rs:1-12)

A table is a list of row groups; one row group is one morsel
(operators/scan.rs:1-56).  Dictionaries are per row group, in first-occurrence
order, and only when the row group has few distinct strings
(minilake-storage/src/parquet_reader.rs:173-212).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import abi

MAX_DICT = 1 << 16  # parquet_reader.rs:173


@dataclass
class HostColumn:
    dtype: int
    values: np.ndarray                 # fixed width values / dict codes (u32) / utf8 bytes (u8)
    offsets: Optional[np.ndarray] = None       # utf8 plain
    validity: Optional[np.ndarray] = None      # u64 words
    dict_offsets: Optional[np.ndarray] = None  # utf8 dict
    dict_bytes: Optional[np.ndarray] = None

    @property
    def is_dict(self) -> bool:
        return self.dict_offsets is not None

    def __len__(self) -> int:
        if self.dtype == abi.UTF8 and not self.is_dict:
            return len(self.offsets) - 1
        return len(self.values)

    def nbytes(self) -> int:
        n = self.values.nbytes
        if self.offsets is not None:
            n += self.offsets.nbytes
        if self.validity is not None:
            n += self.validity.nbytes
        return n

    def valid_mask(self) -> np.ndarray:
        n = len(self)
        if self.validity is None:
            return np.ones(n, dtype=bool)
        bits = np.unpackbits(self.validity.view(np.uint8), bitorder="little")[:n]
        return bits.astype(bool)

    def strings(self) -> List[bytes]:
        if self.is_dict:
            d = [bytes(self.dict_bytes[self.dict_offsets[i]:self.dict_offsets[i + 1]])
                 for i in range(len(self.dict_offsets) - 1)]
            return [d[c] for c in self.values]
        o = self.offsets
        b = self.values.tobytes()
        return [b[o[i]:o[i + 1]] for i in range(len(o) - 1)]

    def to_ml(self, location: int = abi.LOC_HOST) -> abi.MlColumn:
        m = abi.MlColumn()
        m.dtype = self.dtype
        m.location = location
        m.len = len(self)
        m.data = self.values.ctypes.data if self.values.size else _EMPTY.ctypes.data
        if self.dtype == abi.UTF8 and not self.is_dict:
            m.encoding = abi.ENC_PLAIN
            m.offsets = self.offsets.ctypes.data
        elif self.is_dict:
            m.encoding = abi.ENC_DICT
            m.dict_len = len(self.dict_offsets) - 1
            m.dict_offsets = self.dict_offsets.ctypes.data
            m.dict_data = (self.dict_bytes.ctypes.data if self.dict_bytes.size else _EMPTY.ctypes.data)
        if self.validity is not None:
            m.validity = self.validity.ctypes.data
        return m


_EMPTY = np.zeros(16, dtype=np.uint8)


def validity_words(mask: np.ndarray) -> np.ndarray:
    """Pack a bool mask into LSB-first u64 words."""
    n = len(mask)
    nw = (n + 63) // 64
    b = np.packbits(np.asarray(mask, dtype=np.uint8), bitorder="little")
    out = np.zeros(nw * 8, dtype=np.uint8)
    out[:len(b)] = b
    return out.view(np.uint64)


def fixed(dtype: int, values, valid: Optional[np.ndarray] = None) -> HostColumn:
    v = np.ascontiguousarray(np.asarray(values, dtype=abi.NP_DTYPE[dtype]))
    return HostColumn(dtype, v, validity=None if valid is None else validity_words(valid))


def utf8_plain(strings: Sequence[bytes], valid: Optional[np.ndarray] = None) -> HostColumn:
    lens = np.fromiter((len(s) for s in strings), dtype=np.int64, count=len(strings))
    off = np.zeros(len(strings) + 1, dtype=np.uint32)
    np.cumsum(lens, out=off[1:])
    data = np.frombuffer(b"".join(strings), dtype=np.uint8).copy()
    return HostColumn(abi.UTF8, data, offsets=off,
                      validity=None if valid is None else validity_words(valid))


def utf8_dict(dictionary: Sequence[bytes], codes: np.ndarray,
              valid: Optional[np.ndarray] = None) -> HostColumn:
    d = utf8_plain(dictionary)
    return HostColumn(abi.UTF8, np.ascontiguousarray(codes, dtype=np.uint32),
                      validity=None if valid is None else validity_words(valid),
                      dict_offsets=d.offsets, dict_bytes=d.values)


def encode_strings(pool: Sequence[bytes], idx: np.ndarray,
                   valid: Optional[np.ndarray] = None) -> HostColumn:
    """Row-group string column whose row i is pool[idx[i]]: dictionary-encoded (first
    occurrence order) when distinct <= clamp(n/8, 1, 65536), else plain
    (parquet_reader.rs:176-212)."""
    n = len(idx)
    limit = min(max(n // 8, 1), MAX_DICT)
    uniq, first = np.unique(idx, return_index=True)
    if len(uniq) <= limit:
        order = np.argsort(first, kind="stable")
        ordered = uniq[order]
        remap = np.empty(int(idx.max()) + 1 if n else 1, dtype=np.uint32)
        remap[ordered] = np.arange(len(ordered), dtype=np.uint32)
        return utf8_dict([pool[i] for i in ordered], remap[idx] if n else np.zeros(0, np.uint32),
                         valid)
    return utf8_plain([pool[i] for i in idx], valid)


class Table:
    """Row groups of host columns; morsel i = row group i."""

    def __init__(self, name: str, names: Sequence[str], row_groups: List[List[HostColumn]]):
        self.name = name
        self.names = list(names)
        self.row_groups = row_groups

    @property
    def num_rows(self) -> int:
        return sum(len(rg[0]) for rg in self.row_groups)

    @property
    def types(self) -> List[int]:
        return [c.dtype for c in self.row_groups[0]]

    def col_index(self, name: str) -> int:
        return self.names.index(name)

    def project(self, names: Sequence[str]) -> "Table":
        """Projection pushdown: only these columns are read (scan.rs:16-17)."""
        idx = [self.col_index(n) for n in names]
        return Table(self.name, names, [[rg[i] for i in idx] for rg in self.row_groups])

    def morsels(self, keep: abi.Keep):
        """Flat ml_column array [morsel][col] + row counts, for the sinks' drivers."""
        nm, nc = len(self.row_groups), len(self.names)
        arr = keep.add((abi.MlColumn * max(nm * nc, 1))())
        rows = keep.add(np.array([len(rg[0]) for rg in self.row_groups], dtype=np.int64))
        for m, rg in enumerate(self.row_groups):
            for c, col in enumerate(rg):
                arr[m * nc + c] = col.to_ml()
        return arr, nm, nc, rows

    def nbytes(self) -> int:
        return sum(c.nbytes() for rg in self.row_groups for c in rg)
