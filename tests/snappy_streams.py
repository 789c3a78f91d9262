"""Snappy streams of chosen shapes, and Parquet column chunks re-compressed with them, for the
device Snappy decode's tests.

The public Snappy format (a varint length, then literal and copy elements) allows streams that
the reference compressor never writes: elements that cross a 64 KB boundary of the output, and
copies that reach back into an earlier 64 KB fragment.  `encode` writes either kind (or the
compressor's own shape), so the tests can check that every valid stream decodes, whichever pass
decodes it.  Page headers are Thrift compact structs; `recompress_chunk` rewrites each page's
compressed size after compressing its payload."""
from __future__ import annotations

from typing import Optional


def varint(n: int) -> bytes:
    out = bytearray()
    while True:
        b = n & 0x7F
        n >>= 7
        out.append(b | (0x80 if n else 0))
        if not n:
            return bytes(out)


def literal(b: bytes) -> bytes:
    n = len(b) - 1
    if n < 60:
        return bytes([n << 2]) + b
    nb = (n.bit_length() + 7) // 8
    return bytes([(59 + nb) << 2]) + n.to_bytes(nb, "little") + b


def copy(off: int, ln: int) -> bytes:
    assert 1 <= off and 1 <= ln <= 64
    if 4 <= ln <= 11 and off < 2048:
        return bytes([1 | ((ln - 4) << 2) | ((off >> 8) << 5), off & 0xFF])
    if off < 65536:
        return bytes([2 | ((ln - 1) << 2)]) + off.to_bytes(2, "little")
    return bytes([3 | ((ln - 1) << 2)]) + off.to_bytes(4, "little")


def encode(data: bytes, block: Optional[int] = 65536, reach: int = 65535, max_literal: int = 1 << 32,
           matches: bool = True) -> bytes:
    """A greedy Snappy encoder.  block: no element crosses a multiple of `block` bytes of output
    (None: elements run across them); reach: the largest copy offset (copies may reach into an
    earlier block when reach exceeds the distance to the block start); max_literal: longer
    literals are cut; matches=False: literals only."""
    n = len(data)
    out = [varint(n)]
    table = {}
    lit_start = 0

    def flush(upto):
        s = lit_start
        while s < upto:
            e = min(upto, s + max_literal)
            if block is not None:
                e = min(e, (s // block + 1) * block)
            out.append(literal(data[s:e]))
            s = e

    i = 0
    while matches and i + 4 <= n:
        blk_end = n if block is None else min(n, (i // block + 1) * block)
        key = data[i:i + 4]
        j = table.get(key)
        table[key] = i
        if j is not None and i - j <= reach and i + 4 <= blk_end:
            ln = 4
            while i + ln < blk_end and ln < 64 and data[j + ln] == data[i + ln]:
                ln += 1
            flush(i)
            out.append(copy(i - j, ln))
            i += ln
            lit_start = i
        else:
            i += 1
    flush(n)
    return b"".join(out)


# ---- Thrift compact protocol: enough to find and rewrite a PageHeader's fields
def _uvarint(buf: bytes, p: int):
    v = shift = 0
    while True:
        b = buf[p]
        p += 1
        v |= (b & 0x7F) << shift
        shift += 7
        if b < 0x80:
            return v, p


def _skip(buf: bytes, p: int, t: int, element: bool = False) -> int:
    if t in (1, 2):  # booleans: in the field header, or one byte as a list element
        return p + 1 if element else p
    if t == 3:
        return p + 1
    if t in (4, 5, 6):
        return _uvarint(buf, p)[1]
    if t == 7:
        return p + 8
    if t == 8:
        n, p = _uvarint(buf, p)
        return p + n
    if t in (9, 10):
        h = buf[p]
        p += 1
        n, et = h >> 4, h & 15
        if n == 15:
            n, p = _uvarint(buf, p)
        for _ in range(n):
            p = _skip(buf, p, et, True)
        return p
    if t == 11:
        n, p = _uvarint(buf, p)
        if n:
            kv = buf[p]
            p += 1
            for _ in range(n):
                p = _skip(buf, p, kv >> 4, True)
                p = _skip(buf, p, kv & 15, True)
        return p
    if t == 12:
        return struct_fields(buf, p)[1]
    raise ValueError(f"thrift compact type {t}")


def struct_fields(buf: bytes, p: int):
    """{field id: (start, end, type)} of the struct at p, and the position after it."""
    spans, fid = {}, 0
    while True:
        b = buf[p]
        p += 1
        if b == 0:
            return spans, p
        t, d = b & 15, b >> 4
        if d:
            fid += d
        else:
            v, p = _uvarint(buf, p)
            fid = (v >> 1) ^ -(v & 1)
        s = p
        p = _skip(buf, p, t)
        spans[fid] = (s, p, t)


def _zigzag32(buf: bytes, span) -> int:
    v = _uvarint(buf, span[0])[0]
    return (v >> 1) ^ -(v & 1)


def pages(chunk: bytes):
    """(header bytes, page type, payload) of every page of a column chunk."""
    p, out = 0, []
    while p < len(chunk):
        spans, hend = struct_fields(chunk, p)
        size = _zigzag32(chunk, spans[3])
        out.append((chunk[p:hend], _zigzag32(chunk, spans[1]), chunk[hend:hend + size]))
        p = hend + size
    return out


def recompress_chunk(chunk: bytes, compress) -> bytes:
    """An uncompressed chunk of v1 data pages (and a dictionary page) with every payload replaced
    by compress(payload) and each header's compressed_page_size (field 3) rewritten."""
    out = []
    for header, ptype, payload in pages(chunk):
        assert ptype in (0, 2), "v1 data pages and dictionary pages only"
        z = compress(payload)
        spans, _ = struct_fields(header, 0)
        s, e, _ = spans[3]
        n = len(z)
        out.append(header[:s] + varint((n << 1) ^ (n >> 31)) + header[e:] + z)
    return b"".join(out)
