"""The test streams themselves (CPU): every shape `snappy_streams.encode` writes is a valid Snappy
stream (pyarrow's decompressor gives the input back), the shapes are the ones their names say,
and a re-compressed Parquet chunk keeps its page headers apart from the compressed size."""
import numpy as np
import pytest

import snappy_streams as ss


def _data(n=300_000, seed=3):
    rng = np.random.default_rng(seed)
    runs = np.repeat(rng.integers(0, 1 << 40, n // 800), 100).astype(np.int64).tobytes()
    rnd = rng.integers(0, 256, n // 4, dtype=np.uint8).tobytes()
    words = b"".join(rng.choice([b"alpha", b"beta", b"gamma", b"delta"], n // 20))
    return (runs + rnd + words)[:n]


def _elements(z):
    """(output start, output length, copy offset or 0) of every element."""
    n, p = ss._uvarint(z, 0)
    out, res = 0, []
    while p < len(z):
        tag = z[p]
        t = tag & 3
        if t == 0:
            ln = tag >> 2
            p += 1
            if ln >= 60:
                nb = ln - 59
                ln = int.from_bytes(z[p:p + nb], "little")
                p += nb
            ln += 1
            res.append((out, ln, 0))
            p += ln
        elif t == 1:
            res.append((out, 4 + ((tag >> 2) & 7), ((tag >> 5) << 8) | z[p + 1]))
            p += 2
        else:
            nb = 2 if t == 2 else 4
            res.append((out, (tag >> 2) + 1, int.from_bytes(z[p + 1:p + 1 + nb], "little")))
            p += 1 + nb
        out += res[-1][1]
    assert out == n
    return res


@pytest.mark.parametrize("kw", [{}, {"block": None}, {"reach": 65535, "block": 65536}, {"matches": False},
                                {"max_literal": 1000}])
def test_streams_decode_with_pyarrow(kw):
    import pyarrow as pa
    data = _data()
    z = ss.encode(data, **kw)
    assert pa.Codec("snappy").decompress(z, decompressed_size=len(data)).to_pybytes() == data


def test_the_shapes():
    data = _data()
    F = 1 << 16
    crossing = lambda els: any(s // F != (s + ln - 1) // F for s, ln, _ in els)  # noqa: E731
    reaching = lambda els: any(off and s - off < (s // F) * F for s, ln, off in els)  # noqa: E731
    aligned = _elements(ss.encode(data, reach=65535))
    assert not crossing(aligned) and reaching(aligned)
    local = _elements(ss.encode(data, reach=1 << 30, block=F))
    assert not crossing(local)
    free = _elements(ss.encode(data, block=None))
    assert crossing(free)
    one = _elements(ss.encode(data, block=None, matches=False))
    assert len(one) == 1 and crossing(one)


def test_a_recompressed_chunk_keeps_its_headers(tmp_path):
    import pyarrow as pa
    import pyarrow.parquet as pq
    from minilake_b200 import parquet
    path = str(tmp_path / "u.parquet")
    pq.write_table(pa.table({"v": np.arange(50_000, dtype=np.int64)}), path, compression="NONE",
                   use_dictionary=False, data_page_size=1 << 16)
    meta = pq.ParquetFile(path).metadata.row_group(0).column(0)
    chunk = parquet.chunk_bytes(path, meta)
    z = ss.recompress_chunk(chunk, ss.encode)
    a, b = ss.pages(chunk), ss.pages(z)
    assert len(a) == len(b) > 3
    codec = pa.Codec("snappy")
    for (ha, ta, pa_), (hb, tb, pb) in zip(a, b):
        assert ta == tb
        assert codec.decompress(pb, decompressed_size=len(pa_)).to_pybytes() == pa_
        fa, _ = ss.struct_fields(ha, 0)
        fb, _ = ss.struct_fields(hb, 0)
        assert sorted(fa) == sorted(fb)
        assert ss._zigzag32(hb, fb[2]) == len(pa_) and ss._zigzag32(hb, fb[3]) == len(pb)
