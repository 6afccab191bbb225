"""The reference's Parquet decoding tests regenerated: the same encoder, seeds,
draw order and page builders, so the byte streams are the ones those tests
decode, with the values they assert.

Restates (test code of the reference):
  RleBitPackingReaderTest.encode / packBits / writeUleb128 and its cases
      parquet/src/test/java/io/vecruntime/parquet/codec/RleBitPackingReaderTest.java:39-344
  ParquetPageDecoderTest page builders and fixed-width / dictionary cases
      parquet/src/test/java/io/vecruntime/parquet/codec/ParquetPageDecoderTest.java:45-250
`java.util.Random` comes from jrandom.py. Values are unsigned 32-bit here
(the reference's ints, read as their bit patterns).
"""
from __future__ import annotations

import struct
from typing import Iterator, List, Tuple

from .jrandom import JavaRandom


def _uleb(out: bytearray, v: int) -> None:
    v &= 0xFFFFFFFF
    while True:
        b = v & 0x7F
        v >>= 7
        if v:
            out.append(b | 0x80)
        else:
            out.append(b)
            return


def _mask(width: int) -> int:
    return 0xFFFFFFFF if width == 32 else (1 << width) - 1


def _pack(out: bytearray, values, start: int, count: int, padded: int, width: int) -> None:
    buf = bits = 0
    m = _mask(width)
    for j in range(padded):
        v = values[start + j] if j < count else 0
        buf |= (v & m) << bits
        bits += width
        while bits >= 8:
            out.append(buf & 0xFF)
            buf >>= 8
            bits -= 8
    if bits > 0:
        out.append(buf & 0xFF)


def encode(values: List[int], width: int, force_bit_packed: bool) -> bytes:
    """RleBitPackingReaderTest.encode: runs of 8+ equal values as RLE runs
    (unless forced), everything else in bit-packed runs of whole groups."""
    out = bytearray()
    if width == 0:
        return bytes(out)
    values = [v & 0xFFFFFFFF for v in values]
    byte_width = (width + 7) // 8
    n = len(values)
    i = 0
    while i < n:
        run = 1
        while i + run < n and values[i + run] == values[i]:
            run += 1
        if not force_bit_packed and run >= 8:
            _uleb(out, run << 1)
            for b in range(byte_width):
                out.append((values[i] >> (8 * b)) & 0xFF)
            i += run
        else:
            start, count = i, 0
            while i < n:
                rl = 1
                while i + rl < n and values[i + rl] == values[i]:
                    rl += 1
                if not force_bit_packed and rl >= 8 and count % 8 == 0:
                    break
                i += rl
                count += rl
            groups = (count + 7) // 8
            _uleb(out, (groups << 1) | 1)
            _pack(out, values, start, count, groups * 8, width)
    return bytes(out)


def _u32(x: int) -> int:
    return x & 0xFFFFFFFF


def rle_cases() -> Iterator[Tuple[str, int, List[int], bytes]]:
    """(name, bit width, values, encoded stream) for every decode the
    reference's RleBitPackingReaderTest checks."""
    yield "widthZeroAlwaysZero", 0, [0] * 100, encode([0] * 100, 0, False)
    rnd = JavaRandom(559)
    for w in range(1, 33):
        mx = _mask(w)
        for n in (1, 7, 8, 9, 63, 64, 65, 200):
            v = [_u32(rnd.nextLong() % (mx + 1)) for _ in range(n)]
            yield f"allWidthsRoundTrip w{w} n{n} packed", w, v, encode(v, w, True)
            yield f"allWidthsRoundTrip w{w} n{n} mixed", w, v, encode(v, w, False)
    v = [12345] * 1000
    yield "longRleRun", 20, v, encode(v, 20, False)
    v = [i % 4 for i in range(100)]
    yield "alternatingForcesBitPacked", 2, v, encode(v, 2, False)
    v = [3] * 10 + list(range(10, 15)) + [7] * 12
    yield "runThenPackedThenRunBoundaries", 6, v, encode(v, 6, False)
    rnd = JavaRandom(1234)
    for w in range(0, 33):
        mx = 0 if w == 0 else _mask(w)
        for n in (0, 1, 3, 8, 15, 16, 100, 257):
            v = [0 if w == 0 else _u32(rnd.nextLong() % (mx + 1)) for _ in range(n)]
            yield f"readIntsMatchesReadIntAllWidths w{w} n{n}", w, v, encode(v, w, False)
    rnd = JavaRandom(5591)
    for trial in range(400):
        n = rnd.nextInt(1200)
        v = [0] * n
        mode = trial % 3
        cur = rnd.nextInt(2)
        i = 0
        while i < n:
            run = 1 if mode == 0 else (8 + rnd.nextInt(200) if mode == 1 else 1 + rnd.nextInt(20))
            j = 0
            while j < run and i < n:
                v[i] = rnd.nextInt(2) if mode == 0 else cur
                j += 1
                i += 1
            cur ^= 1
        data = encode(v, 1, trial % 7 == 0)
        rnd.nextInt(130)  # the destination bit offset
        o = 0
        while o < n:  # the test's chunking draws, kept for the draw order
            take = min(1 + rnd.nextInt(9 if trial % 2 == 0 else 300), n - o)
            if take == 1:
                rnd.nextBoolean()
            o += take
        yield f"readBitsMatchesReadIntAtWidthOne trial {trial}", 1, v, data
    rnd = JavaRandom(99)
    for w in range(1, 33):
        mx = _mask(w)
        for n in (1, 8, 15, 100, 257):
            v = [_u32(rnd.nextLong() % (mx + 1)) for _ in range(n)]
            yield f"injectedUnpackerMatchesScalar w{w} n{n}", w, v, encode(v, w, True)


# ---------------------------------------------------------------- pages
def _level_bytes(present, max_def: int) -> bytes:
    levels = [max_def if p else 0 for p in present]
    return encode(levels, max_def.bit_length(), False)


def _plain_fixed(values, present, vb: int) -> bytes:
    fmt = "<i" if vb == 4 else "<q"
    return b"".join(struct.pack(fmt, (v if vb == 8 else ((v + 2**31) % 2**32 - 2**31))) for v, p in zip(values, present)
                    if p)


def _dict_ids(ids, present, id_width: int) -> bytes:
    live = [i for i, p in zip(ids, present) if p]
    return bytes([id_width]) + encode(live, id_width, False)


def build_page(value_bytes: bytes, present, max_def: int, v2: bool):
    """ParquetPageDecoderTest.v1Page / v2Page: (page bytes, levels_length)."""
    if v2:
        lvl = _level_bytes(present, max_def) if max_def > 0 else b""
        return lvl + value_bytes, len(lvl)
    out = b""
    if max_def > 0:
        lvl = _level_bytes(present, max_def)
        out += struct.pack("<i", len(lvl)) + lvl
    return out + value_bytes, 0


def page_cases():
    """(name, page bytes, page fields, expected slot values, expected
    validity) for the reference's fixed-width and dictionary page tests; a
    dictionary page decodes to its ids, a null slot to 0."""
    T, F = True, False
    v = [1, -2, 3, 2_000_000_000, -1]
    p = [T] * 5
    for v2 in (False, True):
        data, ll = build_page(_plain_fixed(v, p, 4), p, 0, v2)
        yield (f"plainInt32NoNulls v2={v2}", data, dict(num_values=5, max_def_level=0, v2=int(v2), levels_length=ll,
                                                        encoding=0, value_bytes=4), [_u32(x) for x in v], p)
    v = [10, 0, 30, 0, 50, 60, 0, 80]
    p = [T, F, T, F, T, T, F, T]
    for v2 in (False, True):
        data, ll = build_page(_plain_fixed(v, p, 8), p, 1, v2)
        yield (f"plainInt64WithNullsV1andV2 v2={v2}", data, dict(num_values=8, max_def_level=1, v2=int(v2),
                                                                 levels_length=ll, encoding=0, value_bytes=8),
               [x if q else 0 for x, q in zip(v, p)], p)
    p = [F] * 16
    data, ll = build_page(_plain_fixed([0] * 16, p, 8), p, 1, False)
    yield ("plainDoubleAllNull", data, dict(num_values=16, max_def_level=1, v2=0, levels_length=ll, encoding=0,
                                            value_bytes=8), [0] * 16, p)
    d = [1.5, -0.0, 3.141592653589793, 1e300, float("nan")]
    bits = [struct.unpack("<q", struct.pack("<d", x))[0] for x in d]
    p = [T] * 5
    data, ll = build_page(_plain_fixed(bits, p, 8), p, 0, True)
    yield ("plainDoubleValues", data, dict(num_values=5, max_def_level=0, v2=1, levels_length=ll, encoding=0,
                                           value_bytes=8), bits, p)
    ids = [0, 3, 1, 2, 0, 0, 2, 3]
    p = [T, T, F, T, T, F, T, T]
    vb = _dict_ids(ids, p, 2)  # idBitWidth(dict.length - 1) for a 4-entry dictionary
    for v2 in (False, True):
        data, ll = build_page(vb, p, 1, v2)
        yield (f"dictionaryInt64WithNulls v2={v2}", data, dict(num_values=8, max_def_level=1, v2=int(v2),
                                                               levels_length=ll, encoding=1, value_bytes=4),
               [i if q else 0 for i, q in zip(ids, p)], p)
    ids = [2, 0, 1, 1, 2]
    p = [T, T, T, F, T]
    vb = _dict_ids(ids, p, 2)  # a 3-entry string dictionary: idBitWidth(2) = 2
    data, ll = build_page(vb, p, 1, False)
    yield ("dictionaryStringsThenPlainSameColumn page 1", data, dict(num_values=5, max_def_level=1, v2=0,
                                                                     levels_length=ll, encoding=1, value_bytes=4),
           [i if q else 0 for i, q in zip(ids, p)], p)


def plain_binary(values) -> bytes:
    """ParquetPageDecoderTest.plainBinary with every slot present (a dictionary page)."""
    return b"".join(struct.pack("<i", len(b)) + b for b in values)
