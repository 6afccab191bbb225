"""Known answers of the reference's row hash, pinning the oracle's
restatement on CPU. The expected values come from a second, independent
restatement below, written straight from HashKernels.java in Java's 32-bit
int arithmetic (mix32 :50-53, finish :56-63, fold :178-180, hashBytes
:183-197, mixUtf8 :199-213, mixDictionary :215-236), and are also written
out as literals, so a change to either restatement shows up here."""
import numpy as np

from oracle.pyoracle import hash_rows
from vecruntime_b200 import columns as Cc

M32 = 0xFFFFFFFF
SEED, MULT, NULL_MARK = 0x2545F491, 0x9E3779B1, 0x7F4A7C15


def mix32(h, v):
    h = ((h ^ v) * MULT) & M32
    return h ^ (h >> 15)  # >>> on an int: a logical shift of the 32-bit pattern


def finish(h):
    h ^= h >> 16
    h = (h * 0x85EBCA6B) & M32
    h ^= h >> 13
    h = (h * 0xC2B2AE35) & M32
    return h ^ (h >> 16)


def hash_bytes(b: bytes) -> int:
    h = 0x1B873593
    p = 0
    while p + 4 <= len(b):
        h = mix32(h, int.from_bytes(b[p:p + 4], "little"))
        p += 4
    tail, shift = 0, 0
    while p < len(b):
        tail |= b[p] << shift
        p += 1
        shift += 8
    return mix32(h, tail ^ len(b))


def row_hash(values, fin=True):
    """One row: each key column's 32-bit value (None = null) mixed in order."""
    h = SEED
    for v in values:
        h = mix32(h, NULL_MARK if v is None else v)
    return finish(h) if fin else h


def test_hash_bytes_known_answers():
    assert hash_bytes(b"") == 0x2D63DF64
    assert hash_bytes(b"a") == 0x82302C61
    assert hash_bytes(b"abcd") == 0xAA6AFD01
    assert hash_bytes(b"hello world") == 0xB5EBA779


def test_utf8_rows_match_the_oracle():
    vals = ["", "a", "abcd", "hello world", None, "é中ß", "x" * 13]
    col = Cc.strings(vals, nullable=True)
    got = hash_rows([col], len(vals), finish=False)
    want = [row_hash([None if v is None else hash_bytes(v.encode())], fin=False) for v in vals]
    assert [int(x) for x in got] == want
    assert int(got[0]) == 0x54CE98F9  # mix32(SEED, hashBytes(""))
    assert int(got[4]) == row_hash([None], fin=False) == 0x689F167B


def test_dictionary_rows_hash_the_entry_bytes_not_the_id():
    entries = ["R", "A", "N", None]
    d = Cc.dictionary(entries)
    ids = np.array([0, 1, 2, 3, 0], np.int32)
    got = hash_rows([Cc.dict_strings(ids, d)], len(ids), finish=True)
    want = [row_hash([None if entries[i] is None else hash_bytes(entries[i].encode())]) for i in ids]
    assert [int(x) for x in got] == want == [0x5F38A534, 0xB17DEDD6, 0x54B794A6, 0x6A2ED7D1, 0x5F38A534]
    # the same strings under another dictionary order hash the same
    d2 = Cc.dictionary(["N", "R", "A"])
    got2 = hash_rows([Cc.dict_strings(np.array([1, 2, 0], np.int32), d2)], 3, finish=True)
    assert [int(x) for x in got2] == want[:3]


def test_composite_rows_mix_every_column_in_order():
    ints = np.array([7, -1, 0], np.int32)
    longs = np.array([1 << 40, -5, 0], np.int64)
    d = Cc.dictionary(["MAIL", "SHIP"])
    cols = [Cc.ints(ints), Cc.longs(longs, [False, False, True]), Cc.dict_strings(np.array([1, 0, 1], np.int32), d)]
    got = hash_rows(cols, 3, finish=True)
    fold = lambda v: ((v & 0xFFFFFFFFFFFFFFFF) ^ ((v & 0xFFFFFFFFFFFFFFFF) >> 32)) & M32
    want = [row_hash([int(ints[i]) & M32, None if i == 2 else fold(int(longs[i])),
                      hash_bytes(["MAIL", "SHIP"][[1, 0, 1][i]].encode())]) for i in range(3)]
    assert [int(x) for x in got] == want
