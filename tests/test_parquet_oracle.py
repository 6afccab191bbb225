"""The Parquet page oracle against the reference's own decoding tests
(RleBitPackingReaderTest, ParquetPageDecoderTest), regenerated by
tests/golden/parquet_cases.py: every stream those tests decode, with the
values they assert. CPU only."""
import struct

import numpy as np
import pytest

from oracle import pyoracle as O
from tests.golden import parquet_cases as PC
from vecruntime_b200 import native as N

RLE = list(PC.rle_cases())


def test_case_families_complete():
    names = [c[0] for c in RLE]
    assert len(names) == len(set(names))
    # 1 + 32*8*2 + 3 + 33*8 + 400 + 32*5 decodes, as in the reference's tests
    assert len(RLE) == 1 + 512 + 3 + 264 + 400 + 160


@pytest.mark.parametrize("case", range(len(RLE)), ids=[c[0] for c in RLE])
def test_rle_stream_decodes_to_the_tests_values(case):
    name, width, values, data = RLE[case]
    got = O.rle_decode(data, width, len(values))
    np.testing.assert_array_equal(got, np.array(values, dtype=np.uint32), err_msg=name)


def test_encoder_matches_the_format_by_hand():
    # an RLE run of 10 threes at width 6: header 10 << 1 = 20, one value byte
    assert PC.encode([3] * 10, 6, False) == bytes([20, 3])
    # one bit-packed group of 0..7 at width 3: header (1 << 1) | 1 = 3, then
    # 24 bits LSB first: 0b_111_110_101_100_011_010_001_000
    assert PC.encode(list(range(8)), 3, True) == bytes([3]) + (0b111110101100011010001000).to_bytes(3, "little")
    # ULEB128 header of a 300-value RLE run: 600 = 0x258 -> 0xD8 0x04
    assert PC.encode([1] * 300, 1, False) == bytes([0xD8, 0x04, 1])


PAGES = list(PC.page_cases())


@pytest.mark.parametrize("case", range(len(PAGES)), ids=[c[0] for c in PAGES])
def test_page_decodes_to_the_tests_values(case):
    name, data, fields, want, present = PAGES[case]
    out, valid, npresent = O.pq_decode_page(data, **fields)
    vb = 4 if fields["encoding"] == N.VR_PQ_RLE_DICTIONARY else fields["value_bytes"]
    dt = np.uint32 if vb == 4 else np.int64
    np.testing.assert_array_equal(out.view(dt), np.array(want, dtype=dt), err_msg=name)
    bits = np.unpackbits(valid, bitorder="little")[:len(present)].astype(bool)
    np.testing.assert_array_equal(bits, np.array(present), err_msg=name)
    assert npresent == sum(present)


def test_dictionary_page_of_strings():
    words = [b"apple", b"banana", b"cherry"]
    offs, data = O.pq_plain_dictionary(PC.plain_binary(words), 3)
    assert list(offs) == [0, 5, 11, 17]
    assert bytes(data) == b"applebananacherry"
    # an empty entry and a zero-entry page
    offs, data = O.pq_plain_dictionary(PC.plain_binary([b"", b"x"]), 2)
    assert list(offs) == [0, 0, 1] and bytes(data) == b"x"
    offs, data = O.pq_plain_dictionary(b"", 0)
    assert list(offs) == [0]


def test_malformed_streams_are_errors():
    with pytest.raises(O.OracleError, match="run header"):
        O.rle_decode(b"", 3, 1)                      # no header at all
    with pytest.raises(O.OracleError, match="bit-packed run"):
        O.rle_decode(bytes([3, 0xFF]), 3, 8)         # a group of 3 bytes cut to 1
    with pytest.raises(O.OracleError, match="run header"):
        O.rle_decode(bytes([0x80]), 3, 1)            # a header whose varint never ends
    with pytest.raises(O.OracleError, match="past the end"):
        O.pq_plain_dictionary(struct.pack("<i", 10) + b"abc", 1)
    # ten present slots, one group of 8 ids: the stream ends before the ninth
    data, ll = PC.build_page(bytes([2]) + PC.encode([1, 2], 2, False), [True] * 10, 1, False)
    with pytest.raises(O.OracleError, match="run header"):
        O.pq_decode_page(data, num_values=10, max_def_level=1, v2=0, levels_length=ll, encoding=1, value_bytes=4)


def test_writer_style_encoder_round_trips_through_the_oracle():
    from vecruntime_b200 import datagen as G

    rng = np.random.default_rng(5)
    for width in (1, 2, 7, 17, 32):
        for n in (0, 1, 8, 9, 1000, 5003):
            v = rng.integers(0, 1 << width, size=n, dtype=np.uint64).astype(np.uint32)
            v[n // 3: n // 3 + min(n // 3, 700)] = v[n // 3] if n else 0  # a long repeat -> RLE runs
            data = G.encode_hybrid(v, width)
            np.testing.assert_array_equal(O.rle_decode(data, width, n), v)
    ids = rng.integers(0, 100_000, size=20_000).astype(np.int32)
    nulls = rng.random(20_000) < 0.01
    for v2 in (False, True):
        pages = G.dictionary_pages(ids, nulls, 17, 7_000, v2=v2)
        assert len(pages) == 3
        lo = 0
        for data, f in pages:
            out, valid, npresent = O.pq_decode_page(data, **f)
            hi = lo + f["num_values"]
            want = np.where(nulls[lo:hi], 0, ids[lo:hi]).astype(np.uint32)
            np.testing.assert_array_equal(out.view(np.uint32), want)
            np.testing.assert_array_equal(np.unpackbits(valid, bitorder="little")[:hi - lo].astype(bool),
                                          ~nulls[lo:hi])
            lo = hi


def test_library_dictionary_page_matches_the_oracle():
    from vecruntime_b200 import parquet as P

    words = [b"apple", b"", b"banana", "kéy".encode(), b"x" * 300]
    page = PC.plain_binary(words)
    d = P.dictionary_page(page, len(words))
    offs, data = O.pq_plain_dictionary(page, len(words))
    np.testing.assert_array_equal(d.offsets, offs)
    assert bytes(d.data[:offs[-1]]) == bytes(data)
    from vecruntime_b200 import native as NN
    with pytest.raises(NN.VrError, match="past the end"):
        P.dictionary_page(page[:-1], len(words))


def test_threaded_page_decode_matches_page_by_page():
    """The CPU baseline's threaded decode gives every page's slots and
    validity exactly as the single-page decode does."""
    from vecruntime_b200 import datagen as G

    rng = np.random.default_rng(12)
    ids = rng.integers(0, 3000, size=50_003).astype(np.int32)
    nulls = rng.random(50_003) < 0.05
    pages = G.dictionary_pages(ids, nulls, 12, 7_001)
    out, valid, secs = O.pq_decode_pages_threads(pages, 4)
    want = np.concatenate([O.pq_decode_page(b, **f)[0] for b, f in pages])
    np.testing.assert_array_equal(out, want)
    at = 0
    for b, f in pages:
        vb = (f["num_values"] + 7) // 8
        np.testing.assert_array_equal(valid[at:at + vb], O.pq_decode_page(b, **f)[1][:vb])
        at += vb
    assert secs > 0
