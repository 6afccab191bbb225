"""GPU Parquet page decoding (vr_pq_*) against the oracle: the reference's
own decoding tests (RleBitPackingReaderTest, ParquetPageDecoderTest) through
the device decoder, seeded random column chunks (v1 and v2 pages, nulls,
every bit width, long RLE runs), malformed pages, and the decoded column fed
straight into the aggregate as a batch-dictionary key."""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests.golden import parquet_cases as PC
from vecruntime_b200 import native as N

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def device_pages(pages):
    """[(bytes, fields)] -> (keep-alive tensor, [parquet.Page]) with every
    page's bytes in one device buffer."""
    from vecruntime_b200 import parquet as P

    blob = b"".join(b for b, _ in pages) + b"\0" * 16
    t = torch.frombuffer(bytearray(blob), dtype=torch.uint8).to("cuda")
    out, at = [], 0
    for b, f in pages:
        out.append(P.Page(t.data_ptr() + at, len(b), f["num_values"], f["max_def_level"], bool(f["v2"]),
                          f["levels_length"], f["encoding"], f["value_bytes"]))
        at += len(b)
    return t, out


def oracle_column(pages):
    datas, valids = [], []
    present = 0
    for b, f in pages:
        out, valid, npres = O.pq_decode_page(b, **f)
        datas.append(out)
        valids.append(np.unpackbits(valid, bitorder="little")[:f["num_values"]].astype(bool))
        present += npres
    return np.concatenate(datas) if datas else np.zeros(0, np.uint8), \
        np.concatenate(valids) if valids else np.zeros(0, bool), present


def gpu_column(pages, decoder=None):
    from vecruntime_b200 import parquet as P

    keep, dpages = device_pages(pages)
    n = sum(f["num_values"] for _, f in pages)
    vb = 4 if pages[0][1]["encoding"] == N.VR_PQ_RLE_DICTIONARY else pages[0][1]["value_bytes"]
    dec = decoder or P.PageDecoder(max(n, 1), len(keep), device=0)
    try:
        data, valid, present = dec.decode_to_tensors(dpages)
    finally:
        if decoder is None:
            dec.close()
    d = data.cpu().numpy()[:n * vb]
    v = np.unpackbits(valid.cpu().numpy(), bitorder="little")[:n].astype(bool) if valid is not None \
        else np.ones(n, bool)
    return d, v, present


def check_same(pages, decoder=None):
    want_d, want_v, want_p = oracle_column(pages)
    got_d, got_v, got_p = gpu_column(pages, decoder)
    np.testing.assert_array_equal(got_v, want_v)
    np.testing.assert_array_equal(got_d, want_d)
    assert got_p == want_p


def test_reference_rle_cases_as_one_chunk():
    """Every stream of RleBitPackingReaderTest, each as a dictionary page
    without levels (its values are the page's ids), all in one call."""
    pages = []
    for name, width, values, data in PC.rle_cases():
        pages.append((bytes([width]) + data, dict(num_values=len(values), max_def_level=0, v2=0, levels_length=0,
                                                  encoding=1, value_bytes=4)))
    got_d, got_v, present = gpu_column(pages)
    want = np.concatenate([np.array(v, np.uint32) for _, _, v, _ in PC.rle_cases()])
    np.testing.assert_array_equal(got_d.view(np.uint32), want)
    assert got_v.all() and present == len(want)


@pytest.mark.parametrize("case", [c[0] for c in PC.page_cases()])
def test_reference_page_cases(case):
    name, data, fields, want, present = next(c for c in PC.page_cases() if c[0] == case)
    pages = [(data, fields)]
    check_same(pages)
    got_d, got_v, _ = gpu_column(pages)
    dt = np.uint32 if (fields["encoding"] == 1 or fields["value_bytes"] == 4) else np.int64
    np.testing.assert_array_equal(got_d.view(dt), np.array(want, dtype=dt))
    np.testing.assert_array_equal(got_v, np.array(present))


@pytest.mark.parametrize("v2", [False, True])
@pytest.mark.parametrize("width", [1, 3, 8, 13, 17, 24, 32])
def test_random_dictionary_chunks(width, v2):
    from vecruntime_b200 import datagen as G

    rng = np.random.default_rng(width * 2 + v2)
    n = 300_000
    ids = rng.integers(0, 1 << width, size=n, dtype=np.uint64).astype(np.uint32).view(np.int32)
    ids[1000:200_000] = ids[1000]  # a long run: RLE entries split across warps
    nulls = rng.random(n) < 0.03
    nulls[50_000:60_000] = True     # an all-null stretch
    for page_rows in (1000, 65_536, n):
        check_same(G.dictionary_pages(ids, nulls, width, page_rows, v2=v2))
    check_same(G.dictionary_pages(ids, None, width, 70_000))


def plain_pages(values: np.ndarray, nulls, page_rows, v2):
    from vecruntime_b200 import datagen as G

    vb = values.dtype.itemsize
    out = []
    for lo in range(0, len(values), page_rows):
        hi = min(len(values), lo + page_rows)
        present = ~nulls[lo:hi]
        vals = values[lo:hi][present].tobytes()
        lv = G.encode_hybrid(present.astype(np.uint32), 1)
        page, ll = (lv + vals, len(lv)) if v2 else (len(lv).to_bytes(4, "little") + lv + vals, 0)
        out.append((page, dict(num_values=hi - lo, max_def_level=1, v2=int(v2), levels_length=ll, encoding=0,
                               value_bytes=vb)))
    return out


@pytest.mark.parametrize("dtype", [np.int32, np.int64, np.float64])
def test_random_plain_chunks(dtype):
    rng = np.random.default_rng(11)
    n = 200_003
    values = rng.integers(-(1 << 40), 1 << 40, size=n).astype(dtype) if dtype != np.float64 else rng.standard_normal(n)
    nulls = rng.random(n) < 0.1
    for v2 in (False, True):
        check_same(plain_pages(values, nulls, 30_000, v2))


def test_definition_levels_above_one():
    """A max level of 3 (levels 0..3; a slot is present only at 3)."""
    from vecruntime_b200 import datagen as G

    rng = np.random.default_rng(3)
    n = 50_000
    levels = rng.integers(0, 4, size=n).astype(np.uint32)
    levels[:20_000] = 3
    present = levels == 3
    ids = rng.integers(0, 1000, size=int(present.sum())).astype(np.uint32)
    lv = G.encode_hybrid(levels, 2)
    page = len(lv).to_bytes(4, "little") + lv + bytes([10]) + G.encode_hybrid(ids, 10)
    check_same([(page, dict(num_values=n, max_def_level=3, v2=0, levels_length=0, encoding=1, value_bytes=4))])


def test_one_decoder_many_calls_and_growth():
    from vecruntime_b200 import datagen as G
    from vecruntime_b200 import parquet as P

    rng = np.random.default_rng(8)
    dec = P.PageDecoder(1_000_000, 8 << 20, device=0)
    try:
        for k in range(4):
            n = 1000 * (10 ** (k % 3)) + k
            ids = rng.integers(0, 5000, size=n).astype(np.int32)
            nulls = rng.random(n) < 0.2
            check_same(G.dictionary_pages(ids, nulls, 13, 333 + 700 * k), decoder=dec)
    finally:
        dec.close()


def test_malformed_pages_report_and_leave_the_context_usable():
    from vecruntime_b200 import datagen as G

    ids = np.arange(100, dtype=np.uint32) % 7
    stream = G.encode_hybrid(ids, 3)
    short = bytes([3]) + stream[:len(stream) // 2]
    bad = [(short, dict(num_values=100, max_def_level=0, v2=0, levels_length=0, encoding=1, value_bytes=4))]
    with pytest.raises(O.OracleError):
        oracle_column(bad)
    with pytest.raises(N.VrError, match="page 0: the dictionary-id stream"):
        gpu_column(bad)
    wide = [(bytes([40]) + stream, bad[0][1])]
    with pytest.raises(N.VrError, match="bit width above 32"):
        gpu_column(wide)
    lv = G.encode_hybrid(np.ones(100, np.uint32), 1)
    cut = [((len(lv) + 50).to_bytes(4, "little") + lv, dict(num_values=100, max_def_level=1, v2=0,
                                                            levels_length=0, encoding=1, value_bytes=4))]
    with pytest.raises(N.VrError, match="levels run past the end"):
        gpu_column(cut)
    check_same([(bytes([3]) + stream, bad[0][1])])  # the next good call decodes


def test_decoded_column_feeds_the_aggregate(cuda):
    """Pages -> VR_DICT32 ids with the chunk's dictionary -> count/sum per
    string key: the same groups as the oracle over the host ids."""
    import vecruntime_b200 as vr
    from vecruntime_b200 import aggregate as A
    from vecruntime_b200 import columns as Cc
    from vecruntime_b200 import datagen as G
    from vecruntime_b200 import parquet as P
    from dictkeys import canonical
    from parity import compare_arrays

    rng = np.random.default_rng(21)
    words = [f"key-{i:05d}".encode() for i in range(3000)]
    dict_ = P.dictionary_page(PC.plain_binary(words), len(words))
    n = 400_000
    ids = rng.integers(0, len(words), size=n).astype(np.int32)
    nulls = rng.random(n) < 0.02
    vals = rng.integers(-1000, 1000, size=n).astype(np.int64)
    keep, dpages = device_pages(G.dictionary_pages(ids, nulls, 12, 100_000))
    with P.PageDecoder(n, len(keep)) as dec:
        data, valid, present = dec.decode_to_tensors(dpages)
    assert present == int((~nulls).sum())
    host = Cc.HostBatch([Cc.dict_strings(ids, dict_, nulls), Cc.longs(vals)], n)
    dev_dict_batch, tensors = Cc.to_device(host, 0)  # the dictionary (and values) in device memory
    batch = Cc.DeviceBatch(n, [data.data_ptr(), dev_dict_batch.data_ptrs[1]], [valid.data_ptr(), None],
                           dictionaries=dev_dict_batch.dictionaries)
    fns = [A.CountAgg(), A.SumLongAgg(1), A.MinMaxAgg(1, True)]
    spec = A.Spec(host.columns, [0], fns)
    agg = vr.GpuHashAggregate(host.columns, [0], fns, est_groups=len(words), max_batch_rows=n)
    try:
        agg.consume(batch)
        got_n = agg.num_groups()
        got = canonical(agg.emit(), got_n, 0, agg.key_dictionary(0))
        types = agg.output_types
    finally:
        agg.close()
    o = O.Oracle(spec)
    o.update(host)
    want = canonical(o.emit(O.ORC_FP_COMPENSATED), o.num_groups(), 0, o.key_dictionary(0))
    bad, ex = compare_arrays(spec, types, got, got_n, o.output_types, want, o.num_groups())
    assert got_n == o.num_groups() and bad == 0, ex
