"""GPU parity: libvrgpu (through the C ABI) against the CPU oracle on the
same seeded inputs, compared as sorted multisets of groups (tests/parity.py):
keys, counts, integer/decimal sums and min/max bit-exact; FP64 sums within
1e-12 relative of the oracle's compensated sum."""
import numpy as np
import pytest

import vecruntime_b200 as vr
from vecruntime_b200 import aggregate as A
from vecruntime_b200 import columns as Cc
from vecruntime_b200 import datagen as G
from vecruntime_b200 import native as N

from oracle.pyoracle import ORC_FP_COMPENSATED, Oracle
from parity import compare

pytestmark = pytest.mark.gpu


def run_gpu(w, batches, flags=0, tune=None, est=None, device_batches=False):
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups if est is None else est,
                              max_batch_rows=max(b.num_rows for b in batches), flags=flags, tune=tune)
    keep = []
    for b in batches:
        if device_batches:
            db, t = Cc.to_device(b)
            keep.append(t)
            agg.consume(db)
        else:
            agg.consume(b)
    n = agg.num_groups()
    out = agg.emit()
    st = agg.stats()
    types = agg.output_types
    agg.close()
    return types, out, n, st


def run_oracle(w, batches):
    o = Oracle(w.spec())
    for b in batches:
        o.update(b)
    n = o.num_groups()
    return o.output_types, o.emit(ORC_FP_COMPENSATED), n


def check(w, batches, **kw):
    gt, ga, gn, st = run_gpu(w, batches, **kw)
    ot, oa, on = run_oracle(w, batches)
    compare(w.spec(), gt, ga, gn, ot, oa, on)
    return st


def batches_of(w, size):
    return [w.batch(lo, min(w.rows, lo + size)) for lo in range(0, w.rows, size)]


@pytest.fixture(scope="module")
def plain():
    return G.plain()


def test_plain_256_batches_default(cuda, plain):
    st = check(plain, batches_of(plain, 4096))
    assert st.rows == plain.rows and st.batches == 256


@pytest.mark.parametrize("flags", [N.VR_SPEC_FORCE_GLOBAL, N.VR_SPEC_FORCE_SHARED,
                                   N.VR_SPEC_FORCE_GLOBAL | N.VR_SPEC_WARP_AGG,
                                   N.VR_SPEC_FORCE_SHARED | N.VR_SPEC_WARP_AGG, N.VR_SPEC_NO_TMA])
def test_plain_every_tier(cuda, plain, flags):
    check(plain, [plain.batch()], flags=flags)


def test_plain_device_resident(cuda, plain):
    check(plain, batches_of(plain, 1 << 18), device_batches=True)


def test_decimal_report_direct_tier(cuda):
    w = G.decimal_report(rows=300_000)
    st = check(w, [w.batch()])
    assert st.tier == 0


@pytest.mark.parametrize("how", ["no_tma", "device", "device_unaligned"])
def test_decimal_report_direct_tier_tile_paths(cuda, how):
    """Direct-tier tiles are read from the stage in shared memory when the
    producer bulk-copied them (full tiles of 16-byte aligned batches), and
    from the batch's own buffers otherwise (the last partial tile, NO_TMA,
    buffers that are not 16-byte aligned): every path against the oracle."""
    import torch

    w = G.decimal_report(rows=300_001)
    if how == "no_tma":
        check(w, [w.batch()], flags=N.VR_SPEC_NO_TMA)
        return
    if how == "device":
        check(w, [w.batch()], device_batches=True)
        return
    # every column one element past a 256-byte aligned allocation: 4- and
    # 8-byte aligned, never 16-byte aligned
    hb = w.batch()
    keep, ptrs = [], []
    for c in hb.columns:
        t = torch.empty(c.data.nbytes + c.data.itemsize, dtype=torch.uint8, device="cuda")
        t[c.data.itemsize:].copy_(torch.from_numpy(c.data.view(np.uint8)))
        keep.append(t)
        ptrs.append(t.data_ptr() + c.data.itemsize)
    db = Cc.DeviceBatch(hb.num_rows, ptrs, [None] * len(ptrs))
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=hb.num_rows)
    agg.consume(db)
    n = agg.num_groups()
    out, types, st = agg.emit(), agg.output_types, agg.stats()
    agg.close()
    assert st.tier == 0
    compare(w.spec(), types, out, n, *run_oracle(w, [hb]))


@pytest.mark.parametrize("threads,tile,ctas", [(96, 384, 3), (64, 256, 4), (160, 640, 2)])
def test_decimal_report_direct_tier_block_shapes(cuda, threads, tile, ctas):
    """A tuning choice may put up to four CTAs on an SM: each direct-tier
    block shape gives the oracle's groups."""
    t = N.TuneChoice()
    t.tier, t.threads, t.tile_rows, t.blocks_per_sm = 0, threads, tile, ctas
    w = G.decimal_report(rows=200_003)
    st = check(w, [w.batch()], tune=t)
    assert st.tier == 0 and st.tile_rows == tile and st.blocks == 148 * ctas


def test_decimal_report_hash_tier(cuda):
    w = G.decimal_report(rows=300_000)
    check(w, [w.batch()], flags=N.VR_SPEC_FORCE_SHARED)


def test_high_cardinality_small_with_growth(cuda):
    w = G.high_cardinality(rows=400_000, domain=200_000)
    # an estimate far too small: rows are deferred, the table grows, rows replay
    st = check(w, batches_of(w, 100_000), est=1000)
    assert st.rehashes >= 1


def test_high_cardinality_small_warp_agg(cuda):
    w = G.high_cardinality(rows=400_000, domain=200_000)
    check(w, [w.batch()], flags=N.VR_SPEC_WARP_AGG)


@pytest.mark.parametrize("finish", [1, 0])
def test_row_hash_matches_the_oracle(cuda, finish):
    """vr_hash_rows against the oracle's restatement of HashKernels
    (HashKernels.java:42-236): every lane, nulls mixing NULL_MARK, NaN and
    signed zeros in doubles, both limbs of DECIMAL128, plain UTF8 strings
    (mixUtf8) and dictionary strings with a null entry (mixDictionary: the
    entry's bytes are hashed, not its id)."""
    import ctypes as C

    from keycols import device_key_columns, string_values
    from oracle.pyoracle import hash_rows

    torch = cuda
    rng = np.random.default_rng(4242)
    n = 10_007
    nulls = lambda p: rng.random(n) < p
    d = rng.normal(size=n)
    d[rng.random(n) < 0.05] = np.nan
    d[rng.random(n) < 0.05] = -0.0
    d[rng.random(n) < 0.05] = 0.0
    entries = string_values(rng, 300, 0.0)
    entries[7] = None  # a null entry: its rows hash as null
    dic = Cc.dictionary(entries)
    cols = [Cc.ints(rng.integers(-2**31, 2**31, n), nulls(0.1), nullable=True),
            Cc.longs(rng.integers(-2**63, 2**63 - 1, n, dtype=np.int64), nulls(0.05), nullable=True),
            Cc.doubles(d, nulls(0.02), nullable=True),
            Cc.bools(rng.random(n) < 0.5, nulls(0.1), nullable=True),
            Cc.decimals128([int(x) * (1 << 64) + int(y) for x, y in zip(rng.integers(-2**62, 2**62, n),
                                                                        rng.integers(0, 2**63, n))],
                           38, 0, nulls(0.1), nullable=True),
            Cc.dict_strings(rng.integers(0, len(entries), n), dic, nulls(0.01), nullable=True),
            Cc.strings(string_values(rng, n, 0.05), nullable=True)]
    want = hash_rows(cols, n, finish=bool(finish))
    for with_hashes in (False, True):
        types, dev, keep = device_key_columns(torch, cols, dict_hashes=with_hashes)
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        rc = N.lib().vr_hash_rows(len(cols), types, dev, n, C.c_void_p(out.data_ptr()), finish, C.c_void_p(stream))
        assert rc == N.VR_OK, N.lib().vr_thread_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want), f"{int((got != want).sum())} of {n} hashes differ"


def test_row_hash_refuses_ids_without_strings_and_ids_outside_the_dictionary(cuda):
    """A VR_DICT32 key without its dictionary has no reference hash (the
    reference always hashes the strings); an id past the dictionary's end is
    reported, not read."""
    import ctypes as C

    from keycols import device_key_columns

    torch = cuda
    L = N.lib()
    out = torch.empty(64, dtype=torch.int32, device="cuda")
    bare = Cc.dict_ids(np.arange(64) % 5, 5)
    types, dev, keep = device_key_columns(torch, [bare])
    assert L.vr_hash_rows(1, types, dev, 64, C.c_void_p(out.data_ptr()), 1, None) == N.VR_ERR_INVALID
    assert b"dictionary" in L.vr_thread_last_error()
    past = Cc.dict_strings(np.arange(64) % 6, Cc.dictionary(["a", "b", "c", "d", "e"]))  # id 5 is past the end
    types, dev, keep = device_key_columns(torch, [past])
    assert L.vr_hash_rows(1, types, dev, 64, C.c_void_p(out.data_ptr()), 1, None) == N.VR_ERR_INVALID
    assert b"outside" in L.vr_thread_last_error()


def dictionary_workload(rows, seed, with_nulls=True):
    """Two dictionary keys (5 and 3 ids, nullable), an int64 value with nulls,
    a double, decimal columns for a fused product: the direct tier's shape
    with everything that can make a row not count."""
    rng = np.random.default_rng(seed)
    n1 = rng.random(rows) < (0.1 if with_nulls else 0)
    n2 = rng.random(rows) < (0.05 if with_nulls else 0)
    cols = [Cc.dict_ids(rng.integers(0, 5, rows), 5, n1, nullable=True),
            Cc.dict_ids(rng.integers(0, 3, rows), 3, n2, nullable=True),
            Cc.longs(rng.integers(-(1 << 40), 1 << 40, rows, dtype=np.int64), rng.random(rows) < 0.1, nullable=True),
            Cc.doubles(rng.standard_normal(rows), nullable=False),
            Cc.decimals(rng.integers(0, 10**9, rows, dtype=np.int64), 12, 2, nullable=False),
            Cc.decimals(rng.integers(0, 11, rows, dtype=np.int64), 12, 2, nullable=False)]
    fns = [A.CountAgg(), A.CountAgg(2), A.SumLongAgg(2), A.SumDoubleAgg(3), A.MinMaxAgg(2, True),
           A.MinMaxAgg(2, False), A.WideDecimalSumAgg(A.DecimalProduct([(4, 1, 0), (5, -1, 100)], precision=26), 36, 4)]
    return G.Workload("dict", cols, [0, 1], fns, 24, rows)


@pytest.mark.parametrize("rows", [1, 777, 100_003])
def test_direct_tier_with_selection_nulls_and_partial_tiles(cuda, rows):
    w = dictionary_workload(rows, 900 + rows)
    sel = Cc.pack_bits(np.random.default_rng(rows).random(rows) < 0.6)
    batches = [w.batch(0, rows, selection=sel)]
    st = check(w, batches)
    assert st.tier == 0, "expected the direct tier"


def test_direct_tier_id_outside_its_dictionary_is_an_error(cuda):
    w = dictionary_workload(5000, 5)
    w.columns[1].data[4321] = 7  # dictionary size 3
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=w.rows)
    with pytest.raises(vr.VrError) as e:
        agg.consume(w.batch())
        agg.sync()
    assert e.value.status == N.VR_ERR_INVALID
    agg.close()


@pytest.mark.parametrize("flags", [0, N.VR_SPEC_FORCE_SHARED, N.VR_SPEC_FORCE_GLOBAL])
@pytest.mark.parametrize("shape", ["shared_last_word", "zero_first_word"])
def test_two_word_keys_under_concurrent_inserts(cuda, flags, shape):
    """Composite int64 x int32 keys take two key words, claimed and published
    by one 128-bit CAS and probed with plain 16-byte reads. Every CTA meets
    the same new keys at once; keys that share their last word, or whose
    first word is zero (so a stale zero word reads like part of the key),
    drive the probe from the plain read into the CAS fallback."""
    rng = np.random.default_rng(20261204)
    n = 1 << 20
    if shape == "shared_last_word":
        k1 = rng.integers(0, 4096, size=n).astype(np.int64)
        k2 = np.full(n, 3, np.int32)
    else:
        k1 = np.where(rng.random(n) < 0.5, 0, rng.integers(-50, 50, size=n)).astype(np.int64)
        k2 = rng.integers(0, 64, size=n).astype(np.int32)
    nulls = rng.random(n) < 0.02
    v = rng.integers(-1000, 1000, size=n).astype(np.int64)
    cols = [Cc.longs(k1, nulls), Cc.ints(k2, nullable=False), Cc.longs(v, nullable=False)]
    fns = [A.CountAgg(), A.SumLongAgg(2), A.MinMaxAgg(2, True), A.MinMaxAgg(2, False)]
    groups = len(set(zip(np.where(nulls, -1 << 62, k1).tolist(), k2.tolist())))
    w = G.Workload("two_word_keys", cols, [0, 1], fns, groups, n)
    check(w, batches_of(w, n // 4), flags=flags, device_batches=True)


def test_emit_into_caller_buffers(cuda):
    """vr_agg_emit into caller-owned host buffers reused across calls (pinned
    here, as a caller with a pinned output pool would pass): the same
    groups as freshly allocated outputs, and a buffer too small for the
    range is refused before anything is written."""
    import ctypes as C

    w = G.high_cardinality(rows=200_000, domain=50_000)
    lib = N.lib()
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=w.rows)
    agg.consume(w.batch())
    n = agg.num_groups()
    fresh = agg.emit()
    bufs = []

    def pinned(a):
        p = C.c_void_p()
        assert lib.vr_host_alloc(max(a.nbytes, 16), C.byref(p)) == 0
        bufs.append(p)
        return np.ctypeslib.as_array((C.c_uint8 * a.nbytes).from_address(p.value)).view(a.dtype).reshape(a.shape)

    try:
        out = [(pinned(d), pinned(v)) for d, v in fresh]
        for _ in range(2):
            got = agg.emit(out=out)
            for (d0, v0), (d1, v1) in zip(fresh, got):
                assert np.array_equal(d0.view(np.uint8), d1.view(np.uint8))
                assert np.array_equal(v0, v1)
        half = n // 2
        part = agg.emit(0, half, out=out)
        assert np.array_equal(part[0][0][:half], fresh[0][0][:half])
        small = [(d[:1], v[:1]) for d, v in out]
        with pytest.raises(ValueError):
            agg.emit(out=small)
        compare(w.spec(), agg.output_types, fresh, n, *run_oracle(w, [w.batch()]))
    finally:
        agg.close()
        for p in bufs:
            lib.vr_host_free(p)


def test_autotuner_records_a_choice_that_meets_the_oracle(cuda):
    """vr_tune_search times every candidate shape on one device batch and
    records the fastest; vr_tune_lookup returns it, and a handle created
    with it gives the oracle's groups."""
    import ctypes as C

    w = G.plain(rows=200_017)
    db, keep = Cc.to_device(w.batch())
    sp = w.spec()
    batch = db.ctypes()
    best, rps = N.TuneChoice(), C.c_double()
    rc = N.lib().vr_tune_search(C.byref(sp.spec), C.byref(batch), 1, C.byref(best), C.byref(rps))
    assert rc == N.VR_OK and rps.value > 0
    got = N.TuneChoice()
    assert N.lib().vr_tune_lookup(C.byref(sp.spec), w.rows, C.byref(got)) == 1  # 1: a choice is recorded
    assert (got.tier, got.threads, got.tile_rows, got.smem_slots, got.blocks_per_sm) == \
        (best.tier, best.threads, best.tile_rows, best.smem_slots, best.blocks_per_sm)
    check(w, [w.batch()], tune=best)
