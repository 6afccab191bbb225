"""GPU parity on Spark's null and overflow rules and on the final-mode merges,
against the oracle (tests/parity.py comparison; for error cases the same
status from both):

  * ANSI bigint sum overflow -> VR_ERR_OVERFLOW; non-ANSI sums wrap exactly
    (SumLongAgg, VectorAggregates.scala:142-200)
  * decimal sums past their buffer precision: null, or VR_ERR_DECIMAL_PRECISION
    for a final ANSI result (WideDecimalSumAgg, VectorAggregates.scala:318-395)
  * fused decimal products: 128-bit products, null factors, products past
    their precision (null, or an error with ANSI) -- every row that leaves
    the int64 fast path (SpeculativeDecimalMulExpr, DecimalExprs.scala:470-516)
  * final-mode merges of partial buffers: CountMergeAgg, AverageMergeAgg,
    WideDecimalSumMergeAgg (isEmpty, null sums, overflow), WideDecimalAvgMergeAgg
    (VectorAggregates.scala:526-781, 1042-1090)
each in the hash tier (int64 key) and, where the keys allow, the direct tier."""
import numpy as np
import pytest

import vecruntime_b200 as vr
from vecruntime_b200 import aggregate as A
from vecruntime_b200 import columns as Cc
from vecruntime_b200 import datagen as G
from vecruntime_b200 import native as N

from oracle.pyoracle import ORC_FP_COMPENSATED, Oracle, OracleError
from parity import compare

pytestmark = pytest.mark.gpu


def gpu_result(w, batches, flags=0):
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups,
                              max_batch_rows=max(b.num_rows for b in batches), flags=flags)
    try:
        for b in batches:
            agg.consume(b)
        n = agg.num_groups()
        return ("ok", agg.output_types, agg.emit(), n)
    except vr.VrError as e:
        return ("err", e.status)
    finally:
        agg.close()


def oracle_result(w, batches):
    o = Oracle(w.spec())
    try:
        for b in batches:
            o.update(b)
        return ("ok", o.output_types, o.emit(ORC_FP_COMPENSATED), o.num_groups())
    except OracleError as e:
        return ("err", e.status)


def same(w, batches, flags=0):
    got, want = gpu_result(w, batches, flags), oracle_result(w, batches)
    assert got[0] == want[0], f"gpu {got[:2]} vs oracle {want[:2]}"
    if got[0] == "err":
        assert got[1] == want[1], f"status {got[1]} vs oracle {want[1]}"
        return got[1]
    compare(w.spec(), got[1], got[2], got[3], want[1], want[2], want[3])
    return N.VR_OK


def keys(rng, rows, card, direct):
    if direct:
        return Cc.dict_ids(rng.integers(0, card, rows), card, nullable=False)
    dom = rng.integers(-(1 << 62), 1 << 62, card, dtype=np.int64)
    return Cc.longs(dom[rng.integers(0, card, rows)], nullable=False)


@pytest.mark.parametrize("checked", [False, True])
def test_bigint_sum_overflow(cuda, checked):
    rng = np.random.default_rng(1)
    rows = 4096
    v = np.full(rows, (1 << 62) - 7, np.int64)
    v[::2] *= -1
    v[:3] = (1 << 62)  # the first group (id 0) drifts past 2^63
    k = np.arange(rows) % 64
    k[:40] = 0
    cols = [Cc.longs(k, nullable=False), Cc.longs(v, nullable=False)]
    w = G.Workload("ovf", cols, [0], [A.SumLongAgg(1, checked=checked), A.CountAgg()], 64, rows)
    status = same(w, [w.batch()])
    assert status == (N.VR_ERR_OVERFLOW if checked else N.VR_OK)


@pytest.mark.parametrize("direct", [False, True])
@pytest.mark.parametrize("final,null_on_overflow", [(False, True), (True, True), (True, False)])
def test_decimal_sum_past_its_precision(cuda, direct, final, null_on_overflow):
    rng = np.random.default_rng(2)
    rows = 5000
    v = rng.integers(10**16, 10**17, rows, dtype=np.int64)  # DECIMAL(18, 0): only the big group passes 10^20
    k = keys(rng, rows, 8, direct)
    k.data[: rows // 2] = k.data[0]  # one group sums ~2,500 values: past 10^20
    cols = [k, Cc.decimals(v, 18, 0, rng.random(rows) < 0.02, nullable=True)]
    fns = [A.WideDecimalSumAgg(1, 20, 0, final_result=final, null_on_overflow=null_on_overflow), A.CountAgg(1)]
    w = G.Workload("decprec", cols, [0], fns, 8, rows)
    status = same(w, [w.batch()])
    assert status == (N.VR_ERR_DECIMAL_PRECISION if final and not null_on_overflow else N.VR_OK)


@pytest.mark.parametrize("direct", [False, True])
@pytest.mark.parametrize("checked", [False, True])
def test_decimal_products_leave_the_fast_path(cuda, direct, checked):
    """Most rows' products fit int64; some need 128 bits, some have a null
    factor, some pass the product's precision (null, or an error with ANSI)."""
    rng = np.random.default_rng(3 + direct)
    rows = 20_000
    a = rng.integers(-10**9, 10**9, rows, dtype=np.int64)
    b = rng.integers(-10**9, 10**9, rows, dtype=np.int64)
    c = rng.integers(0, 100, rows, dtype=np.int64)
    big = rng.random(rows) < 0.05
    a[big] = rng.integers(10**16, 10**17, int(big.sum()), dtype=np.int64)  # 128-bit products
    b[big] = rng.integers(10**16, 10**17, int(big.sum()), dtype=np.int64)
    huge = rng.random(rows) < (0.002 if checked else 0.01)
    a[huge] = 10**17 + 3  # with c >= 100 these pass 38 digits
    b[huge] = 10**17 + 7
    c[huge] = 10**6
    k = keys(rng, rows, 16, direct)
    na = rng.random(rows) < 0.03
    cols = [k, Cc.decimals(a, 18, 2, na, nullable=True), Cc.decimals(b, 18, 2, nullable=False),
            Cc.decimals(c, 18, 2, nullable=False)]
    prod = A.DecimalProduct([(1, 1, 0), (2, 1, 0), (3, 1, 0)], precision=38)
    fns = [A.WideDecimalSumAgg(prod, 38, 6, checked_product=checked), A.CountAgg(),
           A.WideDecimalSumAgg(A.DecimalProduct([(1, 1, 0), (2, -1, 100)], precision=38), 38, 4)]
    w = G.Workload("prod", cols, [0], fns, 16, rows)
    status = same(w, [w.batch(0, 12_000), w.batch(12_000, rows)])
    assert status == (N.VR_ERR_DECIMAL_PRECISION if checked else N.VR_OK)


@pytest.mark.parametrize("direct", [False, True])
def test_three_factor_product_reuses_the_two_factor_one(cuda, direct):
    """sum(a*(1-b)) and sum(a*(1-b)*c) over the same a, b (the decimal
    report's two product sums): the direct tier reuses the chunk's a*(1-b)
    for the three-factor sum when every row of the chunk took the 32-bit
    path. Row ranges where a*(1-b) leaves 32 bits (no reuse), where a factor
    leaves 32 bits (the 64-bit path) and where factors are null meet the
    oracle like the rest."""
    rng = np.random.default_rng(11 + direct)
    rows = 60_000
    a = rng.integers(1, 10**6, rows, dtype=np.int64)
    b = rng.integers(0, 11, rows, dtype=np.int64)
    c = rng.integers(0, 9, rows, dtype=np.int64)
    a[20_000:22_000] = rng.integers(10**8, 10**9, 2_000, dtype=np.int64)  # a*(1-b) past 32 bits
    a[30_000:30_100] = rng.integers(10**12, 10**13, 100, dtype=np.int64)  # a factor past 32 bits
    na = np.zeros(rows, bool)
    na[40_000:41_000] = rng.random(1_000) < 0.5
    k = keys(rng, rows, 16, direct)
    cols = [k, Cc.decimals(a, 18, 2, na, nullable=True), Cc.decimals(b, 18, 2, nullable=False),
            Cc.decimals(c, 18, 2, nullable=False)]
    two = A.DecimalProduct([(1, 1, 0), (2, -1, 100)], precision=38)
    three = A.DecimalProduct([(1, 1, 0), (2, -1, 100), (3, 1, 100)], precision=38)
    fns = [A.WideDecimalSumAgg(two, 38, 4), A.WideDecimalSumAgg(three, 38, 6), A.CountAgg()]
    w = G.Workload("prefix", cols, [0], fns, 16, rows)
    assert same(w, [w.batch(0, 45_000), w.batch(45_000, rows)]) == N.VR_OK


def merge_inputs(rng, rows, card, overflow=False):
    """Partial-aggregation buffers as a final aggregate receives them."""
    k = keys(rng, rows, card, False)
    cnt = rng.integers(0, 1000, rows, dtype=np.int64)
    dsum = rng.standard_normal(rows) * 1e3
    dcnt = rng.integers(0, 50, rows, dtype=np.int64)
    # overflow: positive sums of ~2,000 values near 10^36 each pass 10^38
    decsum = ([int(x) * 10**36 // 1000 for x in rng.integers(0, 1000, rows)] if overflow else
              [int(x) * 10**25 // 1000 for x in rng.integers(-1000, 1000, rows)])
    empty = rng.random(rows) < 0.2
    empty_null = rng.random(rows) < 0.05
    sum_null = rng.random(rows) < 0.05
    avgsum = [int(x) * 10**20 for x in rng.integers(-1000, 1000, rows)]
    avgcnt = rng.integers(0, 100, rows, dtype=np.int64)
    cols = [k, Cc.longs(cnt, nullable=False), Cc.doubles(dsum, rng.random(rows) < 0.05, nullable=True),
            Cc.longs(dcnt, nullable=False), Cc.decimals128(decsum, 38, 2, sum_null, nullable=True),
            Cc.bools(empty, empty_null, nullable=True), Cc.decimals128(avgsum, 38, 2, rng.random(rows) < 0.05,
                                                                      nullable=True),
            Cc.longs(avgcnt, rng.random(rows) < 0.05, nullable=True)]
    return cols


@pytest.mark.parametrize("final,null_on_overflow", [(False, True), (True, True)])
def test_final_merges_match_the_oracle(cuda, final, null_on_overflow):
    rng = np.random.default_rng(4)
    rows = 30_000
    cols = merge_inputs(rng, rows, 300)
    fns = [A.CountMergeAgg(1), A.AverageMergeAgg(2, 3), A.SumLongAgg(1),
           A.WideDecimalSumMergeAgg(4, 5, 38, 2, final_result=final, null_on_overflow=null_on_overflow),
           A.WideDecimalAvgMergeAgg(6, 7, 38, 2), A.MinMaxAgg(2, True), A.MinMaxAgg(2, False)]
    w = G.Workload("merge", cols, [0], fns, 300, rows)
    assert same(w, [w.batch(0, 16_384), w.batch(16_384, rows)]) == N.VR_OK


@pytest.mark.parametrize("final,null_on_overflow", [(False, True), (True, True), (True, False)])
def test_merged_decimal_sum_overflow(cuda, final, null_on_overflow):
    rng = np.random.default_rng(5)
    rows = 8_000
    cols = merge_inputs(rng, rows, 4, overflow=True)
    fns = [A.WideDecimalSumMergeAgg(4, 5, 38, 2, final_result=final, null_on_overflow=null_on_overflow),
           A.CountMergeAgg(1)]
    w = G.Workload("mergeovf", cols, [0], fns, 4, rows)
    status = same(w, [w.batch()])
    assert status in (N.VR_OK, N.VR_ERR_DECIMAL_OVERFLOW)
    if final and not null_on_overflow:
        assert status == N.VR_ERR_DECIMAL_OVERFLOW
