"""Final results of averages on CPU: the oracle's decimal average against an
independent computation with Python's decimal module, which follows Spark's
Decimal./ literally -- BigDecimal.divide(count, 39, HALF_UP), then
setScale(result scale, HALF_UP) (DecimalAvgResult, VectorAggregates.scala:405-430;
DecimalKernels.java:44-48) -- on hand-picked ties, negative sums, results
past their precision, and random buffers; and avg(double) = sum / count."""
import decimal

import numpy as np
import pytest

from oracle.pyoracle import ORC_FP_COMPENSATED, Oracle
from parity import compare_arrays
from vecruntime_b200 import aggregate as A
from vecruntime_b200 import columns as Cc
from vecruntime_b200 import native as N

CTX = decimal.Context(prec=200)


def spark_avg(sum_unscaled: int, count: int, sum_scale: int, rs: int, rp: int):
    """Unscaled result, or None past the result precision."""
    q = CTX.divide(decimal.Decimal(sum_unscaled).scaleb(-sum_scale, CTX), decimal.Decimal(count))
    q = q.quantize(decimal.Decimal(1).scaleb(-39), rounding=decimal.ROUND_HALF_UP, context=CTX)
    q = q.quantize(decimal.Decimal(1).scaleb(-rs), rounding=decimal.ROUND_HALF_UP, context=CTX)
    u = int(q.scaleb(rs, CTX))
    return None if abs(u) >= 10 ** rp else u


# (sum unscaled at scale 2, count): exact ties at the result scale 6, their negatives,
# repeating quotients, counts near 2^63, a sum at the edge of Decimal(22,2)
CASES = [(1, 20_000), (-1, 20_000), (3, 40_000), (-3, 40_000), (1, 3), (-2, 3), (10 ** 21 - 1, 7),
         (-(10 ** 21 - 1), 9_223_372_036_854_775_807), (123456789, 1), (0, 5), (5, 8), (99, 2 ** 40 + 1),
         (10 ** 20, 3), (-(10 ** 20) - 7, 11), (1, 9_223_372_036_854_775_807)]


def merge_batch(cases, nulls=()):
    n = len(cases)
    keys = Cc.longs(np.arange(n, dtype=np.int64), nullable=False)
    sums = Cc.decimals128([s for s, _ in cases], 22, 2, [i in nulls for i in range(n)], nullable=True)
    counts = Cc.longs(np.array([c for _, c in cases], np.int64), nullable=False)
    return [keys, sums, counts], n


def emit_of(o):
    return o.emit(ORC_FP_COMPENSATED)


def test_decimal_average_matches_sparks_two_roundings():
    cols, n = merge_batch(CASES)
    fns = [A.WideDecimalAvgMergeAgg(1, 2, 22, 2, final_result=True)]
    o = Oracle(A.Spec(cols, [0], fns))
    o.update(Cc.host_batch(cols))
    out = emit_of(o)
    assert o.output_types[1].lane == N.VR_INT64 and o.output_types[1].precision == 16
    keys = out[0][0]
    vals, valid = out[1][0], Cc.unpack_bits(out[1][1], n)
    for i in range(n):
        s, c = CASES[int(keys[i])]
        want = spark_avg(s, c, 2, 6, 16)
        got = int(vals[i]) if valid[i] else None
        assert got == want, (s, c, got, want)


def test_decimal_average_ties_round_half_away_from_zero():
    assert spark_avg(1, 20_000, 2, 6, 16) == 1  # 0.0000005 -> 0.000001
    assert spark_avg(-1, 20_000, 2, 6, 16) == -1
    assert spark_avg(1, 3, 2, 6, 16) == 3333  # 0.003333...


def test_decimal_average_null_sum_and_zero_count():
    """A partial's null sum (overflowed) makes the result null, or the ANSI
    overflow error; a zero count is null before anything else."""
    cols, n = merge_batch([(5, 2), (7, 0), (9, 3)], nulls=(2,))
    o = Oracle(A.Spec(cols, [0], [A.WideDecimalAvgMergeAgg(1, 2, 22, 2, final_result=True)]))
    o.update(Cc.host_batch(cols))
    out = emit_of(o)
    valid = Cc.unpack_bits(out[1][1], n)
    by_key = {int(k): (bool(v), int(x)) for k, v, x in zip(out[0][0], valid, out[1][0])}
    assert by_key[0] == (True, 25000) and not by_key[1][0] and not by_key[2][0]
    o2 = Oracle(A.Spec(cols, [0], [A.WideDecimalAvgMergeAgg(1, 2, 22, 2, final_result=True,
                                                             null_on_overflow=False)]))
    o2.update(Cc.host_batch(cols))
    with pytest.raises(Exception) as e:
        emit_of(o2)
    assert getattr(e.value, "status", None) == N.VR_ERR_DECIMAL_OVERFLOW


def test_decimal_average_past_the_result_precision():
    """Decimal(38,2) buffers averaged at a given Decimal(20,6): a quotient of
    more than 14 integer digits is null (non-ANSI) or out of range (ANSI)."""
    cases = [(10 ** 30, 1), (10 ** 15, 1), (-(10 ** 16) + 1, 1)]
    n = len(cases)
    cols = [Cc.longs(np.arange(n, dtype=np.int64), nullable=False),
            Cc.decimals128([s for s, _ in cases], 38, 2, nullable=True),
            Cc.longs(np.array([c for _, c in cases], np.int64), nullable=False)]
    f = A.WideDecimalAvgMergeAgg(1, 2, 38, 2, final_result=True, result_precision=20, result_scale=6)
    o = Oracle(A.Spec(cols, [0], [f]))
    o.update(Cc.host_batch(cols))
    out = emit_of(o)
    assert o.output_types[1].lane == N.VR_DECIMAL128
    valid = Cc.unpack_bits(out[1][1], n)
    got = {int(k): (Cc.dec128_to_ints(out[1][0][i:i + 1])[0] if valid[i] else None) for i, k in enumerate(out[0][0])}
    for i, (s, c) in enumerate(cases):
        assert got[i] == spark_avg(s, c, 2, 6, 20)
    assert got[0] is None and got[1] == 10 ** 19
    f2 = A.WideDecimalAvgMergeAgg(1, 2, 38, 2, final_result=True, null_on_overflow=False, result_precision=20,
                                  result_scale=6)
    o2 = Oracle(A.Spec(cols, [0], [f2]))
    o2.update(Cc.host_batch(cols))
    with pytest.raises(Exception) as e:
        emit_of(o2)
    assert getattr(e.value, "status", None) == N.VR_ERR_DECIMAL_PRECISION


def test_random_decimal_averages():
    rng = np.random.default_rng(11)
    cases = [(int(rng.integers(-10 ** 18, 10 ** 18)) * int(rng.integers(1, 1000)), int(rng.integers(1, 10 ** 12)))
             for _ in range(2000)]
    cols, n = merge_batch(cases)
    o = Oracle(A.Spec(cols, [0], [A.WideDecimalAvgMergeAgg(1, 2, 22, 2, final_result=True)]))
    o.update(Cc.host_batch(cols))
    out = emit_of(o)
    valid = Cc.unpack_bits(out[1][1], n)
    for i, k in enumerate(out[0][0]):
        s, c = cases[int(k)]
        assert (int(out[1][0][i]) if valid[i] else None) == spark_avg(s, c, 2, 6, 16)


def test_double_average_final_is_sum_over_count():
    rng = np.random.default_rng(5)
    n = 5000
    k = rng.integers(0, 50, n)
    v = rng.standard_normal(n)
    nulls = rng.random(n) < 0.3
    nulls[k == 7] = True  # a group with no valid value: null average
    cols = [Cc.longs(k, nullable=False), Cc.doubles(v, nulls, nullable=True)]
    spec = A.Spec(cols, [0], [A.AverageAgg(1, final_result=True), A.SumDoubleAgg(1), A.CountAgg(1)])
    o = Oracle(spec)
    o.update(Cc.host_batch(cols))
    out = emit_of(o)
    g = o.num_groups()
    avg_ok = Cc.unpack_bits(out[1][1], g)
    for i in range(g):
        cnt = int(out[4][0][i])
        assert avg_ok[i] == (cnt > 0)
        if cnt:
            assert out[1][0][i] == pytest.approx(out[3][0][i] / cnt, rel=1e-14)
    assert compare_arrays(spec, o.output_types, out, g, o.output_types, out, g)[0] == 0
