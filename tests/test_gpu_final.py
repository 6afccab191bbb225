"""Final and Complete results on the GPU against the oracle.

* The decimal average (DecimalAvgResult, VectorAggregates.scala:405-430):
  merged (sum, count) buffers, and raw rows in Complete mode, at the result
  type with Spark's two half-up roundings; ties, negative sums, null and
  overflowed sums, results past their precision, and the ANSI errors.
* avg(double) = sum / count, null for no rows.
* The plain aggregation run as Spark runs it: partial aggregates over four
  "tasks" of the 1,048,576 rows, their emitted buffers concatenated (the
  exchange), then a Final aggregate over them -- against the oracle's
  aggregate of the raw rows in Complete mode (VectorHashAggregateExec.scala:
  295-300, 1089-1165)."""
import numpy as np
import pytest

import vecruntime_b200 as vr
from vecruntime_b200 import aggregate as A
from vecruntime_b200 import columns as Cc
from vecruntime_b200 import datagen as G
from vecruntime_b200 import native as N

from oracle.pyoracle import ORC_FP_COMPENSATED, Oracle
from parity import compare, compare_arrays
from test_final_results_oracle import CASES, merge_batch

pytestmark = pytest.mark.gpu


def gpu_and_oracle(cols, keys, fns, est=0, flags=0):
    spec = A.Spec(cols, keys, fns)
    batch = Cc.host_batch(cols)
    agg = vr.GpuHashAggregate(cols, keys, fns, est_groups=est, max_batch_rows=batch.num_rows, flags=flags)
    try:
        agg.consume(batch)
        n = agg.num_groups()
        got = agg.emit()
        types = agg.output_types
    finally:
        agg.close()
    o = Oracle(spec)
    o.update(batch)
    return spec, types, got, n, o.output_types, o.emit(ORC_FP_COMPENSATED), o.num_groups()


@pytest.mark.parametrize("flags", [0, N.VR_SPEC_FORCE_GLOBAL, N.VR_SPEC_NO_JIT])
def test_decimal_average_of_merged_buffers(cuda, flags):
    rng = np.random.default_rng(3)
    cases = CASES + [(int(rng.integers(-10 ** 18, 10 ** 18)) * int(rng.integers(1, 1000)),
                      int(rng.integers(1, 10 ** 12))) for _ in range(5000)]
    cols, n = merge_batch(cases, nulls=(3, 17, 400))
    res = gpu_and_oracle(cols, [0], [A.WideDecimalAvgMergeAgg(1, 2, 22, 2, final_result=True)], est=n, flags=flags)
    bad, ex = compare_arrays(*res)
    assert bad == 0, ex


def test_decimal_average_wide_result_and_its_errors(cuda):
    """A DECIMAL128 result type; past its precision: null, or
    VR_ERR_DECIMAL_PRECISION under ANSI; a null partial sum: null, or
    VR_ERR_DECIMAL_OVERFLOW under ANSI."""
    cases = [(10 ** 30, 1), (10 ** 15, 1), (-(10 ** 16) + 1, 1), (-(10 ** 25) - 3, 7), (4, 8)]
    n = len(cases)
    cols = [Cc.longs(np.arange(n, dtype=np.int64), nullable=False),
            Cc.decimals128([s for s, _ in cases], 38, 2, [i == 4 for i in range(n)], nullable=True),
            Cc.longs(np.array([c for _, c in cases], np.int64), nullable=False)]
    f = A.WideDecimalAvgMergeAgg(1, 2, 38, 2, final_result=True, result_precision=20, result_scale=6)
    res = gpu_and_oracle(cols, [0], [f], est=n)
    assert res[1][1].lane == N.VR_DECIMAL128
    bad, ex = compare_arrays(*res)
    assert bad == 0, ex
    for i, status in ((0, N.VR_ERR_DECIMAL_PRECISION), (4, N.VR_ERR_DECIMAL_OVERFLOW)):
        one = [Cc.longs(np.array([i], np.int64), nullable=False),
               Cc.decimals128([cases[i][0]], 38, 2, [i == 4], nullable=True),
               Cc.longs(np.array([cases[i][1]], np.int64), nullable=False)]
        fa = A.WideDecimalAvgMergeAgg(1, 2, 38, 2, final_result=True, null_on_overflow=False, result_precision=20,
                                      result_scale=6)
        agg = vr.GpuHashAggregate(one, [0], [fa], est_groups=1, max_batch_rows=1)
        try:
            agg.consume(Cc.host_batch(one))
            with pytest.raises(vr.VrError) as e:
                agg.emit()
            assert e.value.status == status
            if status == N.VR_ERR_DECIMAL_PRECISION:  # the value Spark's message names
                assert agg.error_value() == (10 ** 34, 20, 6)
            else:
                assert agg.error_value() is None
        finally:
            agg.close()


def test_complete_mode_decimal_and_double_averages(cuda):
    """Complete mode over raw rows: the decimal report's averages (qty and
    disc, DECIMAL(12,2) -> Decimal(16,6)) and a double average, per group."""
    w = G.decimal_report(rows=300_000)
    fns = [A.WideDecimalAvgAgg(2, 22, 2, final_result=True), A.WideDecimalAvgAgg(4, 22, 2, final_result=True),
           A.CountAgg()]
    res = gpu_and_oracle(w.columns, w.keys, fns, est=6)
    bad, ex = compare_arrays(*res)
    assert bad == 0, ex
    rng = np.random.default_rng(8)
    n = 200_000
    k = rng.integers(0, 3000, n)
    v = rng.lognormal(0, 1, n)
    nulls = rng.random(n) < 0.2
    nulls[k % 97 == 0] = True  # groups with no valid value
    cols = [Cc.longs(k, nullable=False), Cc.doubles(v, nulls, nullable=True)]
    res = gpu_and_oracle(cols, [0], [A.AverageAgg(1, final_result=True), A.CountAgg(1)], est=3000)
    bad, ex = compare_arrays(*res)
    assert bad == 0, ex


def test_plain_partial_then_final(cuda):
    """The plain aggregation (1,048,576 rows, 1,000 groups; count(*),
    count(v1), sum(v1) checked, min/max(v1), sum(v2), avg(v2)) as four partial
    tasks, their buffers exchanged, then one Final aggregate: the result
    equals the oracle's Complete aggregate of the raw rows."""
    w = G.plain()
    tasks = 4
    rows = w.rows // tasks
    parts = []
    for t in range(tasks):
        agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=4096)
        for lo in range(t * rows, (t + 1) * rows, 4096):  # 4,096-row batches, as the reference's iterator
            agg.consume(w.batch(lo, lo + 4096))
        n = agg.num_groups()
        parts.append((agg.output_types, agg.emit(), n))
        agg.close()
    # the exchange: every task's buffer rows, one after another
    types = parts[0][0]

    def column(j):
        t = types[j]
        data = np.concatenate([p[1][j][0][:p[2]] for p in parts])
        valid = np.concatenate([Cc.unpack_bits(p[1][j][1], p[2]) for p in parts])
        mk = {N.VR_INT64: Cc.longs, N.VR_FLOAT64: Cc.doubles}[t.lane]
        return mk(data, ~valid, nullable=True)

    # buffers: key, count(*), count(v1), sum(v1), min(v1), max(v1), sum(v2), avg(v2) sum, avg(v2) count
    buf = [column(j) for j in range(len(types))]
    final_fns = [A.CountMergeAgg(1), A.CountMergeAgg(2), A.SumLongAgg(3, checked=True), A.MinMaxAgg(4, True),
                 A.MinMaxAgg(5, False), A.SumDoubleAgg(6), A.AverageMergeAgg(7, 8, final_result=True)]
    buf[0] = Cc.longs(buf[0].data, nullable=False)
    final = vr.GpuHashAggregate(buf, [0], final_fns, est_groups=1000, max_batch_rows=len(buf[0].data))
    try:
        final.consume(Cc.host_batch(buf))
        n = final.num_groups()
        got = final.emit()
        got_types = final.output_types
    finally:
        final.close()
    complete = [A.CountAgg(), A.CountAgg(1), A.SumLongAgg(1, checked=True), A.MinMaxAgg(1, True),
                A.MinMaxAgg(1, False), A.SumDoubleAgg(2), A.AverageAgg(2, final_result=True)]
    o = Oracle(A.Spec(w.columns, w.keys, complete))
    o.update(w.batch())
    assert n == 1000
    # the partial double sums are rounded once each when emitted, so the
    # final sums carry an absolute error of a few ulps of the partials:
    # the tolerance floor is 1e-15 of the group's sum of magnitudes (rows x 6
    # bounds it for N(0,1) values)
    compare(A.Spec(buf, [0], final_fns), got_types, got, n, o.output_types, o.emit(ORC_FP_COMPENSATED),
            o.num_groups(), fsum_scale=lambda row: 6.0 * row[1])
