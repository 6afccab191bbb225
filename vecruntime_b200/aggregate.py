"""Host-side mirror of the reference's aggregate operator interface.

Function classes carry the reference's names and argument meaning
(spark/src/main/scala/io/vecruntime/spark/agg/VectorAggregates.scala):
each compiles to one `vr_agg_fn`; `GpuHashAggregate` plays the role of
VectorGroupedAggregateIterator (VectorHashAggregateExec.scala:463-1039):
`consume` a batch, ask `num_groups`, `emit` Spark buffer columns, `reset`,
`close`. Everything below runs through libvrgpu; nothing computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import native as N
from .columns import Col, DeviceBatch, HostBatch


# ---------------------------------------------------------------- functions
@dataclass
class AggFunction:
    kind: int
    input: int = -1
    input2: int = -1
    flags: int = 0
    precision: int = 0
    scale: int = 0
    terms: Tuple[Tuple[int, int, int], ...] = ()  # (column, sign, addend)
    product_precision: int = 0

    def to_ctypes(self) -> N.AggFn:
        f = N.AggFn()
        f.kind, f.input, f.input2, f.flags = self.kind, self.input, self.input2, self.flags
        f.precision, f.scale, f.num_terms = self.precision, self.scale, len(self.terms)
        f.product_precision = self.product_precision
        for i, (c, s, a) in enumerate(self.terms):
            f.terms[i] = N.Term(c, s, a)
        return f


def CountAgg(input: Optional[int] = None) -> AggFunction:
    """count(*) when input is None, else count of non-null values (VectorAggregates.scala:906-926)."""
    return AggFunction(N.VR_FN_COUNT_STAR) if input is None else AggFunction(N.VR_FN_COUNT, input)


def SumLongAgg(input: int, checked: bool = False) -> AggFunction:
    """sum over INT32/INT64 into bigint; `checked` is ANSI (VectorAggregates.scala:142-200)."""
    return AggFunction(N.VR_FN_SUM_LONG, input, flags=N.VR_FN_CHECKED if checked else 0)


def SumDoubleAgg(input: int, strict: bool = True) -> AggFunction:
    """sum over doubles, null when empty (VectorAggregates.scala:118-136)."""
    return AggFunction(N.VR_FN_SUM_DOUBLE, input, flags=N.VR_FN_STRICT if strict else 0)


def AverageAgg(input: int, strict: bool = True) -> AggFunction:
    """avg over doubles: buffer (sum, count) (VectorAggregates.scala:1021-1039)."""
    return AggFunction(N.VR_FN_AVG_DOUBLE, input, flags=N.VR_FN_STRICT if strict else 0)


def MinMaxAgg(input: int, is_min: bool) -> AggFunction:
    """min/max with Spark's NaN order (VectorAggregates.scala:929-1018)."""
    return AggFunction(N.VR_FN_MIN if is_min else N.VR_FN_MAX, input)


def _dec_flags(final_result, null_on_overflow):
    return (N.VR_FN_FINAL if final_result else 0) | (N.VR_FN_NULL_ON_OVERFLOW if null_on_overflow else 0)


@dataclass
class DecimalProduct:
    """The exact product of factors (addend + sign * column), e.g.
    price * (1 - disc): DecimalProduct([(price, 1, 0), (disc, -1, 100)]).
    Stands in for SpeculativeDecimalMulExpr (DecimalExprs.scala:470-516)."""
    factors: Sequence[Tuple[int, int, int]]
    precision: int = 38


def WideDecimalSumAgg(input, buffer_precision: int, scale: int, final_result: bool = False,
                      null_on_overflow: bool = True, checked_product: bool = False) -> AggFunction:
    """sum over a decimal into Decimal(p+10, s): buffer (sum, isEmpty) (VectorAggregates.scala:318-395)."""
    flags = _dec_flags(final_result, null_on_overflow) | (N.VR_FN_CHECKED if checked_product else 0)
    if isinstance(input, DecimalProduct):
        return AggFunction(N.VR_FN_SUM_DECIMAL, -1, flags=flags, precision=buffer_precision, scale=scale,
                           terms=tuple(input.factors), product_precision=input.precision)
    return AggFunction(N.VR_FN_SUM_DECIMAL, input, flags=flags, precision=buffer_precision, scale=scale)


def WideDecimalAvgAgg(input, buffer_precision: int, scale: int) -> AggFunction:
    """avg over a decimal: buffer (sum: Decimal(p+10, s), count) (VectorAggregates.scala:444-516)."""
    if isinstance(input, DecimalProduct):
        return AggFunction(N.VR_FN_AVG_DECIMAL, -1, precision=buffer_precision, scale=scale,
                           terms=tuple(input.factors), product_precision=input.precision)
    return AggFunction(N.VR_FN_AVG_DECIMAL, input, precision=buffer_precision, scale=scale)


def CountMergeAgg(count: int) -> AggFunction:
    """Final count: partial counts summed (VectorAggregates.scala:1042-1059)."""
    return AggFunction(N.VR_FN_COUNT_MERGE, count)


def AverageMergeAgg(sum_col: int, count_col: int) -> AggFunction:
    """Final avg: (sum, count) buffers summed (VectorAggregates.scala:1065-1090)."""
    return AggFunction(N.VR_FN_AVG_DOUBLE_MERGE, sum_col, count_col)


def WideDecimalSumMergeAgg(sum_col: int, is_empty_col: int, buffer_precision: int, scale: int,
                           final_result: bool = False, null_on_overflow: bool = True) -> AggFunction:
    """Merge of (sum, isEmpty) buffers (VectorAggregates.scala:658-781)."""
    return AggFunction(N.VR_FN_SUM_DECIMAL_MERGE, sum_col, is_empty_col,
                       flags=_dec_flags(final_result, null_on_overflow), precision=buffer_precision, scale=scale)


def WideDecimalAvgMergeAgg(sum_col: int, count_col: int, buffer_precision: int, scale: int) -> AggFunction:
    """Merge of (sum, count) decimal average buffers (VectorAggregates.scala:526-642)."""
    return AggFunction(N.VR_FN_AVG_DECIMAL_MERGE, sum_col, count_col, precision=buffer_precision, scale=scale)


# --------------------------------------------------------------------- spec
class Spec:
    """A vr_agg_spec with its backing arrays kept alive."""

    def __init__(self, columns: Sequence, keys: Sequence[int], functions: Sequence[AggFunction],
                 est_groups: int = 0, max_batch_rows: int = 0, device: int = 0, flags: int = 0):
        types = [c.ctype() if isinstance(c, Col) else c for c in columns]
        self.col_arr = (N.ColumnType * max(1, len(types)))(*types)
        self.key_arr = (C.c_int32 * max(1, len(keys)))(*keys)
        fns = [f.to_ctypes() for f in functions]
        self.fn_arr = (N.AggFn * max(1, len(fns)))(*fns)
        self.spec = N.AggSpec(len(types), self.col_arr, len(keys), self.key_arr, len(fns), self.fn_arr,
                              est_groups, max_batch_rows, device, flags)
        self.columns = types
        self.keys = list(keys)
        self.functions = list(functions)

    def plan(self):
        """Host-only plan inspection (no GPU): vr_plan_info and output types."""
        info = N.PlanInfo()
        outs = (N.ColumnType * 64)()
        rc = N.lib().vr_agg_plan(C.byref(self.spec), C.byref(info), outs, 64)
        return rc, info, [outs[i] for i in range(info.num_outputs)]


def _out_arrays(t: N.ColumnType, n: int):
    nb = (n + 7) // 8
    if t.lane in (N.VR_INT32, N.VR_DICT32):
        data = np.zeros(n, np.int32)
    elif t.lane == N.VR_INT64:
        data = np.zeros(n, np.int64)
    elif t.lane == N.VR_FLOAT64:
        data = np.zeros(n, np.float64)
    elif t.lane == N.VR_DECIMAL128:
        data = np.zeros((n, 2), np.uint64)
    else:  # BOOL
        data = np.zeros(max(nb, 1), np.uint8)
    return data, np.zeros(max(nb, 1), np.uint8)


# ------------------------------------------------------------------ operator
class GpuHashAggregate:
    """One task's grouped aggregate on the GPU (the GPU twin of
    VectorGroupedAggregateIterator: consume / num_groups / emit / reset / close)."""

    def __init__(self, columns, keys, functions, est_groups=0, max_batch_rows=0, device=0, flags=0,
                 tune: Optional[N.TuneChoice] = None):
        self.spec = Spec(columns, keys, functions, est_groups, max_batch_rows, device, flags)
        self._lib = N.lib()
        h = C.c_void_p()
        if tune is not None:
            rc = self._lib.vr_agg_create_tuned(C.byref(self.spec.spec), C.byref(tune), C.byref(h))
        else:
            rc = self._lib.vr_agg_create(C.byref(self.spec.spec), C.byref(h))
        N.check(rc, "vr_agg_create")
        self.h = h
        self._pending = []  # batches kept alive until sync
        n = C.c_int32()
        types = (N.ColumnType * 64)()
        N.check(self._lib.vr_agg_output_schema(self.h, C.byref(n), types, 64), "output schema")
        self.output_types = [types[i] for i in range(n.value)]

    # -- lifecycle ------------------------------------------------------
    def consume(self, batch) -> None:
        """vr_agg_update: GroupKeyTable.assign + GroupedAggState.update for one batch."""
        cb = batch.ctypes()
        self._pending.append((batch, cb))
        N.check(self._lib.vr_agg_update(self.h, C.byref(cb)), "vr_agg_update", self.h)

    def sync(self) -> None:
        N.check(self._lib.vr_agg_sync(self.h), "vr_agg_sync", self.h)
        self._pending.clear()

    def num_groups(self) -> int:
        g = C.c_int64()
        N.check(self._lib.vr_agg_num_groups(self.h, C.byref(g)), "vr_agg_num_groups", self.h)
        self._pending.clear()
        return g.value

    def emit(self, start: int = 0, end: Optional[int] = None):
        """Groups [start, end) as a list of (data, validity) numpy pairs, one per output column."""
        total = self.num_groups()
        end = total if end is None else end
        n = end - start
        arrays = [_out_arrays(t, n) for t in self.output_types]
        outs = (N.OutColumn * max(1, len(arrays)))()
        for i, (d, v) in enumerate(arrays):
            outs[i].data = d.ctypes.data
            outs[i].validity = v.ctypes.data
        N.check(self._lib.vr_agg_emit(self.h, start, end, outs, N.VR_HOST), "vr_agg_emit", self.h)
        return arrays

    def reset(self) -> None:
        N.check(self._lib.vr_agg_reset(self.h), "vr_agg_reset", self.h)

    def stats(self) -> N.AggStats:
        st = N.AggStats()
        self._lib.vr_agg_get_stats(self.h, C.byref(st))
        return st

    def stream(self) -> int:
        return self._lib.vr_agg_stream(self.h) or 0

    def close(self) -> None:
        if self.h:
            self._lib.vr_agg_destroy(self.h)
            self.h = None
            self._pending.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
