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
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

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
    result_precision: int = 0  # final decimal average: result type (0 = Spark's from the buffer type)
    result_scale: int = 0

    def to_ctypes(self) -> N.AggFn:
        f = N.AggFn()
        f.kind, f.input, f.input2, f.flags = self.kind, self.input, self.input2, self.flags
        f.precision, f.scale, f.num_terms = self.precision, self.scale, len(self.terms)
        f.product_precision = self.product_precision
        f.result_precision, f.result_scale = self.result_precision, self.result_scale
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


def AverageAgg(input: int, strict: bool = True, final_result: bool = False) -> AggFunction:
    """avg over doubles: buffer (sum, count) (VectorAggregates.scala:1021-1039);
    `final_result` (Complete mode): the average itself, null for no rows, then the count."""
    return AggFunction(N.VR_FN_AVG_DOUBLE, input,
                       flags=(N.VR_FN_STRICT if strict else 0) | (N.VR_FN_FINAL if final_result else 0))


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


def WideDecimalAvgAgg(input, buffer_precision: int, scale: int, final_result: bool = False,
                      null_on_overflow: bool = True, result_precision: int = 0, result_scale: int = 0) -> AggFunction:
    """avg over a decimal: buffer (sum: Decimal(p+10, s), count) (VectorAggregates.scala:444-516);
    `final_result` (Complete mode): DecimalAvgResult at Decimal(p+4, s+4) (or the given result
    type), then the count (VectorAggregates.scala:405-430)."""
    flags = (N.VR_FN_FINAL if final_result else 0) | (N.VR_FN_NULL_ON_OVERFLOW if null_on_overflow else 0)
    if isinstance(input, DecimalProduct):
        return AggFunction(N.VR_FN_AVG_DECIMAL, -1, flags=flags, precision=buffer_precision, scale=scale,
                           terms=tuple(input.factors), product_precision=input.precision,
                           result_precision=result_precision, result_scale=result_scale)
    return AggFunction(N.VR_FN_AVG_DECIMAL, input, flags=flags, precision=buffer_precision, scale=scale,
                       result_precision=result_precision, result_scale=result_scale)


def CountMergeAgg(count: int) -> AggFunction:
    """Final count: partial counts summed (VectorAggregates.scala:1042-1059)."""
    return AggFunction(N.VR_FN_COUNT_MERGE, count)


def AverageMergeAgg(sum_col: int, count_col: int, final_result: bool = False) -> AggFunction:
    """avg merge: (sum, count) buffers summed (VectorAggregates.scala:1065-1090); `final_result`:
    Average's evaluateExpression, sum / count (null for no rows), then the count."""
    return AggFunction(N.VR_FN_AVG_DOUBLE_MERGE, sum_col, count_col, flags=N.VR_FN_FINAL if final_result else 0)


def WideDecimalSumMergeAgg(sum_col: int, is_empty_col: int, buffer_precision: int, scale: int,
                           final_result: bool = False, null_on_overflow: bool = True) -> AggFunction:
    """Merge of (sum, isEmpty) buffers (VectorAggregates.scala:658-781)."""
    return AggFunction(N.VR_FN_SUM_DECIMAL_MERGE, sum_col, is_empty_col,
                       flags=_dec_flags(final_result, null_on_overflow), precision=buffer_precision, scale=scale)


def WideDecimalAvgMergeAgg(sum_col: int, count_col: int, buffer_precision: int, scale: int,
                           final_result: bool = False, null_on_overflow: bool = True, result_precision: int = 0,
                           result_scale: int = 0) -> AggFunction:
    """Merge of (sum, count) decimal average buffers (VectorAggregates.scala:526-642); `final_result`:
    DecimalAvgResult in the sum slot (VectorAggregates.scala:405-430), then the count."""
    flags = (N.VR_FN_FINAL if final_result else 0) | (N.VR_FN_NULL_ON_OVERFLOW if null_on_overflow else 0)
    return AggFunction(N.VR_FN_AVG_DECIMAL_MERGE, sum_col, count_col, flags=flags, precision=buffer_precision,
                       scale=scale, result_precision=result_precision, result_scale=result_scale)


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


def _out_bytes(t: N.ColumnType, n: int) -> int:
    """Bytes of an output column's data for n groups."""
    if t.lane in (N.VR_INT32, N.VR_DICT32):
        return 4 * n
    if t.lane in (N.VR_INT64, N.VR_FLOAT64):
        return 8 * n
    if t.lane == N.VR_DECIMAL128:
        return 16 * n
    return max((n + 7) // 8, 1)  # BOOL: a bitmap


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

    def emit(self, start: int = 0, end: Optional[int] = None, out=None):
        """Groups [start, end) as a list of (data, validity) numpy pairs, one per
        output column. `out`: such pairs to write into instead of new arrays
        (e.g. views of pinned memory, reused batch after batch); each buffer
        must hold the range."""
        total = self.num_groups()
        end = total if end is None else end
        n = end - start
        if out is None:
            arrays = [_out_arrays(t, n) for t in self.output_types]
        else:
            arrays = list(out)
            if len(arrays) != len(self.output_types):
                raise ValueError("emit: one (data, validity) pair per output column")
            for t, (d, v) in zip(self.output_types, arrays):
                if d.nbytes < _out_bytes(t, n) or v.nbytes < max((n + 7) // 8, 1):
                    raise ValueError("emit: an output buffer is smaller than the range")
        outs = (N.OutColumn * max(1, len(arrays)))()
        for i, (d, v) in enumerate(arrays):
            outs[i].data = d.ctypes.data
            outs[i].validity = v.ctypes.data
        N.check(self._lib.vr_agg_emit(self.h, start, end, outs, N.VR_HOST), "vr_agg_emit", self.h)
        return arrays

    def reset(self) -> None:
        N.check(self._lib.vr_agg_reset(self.h), "vr_agg_reset", self.h)

    def error_value(self):
        """After a VR_ERR_DECIMAL_PRECISION emit: (unscaled value, precision,
        scale) of the decimal that left its type, or None."""
        lo, hi, p, s = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
        if self._lib.vr_agg_error_value(self.h, C.byref(lo), C.byref(hi), C.byref(p), C.byref(s)) != N.VR_OK:
            return None
        u = ((hi.value & ((1 << 64) - 1)) << 64) | (lo.value & ((1 << 64) - 1))
        return (u - (1 << 128) if u >> 127 else u), p.value, s.value

    def key_dictionary(self, key: int):
        """The strings (bytes) behind key `key`'s emitted table ids, when its
        batches bring their own dictionaries (vr_agg_key_dictionary)."""
        n, nb = C.c_int32(), C.c_int64()
        N.check(self._lib.vr_agg_key_dictionary(self.h, key, C.byref(n), None, None, 0, C.byref(nb)),
                "vr_agg_key_dictionary", self.h)
        offs = np.zeros(n.value + 1, np.int32)
        data = np.zeros(max(1, nb.value), np.uint8)
        N.check(self._lib.vr_agg_key_dictionary(self.h, key, C.byref(n), offs.ctypes.data, data.ctypes.data,
                                                nb.value, C.byref(nb)), "vr_agg_key_dictionary", self.h)
        return [data[offs[i]:offs[i + 1]].tobytes() for i in range(n.value)]

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


def tune_search(columns, keys, functions, device_batch, est_groups: int = 0, max_batch_rows: int = 0,
                device: int = 0, iters: int = 2):
    """vr_tune_search: times every candidate launch configuration of the spec
    on one device-resident batch and records the fastest in the autotuner's
    table for (spec, rows, estimated groups), where handles created afterwards
    find it. Returns (choice, rows/s)."""
    spec = Spec(columns, keys, functions, est_groups, max_batch_rows, device)
    cb = device_batch.ctypes()
    best = N.TuneChoice()
    rps = C.c_double()
    N.check(N.lib().vr_tune_search(C.byref(spec.spec), C.byref(cb), iters, C.byref(best), C.byref(rps)),
            "vr_tune_search")
    return best, rps.value


# ------------------------------------------------------------------ batched
class GpuBatchedAggregate:
    """Many independent aggregates (one Spark task's batch each) run by one
    persistent launch (mode VR_BATCHED_PERSISTENT, optionally replayed from a
    CUDA graph) or by one launch per instance (VR_BATCHED_PLAIN). The
    instances share one spec (the same functions over the same column types)
    and one tier; each keeps its own table and shared-memory strategy (whole
    table, hot-key cache or HBM only), which `tune` chooses per estimated-groups
    bucket. No reference counterpart: the reference runs one task per thread
    (VectorHashAggregateExec.scala:248-302)."""

    def __init__(self, instances: Sequence["GpuHashAggregate"], device_batches: Sequence, mode: int = 0,
                 use_graph: bool = False, shape: Optional[N.TuneChoice] = None):
        self._lib = N.lib()
        self.instances = list(instances)
        self._batches = list(device_batches)
        self._hs = (C.c_void_p * len(self.instances))(*[a.h.value for a in self.instances])
        self._bs = (N.Batch * len(self._batches))(*[b.ctypes() for b in self._batches])
        self._shape = shape
        plan = N.BatchedPlan(len(self.instances), self._hs, self._bs, mode, 1 if use_graph else 0,
                             C.pointer(shape) if shape is not None else None)
        h = C.c_void_p()
        rc = self._lib.vr_batched_create(C.byref(plan), C.byref(h))
        if rc:
            raise N.VrError(rc, "vr_batched_create: " + (self._lib.vr_thread_last_error() or b"").decode())
        self.h = h

    def run(self, stream: int = 0) -> None:
        """Resets every instance's table and aggregates every instance's batch
        on `stream` (0: the legacy default stream); returns once the device
        has finished and every instance's group count is known."""
        rc = self._lib.vr_batched_run(self.h, C.c_void_p(stream) if stream else None)
        if rc:
            raise N.VrError(rc, "vr_batched_run: " + (self._lib.vr_thread_last_error() or b"").decode())

    def tune(self, iters: int = 2) -> float:
        """vr_batched_tune: each estimated-groups bucket's shared-memory
        strategy chosen by measurement; returns the launch's ms with them."""
        ms = C.c_double()
        rc = self._lib.vr_batched_tune(self.h, iters, C.byref(ms))
        if rc:
            raise N.VrError(rc, "vr_batched_tune: " + (self._lib.vr_thread_last_error() or b"").decode())
        return ms.value

    def info(self) -> dict:
        """The persistent launch's block shape and how many instances use a
        whole shared-memory table, a hot-key cache or HBM alone."""
        i = N.BatchedInfo()
        N.check(self._lib.vr_batched_get_info(self.h, C.byref(i)), "vr_batched_get_info")
        return {name: getattr(i, name) for name, _ in N.BatchedInfo._fields_}

    def close(self) -> None:
        if self.h:
            self._lib.vr_batched_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ serving
class AggregateServer:
    """Continuous batching of partial-aggregation requests over resident
    per-query tables (vr_srv_*): requests from many tasks are admitted as soon
    as a device slot and the HBM budget allow; latency is submit -> device
    completion. No reference counterpart."""

    def __init__(self, device: int = 0, slots: int = 8, hbm_cap_bytes: int = 120 << 30,
                 staging_bytes_per_slot: int = 0):
        self._lib = N.lib()
        cfg = N.SrvConfig(device, slots, hbm_cap_bytes, staging_bytes_per_slot, 0, 0)
        h = C.c_void_p()
        rc = self._lib.vr_srv_create(C.byref(cfg), C.byref(h))
        if rc:
            raise N.VrError(rc, "vr_srv_create: " + (self._lib.vr_thread_last_error() or b"").decode())
        self.h = h
        self._specs = {}
        self._pending = {}  # ticket -> batch kept alive until it completes

    def _check(self, rc, what):
        if rc:
            raise N.VrError(rc, f"{what}: " + (self._lib.vr_thread_last_error() or b"").decode())

    def open_query(self, columns, keys, functions, est_groups: int = 0, max_batch_rows: int = 0) -> int:
        spec = Spec(columns, keys, functions, est_groups, max_batch_rows)
        q = C.c_int32()
        self._check(self._lib.vr_srv_open_query(self.h, C.byref(spec.spec), C.byref(q)), "vr_srv_open_query")
        self._specs[q.value] = spec
        return q.value

    def submit(self, query: int, batch) -> int:
        cb = batch.ctypes()
        t = C.c_uint64()
        self._check(self._lib.vr_srv_submit(self.h, query, C.byref(cb), C.byref(t)), "vr_srv_submit")
        self._pending[t.value] = (batch, cb)
        return t.value

    def wait(self, ticket: int) -> float:
        ms = C.c_double()
        self._check(self._lib.vr_srv_wait(self.h, ticket, C.byref(ms)), "vr_srv_wait")
        self._pending.pop(ticket, None)
        return ms.value

    def drain(self) -> None:
        self._check(self._lib.vr_srv_drain(self.h), "vr_srv_drain")
        self._pending.clear()

    def results(self, query: int):
        """(output types, arrays, group count) of a query after its queued requests."""
        h = C.c_void_p()
        self._check(self._lib.vr_srv_query_handle(self.h, query, C.byref(h)), "vr_srv_query_handle")
        n = C.c_int32()
        types = (N.ColumnType * 64)()
        N.check(self._lib.vr_agg_output_schema(h, C.byref(n), types, 64), "output schema")
        out_types = [types[i] for i in range(n.value)]
        g = C.c_int64()
        N.check(self._lib.vr_agg_num_groups(h, C.byref(g)), "vr_agg_num_groups")
        arrays = [_out_arrays(t, g.value) for t in out_types]
        outs = (N.OutColumn * max(1, len(arrays)))()
        for i, (d, v) in enumerate(arrays):
            outs[i].data = d.ctypes.data
            outs[i].validity = v.ctypes.data
        N.check(self._lib.vr_agg_emit(h, 0, g.value, outs, N.VR_HOST), "vr_agg_emit")
        return out_types, arrays, g.value

    def close_query(self, query: int) -> None:
        self._check(self._lib.vr_srv_close_query(self.h, query), "vr_srv_close_query")

    def stats(self) -> N.SrvStats:
        st = N.SrvStats()
        self._lib.vr_srv_get_stats(self.h, C.byref(st))
        return st

    def close(self) -> None:
        if self.h:
            self._lib.vr_srv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
