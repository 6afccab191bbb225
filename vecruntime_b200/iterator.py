"""One task's aggregate driven batch by batch with a memory budget: the GPU
twin of the reference's VectorGroupedAggregateIterator
(spark/src/main/scala/org/apache/spark/sql/vecruntime/VectorHashAggregateExec.scala:463-1039).

Batches are consumed into a GPU table (`GpuHashAggregate`) until the input
ends or the table passes its budget; what happens then is the operator's
spill policy (`spillPolicy`, :185-246; `advance`, :689-757):

* InMemory        -- no budget: the whole input, then the groups.
* EmitAndReset    -- buffer-emitting modes (Partial, PartialMerge): a table
                     past the budget is emitted and the table starts over;
                     the next stage merges the pieces. A table that reduced
                     its rows by less than `pass_through_ratio` shows the
                     input does not aggregate here: every later batch is
                     aggregated on its own and emitted (pass-through, #376).
* GraceHash       -- a Final whose buffers are re-mergeable as emitted: past
                     the budget, the table's groups are spilled into
                     `buckets` partitions by the reference row hash of their
                     keys (vr_hash_rows) and the table starts over; at the end
                     each bucket is merged on its own, so no group is emitted
                     twice (AggregateSpill.scala:49-289). The spill lives in
                     host memory, the tier below HBM on a GPU node.

The budget is checked after every batch against the device bytes the
table's groups need, as of the last batch the handle has settled, and, with a shared
`HbmPool`, against what the pool grants (AggregateMemory, :423-452).
Groups come out in batches of `output_batch_rows` (the reference's
OutputBatchSize), each a (rows, [(data, validity), ...]) pair in the
handle's output schema.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass
from typing import Iterable, List, Optional

import numpy as np

from . import native as N
from .aggregate import GpuHashAggregate
from .columns import Col, HostBatch, pack_bits, unpack_bits


@dataclass
class InMemory:
    pass


@dataclass
class EmitAndReset:
    budget: int                     # device bytes of the table; 0 = no budget
    pass_through_ratio: float = 0.0  # rows per group below which the input does not reduce


@dataclass
class GraceHash:
    budget: int
    buckets: int = 16


class HbmPool:
    """Device memory shared by the aggregates of one GPU (the task memory
    manager's role for the reference's AggregateMemory): grants up to
    `capacity` bytes in total; what a table holds goes back at close."""

    def __init__(self, capacity: int):
        self.capacity = int(capacity)
        self.granted = 0
        self._lock = threading.Lock()

    def acquire(self, want: int) -> int:
        with self._lock:
            got = max(0, min(want, self.capacity - self.granted))
            self.granted += got
            return got

    def release(self, n: int) -> None:
        with self._lock:
            self.granted -= n


class AggregateMemory:
    """A table's reservation: over budget past the hard cap, or when the pool
    grants less than the table holds and the table is past
    `min_refusal_bytes` (AggregateMemory.overBudget,
    VectorHashAggregateExec.scala:436-445). Kept across resets, returned at close."""

    def __init__(self, pool: Optional[HbmPool] = None, min_refusal_bytes: int = 64 << 20):
        self.pool = pool
        self.min_refusal = min_refusal_bytes
        self.reserved = 0

    def over_budget(self, estimate: int, budget: int) -> bool:
        if budget > 0 and estimate > budget:
            return True
        if self.pool is not None and estimate > self.reserved:
            self.reserved += self.pool.acquire(estimate - self.reserved)
            if self.reserved < estimate and estimate >= self.min_refusal:
                return True
        return False

    def release(self) -> None:
        if self.pool is not None and self.reserved:
            self.pool.release(self.reserved)
            self.reserved = 0


def _take(t: N.ColumnType, data, validity, n, idx, nullable: bool) -> Col:
    """Rows `idx` of an emitted column as a new input column (with a validity
    bitmap only when the input column it feeds is nullable)."""
    valid = pack_bits(unpack_bits(validity, n)[idx]) if nullable else None
    if t.lane == N.VR_BOOL:
        vals = unpack_bits(data, n)[idx]
        c = Col(t.lane, pack_bits(vals), valid, t.precision, t.scale, t.dict_size, nullable)
        c._n = len(idx)
        return c
    return Col(t.lane, np.ascontiguousarray(data[:n][idx]), valid, t.precision, t.scale, t.dict_size, nullable)


class GpuGroupedAggregateIterator:
    """Consumes `source` (an iterable of HostBatch / DeviceBatch) into a GPU
    table under `policy` and yields output batches."""

    def __init__(self, source: Iterable, columns, keys, functions, policy=None, est_groups: int = 0,
                 max_batch_rows: int = 0, device: int = 0, memory: Optional[AggregateMemory] = None,
                 output_batch_rows: int = 4096, flags: int = 0):
        self.source = source
        self.policy = policy or InMemory()
        self.columns = list(columns)
        self.keys = list(keys)
        self.agg = GpuHashAggregate(columns, keys, functions, est_groups=est_groups, max_batch_rows=max_batch_rows,
                                    device=device, flags=flags)
        self.output_types = self.agg.output_types
        self.memory = memory or AggregateMemory()
        self.output_batch_rows = output_batch_rows
        self.pass_through = False
        self.tables_emitted = 0  # tables that went out before the input ended (spills / emit-and-reset)
        self.fill_rows = 0
        self.device = device
        self._types = [c.ctype() if isinstance(c, Col) else c for c in self.columns]
        if isinstance(self.policy, GraceHash):
            types = self._types
            if self.keys != list(range(len(self.keys))) or \
                    [t.lane for t in self.output_types] != [t.lane for t in types] or \
                    any(f.flags & N.VR_FN_FINAL for f in functions):
                raise ValueError("grace hash needs a merge whose output is its input's layout (keys first, "
                                 "then every buffer as declared, no result in a buffer slot): only such "
                                 "buffers can be merged again")

    # ------------------------------------------------------------ table
    def table_bytes(self) -> int:
        """Device bytes the table's groups need (slots at the load of 1/2 the
        table keeps), as of the last batch the handle settled: the
        reference's estimatedBytes. A reset empties it (the allocation itself
        stays for the next table to regrow into, as the reference keeps its
        reservation)."""
        st = self.agg.stats()
        return int(2 * st.groups * st.slot_bytes)

    def _fill(self, it, budget: int) -> bool:
        """Consumes batches until the input ends (True) or the table passes
        the budget (False) (`fill`, VectorHashAggregateExec.scala:643-657)."""
        for batch in it:
            self.fill_rows += batch.num_rows
            self.agg.consume(batch)
            if self.memory.over_budget(self.table_bytes(), budget):
                return False
        return True

    def _emit_table(self):
        n = self.agg.num_groups()
        for lo in range(0, n, self.output_batch_rows):
            hi = min(n, lo + self.output_batch_rows)
            yield hi - lo, self.agg.emit(lo, hi)

    def _reset(self):
        self.agg.reset()
        self.fill_rows = 0

    # ------------------------------------------------------------ grace hash
    def _buckets_of(self, arrays, n: int, buckets: int) -> np.ndarray:
        """Bucket of every emitted group: the reference row hash of its keys
        (vr_hash_rows on the device), modulo the bucket count."""
        import torch

        dev = torch.device("cuda", self.device)
        nk = len(self.keys)
        types = (N.ColumnType * nk)(*self.output_types[:nk])
        cols = (N.Column * nk)()
        keep = []
        for k in range(nk):
            d, v = arrays[k]
            t = torch.from_numpy(np.ascontiguousarray(d).view(np.uint8).reshape(-1).copy()).to(dev)
            tv = torch.from_numpy(np.ascontiguousarray(v).copy()).to(dev)
            keep += [t, tv]
            cols[k].data = t.data_ptr()
            cols[k].validity = tv.data_ptr()
        out = torch.empty(max(1, n), dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        N.check(N.lib().vr_hash_rows(nk, types, cols, n, C.c_void_p(out.data_ptr()), 1, C.c_void_p(stream)),
                "vr_hash_rows")
        h = out[:n].cpu().numpy().view(np.uint32)
        return (h % np.uint32(buckets)).astype(np.int64)

    def _spill(self, spill: List[list]) -> None:
        """The whole table into the buckets, as input batches of the same layout."""
        n = self.agg.num_groups()
        if n == 0:
            return
        arrays = self.agg.emit()
        b = self._buckets_of(arrays, n, len(spill))
        nullable = [bool(t.nullable) for t in self._types]
        for k in range(len(spill)):
            idx = np.flatnonzero(b == k)
            if len(idx):
                spill[k].append(HostBatch([_take(t, d, v, n, idx, nl) for t, (d, v), nl in
                                           zip(self.output_types, arrays, nullable)], len(idx)))

    # ------------------------------------------------------------ driving
    def __iter__(self):
        it = iter(self.source)
        p = self.policy
        if isinstance(p, InMemory):
            self._fill(it, 0)
            yield from self._emit_table()
        elif isinstance(p, EmitAndReset):
            done = False
            while not done:
                if self.pass_through:  # every later batch is its own table
                    for batch in it:
                        self._reset()
                        self.agg.consume(batch)
                        yield from self._emit_table()
                    break
                self._reset()
                done = self._fill(it, p.budget)
                if not done:
                    self.tables_emitted += 1
                    groups = self.agg.num_groups()
                    if p.pass_through_ratio > 0 and groups > 0 and self.fill_rows < p.pass_through_ratio * groups:
                        self.pass_through = True
                yield from self._emit_table()
        elif isinstance(p, GraceHash):
            spill = None
            while True:
                done = self._fill(it, p.budget)
                if done and spill is None:  # never spilled: the table is the answer
                    yield from self._emit_table()
                    break
                if spill is None:
                    spill = [[] for _ in range(max(2, p.buckets))]
                self._spill(spill)
                self.tables_emitted += 1
                self._reset()
                if done:
                    for bucket in spill:  # one bucket at a time, merged like the exchange's batches
                        self._reset()
                        for batch in bucket:
                            self.agg.consume(batch)
                        yield from self._emit_table()
                    break
        else:
            raise TypeError(f"unknown policy {p!r}")

    def close(self) -> None:
        self.memory.release()
        self.agg.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
