"""The task-level driver with a memory budget (the GPU twin of
VectorGroupedAggregateIterator's spill policies, VectorHashAggregateExec.scala:
185-246, 643-757), against the oracle's aggregate of the raw rows:

* EmitAndReset: a partial aggregate past its budget emits its table and
  starts over; a Final over every emitted piece gives the oracle's groups.
* pass-through: a table that does not reduce its rows switches every later
  batch to its own table.
* GraceHash: a Final past its budget spills its groups into buckets by key
  hash and merges one bucket at a time: the oracle's groups, none twice.
* a shared HBM pool that grants less than a table holds is a budget too."""
import numpy as np
import pytest

from vecruntime_b200 import aggregate as A
from vecruntime_b200 import columns as Cc
from vecruntime_b200 import iterator as I
from vecruntime_b200 import native as N

from oracle.pyoracle import ORC_FP_COMPENSATED, Oracle
from parity import compare_arrays

pytestmark = pytest.mark.gpu

PARTIAL = [A.CountAgg(), A.CountAgg(1), A.SumLongAgg(1), A.MinMaxAgg(1, True), A.MinMaxAgg(1, False),
           A.SumDoubleAgg(2), A.AverageAgg(2)]
FINAL = [A.CountMergeAgg(1), A.CountMergeAgg(2), A.SumLongAgg(3), A.MinMaxAgg(4, True), A.MinMaxAgg(5, False),
         A.SumDoubleAgg(6), A.AverageMergeAgg(7, 8)]
COMPLETE = [A.CountAgg(), A.CountAgg(1), A.SumLongAgg(1), A.MinMaxAgg(1, True), A.MinMaxAgg(1, False),
            A.SumDoubleAgg(2), A.AverageAgg(2)]


def rows_of_keys(seed, rows, groups, batch=8192):
    """`rows` rows over `groups` distinct int64 keys (groups=None: every row its own key)."""
    rng = np.random.default_rng(seed)
    if groups is None:
        k = rng.permutation(rows).astype(np.int64) * 7919 + 13
    else:
        domain = rng.integers(-(1 << 62), 1 << 62, groups, dtype=np.int64)
        k = domain[rng.integers(0, groups, rows)]
    v1 = rng.integers(-10 ** 6, 10 ** 6, rows, dtype=np.int64)
    nulls = rng.random(rows) < 0.05
    v2 = rng.standard_normal(rows)
    cols = [Cc.longs(k, nullable=False), Cc.longs(v1, nulls, nullable=True), Cc.doubles(v2, nullable=False)]
    batches = []
    for lo in range(0, rows, batch):
        hi = min(rows, lo + batch)
        batches.append(Cc.host_batch([Cc.Col(c.lane, c.data[lo:hi],
                                             None if c.validity is None else Cc.pack_bits(
                                                 Cc.unpack_bits(c.validity, rows)[lo:hi]), nullable=c.nullable)
                                      for c in cols]))
    return cols, batches


def concat(types, pieces):
    """Output batches of an iterator as one host batch of input columns."""
    cols = []
    for j, t in enumerate(types):
        data = np.concatenate([a[j][0][:n] for n, a in pieces])
        valid = np.concatenate([Cc.unpack_bits(a[j][1], n) for n, a in pieces])
        cols.append(Cc.Col(t.lane, data, Cc.pack_bits(valid), t.precision, t.scale, 0, True))
    cols[0] = Cc.Col(cols[0].lane, cols[0].data, None, nullable=False)
    return cols


def final_over(cols, est):
    it = I.GpuGroupedAggregateIterator([Cc.host_batch(cols)], cols, [0], FINAL, est_groups=est,
                                       max_batch_rows=len(cols[0].data))
    with it:
        pieces = list(it)
        types = it.output_types
    return types, pieces


def check_against_complete(cols_raw, types, pieces):
    spec = A.Spec(cols_raw, [0], COMPLETE)
    o = Oracle(spec)
    o.update(Cc.host_batch(cols_raw))
    got = [np.concatenate([a[j][0][:n] for n, a in pieces]) for j in range(len(types))]
    gv = [Cc.pack_bits(np.concatenate([Cc.unpack_bits(a[j][1], n) for n, a in pieces])) for j in range(len(types))]
    n = sum(n for n, _ in pieces)
    bad, ex = compare_arrays(A.Spec(cols_raw, [0], FINAL), types, list(zip(got, gv)), n, o.output_types,
                             o.emit(ORC_FP_COMPENSATED), o.num_groups(), rtol=1e-11)
    assert bad == 0, ex
    assert len(np.unique(got[0])) == n  # no group emitted twice


def test_emit_and_reset_past_the_budget(cuda):
    cols, batches = rows_of_keys(1, 300_000, 60_000)
    it = I.GpuGroupedAggregateIterator(batches, cols, [0], PARTIAL, policy=I.EmitAndReset(1 << 20), est_groups=1024,
                                       max_batch_rows=8192)
    with it:
        pieces = list(it)
        types = it.output_types
        assert it.tables_emitted >= 2  # the budget was passed more than once
    assert sum(n for n, _ in pieces) > 60_000  # groups repeat across the emitted tables
    ftypes, fpieces = final_over(concat(types, pieces), 60_000)
    check_against_complete(cols, ftypes, fpieces)


def test_pass_through_when_the_input_does_not_reduce(cuda):
    cols, batches = rows_of_keys(2, 100_000, None)  # every row its own group
    it = I.GpuGroupedAggregateIterator(batches, cols, [0], PARTIAL,
                                       policy=I.EmitAndReset(256 << 10, pass_through_ratio=2.0), est_groups=1024,
                                       max_batch_rows=8192)
    with it:
        pieces = list(it)
        types = it.output_types
        assert it.pass_through
    ftypes, fpieces = final_over(concat(types, pieces), 100_000)
    check_against_complete(cols, ftypes, fpieces)


@pytest.mark.parametrize("pool", [False, True])
def test_grace_hash_final_past_the_budget(cuda, pool):
    cols, batches = rows_of_keys(3, 240_000, 50_000)
    # partial buffers of four tasks: the exchange's input to the Final
    pieces = []
    for t in range(4):
        with I.GpuGroupedAggregateIterator(batches[t::4], cols, [0], PARTIAL, est_groups=50_000,
                                           max_batch_rows=8192) as it:
            pieces += list(it)
            types = it.output_types
    buf = concat(types, pieces)
    chunks = [Cc.host_batch([Cc.Col(c.lane, c.data[lo:lo + 8192],
                                    None if c.validity is None else Cc.pack_bits(
                                        Cc.unpack_bits(c.validity, len(c.data))[lo:lo + 8192]),
                                    nullable=c.nullable) for c in buf])
              for lo in range(0, len(buf[0].data), 8192)]
    if pool:
        memory = I.AggregateMemory(I.HbmPool(512 << 10), min_refusal_bytes=0)
        policy = I.GraceHash(0, buckets=8)
    else:
        memory = None
        policy = I.GraceHash(1 << 20, buckets=8)
    it = I.GpuGroupedAggregateIterator(chunks, buf, [0], FINAL, policy=policy, est_groups=1024, max_batch_rows=8192,
                                       memory=memory)
    with it:
        out = list(it)
        otypes = it.output_types
        assert it.tables_emitted >= 1
    check_against_complete(cols, otypes, out)


def test_grace_hash_refuses_a_final_with_results_in_buffer_slots(cuda):
    cols, _ = rows_of_keys(4, 1000, 10)
    buf = [Cc.longs(np.zeros(1, np.int64), nullable=False), Cc.doubles(np.zeros(1)), Cc.longs(np.zeros(1))]
    with pytest.raises(ValueError):
        I.GpuGroupedAggregateIterator([], buf, [0], [A.AverageMergeAgg(1, 2, final_result=True)],
                                      policy=I.GraceHash(1 << 20))
