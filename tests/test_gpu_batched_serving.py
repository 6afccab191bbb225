"""GPU parity of the batched and serving entry points.

Batched: many uneven instances (rows 2^8..2^14, cardinality 1..2^12) in one
persistent launch, with and without CUDA-graph replay, and one launch per
instance; every instance's groups must equal the oracle's, on the first run
and on a replay (the run resets the tables).

Serving: several live queries whose requests arrive interleaved; each
query's result must equal the oracle's and the same query run alone."""
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


def oracle_of(w, batches):
    o = Oracle(w.spec())
    for b in batches:
        o.update(b)
    return o.output_types, o.emit(ORC_FP_COMPENSATED), o.num_groups()


def shared_choice():
    """One launch configuration for every instance (a batched launch needs it)."""
    t = N.TuneChoice()
    t.tier = 1
    t.threads = 256
    t.tile_rows = 1024
    t.smem_slots = 256
    return t


def test_reset_is_ordered_before_later_work(cuda):
    """vr_agg_reset only queues its clear on the handle's stream: updates and
    emits issued right after it, and a batched launch on another stream, must
    all see an empty table."""
    ws = G.batched_instances(n=6, max_log_rows=14, max_log_card=12)
    aggs, dbs, keep = [], [], []
    for w in ws:
        aggs.append(vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups,
                                        max_batch_rows=w.rows, tune=shared_choice()))
        db, t = Cc.to_device(w.batch())
        dbs.append(db)
        keep.append(t)
    try:
        for a, db in zip(aggs, dbs):
            a.consume(db)
            a.consume(db)
        for w, a, db in zip(ws, aggs, dbs):  # no sync between the clear and the next update
            a.reset()
            a.consume(db)
            n = a.num_groups()
            compare(w.spec(), a.output_types, a.emit(), n, *oracle_of(w, [w.batch()]))
        for a, db in zip(aggs, dbs):
            a.consume(db)
        for a in aggs:
            a.reset()
        b = vr.GpuBatchedAggregate(aggs, dbs, mode=N.VR_BATCHED_PERSISTENT)
        try:
            b.run()
            for w, a in zip(ws, aggs):
                n = a.num_groups()
                compare(w.spec(), a.output_types, a.emit(), n, *oracle_of(w, [w.batch()]))
        finally:
            b.close()
    finally:
        for a in aggs:
            a.close()


def _instances(n, max_log_rows=14, max_log_card=12, tune=None):
    ws = G.batched_instances(n=n, max_log_rows=max_log_rows, max_log_card=max_log_card)
    aggs, dbs, keep = [], [], []
    for w in ws:
        aggs.append(vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups,
                                        max_batch_rows=w.rows, tune=tune))
        db, t = Cc.to_device(w.batch())
        dbs.append(db)
        keep.append(t)
    return ws, aggs, dbs, keep


@pytest.mark.parametrize("mode,use_graph", [(N.VR_BATCHED_PERSISTENT, False), (N.VR_BATCHED_PERSISTENT, True),
                                            (N.VR_BATCHED_PLAIN, False)])
@pytest.mark.parametrize("own_choice", [True, False])
def test_batched_instances_match_the_oracle(cuda, mode, use_graph, own_choice):
    """Instances with their own launch choices (whole shared-memory tables for
    the small cardinalities, hot-key caches for the large ones) or one shared
    choice, in one persistent launch or one launch each."""
    ws, aggs, dbs, keep = _instances(24, tune=None if own_choice else shared_choice())
    b = vr.GpuBatchedAggregate(aggs, dbs, mode=mode, use_graph=use_graph)
    try:
        if mode == N.VR_BATCHED_PERSISTENT and own_choice:
            info = b.info()
            assert info["whole_tables"] > 0 and info["caches"] > 0, info
            assert info["whole_tables"] + info["caches"] + info["hbm_only"] == len(ws)
        for run in range(2):  # the second run replays (graph) and must reset the tables
            b.run()
            for w, a in zip(ws, aggs):
                n = a.num_groups()
                compare(w.spec(), a.output_types, a.emit(), n, *oracle_of(w, [w.batch()]))
    finally:
        b.close()
        for a in aggs:
            a.close()


@pytest.mark.parametrize("threads,tile,ctas,cache", [(128, 256, 2, 512), (256, 1024, 2, 0), (512, 512, 1, 1024)])
def test_batched_launch_shapes_match_the_oracle(cuda, threads, tile, ctas, cache):
    """The persistent launch's block shape is the caller's to choose (or the
    default); every shape must give the oracle's groups, growth included
    (cardinalities up to 2^15 against tables sized for far fewer)."""
    ws, aggs, dbs, keep = _instances(16, max_log_rows=16, max_log_card=15)
    shape = N.TuneChoice()
    shape.threads, shape.tile_rows, shape.blocks_per_sm, shape.smem_slots = threads, tile, ctas, cache
    b = vr.GpuBatchedAggregate(aggs, dbs, mode=N.VR_BATCHED_PERSISTENT, use_graph=True, shape=shape)
    try:
        info = b.info()
        assert info["threads"] == threads and info["tile_rows"] == tile
        b.run()
        for w, a in zip(ws, aggs):
            n = a.num_groups()
            compare(w.spec(), a.output_types, a.emit(), n, *oracle_of(w, [w.batch()]))
    finally:
        b.close()
        for a in aggs:
            a.close()


def test_batched_refuses_different_specs(cuda):
    """One persistent launch runs one kernel: instances whose specs differ
    (here fewer functions, so other accumulators) are refused."""
    ws = G.batched_instances(n=2, max_log_rows=12, max_log_card=4)
    aggs = [vr.GpuHashAggregate(ws[0].columns, ws[0].keys, ws[0].functions, max_batch_rows=ws[0].rows),
            vr.GpuHashAggregate(ws[1].columns, ws[1].keys, ws[1].functions[:3], max_batch_rows=ws[1].rows)]
    dbs, keep = [], []
    for w in ws:
        db, t = Cc.to_device(w.batch())
        dbs.append(db)
        keep.append(t)
    with pytest.raises(vr.VrError):
        vr.GpuBatchedAggregate(aggs, dbs)
    for a in aggs:
        a.close()


def test_serving_mix_equals_alone_and_the_oracle(cuda):
    rng = np.random.default_rng(77)
    queries = []
    for q, (card, rows) in enumerate([(50, 40_000), (5_000, 60_000), (300_000, 50_000)]):
        domain = rng.integers(-(1 << 62), 1 << 62, size=card, dtype=np.int64)
        k = domain[rng.integers(0, card, size=rows)]
        v1 = rng.integers(-10**6, 10**6, size=rows, dtype=np.int64)
        v2 = rng.standard_normal(rows)
        nulls = rng.random(rows) < 0.05
        cols = [Cc.longs(k, nullable=False), Cc.longs(v1, nulls, nullable=True), Cc.doubles(v2, nullable=False)]
        w = G.Workload(f"q{q}", cols, [0], [A.CountAgg(), A.CountAgg(1), A.SumLongAgg(1), A.MinMaxAgg(1, True),
                                           A.MinMaxAgg(1, False), A.SumDoubleAgg(2)], card, rows)
        chunks = [w.batch(lo, min(rows, lo + 8192)) for lo in range(0, rows, 8192)]
        queries.append((w, chunks))
    srv = vr.AggregateServer(slots=4, hbm_cap_bytes=8 << 30)
    try:
        qids = [srv.open_query(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=8192)
                for w, _ in queries]
        tickets = []
        longest = max(len(c) for _, c in queries)
        for i in range(longest):  # interleaved arrivals
            for qid, (w, chunks) in zip(qids, queries):
                if i < len(chunks):
                    tickets.append(srv.submit(qid, chunks[i]))
        lat = [srv.wait(t) for t in tickets]
        assert all(x >= 0 for x in lat)
        for qid, (w, chunks) in zip(qids, queries):
            types, arrays, n = srv.results(qid)
            want = oracle_of(w, chunks)
            compare(w.spec(), types, arrays, n, *want)
            alone = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=8192)
            for c in chunks:
                alone.consume(c)
            compare(w.spec(), types, arrays, n, alone.output_types, alone.emit(), alone.num_groups())
            alone.close()
        st = srv.stats()
        assert st.completed == len(tickets) and st.rejected == 0
        # requests of different queries were on the device at the same time
        # (admitted and not yet complete), not drained one at a time
        assert st.max_in_flight > 1, st.max_in_flight
        # the latency splits into waiting for admission and running on the device
        assert 0 <= st.p99_wait_ms <= st.max_ms and 0 < st.p99_service_ms <= st.max_ms
    finally:
        srv.close()


def test_serving_accounts_for_table_growth(cuda):
    """A query whose table grows past its estimate holds more HBM: the
    server's footprint follows the table, not the size it opened with."""
    rng = np.random.default_rng(5)
    rows = 200_000
    cols = [Cc.longs(rng.integers(-(1 << 62), 1 << 62, rows, dtype=np.int64), nullable=False),
            Cc.longs(rng.integers(0, 100, rows, dtype=np.int64), nullable=False),
            Cc.doubles(rng.standard_normal(rows), nullable=False)]
    w = G.Workload("grow", cols, [0], [A.CountAgg(), A.SumLongAgg(1), A.SumDoubleAgg(2)], 1024, rows)
    srv = vr.AggregateServer(slots=4, hbm_cap_bytes=8 << 30)
    try:
        qid = srv.open_query(w.columns, w.keys, w.functions, est_groups=1024, max_batch_rows=20_000)
        tickets = [srv.submit(qid, w.batch(lo, lo + 20_000)) for lo in range(0, rows, 20_000)]
        for t in tickets:
            srv.wait(t)
        types, arrays, n = srv.results(qid)
        assert n == rows  # every key distinct: the table grew well past 1,024 groups
        compare(w.spec(), types, arrays, n, *oracle_of(w, [w.batch()]))
        st = srv.stats()
        # 200,000 groups need a table of 2^19 slots of 48 bytes (25 MB); what the
        # query held at open (staging for 20,000 rows, 2,048 slots) is under 4 MB
        assert st.hbm_peak > n * 40, st.hbm_peak
    finally:
        srv.close()


def test_batched_autotuner_keeps_results_and_records_its_choices(cuda):
    """vr_batched_tune picks each estimated-groups bucket's strategy by timing
    the launch; the results stay the oracle's, and handles created afterwards
    find the tuner's choice for their (spec, rows, groups) bucket."""
    import ctypes as C

    ws, aggs, dbs, keep = _instances(24, max_log_rows=15, max_log_card=13)
    b = vr.GpuBatchedAggregate(aggs, dbs, mode=N.VR_BATCHED_PERSISTENT, use_graph=True)
    try:
        ms = b.tune(iters=1)
        assert ms > 0
        info = b.info()
        assert info["whole_tables"] + info["caches"] + info["hbm_only"] == len(ws)
        b.run()
        for w, a in zip(ws, aggs):
            n = a.num_groups()
            compare(w.spec(), a.output_types, a.emit(), n, *oracle_of(w, [w.batch()]))
        choice = N.TuneChoice()
        w = ws[0]
        assert N.lib().vr_tune_lookup(C.byref(w.spec().spec), w.rows, C.byref(choice)) == 1
        assert choice.tier in (1, 2)
    finally:
        b.close()
        for a in aggs:
            a.close()
