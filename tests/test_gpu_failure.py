"""Failure detection without a GPU fault: every barrier wait in the aggregate
kernel is bounded. With the test hook that stops the producer warp before it
issues any copy (VRGPU_TEST_STALL_PRODUCER) and a short poll budget
(VRGPU_TEST_WAIT_POLLS), the consumers' waits run out, the kernel records
the timeout and returns, the host reports VR_ERR_TIMEOUT for that handle,
and the next handle on the same device runs normally."""
import time

import pytest

import vecruntime_b200 as vr
from vecruntime_b200 import columns as Cc
from vecruntime_b200 import datagen as G
from vecruntime_b200 import native as N

from oracle.pyoracle import ORC_FP_COMPENSATED, Oracle
from parity import compare

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("workload", ["decimal", "plain"])
def test_a_wait_that_nothing_satisfies_returns_timeout(cuda, workload, monkeypatch):
    w = G.decimal_report(rows=50_000) if workload == "decimal" else G.plain(rows=50_000)
    db, keep = Cc.to_device(w.batch())
    monkeypatch.setenv("VRGPU_TEST_STALL_PRODUCER", "1")
    monkeypatch.setenv("VRGPU_TEST_WAIT_POLLS", "16")
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=w.rows)
    t0 = time.time()
    with pytest.raises(vr.VrError) as e:
        agg.consume(db)
        agg.sync()
    assert e.value.status == N.VR_ERR_TIMEOUT
    assert time.time() - t0 < 10, "the bounded wait took too long"
    with pytest.raises(vr.VrError) as dead:  # the handle is dead after the error
        agg.consume(db)
    assert dead.value.status == N.VR_ERR_STATE
    agg.close()
    # the context is still usable: a fresh handle aggregates correctly
    monkeypatch.delenv("VRGPU_TEST_STALL_PRODUCER")
    monkeypatch.delenv("VRGPU_TEST_WAIT_POLLS")
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=w.rows)
    agg.consume(db)
    n = agg.num_groups()
    o = Oracle(w.spec())
    o.update(w.batch())
    compare(w.spec(), agg.output_types, agg.emit(), n, o.output_types, o.emit(ORC_FP_COMPENSATED), o.num_groups())
    agg.close()
    cuda.cuda.synchronize()
