"""GPU parity: libvrgpu (through the C ABI) against the CPU oracle on the
same seeded inputs, compared as sorted multisets of groups (tests/parity.py):
keys, counts, integer/decimal sums and min/max bit-exact; FP64 sums within
1e-12 relative of the oracle's compensated sum."""
import numpy as np
import pytest

import vecruntime_b200 as vr
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
