"""Batches whose string key brings its own dictionary, on the GPU: the
handle maps each batch's entries onto its table dictionary
(GroupKeyTable.toIds, GroupKeyTable.java:1308-1430) and aggregates table
ids; the groups, translated back to strings through vr_agg_key_dictionary,
equal the oracle's. Hash tier (no declared size) and direct tier (a
declared size), host and device batches, null rows and null entries."""
import numpy as np
import pytest

import vecruntime_b200 as vr
from vecruntime_b200 import aggregate as A
from vecruntime_b200 import columns as Cc
from vecruntime_b200 import native as N

from dictkeys import canonical, dictionary_batches
from oracle.pyoracle import ORC_FP_COMPENSATED, Oracle
from parity import compare_arrays

pytestmark = pytest.mark.gpu

FNS = [A.CountAgg(), A.SumLongAgg(2), A.MinMaxAgg(2, True), A.MinMaxAgg(2, False), A.SumDoubleAgg(3)]


@pytest.mark.parametrize("dict_size,location", [(0, "host"), (16, "host"), (0, "device"), (16, "device")])
def test_batch_dictionaries_match_the_oracle(cuda, dict_size, location):
    batches = dictionary_batches(33, batches=5, dict_size=dict_size)
    keys = [0] if dict_size else [0, 1]  # the direct tier needs every key dictionary-encoded
    spec = A.Spec(batches[0].columns, keys, FNS)
    agg = vr.GpuHashAggregate(batches[0].columns, keys, FNS, est_groups=100, max_batch_rows=5000)
    keep = []
    try:
        st = agg.stats()
        assert (st.tier == 0) == (dict_size > 0)  # a declared size makes the key directly indexable
        for b in batches:
            if location == "device":
                db, t = Cc.to_device(b)
                keep.append(t)
                agg.consume(db)
            else:
                agg.consume(b)
        n = agg.num_groups()
        got = canonical(agg.emit(), n, 0, agg.key_dictionary(0))
        types = agg.output_types
    finally:
        agg.close()
    o = Oracle(spec)
    for b in batches:
        o.update(b)
    want = canonical(o.emit(ORC_FP_COMPENSATED), o.num_groups(), 0, o.key_dictionary(0))
    bad, ex = compare_arrays(spec, types, got, n, o.output_types, want, o.num_groups())
    assert bad == 0, ex


def test_a_declared_size_too_small_is_refused(cuda):
    """More distinct strings than the key's declared dictionary size cannot be
    indexed directly: the update is refused before anything runs."""
    batches = dictionary_batches(2, batches=1, dict_size=4)
    agg = vr.GpuHashAggregate(batches[0].columns, [0, 1], FNS, max_batch_rows=5000)
    try:
        with pytest.raises(vr.VrError) as e:
            agg.consume(batches[0])
        assert e.value.status == N.VR_ERR_INVALID
    finally:
        agg.close()


def test_reset_starts_a_new_table_dictionary(cuda):
    batches = dictionary_batches(9, batches=2)
    agg = vr.GpuHashAggregate(batches[0].columns, [0, 1], FNS, max_batch_rows=5000)
    try:
        agg.consume(batches[0])
        agg.num_groups()
        first = agg.key_dictionary(0)
        agg.reset()
        agg.consume(batches[1])
        n = agg.num_groups()
        second = agg.key_dictionary(0)
        d = batches[1].columns[0].dictionary
        order = [d.data[d.offsets[e]:d.offsets[e + 1]].tobytes() for e in range(d.size - 1)]
        assert second == order and sorted(first[:10]) == sorted(second[:10])
        assert n > 0
    finally:
        agg.close()
