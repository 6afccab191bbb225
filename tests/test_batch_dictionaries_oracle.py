"""Batches whose string key brings its own dictionary, on CPU: the oracle's
mapping of every batch's entries onto one table dictionary
(GroupKeyTable.toIds, GroupKeyTable.java:1308-1430) against an independent
Python computation over the strings themselves: batches whose dictionaries
list the same strings in different orders, with unused and null entries,
give the groups of the strings."""
from collections import defaultdict

import numpy as np

from dictkeys import dictionary_batches
from oracle.pyoracle import ORC_FP_COMPENSATED, Oracle
from vecruntime_b200 import aggregate as A
from vecruntime_b200 import columns as Cc

FNS = [A.CountAgg(), A.SumLongAgg(2), A.MinMaxAgg(2, True), A.MinMaxAgg(2, False)]


def test_batches_with_their_own_dictionaries_group_by_string():
    batches = dictionary_batches(21)
    o = Oracle(A.Spec(batches[0].columns, [0, 1], FNS))
    want = defaultdict(lambda: [0, 0, None, None])
    for b in batches:
        o.update(b)
        key = b.columns[0]
        d = key.dictionary
        valid = Cc.unpack_bits(key.validity, b.num_rows)
        dvalid = Cc.unpack_bits(d.validity, d.size) if d.validity is not None else np.ones(d.size, bool)
        for i in range(b.num_rows):
            e = int(key.data[i])
            s = d.data[d.offsets[e]:d.offsets[e + 1]].tobytes() if valid[i] and dvalid[e] else None
            g = want[(s, int(b.columns[1].data[i]))]
            v = int(b.columns[2].data[i])
            g[0] += 1
            g[1] += v
            g[2] = v if g[2] is None else min(g[2], v)
            g[3] = v if g[3] is None else max(g[3], v)
    n = o.num_groups()
    out = o.emit(ORC_FP_COMPENSATED)
    strings = o.key_dictionary(0)
    assert set(strings) <= set(k[0] for k in want if k[0] is not None)
    got = {}
    kvalid = Cc.unpack_bits(out[0][1], n)
    for g in range(n):
        s = strings[int(out[0][0][g])] if kvalid[g] else None
        got[(s, int(out[1][0][g]))] = [int(out[2][0][g]), int(out[3][0][g]), int(out[4][0][g]), int(out[5][0][g])]
    assert got == {k: v for k, v in want.items()}


def test_same_strings_any_dictionary_order_same_result():
    """One batch per dictionary order, or every row re-encoded against one
    shared dictionary: the same groups, string for string."""
    batches = dictionary_batches(5, batches=3)
    shared = sorted({w for b in batches for w in
                     [b.columns[0].dictionary.data[b.columns[0].dictionary.offsets[e]:
                                                   b.columns[0].dictionary.offsets[e + 1]].tobytes()
                      for e in range(b.columns[0].dictionary.size)]})
    one = Oracle(A.Spec(batches[0].columns, [0, 1], FNS))
    sep = Oracle(A.Spec(batches[0].columns, [0, 1], FNS))
    for b in batches:
        sep.update(b)
        d = b.columns[0].dictionary
        dvalid = Cc.unpack_bits(d.validity, d.size) if d.validity is not None else np.ones(d.size, bool)
        remap = np.array([shared.index(d.data[d.offsets[e]:d.offsets[e + 1]].tobytes()) if dvalid[e] else -1
                          for e in range(d.size)])
        ids = remap[b.columns[0].data]
        nulls = ~Cc.unpack_bits(b.columns[0].validity, b.num_rows) | (ids < 0)
        shared_dict = Cc.dictionary([s.decode() for s in shared])
        cols = [Cc.dict_strings(np.where(ids < 0, 0, ids), shared_dict, nulls, nullable=True)] + b.columns[1:]
        one.update(Cc.host_batch(cols))

    def rows(o):
        n = o.num_groups()
        out = o.emit(ORC_FP_COMPENSATED)
        strs = o.key_dictionary(0)
        kv = Cc.unpack_bits(out[0][1], n)
        return sorted(((strs[int(out[0][0][g])] if kv[g] else b""), int(out[1][0][g]),
                       tuple(int(out[j][0][g]) for j in range(2, 6))) for g in range(n))

    assert rows(one) == rows(sep)
