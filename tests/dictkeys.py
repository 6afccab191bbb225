"""Batches whose dictionary-encoded string key brings its own dictionary
(as Parquet row groups do), and the translation of emitted table ids back to
strings, so two aggregates with different id orders compare."""
import numpy as np

from vecruntime_b200 import columns as Cc

WORDS = ["AIR", "MAIL", "SHIP", "TRUCK", "RAIL", "FOB", "REG AIR", "", "é中", "x" * 40]


def dictionary_batches(seed, batches=4, rows=5000, null_rows=0.05, dict_size=0):
    """`batches` host batches of (string key with its own dictionary, int64
    key, int64 value, double value): every batch's dictionary lists the words
    in its own shuffled order, with entries no row uses and a null entry."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(batches):
        order = list(rng.permutation(len(WORDS)))
        entries = [WORDS[i] for i in order] + ["unused-%d" % b, None]
        pick = rng.integers(0, len(WORDS), rows)  # word index
        pos = {w: i for i, w in enumerate(order)}
        ids = np.array([pos[int(p)] for p in pick], np.int32)
        ids[rng.random(rows) < 0.03] = len(entries) - 1  # rows pointing at the null entry
        nulls = rng.random(rows) < null_rows
        cols = [Cc.dict_strings(ids, Cc.dictionary(entries), nulls, nullable=True, dict_size=dict_size),
                Cc.longs(rng.integers(0, 7, rows), nullable=False),
                Cc.longs(rng.integers(-1000, 1000, rows), nullable=False),
                Cc.doubles(rng.standard_normal(rows), nullable=False)]
        out.append(Cc.host_batch(cols))
    return out


def canonical(arrays, n, key, strings):
    """The emitted arrays with key column `key`'s table ids replaced by the
    position of their string in the sorted word list (nulls stay null)."""
    # one universe for both sides: a table may hold strings no row used (the
    # GPU maps every entry of a batch dictionary, the oracle the ones rows use)
    universe = sorted(set(w.encode() for w in WORDS) | {b"unused-%d" % b for b in range(64)} | set(strings))
    rank = {s: i for i, s in enumerate(universe)}
    ids = arrays[key][0][:n]
    mapped = np.array([rank[strings[int(i)]] for i in ids], np.int32) if n else np.zeros(0, np.int32)
    valid = Cc.unpack_bits(arrays[key][1], n)
    mapped[~valid] = 0
    out = list(arrays)
    out[key] = (mapped, arrays[key][1])
    return out
