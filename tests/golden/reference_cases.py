"""The reference's own aggregation tests, regenerated as golden cases.

The reference keeps no golden files for this path: each of its kernel tests
draws inputs from a seeded java.util.Random and computes the expected
answers inside the test with plain Java (a HashMap of running values,
BigInteger sums, CompareOp.nanSafeCompare). Each case below restates one of
those tests: the same seed, the same draw order, the same batch lengths, and
the same expectation logic, written out per group in the output schema of
this library's functions (Spark buffer columns). Literal known answers from
the reference tests are cases too.

A case holds the input batches (host Arrow layout), the spec (columns, key
columns, functions) and the expected rows (keys first, then each function's
output columns), with a role per output column saying how it compares:
  key / int / dec / bool   exact
  exact                    min/max doubles: NaN == NaN, -0.0 == 0.0
                           (CompareOp.nanSafeCompare, CompareOp.java:68-81)
  fsum                     FP64 sums: the expected value is the reference's
                           sequential per-group `sum += x` in row order
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

from vecruntime_b200 import aggregate as A
from vecruntime_b200 import columns as Cc

from .jrandom import JavaRandom, bit_length, random_biginteger, string_hash

INT_MIN, INT_MAX = -(1 << 31), (1 << 31) - 1
LONG_MIN, LONG_MAX = -(1 << 63), (1 << 63) - 1
MAX_DECIMAL38 = 10 ** 38 - 1
# TestData.LENGTHS (kernels/src/test/java/io/vecruntime/kernels/TestData.java:27-46)
LENGTHS = [0, 1, 3, 7, 8, 15, 16, 31, 63, 64, 65, 100, 127, 128, 129, 1000, 1023, 4097]


@dataclass
class Case:
    name: str
    source: str                 # reference test, file:line
    columns: list               # Col per input column (types of the spec)
    keys: List[int]
    functions: list
    batches: list               # HostBatch per reference batch
    expected: list              # rows: (keys..., outputs...)
    roles: List[str]
    fsum_tol: Optional[Callable[[float], float]] = None  # |got - want| bound for "fsum" columns on the GPU
    notes: str = ""
    meta: Dict = field(default_factory=dict)

    def spec(self, **kw) -> A.Spec:
        rows = max([b.num_rows for b in self.batches] + [1])
        return A.Spec(self.columns, self.keys, self.functions, max_batch_rows=rows, **kw)


# ------------------------------------------------------------ helpers
def nan_safe_compare(x: float, y: float) -> int:
    """CompareOp.nanSafeCompare (CompareOp.java:68-81)."""
    xn, yn = math.isnan(x), math.isnan(y)
    if (xn and yn) or x == y:
        return 0
    if xn:
        return 1
    if yn:
        return -1
    return 1 if x > y else -1


def random_bitmap(rnd: JavaRandom, n: int) -> List[bool]:
    """TestData.randomBitmap (TestData.java:139-147): one nextBoolean per row."""
    return [rnd.nextBoolean() for _ in range(n)]


def random_decimal128(rnd: JavaRandom) -> int:
    """TestData.randomDecimal128 (TestData.java:95-118)."""
    c = rnd.nextInt(12)
    if c == 0:
        return MAX_DECIMAL38
    if c == 1:
        return -MAX_DECIMAL38
    if c == 2:
        return -(1 << 127)
    if c == 3:
        return LONG_MIN
    if c == 4:
        return LONG_MIN << 64
    if c == 5:
        return LONG_MAX + 1
    if c == 6:
        return 0
    if c == 7:
        return rnd.nextInt(2000) - 1000
    bits = rnd.nextInt(127)
    mag = random_biginteger(bits, rnd)
    return mag * (1 if rnd.nextBoolean() else -1)


def java_nulls(rnd: JavaRandom, n: int, fraction: float) -> List[bool]:
    """TestData.nulls (TestData.java:50-56)."""
    return [rnd.nextDouble() < fraction for _ in range(n)]


def bitmap(mask) -> Optional[np.ndarray]:
    return None if mask is None else Cc.pack_bits(np.asarray(mask, dtype=bool))


class Dictionary:
    """UTF8 keys as dictionary ids in first-seen order (the library takes
    string keys as VR_DICT32 ids; GroupKeyTable keeps strings as ids too,
    GroupKeyTable.java:27-36)."""

    def __init__(self):
        self.ids: Dict[str, int] = {}

    def encode(self, values):
        out = []
        for s in values:
            if s is None:
                out.append(0)
            else:
                out.append(self.ids.setdefault(s, len(self.ids)))
        return out


def seq_sum(values) -> float:
    s = 0.0
    for v in values:
        s += v
    return s


# ------------------------------------------- GroupedAggregationTest cases
def grouped_accumulators(cardinality: int, with_selection: bool) -> Case:
    """GroupedAggregationTest.groupedAccumulatorsMatchReference / ...HonourSelection
    (GroupedAggregationTest.java:59-193): INT32 + UTF8 keys with null keys,
    count(*), count(v), sum(double), sum(long), min/max(double) with NaN."""
    rnd = JavaRandom(cardinality)
    d = Dictionary()
    batches = []
    ref: Dict[tuple, dict] = {}
    for n in (1000, 37, 2048, 64, 999):
        k1, k2, vals, lvals, key_nulls, val_nulls = [], [], [], [], [], []
        for _ in range(n):
            g = rnd.nextInt(cardinality)
            a = g % 7
            b = None if g % 13 == 0 else "k" + str(g // 7)
            kn = a == 3 and rnd.nextInt(5) == 0  # `&&` draws only when k1 == 3
            v = math.nan if rnd.nextInt(6) == 0 else rnd.nextInt(-100, 100) / 4.0
            lv = rnd.nextInt(-1000, 1000)
            vn = rnd.nextInt(4) == 0
            k1.append(a), k2.append(b), vals.append(v), lvals.append(lv), key_nulls.append(kn), val_nulls.append(vn)
        sel = random_bitmap(rnd, n) if with_selection else None
        cols = [Cc.ints(k1, key_nulls, nullable=True),
                Cc.dict_ids(d.encode(k2), 0, [s is None for s in k2], nullable=True),
                Cc.doubles(vals, val_nulls, nullable=True),
                Cc.longs(lvals, val_nulls, nullable=True)]
        batches.append(Cc.HostBatch(cols, n, bitmap(sel)))
        for i in range(n):
            if sel is not None and not sel[i]:
                continue
            key = (None if key_nulls[i] else k1[i], None if k2[i] is None else d.ids[k2[i]])
            r = ref.setdefault(key, {"rows": 0, "count": 0, "sum": 0.0, "lsum": 0, "min": None, "max": None})
            r["rows"] += 1
            if not val_nulls[i]:
                x = vals[i]
                r["count"] += 1
                r["sum"] += x
                r["lsum"] += lvals[i]
                if r["min"] is None or nan_safe_compare(x, r["min"]) < 0:
                    r["min"] = x
                if r["max"] is None or nan_safe_compare(x, r["max"]) > 0:
                    r["max"] = x
    fns = [A.CountAgg(), A.CountAgg(2), A.SumDoubleAgg(2), A.SumLongAgg(3), A.MinMaxAgg(2, True),
           A.MinMaxAgg(2, False)]
    expected = []
    for key, r in ref.items():
        some = r["count"] > 0
        expected.append(key + (r["rows"], r["count"], r["sum"] if some else None, r["lsum"] if some else None,
                               r["min"], r["max"]))
    return Case(f"grouped_accumulators[card={cardinality},sel={int(with_selection)}]",
                "GroupedAggregationTest.java:59-193", batches[0].columns, [0, 1], fns, batches, expected,
                ["key", "key", "int", "int", "fsum", "int", "exact", "exact"],
                fsum_tol=lambda want: 1e-9)


def strict_double_sum(cardinality: int) -> Case:
    """GroupedAggregationTest.strictDoubleSumIsBitIdenticalToSequentialReference
    (GroupedAggregationTest.java:201-244): per-group sequential sums of mixed
    magnitudes (up to 1e15) with nulls and, on even lengths, a selection."""
    rnd = JavaRandom(7 * cardinality + 1)
    batches = []
    sums: Dict[int, float] = {}
    counts: Dict[int, int] = {}
    rows: Dict[int, int] = {}
    for n in (1000, 37, 2048, 64, 999, 4097):
        ids, vals, nulls = [], [], []
        for _ in range(n):
            ids.append(rnd.nextInt(cardinality))
            sign = 1 if rnd.nextBoolean() else -1
            x = sign * rnd.nextDouble()
            vals.append(x * (10.0 ** rnd.nextInt(16)))
            nulls.append(rnd.nextInt(5) == 0)
        sel = random_bitmap(rnd, n) if n % 2 == 0 else None
        batches.append(Cc.HostBatch([Cc.ints(ids, nullable=False), Cc.doubles(vals, nulls, nullable=True)], n,
                                    bitmap(sel)))
        for i in range(n):
            if sel is not None and not sel[i]:
                continue
            g = ids[i]
            rows[g] = rows.get(g, 0) + 1
            if not nulls[i]:
                sums[g] = sums.get(g, 0.0) + vals[i]
                counts[g] = counts.get(g, 0) + 1
    fns = [A.CountAgg(), A.SumDoubleAgg(1), A.CountAgg(1)]
    expected = [(g, rows[g], sums.get(g) if counts.get(g) else None, counts.get(g, 0)) for g in rows]
    return Case(f"strict_double_sum[card={cardinality}]", "GroupedAggregationTest.java:201-244",
                batches[0].columns, [0], fns, batches, expected, ["key", "int", "fsum", "int"],
                fsum_tol=lambda want: abs(want) * 1e-12 + 1e-9)


def wide_decimal_keys() -> Case:
    """GroupedAggregationTest.wideDecimalKeysGroupByBothLimbs
    (GroupedAggregationTest.java:246-348): DECIMAL128 keys that share one limb
    and differ in the other, plus an INT32 key; min/max/count of a DECIMAL128
    value column against BigInteger. Groups come from every row (the test
    assigns keys without the selection); values count only on selected,
    non-null rows, so here the selection is folded into the value validity."""
    rnd = JavaRandom(128)
    pool: List[int] = []
    for i in range(40):
        base = random_decimal128(rnd) if i < 8 else pool[i % 8]
        c = i // 8
        v = base if c == 0 else base + (1 << 64) if c == 1 else base ^ 1 if c == 2 else -base if c == 3 else base << 1
        if bit_length(v) > 127:
            v >>= 2
        pool.append(v)
    batches = []
    ref: Dict[tuple, dict] = {}
    for n in (1000, 37, 2048, 64, 999):
        k1, k2, knull = [], [], []
        for _ in range(n):
            k1.append(pool[rnd.nextInt(len(pool))])
            k2.append(rnd.nextInt(3))
            knull.append(rnd.nextInt(11) == 0)
        vals, vnull = [], []
        for _ in range(n):
            vals.append(random_decimal128(rnd))
            vnull.append(rnd.nextInt(4) == 0)
        sel = random_bitmap(rnd, n) if n % 2 == 0 else None
        counted = [not vnull[i] and (sel is None or sel[i]) for i in range(n)]
        cols = [Cc.decimals128(k1, 38, 0, knull, nullable=True),  # values stay under the nulls
                Cc.ints(k2, nullable=False),
                Cc.decimals128(vals, 38, 0, [not c for c in counted], nullable=True)]
        batches.append(Cc.HostBatch(cols, n, None))
        for i in range(n):
            key = (None if knull[i] else k1[i], k2[i])
            r = ref.setdefault(key, {"min": None, "max": None, "count": 0})
            if counted[i]:
                r["count"] += 1
                r["min"] = vals[i] if r["min"] is None else min(r["min"], vals[i])
                r["max"] = vals[i] if r["max"] is None else max(r["max"], vals[i])
    fns = [A.MinMaxAgg(2, True), A.MinMaxAgg(2, False), A.CountAgg(2)]
    expected = [key + (r["min"], r["max"], r["count"]) for key, r in ref.items()]
    return Case("wide_decimal_keys", "GroupedAggregationTest.java:246-348", batches[0].columns, [0, 1], fns,
                batches, expected, ["key", "key", "dec", "dec", "int"])


def wide_long_sum(grouped: bool) -> Case:
    """GroupedAggregationTest.wideLongSumIsExactPast64Bits
    (GroupedAggregationTest.java:831-888): 18-digit values of either sign and
    Long.MIN_VALUE extremes summed exactly past 64 bits (WideLongSum), per
    group under a selection, and ungrouped over every non-null row."""
    rnd = JavaRandom(128)
    groups = 5
    ref = [0] * groups
    ref_count = [0] * groups
    ref_rows = [0] * groups
    ref_all = 0
    all_count = 0
    all_rows = 0
    batches = []
    for n in (1000, 37, 2048, 64, 999):
        vals, nulls, ids = [], [], []
        for i in range(n):
            sign = 1 if rnd.nextBoolean() else -1
            v = sign * (900_000_000_000_000_000 - rnd.nextInt(1_000_000))
            if i % 97 == 5:
                v = LONG_MIN + rnd.nextInt(10)
            vals.append(v)
            nulls.append(rnd.nextInt(9) == 0)
            ids.append(rnd.nextInt(groups))
        sel = random_bitmap(rnd, n)
        for i in range(n):
            all_rows += 1
            if not nulls[i]:
                ref_all += vals[i]
                all_count += 1
            if sel[i]:
                ref_rows[ids[i]] += 1
                if not nulls[i]:
                    ref[ids[i]] += vals[i]
                    ref_count[ids[i]] += 1
        # a plain INT64 lane (precision 0): the values use the whole long range
        v = Cc.longs(vals, nulls, nullable=True)
        if grouped:
            batches.append(Cc.HostBatch([Cc.ints(ids, nullable=False), v], n, bitmap(sel)))
        else:
            batches.append(Cc.HostBatch([v], n, None))
    if grouped:
        fns = [A.WideDecimalSumAgg(1, 38, 0), A.CountAgg(1), A.CountAgg()]
        expected = [(g, ref[g], ref_count[g] == 0, ref_count[g], ref_rows[g]) for g in range(groups) if ref_rows[g]]
        return Case("wide_long_sum[grouped]", "GroupedAggregationTest.java:831-880", batches[0].columns, [0], fns,
                    batches, expected, ["key", "dec", "bool", "int", "int"],
                    meta={"left_long_range": any(abs(x) >= 1 << 63 for x in ref)})
    fns = [A.WideDecimalSumAgg(0, 38, 0), A.CountAgg(0), A.CountAgg()]
    expected = [(ref_all, all_count == 0, all_count, all_rows)]
    return Case("wide_long_sum[ungrouped]", "GroupedAggregationTest.java:831-882", batches[0].columns, [], fns,
                batches, expected, ["dec", "bool", "int", "int"], meta={"left_long_range": abs(ref_all) >= 1 << 63})


# ------------------------------------------------ literal known answers
def known_wide_sum_int32() -> Case:
    """GroupedAggregationTest.java:884-898: INT32 lanes summed exactly:
    MAX + MIN = -1, 7 + -7 = 0, 1 + null = 1 (count 1)."""
    ints = [INT_MAX, INT_MIN, 7, -7, 1, 0]
    nulls = [False, False, False, False, False, True]
    ids = [0, 0, 1, 1, 2, 2]
    cols = [Cc.ints(ids, nullable=False), Cc.ints(ints, nulls, nullable=True)]
    fns = [A.WideDecimalSumAgg(1, 38, 0), A.CountAgg(1), A.SumLongAgg(1)]
    expected = [(0, -1, False, 2, -1), (1, 0, False, 2, 0), (2, 1, False, 1, 1)]
    return Case("known_wide_sum_int32", "GroupedAggregationTest.java:884-898", cols, [0], fns,
                [Cc.HostBatch(cols, 6, None)], expected, ["key", "dec", "bool", "int", "int"])


def known_null_vs_zero_keys() -> Case:
    """GroupedAggregationTest.longKeysAndBooleanKeysDistinguishNullFromZero
    (GroupedAggregationTest.java:781-799): 4 groups, a null key is not 0."""
    cols = [Cc.longs([0, 0, 1 << 40, 0], [False, True, False, False], nullable=True),
            Cc.bools([False, False, True, False], [False, False, False, True], nullable=True)]
    expected = [(0, False, 1), (None, False, 1), (1 << 40, True, 1), (0, None, 1)]
    return Case("known_null_vs_zero_keys", "GroupedAggregationTest.java:781-799", cols, [0, 1], [A.CountAgg()],
                [Cc.HostBatch(cols, 4, None)], expected, ["key", "key", "int"])


def known_write_keys_layout() -> Case:
    """GroupedAggregationTest.writeKeysProducesArrowLayoutColumns
    (GroupedAggregationTest.java:801-829): (5, "xx") twice, (6, "y"),
    (null, null): 3 groups."""
    d = Dictionary()
    k2 = ["xx", "y", "xx", None]
    cols = [Cc.ints([5, 6, 5, 7], [False, False, False, True], nullable=True),
            Cc.dict_ids(d.encode(k2), 0, [s is None for s in k2], nullable=True)]
    expected = [(5, d.ids["xx"], 2), (6, d.ids["y"], 1), (None, None, 1)]
    return Case("known_write_keys_layout", "GroupedAggregationTest.java:801-829", cols, [0, 1], [A.CountAgg()],
                [Cc.HostBatch(cols, 4, None)], expected, ["key", "key", "int"])


def known_memoised_dictionary_keys() -> Case:
    """GroupedAggregationTest.memoisedDictionaryKeysMatchPlainKeys
    (GroupedAggregationTest.java:360-426): two dictionary-encoded keys
    (dictionaries R,A,N and O,F) with nulls; the dictionary ids are the
    test's own, so the keys take the direct (memoised) path: 7 groups."""
    flag_ids = [1, 2, 0, 2, 0, 1, 0, 0]
    flag_null = [False, False, False, False, True, False, False, False]
    status_ids = [1, 0, 1, 1, 0, 0, 0, 1]
    status_null = [False, False, False, False, False, True, False, False]
    cols = [Cc.dict_ids(flag_ids, 3, flag_null, nullable=True), Cc.dict_ids(status_ids, 2, status_null, nullable=True)]
    counts: Dict[tuple, int] = {}
    for i in range(8):
        key = (None if flag_null[i] else flag_ids[i], None if status_null[i] else status_ids[i])
        counts[key] = counts.get(key, 0) + 1
    expected = [k + (c,) for k, c in counts.items()]
    assert len(expected) == 7
    return Case("known_memoised_dictionary_keys", "GroupedAggregationTest.java:360-426", cols, [0, 1],
                [A.CountAgg()], [Cc.HostBatch(cols, 8, None)], expected, ["key", "key", "int"])


def known_record_strings() -> Case:
    """GroupedAggregationTest.aTableBuiltForRecordsKeepsStringKeysAsBytesFromTheStart
    (GroupedAggregationTest.java:617-660): 50 names x 3 ints plus (null, int)
    for the three ints: 153 groups from 500 rows."""
    n = 500
    d = Dictionary()
    names = [None if i % 7 == 6 else f"name {i % 50} long enough not to pack into a long" for i in range(n)]
    ints = [i % 3 for i in range(n)]
    cols = [Cc.dict_ids(d.encode(names), 0, [s is None for s in names], nullable=True), Cc.ints(ints, nullable=False)]
    counts: Dict[tuple, int] = {}
    for i in range(n):
        key = (None if names[i] is None else d.ids[names[i]], ints[i])
        counts[key] = counts.get(key, 0) + 1
    expected = [k + (c,) for k, c in counts.items()]
    assert len(expected) == 153
    return Case("known_record_strings", "GroupedAggregationTest.java:617-660", cols, [0, 1], [A.CountAgg()],
                [Cc.HostBatch(cols, n, None)], expected, ["key", "key", "int"])


def known_high_cardinality_strings() -> Case:
    """GroupedAggregationTest.highCardinalityPlainStringsGroupByIdsAndEmitFromTheDictionary
    (GroupedAggregationTest.java:510-555): 1000 strings x 3 ints = 3000
    groups, then the same strings with int 7 add 1000 more."""
    n = 3000
    d = Dictionary()
    comments = [f"comment number {i % 1000} of a high-cardinality column" for i in range(n)]
    ids = d.encode(comments)
    b1 = [Cc.dict_ids(ids, 0, nullable=False), Cc.ints([i % 3 for i in range(n)], nullable=False)]
    b2 = [Cc.dict_ids(ids, 0, nullable=False), Cc.ints([7] * n, nullable=False)]
    expected = [(ids[i], i % 3, 1) for i in range(n)] + [(ids[i], 7, 3) for i in range(1000)]
    return Case("known_high_cardinality_strings", "GroupedAggregationTest.java:510-555", b1, [0, 1], [A.CountAgg()],
                [Cc.HostBatch(b1, n, None), Cc.HostBatch(b2, n, None)], expected, ["key", "key", "int"])


def known_nan_handling() -> List[Case]:
    """AggKernelsTest.nanHandlingFollowsSpark (AggKernelsTest.java:123-143):
    min ignores NaN unless every value is NaN, max is NaN when any value is,
    a NaN in a null slot is ignored."""
    nan = math.nan
    out = []
    fns = [A.MinMaxAgg(0, True), A.MinMaxAgg(0, False), A.SumDoubleAgg(0), A.CountAgg(0)]
    roles = ["exact", "exact", "fsum", "int"]
    for name, vals, nulls, want in (
            ("mixed", [3.0, nan, 1.0, 2.0, nan], None, (1.0, nan, nan, 5)),
            ("all_nan", [nan, nan, nan], None, (nan, nan, nan, 3)),
            ("null_nan", [nan, 5.0, 7.0], [True, False, False], (5.0, 7.0, 12.0, 2))):
        cols = [Cc.doubles(vals, nulls, nullable=True)]
        out.append(Case(f"known_nan_handling[{name}]", "AggKernelsTest.java:123-143", cols, [], fns,
                        [Cc.HostBatch(cols, len(vals), None)], [want], roles, fsum_tol=lambda want: 0.0))
    return out


def known_sequential_running_sum() -> Case:
    """AggKernelsTest.sequentialDoubleSumIsSparksRunningSum
    (AggKernelsTest.java:145-170): 1000 values whose sum depends on the
    order of addition, every 7th null; the running sum from 0 in row order."""
    vals = [1.0 / (i % 10 + 1) * (1e10 if i % 3 == 0 else 1.0) for i in range(1000)]
    nulls = [i % 7 == 0 for i in range(1000)]
    cols = [Cc.doubles(vals, nulls, nullable=True)]
    want = seq_sum(v for v, z in zip(vals, nulls) if not z)
    return Case("known_sequential_running_sum", "AggKernelsTest.java:145-170", cols, [], [A.SumDoubleAgg(0)],
                [Cc.HostBatch(cols, 1000, None)], [(want,)], ["fsum"], fsum_tol=lambda w: abs(w) * 1e-12)


# ------------------------------------------------------ AggKernelsTest
def _ungrouped_rows(vals, nulls):
    return [v for v, z in zip(vals, nulls) if not z]


def agg_kernel_sums() -> List[Case]:
    """AggKernelsTest.sumsMatchReferenceWithAndWithoutNulls
    (AggKernelsTest.java:39-64): countValid, sum(double), sum(int),
    sum(long) over TestData.LENGTHS x null fractions, ungrouped (one
    group per input; a length-0 input is skipped: the reference checks no
    group there)."""
    rnd = JavaRandom(21)
    out = []
    for n in LENGTHS:
        for frac in (0.0, 0.01, 0.3, 1.0):
            nulls = java_nulls(rnd, n, frac)
            dv, iv, lv = [], [], []
            for _ in range(n):
                dv.append(rnd.nextInt(-1000, 1000) / 8.0)
                iv.append(rnd.nextInt())
                lv.append(rnd.nextLong(-(1 << 40), 1 << 40))
            if n == 0:
                continue
            cols = [Cc.doubles(dv, nulls, nullable=True), Cc.ints(iv, nulls, nullable=True),
                    Cc.longs(lv, nulls, nullable=True)]
            valid = [not z for z in nulls]
            c = sum(valid)
            some = c > 0
            want = (c, seq_sum(_ungrouped_rows(dv, nulls)) if some else None,
                    sum(_ungrouped_rows(iv, nulls)) if some else None,
                    sum(_ungrouped_rows(lv, nulls)) if some else None)
            fns = [A.CountAgg(0), A.SumDoubleAgg(0), A.SumLongAgg(1), A.SumLongAgg(2)]
            out.append(Case(f"agg_kernel_sums[n={n},nulls={frac}]", "AggKernelsTest.java:39-64", cols, [], fns,
                            [Cc.HostBatch(cols, n, None)], [want], ["int", "fsum", "int", "int"],
                            fsum_tol=lambda w: abs(w) * 1e-12))
    return out


def agg_kernel_sequential_sums() -> List[Case]:
    """AggKernelsTest.sequentialSumIsBitIdenticalToReference
    (AggKernelsTest.java:71-103): mixed-magnitude doubles whose sum depends
    on the order of addition; the reference's sequential sum, bit for bit."""
    rnd = JavaRandom(23)
    out = []
    for n in LENGTHS:
        for frac in (0.0, 0.01, 0.3, 1.0):
            nulls = java_nulls(rnd, n, frac)
            dv = []
            for _ in range(n):
                sign = 1 if rnd.nextBoolean() else -1
                x = sign * rnd.nextDouble()
                dv.append(x * (10.0 ** rnd.nextInt(16)))
            if n == 0:
                continue
            cols = [Cc.doubles(dv, nulls, nullable=True)]
            kept = _ungrouped_rows(dv, nulls)
            want = (seq_sum(kept) if kept else None, len(kept))
            out.append(Case(f"agg_kernel_sequential_sums[n={n},nulls={frac}]", "AggKernelsTest.java:71-103", cols,
                            [], [A.SumDoubleAgg(0), A.CountAgg(0)], [Cc.HostBatch(cols, n, None)], [want],
                            ["fsum", "int"], fsum_tol=lambda w: abs(w) * 1e-12 + 1e-9))
    return out


def _test_doubles(rnd: JavaRandom, n: int) -> List[float]:
    """TestData.doubles (TestData.java:120-137)."""
    out = []
    for _ in range(n):
        c = rnd.nextInt(12)
        if c == 0:
            v = math.nan
        elif c == 1:
            v = math.inf
        elif c == 2:
            v = -math.inf
        elif c == 3:
            v = -0.0
        elif c == 4:
            v = 0.0
        elif c == 5:
            v = 1.5
        else:
            a = rnd.nextInt(-5, 5)
            v = a + (0.0 if rnd.nextBoolean() else 0.5)
        out.append(v)
    return out


def agg_kernel_min_max() -> List[Case]:
    """AggKernelsTest.minMaxMatchReferenceIncludingNaNAndInfinities
    (AggKernelsTest.java:105-121): min/max of doubles with NaN, +-Inf and
    -0.0, of small ints and of longs (TestData.ints / longs / doubles)."""
    rnd = JavaRandom(22)
    out = []
    for n in LENGTHS:
        for frac in (0.0, 0.2, 1.0):
            nulls = java_nulls(rnd, n, frac)
            dv = _test_doubles(rnd, n)
            iv = [rnd.nextInt(-20, 20) for _ in range(n)]
            lv = [rnd.nextLong() if rnd.nextInt(3) == 0 else rnd.nextLong(-20, 20) for _ in range(n)]
            valid = [not z for z in nulls]
            if sum(valid) == 0:
                continue  # the reference checks nothing when no value is valid
            cols = [Cc.doubles(dv, nulls, nullable=True), Cc.ints(iv, nulls, nullable=True),
                    Cc.longs(lv, nulls, nullable=True)]

            def mm(vals, lt):
                best = None
                for v, ok in zip(vals, valid):
                    if ok and (best is None or lt(v, best)):
                        best = v
                return best
            want = (mm(dv, lambda a, b: nan_safe_compare(a, b) < 0), mm(dv, lambda a, b: nan_safe_compare(a, b) > 0),
                    mm(iv, lambda a, b: a < b), mm(iv, lambda a, b: a > b),
                    mm(lv, lambda a, b: a < b), mm(lv, lambda a, b: a > b))
            fns = [A.MinMaxAgg(0, True), A.MinMaxAgg(0, False), A.MinMaxAgg(1, True), A.MinMaxAgg(1, False),
                   A.MinMaxAgg(2, True), A.MinMaxAgg(2, False)]
            out.append(Case(f"agg_kernel_min_max[n={n},nulls={frac}]", "AggKernelsTest.java:105-121", cols, [], fns,
                            [Cc.HostBatch(cols, n, None)], [want], ["exact"] * 6))
    return out


# ------------------------------------------ GroupKeyTableInlineKeysTest
INLINE_TWISTS = [("INT32", 1, "none"), ("INT32", 2, "none"), ("INT64", 1, "none"), ("INT32", 1, "nullsLater"),
                 ("INT32", 2, "nullsLater"), ("INT64", 1, "nullsLater"), ("INT32", 2, "selection"),
                 ("INT32", 1, "validBitmap"), ("INT32", 2, "validBitmap"), ("INT64", 1, "validBitmap"),
                 ("INT32", 1, "selectedNoNulls"), ("INT32", 2, "selectedNoNulls"), ("INT32", 1, "large"),
                 ("INT64", 1, "large")]


def inline_keys(t: str, keys: int, twist: str) -> Case:
    """GroupKeyTableInlineKeysTest.groupsMatchTheReference
    (GroupKeyTableInlineKeysTest.java:64-190): one INT32, two INT32 or one
    INT64 key; negative values, values equal in their low 32 bits, swapped
    pairs, null keys arriving in a later batch, selections; 40 batches of
    4096 (17 every seventh) rows. Expected: the HashMap of key tuples, here
    with count(*) per group."""
    rnd = JavaRandom(677 + keys * 31 + string_hash(twist))
    distinct = 400_000 if twist == "large" else 30_000
    is64 = t == "INT64"
    counts: Dict[tuple, int] = {}
    batches = []
    for b in range(40):
        n = 17 if b % 7 == 3 else 4096
        filtered = twist == "selectedNoNulls"
        with_nulls = (twist == "nullsLater" and b == 25) or filtered
        with_sel = (twist == "selection" and b % 5 == 4) or filtered
        v = [[0] * n for _ in range(keys)]
        nul = [[False] * n if with_nulls else None for _ in range(keys)]
        for c in range(keys):
            for i in range(n):
                g = rnd.nextInt(distinct)
                k = rnd.nextInt(4)
                x = -g if k == 0 else (g + (1 << 32) if is64 else g) if k == 1 else g
                v[c][i] = x
                if with_nulls and rnd.nextInt(5) == 0 and (not filtered or i % 3 == 0):
                    nul[c][i] = True
                    v[c][i] = 0
        if keys == 2:
            for i in range(0, n, 11):
                v[1][i] = v[0][i]
                v[0][i] = v[1][(i + 1) % n]
        cols = []
        for c in range(keys):
            # "validBitmap": a nullable column with no null, its bitmap all set
            nulls = nul[c] if nul[c] is not None else ([False] * n if twist == "validBitmap" else None)
            vals = v[c] if is64 else [((x + (1 << 31)) % (1 << 32)) - (1 << 31) for x in v[c]]
            cols.append((Cc.longs if is64 else Cc.ints)(vals, nulls, nullable=True))
        selected = [i % 3 != 0 for i in range(n)] if with_sel else [True] * n
        batches.append(Cc.HostBatch(cols, n, bitmap(selected) if with_sel else None))
        for i in range(n):
            if not selected[i]:
                continue
            tup = []
            for c in range(keys):
                if nul[c] is not None and nul[c][i]:
                    tup.append(None)
                else:
                    x = v[c][i]
                    tup.append(x if is64 else ((x + (1 << 31)) % (1 << 32)) - (1 << 31))
            tup = tuple(tup)
            counts[tup] = counts.get(tup, 0) + 1
    expected = [k + (c,) for k, c in counts.items()]
    return Case(f"inline_keys[{t},{keys},{twist}]", "GroupKeyTableInlineKeysTest.java:64-190", batches[0].columns,
                list(range(keys)), [A.CountAgg()], batches, expected, ["key"] * keys + ["int"])


# ------------------------------------------------------------ registry
def all_case_builders():
    """(builder, args) pairs, in a stable order; each builds one case."""
    out = []

    def add(fn, *args):
        out.append((fn, args))
    for card in (1, 4, 64, 65, 300, 5000):
        for sel in (False, True):
            add(grouped_accumulators, card, sel)
    for card in (1, 3, 64, 300, 5000):
        add(strict_double_sum, card)
    add(wide_decimal_keys)
    add(wide_long_sum, True)
    add(wide_long_sum, False)
    for fn in (known_wide_sum_int32, known_null_vs_zero_keys, known_write_keys_layout, known_memoised_dictionary_keys,
               known_record_strings, known_high_cardinality_strings, known_sequential_running_sum):
        add(fn)
    for t, k, tw in INLINE_TWISTS:
        add(inline_keys, t, k, tw)
    return out


def multi_case_builders():
    """Builders that return several cases at once (one per length x null fraction)."""
    return [known_nan_handling, agg_kernel_sums, agg_kernel_sequential_sums, agg_kernel_min_max]


def build_all() -> List[Case]:
    cases = [fn(*args) for fn, args in all_case_builders()]
    for b in multi_case_builders():
        cases += b()
    return cases
