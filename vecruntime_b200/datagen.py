"""Seeded synthetic inputs with the shapes of the benchmark workloads.

Every generator is numpy's PCG64 with a fixed per-workload seed; Zipf keys
are numpy's Zipf(s) sampler truncated to the domain by resampling. These
stand in for data the reference benchmarks on (TPC-H lineitem shapes and
its JMH generators); no benchmark data is reproduced.

Workloads (rows, keys, values, functions):
  plain      1,048,576 rows (256 batches of 4,096); int64 key over 1,000 seeded
             distinct values; v1 int64 U[-1e6, 1e6] 5% null; v2 f64 N(0,1);
             count(*), count(v1), sum(v1), min(v1), max(v1), sum(v2), avg(v2)
  decimal    low-cardinality decimal report: two dictionary keys (3 and 2
             values), qty/price/disc/tax DECIMAL(12,2); sum(qty), sum(price),
             sum(price*(1-disc)), sum(price*(1-disc)*(1+tax)), avg(qty),
             avg(disc), count(*)
  highcard   key1 int64 Zipf(1.1) over 50M with 1% nulls, key2 int32 U[0,15];
             v_i int32 U[0,1e4], v_f f64 lognormal(0,1); sum/count/min/max/avg
  batched    instances with log-uniform rows 2^10..2^22 and cardinality
             1..2^20; int64 key, int64 + f64 values; sum/count/min/max
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import aggregate as A
from . import columns as Cc

SEEDS = {"plain": 1001, "decimal": 1002, "highcard": 1003, "batched": 1004, "serving": 1005, "parquet": 1006}


@dataclass
class Workload:
    name: str
    columns: list          # Col per input column
    keys: List[int]
    functions: list
    est_groups: int
    rows: int

    def spec(self, **kw) -> A.Spec:
        return A.Spec(self.columns, self.keys, self.functions, est_groups=self.est_groups,
                      max_batch_rows=self.rows, **kw)

    def batch(self, lo: int = 0, hi: int = None, selection=None) -> Cc.HostBatch:
        hi = self.rows if hi is None else hi
        cols = [slice_col(c, lo, hi) for c in self.columns]
        return Cc.HostBatch(cols, hi - lo, selection)


def slice_col(c: Cc.Col, lo: int, hi: int) -> Cc.Col:
    """Rows [lo, hi) of a column; lo must be a multiple of 8 when bitmaps are sliced."""
    assert lo % 8 == 0 or (c.validity is None and c.lane != 4)
    if c.lane == 4:  # BOOL bit-packed
        d = c.data[lo // 8:(hi + 7) // 8]
    else:
        d = c.data[lo:hi]
    v = None if c.validity is None else c.validity[lo // 8:(hi + 7) // 8]
    out = Cc.Col(c.lane, d, v, c.precision, c.scale, c.dict_size, c.nullable)
    if c.lane == 4:
        out._n = hi - lo
    return out


def plain(rows: int = 1 << 20, seed: int = SEEDS["plain"]) -> Workload:
    rng = np.random.default_rng(seed)
    domain = rng.integers(-(1 << 62), 1 << 62, size=1000, dtype=np.int64)
    k = domain[rng.integers(0, 1000, size=rows)]
    v1 = rng.integers(-1_000_000, 1_000_001, size=rows, dtype=np.int64)
    v1_null = rng.random(rows) < 0.05
    v2 = rng.standard_normal(rows)
    cols = [Cc.longs(k, nullable=False), Cc.longs(v1, v1_null), Cc.doubles(v2, nullable=False)]
    fns = [A.CountAgg(), A.CountAgg(1), A.SumLongAgg(1, checked=True), A.MinMaxAgg(1, True), A.MinMaxAgg(1, False),
           A.SumDoubleAgg(2), A.AverageAgg(2)]
    return Workload("plain", cols, [0], fns, 1000, rows)


def decimal_report(rows: int = 60_000_000, seed: int = SEEDS["decimal"]) -> Workload:
    rng = np.random.default_rng(seed)
    k1 = rng.integers(0, 3, size=rows, dtype=np.int32)
    k2 = rng.integers(0, 2, size=rows, dtype=np.int32)
    qty = rng.integers(1, 51, size=rows, dtype=np.int64) * 100            # DECIMAL(12,2)
    price = rng.integers(90_000, 10_500_001, size=rows, dtype=np.int64)   # 900.00 .. 105000.00
    disc = rng.integers(0, 11, size=rows, dtype=np.int64)                 # 0.00 .. 0.10
    tax = rng.integers(0, 9, size=rows, dtype=np.int64)                   # 0.00 .. 0.08
    cols = [Cc.dict_ids(k1, 3, nullable=False), Cc.dict_ids(k2, 2, nullable=False),
            Cc.decimals(qty, 12, 2, nullable=False), Cc.decimals(price, 12, 2, nullable=False),
            Cc.decimals(disc, 12, 2, nullable=False), Cc.decimals(tax, 12, 2, nullable=False)]
    disc_price = A.DecimalProduct([(3, 1, 0), (4, -1, 100)], precision=26)            # DECIMAL(26,4)
    charge = A.DecimalProduct([(3, 1, 0), (4, -1, 100), (5, 1, 100)], precision=38)   # DECIMAL(38,6)
    fns = [A.WideDecimalSumAgg(2, 22, 2), A.WideDecimalSumAgg(3, 22, 2), A.WideDecimalSumAgg(disc_price, 36, 4),
           A.WideDecimalSumAgg(charge, 38, 6), A.WideDecimalAvgAgg(2, 22, 2), A.WideDecimalAvgAgg(4, 22, 2),
           A.CountAgg()]
    return Workload("decimal", cols, [0, 1], fns, 6, rows)


def zipf_keys(rng, n: int, s: float, domain: int) -> np.ndarray:
    out = rng.zipf(s, size=n).astype(np.int64)
    bad = out > domain
    while bad.any():
        out[bad] = rng.zipf(s, size=int(bad.sum()))
        bad = out > domain
    return out


def high_cardinality(rows: int = 100_000_000, seed: int = SEEDS["highcard"], domain: int = 50_000_000) -> Workload:
    rng = np.random.default_rng(seed)
    k1 = zipf_keys(rng, rows, 1.1, domain)
    k1_null = rng.random(rows) < 0.01
    k1[k1_null] = 0
    k2 = rng.integers(0, 16, size=rows, dtype=np.int32)
    vi = rng.integers(0, 10_001, size=rows, dtype=np.int32)
    vf = rng.lognormal(0.0, 1.0, size=rows)
    cols = [Cc.longs(k1, k1_null), Cc.ints(k2, nullable=False), Cc.ints(vi, nullable=False),
            Cc.doubles(vf, nullable=False)]
    fns = [A.CountAgg(), A.SumLongAgg(2), A.MinMaxAgg(2, True), A.MinMaxAgg(2, False), A.SumDoubleAgg(3),
           A.AverageAgg(3), A.MinMaxAgg(3, True), A.MinMaxAgg(3, False)]
    est = expected_distinct_pairs(rows, domain)
    return Workload("highcard", cols, [0, 1], fns, est, rows)


def expected_distinct_pairs(rows: int, domain: int, s: float = 1.1, fanout: int = 16) -> int:
    """Expected distinct (key1, key2) pairs for the high-cardinality shape."""
    k = np.arange(1, domain + 1, dtype=np.float64)
    p = k ** -s
    p /= p.sum()
    lam = rows * p / fanout
    return int(fanout * np.sum(-np.expm1(-lam))) + 1


def batched_instances(n: int = 512, seed: int = SEEDS["batched"], max_log_rows: int = 22,
                      max_log_card: int = 20) -> List[Workload]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        rows = int(round(2 ** rng.uniform(10, max_log_rows)))
        card = max(1, int(round(2 ** rng.uniform(0, max_log_card))))
        domain = rng.integers(-(1 << 62), 1 << 62, size=card, dtype=np.int64)
        k = domain[rng.integers(0, card, size=rows)]
        vi = rng.integers(-1_000_000, 1_000_001, size=rows, dtype=np.int64)
        vf = rng.standard_normal(rows)
        cols = [Cc.longs(k, nullable=False), Cc.longs(vi, nullable=False), Cc.doubles(vf, nullable=False)]
        out.append(Workload(f"inst{i}", cols, [0], batched_functions(), expected_distinct(rows, card), rows))
    return out


def expected_distinct(rows: int, card: int) -> int:
    """Expected distinct keys among `rows` uniform draws from `card` values:
    the cardinality estimate a planner that knows the batch size would pass."""
    return max(1, int(np.ceil(card * -np.expm1(-rows / card))))


def batched_functions():
    return [A.CountAgg(), A.SumLongAgg(1), A.MinMaxAgg(1, True), A.MinMaxAgg(1, False), A.SumDoubleAgg(2),
            A.MinMaxAgg(2, True), A.MinMaxAgg(2, False)]


def input_bytes(w: Workload) -> int:
    """Algorithmic input bytes: every column's values plus validity bits."""
    b = 0
    for c in w.columns:
        b += c.data.nbytes if c.lane != 4 else (w.rows + 7) // 8
        if c.validity is not None:
            b += (w.rows + 7) // 8
    return b


# ------------------------------------------------------------------ Parquet pages
def _uleb(v: int) -> bytes:
    out = bytearray()
    while True:
        b = v & 0x7F
        v >>= 7
        if v:
            out.append(b | 0x80)
        else:
            out.append(b)
            return bytes(out)


def encode_hybrid(values: np.ndarray, width: int, max_groups: int = 63) -> bytes:
    """Parquet's RLE / bit-packed hybrid encoding of `values` at `width`
    bits, as a writer emits it: groups of 8 values (aligned from the
    stream's start) that all hold one value and repeat the previous group's
    value form RLE runs, the rest bit-packed runs of at most `max_groups`
    groups; the last group is zero-padded (a reader stops at its count)."""
    v = np.ascontiguousarray(values, dtype=np.uint32)
    n = len(v)
    if width == 0 or n == 0:
        return b""
    g = (n + 7) // 8
    pad = np.zeros(g * 8, np.uint32)
    pad[:n] = v
    grp = pad.reshape(g, 8)
    const = (grp == grp[:, :1]).all(axis=1)
    const[-1] &= n % 8 == 0  # a padded last group is bit-packed
    # bit-packed bytes of every group: width bytes each, LSB first
    bits = ((pad[:, None] >> np.arange(width, dtype=np.uint32)) & 1).astype(np.uint8)
    packed = np.packbits(bits.reshape(-1), bitorder="little").reshape(g, width)
    first = grp[:, 0]
    vbytes = (width + 7) // 8
    out = []
    i = 0
    while i < g:
        if const[i]:
            j = i + 1
            while j < g and const[j] and first[j] == first[i]:
                j += 1
            out.append(_uleb((j - i) * 8 << 1))
            out.append(int(first[i]).to_bytes(4, "little")[:vbytes])
        else:
            j = i + 1
            while j < g and j - i < max_groups and not const[j]:
                j += 1
            out.append(_uleb(((j - i) << 1) | 1))
            out.append(packed[i:j].tobytes())
        i = j
    return b"".join(out)


def dictionary_pages(ids: np.ndarray, nulls: Optional[np.ndarray], width: int, page_rows: int,
                     v2: bool = False) -> list:
    """A column chunk of RLE_DICTIONARY data pages for `ids` (a null slot
    has no id in its page): [(page bytes, page fields)] with v1 or v2
    framing and definition levels (max level 1) when `nulls` is given."""
    out = []
    n = len(ids)
    for lo in range(0, n, page_rows):
        hi = min(n, lo + page_rows)
        present = np.ones(hi - lo, bool) if nulls is None else ~np.asarray(nulls[lo:hi], bool)
        values = bytes([width]) + encode_hybrid(np.asarray(ids[lo:hi])[present], width)
        lv = b"" if nulls is None else encode_hybrid(present.astype(np.uint32), 1)
        if nulls is None:
            page, ll = values, 0
        elif v2:
            page, ll = lv + values, len(lv)
        else:
            page, ll = len(lv).to_bytes(4, "little") + lv + values, 0
        out.append((page, dict(num_values=hi - lo, max_def_level=0 if nulls is None else 1, v2=int(v2),
                               levels_length=ll, encoding=1, value_bytes=4)))
    return out
