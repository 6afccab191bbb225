"""Comparison of aggregate outputs as sorted multisets of groups.

Keys, counts, integer and decimal sums, min and max compare bit-exact
(min/max of doubles by Spark's NaN-safe equality: NaN == NaN, -0.0 == 0.0);
FP64 sums compare within RTOL relative of the oracle's compensated sum, with
an absolute floor of ATOL_SCALE times the sum of magnitudes in the group
(1e-12 relative).
"""
from __future__ import annotations

import math
from typing import List

import numpy as np

from vecruntime_b200 import native as N
from vecruntime_b200.columns import dec128_to_ints, unpack_bits

RTOL = 1e-12


def roles_of(spec) -> List[str]:
    """Per output column: key / int / fsum / fexact / dec / bool."""
    roles = ["key"] * len(spec.keys)
    for f in spec.functions:
        k = f.kind
        if k in (N.VR_FN_COUNT_STAR, N.VR_FN_COUNT, N.VR_FN_SUM_LONG, N.VR_FN_COUNT_MERGE):
            roles.append("int")
        elif k == N.VR_FN_SUM_DOUBLE:
            roles.append("fsum")
        elif k in (N.VR_FN_AVG_DOUBLE, N.VR_FN_AVG_DOUBLE_MERGE):
            roles += ["fsum", "int"]
        elif k in (N.VR_FN_MIN, N.VR_FN_MAX):
            roles.append("exact")
        elif k in (N.VR_FN_SUM_DECIMAL, N.VR_FN_SUM_DECIMAL_MERGE):
            roles += ["dec", "bool"]
        elif k in (N.VR_FN_AVG_DECIMAL, N.VR_FN_AVG_DECIMAL_MERGE):
            roles += ["dec", "int"]
        else:
            raise ValueError(k)
    return roles


def column_values(t, data, validity, n) -> list:
    valid = unpack_bits(validity, n) if n else np.zeros(0, bool)
    lane = t.lane
    if lane == N.VR_BOOL:
        vals = unpack_bits(data, n).tolist()
    elif lane == N.VR_DECIMAL128:
        vals = dec128_to_ints(data[:n])
    elif lane == N.VR_FLOAT64:
        vals = [float(x) for x in data[:n]]
    else:
        vals = [int(x) for x in data[:n]]
    return [v if ok else None for v, ok in zip(vals, valid)]


def rows_of(types, arrays, n) -> list:
    cols = [column_values(t, d, v, n) for t, (d, v) in zip(types, arrays)]
    return list(zip(*cols)) if cols else []


def _key(v):
    # None sorts first; floats by bits so NaN payloads and -0.0 order deterministically
    if v is None:
        return (0, 0)
    if isinstance(v, float):
        return (1, np.float64(v).view(np.int64).item())
    return (1, v)


def sort_rows(rows, nkeys):
    return sorted(rows, key=lambda r: tuple(_key(x) for x in r[:nkeys]))


def float_equal_exact(a, b) -> bool:
    if a is None or b is None:
        return a is b
    if math.isnan(a) and math.isnan(b):
        return True
    return a == b  # -0.0 == 0.0 (CompareOp.nanSafeCompare)


def float_close(got, want, scale=None, rtol=RTOL) -> bool:
    if got is None or want is None:
        return got is want
    if math.isnan(want) or math.isnan(got):
        return math.isnan(want) and math.isnan(got)
    if math.isinf(want) or math.isinf(got):
        return got == want
    tol = rtol * abs(want)
    if scale is not None:
        tol = max(tol, 1e-15 * scale)
    return abs(got - want) <= tol


def compare(spec, got_types, got_arrays, got_n, want_types, want_arrays, want_n, fsum_scale=None):
    """Asserts the GPU output equals the oracle output as multisets of groups."""
    assert got_n == want_n, f"group count {got_n} != {want_n}"
    assert [t.lane for t in got_types] == [t.lane for t in want_types], "output lanes differ"
    roles = roles_of(spec)
    nk = len(spec.keys)
    g = sort_rows(rows_of(got_types, got_arrays, got_n), nk)
    w = sort_rows(rows_of(want_types, want_arrays, want_n), nk)
    bad = []
    for i, (rg, rw) in enumerate(zip(g, w)):
        for j, role in enumerate(roles):
            a, b = rg[j], rw[j]
            if role == "fsum":
                ok = float_close(a, b, None if fsum_scale is None else fsum_scale(rw))
            elif role == "exact" and (isinstance(a, float) or isinstance(b, float)):
                ok = float_equal_exact(a, b)
            elif role == "key" and isinstance(b, float):
                ok = (a is None and b is None) or (a is not None and b is not None and
                                                   np.float64(a).view(np.int64) == np.float64(b).view(np.int64))
            else:
                ok = a == b
            if not ok:
                bad.append((i, j, role, rg[:nk], a, b))
                if len(bad) > 10:
                    break
        if len(bad) > 10:
            break
    assert not bad, "mismatches (row, col, role, key, got, want): " + repr(bad[:10])


# ------------------------------------------------------------- vectorised
def _key_sort_columns(t, data, validity, n):
    """Sort columns of one key output: its validity, then its raw bits (0 when null)."""
    valid = unpack_bits(validity, n)
    if t.lane == N.VR_BOOL:
        parts = [unpack_bits(data, n).astype(np.uint64)]
    elif t.lane == N.VR_DECIMAL128:
        limbs = np.asarray(data[:n], dtype=np.uint64).reshape(n, 2)
        parts = [limbs[:, 1], limbs[:, 0]]
    else:
        raw = np.ascontiguousarray(data[:n])
        parts = [raw.view(np.uint64 if raw.itemsize == 8 else np.uint32).astype(np.uint64)]
    return [valid.astype(np.uint64)] + [np.where(valid, p, np.uint64(0)) for p in parts]


def _sorted_order(types, arrays, n, nk):
    cols = []
    for t, (d, v) in zip(types[:nk], arrays[:nk]):
        cols += _key_sort_columns(t, d, v, n)
    if not cols:
        return np.arange(n)
    return np.lexsort(cols[::-1])  # lexsort: last key is the primary one


def _values(t, data, n):
    if t.lane == N.VR_BOOL:
        return unpack_bits(data, n)
    if t.lane == N.VR_DECIMAL128:
        return np.asarray(data[:n], dtype=np.uint64).reshape(n, 2)
    return np.asarray(data[:n])


def compare_arrays(spec, got_types, got_arrays, got_n, want_types, want_arrays, want_n, rtol=RTOL, limit=10):
    """The rule of `compare` (groups as a sorted multiset; keys, counts,
    integer and decimal sums and min/max bit-exact with NaN-safe equality for
    doubles; FP64 sums within `rtol` relative), vectorised with numpy for
    millions of groups. Returns (mismatching groups, up to `limit` examples
    as (sorted row, output column, role, got, want))."""
    if got_n != want_n:
        return max(got_n, want_n), [("group count", got_n, want_n)]
    if [t.lane for t in got_types] != [t.lane for t in want_types]:
        return got_n or 1, [("output lanes", [t.lane for t in got_types], [t.lane for t in want_types])]
    n = got_n
    roles = roles_of(spec)
    nk = len(spec.keys)
    og = _sorted_order(got_types, got_arrays, n, nk)
    ow = _sorted_order(want_types, want_arrays, n, nk)
    bad_rows = np.zeros(n, dtype=bool)
    examples = []
    for j, role in enumerate(roles):
        t = got_types[j]
        (gd, gv), (wd, wv) = got_arrays[j], want_arrays[j]
        g_ok = unpack_bits(gv, n)[og]
        w_ok = unpack_bits(wv, n)[ow]
        a = _values(t, gd, n)[og]
        b = _values(t, wd, n)[ow]
        if t.lane == N.VR_DECIMAL128:
            same = (a == b).all(axis=1)
        elif t.lane == N.VR_FLOAT64 and role == "fsum":
            with np.errstate(invalid="ignore", over="ignore"):
                both_nan = np.isnan(a) & np.isnan(b)
                inf = np.isinf(a) | np.isinf(b)
                close = np.abs(a - b) <= rtol * np.abs(b)
                same = both_nan | np.where(inf, a == b, close)
        elif t.lane == N.VR_FLOAT64 and role != "key":
            same = (a == b) | (np.isnan(a) & np.isnan(b))  # nanSafeCompare equality; -0.0 == 0.0
        elif t.lane == N.VR_FLOAT64:
            same = a.view(np.uint64) == b.view(np.uint64)
        else:
            same = a == b
        ok = (g_ok == w_ok) & (same | ~w_ok)
        wrong = ~ok
        if wrong.any():
            bad_rows |= wrong
            for i in np.flatnonzero(wrong)[:max(0, limit - len(examples))]:
                examples.append((int(i), j, role, a[i].tolist() if g_ok[i] else None,
                                 b[i].tolist() if w_ok[i] else None))
    return int(bad_rows.sum()), examples
