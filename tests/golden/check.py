"""Digests, canonical rows and the comparison rule for the golden cases."""
from __future__ import annotations

import hashlib
import json
import math
import struct
from typing import Callable, List, Optional

import numpy as np


def _canon(v):
    if v is None or isinstance(v, bool):
        return v
    if isinstance(v, float):
        return {"f64": struct.pack("<d", v).hex()}
    return int(v)


def canonical_rows(rows, nkeys: int) -> list:
    """Rows as JSON values (doubles by their bits), sorted by key."""
    from parity import sort_rows

    return [[_canon(x) for x in r] for r in sort_rows([tuple(r) for r in rows], nkeys)]


def decanon(v):
    if isinstance(v, dict):
        return struct.unpack("<d", bytes.fromhex(v["f64"]))[0]
    return v


def rows_digest(rows, nkeys: int) -> str:
    return hashlib.sha256(json.dumps(canonical_rows(rows, nkeys), separators=(",", ":")).encode()).hexdigest()


def inputs_digest(case) -> str:
    """Every byte the spec and the batches hand to the library."""
    h = hashlib.sha256()
    for c in case.columns:
        t = c.ctype()
        h.update(struct.pack("<6i", t.lane, t.precision, t.scale, t.nullable, t.dict_size, t.flags))
    h.update(json.dumps([case.keys, [f.to_ctypes().kind for f in case.functions]]).encode())
    for b in case.batches:
        h.update(struct.pack("<q", b.num_rows))
        for c in b.columns:
            h.update(np.ascontiguousarray(c.data).tobytes())
            h.update(b"v" if c.validity is None else np.ascontiguousarray(c.validity).tobytes())
        h.update(b"s" if b.selection is None else np.ascontiguousarray(b.selection).tobytes())
    return h.hexdigest()


def _same_float_bits(a: float, b: float) -> bool:
    return struct.pack("<d", a) == struct.pack("<d", b)


def compare_rows(got, want, roles: List[str], nkeys: int, fsum: Optional[Callable[[float], float]] = None) -> List:
    """Mismatches between two row sets compared as sorted multisets.

    `fsum` None: FP64 sums must be bit-identical (the oracle's sequential
    mode against the reference's sequential sums); else |got - want| <=
    fsum(want). Min/max doubles: NaN == NaN and -0.0 == 0.0
    (CompareOp.nanSafeCompare). Everything else exact."""
    from parity import sort_rows

    g = sort_rows([tuple(r) for r in got], nkeys)
    w = sort_rows([tuple(r) for r in want], nkeys)
    bad = []
    if len(g) != len(w):
        return [("group count", len(g), len(w))]
    for i, (rg, rw) in enumerate(zip(g, w)):
        for j, role in enumerate(roles):
            a, b = rg[j], rw[j]
            if a is None or b is None:
                ok = a is None and b is None
            elif role == "fsum":
                if math.isnan(b) or math.isnan(a):
                    ok = math.isnan(a) and math.isnan(b)
                elif fsum is None:
                    ok = _same_float_bits(a, b)
                elif math.isinf(b) or math.isinf(a):
                    ok = a == b
                else:
                    ok = abs(a - b) <= fsum(b)
            elif role == "exact" and isinstance(b, float):
                ok = (math.isnan(a) and math.isnan(b)) or a == b
            elif role == "key" and isinstance(b, float):
                ok = _same_float_bits(a, b)
            else:
                ok = a == b
            if not ok:
                bad.append((i, j, role, rw[:nkeys], a, b))
                if len(bad) >= 10:
                    return bad
    return bad
