"""Writes tests/golden/expected.json: for every golden case (the reference's
seeded aggregation tests and literal known answers, reference_cases.py) the
digest of its regenerated inputs, its group count, the digest of its
expected rows and, for cases of at most 200 groups, the rows themselves.

    python tests/golden/make_golden.py

The expected rows come from the reference tests' own expectation logic as
restated in reference_cases.py, never from this library or its oracle.
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.dirname(HERE)]

from golden import check, reference_cases  # noqa: E402

MAX_LISTED = 200


def main() -> None:
    out = {}
    for case in reference_cases.build_all():
        nk = len(case.keys)
        entry = {"source": case.source, "inputs_sha256": check.inputs_digest(case), "groups": len(case.expected),
                 "rows_sha256": check.rows_digest(case.expected, nk)}
        if len(case.expected) <= MAX_LISTED:
            entry["rows"] = check.canonical_rows(case.expected, nk)
        out[case.name] = entry
    path = os.path.join(HERE, "expected.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
        f.write("\n")
    print(f"{len(out)} cases -> {path}")


if __name__ == "__main__":
    main()
