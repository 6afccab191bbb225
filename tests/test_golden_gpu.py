"""GPU parity on the golden cases (tests/golden/): the reference's seeded
aggregation tests regenerated, and its literal known answers, run through
the C ABI (host batches, one vr_agg_update per reference batch) and
compared with the reference tests' expected rows: keys, counts, integer and
decimal sums, min/max exact; FP64 sums within the tolerance each reference
test states for a non-sequential sum (1e-9 absolute for the quarter-valued
grouped sums, |x| * 1e-12 + 1e-9 for mixed magnitudes). Each case runs with
the spec's own compiled kernel and with the prebuilt one."""
import json
import os

import pytest

import vecruntime_b200 as vr
from vecruntime_b200 import native as N

from golden import check
from golden import reference_cases as R
from parity import rows_of

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "expected.json")) as f:
    NAMES = sorted(json.load(f))

_cases = {}


def golden_case(name):
    if not _cases:
        for c in R.build_all():
            _cases[c.name] = c
    return _cases[name]


@pytest.mark.parametrize("mode", ["jit", "prebuilt"])
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_the_reference_tests(cuda, name, mode):
    case = golden_case(name)
    flags = N.VR_SPEC_NO_JIT if mode == "prebuilt" else 0
    rows = max([b.num_rows for b in case.batches] + [1])
    agg = vr.GpuHashAggregate(case.columns, case.keys, case.functions, max_batch_rows=rows, flags=flags)
    try:
        for b in case.batches:
            agg.consume(b)
        n = agg.num_groups()
        got = rows_of(agg.output_types, agg.emit(), n)
        st = agg.stats()
    finally:
        agg.close()
    if mode == "jit":
        assert st.jit == 1, "the spec's own kernel did not load"
    tol = case.fsum_tol or (lambda want: abs(want) * 1e-12)
    bad = check.compare_rows(got, case.expected, case.roles, len(case.keys), fsum=tol)
    assert not bad, f"{case.source}: (row, col, role, key, got, want) {bad}"
