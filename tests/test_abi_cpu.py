"""CPU-only checks of the C ABI library: it loads, exports exactly what
include/vrgpu.h declares, and its host-side planner (the GPU gate) compiles
specs the way the reference's planner would accept or refuse them."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import vecruntime_b200 as vr
from vecruntime_b200 import native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "vrgpu.h")).read()
    return set(re.findall(r"^(?:int|void|const char\*|void\*)\s+(vr_[a-z0-9_]+)\(", text, re.M))


def test_library_loads_and_exports_every_declared_symbol():
    lib = N.lib()
    declared = declared_symbols()
    assert len(declared) > 30
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {l.split()[-1] for l in out.stdout.splitlines() if " T " in l}
    assert declared == exported, (declared ^ exported)


def test_ctypes_prototypes_cover_the_header():
    names = {p[0] for p in N.PROTOTYPES}
    assert names == declared_symbols()


def test_status_strings():
    assert N.status_string(N.VR_OK) == "ok"
    assert "overflow" in N.status_string(N.VR_ERR_OVERFLOW)


def spec_of(cols, keys, fns, **kw):
    return vr.Spec(cols, keys, fns, **kw)


def test_plan_plain_int64_key_uses_sentinel_layout():
    cols = [vr.longs(np.zeros(1, np.int64), nullable=False), vr.longs(np.zeros(1, np.int64), nullable=True),
            vr.doubles(np.zeros(1), nullable=False)]
    fns = [vr.CountAgg(), vr.CountAgg(1), vr.SumLongAgg(1, checked=True), vr.MinMaxAgg(1, True),
           vr.MinMaxAgg(1, False), vr.SumDoubleAgg(2), vr.AverageAgg(2)]
    rc, info, outs = spec_of(cols, [0], fns).plan()
    assert rc == N.VR_OK
    assert info.key_words == 1 and info.sentinel_layout == 1
    assert info.direct_ok == 0
    # keys + count, count, sum, min, max, sum, (avg sum, avg count)
    assert [o.lane for o in outs] == [N.VR_INT64, N.VR_INT64, N.VR_INT64, N.VR_INT64, N.VR_INT64, N.VR_INT64,
                                      N.VR_FLOAT64, N.VR_FLOAT64, N.VR_INT64]
    # rows, count(v1), sum(v1), min(v1), max(v1), sum(v2); count(*) is the rows op and
    # avg(v2)'s count of a non-nullable column is count(*) too: no extra ops
    assert info.num_ops == 6


def test_plan_dictionary_keys_are_direct_indexed():
    cols = [vr.dict_ids(np.zeros(1), 3, nullable=False), vr.dict_ids(np.zeros(1), 2, nullable=True),
            vr.decimals(np.zeros(1), 12, 2, nullable=False)]
    fns = [vr.WideDecimalSumAgg(2, 22, 2), vr.CountAgg()]
    rc, info, outs = spec_of(cols, [0, 1], fns).plan()
    assert rc == N.VR_OK
    assert info.direct_ok == 1 and info.direct_slots == 3 * 3  # (3) x (2 + null)
    assert [o.lane for o in outs] == [N.VR_DICT32, N.VR_DICT32, N.VR_DECIMAL128, N.VR_BOOL, N.VR_INT64]
    assert outs[2].precision == 22 and outs[2].scale == 2


def test_plan_composite_nullable_key_needs_two_words():
    cols = [vr.longs(np.zeros(1, np.int64), nullable=True), vr.ints(np.zeros(1), nullable=False),
            vr.ints(np.zeros(1), nullable=False)]
    rc, info, _ = spec_of(cols, [0, 1], [vr.CountAgg(), vr.SumLongAgg(2)]).plan()
    assert rc == N.VR_OK and info.key_words == 2 and info.sentinel_layout == 0


def test_plan_refuses_what_the_gpu_gate_does_not_cover():
    cols = [vr.longs(np.zeros(1, np.int64), nullable=False), vr.decimals(np.zeros(1), 12, 2, nullable=False),
            vr.decimals(np.zeros(1), 12, 3, nullable=False)]
    # a 38-digit average buffer hides its input's precision: the result type must be given
    f = vr.AggFunction(N.VR_FN_AVG_DECIMAL, 1, flags=N.VR_FN_FINAL, precision=38, scale=2)
    rc, info, _ = spec_of(cols, [0], [f]).plan()
    assert rc == N.VR_ERR_INVALID and b"result type" in info.reason
    # a product whose scale needs rounding
    p = vr.DecimalProduct([(1, 1, 0), (2, 1, 0)])
    rc, info, _ = spec_of(cols, [0], [vr.WideDecimalSumAgg(p, 38, 4)]).plan()
    assert rc == N.VR_ERR_UNSUPPORTED
    # min over a boolean lane
    cols2 = [vr.longs(np.zeros(1, np.int64), nullable=False), vr.bools(np.zeros(1, bool))]
    rc, info, _ = spec_of(cols2, [0], [vr.MinMaxAgg(1, True)]).plan()
    assert rc == N.VR_ERR_UNSUPPORTED


def test_plan_types_final_averages_as_spark_does():
    """Final / Complete averages: avg(double) a FLOAT64 result then the count;
    avg(decimal(12,2)) over its Decimal(22,2) buffer a Decimal(16,6) result (an
    INT64 lane up to 18 digits, DECIMAL128 beyond) then the count."""
    cols = [vr.longs(np.zeros(1, np.int64), nullable=False), vr.decimals(np.zeros(1), 12, 2, nullable=False),
            vr.doubles(np.zeros(1), nullable=False), vr.decimals128([0], 38, 2)]
    fns = [vr.WideDecimalAvgAgg(1, 22, 2, final_result=True), vr.AverageAgg(2, final_result=True),
           vr.WideDecimalAvgAgg(3, 38, 2, final_result=True, result_precision=38, result_scale=6)]
    rc, info, outs = spec_of(cols, [0], fns).plan()
    assert rc == N.VR_OK, info.reason
    got = [(t.lane, t.precision, t.scale) for t in outs[1:]]
    assert got == [(N.VR_INT64, 16, 6), (N.VR_INT64, 0, 0), (N.VR_FLOAT64, 0, 0), (N.VR_INT64, 0, 0),
                   (N.VR_DECIMAL128, 38, 6), (N.VR_INT64, 0, 0)]


def test_plan_too_many_accumulators_is_refused():
    cols = [vr.longs(np.zeros(1, np.int64), nullable=False)] + [vr.decimals128([0], 38, 0) for _ in range(15)]
    fns = [vr.WideDecimalSumAgg(i, 38, 0) for i in range(1, 16)] * 3
    rc, info, _ = spec_of(cols, [0], fns).plan()
    assert rc == N.VR_ERR_UNSUPPORTED


def test_create_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cols = [vr.longs(np.zeros(1, np.int64), nullable=False)]
    with pytest.raises(vr.VrError):
        vr.GpuHashAggregate(cols, [0], [vr.CountAgg()])


@pytest.mark.parametrize("workload,tier", [("decimal_report", 0), ("plain", 1), ("high_cardinality", 1)])
def test_jit_specialises_the_aggregate_kernel_without_a_gpu(workload, tier):
    """NVRTC compiles the per-spec aggregate kernel for sm_100a on the host;
    the same source the runtime launches, so a compile error shows here."""
    from vecruntime_b200 import datagen as G

    w = getattr(G, workload)(rows=1000)
    sp = w.spec()
    log = C.create_string_buffer(8192)
    nbytes = C.c_int64()
    rc = N.lib().vr_jit_compile(C.byref(sp.spec), tier, C.byref(nbytes), log, len(log))
    if rc == N.VR_ERR_UNSUPPORTED and b"nvrtc" in log.value.lower():
        pytest.skip("libnvrtc is not loadable here: " + log.value.decode())
    assert rc == N.VR_OK, log.value.decode()
    assert nbytes.value > 10_000


def test_tuner_table_records_keeps_the_fastest_and_round_trips(tmp_path):
    """The autotuner's table (host only): a choice recorded for (spec, rows)
    is found for rows of the same power of two and not for others; a slower
    measurement does not replace a faster one; save and load carry every
    field."""
    from vecruntime_b200 import datagen as G

    lib = N.lib()
    sp = G.plain(rows=1000).spec()
    rows = 3_000_001  # a power-of-two bucket no GPU test's batches fall in
    t = N.TuneChoice()
    t.tier, t.warp_agg, t.threads, t.blocks_per_sm, t.tile_rows, t.smem_slots = 1, 1, 256, 2, 512, 512
    t.table_capacity = 1 << 20
    assert lib.vr_tune_record(C.byref(sp.spec), rows, C.byref(t), C.c_double(2e9)) == N.VR_OK
    slower = N.TuneChoice()
    slower.tier, slower.threads, slower.tile_rows = 2, 128, 1024
    assert lib.vr_tune_record(C.byref(sp.spec), rows, C.byref(slower), C.c_double(1e9)) == N.VR_OK

    fields = ("tier", "warp_agg", "threads", "blocks_per_sm", "tile_rows", "smem_slots", "table_capacity")
    got = N.TuneChoice()
    assert lib.vr_tune_lookup(C.byref(sp.spec), rows + 100_000, C.byref(got)) == 1
    assert [getattr(got, f) for f in fields] == [getattr(t, f) for f in fields]
    assert lib.vr_tune_lookup(C.byref(sp.spec), 1000, C.byref(got)) == 0

    path = tmp_path / "tune.txt"
    assert lib.vr_tune_save(str(path).encode()) == N.VR_OK
    text = path.read_text()
    # a file with that entry's threads changed, loaded back: the lookup follows it
    lines = [ln for ln in text.splitlines() if ln and not ln.startswith("#")]
    assert lines
    edited = []
    for ln in lines:
        f = ln.split()
        if int(f[5]) == 256 and int(f[7]) == 512:  # threads, tile_rows of the recorded choice
            f[5] = "192"
        edited.append(" ".join(f))
    path.write_text("\n".join(edited) + "\n")
    assert lib.vr_tune_load(str(path).encode()) == N.VR_OK
    assert lib.vr_tune_lookup(C.byref(sp.spec), rows, C.byref(got)) == 1
    assert got.threads == 192 and got.tile_rows == 512 and got.smem_slots == 512


def test_plan_shares_accumulators_between_functions():
    """The decimal report's seven functions need six accumulators: avg(qty)
    reuses sum(qty)'s sum, and every count of a non-nullable input is the
    row count."""
    from vecruntime_b200 import datagen as G

    sp = G.decimal_report(rows=100).spec()
    info = N.PlanInfo()
    types = (N.ColumnType * 64)()
    assert N.lib().vr_agg_plan(C.byref(sp.spec), C.byref(info), types, 64) == N.VR_OK
    assert info.num_ops == 6 and info.direct_ok == 1


def test_tuner_key_tells_apart_specs_that_differ_only_in_types_or_flags():
    """Two specs that differ only in a decimal precision, a function flag or
    a product term get separate tuner entries."""
    lib = N.lib()
    cols = [vr.longs(np.zeros(1, np.int64), nullable=False), vr.decimals(np.zeros(1), 12, 2, nullable=False)]
    base = vr.Spec(cols, [0], [vr.WideDecimalSumAgg(1, 22, 2)])
    other_prec = vr.Spec(cols, [0], [vr.WideDecimalSumAgg(1, 23, 2)])
    other_flag = vr.Spec(cols, [0], [vr.WideDecimalSumAgg(1, 22, 2, null_on_overflow=False)])
    rows = 5_000_011
    t = N.TuneChoice()
    t.tier, t.threads, t.tile_rows = 2, 128, 512
    assert lib.vr_tune_record(C.byref(base.spec), rows, C.byref(t), C.c_double(1e9)) == N.VR_OK
    out = N.TuneChoice()
    assert lib.vr_tune_lookup(C.byref(base.spec), rows, C.byref(out)) == 1
    assert lib.vr_tune_lookup(C.byref(other_prec.spec), rows, C.byref(out)) == 0
    assert lib.vr_tune_lookup(C.byref(other_flag.spec), rows, C.byref(out)) == 0
