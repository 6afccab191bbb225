"""Benchmark of the GPU grouped aggregate (one JSON line on stdout, rank 0).

The default run (`--workload all`) measures the metric's own comparison and
every other workload in one line:

* top level -- batched uneven instances: 512 independent aggregates (rows
  log-uniform 2^10..2^22, cardinality log-uniform 1..2^20; int64 key, int64 +
  float64 values; count/sum/min/max) in ONE persistent launch replayed from a
  CUDA graph. `value` = rows/s of that launch with the inputs resident in HBM
  (6.7 GB, larger than the 126 MB L2); `one_launch_per_instance` times the
  same instances with one launch per instance, each with its own launch
  configuration, and `speedup_vs_one_launch_per_instance` is their ratio.
  `e2e` is the same step through the public API from pinned host memory:
  every instance's inputs copied host->device, the persistent launch, and
  every instance's groups emitted into pinned host buffers.
* `workloads.{decimal,highcard,plain}` -- the low-cardinality decimal report
  (60M rows, dictionary keys, exact decimal sums of fused products), the
  high-cardinality composite key (100M rows, Zipf(1.1) int64 x int32[16],
  1% null keys) and the plain aggregation (1,048,576 rows, 1,000 groups).
  A step is one table clear + one aggregate launch over a device-resident
  batch; a 1 GiB write on the stream precedes each step's start event, so
  L2 is cold and the device is busy while the host submits the step. `e2e`
  goes through the public C ABI with pinned host buffers (chunked H2D
  overlapping the kernels, groups emitted into pinned buffers).
* `workloads.parquet` -- the scan that feeds the aggregate: a 60M-slot
  dictionary-encoded string column chunk (3,000 v1 RLE_DICTIONARY data pages
  of 20,000 slots, 17-bit ids, 1% nulls) resident in HBM, decoded into Arrow int32 ids and a
  validity bitmap by one vr_pq_decode per step; parity is bit-exact against
  the oracle's page decode, `e2e` copies the pages in and the column out.
* `serving` -- 16 live queries fed by a seeded Poisson trace of 2,000
  requests/s for 5 minutes (one GPU): p50/p99 latency, queue wait, rows/s,
  the most requests in flight at once.

Every record carries `roofline` (algorithmic bytes / kernel time against the
measured HBM copy bandwidth), `cpu_baseline` (the CPU port of the reference's
aggregate on the host cores, a bounded sample) and `parity`: after the timed
steps, the groups of the full-size run are compared with the CPU port of the
reference (groups as a sorted multiset; keys, counts, integer and decimal
sums and min/max bit-exact; FP64 sums within 1e-12 relative of a compensated
sum). --workload decimal|plain|highcard|batched|serving|parquet prints one of them as
its own line; --impl reference times the CPU port on the host cores instead.

Multi-GPU (torchrun): every rank aggregates its own replica (weak scaling, no
collective on the data path); time = max over ranks; serving, parity and the
CPU legs run at one GPU only.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import ctypes as C
import hashlib
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "rows/s & HBM GB/s (% of peak), batched vs plain on 1 B200; serving p50/p99 ms"
FLUSH_BYTES = 1 << 30  # written on the step's stream before each step's start event
# What the CPU baseline runs: the oracle, a scalar C++ restatement of the
# reference's general probe path, not the reference's Java Vector API code
# (no JDK on the GPU box). The reference's own Q1 aggregate is about 2x faster
# per core than this port (docs/results.md:1654-1666), so a ratio against it
# overstates the lead over the real Vector API path by about that much.
PORT_NOTE = ("scalar C++ restatement of the reference's general-probe aggregate (GroupKeyTable.lookupOrInsert + "
             "GroupedAccumulators), not its SIMD Vector API path; about half the reference's published per-core rate")
# the kernels, the per-spec source generator, the planner (slot layout) and
# the launch-shape choice: what a DRAM byte count depends on (the batched
# launch's also on batched.cu, the page decoder's on its own source alone)
KERNEL_SOURCES = ("agg_main.cuh", "agg_device.cuh", "agg_types.h", "vr_internal.h", "agg_kernels.cu", "jit.cpp",
                  "plan.cpp", "abi.cu")
BATCHED_SOURCES = KERNEL_SOURCES + ("batched.cu",)
PARQUET_SOURCES = ("parquet.cu",)
TRAFFIC_SOURCES = {"batched": BATCHED_SOURCES, "parquet": PARQUET_SOURCES}

# DRAM bytes (read + write) per aggregate launch, dram__bytes_read.sum +
# dram__bytes_write.sum of one ncu capture, with the sha1 prefix of the
# sources it was taken on (KERNEL_SOURCES): a figure whose sources changed
# since is reported as null, not carried over. Scaling to the timed launch:
#   "rows"   -- traffic is the input plus a fixed part: scaled by rows;
#   "approx" -- a hash table's slot traffic per row grows slowly with the
#               group count; scaled by rows from the smaller capture, so a
#               little low (earlier sources: 93 B/row at 8M high-cardinality
#               rows, 103 B/row at 100M);
#   "l2"     -- scaled by rows from a capture whose intermediate arrays
#               stayed in L2: a lower bound at sizes where they do not;
#   "exact"  -- captured at the timed size.
TRAFFIC = {
    # name: (kernel sources sha1 prefix, rows captured, GB per launch, scaling)
    "decimal": ("c54880b41264", 8_000_000, (320.077568e6 + 7.250432e6) / 1e9, "rows"),
    "plain": ("c54880b41264", 1 << 20, (25.449984e6 + 768) / 1e9, "exact"),
    "highcard": ("c54880b41264", 8_000_000, (555.012608e6 + 186.404096e6) / 1e9, "approx"),
    "batched": ("1d46e382ca92", 30_418_299, (1.659858e9 + 712.077568e6) / 1e9, "approx"),
    # the walk, expand and gather kernels (the CUB rank scan not captured)
    "parquet": ("4cc0acd4e6f3", 8 << 20, (8.64768e6 + 20.52864e6 + 35.454464e6 + 0.002048e6 + 0.084224e6 + 1.069056e6)
                / 1e9, "l2"),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def kernel_sha(sources=KERNEL_SOURCES) -> str:
    h = hashlib.sha1()
    for f in sources:
        with open(os.path.join(ROOT, "vecruntime_b200", "csrc", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:12]


def launch_traffic(name, rows):
    """(GB per launch, how it was obtained) or (None, why not)."""
    src = "ncu dram__bytes_read.sum + dram__bytes_write.sum"
    t = TRAFFIC.get(name)
    if t is None:
        return None, "no ncu capture of this workload"
    sha, at, gb, scaling = t
    now = kernel_sha(TRAFFIC_SOURCES.get(name, KERNEL_SOURCES))
    if sha != now:
        return None, f"no ncu capture of the current kernel sources ({now}); the last one was taken on {sha or 'older sources'}"
    if rows == at:
        return gb, f"GB per launch ({src}, capture of this workload on kernel sources {sha})"
    if scaling == "rows":
        return gb * rows / at, f"GB per launch ({src}, {at}-row capture on kernel sources {sha}, scaled by rows)"
    if scaling == "l2":
        return gb * rows / at, (f"GB per launch ({src}, {at}-row capture on kernel sources {sha}, scaled by rows; "
                                "the capture's intermediates stayed in L2, so a lower bound)")
    if scaling == "approx":
        return gb * rows / at, (f"GB per launch ({src}, {at}-row capture on kernel sources {sha}, scaled by rows; "
                                "table traffic per row grows slowly with groups, so a little low)")
    return None, "no capture at this row count (table traffic follows the group count, not the rows)"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if "hbm_gbs" in d:
            return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event reasons of the GPU under test, polled through
    NVML every ~2 ms while the timed region runs (nvidia-smi's fastest period
    is longer than a short timed region). The GPU is found by PCI bus id, so
    the CUDA index and the NVML index may differ."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, cuda_index: int, period_s: float = 0.002):
        self.cuda_index = cuda_index
        self.period = period_s
        self.rows = []  # (sm_mhz, reasons bitmask)
        self.max_mhz = None
        self.error = None
        self._stop = threading.Event()
        self._t = None

    def _handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.cuda_index)
        bus = "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def __enter__(self):
        try:
            self.nvml, self.h = self._handle()
            self.max_mhz = self.nvml.nvmlDeviceGetMaxClockInfo(self.h, self.nvml.NVML_CLOCK_SM)
            self._sample()
            self._t = threading.Thread(target=self._loop, daemon=True)
            self._t.start()
        except Exception as e:  # no NVML: the line says so instead of a number
            self.error = f"{type(e).__name__}: {e}"
        return self

    def _sample(self):
        sm = self.nvml.nvmlDeviceGetClockInfo(self.h, self.nvml.NVML_CLOCK_SM)
        reasons = self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        self.rows.append((sm, reasons))

    def _loop(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception as e:
                self.error = f"{type(e).__name__}: {e}"
                return
            time.sleep(self.period)

    def __exit__(self, *exc):
        self._stop.set()
        if self._t is not None:
            self._t.join(timeout=5)
            try:
                self._sample()
            except Exception:
                pass

    def summary(self):
        sm = [r[0] for r in self.rows]
        reasons = sorted({name for _, bits in self.rows for name, bit in self.REASONS.items() if bits & bit})
        out = {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
               "samples": len(sm), "source": "nvml, polled every %.0f ms during the timed region" % (self.period * 1e3)}
        if self.error:
            out["error"] = self.error
        return out


# ------------------------------------------------------------------ workloads
def make_workload(name, rows=None):
    from vecruntime_b200 import datagen as G

    if name == "decimal":
        return G.decimal_report(rows=rows or 60_000_000)
    if name == "plain":
        return G.plain(rows=rows or (1 << 20))
    if name == "highcard":
        return G.high_cardinality(rows=rows or 100_000_000)
    raise ValueError(name)


def output_row_bytes(types):
    b = 0.0
    for t in types:
        b += {1: 4, 2: 8, 3: 8, 4: 0.125, 5: 16, 6: 4}[t.lane] + 0.125
    return b


def device_batch(w, device):
    import torch

    from vecruntime_b200 import columns as Cc

    db, tensors = Cc.to_device(w.batch(), device)
    torch.cuda.synchronize(device)
    return db, tensors


def pin(a, lib, bufs):
    """A copy of array `a` in pinned host memory (vr_host_alloc); the
    allocation is appended to `bufs` for vr_host_free."""
    if a is None:
        return None
    a = np.ascontiguousarray(a)
    p = C.c_void_p()
    rc = lib.vr_host_alloc(max(a.nbytes, 16), C.byref(p))
    assert rc == 0, "pinned allocation"
    dst = np.ctypeslib.as_array((C.c_uint8 * max(a.nbytes, 1)).from_address(p.value))[:a.nbytes]
    dst = dst.view(a.dtype).reshape(a.shape)
    dst[...] = a
    bufs.append(p)
    return dst


def pinned_copy(w, lib, bufs):
    """The workload's columns copied into pinned host memory (vr_host_alloc)."""
    from vecruntime_b200 import columns as Cc

    cols = []
    for c in w.columns:
        n = Cc.Col(c.lane, pin(c.data, lib, bufs), pin(c.validity, lib, bufs), c.precision, c.scale, c.dict_size,
                   c.nullable)
        if c.lane == 4:
            n._n = c._n
        cols.append(n)
    return cols


def host_threads():
    return os.cpu_count() or 1


# ------------------------------------------------------------------ CPU legs
def cpu_baseline(w, sample_rows, threads):
    """One timed pass of the oracle over the first `sample_rows` rows:
    (rows/s, seconds)."""
    from oracle import pyoracle as O
    from vecruntime_b200 import datagen as G

    sub = G.Workload(w.name, w.columns, w.keys, w.functions, w.est_groups, w.rows)
    batch = sub.batch(0, sample_rows)
    secs, groups = O.run_threads(w.spec(), batch, threads, 4096)
    return sample_rows / secs, secs


def cpu_sample(w, threads, target_s):
    """A bounded sample of about `target_s` seconds of oracle work on the
    workload: a pilot pass on 1M rows sizes it, then whole passes over a row
    prefix (the full input, repeated, when it is fast enough).
    Returns (rows/s, description)."""
    pilot = min(w.rows, 1 << 20)
    rate, _ = cpu_baseline(w, pilot, threads)
    rows = int(min(w.rows, max(pilot, rate * target_s)))
    passes = max(1, min(5000, int(target_s / (rows / rate))))
    done, secs = 0, 0.0
    for _ in range(passes):
        _, s = cpu_baseline(w, rows, threads)
        done += rows
        secs += s
    desc = (f"{passes} pass(es) over {rows} of {w.rows} rows, {threads} threads (one partition each, "
            f"4096-row batches, partitions merged), {secs:.1f} s")
    return done / secs, desc


def cpu_batched(ws, threads, target_s):
    """The oracle over whole instances of the batched workload, one instance
    per host thread at a time (one Spark task each), until about `target_s`
    seconds of wall time have passed or every instance ran once.
    Returns (rows/s, description)."""
    from oracle import pyoracle as O

    def one(w):
        o = O.Oracle(w.spec())
        o.update(w.batch(), 4096)
        o.close()
        return w.rows

    t0 = time.perf_counter()
    rows, done = 0, 0
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        futs = []
        it = iter(ws)
        for w in it:  # keep every thread busy; stop feeding once the time is up
            futs.append(ex.submit(one, w))
            if len(futs) >= threads:
                rows += futs.pop(0).result()
                done += 1
                if time.perf_counter() - t0 > target_s:
                    break
        for f in futs:
            rows += f.result()
            done += 1
    secs = time.perf_counter() - t0
    desc = (f"{done} of {len(ws)} instances ({rows} rows), {threads} threads (one instance per thread, "
            f"4096-row batches), {secs:.1f} s")
    return rows / secs, desc


def check_parity(spec, got_types, got_arrays, got_n, batch, threads):
    """The full-size run's groups against the CPU port of the reference."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import pyoracle as O
    from parity import compare_arrays

    t0 = time.perf_counter()
    o = O.Oracle(spec)
    o.update_threads(batch, threads)
    want_n = o.num_groups()
    want = o.emit(O.ORC_FP_COMPENSATED)
    wt = o.output_types
    o.close()
    bad, ex = compare_arrays(spec, got_types, got_arrays, got_n, wt, want, want_n)
    return {"groups": int(got_n), "oracle_groups": int(want_n), "mismatches": int(bad),
            "examples": [str(e) for e in ex[:3]], "rows_checked": int(batch.num_rows),
            "rule": "sorted multiset of groups; exact but FP64 sums (1e-12 relative of a compensated sum)",
            "oracle_s": round(time.perf_counter() - t0, 1)}


# ------------------------------------------------------------------ single workloads
def run_single(args, name, rank, world, device, check):
    import torch

    import vecruntime_b200 as vr
    from vecruntime_b200 import datagen as G
    from vecruntime_b200 import native as N

    torch.cuda.set_device(device)
    lib = N.lib()
    w = make_workload(name, args.rows if args.workload == name else None)
    log(f"[rank {rank}] workload {w.name}: {w.rows} rows, est groups {w.est_groups}")
    db, tensors = device_batch(w, device)
    tuned = None
    forced = None
    if args.shape:
        # a fixed launch shape (tier, threads, CTAs per SM, tile rows, shared
        # slots, warp pre-aggregation), e.g. the one the autotuner picked at
        # full size, for a profile of a smaller case
        t, th, ctas, tile, slots, wa = (int(x) for x in args.shape.split(","))
        forced = N.TuneChoice(t, wa, th, ctas, tile, slots, 0)
        tuned = {"forced": args.shape}
    elif name in ("highcard", "plain") and not args.no_tune:
        # the autotuner, before anything is timed: every candidate shape and
        # shared-memory size on this batch; the handle below finds the fastest
        from vecruntime_b200 import aggregate as A

        t0 = time.perf_counter()
        best, rps = A.tune_search(w.columns, w.keys, w.functions, db, est_groups=w.est_groups, max_batch_rows=w.rows,
                                  device=device, iters=2)
        tuned = {"tier": best.tier, "threads": best.threads, "ctas_per_sm": best.blocks_per_sm,
                 "tile_rows": best.tile_rows, "smem_slots": best.smem_slots, "warp_agg": best.warp_agg,
                 "seconds": round(time.perf_counter() - t0, 1)}
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=w.rows,
                              device=device, flags=N.VR_SPEC_TRACE, tune=forced)
    launch = agg.stats()
    stream = torch.cuda.ExternalStream(agg.stream(), device=torch.device("cuda", device))
    in_bytes = G.input_bytes(w)
    # before each step's start event, a 1 GiB write on the same stream: it
    # evicts the inputs from L2 (126 MB) when they would fit there, and it
    # keeps the device busy while the host submits the step, so the events
    # time the step's device work rather than the host's submission latency
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=device)
    for _ in range(args.warmup):
        agg.reset()
        agg.consume(db)
        agg.sync()
    st0 = agg.stats()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    dist_barrier(world)
    torch.cuda.synchronize(device)
    with ClockSampler(device) as clocks:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            agg.reset()
            agg.consume(db)
            ev[i][1].record(stream)
            agg.sync()
        torch.cuda.synchronize(device)
    dist_barrier(world)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    st1 = agg.stats()
    kernel_ms = (st1.total_kernel_ms - st0.total_kernel_ms) / args.steps
    launches = st1.kernel_launches - st0.kernel_launches
    ms_per_step, value = weak_scaling(sum(step_ms), args.steps, w.rows, world, device)
    groups = agg.num_groups()
    out_types = agg.output_types
    parity = None
    if check:
        got = agg.emit()
        parity = check_parity(w.spec(), out_types, got, groups, w.batch(), host_threads())
        del got
    agg.close()
    del tensors, flush

    out_bytes = groups * output_row_bytes(out_types)
    alg_bytes = in_bytes + out_bytes
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    traffic, traffic_unit = launch_traffic(w.name, w.rows)
    rec = {
        "value": value, "unit": "rows/s", "ms_per_step": ms_per_step, "steps": args.steps, "warmup": args.warmup,
        "dtype": workload_dtype(w),
        "config": {"workload": workload_label(w), "rows_per_gpu": w.rows, "groups": groups,
                   "batch": "one device-resident batch per step",
                   "launch": {"tier": launch.tier, "threads": launch.threads, "blocks": launch.blocks,
                              "tile_rows": launch.tile_rows, "smem_bytes": launch.smem_bytes, "jit": launch.jit},
                   "autotuner": tuned,
                   "l2": "L2 flushed before each step (%d MB written on the stream outside the timed events; "
                         "inputs %.3f GB)" % (FLUSH_BYTES >> 20, in_bytes / 1e9)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "traffic_unit": traffic_unit,
                     "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": kernel_ms},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
        "parity": parity,
    }
    if not args.no_e2e:
        e2e = run_e2e(args, w, lib, device)
        e2e["value"] = dist_min(e2e["value"], world, device) * world
        rec["e2e"] = e2e
    if check and not args.no_cpu_baseline:
        rate, desc = cpu_sample(w, host_threads(), args.cpu_seconds)
        rec["cpu_baseline"] = {"value": rate, "unit": "rows/s", "cores": host_threads(), "kind": "port", "port": PORT_NOTE,
                               "sample": desc}
    return rec


def workload_dtype(w):
    return "int64 (exact decimal128 sums)" if w.name == "decimal" else "int64/f64"


def workload_label(w):
    n = f"{w.rows // 1_000_000}M rows" if w.rows % 1_000_000 == 0 else f"{w.rows:,} rows"
    return {"decimal": f"low-cardinality decimal report: {n}, 2 dictionary keys (3x2 -> 6 groups), "
                       "4 DECIMAL(12,2) columns, exact decimal(38,6) sums",
            "plain": f"plain grouped aggregation: {n}, int64 key over 1,000 values, 5% nulls",
            "highcard": f"high-cardinality composite key: {n}, Zipf(1.1) int64 x int32[16], 1% null keys"
            }.get(w.name, w.name)


def run_e2e(args, w, lib, device):
    import torch

    import vecruntime_b200 as vr
    from vecruntime_b200 import columns as Cc
    from vecruntime_b200 import datagen as G

    bufs = []
    cols = pinned_copy(w, lib, bufs)
    chunk = min(w.rows, args.chunk_rows)
    chunk -= chunk % 128 if chunk > 128 else 0
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=chunk,
                              device=device)
    stream = torch.cuda.ExternalStream(agg.stream(), device=torch.device("cuda", device))
    bl = []
    for lo in range(0, w.rows, chunk):
        hi = min(w.rows, lo + chunk)
        bl.append(Cc.HostBatch([G.slice_col(c, lo, hi) for c in cols], hi - lo))
    in_bytes = G.input_bytes(w)
    d2h = 0
    times = []
    # the groups come back into pinned buffers allocated once (the first
    # warm-up step sizes them), as a caller with a pinned output pool would
    out_pinned = None
    for it in range(max(1, args.warmup) + args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        agg.reset()
        for hb in bl:
            agg.consume(hb)
        out = agg.emit(out=out_pinned) if out_pinned is not None else agg.emit()
        b.record(stream)
        torch.cuda.synchronize(device)
        if it >= max(1, args.warmup):
            times.append(a.elapsed_time(b))
        d2h = sum(d.nbytes + v.nbytes for d, v in out)
        if out_pinned is None:
            out_pinned = [(pin(d, lib, bufs), pin(v, lib, bufs)) for d, v in out]
    agg.close()
    for p in bufs:
        lib.vr_host_free(p)
    ms = float(np.mean(times))
    return {"value": w.rows / (ms * 1e-3), "unit": "rows/s", "h2d_bytes_per_step": in_bytes,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms, "chunk_rows": chunk}


# ------------------------------------------------------------------ Parquet pages
# pages of 20,000 slots: the page row limit the reference's writer uses by
# default (IcebergParquetAppender.java:151-153, Iceberg's page row limit)
PQ_ROWS, PQ_PAGE_ROWS, PQ_DICT, PQ_NULLS = 60_000_000, 20_000, 100_000, 0.01


def parquet_ids(rows):
    """The chunk's ids (uniform over 100,000 entries, 17-bit) and nulls (1%)."""
    from vecruntime_b200 import datagen as G

    rng = np.random.default_rng(G.SEEDS["parquet"])
    ids = rng.integers(0, PQ_DICT, size=rows).astype(np.int32)
    nulls = rng.random(rows) < PQ_NULLS
    return ids, nulls


def parquet_chunk(rows):
    """A dictionary-encoded string column chunk: v1 RLE_DICTIONARY data pages
    of 20,000 slots over `parquet_ids`."""
    from vecruntime_b200 import datagen as G

    ids, nulls = parquet_ids(rows)
    return G.dictionary_pages(ids, nulls, 17, PQ_PAGE_ROWS)


def run_parquet_aggregate(args, out, valid, rows, device, check):
    """The decoded column straight into the aggregate: count(*) grouped by
    the string key, the chunk's 100,000-entry dictionary attached as a batch
    dictionary (the aggregate maps it onto its table's once per batch). A
    step resets the table and consumes the device-resident decoded column."""
    import torch

    import vecruntime_b200 as vr
    from vecruntime_b200 import aggregate as A
    from vecruntime_b200 import columns as Cc

    words = [f"customer-{i:06d}" for i in range(PQ_DICT)]
    dict_ = Cc.dictionary(words)
    key = Cc.dict_strings(np.zeros(1, np.int32), dict_, np.zeros(1, bool), nullable=True)
    db1, keep = Cc.to_device(Cc.HostBatch([key], 1), device)  # the dictionary in device memory
    batch = Cc.DeviceBatch(rows, [out.data_ptr()], [valid.data_ptr()], dictionaries=db1.dictionaries)
    from vecruntime_b200 import native as N

    agg = vr.GpuHashAggregate([key], [0], [A.CountAgg()], est_groups=PQ_DICT + 1, max_batch_rows=rows,
                              device=device, flags=N.VR_SPEC_TRACE)
    stream = torch.cuda.ExternalStream(agg.stream(), device=torch.device("cuda", device))
    times = []
    k0 = 0.0
    for it in range(args.warmup + args.steps):
        if it == args.warmup:
            k0 = agg.stats().total_kernel_ms
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        agg.reset()
        agg.consume(batch)
        b.record(stream)
        agg.sync()
        if it >= args.warmup:
            times.append(a.elapsed_time(b))
    kernel_ms = (agg.stats().total_kernel_ms - k0) / max(1, args.steps)
    groups = agg.num_groups()
    rec = {"ms_per_step": float(np.mean(times)), "rows/s": rows / (float(np.mean(times)) * 1e-3), "groups": groups,
           "kernel_ms": kernel_ms,
           "what": "count(*) group by the decoded string key (VR_DICT32 + batch dictionary), device-resident; "
                   "the step includes the host's mapping of the 100,000-entry dictionary"}
    if check:
        got = agg.emit()
        strings = agg.key_dictionary(0)
        kd, kv = got[0]
        cd = np.asarray(got[1][0])[:groups].astype(np.int64)
        kvalid = Cc.unpack_bits(kv, groups)
        ids, nulls = parquet_ids(rows)
        want = np.bincount(ids[~nulls], minlength=PQ_DICT)
        counts = np.zeros(PQ_DICT, np.int64)
        null_count = 0
        for g in range(groups):
            if kvalid[g]:
                counts[int(strings[int(kd[g])][len("customer-"):])] += cd[g]
            else:
                null_count += int(cd[g])
        bad = int((counts != want).sum()) + int(null_count != int(nulls.sum()))
        rec["parity"] = {"groups": groups, "want_groups": int((want > 0).sum()) + int(nulls.any()),
                         "mismatches": bad, "rule": "per-string counts and the null group's count, exact"}
    agg.close()
    return rec


def pq_pages_on(blob_ptr, pages):
    from vecruntime_b200 import parquet as P

    out, at = [], 0
    for b, f in pages:
        out.append(P.Page(blob_ptr + at, len(b), f["num_values"], f["max_def_level"], bool(f["v2"]),
                          f["levels_length"], f["encoding"], f["value_bytes"]))
        at += len(b)
    return out


def pq_oracle(pages, threads):
    """The oracle's decode of every page (ParquetPageDecoder.decode restated),
    pages spread over `threads` host threads: (ids, validity bits, seconds)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import pyoracle as O

    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        res = list(ex.map(lambda pf: O.pq_decode_page(pf[0], **pf[1]), pages))
    secs = time.perf_counter() - t0
    ids = np.concatenate([r[0].view(np.int32) for r in res])
    valid = np.concatenate([np.unpackbits(r[1], bitorder="little")[:f["num_values"]] for r, (_, f) in zip(res, pages)])
    return ids, valid.astype(bool), secs


def run_parquet(args, rank, world, device, check):
    """Parquet feed: a 60M-slot column chunk's RLE_DICTIONARY data pages,
    resident in HBM, decoded into Arrow ids + validity (vr_pq_decode)."""
    import torch

    from vecruntime_b200 import parquet as P

    torch.cuda.set_device(device)
    rows = args.rows if (args.rows and args.workload == "parquet") else PQ_ROWS
    pages = parquet_chunk(rows)
    blob = b"".join(b for b, _ in pages)
    page_bytes = len(blob)
    log(f"[rank {rank}] parquet: {rows} slots in {len(pages)} pages, {page_bytes / 1e6:.1f} MB")
    dev = torch.device("cuda", device)
    dblob = torch.frombuffer(bytearray(blob + b"\0" * 16), dtype=torch.uint8).to(dev)
    dpages = pq_pages_on(dblob.data_ptr(), pages)
    out = torch.empty(rows * 4 + 16, dtype=torch.uint8, device=dev)
    vbytes = ((rows + 7) // 8 + 15) // 16 * 16 + 16
    valid = torch.zeros(vbytes, dtype=torch.uint8, device=dev)
    dec = P.PageDecoder(rows, page_bytes, device=device)
    dpages = dec.descriptors(dpages)  # built once: the chunk's page descriptors
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        dec.decode(dpages, out.data_ptr(), valid.data_ptr(), stream.cuda_stream)
        dec.sync()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    dist_barrier(world)
    torch.cuda.synchronize(device)
    present = 0
    with ClockSampler(device) as clocks:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            dec.decode(dpages, out.data_ptr(), valid.data_ptr(), stream.cuda_stream)
            ev[i][1].record(stream)
            present = dec.sync()
        torch.cuda.synchronize(device)
    dist_barrier(world)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ms_per_step, value = weak_scaling(sum(step_ms), args.steps, rows, world, device)
    parity = None
    if check:
        want_ids, want_valid, osecs = pq_oracle(pages, host_threads())
        got_ids = out[:rows * 4].cpu().numpy().view(np.int32)
        got_valid = np.unpackbits(valid.cpu().numpy(), bitorder="little")[:rows].astype(bool)
        bad = int((got_ids != want_ids).sum() + (got_valid != want_valid).sum())
        parity = {"slots": rows, "present": int(present), "oracle_present": int(want_valid.sum()),
                  "mismatches": bad, "rule": "bit-exact ids and validity against the oracle's page decode",
                  "oracle_s": round(osecs, 1)}
    del flush
    out_bytes = rows * 4 + (rows + 7) // 8
    alg = page_bytes + out_bytes
    peak, peak_kind = measured_peaks()
    traffic, traffic_unit = launch_traffic("parquet", rows)
    kernel_ms = float(np.mean(step_ms))
    rec = {
        "value": value, "unit": "rows/s", "ms_per_step": ms_per_step, "steps": args.steps, "warmup": args.warmup,
        "dtype": "u8/u32 (bit unpacking)",
        "config": {"workload": f"Parquet feed: {rows} slots of a dictionary-encoded string column (100,000 entries, "
                               f"17-bit ids, 1% nulls) in {len(pages)} v1 RLE_DICTIONARY data pages of 20,000 slots "
                               "-> Arrow int32 ids + validity",
                   "rows_per_gpu": rows, "page_bytes": page_bytes, "pages": len(pages),
                   "batch": "the column chunk's pages resident in HBM, one vr_pq_decode per step",
                   "l2": "L2 flushed before each step (%d MB written on the stream outside the timed events)"
                         % (FLUSH_BYTES >> 20)},
        "roofline": {"bound": "hbm", "achieved": alg / (kernel_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (kernel_ms * 1e-3) / 1e9 / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "traffic_unit": traffic_unit, "algorithmic_bytes_per_launch": alg,
                     "kernel_ms": kernel_ms, "kernel_ms_is": "the decode's kernels (run walk, expand, rank scan, gather)"},
        "gpu_launches": 5 * args.steps,
        "clocks": clocks.summary(),
        "parity": parity,
    }
    rec["then_aggregate"] = run_parquet_aggregate(args, out, valid, rows, device, check)
    if not args.no_e2e:
        rec["e2e"] = run_parquet_e2e(args, dec, pages, blob, rows, device)
        rec["e2e"]["value"] = dist_min(rec["e2e"]["value"], world, device) * world
    if check and not args.no_cpu_baseline:
        from oracle import pyoracle as O

        # every page, each into its own buffers as the reference's decoder
        # returns them, on all host threads; best of three passes
        secs = min(O.pq_decode_pages_threads(pages, host_threads())[2] for _ in range(3))
        rec["cpu_baseline"] = {"value": rows / secs, "unit": "rows/s", "cores": host_threads(), "kind": "port",
                               "port": "scalar C++ restatement of the reference's ParquetPageDecoder.decode + "
                                       "RleBitPackingReader.readInts (ids not resolved), pages spread over threads",
                               "sample": f"all {len(pages)} pages ({rows} slots), {host_threads()} threads, "
                                         f"{secs:.3f} s (best of 3)"}
    dec.close()
    return rec


def run_parquet_e2e(args, dec, pages, blob, rows, device):
    """The same decode through the public API from host memory: every step
    copies the pages from pinned host memory to the device, decodes them, and
    copies the ids and validity back into pinned buffers."""
    import torch

    dev = torch.device("cuda", device)
    hblob = torch.frombuffer(bytearray(blob + b"\0" * 16), dtype=torch.uint8).pin_memory()
    dblob = torch.empty_like(hblob, device=dev)
    dpages = dec.descriptors(pq_pages_on(dblob.data_ptr(), pages))
    out = torch.empty(rows * 4 + 16, dtype=torch.uint8, device=dev)
    vbytes = ((rows + 7) // 8 + 15) // 16 * 16 + 16
    valid = torch.zeros(vbytes, dtype=torch.uint8, device=dev)
    hout = torch.empty(rows * 4, dtype=torch.uint8).pin_memory()
    hvalid = torch.empty((rows + 7) // 8, dtype=torch.uint8).pin_memory()
    stream = torch.cuda.Stream(device=dev)
    times = []
    for it in range(max(1, args.warmup) + args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
            dblob.copy_(hblob, non_blocking=True)
            dec.decode(dpages, out.data_ptr(), valid.data_ptr(), stream.cuda_stream)
            hout.copy_(out[:rows * 4], non_blocking=True)
            hvalid.copy_(valid[:(rows + 7) // 8], non_blocking=True)
            b.record(stream)
        dec.sync()
        torch.cuda.synchronize(device)
        if it >= max(1, args.warmup):
            times.append(a.elapsed_time(b))
    ms = float(np.mean(times))
    return {"value": rows / (ms * 1e-3), "unit": "rows/s", "h2d_bytes_per_step": len(blob),
            "d2h_bytes_per_step": rows * 4 + (rows + 7) // 8, "ms_per_step": ms}


# ------------------------------------------------------------------ batched
def run_batched(args, rank, world, device, check):
    """512 uneven instances: one persistent launch replayed from a CUDA graph
    against one launch per instance. A step resets every table and
    aggregates every instance's device-resident batch."""
    import torch

    import vecruntime_b200 as vr
    from vecruntime_b200 import columns as Cc
    from vecruntime_b200 import datagen as G
    from vecruntime_b200 import native as N

    torch.cuda.set_device(device)
    lib = N.lib()
    ws = G.batched_instances(n=args.instances)
    rows = sum(w.rows for w in ws)
    in_bytes = sum(G.input_bytes(w) for w in ws)
    log(f"[rank {rank}] batched: {len(ws)} instances, {rows} rows, {sum(w.est_groups for w in ws)} est groups")
    dbs, keep = [], []
    for w in ws:
        db, t = Cc.to_device(w.batch(), device)
        dbs.append(db)
        keep.append(t)

    def handles():
        # each instance's own launch configuration: the autotuner's choice for
        # its (rows, estimated groups) bucket when it has one, else the default
        return [vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=w.rows,
                                    device=device) for w in ws]

    # the autotuner, before anything is timed: each estimated-groups bucket's
    # shared-memory strategy chosen by timing the persistent launch; handles
    # made afterwards (for both forms below) find its choices
    aggs = handles()
    tuned_ms, tune_s = None, 0.0
    if not args.no_tune:
        tuner = vr.GpuBatchedAggregate(aggs, dbs, mode=N.VR_BATCHED_PERSISTENT)
        t0 = time.perf_counter()
        tuned_ms = tuner.tune(iters=2)
        tune_s = time.perf_counter() - t0
        tuner.close()
        for a in aggs:
            a.close()
        aggs = handles()
    stream = torch.cuda.Stream(device=device)

    def timed(b, steps, warmup):
        for _ in range(warmup):
            b.run(stream.cuda_stream)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        dist_barrier(world)
        torch.cuda.synchronize(device)
        for e0, e1 in ev:
            e0.record(stream)
            b.run(stream.cuda_stream)
            e1.record(stream)
        torch.cuda.synchronize(device)
        dist_barrier(world)
        return sum(a.elapsed_time(b) for a, b in ev)

    with ClockSampler(device) as clocks:
        persistent = vr.GpuBatchedAggregate(aggs, dbs, mode=N.VR_BATCHED_PERSISTENT, use_graph=True)
        ms_p, value = weak_scaling(timed(persistent, args.steps, args.warmup), args.steps, rows, world, device)
    info = persistent.info()
    plain = vr.GpuBatchedAggregate(aggs, dbs, mode=N.VR_BATCHED_PLAIN)
    ms_l, value_l = weak_scaling(timed(plain, args.steps, args.warmup), args.steps, rows, world, device)
    plain.close()
    # the groups of the persistent launch (the plain one ran last: run it once more)
    persistent.run(stream.cuda_stream)
    groups = [a.num_groups() for a in aggs]
    out_types = aggs[0].output_types
    parity = None
    if check:
        parity = check_batched(aggs, ws)
    persistent.close()
    peak, peak_kind = measured_peaks()
    out_bytes = sum(groups) * output_row_bytes(out_types)
    alg = in_bytes + out_bytes
    traffic, traffic_unit = launch_traffic("batched", rows)
    rec = {
        "value": value, "unit": "rows/s", "ms_per_step": ms_p, "steps": args.steps, "warmup": args.warmup,
        "dtype": "int64/f64",
        "config": {"workload": f"batched uneven instances: {len(ws)} aggregates, {rows} rows, rows log-uniform "
                               "2^10..2^22, cardinality log-uniform 1..2^20, int64 key, int64 + float64 values, "
                               "count/sum/min/max", "rows_per_gpu": rows, "groups": int(sum(groups)),
                   "mode": "one persistent launch replayed from a CUDA graph (table clears, aggregate, "
                           "status gather)",
                   "launch": info,
                   "autotuner": None if args.no_tune else {"tuned_ms": tuned_ms, "seconds": round(tune_s, 1),
                                 "what": "per estimated-groups bucket: whole shared-memory table, 256/512/1024-slot "
                                         "hot-key cache or HBM only, by coordinate descent on the launch's time; "
                                         "both forms below use the tuned choices"},
                   "l2": "inputs larger than L2 (%.2f GB)" % (in_bytes / 1e9)},
        "roofline": {"bound": "hbm", "achieved": alg / (ms_p * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (ms_p * 1e-3) / 1e9 / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "traffic_unit": traffic_unit,
                     "algorithmic_bytes_per_launch": alg,
                     "kernel_ms": ms_p, "kernel_ms_is": "the whole graph (table clears + aggregate + status gather)"},
        "one_launch_per_instance": {"value": value_l, "unit": "rows/s", "ms_per_step": ms_l,
                                    "launches_per_step": "per instance: table clear, control clear, aggregate"},
        "speedup_vs_one_launch_per_instance": ms_l / ms_p,
        "gpu_launches": 3 * args.steps,
        "clocks": clocks.summary(),
        "parity": parity,
    }
    if not args.no_e2e:
        e2e = run_batched_e2e(args, ws, aggs, dbs, keep, lib, device, stream)
        e2e["value"] = dist_min(e2e["value"], world, device) * world
        rec["e2e"] = e2e
    if check and not args.no_cpu_baseline:
        rate, desc = cpu_batched(ws, host_threads(), args.cpu_seconds)
        rec["cpu_baseline"] = {"value": rate, "unit": "rows/s", "cores": host_threads(), "kind": "port", "port": PORT_NOTE,
                               "sample": desc}
    for a in aggs:
        a.close()
    return rec


def check_batched(aggs, ws):
    """Every instance's groups against the oracle (one instance per host thread)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import pyoracle as O
    from parity import compare_arrays

    t0 = time.perf_counter()
    got = []
    for a in aggs:
        n = a.num_groups()
        got.append((n, a.emit()))

    def one(i):
        w = ws[i]
        o = O.Oracle(w.spec())
        o.update(w.batch(), 4096)
        want_n = o.num_groups()
        want = o.emit(O.ORC_FP_COMPENSATED)
        wt = o.output_types
        o.close()
        n, arrays = got[i]
        bad, ex = compare_arrays(w.spec(), aggs[i].output_types, arrays, n, wt, want, want_n)
        return bad, ex, want_n

    bad, groups, examples, wrong = 0, 0, [], 0
    with cf.ThreadPoolExecutor(max_workers=host_threads()) as ex:
        for i, (b, e, g) in enumerate(ex.map(one, range(len(ws)))):
            bad += b
            groups += g
            if b:
                wrong += 1
                examples += [f"instance {i}: {x}" for x in e[:1]]
    return {"groups": int(sum(n for n, _ in got)), "oracle_groups": int(groups), "mismatches": int(bad),
            "instances_with_mismatches": wrong, "examples": examples[:3],
            "rows_checked": int(sum(w.rows for w in ws)),
            "rule": "per instance, sorted multiset of groups; exact but FP64 sums (1e-12 relative of a compensated sum)",
            "oracle_s": round(time.perf_counter() - t0, 1)}


def run_batched_e2e(args, ws, aggs, dbs, keep, lib, device, stream):
    """The batched step through the public API from pinned host memory: every
    instance's input columns copied into its device batch, the persistent
    launch, every instance's groups emitted into pinned host buffers."""
    import torch

    import vecruntime_b200 as vr
    from vecruntime_b200 import native as N

    bufs = []
    src = []  # (pinned host tensor, device tensor) per input buffer
    for w, tensors in zip(ws, keep):
        arrays = [c.data for c in w.columns] + [c.validity for c in w.columns if c.validity is not None]
        for a, t in zip(arrays, tensors):
            p = pin(np.frombuffer(np.ascontiguousarray(a).tobytes(), np.uint8), lib, bufs)
            src.append((torch.from_numpy(p), t[:p.nbytes]))
    h2d = sum(h.numel() for h, _ in src)
    persistent = vr.GpuBatchedAggregate(aggs, dbs, mode=N.VR_BATCHED_PERSISTENT, use_graph=True)
    outs = None
    times = []
    for it in range(max(1, args.warmup) + args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        with torch.cuda.stream(stream):
            for h, d in src:
                d.copy_(h, non_blocking=True)
        persistent.run(stream.cuda_stream)
        if outs is None:
            res = [agg.emit() for agg in aggs]
            outs = [[(pin(d, lib, bufs), pin(v, lib, bufs)) for d, v in r] for r in res]
        else:
            for agg, o in zip(aggs, outs):
                agg.emit(out=o)
        b.record(stream)
        torch.cuda.synchronize(device)
        if it >= max(1, args.warmup):
            times.append(a.elapsed_time(b))
    d2h = sum(d.nbytes + v.nbytes for o in outs for d, v in o)
    persistent.close()
    for p in bufs:
        lib.vr_host_free(p)
    ms = float(np.mean(times))
    rows = sum(w.rows for w in ws)
    return {"value": rows / (ms * 1e-3), "unit": "rows/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": ms}


# ------------------------------------------------------------------ serving
def run_serving(args, device):
    """16 live queries (resident tables of 1e3..1e7 groups) fed by Poisson
    arrivals (args.rate requests/s in total) of batches with log-uniform
    4,096..1,048,576 rows, for args.seconds: p50/p99 latency (submit ->
    device completion) and rows/s. Request batches come from a pinned pool
    (4 per query) reused by the seeded trace."""
    import torch

    import vecruntime_b200 as vr
    from vecruntime_b200 import aggregate as A
    from vecruntime_b200 import columns as Cc
    from vecruntime_b200 import datagen as G
    from vecruntime_b200 import native as N

    torch.cuda.set_device(device)
    lib = N.lib()
    rng = np.random.default_rng(G.SEEDS["serving"])
    fns = [A.CountAgg(), A.SumLongAgg(1), A.MinMaxAgg(1, True), A.MinMaxAgg(1, False), A.SumDoubleAgg(2),
           A.MinMaxAgg(2, True), A.MinMaxAgg(2, False)]
    srv = vr.AggregateServer(device=device, slots=args.slots, hbm_cap_bytes=120 << 30)
    queries, pool, bufs = [], [], []
    max_rows = 1 << 20
    for q in range(16):
        card = int(round(10 ** rng.uniform(3, 7)))
        domain = rng.integers(-(1 << 62), 1 << 62, size=card, dtype=np.int64)
        batches = []
        for _ in range(4):
            n = int(round(2 ** rng.uniform(12, 20)))
            cols = [Cc.longs(domain[rng.integers(0, card, size=n)], nullable=False),
                    Cc.longs(rng.integers(-10**6, 10**6, size=n, dtype=np.int64), nullable=False),
                    Cc.doubles(rng.standard_normal(n), nullable=False)]
            w = G.Workload(f"q{q}", cols, [0], fns, card, n)
            batches.append(Cc.HostBatch(pinned_copy(w, lib, bufs), n))
        qid = srv.open_query(cols, [0], fns, est_groups=card, max_batch_rows=max_rows)
        queries.append(qid)
        pool.append(batches)
    # the seeded trace: arrival times and (query, batch) picks
    n_req = int(args.rate * args.seconds)
    gaps = rng.exponential(1.0 / args.rate, size=n_req)
    picks = rng.integers(0, 16, size=n_req), rng.integers(0, 4, size=n_req)
    tickets, rows_done = [], 0
    lat = []
    with ClockSampler(device, period_s=0.05) as clocks:
        t0 = time.perf_counter()
        due = t0
        for gap, q, b in zip(gaps, picks[0], picks[1]):
            due += gap
            d = due - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets.append(srv.submit(queries[q], pool[q][b]))
            rows_done += pool[q][b].num_rows
            if len(tickets) > 4096:  # collect finished tickets as the trace goes on
                lat += [srv.wait(t) for t in tickets[:2048]]
                del tickets[:2048]
        lat += [srv.wait(t) for t in tickets]
        wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    for p in bufs:
        lib.vr_host_free(p)
    lat = np.array(lat)
    return {
        "value": rows_done / wall, "unit": "rows/s", "steps": n_req, "ms_per_step": float(np.mean(lat)),
        "config": {"workload": f"serving loop: 16 live queries (1e3..1e7 groups), Poisson arrivals at "
                               f"{args.rate:g} requests/s for {args.seconds:g} s, batches of 4,096..1,048,576 "
                               "rows from pinned host memory", "hbm_cap_gb": 120, "slots": args.slots},
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "max_ms": float(lat.max()), "p99_wait_ms": st.p99_wait_ms, "p99_service_ms": st.p99_service_ms,
        "requests": n_req, "admitted_immediately": st.admitted_immediately, "queued": st.queued,
        "rejected": st.rejected, "max_in_flight": st.max_in_flight, "hbm_peak_gb": st.hbm_peak / 1e9,
        "offered_rows_per_s": rows_done / float(np.sum(gaps)), "gpu_launches": int(st.completed),
        "clocks": clocks.summary(),
    }


# ------------------------------------------------------------------ reference arm
def run_reference(args):
    """The CPU port of the reference's aggregate (oracle/) on the host cores,
    every host thread: bounded samples of the same workload as our arm."""
    from vecruntime_b200 import datagen as G

    threads = host_threads()
    name = "batched" if args.workload in ("all", "batched") else args.workload
    if name == "serving":
        name = "batched"
    per_step = min(args.cpu_seconds, 150.0 / max(1, args.steps + args.warmup))
    rates, desc = [], ""
    if name == "batched":
        ws = G.batched_instances(n=args.instances)
        label = (f"batched uneven instances: {len(ws)} aggregates, {sum(w.rows for w in ws)} rows, rows log-uniform "
                 "2^10..2^22, cardinality log-uniform 1..2^20, int64 key, int64 + float64 values, count/sum/min/max")
        for _ in range(args.warmup):
            cpu_batched(ws[:threads], threads, 1.0)
        for _ in range(args.steps):
            r, desc = cpu_batched(ws, threads, per_step)
            rates.append(r)
        rows, dtype = sum(w.rows for w in ws), "int64/f64"
    else:
        w = make_workload(name, args.rows)
        label, rows, dtype = workload_label(w), w.rows, workload_dtype(w)
        for _ in range(args.warmup):
            cpu_baseline(w, min(w.rows, 1 << 20), threads)
        for _ in range(args.steps):
            r, desc = cpu_sample(w, threads, per_step)
            rates.append(r)
    value = float(np.median(rates))
    return {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": rows / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic (seeded)", "config": {"workload": label, "rows_per_gpu": rows},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port", "port": PORT_NOTE,
                         "sample": "per step: " + desc},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------------ distributed
def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def dist_max(x, world, device):
    """Max of x over the ranks (a CUDA tensor under NCCL, a CPU one under gloo)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    where = torch.device("cuda", device) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([x], dtype=torch.float64, device=where)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_min(x, world, device):
    return -dist_max(-x, world, device)


def weak_scaling(total_ms, steps, rows_per_rank, world, device):
    """(ms per step, whole-job rows/s): every rank aggregates its own replica,
    the job's time is the slowest rank's."""
    ms_per_step = dist_max(total_ms, world, device) / steps
    return ms_per_step, rows_per_rank * world / (ms_per_step * 1e-3)


def line(rec, world, args):
    """The contract's JSON line around a record."""
    out = {"metric": METRIC, "value": rec["value"], "unit": rec["unit"], "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": rec["ms_per_step"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": rec.get("dtype", "int64/f64"),
           "data": "synthetic (seeded; shapes of the workload, no benchmark data reproduced)"}
    cfg = dict(rec["config"])
    cfg["parallelism"] = f"replicas x{world}"
    out["config"] = cfg
    for k, v in rec.items():
        if k not in out and k not in ("config",):
            out[k] = v
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="all",
                    choices=["all", "decimal", "plain", "highcard", "batched", "serving", "parquet"])
    ap.add_argument("--instances", type=int, default=512, help="batched: instances")
    ap.add_argument("--rate", type=float, default=2000.0, help="serving: requests/s")
    ap.add_argument("--seconds", type=float, default=300.0, help="serving: trace length")
    ap.add_argument("--slots", type=int, default=32, help="serving: requests in flight on the device")
    ap.add_argument("--rows", type=int, default=None)
    ap.add_argument("--chunk-rows", type=int, default=8 << 20)
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline sample length")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (default launch shapes)")
    ap.add_argument("--shape", default=None,
                    help="decimal/plain/highcard: a fixed launch shape tier,threads,ctas,tile,slots,warp_agg")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if args.workload == "serving":
        if rank == 0:  # one GPU: serving is about one device's scheduling
            rec = run_serving(args, local)
            print(json.dumps(line(rec, 1, args)), flush=True)
        return

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    check = rank == 0 and world == 1 and not args.no_parity
    if args.workload == "all":
        serving = None
        if world == 1 and not args.no_serving:
            # first, in a fresh process: nothing else has touched host or device memory yet
            serving = run_serving(args, local)
        rec = run_batched(args, rank, world, local, check)
        rec["workloads"] = {}
        for name in ("decimal", "highcard", "plain"):
            rec["workloads"][name] = run_single(args, name, rank, world, local, check)
        rec["workloads"]["parquet"] = run_parquet(args, rank, world, local, check)
        if serving is not None:
            rec["serving"] = serving
    elif args.workload == "batched":
        rec = run_batched(args, rank, world, local, check)
    elif args.workload == "parquet":
        rec = run_parquet(args, rank, world, local, check)
    else:
        rec = run_single(args, args.workload, rank, world, local, check)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line(rec, world, args)), flush=True)


if __name__ == "__main__":
    main()
