"""Benchmark of the GPU grouped aggregate (one JSON line on stdout, rank 0).

Default workload: the low-cardinality decimal report aggregate (60M rows,
two dictionary keys -> 6 groups, four DECIMAL(12,2) columns; sum(qty),
sum(price), sum(price*(1-disc)), sum(price*(1-disc)*(1+tax)) in exact
decimal, avg(qty), avg(disc), count(*)) -- the TPC-H Q1 shape the reference
quotes its headline numbers on. A step is one pass of the aggregate over the
whole input: table clear + aggregate kernel, inputs resident in HBM (2.4 GB,
larger than the 126 MB L2; a 1 GiB write on the stream precedes each step's
start event, so L2 is cold and the device is busy while the host submits the
step). `e2e` is the same work through the public C ABI
with pinned host buffers: H2D of the step's inputs (chunked, copies
overlapping kernels) + the emitted groups copied back into pinned output
buffers allocated once and reused every step.

Other workloads (--workload plain|highcard|batched|serving) print the same
line for their own shape. --impl reference times the CPU port of the
reference's aggregate (oracle/) on the host cores instead.

Multi-GPU (torchrun): every rank aggregates its own replica of the workload
(weak scaling, no collective on the data path); time = max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "rows/s & HBM GB/s (% of peak), batched vs plain on 1 B200; serving p50/p99 ms"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# DRAM bytes (read + write) of one aggregate launch, from ncu captures
# (dram__bytes_read.sum + dram__bytes_write.sum). The decimal report's traffic
# is its input plus a fixed flush, so an 8M-row capture scales with rows
# (profiles/aggregate_decimal_report_8M.md). A hash table's traffic follows
# its group count, not the rows, so those figures hold only at the row count
# they were captured at (profiles/aggregate_plain_1M.md,
# profiles/aggregate_high_cardinality_100M.md).
TRAFFIC_PER_ROW = {"decimal": (320.097792e6 + 4.176128e6) / 8_000_000}
TRAFFIC_AT_ROWS = {"plain": (1 << 20, 25.473792e6 + 6.912e3), "highcard": (100_000_000, 7.72e9 + 2.57e9)}
FLUSH_BYTES = 1 << 30  # written on the step's stream before each step's start event


def launch_traffic(w):
    """(GB per launch, how it was obtained) or (None, why not)."""
    src = "ncu dram__bytes_read.sum + dram__bytes_write.sum"
    if w.name in TRAFFIC_PER_ROW:
        return TRAFFIC_PER_ROW[w.name] * w.rows / 1e9, f"GB per launch ({src}, 8M-row capture scaled by rows)"
    at = TRAFFIC_AT_ROWS.get(w.name)
    if at is not None and at[0] == w.rows:
        return at[1] / 1e9, f"GB per launch ({src}, capture of this workload at {w.rows} rows)"
    return None, "no capture at this row count (table traffic follows the group count, not the rows)"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
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
    dst = np.ctypeslib.as_array((C.c_uint8 * a.nbytes).from_address(p.value)).view(a.dtype).reshape(a.shape)
    dst[...] = a
    bufs.append(p)
    return dst


def pinned_copy(w, lib):
    """The workload's columns copied into pinned host memory (vr_host_alloc)."""
    from vecruntime_b200 import columns as Cc

    bufs = []

    def pin_one(a):
        return pin(a, lib, bufs)

    cols = []
    for c in w.columns:
        n = Cc.Col(c.lane, pin_one(c.data), pin_one(c.validity), c.precision, c.scale, c.dict_size, c.nullable)
        if c.lane == 4:
            n._n = c._n
        cols.append(n)
    return cols, bufs


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


# ------------------------------------------------------------------ our arm
def run_ours(args, rank, world, device):
    import torch

    import vecruntime_b200 as vr
    from vecruntime_b200 import native as N

    torch.cuda.set_device(device)
    lib = N.lib()
    w = make_workload(args.workload, args.rows)
    log(f"[rank {rank}] workload {w.name}: {w.rows} rows, est groups {w.est_groups}")
    db, tensors = device_batch(w, device)
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=w.rows,
                              device=device, flags=N.VR_SPEC_TRACE)
    stream = torch.cuda.ExternalStream(agg.stream(), device=torch.device("cuda", device))
    from vecruntime_b200 import datagen as G

    in_bytes = G.input_bytes(w)
    # before each step's start event, a 1 GiB write on the same stream: it
    # evicts the inputs from L2 (126 MB) when they would fit there, and it
    # keeps the device busy while the host submits the step, so the events
    # time the step's device work rather than the host's submission latency
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=device)
    # warm-up
    for _ in range(args.warmup):
        agg.reset()
        agg.consume(db)
        agg.sync()
    groups = agg.num_groups()
    st0 = agg.stats()
    kms0 = st0.total_kernel_ms
    launches0 = st0.kernel_launches
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
    kernel_ms = (st1.total_kernel_ms - kms0) / args.steps
    launches = st1.kernel_launches - launches0
    ms_per_step, value = weak_scaling(sum(step_ms), args.steps, w.rows, world, device)

    out_types = agg.output_types
    out_bytes = groups * output_row_bytes(out_types)
    alg_bytes = in_bytes + out_bytes
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    traffic, traffic_unit = launch_traffic(w)
    agg.close()
    del tensors, flush

    # end to end through the public API: pinned host buffers, H2D + D2H in the step
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, w, lib, device, out_types)
        if e2e is not None:
            e2e["value"] = dist_min(e2e["value"], world, device) * world

    result = {
        "metric": METRIC,
        "value": value,
        "unit": "rows/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": workload_dtype(w),
        "data": "synthetic (seeded; shapes of the workload, no benchmark data reproduced)",
        "config": {"workload": workload_label(w), "rows_per_gpu": w.rows, "groups": groups,
                   "batch": "one device-resident batch per step",
                   "l2": "L2 flushed before each step (%d MB written on the stream outside the timed events; "
                         "inputs %.3f GB)" % (FLUSH_BYTES >> 20, in_bytes / 1e9),
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "traffic_unit": traffic_unit,
                     "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": kernel_ms},
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    return result, w


def workload_dtype(w):
    return "int64 (exact decimal128 sums)" if w.name == "decimal" else "int64/f64"


def workload_label(w):
    n = f"{w.rows // 1_000_000}M rows" if w.rows % 1_000_000 == 0 else f"{w.rows:,} rows"
    return {"decimal": f"low-cardinality decimal report: {n}, 2 dictionary keys (3x2 -> 6 groups), "
                       "4 DECIMAL(12,2) columns, exact decimal(38,6) sums",
            "plain": f"plain grouped aggregation: {n}, int64 key over 1,000 values, 5% nulls",
            "highcard": f"high-cardinality composite key: {n}, Zipf(1.1) int64 x int32[16], 1% null keys"
            }.get(w.name, w.name)


def run_e2e(args, w, lib, device, out_types):
    import torch

    import vecruntime_b200 as vr
    from vecruntime_b200 import columns as Cc
    from vecruntime_b200 import datagen as G

    cols, bufs = pinned_copy(w, lib)
    chunk = min(w.rows, args.chunk_rows)
    chunk -= chunk % 128 if chunk > 128 else 0
    agg = vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups, max_batch_rows=chunk,
                              device=device)
    stream = torch.cuda.ExternalStream(agg.stream(), device=torch.device("cuda", device))

    def batches():
        out = []
        for lo in range(0, w.rows, chunk):
            hi = min(w.rows, lo + chunk)
            out.append(Cc.HostBatch([G.slice_col(c, lo, hi) for c in cols], hi - lo))
        return out

    bl = batches()
    groups = 0
    in_bytes = G.input_bytes(w)
    d2h = 0
    times = []
    # the groups come back into pinned buffers allocated once (the first
    # warm-up step sizes them), as a caller with a pinned output pool would
    out_pinned, out_bufs = None, []
    for it in range(args.warmup + args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        agg.reset()
        for hb in bl:
            agg.consume(hb)
        groups = agg.num_groups()
        out = agg.emit(out=out_pinned) if out_pinned is not None else agg.emit()
        b.record(stream)
        torch.cuda.synchronize(device)
        if it >= args.warmup:
            times.append(a.elapsed_time(b))
        d2h = sum(d.nbytes + v.nbytes for d, v in out)
        if out_pinned is None:
            out_pinned = [(pin(d, lib, out_bufs), pin(v, lib, out_bufs)) for d, v in out]
    agg.close()
    for p in bufs + out_bufs:
        lib.vr_host_free(p)
    ms = float(np.mean(times))
    return {"value": w.rows / (ms * 1e-3), "unit": "rows/s", "h2d_bytes_per_step": in_bytes,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms, "chunk_rows": chunk}


# ------------------------------------------------------------------ batched (C4)
def batched_choice():
    """The one launch configuration every instance of a batched launch shares:
    the hash tier's two-CTAs-per-SM shape (1024-row tiles, 256 consumer
    threads, a 256-slot shared hot-key cache in front of each instance's HBM
    table). Measured on this workload (persistent launch, CUDA graph):
    1024-row tiles x 256 slots 27.3 ms, 512 x 512 27.4, 512 x 256 28.2,
    256 x 256 29.1, 1024 x 128 29.1, 256 x 1024 29.6 (every change of
    instance flushes the whole cache, so the larger caches that pay for one
    long batch do not pay here)."""
    from vecruntime_b200 import native as N

    t = N.TuneChoice()
    t.tier, t.threads, t.tile_rows, t.smem_slots = 1, 256, 1024, 256
    return t


def run_batched(args, device):
    """512 uneven instances (rows log-uniform 2^10..2^22, cardinality
    log-uniform 1..2^20): one persistent launch replayed from a CUDA graph,
    against one launch per instance. A step resets every table and
    aggregates every instance's device-resident batch."""
    import torch

    import vecruntime_b200 as vr
    from vecruntime_b200 import columns as Cc
    from vecruntime_b200 import datagen as G
    from vecruntime_b200 import native as N

    torch.cuda.set_device(device)
    ws = G.batched_instances(n=args.instances)
    log(f"[batched] {len(ws)} instances, {sum(w.rows for w in ws)} rows")
    aggs, dbs, keep = [], [], []
    for w in ws:
        aggs.append(vr.GpuHashAggregate(w.columns, w.keys, w.functions, est_groups=w.est_groups,
                                        max_batch_rows=w.rows, device=device, tune=batched_choice()))
        db, t = Cc.to_device(w.batch(), device)
        dbs.append(db)
        keep.append(t)
    stream = torch.cuda.Stream(device=device)
    rows = sum(w.rows for w in ws)
    in_bytes = sum(G.input_bytes(w) for w in ws)

    def timed(b):
        for _ in range(args.warmup):
            b.run(stream.cuda_stream)
        ms = []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.run(stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.mean(ms))

    torch.cuda.synchronize(device)
    with ClockSampler(device) as clocks:
        persistent = vr.GpuBatchedAggregate(aggs, dbs, mode=N.VR_BATCHED_PERSISTENT, use_graph=True)
        ms_p = timed(persistent)
        persistent.close()
        plain = vr.GpuBatchedAggregate(aggs, dbs, mode=N.VR_BATCHED_PLAIN)
        ms_l = timed(plain)
        plain.close()
    launches = 3  # zero, aggregate, status gather
    peak, peak_kind = measured_peaks()
    for a in aggs:
        a.close()
    return {
        "metric": METRIC, "value": rows / (ms_p * 1e-3), "unit": "rows/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_p, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int64/f64", "data": "synthetic (seeded; shapes of the workload, no benchmark data reproduced)",
        "config": {"workload": f"batched uneven instances: {len(ws)} aggregates, {rows} rows, rows log-uniform "
                               "2^10..2^22, cardinality log-uniform 1..2^20, int64 key, int64 + float64 values, "
                               "count/sum/min/max", "mode": "one persistent launch replayed from a CUDA graph",
                   "l2": "inputs larger than L2 (%.2f GB)" % (in_bytes / 1e9)},
        "roofline": {"bound": "hbm", "achieved": in_bytes / (ms_p * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": in_bytes / (ms_p * 1e-3) / 1e9 / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_launch": in_bytes, "kernel_ms": ms_p},
        "one_launch_per_instance": {"value": rows / (ms_l * 1e-3), "unit": "rows/s", "ms_per_step": ms_l},
        "speedup_vs_one_launch_per_instance": ms_l / ms_p,
        "gpu_launches": launches * args.steps,
        "clocks": clocks.summary(),
    }


# ------------------------------------------------------------------ serving (C5)
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
            pcols, pb = pinned_copy(w, lib)
            bufs += pb
            batches.append(Cc.HostBatch(pcols, n))
        qid = srv.open_query(cols, [0], fns, est_groups=card, max_batch_rows=max_rows)
        queries.append(qid)
        pool.append(batches)
    # the seeded trace: arrival times and (query, batch) picks
    n_req = int(args.rate * args.seconds)
    gaps = rng.exponential(1.0 / args.rate, size=n_req)
    picks = [(int(rng.integers(0, 16)), int(rng.integers(0, 4))) for _ in range(n_req)]
    tickets, rows_done = [], 0
    with ClockSampler(device) as clocks:
        t0 = time.perf_counter()
        due = t0
        for gap, (q, b) in zip(gaps, picks):
            due += gap
            d = due - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets.append(srv.submit(queries[q], pool[q][b]))
            rows_done += pool[q][b].num_rows
        lat = [srv.wait(t) for t in tickets]
        wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    for p in bufs:
        lib.vr_host_free(p)
    lat = np.array(lat)
    return {
        "metric": METRIC, "value": rows_done / wall, "unit": "rows/s", "n_gpus": 1, "steps": n_req,
        "warmup": 0, "ms_per_step": float(np.mean(lat)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic (seeded trace; no benchmark data reproduced)",
        "config": {"workload": f"serving loop: 16 live queries (1e3..1e7 groups), Poisson arrivals at "
                               f"{args.rate:g} requests/s for {args.seconds:g} s, batches of 4,096..1,048,576 "
                               "rows from pinned host memory", "hbm_cap_gb": 120},
        "serving": {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                    "max_ms": float(lat.max()), "p99_wait_ms": st.p99_wait_ms, "p99_service_ms": st.p99_service_ms,
                    "requests": n_req, "slots": args.slots, "admitted_immediately": st.admitted_immediately,
                    "queued": st.queued, "rejected": st.rejected, "hbm_peak_gb": st.hbm_peak / 1e9,
                    "offered_rows_per_s": rows_done / float(np.sum(gaps))},
        "gpu_launches": int(st.completed),
        "clocks": clocks.summary(),
    }


# ------------------------------------------------------------------ reference arm
def run_reference(args):
    """The CPU port of the reference's aggregate (oracle/) on the host cores:
    bounded samples of the same workload, every host thread."""
    threads = os.cpu_count() or 1
    w = make_workload(args.workload, args.rows)
    for _ in range(args.warmup):
        cpu_baseline(w, min(w.rows, 1 << 20), threads)
    # each step about args.cpu_seconds of work, the whole run about 3 minutes at most
    per_step = min(args.cpu_seconds, 180.0 / max(1, args.steps))
    rates = []
    desc = ""
    for _ in range(args.steps):
        r, desc = cpu_sample(w, threads, per_step)
        rates.append(r)
    value = float(np.median(rates))
    return {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": w.rows / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": workload_dtype(w),
        "data": "synthetic (seeded)", "config": {"workload": workload_label(w), "rows_per_gpu": w.rows},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="decimal", choices=["decimal", "plain", "highcard", "batched", "serving"])
    ap.add_argument("--instances", type=int, default=512, help="batched: instances")
    ap.add_argument("--rate", type=float, default=2000.0, help="serving: requests/s")
    ap.add_argument("--seconds", type=float, default=10.0, help="serving: trace length")
    ap.add_argument("--slots", type=int, default=32, help="serving: requests in flight on the device")
    ap.add_argument("--rows", type=int, default=None)
    ap.add_argument("--chunk-rows", type=int, default=8 << 20)
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline sample length")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if args.workload in ("batched", "serving"):
        if rank == 0:  # one GPU: these shapes are about one device's scheduling
            fn = run_batched if args.workload == "batched" else run_serving
            print(json.dumps(fn(args, local)), flush=True)
        return

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    result, w = run_ours(args, rank, world, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, desc = cpu_sample(w, threads, args.cpu_seconds)
        result["cpu_baseline"] = {"value": rate, "unit": "rows/s", "cores": threads, "kind": "port", "sample": desc}
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


if __name__ == "__main__":
    main()
