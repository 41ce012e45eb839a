"""Benchmark of the compiled-pipeline hot path on B200.

Workload (the configuration the headline metric is quoted on): a batched
uneven panel of 2000 traces × 3001 float32 samples at 2 ms, live lengths
U{1500..3001}, through demean → band-pass 3/6/70/90 Hz with a 50 Hz notch
(2 Hz wide) → AGC 300 ms, src → dst. One step = one apply of the plan to one
panel. Throughput is Msamples/s over the full stored width (rows × cols /
time). Panels rotate through a pool larger than L2 so no step reads inputs
left in cache by the previous one.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 it runs under torchrun, one rank per GPU, each on its own panel
(weak scaling; traces are independent, there is no data-path exchange);
timing is the max over ranks of the device-timed region.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ROWS, COLS, DT = 2000, 3001, 2.0
WORKLOAD = "uneven panel 2000x3001 f32 @2ms, live U{1500..3001}: demean -> bandpass 3/6/70/90 Hz + 50 Hz notch (2 Hz) -> AGC 300 ms"
METRIC = "Msamples/s, band-pass+AGC plan, 2000×3001 fp32; p50/p99 viewer-request latency"


def flow():
    import processseg_b200 as P
    return [P.demeanOp(), P.filterOp(P.bandPass(P.Corners(3, 6, 70, 90)).withNotch(50, 2)),
            P.agcOp(300)]


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def config(world):
    """The workload's config, the same dict in both arms."""
    return {"workload": WORKLOAD, "rows": ROWS, "cols": COLS, "parallelism": f"traces x{world}",
            "l2": "inputs larger than L2: 8 rotating src/dst panel pairs (384 MB)"}


def cpu_baseline(warmup=3, samples=15, min_sample_ms=20.0):
    """The oracle (the C++ restatement of the reference's path) through its
    ProcessPool clone on the same panel, timed by the reference harness's
    method (bench/benchutil.nim:96-126: 3 warm-up applies, then 15 samples of
    doubling batches of at least 20 ms each; median and minimum), on all host
    cores and on one thread. Only the oracle's library is loaded: the rows are
    flattened by the oracle and the ops are plain descriptors."""
    from processseg_b200 import synth
    import processseg_b200 as P
    from oracle import oracle as O
    g = synth.c2()
    live, start = O.rows_flatten(g.status, g.numSamples, g.t0Ms, 0, DT, g.failed, COLS, 0)
    plan = O.OraclePlan(flow(), P.F32, DT, COLS)
    cores = os.cpu_count() or 1
    med, mn, n = plan.bench(g.data, live, start, threads=cores, warm=warmup, samples=samples,
                            min_sample_ms=min_sample_ms)
    med1, mn1, n1 = plan.bench(g.data, live, start, threads=1, warm=warmup, samples=samples,
                               min_sample_ms=min_sample_ms)
    return {"value": ROWS * COLS / med / 1e6, "unit": "Msamples/s", "cores": cores, "kind": "port",
            "sample": f"the full 2000x3001 panel: {warmup} warm-up applies, then {samples} samples of >= "
                      f"{min_sample_ms:g} ms ({n} applies), median {med * 1e3:.2f} ms (min {mn * 1e3:.2f} ms) "
                      f"on {cores} threads of the ProcessPool clone",
            "method": "bench/benchutil.nim:96-126 (3 warm-ups, 15 samples >= 20 ms, median)",
            "samples": samples,
            "one_thread": {"value": ROWS * COLS / med1 / 1e6, "unit": "Msamples/s", "cores": 1,
                           "median_ms": med1 * 1e3, "min_ms": mn1 * 1e3, "applies": n1},
            "all_cores": {"median_ms": med * 1e3, "min_ms": mn * 1e3, "applies": n}}


def trace_errors(got, want, live):
    """Per trace with live samples: max |got - want| over its live samples
    divided by the RMS of ``want`` there (the reference's error measure)."""
    import numpy as np
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    cols = want.shape[1]
    mask = np.arange(cols)[None, :] < np.asarray(live)[:, None]
    n = mask.sum(axis=1)
    keep = n > 0
    rms = np.sqrt(np.where(mask, want * want, 0).sum(axis=1)[keep] / n[keep])
    err = np.where(mask, np.abs(got - want), 0).max(axis=1)[keep]
    ok = rms > 0
    return err[ok] / rms[ok]


def error_summary(e, what):
    import numpy as np
    return {"max": float(np.max(e)), "p99": float(np.percentile(e, 99)), "mean": float(np.mean(e)),
            "traces": int(e.size), "above_1e-5": int(np.sum(e > 1e-5)), "of": what}


def error_report(dst_c2):
    """Each output's max error relative to its trace's RMS, against the FP64
    oracle (and, for parity, against the float32 oracle), computed after the
    timed region: C2 on the bench's own panel (all 2000 traces, the device
    output of the timed steps), C3 on a 32-channel gather and C5 on a
    2000-trace panel of its configuration (same generator, plan and interval)."""
    import numpy as np
    import torch
    import processseg_b200 as P
    from processseg_b200 import synth
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    out = {}
    g = synth.c2()
    live, start = O.rows_flatten(g.status, g.numSamples, g.t0Ms, 0, DT, g.failed, COLS, 0)
    got = dst_c2.cpu().numpy()
    w64 = O.OraclePlan(flow(), P.F64, DT, COLS).apply(g.data.astype(np.float64), live, start, threads=cores)
    w32 = O.OraclePlan(flow(), P.F32, DT, COLS).apply(g.data, live, start, threads=cores)
    out["c2"] = {"vs_fp64": error_summary(trace_errors(got, w64, live), "device float32 vs FP64 oracle"),
                 "vs_f32_oracle": error_summary(trace_errors(got, w32, live), "device vs float32 oracle"),
                 "f32_oracle_vs_fp64": error_summary(trace_errors(w32, w64, live), "float32 oracle vs FP64 oracle")}
    # C5: a 2000-trace panel of the 50000x6001 configuration
    g5 = synth.c5(rows=2000)
    flow5 = [P.demeanOp(), P.filterOp(P.bandPass(P.Corners(2, 5, 120, 150))), P.agcOp(250),
             P.normalizeOp(P.normPercentile, P.perTrace, percentile=99.0)]
    live5, start5 = O.rows_flatten(g5.status, g5.numSamples, g5.t0Ms, 0, 1.0, g5.failed, 6001, 0)
    plan5 = P.initPipeline(flow5).compile(P.float32, 1.0, 6001)
    ws = P.initWorkspace()
    ws.reserve(plan5, rows=2000, cols=6001)
    s5 = torch.from_numpy(g5.data).cuda()
    d5 = torch.empty_like(s5)
    plan5.apply(s5, d5, g5.meta(), ws)
    got5 = d5.cpu().numpy()
    w64 = O.OraclePlan(flow5, P.F64, 1.0, 6001).apply(g5.data.astype(np.float64), live5, start5, threads=cores)
    w32 = O.OraclePlan(flow5, P.F32, 1.0, 6001).apply(g5.data, live5, start5, threads=cores)
    out["c5"] = {"vs_fp64": error_summary(trace_errors(got5, w64, live5), "device float32 vs FP64 oracle"),
                 "vs_f32_oracle": error_summary(trace_errors(got5, w32, live5), "device vs float32 oracle"),
                 "f32_oracle_vs_fp64": error_summary(trace_errors(w32, w64, live5), "float32 oracle vs FP64 oracle"),
                 "sample": "a 2000x6001 panel of the C5 configuration (synth.c5(rows=2000))"}
    # C3: one sweep of a 32-channel gather, correlated to 6 s
    spec = P.linearSweep(8, 80, 12000, 2, P.initSweepTaper(300, 300, P.tpCos2))
    pilot = P.generatePilot(spec, np.float64)
    recs = synth.vibroseis_records(pilot.samples, channels=32, sweeps=1)[0]
    rows3 = recs.shape[0]
    meta3 = P.initChunkMeta(np.full(rows3, P.tsLive, np.int32), np.full(rows3, 10001, np.int32), 2.0)
    cplan = P.initCorrelationPlan(P.float32, pilot, 2.0, 10001, outSamples=3000)
    x3 = torch.from_numpy(np.ascontiguousarray(recs.astype(np.float32))).cuda()
    d3 = torch.zeros(rows3, 3000, device="cuda")
    cplan.correlateInto(x3, d3, meta3)
    got3 = d3.cpu().numpy()
    live3 = np.full(rows3, 10001, np.int32)
    w64, _, _ = O.correlate(pilot.samples, 2.0, 0.0, recs.astype(np.float64), live3, 2.0, 10001, outSamples=3000)
    w32, _, _ = O.correlate(pilot.samples, 2.0, 0.0, recs.astype(np.float32), live3, 2.0, 10001, outSamples=3000)
    l3 = np.full(rows3, 3000)
    out["c3"] = {"vs_fp64": error_summary(trace_errors(got3, w64, l3), "device float32 vs FP64 oracle"),
                 "vs_f32_oracle": error_summary(trace_errors(got3, w32, l3), "device vs float32 oracle"),
                 "vs_fp64_of_peak": float(np.max(np.abs(got3 - w64)) / np.max(np.abs(w64))),
                 "sample": "one sweep of a 32-channel gather (10001 samples, 6 s out)"}
    out["oracle"] = "the C++ restatement of the reference (oracle/psg_oracle.cpp); parity is against it, not the Nim reference, which cannot run here"
    return out


def serving_leg(n_req=150, rates=(2000.0, 5000.0, 10000.0, 20000.0, 40000.0), slots=16):
    """The served viewer load (Poisson arrivals; trace counts log-uniform in
    48..5000; shown windows log-uniform in 200..4000 samples of a 6001-sample
    record, decoded with each plan's margin; three plans) at a sweep of
    offered rates, the request loop against the plain per-call apply (one
    caller, in arrival order, each call waiting for its result) on the same
    request sequence. Two forms: host buffers (copies in and out in every
    request's latency) and device-resident requests (the blocks already in
    HBM). Latency is from each request's scheduled arrival to its completion,
    for both paths (a submit that falls behind the schedule counts its
    delay). ``equal_p99``: at each p99 the
    plain path reached in the sweep, the best throughput each path sustains
    with its p99 within it, and their ratio."""
    import threading
    import numpy as np
    import torch
    import processseg_b200 as P
    from processseg_b200 import synth
    flows = synth.viewer_flows()
    margins = [P.initPipeline(f).requiredMargin(DT) for f in flows]
    base = rates[0]
    reqs = synth.viewer_requests(n_req, rate_hz=base, margins=margins)
    plans = {}
    for r in reqs:
        key = (r.flow, r.cols)
        if key not in plans:
            plans[key] = P.initPipeline(flows[r.flow]).compile(P.float32, DT, r.cols, recordSamples=6001)
    maxn = max(r.rows * r.cols for r in reqs)
    g = synth.shot_gather(5000, 6001, DT, seed=9, workload="c4", live_range=(3000, 6001))
    pool_h = torch.from_numpy(g.data.reshape(-1)[:maxn].copy()).pin_memory()
    outs_h = [torch.empty(maxn, dtype=torch.float32).pin_memory() for _ in range(slots)]
    pool_d = pool_h.cuda()
    outs_d = [torch.empty(maxn, dtype=torch.float32, device="cuda") for _ in range(slots)]
    metas = {}
    jobs = {"host": [], "device": []}
    for i, r in enumerate(reqs):
        key = (r.rows, r.first, r.cols)
        if key not in metas:
            metas[key] = P.initChunkMeta(g.status[:r.rows], g.numSamples[:r.rows], DT, g.t0Ms[:r.rows], r.first)
            metas[key].flat(r.cols)
            metas[key].device(r.cols)
        n = r.rows * r.cols
        plan = plans[(r.flow, r.cols)]
        jobs["host"].append((r.arrival_s, plan, pool_h.numpy()[:n].reshape(r.rows, r.cols),
                             outs_h[i % slots].numpy()[:n].reshape(r.rows, r.cols), metas[key]))
        jobs["device"].append((r.arrival_s, plan, pool_d[:n].view(r.rows, r.cols),
                               outs_d[i % slots][:n].view(r.rows, r.cols), metas[key]))
    total = sum(r.rows * r.cols for r in reqs)
    ws = P.initWorkspace()
    for _, plan, src, dst, meta in jobs["host"]:
        ws.reserve(plan, rows=5000, cols=src.shape[1])

    def spin_until(t0, t):
        while time.perf_counter() - t0 < t:
            pass

    def plain_run(form, scale):
        lat = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for arr, plan, src, dst, meta in jobs[form]:
            spin_until(t0, arr * scale)
            plan.apply(src, dst, meta, ws)
            if form == "device":
                torch.cuda.current_stream().synchronize()
            lat.append(time.perf_counter() - t0 - arr * scale)
        span = time.perf_counter() - t0
        return {"p50_ms": float(np.percentile(lat, 50)) * 1e3, "p99_ms": float(np.percentile(lat, 99)) * 1e3,
                "msamples_per_s": total / span / 1e6}

    def served_run(srv, form, scale):
        srv.stats(reset=True)
        c0 = srv.counters()
        tickets = []
        lat = [0.0] * len(jobs[form])
        arrivals = [arr * scale for arr, *_ in jobs[form]]

        def waiter():
            # latency from each request's scheduled arrival (as the plain
            # path's) to the time the loop saw it finish
            k = 0
            while k < len(jobs[form]):
                if k < len(tickets):
                    lat[k] = srv.wait(tickets[k], 60000) - t0 - arrivals[k]  # the loop's completion time
                    k += 1
                else:
                    time.sleep(0.0001)

        th = threading.Thread(target=waiter)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        th.start()
        for (arr, plan, src, dst, meta), when in zip(jobs[form], arrivals):
            spin_until(t0, when)
            tickets.append(srv.submit(plan, src, dst, meta))
        th.join()
        span = time.perf_counter() - t0
        st, c1 = srv.stats(), srv.counters()
        return {"p50_ms": float(np.percentile(lat, 50)) * 1e3, "p99_ms": float(np.percentile(lat, 99)) * 1e3,
                "msamples_per_s": total / span / 1e6, "requests_per_batch": st["requests_per_launch"],
                "batches_beside_running": c1["overlapped"] - c0["overlapped"]}

    out = {"workload": "served viewer load: Poisson arrivals, traces log-U[48,5000], windows log-U[200,4000] of 6001 "
                       "+ plan margins, 3 plans",
           "requests": n_req, "forms": {}}
    with P.Server(arena_bytes=3 << 30) as srv:
        for form in ("host", "device"):
            for _, plan, src, dst, meta in jobs[form][:3]:  # warm-up (and the tuner, where a plan has one)
                plan.apply(src, dst, meta, ws)
                srv.wait(srv.submit(plan, src, dst, meta), 60000)
            torch.cuda.synchronize()
            sweep = []
            for rate in rates:
                scale = base / rate
                sweep.append({"offered_rps": rate, "plain": plain_run(form, scale),
                              "served": served_run(srv, form, scale)})
            # at each p99 the plain path reached: the best throughput each
            # path sustains with its p99 within it
            eq = []
            for bound in sorted({s["plain"]["p99_ms"] for s in sweep}):
                best = lambda path: max([s[path]["msamples_per_s"] for s in sweep if s[path]["p99_ms"] <= bound]
                                        or [0.0])
                sp, ss = best("plain"), best("served")
                eq.append({"p99_bound_ms": bound, "plain_msamples_per_s": sp, "served_msamples_per_s": ss,
                           "ratio": ss / sp if sp > 0 else None})
            out["forms"][form] = {"sweep": sweep, "equal_p99": eq}
    return out


def multi_gpu_legs(args, world, rank, dist):
    """The two splits beside the weak-scaled panels, run on every rank (their
    collectives are the path's exchanges), timed with events on each rank
    after W warm-up steps, the max over ranks: ``sharded_panel``, a per-panel
    p99 normalization over a panel split by rows (the C2 chain with the
    normalization before the AGC; ``applySharded``: two all-reduces of the
    partial statistics per step; each rank 2000 × 3001 rows, weak scaling),
    and ``c3_by_channel``, the 4-sweep 240-channel gather split by channel
    (each rank correlates and stacks every sweep of its channels, one
    all-gather assembles the 240 × 3000 stack; strong scaling)."""
    import numpy as np
    import torch
    import processseg_b200 as P
    from processseg_b200 import shard, synth

    def timed(fn):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        if dist:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    out = {}
    flow = [P.demeanOp(), P.filterOp(P.bandPass(P.Corners(3, 6, 70, 90)).withNotch(50, 2)),
            P.normalizeOp(P.normPercentile, P.perPanel, percentile=99.0), P.agcOp(300)]
    plan = P.initPipeline(flow).compile(P.float32, DT, COLS)
    g = synth.c2(seed=40 + rank)
    meta = g.meta()
    ws = P.initWorkspace()
    ws.reserve(plan, rows=ROWS, cols=COLS)
    src = torch.from_numpy(g.data).cuda()
    dst = torch.empty_like(src)
    ms = timed(lambda: shard.applySharded(plan, src, dst, meta, ws))
    out["sharded_panel"] = {
        "workload": f"{world} x 2000 x 3001 f32 panel split by rows: demean -> band-pass + notch -> per-panel p99 "
                    "-> AGC 300 ms (applySharded, two all-reduces per step)",
        "ms_per_step": ms, "msamples_per_s": world * ROWS * COLS / (ms * 1e-3) / 1e6, "scaling": "weak"}
    del src, dst

    spec = P.linearSweep(8, 80, 12000, 2, P.initSweepTaper(300, 300, P.tpCos2))
    pilot = P.generatePilot(spec, np.float64)
    recs = synth.vibroseis_records(pilot.samples, channels=240, sweeps=4)
    sweeps, ch, ns = recs.shape
    block = recs.reshape(sweeps * ch, ns)
    rmap = (np.arange(sweeps * ch) % ch).astype(np.int32)
    cmeta = P.initChunkMeta(np.full(sweeps * ch, P.tsLive, np.int32), np.full(sweeps * ch, ns, np.int32), 2.0)
    cplan = P.initCorrelationPlan(P.float32, pilot, 2.0, ns, outSamples=3000)
    idx, _, _ = shard.channelShard(rmap, ch, world, rank)
    x = torch.from_numpy(block).cuda()  # every record in HBM; each rank reads its channels' records
    split = shard.ChannelSplit(cplan, cmeta, rmap, ch)
    ms = timed(lambda: split.run(x))
    out["c3_by_channel"] = {
        "workload": "4 sweeps x 240 channels x 10001 f32, nfft 16200, 6 s out, split by channel, stack all-gathered",
        "ms_per_gather": ms, "records_this_rank": int(idx.size),
        "msamples_per_s": sweeps * ch * ns / (ms * 1e-3) / 1e6, "scaling": "strong"}
    return out


def launch_of(plan, rows):
    """The trace-kernel launch shape the tuner chose for a call of ``rows``
    rows (the first one untuned), with its per-shape times (µs per launch)."""
    tun = plan.tuning()
    if not tun["parts"]:
        return None
    part = tun["parts"][0]
    rec = next((t for t in tun["tuned"] if t["part"] == part["part"] and t["class"] == int(rows).bit_length()), None)
    pick = part["pinned"] if part["pinned"] >= 0 else (rec["choice"] if rec else 0)
    return {"chosen": part["shapes"][pick], "pinned": part["pinned"] >= 0,
            "tuner_us_per_shape": rec["us"] if rec else None, "shapes": part["shapes"]}


def workloads_leg(peak, which=("c1", "c3", "c5", "segy", "spectrum")):
    """The other configurations, device-resident, each timed with CUDA events
    after a warm-up: C1 (48×2001, demean → band-pass 4-8-60-80 → AGC 500 ms),
    C3 (4 sweeps × 240 channels × 10001 samples correlated with a 12 s
    8–80 Hz pilot to 6 s, stacked), C5 (50000×6001 at 1 ms, demean →
    band-pass 2/5/120/150 → AGC 250 ms → per-trace p99 normalization).
    HBM fraction: algorithmic bytes (each input sample read once, each output
    written once) over the time, against the measured copy bandwidth."""
    import numpy as np
    import torch
    import processseg_b200 as P
    from processseg_b200 import synth

    def timed(fn, steps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps * 1e-3

    out = {}
    if "c1" in which:
        g = synth.c1()
        meta = g.meta()
        plan = P.initPipeline([P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 60, 80)), P.agcOp(500)]).compile(P.float32, 2.0, 2001)
        ws = P.initWorkspace()
        ws.reserve(plan, rows=48, cols=2001)
        src = torch.from_numpy(g.data).cuda()
        dst = torch.empty_like(src)
        t = timed(lambda: plan.apply(src, dst, meta, ws), 200)
        # the same apply captured once and replayed: one host call per panel
        gr = plan.capture(src, dst, meta, ws)
        tg = timed(gr.replay, 200)
        del gr
        out["c1"] = {"workload": "48x2001 f32 @2ms: demean -> bandpass 4-8-60-80 -> AGC 500 ms", "us_per_panel": t * 1e6,
                     "msamples_per_s": 48 * 2001 / t / 1e6, "hbm_frac": 2 * 48 * 2001 * 4 / t / 1e9 / peak,
                     "us_per_panel_graph_replay": tg * 1e6, "launch": launch_of(plan, 48)}

    if "c3" in which:
        spec = P.linearSweep(8, 80, 12000, 2, P.initSweepTaper(300, 300, P.tpCos2))
        pilot = P.generatePilot(spec, np.float64)
        recs = synth.vibroseis_records(pilot.samples, channels=240, sweeps=4)
        sweeps, ch, ns = recs.shape
        cplan = P.initCorrelationPlan(P.float32, pilot, 2.0, ns, outSamples=3000)
        stack = P.initRecordStack(ch, 3000, 2.0)
        # the gather's sweeps as one block of records, each stacked on its channel
        x = torch.from_numpy(recs.reshape(sweeps * ch, ns)).cuda()
        rmap = (torch.arange(sweeps * ch, dtype=torch.int32, device="cuda") % ch).contiguous()
        cmeta = P.initChunkMeta(np.full(sweeps * ch, P.tsLive, np.int32), np.full(sweeps * ch, ns, np.int32), 2.0)
        d = torch.empty(sweeps * ch, 3000, device="cuda")
        so = torch.empty(ch, 3000, device="cuda")

        def c3():
            stack.clear()
            cplan.correlateInto(x, d, cmeta, stack=stack, rowMap=rmap)
            stack.stackInto(so)
        t = timed(c3, 20)
        inb = sweeps * ch * ns * 4
        outb = sweeps * ch * 3000 * 4 + ch * 3000 * 4
        out["c3"] = {"workload": "4 sweeps x 240 channels x 10001 f32 @2ms, 12 s 8-80 Hz pilot, nfft 16200, 6 s out, vertical stack (one call of 960 records, rowMap to the channels)",
                     "ms_per_gather": t * 1e3, "msamples_per_s": sweeps * ch * ns / t / 1e6,
                     "hbm_frac": (inb + outb) / t / 1e9 / peak}

    if "c5" in which:
        g = synth.c5()
        meta = g.meta()
        flow = [P.demeanOp(), P.filterOp(P.bandPass(P.Corners(2, 5, 120, 150))), P.agcOp(250),
                P.normalizeOp(P.normPercentile, P.perTrace, percentile=99.0)]
        plan = P.initPipeline(flow).compile(P.float32, 1.0, 6001)
        ws = P.initWorkspace()
        ws.reserve(plan, rows=50000, cols=6001)
        src = torch.from_numpy(g.data).cuda()
        dst = torch.empty_like(src)
        t = timed(lambda: plan.apply(src, dst, meta, ws), 3)
        out["c5"] = {"workload": "50000x6001 f32 @1ms (1.2 GB), live U{4000..6001}: demean -> bandpass 2/5/120/150 -> AGC 250 ms -> per-trace p99",
                     "ms_per_panel": t * 1e3, "msamples_per_s": 50000 * 6001 / t / 1e6,
                     "hbm_frac": 2 * 50000 * 6001 * 4 / t / 1e9 / peak, "launch": launch_of(plan, 50000)}
        del src, dst
        torch.cuda.empty_cache()

    if "segy" in which:
        # SEG-Y decode: 20000 records of 3001 IBM-float samples (random words)
        # to a float32 block, and a viewer's spectrum panel (501-sample windows
        # of the C2 panel, power-averaged)
        from processseg_b200 import _abi as A
        rows, n = 20000, 3001
        st = torch.cuda.current_stream().cuda_stream
        blk = torch.empty(rows, n, dtype=torch.float32, device="cuda")
        out["segy"] = {"workload": "20000 SEG-Y records x 3001 samples (random words) -> f32 block"}
        for fmt, name, sz in ((1, "ibm", 4), (3, "int16", 2), (5, "ieee32", 4)):
            rec = torch.randint(0, 256, (rows, 240 + sz * n), dtype=torch.uint8, device="cuda")
            t = timed(lambda: A.check(A.lib().psg_segy_decode(rec.data_ptr(), rows, 240 + sz * n, 240, n, fmt, 0, A.F32,
                                                              blk.data_ptr(), n, st)), 10)
            nbytes = rec.numel() + blk.numel() * 4
            out["segy"][name] = {"us_per_block": t * 1e6, "gb_per_s": nbytes / t / 1e9, "hbm_frac": nbytes / t / 1e9 / peak}
            del rec
        del blk
    if "spectrum" in which:
        from processseg_b200 import _abi as A
        st = torch.cuda.current_stream().cuda_stream
        g = synth.c2()
        meta = g.meta()
        sp = P.initSpectrumPlan(P.float32, 2.0, 501)
        ws = P.initWorkspace()
        src = torch.from_numpy(g.data).cuda()
        amp = [0.0] * sp.bins
        live, _ = meta.device(3001)
        avg = torch.empty(sp.bins, dtype=torch.float64, device="cuda")
        t = timed(lambda: A.check(A.lib().psg_spectrum_average(sp.h, ws.h, src.data_ptr(), 2000, 3001, live.data_ptr(), 2.0,
                                                               500, 0, 1999, avg.data_ptr(), None, st)), 20)
        out["spectrum"] = {"workload": "spectrum panel: 2000 traces x 501-sample windows from sample 500, nfft 512",
                           "us_per_panel": t * 1e6, "msamples_per_s": 2000 * 501 / t / 1e6}
        del src
        torch.cuda.empty_cache()
    return out


def run_reference(args):
    """The reference arm: the reference's CPU implementation of the path,
    here the oracle port (the reference is Nim, which cannot build here),
    through its ProcessPool clone on all host cores, rank 0 only. It loads
    no part of the CUDA library."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    b = cpu_baseline()
    line = {"impl": "reference", "metric": METRIC, "value": b["value"], "unit": "Msamples/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config(world),
            "cpu_baseline": b,
            "e2e": {"value": b["value"], "unit": "Msamples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch
    import processseg_b200 as P
    from processseg_b200 import synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    g = synth.c2(seed=2 + rank)
    meta = g.meta()
    plan = P.initPipeline(flow()).compile(P.float32, DT, COLS)
    if args.trace_shape is not None:
        plan.pinTrace(0, args.trace_shape)  # a launch shape fixed for a profile (no tuning launches)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=ROWS, cols=COLS)
    # A pool of distinct panels larger than L2 (126 MB): 8 × (24 + 24) MB.
    pool = 8
    srcs = [torch.from_numpy(g.data).cuda() for _ in range(pool)]
    for i, s in enumerate(srcs):
        s.mul_(1.0 + 1e-3 * i)
    dsts = [torch.empty_like(srcs[0]) for _ in range(pool)]
    stream = torch.cuda.current_stream()

    def step(i):
        plan.apply(srcs[i % pool], dsts[i % pool], meta, ws)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    # The K steps run back to back between two events on the launching
    # stream (one trace_kernel launch each): the average launch duration is
    # the region's time over K. Events between the steps would add their own
    # gaps to the region.
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            step(i)
        e1.record(stream)
        torch.cuda.synchronize()
        time.sleep(0.25)  # at least one clock sample after a short region
    ms_total = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms_total], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
        dist.barrier()
    ms_step = ms_total / args.steps
    kernel_ms = [ms_step]
    value = world * ROWS * COLS / (ms_step * 1e-3) / 1e6

    # e2e: the public API with host buffers (pinned): every step copies its
    # panel in, applies the plan and copies the result out. Streamed: the
    # steps are queued back to back (apply(..., wait=False), two result
    # buffers in turn) and the clock stops when the last result has landed;
    # one at a time (each call waits) is reported beside it.
    hsrc = torch.from_numpy(g.data).pin_memory()
    hdst = [torch.empty_like(hsrc).pin_memory() for _ in range(2)]
    hs, hd = hsrc.numpy(), [h.numpy() for h in hdst]
    for _ in range(2):
        plan.apply(hs, hd[0], meta, ws)
    e2e_steps = max(3, min(args.steps, 20))

    def e2e_run(wait):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(e2e_steps):
            plan.apply(hs, hd[i & 1], meta, ws, wait=wait)
        ws.synchronize()
        sec = (time.perf_counter() - t0) / e2e_steps
        if dist:
            t = torch.tensor([sec], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            sec = float(t.item())
        return world * ROWS * COLS / sec / 1e6

    e2e_run(False)  # the first streamed run sizes the pinned staging
    e2e = e2e_run(False)
    e2e_sync = e2e_run(True)
    multi = None if args.no_multi else multi_gpu_legs(args, world, rank, dist)

    if rank == 0:
        peak, peak_kind = peaks()
        kavg = statistics.mean(kernel_ms)
        alg_bytes = 2 * ROWS * COLS * 4
        achieved = alg_bytes / (kavg * 1e-3) / 1e9
        traffic, insts = None, None
        try:
            with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
                tj = json.load(f)
            traffic = tj.get("trace_kernel_c2_bytes")
            insts = tj.get("trace_kernel_c2_warp_instructions")
        except Exception:
            pass
        line = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": config(world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "trace_kernel<RPlan<1944>> (float32 demean/filter/AGC), the tuned launch shape",
                         "algorithmic_bytes": alg_bytes},
            # the bound that sets the time: warp-instruction issue, with the
            # launch's instruction count from its ncu capture over the measured
            # kernel time, against 4 schedulers x SMs x the clock seen
            "issue": None if not insts else {
                "achieved": insts / (kavg * 1e-3) / 1e12, "unit": "T warp-instructions/s",
                "peak": 4 * torch.cuda.get_device_properties(0).multi_processor_count
                * (clk.summary().get("sm_mhz") or 1965.0) * 1e6 / 1e12,
                "warp_instructions_per_launch": insts},
            "e2e": {"value": e2e, "unit": "Msamples/s",
                    "h2d_bytes_per_step": ROWS * COLS * 4 + ROWS * 12,
                    "d2h_bytes_per_step": ROWS * COLS * 4,
                    "mode": "streamed: steps queued back to back, the clock stops at the last result",
                    "one_at_a_time": e2e_sync},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "launch": launch_of(plan, ROWS),
        }
        if multi:
            line["multi_gpu"] = multi
        if line["issue"]:
            line["issue"]["frac"] = line["issue"]["achieved"] / line["issue"]["peak"]
        # the one-GPU legs: the served load, the other configurations and the
        # CPU baseline run at N = 1 only (under torchrun the other ranks wait
        # for rank 0 at the final barrier)
        if world == 1 and not args.no_serving:
            line["serving"] = serving_leg()
        if world == 1 and not args.no_workloads:
            line["workloads"] = workloads_leg(peak, args.workloads.split(","))
        if world == 1 and not args.no_errors:
            line["error_vs_fp64"] = error_report(dsts[0])
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the served-load leg")
    ap.add_argument("--no-multi", action="store_true", help="skip the split-panel and by-channel legs")
    ap.add_argument("--workloads", default="c1,c3,c5,segy,spectrum",
                    help="the other configurations to time (comma-separated: c1, c3, c5, segy, spectrum)")
    ap.add_argument("--trace-shape", type=int, default=None,
                    help="run the headline panel with this trace-kernel launch shape (PipelinePlan.tuning lists them)")
    ap.add_argument("--no-workloads", action="store_true", help="skip the C1/C3/C5 legs")
    ap.add_argument("--no-errors", action="store_true", help="skip the error report against the oracle")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
