"""Parity of the device pipeline (libpsgcuda.so through its C ABI) with the
CPU oracle, on seeded synthetic panels. The bar (the parity tolerance): each
output trace within 1e-5 of its RMS of the oracle's float32 apply, and
within 1e-12 of its RMS for float64 plans. Non-live rows and samples past a
row's live length are copied bit for bit."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import synth
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]

C1_FLOW = [P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 60, 80)), P.agcOp(500)]
C2_FLOW = [P.demeanOp(), P.filterOp(P.bandPass(P.Corners(3, 6, 70, 90)).withNotch(50, 2)),
           P.agcOp(300)]


def rel_rms_err(got, want, live):
    """max over live traces of max|got − want| / rms(want) on the live part."""
    worst = 0.0
    for r in range(want.shape[0]):
        n = int(live[r])
        if n == 0:
            continue
        w = want[r, :n].astype(np.float64)
        g = got[r, :n].astype(np.float64)
        rms = math.sqrt(float(np.mean(w * w)))
        if rms == 0:
            assert np.all(g == 0)
            continue
        worst = max(worst, float(np.max(np.abs(g - w))) / rms)
    return worst


def assert_parity(got, flow, data, meta, dtype, dtMs, samples=None, record=0, tol=None):
    """The device output against the oracle of the same precision: within
    ``tol`` (1e-5 float32, 1e-12 float64) of each trace's RMS. Where the
    oracle's own float32 output is further than that from the float64
    oracle (float32 rounding of a large offset under a low-cut, say), the
    device must be no further from the float64 oracle than twice the
    oracle's own float32 error."""
    tol = tol if tol is not None else (1e-5 if dtype == P.F32 else 1e-12)
    live = meta.flat(data.shape[1])[0]
    want = run_oracle(flow, data, meta, dtype, dtMs, samples, record)
    e = rel_rms_err(got, want, live)
    if e <= tol or dtype == P.F64:
        assert e <= tol, e
        return e
    want64 = run_oracle(flow, data.astype(np.float64), meta, P.F64, dtMs, samples, record)
    own = rel_rms_err(want, want64, live)
    mine = rel_rms_err(got, want64, live)
    assert mine <= max(tol, 2 * own), (e, mine, own)
    return mine


def run_gpu(flow, data, meta, dtype, dtMs, samples=None, record=0, inplace=False, host=False):
    plan = P.initPipeline(flow).compile(dtype, dtMs, samples or data.shape[1], record)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=data.shape[0], cols=data.shape[1])
    if host:
        dst = np.zeros_like(data)
        plan.apply(data, dst, meta, ws)
        return dst
    src = torch.from_numpy(data).cuda()
    if inplace:
        plan.apply(src, meta, ws)
        torch.cuda.synchronize()
        return src.cpu().numpy()
    dst = torch.zeros_like(src)
    plan.apply(src, dst, meta, ws)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


def run_oracle(flow, data, meta, dtype, dtMs, samples=None, record=0):
    plan = O.OraclePlan(flow, dtype, dtMs, samples or data.shape[1], record)
    live, start = meta.flat(data.shape[1], 0)
    return plan.apply(data, live, start)


def test_c1_plain_plan_matches_oracle():
    g = synth.c1()
    meta = g.meta()
    got = run_gpu(C1_FLOW, g.data, meta, P.float32, 2.0)
    want = run_oracle(C1_FLOW, g.data, meta, P.F32, 2.0)
    live = meta.flat(2001)[0]
    assert rel_rms_err(got, want, live) <= 1e-5
    # and against the float64 oracle
    want64 = run_oracle(C1_FLOW, g.data.astype(np.float64), meta, P.F64, 2.0)
    assert rel_rms_err(got, want64, live) <= 1e-5


def test_c2_uneven_panel_src_dst_and_in_place():
    g = synth.c2(rows=300)
    g.status[[5, 77]] = P.tsDead
    g.status[[9]] = P.tsAux
    g.failed = np.array([13, 200], np.int64)
    meta = g.meta()
    want = run_oracle(C2_FLOW, g.data, meta, P.F32, 2.0)
    live = meta.flat(3001)[0]
    for inplace in (False, True):
        got = run_gpu(C2_FLOW, g.data, meta, P.float32, 2.0, inplace=inplace)
        assert rel_rms_err(got, want, live) <= 1e-5
        for r in range(g.data.shape[0]):
            n = live[r]
            assert np.array_equal(got[r, n:], g.data[r, n:]), r  # dead rows and padding
    host = run_gpu(C2_FLOW, g.data, meta, P.float32, 2.0, host=True)
    dev = run_gpu(C2_FLOW, g.data, meta, P.float32, 2.0)
    assert np.array_equal(host, dev)
    # every op alone: in place gives the bits of src -> dst
    for flow in ([P.demeanOp()], C2_FLOW[1:2], C2_FLOW[2:]):
        a = run_gpu(flow, g.data, meta, P.float32, 2.0)
        b = run_gpu(flow, g.data, meta, P.float32, 2.0, inplace=True)
        assert np.array_equal(a, b)
        assert_parity(a, flow, g.data, meta, P.F32, 2.0)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_host_buffers_pinned_pageable_and_in_place_agree(dtype):
    """The host-memory apply reads pinned buffers over the bus from the
    kernel and stages pageable ones through chunk copies: the same bits
    either way, src → dst and in place, as the device-resident apply."""
    g = synth.c2(rows=700, dtype=dtype)
    g.status[[3, 400]] = P.tsDead
    meta = g.meta()
    T = P.float32 if dtype == np.float32 else P.float64
    dev = run_gpu(C2_FLOW, g.data, meta, T, 2.0)
    plan = P.initPipeline(C2_FLOW).compile(T, 2.0, 3001)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=700, cols=3001)
    pageable = np.zeros_like(g.data)
    plan.apply(g.data, pageable, meta, ws)
    hs = torch.from_numpy(g.data.copy()).pin_memory()
    hd = torch.zeros_like(hs).pin_memory()
    plan.apply(hs.numpy(), hd.numpy(), meta, ws)
    plan.apply(hs.numpy(), meta, ws)  # in place, pinned
    assert np.array_equal(pageable, dev)
    assert np.array_equal(hd.numpy(), dev)
    assert np.array_equal(hs.numpy(), dev)


def test_float64_plan_matches_oracle_to_1e12():
    g = synth.c2(rows=64, dtype=np.float64)
    meta = g.meta()
    got = run_gpu(C2_FLOW, g.data, meta, P.float64, 2.0)
    want = run_oracle(C2_FLOW, g.data, meta, P.F64, 2.0)
    assert rel_rms_err(got, want, meta.flat(3001)[0]) <= 1e-12


FLOWS = {
    "basic": [P.detrendOp(), P.scaleOp(2.5), P.gainDbOp(-3), P.clipOp(-1.5, 1.2), P.polarityOp(),
              P.demeanOp()],
    "highcut_reflect": [P.filterOp(P.highCut(60, 80))],
    "zero_dc": [P.filterOp(P.highCut(60, 80).withZeroDc())],
    "trend_none": [P.filterOp(P.lowCut(2, 4), P.trNone)],
    "trend_mean": [P.filterOp(P.bandPass(P.Corners(4, 8, 60, 80)), P.trMean)],
    "butter": [P.filterOp(P.butterBandPass(5, 100, 24)), P.gainCurveOp(P.powerGain(2))],
    "agc_meanabs": [P.agcOp(200, P.agcMeanAbs, target=2.0)],
    "norm_max": [P.normalizeOp(P.normMax, target=3.0)],
    "norm_rms": [P.bandPassOp(P.Corners(4, 8, 60, 80)), P.normalizeOp(P.normRms)],
    "norm_pct": [P.normalizeOp(P.normPercentile, percentile=99.0)],
    "norm_pct_low": [P.normalizeOp(P.normPercentile, percentile=37.5)],
    "panel_rms": [P.agcOp(200), P.normalizeOp(P.normRms, P.perPanel, target=3.0), P.demeanOp()],
    "panel_max": [P.normalizeOp(P.normMax, P.perPanel), P.agcOp(100)],
    "panel_pct": [P.demeanOp(), P.normalizeOp(P.normPercentile, P.perPanel, percentile=99.0)],
    "curves": [P.gainCurveOp(P.exponentialGain(3)),
               P.gainCurveOp(P.knotGain([P.GainKnot(0, 0), P.GainKnot(900, 6), P.GainKnot(3000, 20)]))],
}


@pytest.mark.parametrize("name", sorted(FLOWS))
@pytest.mark.parametrize("dtype", [P.F32, P.F64])
def test_op_flows_match_oracle(name, dtype):
    npd = np.float32 if dtype == P.F32 else np.float64
    g = synth.shot_gather(40, 1201, 2.0, seed=11, dtype=npd, live_range=(2, 1201), sine_hz=30.0,
                          workload="flows")
    g.status[[3]] = P.tsDead
    g.t0Ms = np.linspace(-10, 40, 40)
    g.numSamples[7] = 1
    meta = g.meta()
    flow = FLOWS[name]
    got = run_gpu(flow, g.data, meta, dtype, 2.0)
    tol = 1e-5 if dtype == P.F32 else 1e-12
    if name.startswith("panel_pct"):
        tol = max(tol, 1e-9)  # the histogram bin position is exact; sums reorder in f64
    assert_parity(got, flow, g.data, meta, dtype, 2.0, tol=tol)


def test_gain_curve_zoom_window_matches_whole_record_plan():
    # tests/tpipeline.nim:333-361: a window compiled for its width with the
    # record's length gives the bits of the whole-record plan.
    ns, first, cols = 6001, 3700, 1101
    g = synth.shot_gather(12, ns, 2.0, seed=5, workload="zoom")
    win = np.ascontiguousarray(g.data[:, first:first + cols])
    meta = P.initChunkMeta(g.status, g.numSamples, 2.0, g.t0Ms, first)
    for curve in (P.powerGain(2), P.exponentialGain(3),
                  P.knotGain([P.GainKnot(0, 0), P.GainKnot(9000, 20)])):
        flow = [P.gainCurveOp(curve)]
        a = run_gpu(flow, win, meta, P.float32, 2.0, samples=ns)
        b = run_gpu(flow, win, meta, P.float32, 2.0, samples=cols, record=ns)
        assert np.array_equal(a, b)
        want = run_oracle(flow, win, meta, P.F32, 2.0, samples=cols, record=ns)
        assert rel_rms_err(b, want, meta.flat(cols)[0]) <= 1e-6


def test_nan_stays_in_its_row():
    g = synth.shot_gather(6, 500, 2.0, seed=2, workload="nan")
    g.data[2, 250] = np.nan
    meta = g.meta()
    got = run_gpu(C1_FLOW, g.data, meta, P.float32, 2.0)
    assert np.isnan(got[2]).any()
    for r in (0, 1, 3, 4, 5):
        assert np.all(np.isfinite(got[r]))


def test_errors_change_nothing():
    # tests/tpipeline.nim:227-249
    g = synth.shot_gather(20, 500, 2.0, seed=3, workload="err")
    meta = g.meta()
    src = torch.from_numpy(g.data).cuda()
    orig = src.clone()
    flow = P.initPipeline([P.demeanOp(), P.agcOp(100)])
    ws = P.initWorkspace()
    narrow = flow.compile(P.float32, 2.0, 400)
    ws.reserve(narrow)
    with pytest.raises(ValueError):
        narrow.apply(src, meta, ws)
    other = flow.compile(P.float32, 4.0, 500)
    with pytest.raises(ValueError):
        other.apply(src, meta, ws)
    ok = flow.compile(P.float32, 2.0, 500)
    with pytest.raises(ValueError):
        ok.apply(src, torch.zeros(19, 500, device="cuda"), meta, ws)
    with pytest.raises(ValueError):
        ok.apply(src, torch.zeros(20, 499, device="cuda"), meta, ws)
    with pytest.raises(ValueError):
        ok.apply(src[:, :250], src[:, 250:], meta, ws)  # not contiguous
    with pytest.raises(ValueError):
        ok.apply(src.double(), meta, ws)
    buf = torch.zeros(24, 500, device="cuda")
    with pytest.raises(ValueError, match="overlap"):
        P.initPipeline([P.scaleOp(2)]).compile(P.float32, 2.0, 500).apply(buf[0:20], buf[2:22], meta, ws)
    torch.cuda.synchronize()
    assert torch.equal(src, orig)
    panel = P.initPipeline([P.normalizeOp(P.normRms, P.perPanel)]).compile(P.float32, 2.0, 500)
    with pytest.raises(AssertionError):
        panel.apply(src, meta, P.initWorkspace())
    with pytest.raises(ValueError, match=r"^op 1 \(opFilter\): "):
        P.initPipeline([P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 200, 260))]).compile(P.float32, 2.0, 500)


def test_empty_pipeline_copies():
    g = synth.shot_gather(10, 100, 2.0, seed=1, workload="empty")
    meta = g.meta()
    got = run_gpu([], g.data, meta, P.float32, 2.0)
    assert np.array_equal(got, g.data)
    same = run_gpu([], g.data, meta, P.float32, 2.0, inplace=True)
    assert np.array_equal(same, g.data)


def test_panel_factor_matches_oracle():
    g = synth.shot_gather(50, 800, 2.0, seed=8, workload="pf", live_range=(100, 800))
    meta = g.meta()
    flow = P.initPipeline([P.agcOp(50), P.normalizeOp(P.normPercentile, P.perPanel, target=2)])
    plan = flow.compile(P.float32, 2.0, 800)
    ws = P.initWorkspace()
    ws.reserve(plan)
    b = torch.from_numpy(g.data).cuda()
    f = plan.panelFactorOf(b, meta, 1, ws)
    st = O.panel_stats(g.data, meta.flat(800)[0], 99.0)
    assert abs(f - 2 / st["clip"]) <= 1e-12 * abs(f)


@pytest.mark.parametrize("window_ms", [100, 300, 500, 700])
@pytest.mark.parametrize("dtype", [P.F32, P.F64])
def test_agc_window_edges_match_oracle(window_ms, dtype):
    """AGC at live lengths around the half window h, the whole window
    w = 2h + 1 and its multiples (head, whole-trace, whole-window and tail
    forms of gain/gain.nim:433-461), in both modes, with a row whose second
    half is 120 dB quieter than its first (tests/tgain.nim:187-212)."""
    h = int(round(window_ms / 2.0 / 2))
    w = 2 * h + 1
    cols = 1201
    lens = sorted({n for n in (1, 2, 3, h - 1, h, h + 1, 2 * h - 1, 2 * h, w, w + 1, 2 * w - 1, 2 * w,
                               2 * w + 1, 3 * w + h, 4 * w - 1, cols - 1, cols) if 1 <= n <= cols})
    npd = np.float32 if dtype == P.F32 else np.float64
    g = synth.shot_gather(len(lens) + 1, cols, 2.0, seed=21, dtype=npd, workload="agc_edges")
    g.numSamples[:len(lens)] = lens
    g.numSamples[-1] = cols
    g.data[-1, cols // 2:] *= 1e-6
    for r, n in enumerate(g.numSamples):
        g.data[r, n:] = 0
    meta = g.meta()
    for mode in (P.agcRms, P.agcMeanAbs):
        flow = [P.agcOp(window_ms, mode)]
        got = run_gpu(flow, g.data, meta, dtype, 2.0)
        assert_parity(got, flow, g.data, meta, dtype, 2.0)


@pytest.mark.parametrize("flow", [C2_FLOW, C2_FLOW + [P.normalizeOp(P.normPercentile, percentile=99.0)],
                                  [P.bandPassOp(P.Corners(4, 8, 60, 80)), P.normalizeOp(P.normRms)],
                                  [P.filterOp(P.butterBandPass(5, 100, 24)), P.gainCurveOp(P.powerGain(2))]],
                         ids=["dfa", "dfan", "fn", "fg"])
def test_recipe_kernels_and_step_switch_match_oracle(flow, monkeypatch):
    """The fixed-sequence kernels (demean fused into the filter's pack) and
    the generic step switch (PSG_RECIPES=0, read at compile time) both match
    the oracle on the same uneven panel of an odd number of rows, with a dead
    row and a row holding a NaN that stays in its row."""
    g = synth.c2(rows=161)
    g.status[[4]] = P.tsDead
    g.data[17, 40] = np.nan
    meta = g.meta()
    outs = [run_gpu(flow, g.data, meta, P.float32, 2.0)]
    monkeypatch.setenv("PSG_RECIPES", "0")
    outs.append(run_gpu(flow, g.data, meta, P.float32, 2.0))
    ok = np.ones(g.data.shape[0], bool)
    ok[17] = False
    live = meta.flat(3001)[0]
    for got in outs:
        assert np.isnan(got[17, :live[17]]).any()
        assert np.all(np.isfinite(got[ok]))
        assert_parity(got[ok], flow, g.data[ok], P.initChunkMeta(g.status[ok], g.numSamples[ok], 2.0,
                                                                  g.t0Ms[ok], 0), P.F32, 2.0)


def long_gather(rows, cols, dtMs, dtype, seed):
    g = synth.shot_gather(rows, cols, dtMs, seed, dtype, live_range=(cols // 2, cols), sine_hz=50.0,
                          workload="long")
    g.status[[2]] = P.tsDead
    return g


@pytest.mark.parametrize("dtype,cols,dtMs,flow", [
    (P.F64, 16384, 0.5, [P.demeanOp(), P.bandPassOp(P.Corners(8, 12, 40, 50)), P.agcOp(200)]),
    (P.F32, 30000, 1.0, [P.demeanOp(), P.bandPassOp(P.Corners(2, 5, 120, 150)), P.agcOp(250),
                         P.normalizeOp(P.normPercentile, percentile=99.0)]),
    (P.F64, 20000, 1.0, [P.agcOp(500), P.scaleOp(2)]),
], ids=["f64-16384-filter-agc", "f32-30000-filter-agc-p99", "f64-20000-agc"])
def test_long_traces_match_oracle(dtype, cols, dtMs, flow):
    """Traces whose FFT (or AGC) work areas do not fit beside the row in
    shared memory run with those areas in global memory; the same bar
    against the oracle, on ragged live lengths with a dead row."""
    npdt = np.float32 if dtype == P.F32 else np.float64
    g = long_gather(7, cols, dtMs, npdt, seed=11)
    meta = g.meta()
    got = run_gpu(flow, g.data, meta, dtype, dtMs)
    assert_parity(got, flow, g.data, meta, dtype, dtMs)
    assert np.array_equal(got[2], g.data[2])


@pytest.mark.parametrize("dtype", [P.F32, P.F64])
def test_global_work_layout_matches_shared_bit_for_bit(dtype, monkeypatch):
    """PSG_WIDE=1 (read at compile time) puts any plan's work areas in global
    memory: the step switch then gives the same bits as with them in shared
    memory."""
    npdt = np.float32 if dtype == P.F32 else np.float64
    g = synth.c2(rows=97, dtype=npdt)
    g.data[9, 100] = np.inf
    meta = g.meta()
    flow = C2_FLOW + [P.normalizeOp(P.normRms)]
    monkeypatch.setenv("PSG_RECIPES", "0")
    shared = run_gpu(flow, g.data, meta, dtype, 2.0)
    monkeypatch.setenv("PSG_WIDE", "1")
    wide = run_gpu(flow, g.data, meta, dtype, 2.0)
    wide_host = run_gpu(flow, g.data, meta, dtype, 2.0, host=True)
    np.testing.assert_array_equal(wide, shared)
    np.testing.assert_array_equal(wide_host, shared)


def test_long_trace_workspace_and_limits():
    """A plan with long traces needs its workspace reserved for it (the
    reference's AssertionDefect otherwise); a trace too long for one CTA's
    shared memory is refused at compile time."""
    flow = P.initPipeline([P.bandPassOp(P.Corners(8, 12, 40, 50))])
    long_plan = flow.compile(P.float64, 0.5, 16384)
    short_plan = flow.compile(P.float64, 0.5, 2000)
    ws = P.initWorkspace()
    ws.reserve(short_plan, rows=4, cols=2000)
    src = torch.zeros(4, 16384, dtype=torch.float64, device="cuda")
    meta = P.liveMeta(4, 16384, 0.5)
    with pytest.raises(AssertionError):
        long_plan.apply(src, meta, ws)
    ws.reserve(long_plan, rows=4, cols=16384)
    long_plan.apply(src, meta, ws)
    torch.cuda.synchronize()
    assert ws.bytes >= long_plan.workspaceSize(4, 16384) > short_plan.workspaceSize(4, 16384)
    with pytest.raises(ValueError, match="shared memory"):
        flow.compile(P.float64, 0.5, 40000)


def test_process_pool_apply_matches_plan_apply():
    """newProcessPool / ProcessPool.apply (pool.nim:145-302): the same rows
    as PipelinePlan.apply, on device tensors and host arrays, blocking."""
    g = synth.c2(rows=64)
    meta = g.meta()
    plan = P.initPipeline(C2_FLOW).compile(P.float32, 2.0, 3001)
    want = run_gpu(C2_FLOW, g.data, meta, P.F32, 2.0)
    pool = P.newProcessPool(8)
    assert pool.workers == 8
    dst = np.zeros_like(g.data)
    pool.apply(plan, g.data, dst, meta)
    assert np.array_equal(dst, want)
    x = torch.from_numpy(g.data).cuda()
    pool.apply(plan, x, meta)
    assert np.array_equal(x.cpu().numpy(), want)
    pool.ping()
    with pytest.raises(ValueError):
        P.newProcessPool(0)


def test_scale_rows_matches_reference_rules():
    """scaleRows / scaleRowsInto (calibrate.nim:562-612): each row that is
    not failed times T(factor) up to its live length whatever its status,
    NaN factors fill the live part with NaN, the rest copied; an infinite
    factor is refused before any sample changes."""
    rng = np.random.default_rng(5)
    for npdt in (np.float32, np.float64):
        x = rng.standard_normal((7, 300)).astype(npdt)
        status = np.array([P.tsLive, P.tsDead, P.tsAux, P.tsLive, P.tsLive, P.tsUnknown, P.tsLive], np.int32)
        ns = np.array([300, 200, 100, 0, 300, 150, 299], np.int32)
        meta = P.initChunkMeta(status, ns, 2.0, failed=[4])
        f = np.array([2.0, -1.5, 0.5, 3.0, 7.0, np.nan, 1e-3])
        want = x.copy()
        for r in range(7):
            if r == 4:
                continue
            n = min(ns[r], 300)
            want[r, :n] = x[r, :n] * npdt(f[r])
        dst = np.zeros_like(x)
        P.scaleRowsInto(x, dst, meta, f)
        assert np.array_equal(dst, want, equal_nan=True)
        t = torch.from_numpy(x.copy()).cuda()
        P.scaleRows(t, meta, f)
        assert np.array_equal(t.cpu().numpy(), want, equal_nan=True)
        bad = f.copy()
        bad[2] = np.inf
        t = torch.from_numpy(x.copy()).cuda()
        with pytest.raises(ValueError):
            P.scaleRows(t, meta, bad)
        assert np.array_equal(t.cpu().numpy(), x)
        with pytest.raises(ValueError):
            P.scaleRows(t, meta, f[:3])
    with pytest.raises(ValueError):  # 1e39 overflows float32
        P.scaleRows(torch.ones(1, 4, device="cuda"), P.liveMeta(1, 4, 2.0), [1e39])


@pytest.mark.parametrize("flow", [C2_FLOW, C2_FLOW + [P.normalizeOp(P.normRms, P.perPanel)],
                                  [P.muteTopOp(P.timeMute(300), taperMs=20)] + C2_FLOW],
                         ids=["chunked", "whole-block", "keys"])
def test_async_host_applies_overlap_and_match(flow):
    """apply(..., wait=False) on host arrays: six panels queued back to back
    (their copies overlap), interleaved with a waiting call, each equal to
    the waiting apply of the same panel."""
    plan = P.initPipeline(flow).compile(P.float32, 2.0, 3001)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=300, cols=3001)
    gs = [synch for synch in (synth.c2(seed=40 + i, rows=300) for i in range(6))]
    want = []
    for g in gs:
        d = np.zeros_like(g.data)
        plan.apply(g.data, d, g.meta(), ws)
        want.append(d)
    srcs = [torch.from_numpy(g.data).pin_memory().numpy() for g in gs]
    dsts = [torch.zeros(300, 3001).pin_memory().numpy() for _ in gs]
    metas = [g.meta() for g in gs]
    for i in range(6):
        plan.apply(srcs[i], dsts[i], metas[i], ws, wait=False)
        if i == 2:
            extra = np.zeros_like(gs[0].data)
            plan.apply(gs[0].data, extra, metas[0], ws)
            assert np.array_equal(extra, want[0])
    ws.synchronize()
    for i in range(6):
        assert np.array_equal(dsts[i], want[i]), i


def test_async_host_applies_across_layouts(monkeypatch):
    """Queued host applies whose staging is laid out differently from the
    call before (another width, a whole block, a plan with its work areas in
    global memory, which keeps to one lane) give the waiting results."""
    monkeypatch.setenv("PSG_WIDE", "1")
    wide = P.initPipeline(C2_FLOW).compile(P.float32, 2.0, 3001)
    monkeypatch.delenv("PSG_WIDE")
    plans = [P.initPipeline(C2_FLOW).compile(P.float32, 2.0, 3001), wide,
             P.initPipeline(C2_FLOW).compile(P.float32, 2.0, 1500)]
    ws = P.initWorkspace()
    cases = []
    for i, (plan, rows, cols) in enumerate([(0, 900, 3001), (2, 1200, 1500), (1, 900, 3001), (0, 40, 3001),
                                            (2, 1500, 1500), (0, 900, 3001)]):
        g = synth.shot_gather(rows, cols, 2.0, 70 + i, np.float32, live_range=(cols // 2, cols), sine_hz=50.0,
                              workload="layouts")
        ws.reserve(plans[plan], rows=rows, cols=cols)
        want = np.zeros_like(g.data)
        plans[plan].apply(g.data, want, g.meta(), ws)
        src = torch.from_numpy(g.data).pin_memory()
        dst = torch.zeros_like(src).pin_memory()
        cases.append((plans[plan], src, dst, g.meta(), want))
    for plan, src, dst, meta, _ in cases:
        plan.apply(src.numpy(), dst.numpy(), meta, ws, wait=False)
    ws.synchronize()
    for i, (_, _, dst, _, want) in enumerate(cases):
        assert np.array_equal(dst.numpy(), want), i


def test_check_apply_refuses_what_apply_refuses():
    """checkApply (pipeline.nim:619-641) raises the ValueError apply would,
    for device tensors and host arrays alike, and touches no sample."""
    plan = P.initPipeline(C1_FLOW).compile(P.float32, 2.0, 2001)
    meta = P.liveMeta(8, 2001, 2.0)
    x = torch.randn(16, 2001, device="cuda")
    src, dst = x[:8], torch.empty(8, 2001, device="cuda")
    before = x.clone()
    plan.checkApply(src, dst, meta)
    plan.checkApply(None, dst, meta)
    plan.checkApply(dst, dst, meta)  # the same block: in place
    bad = [
        (lambda: plan.checkApply(x[:8], x[4:12], meta), "overlap"),
        (lambda: plan.checkApply(src, dst, P.liveMeta(8, 2001, 4.0)), "dtMs"),
        (lambda: plan.checkApply(None, torch.empty(8, 2002, device="cuda"), meta), "columns"),
        (lambda: plan.checkApply(None, dst, P.liveMeta(9, 2001, 2.0)), "rows"),
        (lambda: plan.checkApply(None, dst.double(), meta), "float"),
        (lambda: plan.checkApply(torch.empty(8, 100, device="cuda"), dst, meta), "×"),
    ]
    ws = P.initWorkspace()
    ws.reserve(plan, rows=8, cols=2001)
    for f, what in bad:
        with pytest.raises(ValueError, match=what):
            f()
    # apply refuses the same overlap before any sample changes
    with pytest.raises(ValueError, match="overlap"):
        plan.apply(x[:8], x[4:12], meta, ws)
    torch.cuda.synchronize()
    assert torch.equal(x, before)
    h = np.zeros((8, 2001), np.float32)
    plan.checkApply(h.copy(), h, meta)
    with pytest.raises(ValueError, match="dtMs"):
        plan.checkApply(None, h, P.liveMeta(8, 2001, 1.0))
