"""The trace kernel's launch shapes and the tuner that picks among them: for
the three compile-time transform lengths (m = 1944: 2000 × 3001-style panels;
m = 1125: 48 × 2001; m = 3375 with a per-trace p99 normalization: 6001
samples at 1 ms), every shape, pinned, gives the same bits as the first, and
those bits are within the parity bar (1e-5 of each trace's RMS) of the
oracle's float32 apply (filter/apply.nim:81-84 with the reference's FFT
stages, fft/plan.nim:120-160). The tuner's first apply at a row count
records a time for every shape and a choice, leaves the result unchanged,
and tunes in-place applies too."""
import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import synth
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]

C2_FLOW = [P.demeanOp(), P.filterOp(P.bandPass(P.Corners(3, 6, 70, 90)).withNotch(50, 2)), P.agcOp(300)]
C1_FLOW = [P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 60, 80)), P.agcOp(500)]
C5_FLOW = [P.demeanOp(), P.filterOp(P.bandPass(P.Corners(2, 5, 120, 150))), P.agcOp(250),
           P.normalizeOp(P.normPercentile, P.perTrace, percentile=99.0)]


def case(name):
    if name == "m1944":
        return C2_FLOW, synth.c2(rows=300), 2.0
    if name == "m1125":
        return C1_FLOW, synth.c1(), 2.0
    g = synth.shot_gather(150, 6001, 1.0, 9, np.float32, live_range=(4000, 6001), workload="c5")
    return C5_FLOW, g, 1.0


def rel_errs(got, want, live):
    mask = np.arange(want.shape[1])[None, :] < live[:, None]
    w, g = want.astype(np.float64), got.astype(np.float64)
    n = np.maximum(mask.sum(1), 1)
    rms = np.sqrt(np.where(mask, w * w, 0).sum(1) / n)
    d = np.where(mask, np.abs(g - w), 0).max(1)
    return np.where(rms > 0, d / np.where(rms > 0, rms, 1), 0)


def run(plan, ws, src, meta, in_place=False):
    if in_place:
        dst = src.clone()
        plan.apply(None, dst, meta, ws)
    else:
        dst = torch.full_like(src, float("nan"))
        plan.apply(src, dst, meta, ws)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


@pytest.mark.parametrize("name,m", [("m1944", 1944), ("m1125", 1125), ("m3375", 3375)])
def test_every_launch_shape_gives_the_same_bits(name, m):
    flow, g, dt = case(name)
    rows, cols = g.data.shape
    plan = P.initPipeline(flow).compile(P.float32, dt, cols)
    n = plan.traceShapes(0)
    assert n >= 2, "the transform length has trace-kernel builds"
    info = plan.tuning()
    shapes = info["parts"][0]["shapes"]
    assert len(shapes) == n and all(s["m"] == m for s in shapes)
    assert {s["grid"] for s in shapes} == {"persistent", "per_row"}
    meta = g.meta()
    ws = P.initWorkspace()
    ws.reserve(plan, rows=rows, cols=cols)
    src = torch.from_numpy(g.data).cuda()
    outs = []
    for k in range(n):
        plan.pinTrace(0, k)
        outs.append(run(plan, ws, src, meta))
    for k in range(1, n):
        assert np.array_equal(outs[k], outs[0], equal_nan=True), (k, shapes[k])
    live, start = meta.flat(cols)
    want = O.OraclePlan(flow, P.F32, dt, cols).apply(g.data, live, start)
    assert rel_errs(outs[0], want, live).max() <= 1e-5
    # the tuner: unpinned, the first apply at this row count times every shape
    plan.pinTrace(0, -1)
    tuned = run(plan, ws, src, meta)
    assert np.array_equal(tuned, outs[0], equal_nan=True)
    rec = [t for t in plan.tuning()["tuned"] if t["part"] == 0]
    assert len(rec) == 1 and rec[0]["rows"] == rows and len(rec[0]["us"]) == n
    assert 0 <= rec[0]["choice"] < n and all(u > 0 for u in rec[0]["us"])
    assert rec[0]["us"][rec[0]["choice"]] == min(rec[0]["us"])
    # a second apply at the same class keeps the choice (no new record)
    assert np.array_equal(run(plan, ws, src, meta), outs[0], equal_nan=True)
    assert len(plan.tuning()["tuned"]) == 1


def test_tuning_an_in_place_apply_leaves_the_result_as_one_apply():
    flow, g, dt = case("m1944")
    rows, cols = g.data.shape
    meta = g.meta()
    src = torch.from_numpy(g.data).cuda()
    ref_plan = P.initPipeline(flow).compile(P.float32, dt, cols)
    ref_plan.pinTrace(0, 0)
    ws = P.initWorkspace()
    ws.reserve(ref_plan, rows=rows, cols=cols)
    want = run(ref_plan, ws, src, meta)
    plan = P.initPipeline(flow).compile(P.float32, dt, cols)
    got = run(plan, ws, src, meta, in_place=True)
    assert len(plan.tuning()["tuned"]) == 1
    assert np.array_equal(got, want, equal_nan=True)
    # a different row-count class tunes again
    half = torch.from_numpy(np.ascontiguousarray(g.data[:70])).cuda()
    m70 = P.initChunkMeta(g.status[:70], g.numSamples[:70], dt, np.zeros(70))
    out70 = run(plan, ws, half, m70)
    assert len(plan.tuning()["tuned"]) == 2
    ref70 = run(ref_plan, ws, half, m70)
    assert np.array_equal(out70, ref70, equal_nan=True)


def test_pin_rejects_bad_shapes():
    flow, g, dt = case("m1125")
    plan = P.initPipeline(flow).compile(P.float32, dt, g.data.shape[1])
    n = plan.traceShapes(0)
    with pytest.raises(ValueError):
        plan.pinTrace(0, n)
    with pytest.raises(ValueError):
        plan.pinTrace(0, -2)
    with pytest.raises(ValueError):
        plan.pinTrace(3, 0)
    # a float64 plan runs on the general kernel: no shapes
    p64 = P.initPipeline(flow).compile(P.float64, dt, g.data.shape[1])
    assert p64.traceShapes(0) == 0
    assert p64.tuning() == {"parts": [], "tuned": []}
