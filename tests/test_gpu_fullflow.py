"""The reference's full flow (tests/tpipeline.nim:33-49, every op kind:
demean, FFT band-pass, LMO top mute, per-panel RMS normalization, AGC, a
knot gain curve, an IIR high-cut, a per-panel percentile normalization,
clip, scale, gain, polarity, detrend, a bottom mute, a per-trace max
normalization) compiled into one plan of three parts on the device, against
the same ops applied one by one as one-op plans on the device
(apply_equals_ops_one_by_one: float64 within 1e-13 of the largest output
sample, float32 1e-6) and against the oracle's apply of the flow. src → dst
leaves src untouched and copies dead and failed rows as they are."""
import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A
from processseg_b200 import synth
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


def full_flow():
    return [P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 60, 80)),
            P.muteTopOp(P.lmoMute(2500, padMs=-20), taperMs=20),
            P.normalizeOp(P.normRms, P.perPanel, target=2.0), P.agcOp(300),
            P.gainCurveOp(P.knotGain([P.GainKnot(0, 0), P.GainKnot(3000, 12)])),
            P.iirOp(P.butterHighCut(90, 24)),
            P.normalizeOp(P.normPercentile, P.perPanel, percentile=95.0),
            P.clipOp(-3, 3), P.scaleOp(0.5), P.gainDbOp(6), P.polarityOp(), P.detrendOp(),
            P.muteBottomOp(P.timeMute(3500), taperMs=40), P.normalizeOp(P.normMax)]


@pytest.mark.parametrize("T,npdt,tol", [(P.float64, np.float64, 1e-13), (P.float32, np.float32, 1e-6)])
def test_full_flow_equals_ops_one_by_one(T, npdt, tol):
    g = synth.shot_gather(100, 2001, 2.0, 11, npdt, sine_hz=50.0, workload="fullflow")
    g.status[[3, 40, 65]] = P.tsDead
    failed = [7, 64, 90]
    meta = P.initChunkMeta(g.status, g.numSamples, 2.0, g.t0Ms, 0, failed, g.offsets)
    flow = full_flow()
    plan = P.initPipeline(flow).compile(T, 2.0, 2001)
    assert plan.partCount == 3
    ws = P.initWorkspace()
    ws.reserve(plan, rows=100, cols=2001)
    src = torch.from_numpy(g.data.copy()).cuda()
    dst = torch.zeros_like(src)
    plan.apply(src, dst, meta, ws)
    # the same ops as one-op plans, one after the other, in place
    one = torch.from_numpy(g.data.copy()).cuda()
    for op in flow:
        p1 = P.initPipeline([op]).compile(T, 2.0, 2001)
        ws.reserve(p1, rows=100, cols=2001)
        p1.apply(one, meta, ws)
    torch.cuda.synchronize()
    got, want = dst.cpu().numpy(), one.cpu().numpy()
    assert np.array_equal(src.cpu().numpy(), g.data)
    scale = float(np.max(np.abs(want)))
    assert np.max(np.abs(got.astype(np.float64) - want)) <= tol * scale
    for r in (3, 7, 40, 64, 65, 90):
        assert np.array_equal(got[r], g.data[r])
    # and the oracle's apply of the flow
    live, start = meta.flat(2001)
    ref = O.OraclePlan(flow, A.F64 if T == P.float64 else A.F32, 2.0, 2001).apply(
        g.data, live, start, keys=(meta.offsets, meta.t0, 0, 2.0))
    if T == P.float64:
        assert np.max(np.abs(got - ref)) <= 1e-9 * scale
    else:
        ref64 = O.OraclePlan(flow, A.F64, 2.0, 2001).apply(g.data.astype(np.float64), live, start,
                                                           keys=(meta.offsets, meta.t0, 0, 2.0))
        own = np.max(np.abs(ref.astype(np.float64) - ref64))
        assert np.max(np.abs(got.astype(np.float64) - ref64)) <= max(1e-5 * scale, 2 * own)
