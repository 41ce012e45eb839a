"""Top and bottom mutes (core/mute.nim) as steps of the device pipeline,
against the oracle: the reference's known answers (tests/tmute.nim), and
mutes inside filter/AGC flows on uneven gathers whose rows carry their own
offsets and t0Ms, in a window (firstSample > 0), with dead, auxiliary and
NaN-offset rows. float64 within 1e-12 of each trace's RMS, float32 within
1e-5 (the weights' sine is CUDA's against glibc's, ≤ 1 ulp apart)."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A
from processseg_b200 import synth
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


def gpu(flow, data, meta, dtype, dtMs, host=False):
    plan = P.initPipeline(flow).compile(dtype, dtMs, data.shape[1])
    ws = P.initWorkspace()
    ws.reserve(plan, rows=data.shape[0], cols=data.shape[1])
    if host:
        dst = np.zeros_like(data)
        plan.apply(data, dst, meta, ws)
        return dst
    src = torch.from_numpy(data).cuda()
    dst = torch.zeros_like(src)
    plan.apply(src, dst, meta, ws)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


def oracle(flow, data, meta, dtype, dtMs):
    plan = O.OraclePlan(flow, dtype, dtMs, data.shape[1], 0)
    live, start = meta.flat(data.shape[1], 0)
    return plan.apply(data, live, start, keys=(meta.offsets, meta.t0, meta.firstSample, meta.dtMs))


def max_rel(got, want, live):
    worst = 0.0
    for r in range(want.shape[0]):
        n = int(live[r])
        if n == 0:
            continue
        w = want[r, :n].astype(np.float64)
        g = got[r, :n].astype(np.float64)
        rms = math.sqrt(float(np.mean(w * w)))
        d = float(np.max(np.abs(g - w))) if n else 0.0
        worst = max(worst, d / rms if rms > 0 else d)
    return worst


def test_reference_known_answers_on_the_device():
    cases = [  # (op, rows, dtMs, t0, offsets, first, live, status)
        (P.muteTopOp(P.timeMute(6), 4), np.ones((1, 10)), 1.0, [0.0], [0.0], 0, None, None),
        (P.muteTopOp(P.timeMute(2.5), 1), np.ones((1, 5)), 1.0, [0.0], [0.0], 0, None, None),
        (P.muteTopOp(P.timeMute(2), 0), np.ones((1, 5)), 1.0, [0.0], [0.0], 0, None, None),
        (P.muteTopOp(P.timeMute(99), 3), np.ones((1, 4)), 1.0, [0.0], [0.0], 0, None, None),
        (P.muteTopOp(P.timeMute(2), 3), np.ones((1, 4)), 1.0, [math.nan], [0.0], 0, None, None),
        (P.muteBottomOp(P.timeMute(3), 4), np.ones((1, 10)), 1.0, [0.0], [0.0], 0, None, None),
        (P.muteBottomOp(P.timeMute(-1), 0), np.ones((1, 4)), 1.0, [0.0], [0.0], 0, None, None),
        (P.muteTopOp(P.lmoMute(2000), 20), np.ones((3, 150)), 4.0, [0.0] * 3, [0.0, 400, 800], 0, None, None),
        (P.muteTopOp(P.timeMute(140)), np.ones((2, 40)), 4.0, [100.0, 0.0], [0.0, 0.0], 0, None, None),
        (P.muteTopOp(P.timeMute(140)), np.ones((1, 30)), 4.0, [0.0], [0.0], 20, None, None),
        (P.muteBottomOp(P.tableMute([100.0, 400], [200.0, 160])), np.ones((4, 100)), 4.0, [0.0] * 4,
         [100.0, 200, math.nan, 400], 0, [100, 100, 100, 60], [A.TS_LIVE, A.TS_AUX, A.TS_LIVE, A.TS_LIVE]),
        (P.muteTopOp(P.lmoMute(1800, padMs=-20), 30), np.ones((4, 1000)), 2.0, [0.0] * 4, [0.0, 500, 1000, 1500],
         0, None, None),
    ]
    for dtype, npdt in ((P.F64, np.float64), (P.F32, np.float32)):
        for op, rows, dtMs, t0, offsets, first, live, status in cases:
            rows = rows.astype(npdt)
            r, c = rows.shape
            if live is not None:
                rows[3, 60:] = 7
            meta = P.initChunkMeta(status if status is not None else np.full(r, A.TS_LIVE, np.int32),
                                   (np.asarray(live) if live is not None else np.full(r, c)) + first, dtMs, t0,
                                   first, (), offsets)
            got = gpu([op], rows, meta, dtype, dtMs)
            want = oracle([op], rows, meta, dtype, dtMs)
            # zeros and untouched samples exactly; tapered ones to the weights' rounding
            exact = (want == 0) | (want == rows)
            assert np.array_equal(got[exact], want[exact]), (op, dtype)
            assert np.allclose(got, want, rtol=1e-6 if dtype == P.F32 else 1e-14, atol=0), (op, dtype)


def keyed_gather(rows, cols, dtMs, npdt, seed, first=0):
    g = synth.shot_gather(rows, cols + first, dtMs, seed, npdt, live_range=((cols + first) * 2 // 3, cols + first),
                          sine_hz=50.0, workload="mutes")
    g.data = np.ascontiguousarray(g.data[:, first:])
    g.t0Ms = np.random.default_rng(seed).uniform(-40.0, 60.0, rows)
    g.status[[3]] = P.tsDead
    g.status[[5]] = P.tsAux
    g.offsets[7] = math.nan
    g.offsets[8] = -g.offsets[8]
    return g


FLOWS = {
    "lmo-top": [P.muteTopOp(P.lmoMute(2500, t0Ms=20, padMs=-10), taperMs=40)],
    "filter-between-mutes": [P.demeanOp(), P.muteTopOp(P.lmoMute(2000), taperMs=30),
                             P.bandPassOp(P.Corners(4, 8, 60, 80)),
                             P.muteBottomOp(P.tableMute([0.0, 1000, 3000], [2500.0, 3200, 5000]), taperMs=60)],
    # AGC after the filter, mutes last: an AGC after a mute and a filter
    # would scale the filter's far tails inside the muted zone (rounding
    # noise) up to the target, where no two implementations agree
    "agc-then-mutes": [P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 60, 80)), P.agcOp(400),
                       P.muteTopOp(P.lmoMute(2000), taperMs=30),
                       P.muteBottomOp(P.tableMute([0.0, 1000, 3000], [2500.0, 3200, 5000]), taperMs=60)],
    "time-mutes-normalize": [P.muteTopOp(P.timeMute(300), taperMs=17.3), P.muteBottomOp(P.timeMute(3700.5)),
                             P.normalizeOp(P.normRms)],
}


@pytest.mark.parametrize("name", list(FLOWS))
@pytest.mark.parametrize("dtype", [P.F32, P.F64])
def test_mute_flows_match_oracle(name, dtype):
    npdt = np.float32 if dtype == P.F32 else np.float64
    flow = FLOWS[name]
    g = keyed_gather(120, 2001, 2.0, npdt, seed=21, first=7)
    meta = g.meta(firstSample=7)
    got = gpu(flow, g.data, meta, dtype, 2.0)
    want = oracle(flow, g.data, meta, dtype, 2.0)
    live = meta.flat(g.data.shape[1])[0]
    tol = 1e-5 if dtype == P.F32 else 1e-12
    e = max_rel(got, want, live)
    if dtype == P.F32 and e > tol:
        # as the pipeline's parity bar: no further from the float64 oracle
        # than twice the float32 oracle is
        want64 = oracle(flow, g.data.astype(np.float64), meta, P.F64, 2.0)
        assert max_rel(got, want64, live) <= max(tol, 2 * max_rel(want, want64, live))
    else:
        assert e <= tol
    # rows the plan does not process are copied bit for bit
    for r in (3, 5):
        assert np.array_equal(got[r], g.data[r])
    # the host-memory path stages the keys with the rows: the same bits
    host = gpu(flow, g.data, meta, dtype, 2.0, host=True)
    assert np.array_equal(host, got)


def test_mute_plan_needs_keys_and_is_served_with_them():
    plan = P.initPipeline([P.muteTopOp(P.timeMute(100))]).compile(P.float32, 2.0, 500)
    assert plan.needsKeys
    assert not P.initPipeline([P.demeanOp()]).compile(P.float32, 2.0, 500).needsKeys
    ws = P.initWorkspace()
    ws.reserve(plan, rows=4, cols=500)
    src = torch.ones(4, 500, device="cuda")
    meta = P.liveMeta(4, 500, 2.0)
    live, start = meta.device(500)
    with pytest.raises(ValueError, match="mutes"):
        A.check(A.lib().psg_apply(plan.h, ws.h, None, src.data_ptr(), 4, 500, live.data_ptr(), start.data_ptr(),
                                  2.0, None))
    torch.cuda.synchronize()
    assert float(src.min()) == 1.0, "nothing changed"
    plan.apply(src, meta, ws)
    torch.cuda.synchronize()
    assert float(src[:, :50].abs().max()) == 0 and float(src[:, 50:].min()) == 1
    # served: the loop copies the rows' keys in with the block (psg_submit_keyed)
    x = np.ones((4, 500), np.float32)
    y = np.zeros_like(x)
    with P.Server(arena_bytes=16 << 20) as srv:
        srv.wait(srv.submit(plan, x, y, meta), 30000)
    assert np.array_equal(y, src.cpu().numpy())


def test_applied_response_mute_sees_offset_zero_and_t0_zero():
    """appliedResponseInto runs its impulse (sample samples // 2) at t0 = 0
    and offset 0: a top mute after it silences it, one before it passes it."""
    ws = P.initWorkspace()
    g = [0.0, 0.0]
    P.initPipeline([P.muteTopOp(P.lmoMute(2000, t0Ms=300))]).appliedResponseInto(P.float64, 2.0, 256, [10.0, 50.0],
                                                                                 g, ws)
    assert g == [0.0, 0.0]
    P.initPipeline([P.muteTopOp(P.lmoMute(2000, t0Ms=200))]).appliedResponseInto(P.float64, 2.0, 256, [10.0, 50.0],
                                                                                 g, ws)
    assert abs(g[0] - 1) < 1e-12 and abs(g[1] - 1) < 1e-12
