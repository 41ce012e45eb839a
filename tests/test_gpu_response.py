"""``Pipeline.appliedResponseInto`` (pipeline.nim:840-880) through
``psg_applied_response``: the cases of the reference's tests
(tests/tpipeline.nim:403-445, applied_response), its sine/cosine-sum check
(tpipeline.nim:447-518, applied_response_matches_sine_cosine; the same
tolerance, 1e-12 + 1e-9·|want|, against the device-applied impulse), and the
moduli of the oracle's own applied impulse."""
import copy
import math

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A
from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


def sine_cosine_gain(x, hz, dt):
    """|Σ x[j]·exp(−2πi·f·j·dt)|, the angle formed as (((−2π)·f)·j)·dt."""
    j = np.arange(len(x), dtype=np.float64)
    v = np.asarray(x, dtype=np.float64)
    out = np.empty(len(hz))
    for i, f in enumerate(hz):
        p = ((-2 * math.pi * f) * j) * dt
        out[i] = math.hypot(float(np.sum(v * np.cos(p))), float(np.sum(v * np.sin(p))))
    return out


def without_trend(flow):
    ops = [copy.deepcopy(o) for o in flow]
    for o in ops:
        if o.kind == A.OP_FILTER:
            o.filter.trend = A.TR_NONE
        elif o.kind == A.OP_IIR:
            o.iir.trend = A.TR_NONE
    return ops


def impulse_out(flow, T, dtMs, samples, keep_trend=False):
    """The impulse at samples // 2 of one live row at t0 = 0, applied by the
    device plan from host memory."""
    ops = list(flow) if keep_trend else without_trend(flow)
    plan = P.initPipeline(ops).compile(T, dtMs, samples)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=1, cols=samples)
    x = np.zeros((1, samples), dtype=np.float32 if T == P.float32 else np.float64)
    x[0, samples // 2] = 1
    plan.apply(x, P.liveMeta(1, samples, dtMs), ws)
    return x[0]


def log_hz(nyq, n):
    out = np.zeros(n)
    out[n - 1] = nyq
    lo, hi = nyq * 1e-6, nyq * (1 - 1e-9)
    for i in range(1, n - 1):
        out[i] = lo * (hi / lo) ** ((i - 1) / (n - 3))
    return out


def lin_hz(nyq, n):
    if n <= 1:
        return np.zeros(n)
    return np.array([nyq * i / (n - 1) for i in range(n)])


def test_applied_response_reference_cases():
    flow = P.initPipeline([P.bandPassOp(P.Corners(8, 12, 40, 50), trend=A.TR_LINEAR)])
    ws = P.initWorkspace()
    gain = [0.0] * 3
    flow.appliedResponseInto(P.float64, 2, 256, [5.0, 25.0, 80.0], gain, ws)
    assert gain[1] > 0.5, gain
    assert gain[0] < 0.05 and gain[2] < 0.05, gain
    assert flow[0].kind == A.OP_FILTER and flow[0].filter.trend == A.TR_LINEAR
    # the trend removal is off in the applied response: a low-cut with its
    # linear detrend kept gives a different modulus at 2 Hz
    low = P.initPipeline([P.filterOp(P.lowCut(4, 8), A.TR_LINEAR)])
    fh = [2.0, 20.0]
    applied = np.zeros(2)
    low.appliedResponseInto(P.float64, 2, 256, fh, applied, ws)
    by_hand = sine_cosine_gain(impulse_out(low, P.float64, 2, 256, keep_trend=True), fh, 0.002)
    assert abs(applied[0] - by_hand[0]) > 1e-4, (applied, by_hand)
    g2 = [0.0]
    P.initPipeline([P.scaleOp(3)]).appliedResponseInto(P.float64, 2, 64, [10.0], g2, ws)
    assert abs(g2[0] - 3) < 1e-9, g2
    with pytest.raises(ValueError):
        P.initPipeline([P.scaleOp(math.inf)]).appliedResponseInto(P.float64, 2, 32, [1.0], g2, ws)
    with pytest.raises(AssertionError):
        flow.appliedResponseInto(P.float64, 2, 256, [5.0, 25.0], gain, ws)
    # no frequencies: nothing to write, the flow still compiles
    flow.appliedResponseInto(P.float32, 2, 256, [], [], ws)
    with pytest.raises(ValueError):
        flow.appliedResponseInto(P.float32, 2, 0, [], [], ws)


@pytest.mark.parametrize("T", ["float64", "float32"])
def test_applied_response_matches_sine_cosine(T):
    T = getattr(P, T)
    flows = [
        P.initPipeline([P.bandPassOp(P.Corners(8, 12, 40, 50))]),
        P.initPipeline([P.iirOp(P.butterBandPass(4, 60, 24))]),
        P.initPipeline([P.gainDbOp(12), P.filterOp(P.lowCut(4, 8))]),
    ]
    ws = P.initWorkspace()
    for flow in flows:
        for dtMs in (0.5, 2.0, 4.0):
            nyq = 500.0 / dtMs
            for samples in (64, 1000, 4001, 16384):
                try:
                    x = impulse_out(flow, T, dtMs, samples)
                except ValueError as e:
                    # a trace and its FFTs must fit one CTA's shared memory:
                    # only the longest float64 traces here do not
                    assert "shared memory" in str(e) and samples == 16384 and T == P.float64, e
                    with pytest.raises(ValueError, match="shared memory"):
                        flow.appliedResponseInto(T, dtMs, samples, [1.0], [0.0], ws)
                    continue
                for n_hz in (1, 15, 17, 31, 512):
                    for hz in (log_hz(nyq, n_hz), lin_hz(nyq, n_hz)):
                        got = np.zeros(len(hz))
                        flow.appliedResponseInto(T, dtMs, samples, hz, got, ws)
                        want = sine_cosine_gain(x, hz, dtMs / 1000)
                        d = np.abs(got - want)
                        bad = d > 1e-12 + 1e-9 * np.abs(want)
                        assert not bad.any(), (T, dtMs, samples, n_hz, hz[bad], got[bad], want[bad])


@pytest.mark.parametrize("T,tol", [("float64", 1e-10), ("float32", 2e-5)])
def test_applied_response_matches_oracle_impulse(T, tol):
    """Against the moduli of the oracle's apply of the same impulse, within
    ``tol`` of the largest modulus (the per-trace bar of the apply itself)."""
    T = getattr(P, T)
    code = T
    flow = [P.demeanOp(), P.filterOp(P.bandPass(P.Corners(3, 6, 70, 90)).withNotch(50, 2)), P.gainDbOp(6)]
    samples, dtMs = 3001, 2.0
    hz = lin_hz(250.0, 257)
    got = np.zeros(len(hz))
    P.initPipeline(flow).appliedResponseInto(T, dtMs, samples, hz, got, P.initWorkspace())
    x = np.zeros((1, samples), dtype=np.float32 if code == A.F32 else np.float64)
    x[0, samples // 2] = 1
    plan = O.OraclePlan(without_trend(flow), code, dtMs, samples, 0)
    y = plan.apply(x, np.array([samples], np.int32), np.zeros(1))
    want = sine_cosine_gain(y[0], hz, dtMs / 1000)
    assert np.max(np.abs(got - want)) <= tol * np.max(want), np.max(np.abs(got - want))
