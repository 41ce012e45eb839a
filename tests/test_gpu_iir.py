"""IIR filters (filter/iir.nim) as the device pipeline's step: each pass of
each section a chunked linear recurrence over the CTA, against the oracle's
serial restatement (the reference's single-trace form) on uneven gathers
(float64 within 1e-12 of each trace's RMS, 1e-10 with an AGC after the
filter; float32 within 1e-5), and the
reference's properties on the device: the zero-phase impulse response has
the spec's response, minimum phase is causal, zero phase symmetric, a decay
after the input ends is exactly zero, and traces too long for shared memory
run in the global-memory layout."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A
from processseg_b200 import synth
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


def gpu(flow, data, meta, dtype, dtMs, samples=None):
    plan = P.initPipeline(flow).compile(dtype, dtMs, samples or data.shape[1])
    ws = P.initWorkspace()
    ws.reserve(plan, rows=data.shape[0], cols=data.shape[1])
    src = torch.from_numpy(np.ascontiguousarray(data)).cuda()
    dst = torch.zeros_like(src)
    plan.apply(src, dst, meta, ws)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


def oracle(flow, data, meta, dtype, dtMs, samples=None):
    plan = O.OraclePlan(flow, dtype, dtMs, samples or data.shape[1], 0)
    live, start = meta.flat(data.shape[1], 0)
    return plan.apply(data, live, start)


def max_rel(got, want, live):
    worst = 0.0
    for r in range(want.shape[0]):
        n = int(live[r])
        if n == 0:
            continue
        w = want[r, :n].astype(np.float64)
        g = got[r, :n].astype(np.float64)
        rms = math.sqrt(float(np.mean(w * w)))
        d = float(np.max(np.abs(g - w)))
        worst = max(worst, d / rms if rms > 0 else d)
    return worst


# flow, float64 tolerance. A recurrence's float64 rounding, serial or chunked,
# is about 1e-13 of RMS from the exact one on these traces (both measured
# against an extended-precision recurrence); an AGC after the filter scales
# its quiet windows up, and that rounding with them.
FLOWS = {
    "bp-zero": ([P.iirOp(P.butterBandPass(3, 70, 24))], 1e-12),
    "lowcut-min-mean": ([P.demeanOp(), P.iirOp(P.butterLowCut(4, 18), P.ipMinimum, P.trMean)], 1e-12),
    "lowcut-min-mean-agc": ([P.demeanOp(), P.iirOp(P.butterLowCut(4, 18), P.ipMinimum, P.trMean), P.agcOp(500)],
                            1e-10),
    "highcut-zero-48-none": ([P.iirOp(P.butterHighCut(60, 48), P.ipZero, P.trNone), P.scaleOp(2)], 1e-12),
    "bp-min-linear": ([P.iirOp(P.butterBandPass(5, 100, 24, 36), P.ipMinimum)], 1e-12),
}


@pytest.mark.parametrize("name", list(FLOWS))
@pytest.mark.parametrize("dtype", [P.F32, P.F64])
def test_iir_flows_match_oracle(name, dtype):
    npdt = np.float32 if dtype == P.F32 else np.float64
    g = synth.shot_gather(40, 2001, 2.0, 31, npdt, live_range=(1000, 2001), sine_hz=50.0, workload="iir")
    for i, n in enumerate([2001, 1500, 700, 2, 1, 0, 1999]):
        g.numSamples[3 * i] = n
        g.data[3 * i, n:] = 0
    g.status[[4]] = P.tsDead
    g.data[8] += np.linspace(-3, 5, 2001).astype(npdt)  # a drift
    g.data[9] += 1000  # a large DC
    meta = g.meta()
    flow, tol64 = FLOWS[name]
    got = gpu(flow, g.data, meta, dtype, 2.0)
    want = oracle(flow, g.data, meta, dtype, 2.0)
    live = meta.flat(2001)[0]
    assert max_rel(got, want, live) <= (1e-5 if dtype == P.F32 else tol64)
    assert np.array_equal(got[4], g.data[4])
    for r in range(g.data.shape[0]):
        assert np.array_equal(got[r, live[r]:], g.data[r, live[r]:])


def one_trace(spec, phase, trend, x, dtMs, T=P.F64):
    npdt = np.float32 if T == P.F32 else np.float64
    data = np.ascontiguousarray(x, dtype=npdt)[None, :]
    return gpu([P.iirOp(spec, phase, trend)], data, P.liveMeta(1, data.shape[1], dtMs), T, dtMs)[0]


def test_device_properties():
    ns, dt = 4000, 2.0
    x = np.zeros(ns)
    x[ns // 2] = 1
    df = 1000 / (ns * dt)
    for s in (P.butterBandPass(4, 60, 24), P.butterLowCut(2, 24), P.butterHighCut(80, 48)):
        h = one_trace(s, P.ipZero, A.TR_NONE, x, dt)
        mag = np.abs(np.fft.rfft(h))
        want = np.array([s.response(k * df, dt) for k in range(ns // 2 + 1)])
        assert np.max(np.abs(mag - want)) < 1e-4
    x = np.zeros(2001)
    x[1000] = 1
    s = P.butterBandPass(4, 60, 24)
    m = one_trace(s, P.ipMinimum, A.TR_NONE, x, dt)
    assert np.max(np.abs(m[:1000])) == 0 and m[1000] > 0
    z = one_trace(s, P.ipZero, A.TR_NONE, x, dt)
    assert np.max(np.abs(z[1001:] - z[999::-1])) < 1e-12
    # a decay after a spike ends in exact zeros (float64 and float32)
    for T, n in ((P.F64, 20000), (P.F32, 40000)):
        x = np.zeros(n)
        x[10] = 1
        for ph in (P.ipZero, P.ipMinimum):
            y = one_trace(P.butterHighCut(100, 24), ph, A.TR_NONE, x, 0.25, T)
            assert y[n - 10000] == 0 and y[-1] == 0


def test_long_iir_traces_in_the_global_layout():
    """A float64 IIR over 20000 samples whose float64 work area does not fit
    beside the row: the same bar against the oracle."""
    g = synth.shot_gather(5, 20000, 0.5, 41, np.float64, live_range=(12000, 20000), workload="iir-long")
    meta = g.meta()
    flow = [P.iirOp(P.butterBandPass(4, 60, 24))]
    got = gpu(flow, g.data, meta, P.F64, 0.5)
    want = oracle(flow, g.data, meta, P.F64, 0.5)
    assert max_rel(got, want, meta.flat(20000)[0]) <= 1e-12


def test_iir_plan_api_and_serving():
    plan = P.initIirPlan(P.float32, P.butterBandPass(4, 60, 24), 2.0, 500)
    x = torch.randn(6, 500, device="cuda")
    ref = x.clone()
    ws = P.initWorkspace()
    plan.applyFilter(x, P.liveMeta(6, 500, 2.0), ws)
    torch.cuda.synchronize()
    want = oracle([P.iirOp(P.butterBandPass(4, 60, 24))], ref.cpu().numpy(), P.liveMeta(6, 500, 2.0), P.F32, 2.0)
    assert max_rel(x.cpu().numpy(), want, [500] * 6) <= 1e-5
    # the request loop serves an IIR plan with the plain apply's launches: the same bits
    compiled = P.initPipeline([P.iirOp(P.butterBandPass(4, 60, 24))]).compile(P.float32, 2.0, 500)
    src = np.random.default_rng(4).standard_normal((4, 500)).astype(np.float32)
    plain = np.zeros_like(src)
    ws2 = P.initWorkspace()
    ws2.reserve(compiled, rows=4, cols=500)
    compiled.apply(src, plain, P.liveMeta(4, 500, 2.0), ws2)
    served = np.zeros_like(src)
    with P.Server(arena_bytes=16 << 20) as srv:
        srv.wait(srv.submit(compiled, src, served, P.liveMeta(4, 500, 2.0)), 30000)
    assert np.array_equal(served, plain)
