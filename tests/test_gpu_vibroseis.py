"""Vibroseis correlation and the vertical stack on the device against the
oracle: the C3 workload (240 channels × 10001 samples at 2 ms, a 12 s 8-80 Hz
linear sweep with 300 ms cos² tapers, 6 s out, 4 sweeps stacked). Tolerance:
the reference's own float32 bar, 2e-5 of the correlation peak
(tests/tcorrelate.nim:306-364), and 1e-10 of it in float64."""
import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import synth
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


def c3_inputs(channels=240, sweeps=4):
    spec = P.linearSweep(8, 80, 12000, 2, P.initSweepTaper(300, 300, P.tpCos2))
    pilot = P.generatePilot(spec, np.float64)
    recs = synth.vibroseis_records(pilot.samples, channels=channels, sweeps=sweeps)
    return pilot, recs


@pytest.mark.parametrize("dtype", [P.F32, P.F64])
def test_correlation_matches_oracle(dtype):
    pilot, recs = c3_inputs(channels=32, sweeps=1)
    npd = np.float32 if dtype == P.F32 else np.float64
    src = recs[0].astype(npd)
    rows = src.shape[0]
    status = np.full(rows, P.tsLive, np.int32)
    status[3] = P.tsDead
    status[4] = P.tsAux
    ns = np.full(rows, 10001, np.int32)
    ns[5] = 7000
    meta = P.initChunkMeta(status, ns, 2.0, np.zeros(rows), 0, [6])
    plan = P.initCorrelationPlan(dtype, pilot, 2.0, 10001, outSamples=3000)
    assert plan.nfft == 16200 and plan.outSamples == 3000
    s = torch.from_numpy(src).cuda()
    d = torch.zeros(rows, 3000, dtype=s.dtype, device="cuda")
    plan.correlateInto(s, d, meta)
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    live, _ = meta.flat(10001, 1)
    want, nfft, _ = O.correlate(pilot.samples, 2.0, 0.0, src, live, 2.0, 10001, outSamples=3000)
    assert nfft == 16200
    peak = np.max(np.abs(want))
    tol = 2e-5 if dtype == P.F32 else 1e-10
    assert np.max(np.abs(got - want)) <= tol * peak
    assert np.all(got[3] == 0) and np.all(got[6] == 0)  # dead and failed rows give zeros
    assert np.any(got[4] != 0)  # an auxiliary row is correlated


def test_correlate_and_stack_c3():
    pilot, recs = c3_inputs()
    sweeps, ch, ns = recs.shape
    plan = P.initCorrelationPlan(P.float32, pilot, 2.0, ns, outSamples=3000)
    stack = P.initRecordStack(ch, 3000, 2.0)
    meta = P.initChunkMeta(np.full(ch, P.tsLive, np.int32), np.full(ch, ns, np.int32), 2.0)
    num = np.zeros((ch, 3000))
    cnt = np.zeros((ch, 3000), np.int32)
    live, _ = meta.flat(ns, 1)
    for s in range(sweeps):
        x = torch.from_numpy(recs[s]).cuda()
        d = torch.zeros(ch, 3000, device="cuda")
        plan.correlateInto(x, d, meta, stack=stack)
        want, _, _ = O.correlate(pilot.samples, 2.0, 0.0, recs[s], live, 2.0, ns, outSamples=3000)
        O.stack_add(num, cnt, want, np.full(ch, 3000, np.int32))
    out = torch.zeros(ch, 3000, device="cuda")
    stack.stackInto(out)
    fold = torch.zeros(ch, 3000, dtype=torch.int32, device="cuda")
    stack.foldInto(fold)
    torch.cuda.synchronize()
    want = O.stack_result(num, cnt, np.float32)
    assert np.array_equal(fold.cpu().numpy(), cnt)
    assert np.max(np.abs(out.cpu().numpy() - want)) <= 2e-5 * np.max(np.abs(want))


def test_stack_skips_non_finite_rows():
    st = P.initRecordStack(4, 100, 2.0)
    b = torch.ones(4, 100, device="cuda")
    b[1, 50] = float("nan")
    meta = P.initChunkMeta(np.full(4, P.tsLive, np.int32), np.full(4, 100, np.int32), 2.0)
    st.addRecord(b, meta)
    st.addRecord(b, meta, rowMap=[0, 0, -1, 3])
    out = torch.zeros(4, 100, device="cuda")
    st.stackInto(out)
    fold = torch.zeros(4, 100, dtype=torch.int32, device="cuda")
    st.foldInto(fold)
    torch.cuda.synchronize()
    f = fold.cpu().numpy()
    assert f[0, 0] == 2 and f[1, 0] == 0 and f[2, 0] == 1 and f[3, 0] == 2
    assert np.all(out.cpu().numpy()[[0, 2, 3]] == 1)


def test_sweeps_in_one_block_stack_as_sweep_by_sweep():
    """The gather's sweeps correlated as one block of records, each mapped to
    its channel's stack row (a device rowMap), give the stack of the
    sweep-by-sweep calls (float64 sums, added in another order)."""
    pilot, recs = c3_inputs(channels=48, sweeps=3)
    sweeps, ch, ns = recs.shape
    plan = P.initCorrelationPlan(P.float32, pilot, 2.0, ns, outSamples=3000)
    meta1 = P.initChunkMeta(np.full(ch, P.tsLive, np.int32), np.full(ch, ns, np.int32), 2.0)
    a = P.initRecordStack(ch, 3000, 2.0)
    for s in range(sweeps):
        plan.correlateInto(torch.from_numpy(recs[s]).cuda(), None, meta1, stack=a)
    b = P.initRecordStack(ch, 3000, 2.0)
    metan = P.initChunkMeta(np.full(sweeps * ch, P.tsLive, np.int32), np.full(sweeps * ch, ns, np.int32), 2.0)
    rmap = (torch.arange(sweeps * ch, dtype=torch.int32, device="cuda") % ch).contiguous()
    plan.correlateInto(torch.from_numpy(recs.reshape(sweeps * ch, ns)).cuda(), None, metan, stack=b, rowMap=rmap)
    oa, ob = torch.zeros(ch, 3000, device="cuda"), torch.zeros(ch, 3000, device="cuda")
    a.stackInto(oa)
    b.stackInto(ob)
    fa = torch.zeros(ch, 3000, dtype=torch.int32, device="cuda")
    fb = torch.zeros_like(fa)
    a.foldInto(fa)
    b.foldInto(fb)
    torch.cuda.synchronize()
    assert torch.equal(fa, fb) and int(fa.max()) == sweeps
    ref = float(oa.abs().max())
    assert float((oa - ob).abs().max()) <= 1e-6 * ref


@pytest.mark.parametrize("law", ["dbPerOctave", "dbPerHz", "exponential", "table"])
def test_correlation_with_nonlinear_pilots_matches_oracle(law):
    """The non-linear laws' pilots (with Kaiser, Gaussian or power ramps and
    a harmonic-free float32 pilot) correlated on the device against the
    oracle's correlation of the same samples, at the float32 bar."""
    taper = {"dbPerOctave": P.initSweepTaper(300, 300, P.tpKaiser),
             "dbPerHz": P.initSweepTaper(250, 400, P.tpGaussian),
             "exponential": P.initSweepTaper(300, 300, P.tpPower, 3.0),
             "table": P.initSweepTaper(200, 200, P.tpBlackmanHarris)}[law]
    spec = {"dbPerOctave": lambda: P.dbPerOctaveSweep(8, 80, 8000, 2, 3, taper),
            "dbPerHz": lambda: P.dbPerHzSweep(8, 80, 8000, 2, 0.05, taper),
            "exponential": lambda: P.exponentialSweep(6, 90, 8000, 2, taper),
            "table": lambda: P.tableSweep([P.SweepPoint(0, 8), P.SweepPoint(3000, 30),
                                           P.SweepPoint(8000, 80)], 2, taper)}[law]()
    pilot = P.generatePilot(spec, np.float32)
    assert pilot.samples.dtype == np.float32 and len(pilot) == 4000
    recs = synth.vibroseis_records(pilot.samples.astype(np.float64), channels=24, sweeps=1, samples=8001)
    src = recs[0].astype(np.float32)
    rows = src.shape[0]
    meta = P.initChunkMeta(np.full(rows, P.tsLive, np.int32), np.full(rows, 8001, np.int32), 2.0)
    plan = P.initCorrelationPlan(P.float32, pilot, 2.0, 8001, outSamples=2000)
    s = torch.from_numpy(src).cuda()
    d = torch.zeros(rows, 2000, dtype=s.dtype, device="cuda")
    plan.correlateInto(s, d, meta)
    torch.cuda.synchronize()
    live, _ = meta.flat(8001, 1)
    want, _, _ = O.correlate(pilot.samples.astype(np.float64), 2.0, 0.0, src, live, 2.0, 8001, outSamples=2000)
    peak = np.max(np.abs(want))
    assert np.max(np.abs(d.cpu().numpy() - want)) <= 2e-5 * peak
