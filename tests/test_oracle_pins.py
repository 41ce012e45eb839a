"""Pins the CPU oracle (oracle/psg_oracle.cpp) to the reference's own
known-answer tests and tolerances. The reference (Nim) cannot be built
here, so these checks, ported from its test suite, are what make the oracle
a stand-in for it. Each block cites the reference test it restates."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.usefixtures("built")


def fast_lens(limit):
    return [n for n in range(1, limit + 1) if O.is_fast_len(n)]


def test_fast_lengths():
    # tests/tfftplan.nim:46-58
    assert O.is_fast_len(1) and O.is_fast_len(2) and O.is_fast_len(2025) and O.is_fast_len(4096)
    assert not O.is_fast_len(0) and not O.is_fast_len(7) and not O.is_fast_len(2001)
    assert O.next_fast_len(2001) == 2048 and O.next_fast_len(2001, even=False) == 2025
    assert O.next_fast_len(0) == 2 and O.next_fast_len(0, even=False) == 1
    assert O.next_fast_len(7) == 8 and O.next_fast_len(11) == 12 and O.next_fast_len(13) == 16
    assert O.next_fast_len(14, even=False) == 15
    assert O.next_fast_len(4097) == 4320
    for n in range(1, 5001, 7):
        e = O.next_fast_len(n)
        assert O.is_fast_len(e) and e % 2 == 0 and e >= n


@pytest.mark.parametrize("dtype,tol", [(np.float32, 1e-5), (np.float64, 1e-12)])
def test_fft_matches_dft_on_every_smooth_length(dtype, tol):
    # tests/tfftplan.nim:64-94 (numpy's float64 FFT stands in for the naive DFT)
    rng = np.random.default_rng(17)
    worst = 0.0
    for n in fast_lens(4096):
        x64 = rng.uniform(-1, 1, n).astype(np.float32).astype(np.float64)
        ref = np.fft.rfft(x64)
        re, im = O.fft_forward(x64.astype(dtype))
        e = np.max(np.abs(re.astype(np.float64) + 1j * im.astype(np.float64) - ref)) / max(
            np.max(np.abs(ref)), 1e-300)
        assert e <= tol, (n, e)
        back = O.fft_inverse(re, im, n)
        rt = np.max(np.abs(back.astype(np.float64) - x64))
        assert rt <= tol, (n, rt)
        worst = max(worst, e)


def test_known_spectra():
    # tests/tfftplan.nim:96-110
    x = np.zeros(16)
    x[0] = 1
    re, im = O.fft_forward(x)
    assert np.all(np.abs(re - 1) < 1e-15) and np.all(np.abs(im) < 1e-15)
    x = np.cos(2 * np.pi * 3 * np.arange(16) / 16)
    re, im = O.fft_forward(x)
    want = np.where(np.arange(9) == 3, 8.0, 0.0)
    assert np.all(np.abs(re - want) < 1e-13) and np.all(np.abs(im) < 1e-13)


def test_filter_plan_known_answers():
    # bench/README.md:116-117 (L, nfft); tests/tfilterapply.nim:34-61
    bp = P.bandPass(P.Corners(4, 8, 60, 80))
    i = O.filter_plan_info(bp, P.F32, 2.0, 2001)
    assert (i["margin"], i["nfft"], i["reflect"]) == (110, 2250, False)
    lc = P.lowCut(0.5, 1)
    i = O.filter_plan_info(lc, P.F32, 2.0, 2001, with_gain=True)
    assert (i["margin"], i["nfft"]) == (881, 3840)
    assert i["gain"][0] == 0 and i["gain"][i["nfft"] // 2] == 1
    assert i["nfft"] >= 2001 + 2 * i["margin"] and i["nfft"] < 2001 + 4 * i["margin"]
    hc = O.filter_plan_info(P.highCut(60, 80), P.F32, 2.0, 2001)
    assert hc["reflect"] and hc["nfft"] >= 2001 + 4 * hc["margin"]
    flat = O.filter_plan_info(P.bandPass(P.Corners(0, 0, math.inf, math.inf)), P.F64, 2.0, 2001)
    assert flat["margin"] == 0
    # an impulse longer than the trace: pads cut to the trace (tfilterapply.nim:63-73)
    far = O.filter_plan_info(P.lowCut(0.02, 0.04), P.F64, 2.0, 2001)
    assert far["margin"] > 10 * 2001 and 3 * 2001 <= far["nfft"] < 4 * 2001


def test_response_known_answers():
    # src/processSEG/filter/design.nim:8; tests/tfilterdesign.nim:25-50
    bp = P.bandPass(P.Corners(4, 8, 60, 80))
    assert abs(O.response(bp, 6, 2) - 0.5) < 1e-12 and abs(O.response(bp, 70, 2) - 0.5) < 1e-12
    assert O.response(bp, 30, 2) == 1 and O.response(bp, 2, 2) == 0 and O.response(bp, 90, 2) == 0
    lc = P.lowCut(0.5, 1)
    assert O.response(lc, 0, 2) == 0 and abs(O.response(lc, 0.75, 2) - 0.5) < 1e-15
    hc = P.butterHighCut(60, 24)
    assert abs(20 * math.log10(O.response(hc, 60, 2)) - 20 * math.log10(0.5)) < 1e-9
    assert O.response(hc, 250, 2) == 0
    w = math.tan(math.pi * 100 * 0.002) / math.tan(math.pi * 60 * 0.002)
    assert abs(O.response(hc, 100, 2) - 1 / (1 + w ** 4)) < 1e-12
    s = P.bandPass(P.Corners(2, 4, 100, 120)).withNotch(50, 4)
    assert O.response(s, 50, 2) == 0 and abs(O.response(s, 49, 2) - 0.5) < 1e-12
    assert O.response(s, 48, 2) == 1 and O.response(s, 52, 2) == 1


def test_margins_and_agc_windows():
    # tests/tgain.nim:159-160; tests/tpipeline.nim:306-324
    assert O.required_margin([P.agcOp(500)], 2.0) == 125
    assert O.required_margin([P.agcOp(4)], 2.0) == 1  # window of 3 samples
    c1 = [P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 60, 80)), P.agcOp(500)]
    assert O.required_margin(c1, 2.0) == 110 + 125
    plan = O.OraclePlan(c1, P.F32, 2.0, 2001)
    assert plan.margin == 235 and plan.partCount == 1
    assert O.OraclePlan([P.agcOp(20), P.normalizeOp(P.normRms, P.perPanel)], P.F32, 2.0, 50).partCount == 2
    assert O.required_margin([P.gainDbOp(3)], 2.0) == 0
    with pytest.raises(ValueError, match=r"^op 1 \(opAgc\): "):
        O.required_margin([P.demeanOp(), P.agcOp(1)], 2.0)
    assert P.decodeWindow(800, 1200, 110, 2001) == (690, 1310)
    assert P.decodeWindow(50, 300, 110, 2001) == (0, 410)
    assert P.decodeWindow(1900, 2000, 110, 2001) == (1790, 2000)
    assert P.decodeWindow(10, 20, -5, 100) == (10, 20)
    assert P.decodeWindow(10, 20, 2 ** 62, 100) == (0, 99)


def ref_agc(x, h, rms_mode, target, epsilon):
    """tests/tgain.nim:105-121: direct window sums in float64."""
    n = x.size
    eps = epsilon * math.sqrt(np.sum(x * x) / n)
    y = np.empty(n)
    for i in range(n):
        lo, e = max(0, i - h), min(n, i + h + 1)
        seg = x[lo:e]
        s = np.sum(seg * seg) if rms_mode else np.sum(np.abs(seg))
        level = math.sqrt(s / (e - lo)) if rms_mode else s / (e - lo)
        y[i] = x[i] * (target / (level + eps))
    return y


@pytest.mark.parametrize("mode", [P.agcRms, P.agcMeanAbs])
def test_agc_matches_direct_sums(mode):
    # tests/tgain.nim:123-158
    rng = np.random.default_rng(5)
    for n, win in [(1, 6.0), (2, 6.0), (5, 6.0), (7, 6.0), (13, 6.0), (14, 6.0), (100, 6.0),
                   (101, 50.0), (500, 104.0), (2001, 500.0), (30, 200.0)]:
        x = rng.standard_normal(n)
        x[n // 3] += 20
        h = max(1, int(math.floor(win / 4 + 0.5)))  # Nim round: half away from zero
        want = ref_agc(x, h, mode == P.agcRms, 2.0, 1e-9)
        got = O.agc_row(x, win, 2.0, mode, 2.0, 1e-9)
        assert np.all(np.abs(got - want) <= 1e-12 * np.maximum(np.abs(got), np.abs(want))), (n, win)
    for n in (3, 40, 777):
        x = rng.standard_normal(n) * 1e-20
        want = ref_agc(x, int(math.floor(30 / 4 + 0.5)), mode == P.agcRms, 1.0, 1e-9)
        got = O.agc_row(x.astype(np.float32), 30.0, 2.0, mode)
        assert np.all(np.abs(got - want) <= 1e-5 * np.maximum(np.abs(got), np.abs(want)))


def test_agc_precision_at_120_db():
    # tests/tgain.nim:187-212
    rng = np.random.default_rng(11)
    n = 3000
    x = rng.standard_normal(n)
    x[1000:] *= 1e-6
    want = ref_agc(x, 25, True, 1.0, 1e-12)
    got = O.agc_row(x, 100.0, 2.0, P.agcRms, 1.0, 1e-12)
    assert np.all(np.abs(got - want) <= 1e-12 * np.maximum(np.abs(got), np.abs(want)))
    assert abs(math.sqrt(np.mean(got[1200:] ** 2)) - 1) < 0.05


def clean(n=2001, dt=2.0):
    # tests/tfilterapply.nim:15-21: events well inside the trace
    from processseg_b200.synth import ricker
    x = np.zeros(n)
    t = np.arange(n) * dt
    for c, f, a in ((600, 25, 1.0), (1800, 30, -0.7), (3300, 20, 0.5)):
        tau = t - c
        x += np.where(np.abs(tau) <= 3000 / f, a * ricker(tau, f), 0.0)
    return x


def run_filter(x, spec, dtype, trend=P.trLinear, dt=2.0):
    plan = O.OraclePlan([P.filterOp(spec, trend)], dtype, dt, x.size)
    b = np.ascontiguousarray(x.astype(np.float32 if dtype == P.F32 else np.float64)[None, :])
    return plan.apply(b, np.array([x.size], np.int32))[0].astype(np.float64)


@pytest.mark.parametrize("dtype,tol", [(P.F64, 1e-9), (P.F32, 2e-4)])
def test_filter_edges_match_clean_reference(dtype, tol):
    # tests/tfilterapply.nim:75-101
    c = clean()
    reference = run_filter(c, P.lowCut(0.5, 1), dtype)
    assert np.max(np.abs(reference - c)) < 0.02
    dc = c + 1000
    drift = c + (-30 + 50 * np.arange(c.size) * 2.0 / 1000)
    for x in (dc, drift):
        y = run_filter(x, P.lowCut(0.5, 1), dtype)
        assert np.max(np.abs(y - reference)) <= tol


def test_symmetric_impulse_response():
    # tests/tfilterapply.nim:157-176
    for s in (P.bandPass(P.Corners(4, 8, 60, 80)), P.lowCut(1, 2), P.butterBandPass(5, 60),
              P.highCut(60, 80).withNotch(50, 4)):
        x = np.zeros(2001)
        x[1000] = 1
        y = run_filter(x, s, P.F64, trend=P.trNone)
        assert np.max(np.abs(y[1001:2001] - y[999::-1][:1000])) < 1e-12
        assert y[1000] > 0


def direct_corr(x, p, m):
    # tests/tcorrelate.nim:15-20
    lo = max(0, -m)
    hi = min(p.size, x.size - m)
    if hi <= lo:
        return 0.0
    return float(np.dot(x[m + lo:m + hi], p[lo:hi]))


def test_correlation_equals_direct():
    # tests/tcorrelate.nim:40-64
    pilot = O.linear_sweep(8, 60, 1000, 2, 100, 100, 2)
    n = 1201
    x = np.random.default_rng(7).standard_normal(n)
    y, nfft, _ = O.correlate(pilot, 2.0, 0.0, x[None, :], np.array([n]), 2.0, n, normalize=False)
    assert y.shape[1] == n - pilot.size
    d = np.array([direct_corr(x, pilot, m) for m in range(y.shape[1])])
    assert np.max(np.abs(y[0] - d)) < 1e-10 * np.max(np.abs(d))
    y2, _, _ = O.correlate(pilot, 2.0, 0.0, x[None, :], np.array([n]), 2.0, n, outSamples=n,
                           normalize=False)
    for m in (n - pilot.size, n - 100, n - 1):
        assert abs(y2[0, m] - direct_corr(x, pilot, m)) < 1e-10 * np.max(np.abs(d))


def test_correlation_whole_sample_start_times():
    # tests/tcorrelate.nim:66-93
    base = O.linear_sweep(8, 60, 1000, 2, 100, 100, 2)
    n = 1801
    x = np.random.default_rng(11).standard_normal(n)
    for t0 in (-20.0, 20.0, -900.0, 3000.0):
        y, _, _ = O.correlate(base, 2.0, t0, x[None, :], np.array([n]), 2.0, n, outSamples=n,
                              normalize=False)
        s = int(t0 / 2)
        d = np.array([0.0 if (m + s <= -base.size or m + s >= n) else direct_corr(x, base, m + s)
                      for m in range(n)])
        assert np.max(np.abs(y[0] - d)) < 1e-10 * np.max(np.abs(d))


def test_correlation_known_answers():
    # bench/README.md:368-369 (nfft 16200); tests/tcorrelate.nim:95-135
    pilot = O.linear_sweep(8, 80, 12000, 2, 300, 300, 2)
    assert pilot.size == 6000
    _, nfft, _ = O.correlate(pilot, 2.0, 0.0, np.zeros((1, 10001)), np.array([10001]), 2.0, 10001,
                             outSamples=3000)
    assert nfft == 16200
    p = O.linear_sweep(10, 80, 4000, 2, 200, 200, 2)
    n = 3501
    refl = np.zeros(n)
    refl[100], refl[400], refl[900] = 1.0, -0.5, 0.25
    x = np.convolve(refl, p)[:n]
    y, _, _ = O.correlate(p, 2.0, 0.0, x[None, :], np.array([n]), 2.0, n)
    assert abs(y[0, 100] - 1) < 1e-3 and abs(y[0, 400] + 0.5) < 1e-3 and abs(y[0, 900] - 0.25) < 1e-3
    refl = np.zeros(6001)
    refl[300] = 0.7
    for amp, length in ((1.0, 4000.0), (3.5, 8000.0)):
        p = O.linear_sweep(10, 80, length, 2, 200, 200, 2, amplitude=amp)
        x = np.convolve(refl, p)[:6001]
        y, _, scale = O.correlate(p, 2.0, 0.0, x[None, :], np.array([6001]), 2.0, 6001)
        assert abs(y[0, 300] - 0.7) < 1e-6 * 0.7
        assert abs(scale * np.sum(p * p) - 1) < 1e-9


def test_pipeline_parts_and_errors():
    # tests/tpipeline.nim:215-249: an empty pipeline copies; invalid ops name themselves
    g = np.random.default_rng(1).standard_normal((10, 100)).astype(np.float32)
    plan = O.OraclePlan([], P.F32, 2.0, 100)
    assert np.array_equal(plan.apply(g, np.full(10, 100, np.int32)), g)
    with pytest.raises(ValueError, match=r"^op 1 \(opFilter\): "):
        O.OraclePlan([P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 200, 260))], P.F32, 2.0, 100)
    with pytest.raises(ValueError):
        O.OraclePlan([], P.F32, 2.0, 100, recordSamples=99)
