"""Vibroseis sweeps (src/processSEG/vibroseis/sweep.nim) through the C ABI:
the reference's own checks (tests/tsweep.nim: instantaneous frequency of
every law against frequencyAt, the dB/octave and dB/Hz spectral slopes, the
Klauder wavelet, phase accuracy against phaseAt, lengths and amplitude,
validation, specs built as objects, steep boosts, whole samples), and every
law's samples against the oracle's restatement, bit for bit in float32 and
float64, with and without harmonics and for shorter and longer buffers.
Host code only: no GPU."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from oracle import oracle as O


def inst_freq(spec):
    """Mean frequency over each sample interval from the analytic phase: the
    sweep at φ₀ = 0 (sine) and at 90° (cosine), without its ramps."""
    from dataclasses import replace
    s = replace(spec, taper=P.noTaper())
    a = s.samples(np.float64)
    b = replace(s, startPhaseDeg=90.0).samples(np.float64)
    d = np.arctan2(a[1:], b[1:]) - np.arctan2(a[:-1], b[:-1])
    d = np.mod(d, 2 * math.pi)
    return d / (2 * math.pi) / (spec.dtMs / 1000)


def check_law(spec, tol):
    f = inst_freq(spec)
    worst = 0.0
    for j in range(f.size):
        a = j * spec.dtMs
        want = (spec.frequencyAt(a) + 4 * spec.frequencyAt(a + 0.5 * spec.dtMs) + spec.frequencyAt(a + spec.dtMs)) / 6
        worst = max(worst, abs(f[j] - want))
    assert worst < tol, (spec.law, worst)


def test_instantaneous_frequency_follows_the_law():
    taper = P.initSweepTaper(200, 200)
    check_law(P.linearSweep(8, 80, 6000, 2, taper), 1e-6)
    check_law(P.linearSweep(90, 6, 6000, 2, taper), 1e-6)
    check_law(P.exponentialSweep(5, 120, 8000, 2, taper), 1e-4)
    check_law(P.dbPerOctaveSweep(6, 100, 8000, 2, 3, taper), 1e-4)
    check_law(P.dbPerOctaveSweep(100, 6, 8000, 2, -4.5, taper), 1e-4)
    check_law(P.dbPerHzSweep(6, 100, 8000, 2, 0.1, taper), 1e-4)
    check_law(P.dbPerHzSweep(6, 100, 8000, 1, -0.2, taper), 1e-4)
    check_law(P.tableSweep([P.SweepPoint(0, 10), P.SweepPoint(1500, 20), P.SweepPoint(4000, 90)], 2), 1e-6)
    d = P.dbPerHzSweep(6, 100, 8000, 2, 0.1)
    assert abs(d.frequencyAt(0) - 6) < 1e-12 and abs(d.frequencyAt(8000) - 100) < 1e-9
    o = P.dbPerOctaveSweep(6, 100, 8000, 2, 3)
    assert abs(o.frequencyAt(0) - 6) < 1e-12 and abs(o.frequencyAt(8000) - 100) < 1e-9
    assert abs(o.frequencyAt(4000) - math.sqrt((36.0 + 10000) / 2)) < 0.05


def test_short_time_spectrum_peak():
    spec = P.dbPerOctaveSweep(8, 100, 10000, 2, 3)
    x = spec.samples()
    win, nfft = 256, 2048
    w = 0.5 - 0.5 * np.cos(2 * math.pi * (np.arange(win) + 0.5) / win)
    for c in range(600, 4401, 400):
        amp = np.abs(np.fft.rfft(x[c - win // 2:c + win // 2] * w, nfft))
        best = int(np.argmax(amp[1:]) + 1)
        assert abs(best * 1000 / (nfft * 2) - spec.frequencyAt(c * 2)) < 1.0, c


def power_spectrum(x, n):
    buf = np.zeros(n)
    buf[:x.size] = x
    z = np.fft.rfft(buf)
    return z.real ** 2 + z.imag ** 2


def band_db(pw, bin_hz, lo, hi):
    f = np.arange(pw.size) * bin_hz
    sel = (f >= lo) & (f <= hi)
    return 10 * math.log10(pw[sel].sum() / sel.sum())


def test_db_per_octave_and_db_per_hz_slopes():
    for boost in (-3.0, 3.0, 6.0):
        spec = P.dbPerOctaveSweep(5, 200, 16000, 1, boost, P.initSweepTaper(50, 50))
        n = 32768
        pw = power_spectrum(spec.samples(), n)
        levels = [band_db(pw, 1000 / n, fc / 2 ** (1 / 6), fc * 2 ** (1 / 6)) for fc in (40.0, 80.0, 160.0)]
        for i in range(1, len(levels)):
            assert abs(levels[i] - levels[i - 1] - boost) < 0.5, (boost, levels)
    spec = P.dbPerHzSweep(5, 125, 16000, 1, 0.1, P.initSweepTaper(300, 300))
    pw = power_spectrum(spec.samples(), 32768)
    a, b = band_db(pw, 1000 / 32768, 25, 35), band_db(pw, 1000 / 32768, 85, 95)
    assert abs((b - a) / 60 - 0.1) < 0.01


def test_klauder_wavelet():
    from dataclasses import replace
    spec = P.linearSweep(10, 60, 4000, 1)
    s = spec.samples()
    c = replace(spec, startPhaseDeg=90.0).samples()

    def corr(a, b, lag):
        return float(np.dot(a[lag:], b[:a.size - lag]))
    r0 = corr(s, s, 0)
    env_prev, null = math.inf, -1
    for lag in range(1, 61):
        r = corr(s, s, lag)
        assert r < r0
        env = math.hypot(r + corr(c, c, lag), corr(s, c, lag) - corr(c, s, lag)) / 2
        if env > env_prev and null < 0:
            null = lag - 1
        env_prev = env
    assert 18 <= null <= 22, null


def test_phase_accuracy():
    lin = P.linearSweep(8, 80, 8000, 2, startPhaseDeg=30)
    x = lin.samples()
    for j in (0, 1, 1000, 2500, 3999):
        assert abs(x[j] - math.sin(lin.phaseAt(j * 2))) < 1e-12
    e = P.exponentialSweep(5, 120, 8000, 2)
    d = P.dbPerOctaveSweep(5, 120, 8000, 2, -20 * math.log10(2.0) / 2)
    xe, xd = e.samples(), d.samples()
    assert np.max(np.abs(xe - xd)) < 1e-9
    pe = np.array([math.sin(e.phaseAt(j * 2)) for j in range(xe.size)])
    assert np.max(np.abs(xe - pe)) < 1e-9
    assert e.segySweepType() == 3 and d.segySweepType() == 3 and lin.segySweepType() == 1
    t = P.tableSweep([P.SweepPoint(0, 8), P.SweepPoint(8000, 80)], 2)
    assert np.max(np.abs(t.samples() - P.linearSweep(8, 80, 8000, 2).samples())) < 1e-9
    assert t.segySweepType() == 4
    assert math.isnan(d.phaseAt(100)) and math.isnan(P.dbPerHzSweep(6, 100, 8000, 2, 0.1).phaseAt(100))
    assert np.max(np.abs(lin.samples(np.float32).astype(np.float64) - x)) < 1e-6


def test_lengths_and_amplitude():
    s = P.linearSweep(8, 80, 8000, 2, amplitude=2.5, taper=P.initSweepTaper(100, 100))
    assert s.sweepLen() == 4000
    x = s.samples(np.float32)
    assert x[0] == 0 and abs(x[-1]) < 2.5 * 0.03
    peak = float(np.max(np.abs(x)))
    assert 2.49 < peak <= 2.5
    assert P.linearSweep(8, 80, 0.3, 0.1).sweepLen() == 3  # 0.3 / 0.1 is 2.9999999999999996
    with pytest.raises(ValueError):
        s.sweepInto(np.zeros(10))
    buf = np.zeros(4000)
    s.sweepInto(buf)
    assert np.array_equal(buf, s.samples())


def test_validation():
    bad = [lambda: P.linearSweep(8, 210, 8000, 2), lambda: P.linearSweep(8, 260, 8000, 2, maxNyquistFraction=1),
           lambda: P.linearSweep(0, 80, 8000, 2), lambda: P.linearSweep(8, 80, 1, 2),
           lambda: P.linearSweep(8, 80, 8000, 0), lambda: P.linearSweep(8, 80, 8001, 2),
           lambda: P.linearSweep(8, 80, 1e12, 2), lambda: P.linearSweep(8, 80, 1e300, 2),
           lambda: P.linearSweep(8, 80, 1000, 2, P.initSweepTaper(600, 500)),
           lambda: P.dbPerHzSweep(8, 80, 8000, 2, 10), lambda: P.dbPerOctaveSweep(8, 80, 8000, 2, math.nan),
           lambda: P.tableSweep([P.SweepPoint(1, 8), P.SweepPoint(8000, 80)], 2),
           lambda: P.tableSweep([P.SweepPoint(0, 8), P.SweepPoint(0, 80)], 2),
           lambda: P.tableSweep([P.SweepPoint(0, 8)], 2)]
    for f in bad:
        with pytest.raises(ValueError):
            f()
    P.linearSweep(8, 240, 8000, 2, maxNyquistFraction=1)
    from dataclasses import replace
    with pytest.raises(ValueError, match="amplitude"):
        replace(P.linearSweep(8, 80, 8000, 2), amplitude=math.nan).validate()
    with pytest.raises(ValueError, match="720"):
        P.dbPerHzSweep(8, 80, 8000, 2, 10)


def test_specs_built_as_objects():
    for spec in [P.SweepSpec(0, 0, 0, 0), P.SweepSpec(10, 80, 4e12, 2), P.SweepSpec(10, 80, math.nan, 2),
                 P.SweepSpec(10, 80, 8000, -2), P.SweepSpec(10, 80, math.inf, 2), P.SweepSpec(10, 80, 1, 2)]:
        assert spec.sweepLen() == 0, spec.lengthMs
        with pytest.raises(ValueError):
            spec.samples(np.float32)
        with pytest.raises(ValueError):
            P.generatePilot(spec)
        with pytest.raises(ValueError):
            spec.sweepInto(np.zeros(4))
    ok = P.SweepSpec(10, 80, 8000, 2)
    assert ok.sweepLen() == 4000 and len(P.generatePilot(ok, np.float32)) == 4000


def test_steep_boosts_stay_finite():
    for f in [lambda: P.dbPerOctaveSweep(10, 100, 8000, 2, 3000), lambda: P.dbPerOctaveSweep(10, 100, 8000, 2, -100),
              lambda: P.dbPerOctaveSweep(100, 10, 8000, 2, 100), lambda: P.dbPerHzSweep(10, 110, 8000, 2, -2),
              lambda: P.dbPerHzSweep(10, 110, 8000, 2, 1.6)]:
        with pytest.raises(ValueError):
            f()
    steep = [P.dbPerOctaveSweep(10, 100, 8000, 2, 90), P.dbPerOctaveSweep(10, 100, 8000, 2, -90),
             P.dbPerOctaveSweep(100, 10, 8000, 2, -90), P.dbPerHzSweep(10, 110, 8000, 2, 1.5),
             P.dbPerHzSweep(10, 110, 8000, 2, -1.5), P.dbPerHzSweep(110, 10, 8000, 2, 1.5),
             P.dbPerOctaveSweep(900, 1800, 2000, 0.25, 290, maxNyquistFraction=1),
             P.dbPerOctaveSweep(900, 1800, 2000, 0.25, -290, maxNyquistFraction=1)]
    for spec in steep:
        assert spec.frequencyAt(0) == spec.f1Hz and spec.frequencyAt(spec.lengthMs) == spec.f2Hz
        lo, hi = min(spec.f1Hz, spec.f2Hz), max(spec.f1Hz, spec.f2Hz)
        last = spec.f1Hz
        for k in range(0, 4001, 7):
            t = spec.lengthMs * (1 - 10.0 ** (-k / 250))
            f = spec.frequencyAt(t)
            assert lo <= f <= hi, (spec.law, spec.boostDb, t, f)
            assert (f - last) * (spec.f2Hz - spec.f1Hz) >= 0
            last = f
        assert np.isfinite(spec.samples()).all()


def test_whole_samples_long_sweep():
    with pytest.raises(ValueError):
        P.linearSweep(5, 10, 1000.5, 1)
    with pytest.raises(ValueError):
        P.linearSweep(5, 10, 600000.5, 1, maxNyquistFraction=1)
    P.linearSweep(5, 10, 600000, 1, maxNyquistFraction=1)
    assert P.linearSweep(5, 10, 1000 * 0.1, 0.1).sweepLen() == 1000
    assert P.linearSweep(5, 10, 60000 * 0.1, 0.1).sweepLen() == 60000


def specs():
    t = P.initSweepTaper(250, 150, P.tpKaiser)
    return [P.linearSweep(8, 80, 4000, 2, t, startPhaseDeg=30, amplitude=2),
            P.linearSweep(90, 6, 3000, 1, P.initSweepTaper(100, 100)),
            P.exponentialSweep(5, 120, 4000, 2, t),
            P.dbPerOctaveSweep(6, 100, 4000, 2, 3, t, startPhaseDeg=-45),
            P.dbPerOctaveSweep(100, 6, 4000, 2, -4.5, t),
            P.dbPerOctaveSweep(5, 120, 4000, 2, -20 * math.log10(2.0) / 2),
            P.dbPerHzSweep(6, 100, 4000, 2, 0.1, t),
            P.dbPerHzSweep(110, 10, 4000, 2, 1.5),
            P.tableSweep([P.SweepPoint(0, 10), P.SweepPoint(1500, 20), P.SweepPoint(2001, 20),
                          P.SweepPoint(4000, 90)], 2, P.initSweepTaper(300, 300, P.tpGaussian, 0.3)),
            P.tableSweep([P.SweepPoint(0, 8), P.SweepPoint(4000, 80)], 2)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_every_law_matches_the_oracle(dtype):
    """Bit for bit: the same float64 phase, rounding of each sample to the
    sample type, and ramps; frequencyAt at and between the sample times."""
    harmonics = [P.SweepHarmonic(1, 1, 0), P.SweepHarmonic(2, 0.3, 45), P.SweepHarmonic(3.5, 0.1, -20),
                 P.SweepHarmonic(9, 0.05, 0)]
    for spec in specs():
        n0 = spec.sweepLen()
        for hs in ((), harmonics):
            for n in (0, n0 // 3, n0 + 777):
                got = spec.samples(dtype, hs, n)
                want = O.sweep_samples(spec, dtype, hs, n)
                assert got.dtype == dtype and np.array_equal(got, want), (spec.law, len(hs), n)
        for t in np.linspace(-10, spec.lengthMs + 10, 97):
            assert spec.frequencyAt(t) == O.sweep_frequency_at(spec, t), (spec.law, t)


def test_harmonics():
    """sweep.nim:375-420: an empty list or the fundamental alone is the
    sweep; a harmonic at or above Nyquist is cut from those samples; a
    longer buffer ends in zeros; bad harmonics are refused."""
    spec = P.linearSweep(8, 100, 4000, 2, P.initSweepTaper(200, 200))
    x = spec.samples()
    assert np.array_equal(P.sweepHarmonics(spec, np.float64, [P.SweepHarmonic()]), x)
    y = P.sweepHarmonics(spec, np.float64, [], samples=x.size + 500)
    assert np.array_equal(y[:x.size], x) and not y[x.size:].any()
    # the 3rd harmonic of a 100 Hz end at 2 ms (Nyquist 250 Hz) leaves once f ≥ 83.3 Hz
    z = P.sweepHarmonics(spec, np.float64, [P.SweepHarmonic(1, 1, 0), P.SweepHarmonic(3, 0.5, 0)])
    f = np.array([spec.frequencyAt(j * 2) for j in range(x.size)])
    cut = 3 * f >= 250
    assert cut.any() and (~cut).any()
    assert np.array_equal(z[cut], x[cut]) and not np.array_equal(z[~cut], x[~cut])
    for h in (P.SweepHarmonic(0, 1, 0), P.SweepHarmonic(math.inf, 1, 0), P.SweepHarmonic(2, math.nan, 0),
              P.SweepHarmonic(2, 1, math.inf)):
        with pytest.raises(ValueError):
            P.sweepHarmonics(spec, np.float64, [h])
