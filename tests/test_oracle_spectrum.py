"""Spectra on the CPU: the oracle's restatement of fft/spectrum.nim pinned by
the known answers of the reference's tests/tspectrum.nim (window and FFT
lengths, the peak within one bin, amplitudes on a bin whatever the taper and
padding, the phase, DC and demean, the power average over live rows, short
windows, NaN rows left out, a 60 s record at 1 ms), and the host dB and phase
helpers of the product."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A
from oracle import oracle as O


def sinusoid(n, dtMs, f, amp=1.0, phase=0.0):
    return amp * np.sin(2 * math.pi * f * np.arange(n) * dtMs / 1000 + phase)


def one(x, dtMs, win, taper=0.1, nfft=0, demean=True, dtype=np.float64):
    x = np.asarray(x, dtype)[None, :]
    a, p = O.spectrum_amplitudes(x, [x.shape[1]], dtMs, win, 0, taper, nfft, demean)
    return a[0].astype(np.float64), p[0].astype(np.float64)


def bin_hz(nfft, dtMs, k):
    return k * 1000 / (nfft * dtMs)


def test_plan_lengths():
    assert O.spectrum_plan(A.F32, 2.0, 501)[0] == 512
    assert O.spectrum_plan(A.F64, 4.0, 100, nfft=1000)[0] == 1000
    assert O.spectrum_plan(A.F32, 2.0, 512)[0] == 512
    assert O.spectrum_plan(A.F32, 2.0, 1000)[0] == 1024
    assert O.spectrum_plan(A.F32, 1.0, 60001)[0] == 65536
    for bad in (dict(windowLen=0), dict(dtMs=0.0), dict(dtMs=math.inf), dict(taperFraction=0.6),
                dict(nfft=64), dict(nfft=101)):
        kw = dict(dtype=A.F32, dtMs=2.0, windowLen=100)
        kw.update(bad)
        with pytest.raises(ValueError):
            O.spectrum_plan(kw["dtype"], kw["dtMs"], kw["windowLen"], kw.get("taperFraction", 0.1), kw.get("nfft", 0))


def test_peak_within_one_bin():
    for win, nfft, taper in ((501, 0, 0.1), (400, 1024, 0.5), (1000, 0, 0.0), (257, 0, 0.25)):
        n = O.spectrum_plan(A.F64, 2.0, win, taper, nfft)[0]
        for f in (7.3, 25.0, 61.7, 180.2):
            amp, _ = one(sinusoid(win, 2.0, f, 3), 2.0, win, taper, nfft)
            assert abs(bin_hz(n, 2.0, int(np.argmax(amp))) - f) <= bin_hz(n, 2.0, 1)


def test_amplitude_scale_on_a_bin():
    for taper, nfft, b in ((0.0, 1000, 40), (0.1, 0, 40), (0.5, 0, 40), (0.5, 4096, 160)):
        n = O.spectrum_plan(A.F64, 1.0, 1000, taper, nfft)[0]
        f = bin_hz(n, 1.0, b)
        amp, phase = one(sinusoid(1000, 1.0, f, 2.5, 0.3), 1.0, 1000, taper, nfft)
        k = int(np.argmax(amp))
        assert abs(amp[k] - 2.5) <= 0.01
        if taper == 0:
            assert abs(phase[k] - (0.3 - math.pi / 2)) <= 1e-6


def test_dc_and_demean():
    for demean in (True, False):
        amp, _ = one(np.full(200, 4.0), 2.0, 200, 0.0, 0, demean)
        assert abs(amp[0] - (0.0 if demean else 4.0)) <= 1e-9


def test_average_over_live_rows():
    g = np.stack([sinusoid(600, 2.0, 25.0, r + 1) for r in range(6)]).astype(np.float32)
    live = np.full(6, 600, np.int32)
    live[2] = 0  # dead
    live[4] = 0  # failed
    live[5] = 100  # live before the window only
    amp, used = O.spectrum_average(g, live, 2.0, 400, 150, 0.5, 400)
    assert used == 3
    k = int(np.argmax(amp))
    assert k == 20 and abs(amp[k] - math.sqrt(21.0 / 3)) <= 1e-3
    one_row, used = O.spectrum_average(g, live, 2.0, 400, 150, 0.5, 400, rows=(3, 3))
    assert used == 1 and abs(one_row[k] - 4) <= 1e-3
    a32, _ = one(g[3, 150:550], 2.0, 400, 0.5, 400, dtype=np.float32)
    assert np.max(np.abs(a32 - one_row)) <= 1e-4
    none, used = O.spectrum_average(g, live, 2.0, 400, 150, 0.5, 400, rows=(2, 2))
    assert used == 0 and none[k] == 0


def test_nan_rows_are_left_out():
    g = np.stack([sinusoid(400, 2.0, 25.0, 2) for _ in range(4)]).astype(np.float32)
    live = np.full(4, 400, np.int32)
    for bad in (math.nan, math.inf, -math.inf):
        g[2, 10] = bad
        amp, used = O.spectrum_average(g, live, 2.0, 200, 0, 0.1, 200)
        assert used == 3 and np.all(np.isfinite(amp))
        assert abs(amp[int(np.argmax(amp))] - 2) <= 0.02
        assert O.spectrum_average(g, live, 2.0, 200, 200, 0.1, 200)[1] == 4
    x = np.zeros(200, np.float32)
    x[3] = math.nan
    assert math.isnan(one(x, 2.0, 200, 0.1, 200, dtype=np.float32)[0][5])


def test_short_windows_scale_like_full_ones():
    amp, _ = one(sinusoid(300, 1.0, 50, 3), 1.0, 400, 0.2, 400)
    assert int(np.argmax(amp)) == 20 and abs(amp[20] - 3) <= 0.03
    g = np.stack([sinusoid(500, 1.0, 50, 3) for _ in range(11)])
    live = np.array([500 if r % 2 == 0 else 300 + 100 * (r % 3) for r in range(11)], np.int32)
    avg, used = O.spectrum_average(g, live, 1.0, 400, 100, 0.2, 400)
    assert used == 11 and int(np.argmax(avg)) == 20 and abs(avg[20] - 3) <= 0.05


def test_sixty_second_record_at_1_ms():
    n = O.spectrum_plan(A.F32, 1.0, 60001)[0]
    f = bin_hz(n, 1.0, 1000)
    amp, _ = one(sinusoid(60001, 1.0, f, 2), 1.0, 60001, dtype=np.float32)
    assert int(np.argmax(amp)) == 1000 and abs(amp[1000] - 2) <= 2e-3


def test_db_and_phase_helpers():
    db = [0.0] * 4
    P.toDbInto([0.0, 0.01, 0.1, 1.0], db)
    assert db[3] == 0 and abs(db[2] + 20) <= 1e-12 and abs(db[1] + 40) <= 1e-12 and db[0] == -120
    P.toDbInto([math.nan, 1.0, math.inf, 0.1], db)
    assert db[0] == -120 and db[1] == 0 and db[2] == math.inf and abs(db[3] + 20) <= 1e-12
    amp, phase = [0.0, 0.0], [0.0, 0.0]
    P.amplitudePhaseInto([3.0, 0.0], [4.0, -2.0], amp, phase)
    assert amp == [5.0, 2.0] and abs(phase[1] + math.pi / 2) <= 1e-6
    d = [0.0] * 4
    P.unwrapPhaseInto([170.0, -170.0, math.nan, -160.0], [True, True, True, True], d)
    assert d[0] == 170 and d[1] == 190 and math.isnan(d[2]) and d[3] == 200
    m, r = P.circularMeanDeg([170.0, -170.0])
    assert abs(abs(m) - 180) <= 1e-9 and abs(r - math.cos(math.radians(10))) <= 1e-12
    hz = [float(k) for k in range(10)]
    ph = [-360 * 4 / 1000 * f + 5 for f in hz]  # a 4 ms delay
    out = [0.0] * 10
    assert abs(P.removeDelayInto(ph, hz, [True] * 10, out) - 4) <= 1e-9
