"""Spectra on the device (psg_spectrum_average / psg_spectrum_amplitude
through SpectrumPlan) against the oracle and the reference's known answers
(tests/tspectrum.nim): per-row amplitude within 1e-5 (float32) or 1e-12
(float64) of the row's peak, the power average likewise of its peak; even
and odd FFT lengths, short windows, dead and NaN rows, a window offset, and
a 60 s record whose transform runs in global memory."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A
from processseg_b200 import synth
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


def sinusoid(n, dtMs, f, amp=1.0, phase=0.0):
    return amp * np.sin(2 * math.pi * f * np.arange(n) * dtMs / 1000 + phase)


def meta_of(live, dtMs):
    live = np.asarray(live, np.int32)
    return P.initChunkMeta(np.where(live > 0, A.TS_LIVE, A.TS_DEAD).astype(np.int32), live, dtMs)


@pytest.mark.parametrize("T,npdt,tol", [(P.float32, np.float32, 1e-5), (P.float64, np.float64, 1e-12)])
@pytest.mark.parametrize("win,nfft,taper,first", [(501, 0, 0.1, 0), (400, 400, 0.5, 37), (300, 375, 0.25, 11),
                                                  (1, 0, 0.1, 5), (1000, 0, 0.0, 0), (257, 1024, 0.2, 100)])
def test_device_matches_oracle(T, npdt, tol, win, nfft, taper, first):
    g = synth.shot_gather(37, 1200, 2.0, 51, npdt, live_range=(300, 1200), sine_hz=50.0, workload="spectrum")
    g.status[[4]] = P.tsDead
    g.data[9, first + 3] = np.nan
    meta = g.meta()
    live = meta.flat(1200)[0]
    sp = P.initSpectrumPlan(T, 2.0, win, taper, nfft)
    ws = P.initWorkspace()
    amp = np.zeros(sp.bins)
    used = sp.averageAmplitudeInto(g.data, meta, first, amp, ws)
    want, wused = O.spectrum_average(g.data, live, 2.0, win, first, taper, nfft)
    assert used == wused
    assert np.max(np.abs(amp - want)) <= tol * max(np.max(want), 1e-300)
    # the same call again gives the same bits (sums in a fixed order)
    amp2 = np.zeros(sp.bins)
    sp.averageAmplitudeInto(g.data, meta, first, amp2, ws)
    assert np.array_equal(amp, amp2)
    a, p = sp.amplitudes(g.data, meta, first, ws)
    a, p = a.cpu().numpy(), p.cpu().numpy()
    wa, wp = O.spectrum_amplitudes(g.data, live, 2.0, win, first, taper, nfft)
    for r in range(g.data.shape[0]):
        if not np.all(np.isfinite(wa[r])):
            assert np.array_equal(np.isnan(a[r]), np.isnan(wa[r]))
            continue
        peak = float(np.max(np.abs(wa[r])))
        assert np.max(np.abs(a[r].astype(np.float64) - wa[r])) <= tol * max(peak, 1e-30), r
        big = wa[r] > 1e-3 * peak  # the phase where the bin has amplitude
        d = np.angle(np.exp(1j * (p[r][big].astype(np.float64) - wp[r][big])))
        assert np.max(np.abs(d), initial=0) <= (1e-3 if T == P.float32 else 1e-9), r


def test_reference_known_answers_on_the_device():
    ws = P.initWorkspace()
    # amplitude on a bin whatever the taper and padding, and the boxcar phase
    for taper, nfft, b in ((0.0, 1000, 40), (0.1, 0, 40), (0.5, 0, 40), (0.5, 4096, 160)):
        sp = P.initSpectrumPlan(P.float64, 1.0, 1000, taper, nfft)
        amp, phase = np.zeros(sp.bins), np.zeros(sp.bins)
        sp.amplitudeInto(sinusoid(1000, 1.0, sp.binHz(b), 2.5, 0.3), amp, phase, ws)
        k = int(np.argmax(amp))
        assert abs(amp[k] - 2.5) <= 0.01
        if taper == 0:
            assert abs(phase[k] - (0.3 - math.pi / 2)) <= 1e-6
    # the power average over live rows: amplitudes 1, 2, 4 → sqrt(21/3)
    g = np.stack([sinusoid(600, 2.0, 25.0, r + 1) for r in range(6)]).astype(np.float32)
    live = np.full(6, 600)
    live[2] = live[4] = 0
    live[5] = 100
    sp = P.initSpectrumPlan(P.float32, 2.0, 400, 0.5, 400)
    amp = np.zeros(sp.bins)
    before = g.copy()
    assert sp.averageAmplitudeInto(g, meta_of(live, 2.0), 150, amp, ws) == 3
    assert np.array_equal(g, before)
    assert int(np.argmax(amp)) == 20 and abs(amp[20] - math.sqrt(21.0 / 3)) <= 1e-3
    assert sp.averageAmplitudeInto(g, meta_of(live, 2.0), 150, amp, ws, rows=(3, 3)) == 1
    assert abs(amp[20] - 4) <= 1e-3
    assert sp.averageAmplitudeInto(g, meta_of(live, 2.0), 150, amp, ws, rows=(2, 2)) == 0 and amp[20] == 0
    with pytest.raises(ValueError):
        sp.averageAmplitudeInto(g, meta_of(live, 2.0), -1, amp, ws)
    with pytest.raises(AssertionError):
        sp.averageAmplitudeInto(g, meta_of(live, 2.0), 0, amp[:4], ws)
    with pytest.raises(ValueError):
        sp.averageAmplitudeInto(g, meta_of(live, 4.0), 0, amp, ws)
    # 60 s at 1 ms: nfft 65536, the transform in global memory
    sp = P.initSpectrumPlan(P.float32, 1.0, 60001)
    assert sp.nfft == 65536 and sp.bins == 32769
    row = sinusoid(60001, 1.0, sp.binHz(3000), 1.5).astype(np.float32)
    g = np.stack([row] * 10)
    avg = np.zeros(sp.bins)
    assert sp.averageAmplitudeInto(g, meta_of(np.full(10, 60001), 1.0), 0, avg, ws) == 10
    assert int(np.argmax(avg)) == 3000 and abs(avg[3000] - 1.5) <= 2e-3
    want, _ = O.spectrum_average(g, np.full(10, 60001, np.int32), 1.0, 60001, 0)
    assert np.max(np.abs(avg - want)) <= 1e-5 * np.max(want)
