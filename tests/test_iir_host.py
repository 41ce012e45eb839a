"""IIR filters on the CPU: the host design in libpsgcuda.so (order, margin,
magnitude) and the oracle's restatement of filter/iir.nim, both pinned by
the known answers of the reference's tests/tiir.nim (corners at −6 dB zero
phase and −3 dB minimum phase, zero-phase gain equal to the spec's
response, validation), and the oracle's apply by that file's properties
(the impulse response's spectrum, causality and symmetry, the steady-state
start against a DC and a drift, an exactly zero decay, zoom windows)."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A
from oracle import oracle as O

DT = 2.0


def db(g):
    return 20 * math.log10(g)


def test_design_and_corners():
    lp = P.initIirPlan(P.float64, P.butterHighCut(60, 24), DT, 100)
    assert lp.order == 2 and lp.phase == P.ipZero
    assert abs(db(lp.magnitudeAt(60)) - db(0.5)) <= 1e-9
    mp = P.initIirPlan(P.float64, P.butterHighCut(60, 24), DT, 100, phase=P.ipMinimum)
    assert mp.order == 4
    assert abs(db(mp.magnitudeAt(60)) + 3.0103) <= 1e-4
    assert abs(mp.magnitudeAt(0) - 1) <= 1e-12 and mp.magnitudeAt(250) < 1e-12
    odd = P.initIirPlan(P.float64, P.butterLowCut(4, 18), DT, 100, phase=P.ipMinimum)
    assert odd.order == 3 and abs(db(odd.magnitudeAt(4)) + 3.0103) <= 1e-4
    assert odd.magnitudeAt(0) < 1e-12 and abs(odd.magnitudeAt(250) - 1) <= 1e-12
    spec = P.butterBandPass(4, 60, 24, 48)
    bp = P.initIirPlan(P.float64, spec, DT, 100)
    assert bp.order == 6
    for f in (0.5, 2.0, 4.0, 10.0, 30.0, 60.0, 90.0, 200.0):
        assert abs(bp.magnitudeAt(f) - spec.response(f, DT)) <= 1e-9, f
    # the oracle's design agrees
    for s, ph in ((P.butterHighCut(60, 24), P.ipZero), (P.butterHighCut(60, 24), P.ipMinimum),
                  (P.butterLowCut(4, 18), P.ipMinimum), (spec, P.ipZero)):
        o, pad, g, mag = O.iir_info(s, DT, 100, ph, A.TR_LINEAR, [4.0, 60.0, 100.0])
        mine = P.initIirPlan(P.float64, s, DT, 100, phase=ph)
        assert (o, pad) == (mine.order, mine.requiredMargin)
        assert np.allclose(mag, mine.magnitudeAt([4.0, 60.0, 100.0]), rtol=1e-13, atol=1e-15)


def test_validation():
    bad = [(P.lowCut(1, 2), P.ipZero, 100), (P.butterLowCut(4).withNotch(50, 2), P.ipZero, 100),
           (P.butterLowCut(4).withZeroDc(), P.ipZero, 100), (P.butterLowCut(4, 18), P.ipZero, 100),
           (P.butterLowCut(4, 20), P.ipMinimum, 100), (P.butterLowCut(4), P.ipZero, 0)]
    for s, ph, n in bad:
        with pytest.raises(ValueError):
            P.initIirPlan(P.float64, s, DT, n, phase=ph)
        with pytest.raises(ValueError):
            O.iir_info(s, DT, n, ph)
    with pytest.raises(ValueError):
        P.butterHighCut(300)  # no Nyquist check at build time in Python; the plan checks it
        P.initIirPlan(P.float64, P.butterHighCut(300), DT, 100)


def test_margins_match_oracle_and_pipeline():
    for s in (P.butterBandPass(4, 60, 24), P.butterLowCut(2, 24), P.butterLowCut(2, 48), P.butterHighCut(80, 48),
              P.butterBandPass(8, 100, 48, 24), P.butterLowCut(3, 18)):
        for ph in (P.ipZero, P.ipMinimum):
            for dt in (1.0, 2.0, 4.0):
                try:
                    want = O.iir_info(s, dt, 1, ph)[1]
                except ValueError:
                    with pytest.raises(ValueError):
                        P.initIirPlan(P.float64, s, dt, 1, phase=ph)
                    continue
                assert P.initIirPlan(P.float64, s, dt, 1, phase=ph).requiredMargin == want
                flow = P.initPipeline([P.iirOp(s, ph), P.agcOp(500)])
                assert flow.requiredMargin(dt) == want + math.floor(500 / (2 * dt) + 0.5)


def spike(n, at):
    x = np.zeros(n)
    x[at] = 1
    return x


def test_oracle_impulse_response_matches_the_response():
    ns = 4000
    df = 1000 / (ns * DT)
    f = np.arange(ns // 2 + 1) * df
    for s in (P.butterBandPass(4, 60, 24), P.butterLowCut(2, 24), P.butterHighCut(80, 48),
              P.butterBandPass(8, 100, 48, 24)):
        h = O.iir_apply(s, DT, spike(ns, ns // 2), P.ipZero, A.TR_NONE)
        mag = np.abs(np.fft.rfft(h))
        want = np.array([s.response(v, DT) for v in f])
        assert np.max(np.abs(mag - want)) < 1e-4
    for s, s2 in ((P.butterBandPass(4, 60, 24), P.butterBandPass(4, 60, 48)),
                  (P.butterLowCut(3, 18), P.butterLowCut(3, 36))):
        m = P.initIirPlan(P.float64, s, DT, ns, phase=P.ipMinimum).requiredMargin
        h = O.iir_apply(s, DT, spike(ns, m + 1), P.ipMinimum, A.TR_NONE)
        mag = np.abs(np.fft.rfft(h))
        assert np.max(np.abs(mag - np.sqrt([s2.response(v, DT) for v in f]))) < 1e-4


def test_oracle_causal_and_symmetric():
    x = spike(2001, 1000)
    s = P.butterBandPass(4, 60, 24)
    m = O.iir_apply(s, DT, x, P.ipMinimum, A.TR_NONE)
    assert np.max(np.abs(m[:1000])) == 0 and m[1000] > 0
    z = O.iir_apply(s, DT, x, P.ipZero, A.TR_NONE)
    assert np.max(np.abs(z[1001:2001] - z[999::-1][:1000])) < 1e-12


def ricker(n, t_ms, f, amp=1.0):
    t = (np.arange(n) * DT - t_ms) / 1000
    a = (math.pi * f * t) ** 2
    return amp * (1 - 2 * a) * np.exp(-a)


def test_oracle_steady_state_start():
    c = ricker(2001, 900, 25) + ricker(2001, 2400, 15, -0.6)
    t = np.arange(2001) * DT / 1000
    for ph in (P.ipZero, P.ipMinimum):
        for tr in (A.TR_NONE, A.TR_MEAN, A.TR_LINEAR):
            s = P.butterLowCut(2, 24)
            ref = O.iir_apply(s, DT, c, ph, tr)
            assert np.max(np.abs(O.iir_apply(s, DT, c + 1000, ph, tr) - ref)[:200]) < 1e-6
            d = np.max(np.abs(O.iir_apply(s, DT, c + 5 + 20 * t, ph, tr) - ref)[:200])
            if tr == A.TR_LINEAR:
                assert d < 1e-9
            elif ph == P.ipZero:
                assert d < 0.05


def test_oracle_decay_is_exactly_zero():
    for ph in (P.ipZero, P.ipMinimum):
        y = O.iir_apply(P.butterHighCut(100, 24), 0.25, spike(40000, 10), ph, A.TR_NONE)
        assert y[30000] == 0 and y[-1] == 0
        assert np.count_nonzero((y != 0) & (np.abs(y) < 2.2250738585072014e-308)) < 600
