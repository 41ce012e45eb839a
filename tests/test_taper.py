"""Sweep-end tapers (src/processSEG/vibroseis/taper.nim) through the C ABI:
the reference's own checks (tests/ttaper.nim:10-101: closed forms, slopes at
the top, monotonic rise, lengths in ms, no-op lengths, the overlap refusal,
bad arguments, SEG-Y codes, a taper built as an object taking its shape's
default), and every shape's sweep against the oracle, bit for bit in float32
and float64. Host code only: no GPU."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from oracle import oracle as O


def close(a, b, tol=1e-12):
    return abs(a - b) <= tol


def test_closed_forms():
    half = [(P.tpLinear, 0.0, 0.5), (P.tpCosine, 0.0, math.sin(math.pi / 4)), (P.tpCos2, 0.0, 0.5),
            (P.tpHamming, 0.08, 0.54), (P.tpBlackman, 0.0, 0.42 - 0.08),
            (P.tpBlackmanHarris, 0.35875 - 0.48829 + 0.14128 - 0.01168, 0.35875 - 0.14128)]
    for shape, w0, wh in half:
        assert close(P.taperWeight(shape, 0), w0), shape
        assert close(P.taperWeight(shape, 0.5), wh), shape
        assert close(P.taperWeight(shape, 1), 1), shape
    # Kaiser: I0(β·√(1 − (1 − x)²)) / I0(β); I0(6) = 67.23440697647797
    assert close(P.taperWeight(P.tpKaiser, 0, 6), 1 / 67.23440697647797, 1e-13)
    assert close(P.taperWeight(P.tpKaiser, 1, 6), 1)
    assert close(P.taperWeight(P.tpGaussian, 0, 0.5), math.exp(-2.0))
    assert close(P.taperWeight(P.tpGaussian, 0.5, 0.5), math.exp(-0.5))
    assert close(P.taperWeight(P.tpPower, 0.5, 3), 0.125)
    assert close(P.taperWeight(P.tpPower, 0.5), 0.25)  # default p = 2
    # NaN takes the default everywhere: β = 6, σ = 0.4
    assert P.taperWeight(P.tpKaiser, 0.3) == P.taperWeight(P.tpKaiser, 0.3, 6.0)
    assert P.taperWeight(P.tpGaussian, 0.3) == P.taperWeight(P.tpGaussian, 0.3, 0.4)
    # clamped to [0, 1]
    assert P.taperWeight(P.tpLinear, -2) == 0 and P.taperWeight(P.tpLinear, 3) == 1
    h = 1e-6
    for shape in (P.tpCos2, P.tpHamming, P.tpBlackman, P.tpBlackmanHarris, P.tpKaiser, P.tpGaussian):
        d = (P.taperWeight(shape, 1) - P.taperWeight(shape, 1 - h)) / h
        assert abs(d) < 1e-4, (shape, d)
    assert close((P.taperWeight(P.tpLinear, 1) - P.taperWeight(P.tpLinear, 1 - h)) / h, 1, 1e-6)
    assert close((P.taperWeight(P.tpCosine, h) - P.taperWeight(P.tpCosine, 0)) / h, math.pi / 2, 1e-5)
    for shape in range(9):
        prev = -1.0
        for i in range(101):
            w = P.taperWeight(shape, i / 100)
            assert w >= prev - 1e-15, shape
            prev = w


def test_weights_match_the_oracle():
    xs = np.linspace(-0.1, 1.1, 241)
    for shape in range(9):
        for param in (math.nan, 0.7, 3.0, 12.5):
            if shape == P.tpKaiser and param == 0.7:
                param = 0.0  # β = 0: no taper at all
            for x in xs:
                assert P.taperWeight(shape, x, param) == O.taper_weight(shape, x, param), (shape, param, x)
    with pytest.raises(ValueError):
        P.taperWeight(9, 0.5)


def test_apply_lengths_in_ms():
    x = np.ones(100)  # 200 ms at 2 ms: the last sample is at 198 ms
    P.applyTaper(x, 2, P.initSweepTaper(20, 40, P.tpLinear))
    assert x[0] == 0 and close(x[5], 0.5) and x[10] == 1
    assert close(x[99], 0.05) and close(x[90], 0.5) and x[80] == 1
    y = np.ones(11, np.float32)  # 5 ms at 2 ms: not a whole number of samples
    P.applyTaper(y, 2, P.initSweepTaper(5, math.nan, P.tpCos2))
    assert y[0] == 0 and close(y[1], 0.5 - 0.5 * math.cos(math.pi * 0.4), 1e-7)
    assert close(y[2], 0.5 - 0.5 * math.cos(math.pi * 0.8), 1e-7) and y[3] == 1 and y[10] == 1
    # float32: each product rounds to float32, as T(float64(x)·w)
    z = np.full(11, 0.1, np.float32)
    P.applyTaper(z, 2, P.initSweepTaper(5, 5, P.tpKaiser))
    want = np.full(11, 0.1, np.float32)
    for j in range(3):
        want[j] = np.float32(float(want[j]) * O.taper_weight(P.tpKaiser, j * 2 / 5))
    for j in range(10, 7, -1):
        want[j] = np.float32(float(want[j]) * O.taper_weight(P.tpKaiser, (22 - j * 2) / 5))
    assert np.array_equal(z, want), (z, want)


def test_zero_and_nan_lengths_are_no_ops():
    x = np.array([1.0, 2.0, 3.0, 4.0])
    P.applyTaper(x, 1, P.initSweepTaper(0, math.nan))
    assert list(x) == [1, 2, 3, 4]
    P.applyTaper(x, 1, P.noTaper())
    assert list(x) == [1, 2, 3, 4]


def test_overlap_is_refused_meeting_is_not():
    x = np.ones(10)  # 10 ms at 1 ms
    with pytest.raises(ValueError, match="overlap"):
        P.applyTaper(x, 1, P.initSweepTaper(6, 5))
    assert (x == 1).all()  # nothing written
    P.applyTaper(x, 1, P.initSweepTaper(5, 5, P.tpLinear))
    assert x[5] == 1 and x[0] == 0 and close(x[9], 0.2) and close(x[4], 0.8)


def test_bad_arguments():
    for args in [(-1, 0), (math.inf, 0), (1, 1, P.tpGaussian, 0), (1, 1, P.tpKaiser, -1),
                 (1, 1, P.tpKaiser, 51), (1, 1, P.tpPower, 0), (1, 1, P.tpPower, math.inf)]:
        with pytest.raises(ValueError):
            P.initSweepTaper(*args)
    with pytest.raises(ValueError):
        P.applyTaper(np.ones(2), 0, P.noTaper())
    # the C side validates a taper given as an object, as applyTaper does
    with pytest.raises(ValueError, match="Gaussian"):
        P.applyTaper(np.ones(20), 1, P.SweepTaper(2, 2, P.tpGaussian, -1.0))


def test_segy_codes():
    assert P.segyTaperType(P.tpLinear) == 1 and P.segyTaperType(P.tpCos2) == 2
    for s in (P.tpCosine, P.tpHamming, P.tpBlackman, P.tpBlackmanHarris, P.tpKaiser, P.tpGaussian, P.tpPower):
        assert P.segyTaperType(s) == 3
    assert P.initSweepTaper(500, 250, P.tpKaiser).param == 6 and P.initSweepTaper(500, 250, P.tpKaiser).segyTaperType() == 3


def test_a_taper_built_as_an_object_takes_its_shape_default():
    for shape in (P.tpKaiser, P.tpGaussian, P.tpPower):
        built = P.SweepTaper(4, 4, shape)
        assert math.isnan(built.param)
        built.validate()
        x, y = np.ones(21), np.ones(21)
        P.applyTaper(x, 1, built)
        P.applyTaper(y, 1, P.initSweepTaper(4, 4, shape))
        assert np.array_equal(x, y) and x[1] < 0.9 and x[10] == 1, (shape, x[:5])
    assert math.isnan(P.SweepTaper().param) and math.isnan(P.noTaper().param)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_every_shape_in_a_sweep_matches_the_oracle(dtype):
    """A 4 s 8→80 Hz sweep at 2 ms with 300/200 ms ramps of each shape (and a
    non-default parameter), bit for bit: phase in float64, each sample
    rounded to the sample type, then each tapered product rounded again."""
    for shape in range(9):
        for param in (math.nan, 2.5):
            if shape < P.tpKaiser and not math.isnan(param):
                continue
            t = P.initSweepTaper(300, 200, shape, param)
            got = P.linearSweep(8, 80, 4000, 2, t, startPhaseDeg=30).samples(dtype)
            want = O.linear_sweep(8, 80, 4000, 2, 300, 200, shape, 30.0, 1.0, dtype, param=t.param)
            assert got.dtype == dtype and np.array_equal(got, want), (shape, param)
    with pytest.raises(ValueError, match="overlap"):
        P.linearSweep(8, 80, 400, 2, P.initSweepTaper(300, 200))
