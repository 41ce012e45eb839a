"""Pilots (src/processSEG/vibroseis/pilot.nim): the reference's own checks
(tests/tpilot.nim: generated, validation, sweep_overrides, the sweep fields
of other types and of headers that do not fit the trace,
from_row_window_and_t0). Host code only: no GPU."""
import math

import numpy as np
import pytest

import processseg_b200 as P


def test_generated():
    spec = P.linearSweep(8, 80, 8000, 2, P.initSweepTaper(250, 300, P.tpLinear))
    p = P.generatePilot(spec, np.float32)
    assert len(p) == 4000 and p.dtMs == 2 and p.t0Ms == 0 and p.lengthMs == 8000
    assert p.sweep is not None and p.sweep.f1Hz == 8
    assert np.array_equal(p.samples, spec.samples(np.float32))
    p.validate()


def test_validation():
    for args, kw in [(([1.0], 2), {}), (([0.0, 0.0, 0.0], 2), {}), (([1.0, math.nan], 2), {}),
                     (([1.0, 1.0], 0), {}), (([1.0, 1.0], 2), {"t0Ms": math.nan}),
                     (([1.0, 1.0], 1), {"sweep": P.linearSweep(8, 80, 100, 2)})]:
        with pytest.raises(ValueError):
            P.initPilot(*args, **kw)
    assert P.initPilot([1.0, -1.0], 2, 0.6).t0Ms == 0.6


def test_sweep_overrides():
    spec = P.linearSweep(8, 80, 12000, 2, P.initSweepTaper(250, 500, P.tpCos2))
    o = P.sweepOverrides(spec)
    assert len(o) == 7 and o[0][0] == "trace.sweepFreqStart"
    assert [v for _, v in o] == [8, 80, 12000, 1, 250, 500, 2]
    assert P.sweepOverrides(spec, binary=True)[3][0] == "binary.sweepType"
    for s in [P.linearSweep(8, 80, 40000, 2), P.linearSweep(7.5, 80, 12000, 2), P.linearSweep(8, 79.6, 12000, 2),
              P.linearSweep(8, 80, 12000.5, 0.5, maxNyquistFraction=0.1),
              P.linearSweep(8, 80, 12000, 2, P.initSweepTaper(250.5, 0))]:
        with pytest.raises(ValueError):
            P.sweepOverrides(s)
    assert P.sweepOverrides(P.exponentialSweep(8, 80, 12000, 2))[3][1] == 3
    assert P.sweepOverrides(P.dbPerHzSweep(8, 80, 12000, 2, 0.1))[3][1] == 4


def test_sweep_from_headers():
    assert P.sweepFromHeaders(8, 80, 8000, 4, 0, 0, 1, 2) is None
    assert P.sweepFromHeaders(8, 80, 8000, 3, 0, 0, 3, 2).law == P.slExponential
    s = P.sweepFromHeaders(6, 90, 6000, 1, 200, 400, 1, 2)
    assert s.law == P.slLinear and s.f1Hz == 6 and s.f2Hz == 90 and s.lengthMs == 6000
    assert s.taper.startMs == 200 and s.taper.endMs == 400 and s.taper.shape == P.tpLinear
    assert s.maxNyquistFraction == 1
    assert P.sweepFromHeaders(80, 1100, 12000, 1, 500, 300, 5, 1) is None  # above Nyquist
    assert P.sweepFromHeaders(8, 110, 12000, 1, 500, 300, 5, 1) is not None
    assert P.sweepFromHeaders(8, 110, 12000, 1, 500, 300, 5, 1, samples=12001) is not None
    assert P.sweepFromHeaders(8, 110, 12000, 1, 500, 300, 5, 1, samples=16001) is not None
    assert P.sweepFromHeaders(8, 110, 12000, 1, 500, 300, 5, 1, samples=6001) is None
    assert P.sweepFromHeaders(8, 110, 12000, 1, 9000, 9000, 1, 1) is None  # ramps overlap
    assert P.sweepFromHeaders(8, 110, 12000.5, 1, 0, 0, 1, 1) is None  # not whole samples
    assert P.sweepFromHeaders(8, 110, 12000, 1, 0, 0, 1, math.nan) is None
    # a round trip through the fields
    spec = P.linearSweep(6, 90, 6000, 2, P.initSweepTaper(200, 400, P.tpLinear))
    f = dict(P.sweepOverrides(spec))
    back = P.sweepFromHeaders(f["trace.sweepFreqStart"], f["trace.sweepFreqEnd"], f["trace.sweepLength"],
                              f["trace.sweepType"], f["trace.sweepTaperStart"], f["trace.sweepTaperEnd"],
                              f["trace.taperType"], 2)
    assert np.array_equal(back.samples(np.float32), spec.samples(np.float32))


def test_from_row_window_and_t0():
    data = np.zeros((1, 8))
    data[0, :6] = np.arange(1, 7)
    meta = P.initChunkMeta(np.full(1, P.tsLive, np.int32), np.array([6], np.int32), 2.0,
                           np.array([-1.5]), 1)
    p = P.pilotFromRow(meta, data, 0)
    # column 0 is trace sample 1: t0 = −1.5 + 2; the live length is 6 − 1
    assert p.t0Ms == 0.5 and len(p) == 5 and p.sweep is None
    assert np.array_equal(p.samples, [1, 2, 3, 4, 5])
    assert P.pilotFromRow(meta, data, 0, t0Ms=3).t0Ms == 3
    with pytest.raises(ValueError):
        P.pilotFromRow(meta, data, 1)
    failed = P.initChunkMeta(np.full(2, P.tsLive, np.int32), np.array([6, 6], np.int32), 2.0,
                             np.zeros(2), 0, [1])
    with pytest.raises(ValueError, match="decoded"):
        P.pilotFromRow(failed, np.ones((2, 8)), 1)
    # an auxiliary row is a pilot too
    aux = P.initChunkMeta(np.array([P.tsAux], np.int32), np.array([8], np.int32), 2.0, np.zeros(1))
    assert len(P.pilotFromRow(aux, np.ones((1, 8)), 0)) == 8
