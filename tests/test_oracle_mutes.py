"""Mutes on the CPU: the curves and builder checks of the host API, and the
oracle's restatement of core/mute.nim pinned by the known answers of the
reference's tests/tmute.nim (top/bottom kernels with exact taper values,
an LMO mute on a gather, the taper limit, the time axis of t0Ms and a
window, a table mute with auxiliary, NaN-offset and short rows, a NaN t0)."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A
from oracle import oracle as O


def near(a, b, tol=1e-6):
    return abs(a - b) <= tol


def test_curves():
    assert P.timeMute(100).muteTimeMs(math.nan) == 100
    lmo = P.lmoMute(velocity=2000, t0Ms=10, padMs=-5)
    assert near(lmo.muteTimeMs(1000), 505) and near(lmo.muteTimeMs(-1000), 505)
    assert math.isnan(lmo.muteTimeMs(math.nan))
    tab = P.tableMute([0.0, 100, 300], [10.0, 50, 250])
    assert tab.kind == P.mkTable
    assert tab.muteTimeMs(0) == 10 and tab.muteTimeMs(100) == 50
    assert near(tab.muteTimeMs(50), 30) and near(tab.muteTimeMs(-200), 150)
    assert tab.muteTimeMs(1000) == 250
    assert P.tableMute([200.0], [80.0]).muteTimeMs(0) == 80
    assert math.isnan(tab.muteTimeMs(math.nan))


def test_validation():
    for bad in (lambda: P.timeMute(math.nan), lambda: P.tableMute([], []),
                lambda: P.tableMute([0.0, 1], [1.0]), lambda: P.tableMute([1.0, 1], [1.0, 2]),
                lambda: P.tableMute([-1.0], [1.0]), lambda: P.tableMute([0.0], [math.inf]),
                lambda: P.lmoMute(0), lambda: P.lmoMute(-1500), lambda: P.lmoMute(1500, padMs=math.nan)):
        with pytest.raises(ValueError):
            bad()
    # the plan refuses a negative or non-finite taper (pipeline.nim:417-421)
    for taper in (-1.0, math.nan):
        with pytest.raises(ValueError, match="taper"):
            O.OraclePlan([P.muteTopOp(P.timeMute(4), taperMs=taper)], A.F32, 2.0, 10)


def mute_rows(op, rows, dtMs=1.0, dtype=np.float64, t0=None, offsets=None, first=0, live=None, status=None):
    """The oracle's apply of [op] on `rows` (2-D) with the given keys."""
    rows = np.array(rows, dtype=dtype)
    r, c = rows.shape
    live = np.full(r, c, np.int32) if live is None else np.asarray(live, np.int32)
    if status is not None:
        live = np.where(np.asarray(status) == A.TS_LIVE, live, 0).astype(np.int32)
    t0 = np.zeros(r) if t0 is None else np.asarray(t0, np.float64)
    offsets = np.zeros(r) if offsets is None else np.asarray(offsets, np.float64)
    plan = O.OraclePlan([op], A.F64 if dtype == np.float64 else A.F32, dtMs, c)
    return plan.apply(rows, live, None, keys=(offsets, t0, first, dtMs))


def top(x, startCol, taperCols):
    return mute_rows(P.muteTopOp(P.timeMute(startCol), taperMs=taperCols), [x])[0]


def bottom(x, endCol, taperCols):
    return mute_rows(P.muteBottomOp(P.timeMute(endCol), taperMs=taperCols), [x])[0]


def test_top_kernel_exact():
    x = top(np.ones(10), 6, 4)
    assert x[0] == 0 and x[1] == 0 and x[2] == 0
    for j in range(3, 6):
        assert near(x[j], math.sin(math.pi / 2 * (j - 2) / 4) ** 2, 1e-12)
    assert np.all(x[6:] == 1)
    assert top(np.ones(5), 2, 0).tolist() == [0, 0, 1, 1, 1]
    f = top(np.ones(5), 2.5, 1)
    assert f[1] == 0 and near(f[2], math.sin(math.pi / 4) ** 2, 1e-12) and f[3] == 1
    assert top(np.ones(4), 99, 3).tolist() == [0, 0, 0, 0]
    assert top(np.ones(4), -10, 3).tolist() == [1, 1, 1, 1]
    nan_row = mute_rows(P.muteTopOp(P.timeMute(2), taperMs=3), [np.ones(4)], t0=[math.nan])[0]
    assert nan_row.tolist() == [1, 1, 1, 1]


def test_bottom_kernel_exact():
    x = bottom(np.ones(10), 3, 4)
    assert np.all(x[:4] == 1)
    for j in range(4, 7):
        assert near(x[j], math.sin(math.pi / 2 * (7 - j) / 4) ** 2, 1e-12)
    assert np.all(x[7:] == 0)
    assert bottom(np.ones(5), 2, 0).tolist() == [1, 1, 1, 0, 0]
    assert bottom(np.ones(4), -1, 0).tolist() == [0, 0, 0, 0]
    assert bottom(np.ones(4), 50, 2).tolist() == [1, 1, 1, 1]


def test_lmo_top_mute_on_a_gather():
    # offsets 0, 400, 800 at 2000 m/s: columns 0, 50, 100 at 4 ms; the 20 ms
    # taper is the 5 columns before each
    g = mute_rows(P.muteTopOp(P.lmoMute(velocity=2000), taperMs=20), np.ones((3, 150)), dtMs=4,
                  dtype=np.float32, offsets=[0.0, 400, 800])
    for r, col in enumerate([0, 50, 100]):
        assert np.all(g[r, :max(col - 5, 0)] == 0)
        for k in range(5):
            if col - 5 + k >= 0:
                assert near(float(g[r, col - 5 + k]), math.sin(math.pi / 2 * k / 5) ** 2)
        assert np.all(g[r, col:] == 1)


def test_taper_limit_is_continuous():
    for L in (0.0, 1e-3):
        assert top(np.ones(6), 3, L).tolist() == [0, 0, 0, 1, 1, 1]
        assert bottom(np.ones(6), 2, L).tolist() == [1, 1, 1, 0, 0, 0]


def test_time_axis_follows_t0_and_the_window():
    g = mute_rows(P.muteTopOp(P.timeMute(140)), np.ones((2, 40)), dtMs=4, t0=[100.0, 0.0])
    assert g[0, 9] == 0 and g[0, 10] == 1
    assert g[1, 34] == 0 and g[1, 35] == 1
    # a window from trace sample 20 (80 ms): 140 ms is its column 15
    w = mute_rows(P.muteTopOp(P.timeMute(140)), np.ones((1, 30)), dtMs=4, first=20)
    assert w[0, 14] == 0 and w[0, 15] == 1
    w = mute_rows(P.muteBottomOp(P.timeMute(180)), w, dtMs=4, first=20)
    assert w[0, 25] == 1 and w[0, 26] == 0


def test_table_bottom_mute_and_liveness():
    x = np.ones((4, 100))
    x[3, 60:] = 7  # a sentinel past the live end
    tab = P.tableMute([100.0, 400], [200.0, 160])  # columns 50 .. 40 at 4 ms
    g = mute_rows(P.muteBottomOp(tab), x, dtMs=4, offsets=[100.0, 200, math.nan, 400],
                  live=[100, 100, 100, 60], status=[A.TS_LIVE, A.TS_AUX, A.TS_LIVE, A.TS_LIVE])
    assert g[0, 50] == 1 and g[0, 51] == 0
    assert g[1, 99] == 1, "auxiliary rows are untouched"
    assert g[2, 99] == 1, "a NaN offset leaves the row alone"
    assert g[3, 40] == 1 and g[3, 41] == 0 and g[3, 59] == 0
    assert np.all(g[3, 60:] == 7), "nothing past the live end is written"
    g = mute_rows(P.muteTopOp(P.timeMute(400)), g, dtMs=4, offsets=[100.0, 200, math.nan, 400],
                  live=[100, 100, 100, 60], status=[A.TS_LIVE, A.TS_AUX, A.TS_LIVE, A.TS_LIVE])
    assert g[3, 60] == 7, "a top mute also stops at the live end"


def test_float64_lmo_and_table():
    x = np.ones((4, 1000))
    for _ in range(2):
        x = mute_rows(P.muteTopOp(P.lmoMute(1800, padMs=-20), taperMs=30), x, dtMs=2,
                      offsets=[0.0, 500, 1000, 1500])
        x = mute_rows(P.muteBottomOp(P.tableMute([0.0, 1500], [1200.0, 1900]), taperMs=40), x, dtMs=2,
                      offsets=[0.0, 500, 1000, 1500])
    assert x[3, 0] == 0 and x[0, 999] == 0
