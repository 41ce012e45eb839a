"""traceStatsInto and panelStats (gain/stats.nim:186-304) on the device against
the oracle's restatement: float32 and float64 blocks with dead, auxiliary and
failed rows, rows holding NaN or Inf, a live row whose live window is empty
(a zoom window past a short trace: (0, 0) as statsOf gives, counted among the
panel's rows), a row range, and the percentile forms (NaN, 100, 99)."""
import math

import numpy as np
import pytest

import processseg_b200 as P
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


def block_and_meta(dt, rows=300, cols=1001, first=0, seed=5):
    rng = np.random.default_rng(seed)
    data = (rng.standard_normal((rows, cols)) * rng.uniform(0.01, 100, (rows, 1))).astype(dt)
    status = np.full(rows, P.tsLive, np.int32)
    status[3] = P.tsDead
    status[4] = P.tsAux
    status[9] = P.tsUnknown
    ns = rng.integers(1, cols + first + 1, rows).astype(np.int32)
    ns[10] = first  # live, but its live window is empty
    ns[11] = max(first - 5, 0)
    data[12, 7] = np.nan
    ns[12] = max(ns[12], first + 8)
    data[13, 0] = -np.inf
    ns[13] = max(ns[13], first + 1)
    meta = P.initChunkMeta(status, ns, 2.0, np.zeros(rows), first, failed=[20, 21])
    return data, meta


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_trace_stats_match_oracle(dt):
    data, meta = block_and_meta(dt, first=37)
    live3, _ = meta.flat(data.shape[1], 3)
    assert live3[3] == -1 and live3[20] == -1 and live3[10] == 0 and live3[11] == 0
    want_rms, want_mx = O.trace_stats(data, live3)
    got = P.traceStatsInto(torch.from_numpy(data).cuda(), meta)
    assert len(got) == data.shape[0]
    for r, s in enumerate(got):
        for g, w in ((s.rms, want_rms[r]), (s.maxAbs, want_mx[r])):
            if g == w:
                continue
            if math.isnan(w):
                assert math.isnan(g), (r, g, w)
            else:
                assert abs(g - w) <= 1e-12 * max(abs(w), 1e-300), (r, g, w)
    # not live: NaN; live with no samples: (0, 0), as statsOf
    assert math.isnan(got[3].rms) and math.isnan(got[20].maxAbs)
    assert got[10].rms == 0 and got[10].maxAbs == 0
    assert math.isnan(got[12].rms) and got[13].maxAbs == math.inf
    # the list form fills a caller's list, and checks its length
    out = [None] * data.shape[0]
    assert P.traceStatsInto(data, meta, out) is out
    with pytest.raises(ValueError):
        P.traceStatsInto(data, meta, [None] * 3)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("clip", [99.0, math.nan, 100.0, 0.0, 63.0])
def test_panel_stats_match_oracle(dt, clip):
    data, meta = block_and_meta(dt, first=11, seed=8)
    live3, _ = meta.flat(data.shape[1], 3)
    want = O.panel_stats(data, live3, clip, signed=True)
    got = P.panelStats(torch.from_numpy(data).cuda(), meta, clipPercentile=clip)
    assert got.rows == want["rows"] and got.samples == want["samples"]
    for g, w in ((got.rms, want["rms"]), (got.maxAbs, want["maxAbs"]), (got.clip, want["clip"])):
        if g == w:
            continue
        if math.isnan(w):
            assert math.isnan(g)
        else:
            assert abs(g - w) <= 1e-12 * max(abs(w), 1e-300), (g, w)
    # the empty live rows count among the rows the panel used
    n_empty = int(np.sum(live3 == 0))
    assert n_empty >= 1
    usable = [r for r in range(data.shape[0]) if live3[r] >= 0 and r not in (12, 13)]
    assert got.rows == len(usable)


def test_panel_stats_row_range_and_errors():
    data, meta = block_and_meta(np.float32, seed=2)
    live3, _ = meta.flat(data.shape[1], 3)
    sub = live3.copy()
    sub[:50] = -1
    sub[200:] = -1
    want = O.panel_stats(data, sub, 99.0, signed=True)
    got = P.panelStats(data, meta, clipPercentile=99.0, rows=range(50, 200))
    assert (got.rows, got.samples) == (want["rows"], want["samples"])
    assert abs(got.rms - want["rms"]) <= 1e-12 * want["rms"]
    assert abs(got.clip - want["clip"]) <= 1e-12 * want["clip"]
    empty = P.panelStats(data, meta, rows=range(400, 500))
    assert empty.rows == 0 and empty.samples == 0 and math.isnan(empty.clip)
    with pytest.raises(ValueError):
        P.panelStats(data, meta, clipPercentile=101.0)
    with pytest.raises(ValueError):
        P.panelStats(data[:10], meta)
