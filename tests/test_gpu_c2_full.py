"""The headline configuration itself: the 2000 × 3001 float32 panel that the
benchmark times (synth.c2() at its seed, live lengths U{1500..3001}, demean →
band-pass 3/6/70/90 Hz with a 2 Hz notch at 50 Hz → AGC 300 ms), src → dst on
the device, every trace against the float32 oracle (parity: within 1e-5 of
its RMS) and the FP64 oracle (the precision bar: within 1e-5 of its RMS),
with the samples past each live length copied bit for bit. Also the
float64 plan on the same panel against the FP64 oracle (1e-12)."""
import os

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import synth
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]

FLOW = [P.demeanOp(), P.filterOp(P.bandPass(P.Corners(3, 6, 70, 90)).withNotch(50, 2)), P.agcOp(300)]
ROWS, COLS, DT = 2000, 3001, 2.0


def rel_errs(got, want, live):
    """Per trace: max |got − want| over its live samples / the RMS of want there."""
    mask = np.arange(want.shape[1])[None, :] < live[:, None]
    w = want.astype(np.float64)
    g = got.astype(np.float64)
    n = np.maximum(mask.sum(1), 1)
    rms = np.sqrt(np.where(mask, w * w, 0).sum(1) / n)
    d = np.where(mask, np.abs(g - w), 0).max(1)
    return np.where(rms > 0, d / np.where(rms > 0, rms, 1), 0)


def device(dtype, data, meta):
    plan = P.initPipeline(FLOW).compile(dtype, DT, COLS)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=ROWS, cols=COLS)
    src = torch.from_numpy(data).cuda()
    dst = torch.full_like(src, float("nan"))
    plan.apply(src, dst, meta, ws)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


def test_benchmarked_c2_panel_matches_oracles():
    g = synth.c2()
    assert g.data.shape == (ROWS, COLS)
    meta = g.meta()
    live, start = meta.flat(COLS)
    assert live.min() >= 1500 and live.max() <= 3001
    cores = os.cpu_count() or 1
    got = device(P.float32, g.data, meta)
    mask = np.arange(COLS)[None, :] >= live[:, None]
    assert np.array_equal(got[mask], g.data[mask])
    want32 = O.OraclePlan(FLOW, P.F32, DT, COLS).apply(g.data, live, start, threads=cores)
    want64 = O.OraclePlan(FLOW, P.F64, DT, COLS).apply(g.data.astype(np.float64), live, start, threads=cores)
    par = rel_errs(got, want32, live)
    prec = rel_errs(got, want64, live)
    own = rel_errs(want32, want64, live)
    print(f"C2 2000x3001: device vs float32 oracle max {par.max():.3e} p99 {np.percentile(par, 99):.3e};"
          f" device vs FP64 oracle max {prec.max():.3e} p99 {np.percentile(prec, 99):.3e};"
          f" float32 oracle vs FP64 max {own.max():.3e}")
    assert par.max() <= 1e-5
    assert prec.max() <= 1e-5

    got64 = device(P.float64, g.data.astype(np.float64), meta)
    assert rel_errs(got64, want64, live).max() <= 1e-12
