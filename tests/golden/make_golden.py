"""Writes tests/golden/fixtures.npz: small seeded inputs and the oracle's
outputs for them (the reference itself, Nim, cannot run in this build), so
that a change of the oracle or of the device path against the same inputs
shows. Each case: a flow (or a decode / spectrum call), float32 and float64,
4 traces of 1001 samples at 2 ms with ragged live lengths, a dead row and
per-row offsets and t0s. Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import processseg_b200 as P  # noqa: E402
from processseg_b200 import _abi as A  # noqa: E402
from oracle import oracle as O  # noqa: E402

ROWS, COLS, DT = 4, 1001, 2.0


def flows():
    return {
        "dfa": [P.demeanOp(), P.filterOp(P.bandPass(P.Corners(3, 6, 70, 90)).withNotch(50, 2)), P.agcOp(300)],
        "mutes": [P.muteTopOp(P.lmoMute(2500, padMs=-20), taperMs=20), P.bandPassOp(P.Corners(4, 8, 60, 80)),
                  P.muteBottomOp(P.timeMute(1500), taperMs=40)],
        "iir": [P.iirOp(P.butterBandPass(4, 60, 24)), P.normalizeOp(P.normPercentile, percentile=95.0)],
        "curves": [P.detrendOp(), P.gainCurveOp(P.powerGain(2)), P.clipOp(-3, 3),
                   P.normalizeOp(P.normRms, P.perPanel, target=2.0)],
    }


def inputs():
    rng = np.random.default_rng(20261203)
    x = rng.standard_normal((ROWS, COLS)) + np.sin(2 * np.pi * 25 * np.arange(COLS) * DT / 1000)
    live = np.array([1001, 700, 0, 333], np.int32)
    for r in range(ROWS):
        x[r, live[r]:] = 0
    status = np.array([A.TS_LIVE, A.TS_LIVE, A.TS_DEAD, A.TS_LIVE], np.int32)
    t0 = np.array([0.0, 12.0, 0.0, -8.0])
    offsets = np.array([100.0, 900.0, 0.0, 2100.0])
    return x, live, status, t0, offsets


def main():
    x, live, status, t0, offsets = inputs()
    meta = P.initChunkMeta(status, live, DT, t0, 0, (), offsets)
    lv, start = meta.flat(COLS)
    out = {"x": x, "live": live, "status": status, "t0": t0, "offsets": offsets}
    for name, flow in flows().items():
        for code, npdt in ((A.F32, np.float32), (A.F64, np.float64)):
            y = O.OraclePlan(flow, code, DT, COLS).apply(x.astype(npdt), lv, start, keys=(offsets, t0, 0, DT))
            out[f"{name}_{npdt.__name__}"] = y
    rng = np.random.default_rng(7)
    rec = rng.integers(0, 256, (3, 240 + 4 * 64), dtype=np.uint8)
    out["segy_records"] = rec
    out["segy_ibm_f32"] = O.segy_decode(rec, 64, 1, np.float32)
    amp, used = O.spectrum_average(x.astype(np.float32), lv, DT, 501, 100, 0.1, 0)
    out["spectrum_avg_f32"] = amp
    out["spectrum_used"] = np.array([used])
    np.savez_compressed(os.path.join(HERE, "fixtures.npz"), **out)


if __name__ == "__main__":
    main()
