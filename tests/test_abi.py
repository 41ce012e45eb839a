"""The C ABI without a GPU: libpsgcuda.so loads, exports every entry point
include/psg.h declares, and its host-side plan arithmetic (fast lengths,
responses, impulse lengths, margins, row flattening, sweeps) agrees with the
oracle. The device entry points are exercised by the gpu-marked tests."""
import ctypes as C
import math
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A
from oracle import oracle as O

pytestmark = pytest.mark.usefixtures("built")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "psg.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(psg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = A.lib()
    names = declared_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares every one of them
    assert set(names) <= set(A.EXPORTED), set(names) - set(A.EXPORTED)


def test_struct_layout_matches_header():
    # psg_op is shared by ctypes callers: its size is fixed by the header.
    assert C.sizeof(A.FilterSpecC) == 16 + 8 * 8 + 16 * 8
    assert C.sizeof(A.GainCurveC) == 8 + 4 * 8 + 16 * 64
    assert C.sizeof(A.MuteCurveC) == 8 + 4 * 8 + 16 * 64
    assert C.sizeof(A.OpC) == (8 + 8 * 3 + C.sizeof(A.FilterSpecC) + 8 * 3 + 16 + 16 + C.sizeof(A.GainCurveC) + 16
                               + C.sizeof(A.MuteCurveC) + 8)
    # and as the C compiler lays the header out
    prog = r'''
#include <stddef.h>
#include <stdio.h>
#include "psg.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(psg_op), offsetof(psg_op, iir_phase), offsetof(psg_op, curve),
         offsetof(psg_op, mute), offsetof(psg_op, taper_ms), sizeof(psg_keys));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        with open(src, "w") as f:
            f.write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", exe, src], check=True)
        got = [int(v) for v in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(A.OpC), A.OpC.iir_phase.offset, A.OpC.curve.offset, A.OpC.mute.offset, A.OpC.taper_ms.offset,
            C.sizeof(A.KeysC)]
    assert got == want


def test_fast_lengths_match_oracle():
    lib = A.lib()
    for n in range(0, 6000, 3):
        assert lib.psg_is_fast_len(n) == int(O.is_fast_len(n))
        assert lib.psg_next_fast_len(n, 1) == O.next_fast_len(n)
        assert lib.psg_next_fast_len(n, 0) == O.next_fast_len(n, even=False)


SPECS = [
    P.bandPass(P.Corners(4, 8, 60, 80)),
    P.bandPass(P.Corners(3, 6, 70, 90)).withNotch(50, 2),
    P.bandPass(P.Corners(2, 5, 120, 150)),
    P.lowCut(0.5, 1), P.lowCut(1, 2), P.highCut(60, 80), P.highCut(60, 80).withZeroDc(),
    P.butterBandPass(5, 100, 24), P.butterLowCut(2), P.butterBandPass(2, 80, 48),
    P.highCut(60, 80).withNotch(50, 2), P.bandPass(P.Corners(0.5, 1, 60, 80)),
]


@pytest.mark.parametrize("dt", [1.0, 2.0, 4.0])
def test_impulse_lengths_and_responses_match_oracle(dt):
    for s in SPECS:
        try:
            want = O.impulse_length(s, dt)
        except ValueError:
            with pytest.raises(ValueError):
                s.impulseLength(dt)
            continue
        assert s.impulseLength(dt) == want, (s, dt)
        for f in np.linspace(0, 500 / dt, 97):
            assert abs(s.response(f, dt) - O.response(s, f, dt)) <= 1e-15


def test_required_margin_matches_oracle_and_names_the_op():
    flows = [
        [P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 60, 80)), P.agcOp(500)],
        [P.demeanOp(), P.filterOp(SPECS[1]), P.agcOp(300)],
        [P.filterOp(P.butterBandPass(5, 100, 24)), P.gainCurveOp(P.powerGain(2))],
        [P.gainDbOp(3)],
    ]
    for f in flows:
        for dt in (1.0, 2.0):
            assert P.initPipeline(f).requiredMargin(dt) == O.required_margin(f, dt)
    with pytest.raises(ValueError, match=r"^op 1 \(opAgc\): "):
        P.initPipeline([P.demeanOp(), P.agcOp(1)]).requiredMargin(2)
    with pytest.raises(ValueError):
        P.initPipeline([P.agcOp(100)]).requiredMargin(0)


def test_decode_window_matches_reference_answers():
    lib = A.lib()
    out = (C.c_int64 * 2)()
    for (a, b, m, n), want in [((800, 1200, 110, 2001), (690, 1310)), ((50, 300, 110, 2001), (0, 410)),
                               ((1900, 2000, 110, 2001), (1790, 2000)), ((10, 20, -5, 100), (10, 20)),
                               ((10, 20, 2 ** 62, 100), (0, 99))]:
        lib.psg_decode_window(a, b, m, n, out)
        assert (out[0], out[1]) == want


def test_rows_flatten_matches_oracle():
    rng = np.random.default_rng(3)
    rows, cols = 97, 500
    status = rng.integers(0, 4, rows).astype(np.int32)
    ns = rng.integers(0, 700, rows).astype(np.int32)
    t0 = rng.uniform(-100, 100, rows)
    failed = np.array([3, 10, 11, 50], np.int64)
    status[0], ns[0] = P.tsLive, 0  # a live row with no samples
    for first in (0, 37):
        for mode in (0, 1, 3):
            meta = P.initChunkMeta(status, ns, 2.0, t0, first, failed)
            live, start = meta.flat(cols, mode)
            ol, os_ = O.rows_flatten(status, ns, t0, first, 2.0, failed, cols, mode)
            assert np.array_equal(live, ol) and np.array_equal(start, os_)
            for r in range(rows):
                use = meta.isLive(r) if mode in (0, 3) else (status[r] != P.tsDead and not meta.isFailed(r))
                want = meta.liveSamples(r, cols) if use else (-1 if mode == 3 else 0)
                assert live[r] == want
            if mode == 3:
                # a live row with an empty live window stays apart from a row not live
                assert np.any(live == 0) and np.any(live == -1)
    with pytest.raises(ValueError):
        P.initChunkMeta(status, ns, 2.0, t0, 0, [5, 5]).flat(cols)


def test_linear_sweep_matches_oracle():
    for args in [(8, 80, 12000, 2, 300, 300, 2), (8, 60, 1000, 2, 100, 100, 2),
                 (10, 80, 4000, 2, 200, 200, 0)]:
        f1, f2, L, dt, ts, te, shape = args
        spec = P.linearSweep(f1, f2, L, dt, P.initSweepTaper(ts, te, shape))
        x = spec.samples()
        y = O.linear_sweep(f1, f2, L, dt, ts, te, shape)
        assert x.size == y.size == int(L / dt)
        assert np.max(np.abs(x - y)) <= 1e-15
    with pytest.raises(ValueError):
        P.linearSweep(8, 300, 1000, 2)  # above 0.8 × Nyquist
    with pytest.raises(ValueError):
        P.linearSweep(8, 80, 1001, 2)  # not a whole number of samples


def test_builders_validate_like_the_reference():
    with pytest.raises(ValueError):
        P.bandPass(P.Corners(8, 4, 60, 80))
    with pytest.raises(ValueError):
        P.bandPass(P.Corners(4, 8, 80, 60))
    with pytest.raises(ValueError):
        P.butterBandPass(10, 5)
    with pytest.raises(ValueError):
        P.lowCut(1, 2).withNotch(-1, 2)
    with pytest.raises(ValueError):
        P.knotGain([P.GainKnot(0, 0), P.GainKnot(0, 3)])
    with pytest.raises(ValueError):
        P.powerGain(2, refMs=0)
    op = P.agcOp(500)
    with pytest.raises(ValueError):
        op.filter
    assert op.agc.windowMs == 500
    flow = P.initPipeline([P.demeanOp(), op])
    flow[1].agc.windowMs = 300
    assert flow[1].agc.windowMs == 300


def test_no_cpu_fallback_without_a_device():
    """Compiling a plan needs the device: without one the library says so
    (it never computes on the host)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(Exception) as e:
        P.initPipeline([P.demeanOp()]).compile(P.float32, 2.0, 100)
    assert not isinstance(e.value, ValueError) or "device" in str(e.value).lower()


def test_statistics_refuse_a_bad_dtype_before_any_launch():
    # checked before the device is touched: no GPU needed, nothing launched
    lib = A.lib()
    out = (C.c_double * 5)()
    for dtype in (2, -1, 7):
        assert lib.psg_trace_stats(None, dtype, 4, 4, None, out, out, None) == A.EINVAL
        assert "dtype" in lib.psg_last_error().decode()
        assert lib.psg_panel_stats(None, None, dtype, 4, 4, None, 99.0, out, None) == A.EINVAL
        assert "dtype" in lib.psg_last_error().decode()
        assert lib.psg_panel_stats_static(None, dtype, 4, 4, None, 99.0, out, None) == A.EINVAL
        assert "dtype" in lib.psg_last_error().decode()


def test_trace_stats_oracle_follows_stats_of():
    # the checker itself: NaN for rows not live, (0, 0) for an empty live row,
    # float64 sums of squares over the live samples
    b = np.arange(12, dtype=np.float32).reshape(3, 4) - 5
    rms, mx = O.trace_stats(b, np.array([-1, 0, 3], np.int32))
    assert math.isnan(rms[0]) and math.isnan(mx[0])
    assert rms[1] == 0 and mx[1] == 0
    assert rms[2] == math.sqrt((3 * 3 + 4 * 4 + 5 * 5) / 3) and mx[2] == 5
    st = O.panel_stats(b, np.array([-1, 0, 3], np.int32), math.nan, signed=True)
    assert st["rows"] == 2 and st["samples"] == 3
    st = O.panel_stats(b, np.array([0, 0, 3], np.int32), math.nan)
    assert st["rows"] == 1 and st["samples"] == 3
