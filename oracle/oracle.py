"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle
(``oracle/libpsg_oracle.so``, built from ``oracle/psg_oracle.cpp`` by
``oracle/Makefile``). Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py`` use it, as the checker or the timed CPU
reference; the product never does.

The oracle restates the reference's Nim hot path (see the header of
psg_oracle.cpp). It cannot be compared with the reference's own binaries
(no Nim toolchain exists here): it is pinned by the reference's known-answer
tests instead (tests/test_oracle_pins.py).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

from processseg_b200 import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libpsg_oracle.so")
_lib = None

P, I32, I64, DBL = C.c_void_p, C.c_int32, C.c_int64, C.c_double


def build():
    """Compiles the oracle with its Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        sig = {
            "orc_last_error": (C.c_char_p, []),
            "orc_is_fast_len": (C.c_int, [I64]),
            "orc_next_fast_len": (I64, [I64, C.c_int]),
            "orc_fft_forward": (C.c_int, [C.c_int, I64, P, P, P]),
            "orc_fft_inverse": (C.c_int, [C.c_int, I64, P, P, P]),
            "orc_response": (C.c_int, [C.POINTER(A.FilterSpecC), DBL, DBL, C.POINTER(DBL)]),
            "orc_impulse_length": (C.c_int, [C.POINTER(A.FilterSpecC), DBL, C.POINTER(I64)]),
            "orc_filter_plan_info": (C.c_int, [C.POINTER(A.FilterSpecC), C.c_int, DBL, I64, C.c_int,
                                               C.POINTER(I64), C.POINTER(I64), C.POINTER(I64),
                                               C.POINTER(C.c_int), C.POINTER(DBL), P]),
            "orc_required_margin": (C.c_int, [C.POINTER(A.OpC), C.c_int, DBL, C.POINTER(I64)]),
            "orc_plan_compile": (C.c_int, [C.POINTER(A.OpC), C.c_int, C.c_int, DBL, I64, I64,
                                           C.POINTER(P)]),
            "orc_plan_destroy": (None, [P]),
            "orc_plan_margin": (I64, [P]),
            "orc_plan_part_count": (C.c_int, [P]),
            "orc_plan_step_nfft": (I64, [P, C.c_int]),
            "orc_rows_flatten": (C.c_int, [P, P, P, I64, I32, DBL, P, I64, I32, I32, P, P]),
            "orc_plan_apply": (C.c_int, [P, P, P, I64, I64, P, P, C.c_int]),
            "orc_plan_apply_keyed": (C.c_int, [P, P, P, I64, I64, P, P, P, P, I64, C.c_double, C.c_int]),
            "orc_iir_info": (C.c_int, [C.POINTER(A.FilterSpecC), C.c_double, I64, C.c_int, C.c_int,
                                       C.POINTER(C.c_int), C.POINTER(I64), C.POINTER(C.c_double), P, I64, P]),
            "orc_iir_apply": (C.c_int, [C.POINTER(A.FilterSpecC), C.c_double, I64, C.c_int, C.c_int, P, I64]),
            "orc_spectrum": (C.c_int, [C.c_int, C.c_double, I64, C.c_double, I64, C.c_int, P, I64, I64, P, I64,
                                       I64, I64, P, P, P, P, P, P]),
            "orc_bench_apply": (C.c_int, [P, P, P, I64, I64, P, P, C.c_int, C.c_int, C.c_int, DBL,
                                          C.POINTER(DBL), C.POINTER(DBL), C.POINTER(I64)]),
            "orc_agc_row": (C.c_int, [C.c_int, DBL, DBL, C.c_int, DBL, DBL, P, I64]),
            "orc_panel_stats": (C.c_int, [C.c_int, P, I64, I64, P, DBL, C.c_int, P]),
            "orc_trace_stats": (C.c_int, [C.c_int, P, I64, I64, P, P, P]),
            "orc_percentile_abs": (C.c_int, [C.c_int, P, I64, DBL, C.POINTER(DBL)]),
            "orc_linear_sweep": (C.c_int, [DBL, DBL, DBL, DBL, DBL, DBL, C.c_int, DBL, DBL, DBL,
                                           C.c_int, P, C.POINTER(I64)]),
            "orc_taper_weight": (C.c_int, [C.c_int, DBL, DBL, C.POINTER(DBL)]),
            "orc_sweep_samples": (C.c_int, [C.c_int, DBL, DBL, DBL, DBL, DBL, P, C.c_int, P, C.c_int, DBL,
                                            DBL, DBL, DBL, C.c_int, DBL, C.c_int, P, I64]),
            "orc_sweep_frequency_at": (C.c_int, [C.c_int, DBL, DBL, DBL, DBL, DBL, P, C.c_int, DBL,
                                                 C.POINTER(DBL)]),
            "orc_correlate": (C.c_int, [P, I64, DBL, DBL, C.c_int, DBL, I64, I64, C.c_int, DBL,
                                        C.c_int, P, P, I64, I64, P, C.POINTER(I64),
                                        C.POINTER(DBL)]),
            "orc_stack_add": (C.c_int, [C.c_int, P, I64, I64, P, P, P, P, I64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def _check(st):
    if st != 0:
        raise ValueError(lib().orc_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _dt(a):
    return A.F32 if a.dtype == np.float32 else A.F64


def is_fast_len(n):
    return bool(lib().orc_is_fast_len(n))


def next_fast_len(n, even=True):
    return lib().orc_next_fast_len(n, 1 if even else 0)


def fft_forward(x):
    x = np.ascontiguousarray(x)
    n = x.size
    re = np.zeros(n // 2 + 1, x.dtype)
    im = np.zeros(n // 2 + 1, x.dtype)
    _check(lib().orc_fft_forward(_dt(x), n, _ptr(x), _ptr(re), _ptr(im)))
    return re, im


def fft_inverse(re, im, n):
    re = np.ascontiguousarray(re)
    im = np.ascontiguousarray(im)
    x = np.zeros(n, re.dtype)
    _check(lib().orc_fft_inverse(_dt(re), n, _ptr(re), _ptr(im), _ptr(x)))
    return x


def response(spec, f, dtMs):
    out = C.c_double()
    _check(lib().orc_response(C.byref(spec.to_c()), f, dtMs, C.byref(out)))
    return out.value


def impulse_length(spec, dtMs):
    out = C.c_int64()
    _check(lib().orc_impulse_length(C.byref(spec.to_c()), dtMs, C.byref(out)))
    return out.value


def filter_plan_info(spec, dtype, dtMs, samples, trend=A.TR_LINEAR, with_gain=False):
    m, pad, nfft = C.c_int64(), C.c_int64(), C.c_int64()
    refl, dc = C.c_int(), C.c_double()
    s = spec.to_c()
    _check(lib().orc_filter_plan_info(C.byref(s), dtype, dtMs, samples, trend, C.byref(m),
                                      C.byref(pad), C.byref(nfft), C.byref(refl), C.byref(dc),
                                      None))
    info = dict(margin=m.value, pad=pad.value, nfft=nfft.value, reflect=bool(refl.value),
                dcGain=dc.value)
    if with_gain:
        g = np.zeros(nfft.value // 2 + 1)
        _check(lib().orc_filter_plan_info(C.byref(s), dtype, dtMs, samples, trend, C.byref(m),
                                          C.byref(pad), C.byref(nfft), C.byref(refl), C.byref(dc),
                                          _ptr(g)))
        info["gain"] = g
    return info


def required_margin(ops, dtMs):
    arr = A.ops_array(ops)
    out = C.c_int64()
    _check(lib().orc_required_margin(arr, len(ops), dtMs, C.byref(out)))
    return out.value


class OraclePlan:
    """A compiled pipeline in the oracle (pipeline.nim:466-523)."""

    def __init__(self, ops, dtype, dtMs, samples, recordSamples=0):
        self.dtype = dtype
        arr = A.ops_array(list(ops))
        h = C.c_void_p()
        _check(lib().orc_plan_compile(arr, len(list(ops)), dtype, dtMs, samples, recordSamples,
                                      C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.orc_plan_destroy(self.h)
            self.h = None

    @property
    def margin(self):
        return lib().orc_plan_margin(self.h)

    @property
    def partCount(self):
        return lib().orc_plan_part_count(self.h)

    def step_nfft(self, i):
        return lib().orc_plan_step_nfft(self.h, i)

    def apply(self, src, live, startMs=None, threads=1, inplace=False, keys=None):
        """Runs the plan on ``src`` ([rows, cols], the plan's dtype): returns
        dst (src → dst form; the copy fused per row as the reference).
        ``keys`` = (offsets, t0Ms, firstSample, dtMs): the rows' trace keys,
        which mutes read."""
        src = np.ascontiguousarray(src)
        rows, cols = src.shape
        live = np.ascontiguousarray(live, dtype=np.int32)
        st = None if startMs is None else np.ascontiguousarray(startMs, dtype=np.float64)
        if keys is not None:
            off = None if keys[0] is None else np.ascontiguousarray(keys[0], dtype=np.float64)
            t0 = None if keys[1] is None else np.ascontiguousarray(keys[1], dtype=np.float64)
            dst = src.copy() if inplace else np.zeros_like(src)
            _check(lib().orc_plan_apply_keyed(self.h, None if inplace else _ptr(src), _ptr(dst), rows, cols,
                                              _ptr(live), _ptr(st), _ptr(off), _ptr(t0), int(keys[2]),
                                              float(keys[3]), threads))
            return dst
        if inplace:
            dst = src.copy()
            _check(lib().orc_plan_apply(self.h, None, _ptr(dst), rows, cols, _ptr(live), _ptr(st),
                                        threads))
        else:
            dst = np.zeros_like(src)
            _check(lib().orc_plan_apply(self.h, _ptr(src), _ptr(dst), rows, cols, _ptr(live),
                                        _ptr(st), threads))
        return dst

    def bench(self, src, live, startMs=None, threads=1, warm=3, samples=15, min_sample_ms=20.0):
        """Median and minimum seconds of one src → dst apply through the pool
        clone, and the applies run, by the reference harness's method
        (bench/benchutil.nim:96-126): ``warm`` applies, then ``samples``
        samples of doubling batches of at least ``min_sample_ms`` each."""
        src = np.ascontiguousarray(src)
        rows, cols = src.shape
        dst = np.zeros_like(src)
        live = np.ascontiguousarray(live, dtype=np.int32)
        st = None if startMs is None else np.ascontiguousarray(startMs, dtype=np.float64)
        med, mn, n = C.c_double(), C.c_double(), C.c_int64()
        _check(lib().orc_bench_apply(self.h, _ptr(src), _ptr(dst), rows, cols, _ptr(live), _ptr(st),
                                     threads, warm, samples, min_sample_ms, C.byref(med), C.byref(mn),
                                     C.byref(n)))
        return med.value, mn.value, n.value


def iir_info(spec, dtMs, samples, phase=A.IP_ZERO, trend=A.TR_LINEAR, freqs=()):
    """(order, requiredMargin, dcGain, magnitudeAt(freqs)) of an IIR plan."""
    c = spec.to_c()
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    mag = np.zeros(f.size)
    order, pad, g = C.c_int(), C.c_int64(), C.c_double()
    _check(lib().orc_iir_info(C.byref(c), dtMs, samples, phase, trend, C.byref(order), C.byref(pad), C.byref(g),
                              _ptr(f), f.size, _ptr(mag)))
    return order.value, pad.value, g.value, mag


def iir_apply(spec, dtMs, x, phase=A.IP_ZERO, trend=A.TR_LINEAR, samples=None):
    """One trace (float64) through an IIR plan of ``samples`` (default: its
    length), as the reference's single-trace applyFilter."""
    c = spec.to_c()
    y = np.ascontiguousarray(x, dtype=np.float64).copy()
    _check(lib().orc_iir_apply(C.byref(c), dtMs, samples or y.size, phase, trend, _ptr(y), y.size))
    return y


def spectrum_plan(dtype, dtMs, windowLen, taperFraction=0.1, nfft=0, demean=True):
    """(nfft, Σw) of a SpectrumPlan."""
    n, sw = C.c_int64(), C.c_double()
    _check(lib().orc_spectrum(dtype, dtMs, windowLen, taperFraction, nfft, int(demean), None, 0, 0, None, 0, 0, -1,
                              None, None, None, None, C.byref(n), C.byref(sw)))
    return n.value, sw.value


def spectrum_average(b, live, dtMs, windowLen, firstCol, taperFraction=0.1, nfft=0, demean=True, rows=(0, 2 ** 62)):
    """(amp, used): averageAmplitudeInto over the rows ``rows`` (inclusive)."""
    b = np.ascontiguousarray(b)
    dtype = A.F32 if b.dtype == np.float32 else A.F64
    n, _ = spectrum_plan(dtype, dtMs, windowLen, taperFraction, nfft, demean)
    amp = np.zeros(n // 2 + 1)
    used = C.c_int64()
    live = np.ascontiguousarray(live, dtype=np.int32)
    _check(lib().orc_spectrum(dtype, dtMs, windowLen, taperFraction, nfft, int(demean), _ptr(b), b.shape[0],
                              b.shape[1], _ptr(live), firstCol, rows[0], rows[1], _ptr(amp), C.byref(used), None,
                              None, None, None))
    return amp, used.value


def spectrum_amplitudes(b, live, dtMs, windowLen, firstCol, taperFraction=0.1, nfft=0, demean=True):
    """(amp, phase), rows × bins of the block's dtype: amplitudeInto per row."""
    b = np.ascontiguousarray(b)
    dtype = A.F32 if b.dtype == np.float32 else A.F64
    n, _ = spectrum_plan(dtype, dtMs, windowLen, taperFraction, nfft, demean)
    amp = np.zeros((b.shape[0], n // 2 + 1), b.dtype)
    phase = np.zeros_like(amp)
    live = np.ascontiguousarray(live, dtype=np.int32)
    _check(lib().orc_spectrum(dtype, dtMs, windowLen, taperFraction, nfft, int(demean), _ptr(b), b.shape[0],
                              b.shape[1], _ptr(live), firstCol, 0, -1, None, None, _ptr(amp), _ptr(phase), None,
                              None))
    return amp, phase


def segy_decode(records, samples, format, dtype=np.float32, little=False, header=240, out_cols=0):
    """SEG-Y rev 2 data samples of each record (numpy, exact float64 first,
    then rounded to dtype). IBM float: (−1)^s · 0.f · 16^(e − 64), a 24-bit
    fraction f and a 7-bit excess-64 exponent e."""
    sz = {1: 4, 2: 4, 3: 2, 5: 4, 6: 8, 7: 3, 8: 1, 10: 4, 11: 2, 15: 3, 16: 1}[format]
    rec = np.ascontiguousarray(records, dtype=np.uint8)
    raw = rec[:, header:header + samples * sz].reshape(rec.shape[0], samples, sz).astype(np.uint64)
    if little:
        raw = raw[:, :, ::-1]
    u = np.zeros(raw.shape[:2], np.uint64)
    for i in range(sz):
        u = (u << np.uint64(8)) | raw[:, :, i]
    if format == 1:
        frac = (u & np.uint64(0xFFFFFF)).astype(np.float64)
        e = ((u >> np.uint64(24)) & np.uint64(0x7F)).astype(np.int64)
        v = np.ldexp(frac, 4 * e - 280)
        v = np.where((u >> np.uint64(31)) & np.uint64(1), -v, v)
    elif format == 2:
        v = u.astype(np.uint32).view(np.int32).astype(np.float64)
    elif format == 3:
        v = u.astype(np.uint16).view(np.int16).astype(np.float64)
    elif format == 5:
        with np.errstate(invalid="ignore"):
            v = u.astype(np.uint32).view(np.float32).astype(np.float64)
    elif format == 6:
        v = u.view(np.float64).copy()
    elif format == 7:
        v = ((u.astype(np.int64) ^ 0x800000) - 0x800000).astype(np.float64)
    elif format == 8:
        v = u.astype(np.uint8).view(np.int8).astype(np.float64)
    else:
        v = u.astype(np.float64)
    cols = out_cols or samples
    out = np.zeros((rec.shape[0], cols), dtype)
    with np.errstate(over="ignore", invalid="ignore"):
        out[:, :min(cols, samples)] = v[:, :min(cols, samples)].astype(dtype)
    return out


def segy_keys(records, little=False):
    """(status, numSamples, intervalUs, offset, t0Ms) from the trace headers."""
    rec = np.ascontiguousarray(records, dtype=np.uint8)
    o = "<" if little else ">"
    def field(at, t):
        return np.frombuffer(rec[:, at:at + np.dtype(t).itemsize].tobytes(), dtype=np.dtype(o + t))
    code = field(28, "i2")
    status = np.where(code == 1, A.TS_LIVE, np.where(code == 2, A.TS_DEAD, np.where(code == 0, A.TS_UNKNOWN,
                                                                                     A.TS_AUX)))
    return (status.astype(np.int32), field(114, "u2").astype(np.int32), field(116, "u2").astype(np.float64),
            field(36, "i4").astype(np.float64), field(108, "i2").astype(np.float64))


def rows_flatten(status, numSamples, t0Ms, firstSample, dtMs, failed, cols, mode=0):
    status = np.ascontiguousarray(status, dtype=np.int32)
    ns = np.ascontiguousarray(numSamples, dtype=np.int32)
    t0 = None if t0Ms is None else np.ascontiguousarray(t0Ms, dtype=np.float64)
    fl = np.ascontiguousarray(failed if failed is not None else [], dtype=np.int64)
    rows = status.size
    live = np.zeros(rows, np.int32)
    start = np.zeros(rows, np.float64)
    _check(lib().orc_rows_flatten(_ptr(status), _ptr(ns), _ptr(t0), rows, firstSample, dtMs,
                                  _ptr(fl), fl.size, cols, mode, _ptr(live), _ptr(start)))
    return live, start


def agc_row(x, windowMs, dtMs, mode=A.AGC_RMS, target=1.0, eps=1e-9):
    y = np.ascontiguousarray(x).copy()
    _check(lib().orc_agc_row(_dt(y), windowMs, dtMs, mode, target, eps, _ptr(y), y.size))
    return y


def panel_stats(b, live, clipP, signed=False):
    """panelStats (stats.nim:253-304) of the rows ``live`` selects: with
    ``signed`` a row with live < 0 is not live and live == 0 is a live row
    without samples (flattening mode 3); otherwise live == 0 is not live."""
    b = np.ascontiguousarray(b)
    live = np.ascontiguousarray(live, dtype=np.int32)
    out = np.zeros(5)
    _check(lib().orc_panel_stats(_dt(b), _ptr(b), b.shape[0], b.shape[1], _ptr(live), clipP,
                                 1 if signed else 0, _ptr(out)))
    return dict(rms=out[0], maxAbs=out[1], clip=out[2], rows=int(out[3]), samples=int(out[4]))


def trace_stats(b, live):
    """traceStatsInto (stats.nim:186-199): (rms, maxAbs) per row, NaN for a
    row with live < 0, (0, 0) for a live row without samples."""
    b = np.ascontiguousarray(b)
    live = np.ascontiguousarray(live, dtype=np.int32)
    rms = np.zeros(b.shape[0])
    mx = np.zeros(b.shape[0])
    _check(lib().orc_trace_stats(_dt(b), _ptr(b), b.shape[0], b.shape[1], _ptr(live), _ptr(rms), _ptr(mx)))
    return rms, mx


def percentile_abs(x, p):
    x = np.ascontiguousarray(x)
    out = C.c_double()
    _check(lib().orc_percentile_abs(_dt(x), _ptr(x), x.size, p, C.byref(out)))
    return out.value


def linear_sweep(f1, f2, lengthMs, dtMs, taperStart=0.0, taperEnd=0.0, shape=2, phaseDeg=0.0,
                 amplitude=1.0, dtype=np.float64, param=math.nan):
    n = C.c_int64()
    dt = A.F32 if dtype == np.float32 else A.F64
    _check(lib().orc_linear_sweep(f1, f2, lengthMs, dtMs, taperStart, taperEnd, shape, param, phaseDeg,
                                  amplitude, dt, None, C.byref(n)))
    x = np.zeros(n.value, dtype)
    _check(lib().orc_linear_sweep(f1, f2, lengthMs, dtMs, taperStart, taperEnd, shape, param, phaseDeg,
                                  amplitude, dt, _ptr(x), C.byref(n)))
    return x


def _sweep_args(spec):
    tab = np.array([[p.tMs, p.fHz] for p in spec.table] or [[0.0, 0.0]], np.float64)
    return (spec.law, spec.f1Hz, spec.f2Hz, spec.lengthMs, spec.dtMs, spec.boostDb, _ptr(tab),
            len(spec.table)), tab


def sweep_samples(spec, dtype=np.float64, harmonics=(), n=0):
    """The oracle's sweep of a ``processseg_b200.SweepSpec`` (its fields
    only; the spec is assumed valid)."""
    args, tab = _sweep_args(spec)
    if n == 0:
        steps = spec.lengthMs / spec.dtMs
        n = int(round(steps)) if abs(steps - round(steps)) <= 1e-6 else int(math.floor(steps))
    h = np.array([[x.order, x.amp, x.phaseDeg] for x in harmonics] or [[0.0, 0.0, 0.0]], np.float64)
    x = np.zeros(n, dtype)
    t = spec.taper
    _check(lib().orc_sweep_samples(*args, _ptr(h), len(harmonics), spec.startPhaseDeg, spec.amplitude,
                                   t.startMs, t.endMs, t.shape, t.param, _dt(x), _ptr(x), n))
    return x


def sweep_frequency_at(spec, tMs):
    args, tab = _sweep_args(spec)
    out = C.c_double()
    _check(lib().orc_sweep_frequency_at(*args, tMs, C.byref(out)))
    return out.value


def taper_weight(shape, x, param=math.nan):
    out = C.c_double()
    _check(lib().orc_taper_weight(shape, x, param, C.byref(out)))
    return out.value


def correlate(pilot, pilotDt, pilotT0, src, live, dtMs, recordSamples, outSamples=0,
              mode=A.CM_CORRELATE, epsPercent=1.0, normalize=True):
    pilot = np.ascontiguousarray(pilot, dtype=np.float64)
    src = np.ascontiguousarray(src)
    rows, cols = src.shape
    live = np.ascontiguousarray(live, dtype=np.int32)
    nfft, scale = C.c_int64(), C.c_double()
    # First the plan facts (no rows), then the rows.
    _check(lib().orc_correlate(_ptr(pilot), pilot.size, pilotDt, pilotT0, _dt(src), dtMs,
                               recordSamples, outSamples, mode, epsPercent, int(normalize), None,
                               None, 0, cols, None, C.byref(nfft), C.byref(scale)))
    outN = outSamples if outSamples else recordSamples - pilot.size
    dst = np.zeros((rows, outN), src.dtype)
    _check(lib().orc_correlate(_ptr(pilot), pilot.size, pilotDt, pilotT0, _dt(src), dtMs,
                               recordSamples, outSamples, mode, epsPercent, int(normalize),
                               _ptr(src), _ptr(dst), rows, cols, _ptr(live), C.byref(nfft),
                               C.byref(scale)))
    return dst, nfft.value, scale.value


def stack_add(num, cnt, block, live, rowMap=None):
    block = np.ascontiguousarray(block)
    live = np.ascontiguousarray(live, dtype=np.int32)
    rm = None if rowMap is None else np.ascontiguousarray(rowMap, dtype=np.int32)
    _check(lib().orc_stack_add(_dt(block), _ptr(block), block.shape[0], block.shape[1], _ptr(live),
                               _ptr(rm), _ptr(num), _ptr(cnt), num.shape[1]))


def stack_result(num, cnt, dtype, norm=A.FN_FOLD):
    """stackInto, vibroseis/vstack.nim:439-471 (rsVertical)."""
    c = cnt.astype(np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        if norm == A.FN_NONE:
            v = num
        elif norm == A.FN_FOLD:
            v = num / c
        else:
            v = num / np.sqrt(c)
    v = np.where(cnt == 0, 0.0, v)
    return v.astype(dtype)
