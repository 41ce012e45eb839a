"""Vibroseis correlation and vertical stacking: the host side of
src/processSEG/vibroseis/{sweep,taper,pilot,correlate,vstack}.nim over the
C ABI. Sweeps are synthesised in float64 (closed-form linear phase); the
pilot spectrum and the correlation multiplier are computed in float64 at
plan time; correlation and the stack run on the device.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _abi as A
from .meta import ChunkMeta, same_interval

tpLinear, tpCosine, tpCos2, tpHamming, tpBlackman, tpBlackmanHarris, tpKaiser, tpGaussian, tpPower = range(9)

_DEFAULT_PARAM = {tpKaiser: 6.0, tpGaussian: 0.4, tpPower: 2.0}


def defaultTaperParam(shape: int) -> float:
    """β = 6 (Kaiser), σ = 0.4 (Gaussian), p = 2 (power); NaN for the other
    shapes (taper.nim:69-74)."""
    return _DEFAULT_PARAM.get(shape, math.nan)


@dataclass(frozen=True)
class SweepTaper:
    """The ramps at the two ends of a sweep (taper.nim:60-67): lengths in ms
    (0 or NaN: none), one shape for both, and the shape's parameter (NaN:
    its default wherever the taper is used)."""
    startMs: float = 0.0
    endMs: float = 0.0
    shape: int = tpCos2
    param: float = math.nan

    def validate(self):
        """taper.nim:79-97: the lengths ≥ 0 and finite (or NaN), β in 0 .. 50,
        σ and p > 0 and finite. Raises ``ValueError``."""
        if self.shape not in range(9):
            raise ValueError(f"taper shape {self.shape} is not one of 0 .. 8")
        for name, v in (("startMs", self.startMs), ("endMs", self.endMs)):
            if not math.isnan(v) and not (v >= 0 and v < math.inf):
                raise ValueError(f"a taper {name} must be ≥ 0 and finite (or NaN for none), got {v}")
        p = defaultTaperParam(self.shape) if math.isnan(self.param) else self.param
        if self.shape == tpKaiser and not (0 <= p <= 50):
            raise ValueError(f"a Kaiser taper needs 0 ≤ β ≤ 50, got {p}")
        if self.shape == tpGaussian and not (0 < p < math.inf):
            raise ValueError(f"a Gaussian taper needs σ > 0, got {p}")
        if self.shape == tpPower and not (0 < p < math.inf):
            raise ValueError(f"a power taper needs an exponent > 0, got {p}")

    def segyTaperType(self) -> int:
        return segyTaperType(self.shape)


def initSweepTaper(startMs: float, endMs: float, shape: int = tpCos2, param: float = math.nan) -> SweepTaper:
    """taper.nim:99-111: a NaN ``param`` takes the shape's default."""
    t = SweepTaper(float(startMs), float(endMs), shape,
                   defaultTaperParam(shape) if math.isnan(param) else float(param))
    t.validate()
    return t


def noTaper() -> SweepTaper:
    """taper.nim:113-115."""
    return SweepTaper(0.0, 0.0, tpLinear, math.nan)


def segyTaperType(shape: int) -> int:
    """The SEG-Y taper type code: 1 linear, 2 cos², 3 other (taper.nim:117-123)."""
    return 1 if shape == tpLinear else 2 if shape == tpCos2 else 3


def taperWeight(shape: int, x: float, param: float = math.nan) -> float:
    """taper.nim:125-145 through ``psg_taper_weight``."""
    out = C.c_double()
    A.check(A.lib().psg_taper_weight(int(shape), float(x), float(param), C.byref(out)))
    return out.value


def applyTaper(x: np.ndarray, dtMs: float, t: SweepTaper) -> None:
    """taper.nim:160-179 through ``psg_apply_taper``: in place on a
    contiguous float32 or float64 array; ``ValueError`` with nothing written
    for a bad ``dtMs`` or taper, or ramps that overlap."""
    if not isinstance(x, np.ndarray) or x.dtype not in (np.float32, np.float64) or not x.flags.c_contiguous:
        raise TypeError("applyTaper takes a contiguous float32 or float64 numpy array")
    dt = A.F32 if x.dtype == np.float32 else A.F64
    A.check(A.lib().psg_apply_taper(dt, x.ctypes.data_as(C.c_void_p), x.size, float(dtMs), float(t.startMs),
                                    float(t.endMs), int(t.shape), float(t.param)))


slLinear, slDbPerOctave, slDbPerHz, slExponential, slTable = (A.SL_LINEAR, A.SL_DB_PER_OCTAVE, A.SL_DB_PER_HZ,
                                                               A.SL_EXPONENTIAL, A.SL_TABLE)


@dataclass(frozen=True)
class SweepPoint:
    """A point of a table sweep: the frequency ``fHz`` at ``tMs`` (sweep.nim:76-79)."""
    tMs: float
    fHz: float


@dataclass(frozen=True)
class SweepHarmonic:
    """One term ``amp · sin(order·φ + rad(phaseDeg))`` of a distorted sweep,
    φ the fundamental's phase (sweep.nim:96-103)."""
    order: float = 1.0
    amp: float = 1.0
    phaseDeg: float = 0.0


@dataclass(frozen=True)
class SweepSpec:
    """A vibroseis sweep (sweep.nim:81-94). Make one with ``linearSweep``,
    ``dbPerOctaveSweep``, ``dbPerHzSweep``, ``exponentialSweep`` or
    ``tableSweep``, which validate it; the host library computes the
    samples (float64 phase: closed form for the linear and table laws,
    4-point Gauss–Legendre per interval for the others)."""
    f1Hz: float
    f2Hz: float
    lengthMs: float
    dtMs: float
    taper: SweepTaper = SweepTaper(0.0, 0.0, tpLinear, math.nan)
    startPhaseDeg: float = 0.0
    amplitude: float = 1.0
    maxNyquistFraction: float = 0.8
    law: int = slLinear
    boostDb: float = 0.0
    table: tuple = ()

    def _c(self):
        pts = (A.SweepPointC * max(1, len(self.table)))(*[A.SweepPointC(p.tMs, p.fHz) for p in self.table])
        c = A.SweepC(self.law, self.taper.shape, self.f1Hz, self.f2Hz, self.lengthMs, self.dtMs, self.boostDb,
                     C.cast(pts, C.c_void_p), len(self.table), self.startPhaseDeg, self.amplitude,
                     self.taper.startMs, self.taper.endMs, self.taper.param, self.maxNyquistFraction)
        c._keep = pts
        return c

    def validate(self):
        """sweep.nim:132-183. Raises ``ValueError``."""
        A.check(A.lib().psg_sweep_validate(C.byref(self._c())))

    def sweepLen(self) -> int:
        """sweep.nim:112-119: 0 for a length or interval ``validate`` refuses."""
        n = C.c_int64()
        A.check(A.lib().psg_sweep_len(C.byref(self._c()), C.byref(n)))
        return n.value

    def frequencyAt(self, tMs: float) -> float:
        """sweep.nim:248-284."""
        out = C.c_double()
        A.check(A.lib().psg_sweep_frequency_at(C.byref(self._c()), float(tMs), C.byref(out)))
        return out.value

    def phaseAt(self, tMs: float) -> float:
        """sweep.nim:436-463 (NaN for the boosted laws)."""
        out = C.c_double()
        A.check(A.lib().psg_sweep_phase_at(C.byref(self._c()), float(tMs), C.byref(out)))
        return out.value

    def segySweepType(self) -> int:
        """sweep.nim:465-473: 1 linear, 3 exponential, 4 other."""
        t = C.c_int32()
        x = np.zeros(1)
        A.check(A.lib().psg_sweep_samples(C.byref(self._c()), None, 0, A.F64, x.ctypes.data_as(C.c_void_p), 1,
                                          C.byref(t)))
        return t.value

    def samples(self, dtype=np.float64, harmonics=(), samples: int = 0) -> np.ndarray:
        """sweepSamples / sweepHarmonics (sweep.nim:344-349, 422-434):
        ``samples`` 0 is ``sweepLen``; a longer buffer is the sweep followed
        by zeros, a shorter one its first samples."""
        self.validate()
        n = self.sweepLen() if samples == 0 else int(samples)
        if n < 1:
            raise ValueError(f"samples must be ≥ 1, got {n}")
        dt = A.F32 if np.dtype(dtype) == np.float32 else A.F64
        hs = (A.SweepHarmonicC * max(1, len(harmonics)))(
            *[A.SweepHarmonicC(h.order, h.amp, h.phaseDeg) for h in harmonics])
        x = np.zeros(n, np.float32 if dt == A.F32 else np.float64)
        A.check(A.lib().psg_sweep_samples(C.byref(self._c()), hs, len(harmonics), dt,
                                          x.ctypes.data_as(C.c_void_p), n, None))
        return x

    def sweepInto(self, x: np.ndarray, harmonics=()) -> None:
        """sweepInto / sweepHarmonicsInto (sweep.nim:331-342, 375-420) on a
        float32 or float64 array; without harmonics its length must be
        ``sweepLen``."""
        if not harmonics and x.size != self.sweepLen():
            self.validate()
            raise ValueError(f"the sweep has {self.sweepLen()} samples, the buffer {x.size}")
        x[...] = self.samples(x.dtype, harmonics, x.size)


def sweepHarmonics(spec: SweepSpec, dtype=np.float64, harmonics=(), samples: int = 0) -> np.ndarray:
    return spec.samples(dtype, harmonics, samples)


def _built(**kw) -> SweepSpec:
    s = SweepSpec(**kw)
    s.validate()
    return s


def linearSweep(f1Hz, f2Hz, lengthMs, dtMs, taper: SweepTaper = None, startPhaseDeg=0.0,
                amplitude=1.0, maxNyquistFraction=0.8) -> SweepSpec:
    """sweep.nim:185-192."""
    return _built(f1Hz=f1Hz, f2Hz=f2Hz, lengthMs=lengthMs, dtMs=dtMs, taper=taper or noTaper(),
                  startPhaseDeg=startPhaseDeg, amplitude=amplitude, maxNyquistFraction=maxNyquistFraction)


def dbPerOctaveSweep(f1Hz, f2Hz, lengthMs, dtMs, boostDb, taper: SweepTaper = None, startPhaseDeg=0.0,
                     amplitude=1.0, maxNyquistFraction=0.8) -> SweepSpec:
    """sweep.nim:194-201."""
    return _built(f1Hz=f1Hz, f2Hz=f2Hz, lengthMs=lengthMs, dtMs=dtMs, taper=taper or noTaper(),
                  startPhaseDeg=startPhaseDeg, amplitude=amplitude, maxNyquistFraction=maxNyquistFraction,
                  law=slDbPerOctave, boostDb=boostDb)


def dbPerHzSweep(f1Hz, f2Hz, lengthMs, dtMs, boostDb, taper: SweepTaper = None, startPhaseDeg=0.0,
                 amplitude=1.0, maxNyquistFraction=0.8) -> SweepSpec:
    """sweep.nim:203-210."""
    return _built(f1Hz=f1Hz, f2Hz=f2Hz, lengthMs=lengthMs, dtMs=dtMs, taper=taper or noTaper(),
                  startPhaseDeg=startPhaseDeg, amplitude=amplitude, maxNyquistFraction=maxNyquistFraction,
                  law=slDbPerHz, boostDb=boostDb)


def exponentialSweep(f1Hz, f2Hz, lengthMs, dtMs, taper: SweepTaper = None, startPhaseDeg=0.0,
                     amplitude=1.0, maxNyquistFraction=0.8) -> SweepSpec:
    """sweep.nim:212-219."""
    return _built(f1Hz=f1Hz, f2Hz=f2Hz, lengthMs=lengthMs, dtMs=dtMs, taper=taper or noTaper(),
                  startPhaseDeg=startPhaseDeg, amplitude=amplitude, maxNyquistFraction=maxNyquistFraction,
                  law=slExponential)


def tableSweep(points, dtMs, taper: SweepTaper = None, startPhaseDeg=0.0, amplitude=1.0,
               maxNyquistFraction=0.8) -> SweepSpec:
    """sweep.nim:221-232: f1/f2/length from the first and last points."""
    pts = tuple(points)
    if len(pts) < 2:
        raise ValueError("a table sweep needs at least two points")
    return _built(f1Hz=pts[0].fHz, f2Hz=pts[-1].fHz, lengthMs=pts[-1].tMs, dtMs=dtMs, taper=taper or noTaper(),
                  startPhaseDeg=startPhaseDeg, amplitude=amplitude, maxNyquistFraction=maxNyquistFraction,
                  law=slTable, table=pts)


@dataclass
class Pilot:
    """A pilot sweep: its samples at ``dtMs``, sample 0 at ``t0Ms`` from the
    time break, and the sweep it is when known (pilot.nim:55-62)."""
    samples: np.ndarray
    dtMs: float
    t0Ms: float = 0.0
    sweep: Optional[SweepSpec] = None

    def __len__(self):
        return int(self.samples.size)

    @property
    def lengthMs(self) -> float:
        """``len·dtMs`` (pilot.nim:84-87)."""
        return float(self.samples.size) * self.dtMs if self.samples.size > 0 else 0.0

    def validate(self):
        """pilot.nim:89-106: at least two samples, all finite, not all zero; a
        finite positive ``dtMs``; a finite ``t0Ms``; the sweep's ``dtMs`` equal
        to the pilot's. Raises ``ValueError``."""
        x = np.asarray(self.samples, dtype=np.float64).reshape(-1)
        if x.size < 2:
            raise ValueError(f"a pilot needs at least two samples, got {x.size}")
        if not (self.dtMs > 0 and self.dtMs < math.inf):
            raise ValueError(f"a pilot's dtMs must be finite and positive, got {self.dtMs}")
        if not math.isfinite(self.t0Ms):
            raise ValueError(f"a pilot's t0Ms must be finite, got {self.t0Ms}")
        bad = np.flatnonzero(~np.isfinite(x))
        if bad.size:
            raise ValueError(f"pilot sample {int(bad[0])} is not finite")
        if not np.any(x != 0):
            raise ValueError("the pilot is all zeros")
        if self.sweep is not None and not same_interval(self.sweep.dtMs, self.dtMs):
            raise ValueError(f"the pilot's sweep is sampled at {self.sweep.dtMs} ms, the pilot at {self.dtMs} ms")


def generatePilot(spec: SweepSpec, dtype=np.float64) -> Pilot:
    """The pilot of ``spec`` from ``t0Ms = 0``, with ``sweep`` set
    (pilot.nim:115-119). Raises ``ValueError`` for an invalid spec."""
    return Pilot(spec.samples(dtype), spec.dtMs, 0.0, spec)


def initPilot(samples, dtMs, t0Ms=0.0, sweep: Optional[SweepSpec] = None) -> Pilot:
    """A pilot from samples the caller has (pilot.nim:108-113). Raises
    ``ValueError`` as ``Pilot.validate``."""
    p = Pilot(np.asarray(samples), float(dtMs), float(t0Ms), sweep)
    p.validate()
    return p


def pilotFromRow(meta: ChunkMeta, data, row: int, t0Ms: float = math.nan,
                 sweep: Optional[SweepSpec] = None) -> Pilot:
    """The pilot recorded in row ``row`` of a block (pilot.nim:121-141): its
    live samples, the meta's ``dtMs`` and its start time (that of column 0,
    ``firstSample`` included) unless ``t0Ms`` is given. The row need not be
    live but must not be a failed one. ``data`` is a numpy array or a tensor
    ``[rows, cols]``."""
    rows = int(data.shape[0])
    meta.checkShape(rows)
    if not 0 <= row < len(meta):
        raise ValueError(f"row {row} is outside 0 ..< {len(meta)}")
    if meta.isFailed(row):
        raise ValueError(f"row {row} could not be decoded")
    n = meta.liveSamples(row, int(data.shape[1]))
    r = data[row, :n]
    s = r.detach().cpu().numpy().copy() if hasattr(r, "detach") else np.array(r, copy=True)
    t0 = meta.sampleTimeMs(row, 0) if math.isnan(t0Ms) else float(t0Ms)
    if math.isnan(t0):
        raise ValueError(f"row {row} has no start time in its keys: pass t0Ms")
    return initPilot(s, meta.dtMs, t0, sweep)


def _int16_field(v: float, what: str, unit: str) -> int:
    r = math.floor(abs(v) + 0.5) * (1 if v >= 0 else -1) if math.isfinite(v) else v
    if not (-32768 <= r <= 32767):
        raise ValueError(f"{what} = {v} does not fit a SEG-Y int16 field")
    if abs(v - r) > 1e-9 * max(1.0, abs(r)):
        raise ValueError(f"{what} = {v} {unit} is not a whole number: the SEG-Y sweep fields hold whole {unit}, "
                         "and a rounded value would be read back as the sweep (write the trace without them)")
    return int(r)


def sweepOverrides(spec: SweepSpec, binary: bool = False):
    """The SEG-Y sweep fields of ``spec`` as (name, value) pairs, trace bytes
    127-140 or with ``binary`` the binary header's 3233-3248 (pilot.nim:
    164-184): whole Hz and ms, ``ValueError`` for a value that is not a whole
    number or does not fit an int16."""
    pre = "binary." if binary else "trace."
    t = spec.taper
    ts = 0.0 if math.isnan(t.startMs) else t.startMs
    te = 0.0 if math.isnan(t.endMs) else t.endMs
    return [(pre + "sweepFreqStart", _int16_field(spec.f1Hz, "f1Hz", "Hz")),
            (pre + "sweepFreqEnd", _int16_field(spec.f2Hz, "f2Hz", "Hz")),
            (pre + "sweepLength", _int16_field(spec.lengthMs, "lengthMs", "ms")),
            (pre + "sweepType", spec.segySweepType()),
            (pre + "sweepTaperStart", _int16_field(ts, "taper startMs", "ms")),
            (pre + "sweepTaperEnd", _int16_field(te, "taper endMs", "ms")),
            (pre + "taperType", t.segyTaperType())]


def sweepFromHeaders(f1Hz, f2Hz, lengthMs, sweepType, taperStartMs, taperEndMs, taperType, dtMs,
                     samples: int = 0) -> Optional[SweepSpec]:
    """The sweep SEG-Y sweep fields describe when a trace at ``dtMs`` can hold
    it (pilot.nim:186-212): type 1 (linear) or 3 (exponential), valid at
    ``dtMs`` with frequencies up to Nyquist, and with ``samples`` no longer
    than the trace; else None. The ramps are linear for taper type 1, cos²
    otherwise."""
    if sweepType not in (1.0, 3.0) or not (dtMs > 0 and dtMs < math.inf):
        return None
    if samples > 0 and not (lengthMs <= float(samples) * dtMs):
        return None
    spec = SweepSpec(f1Hz, f2Hz, lengthMs, dtMs,
                     SweepTaper(max(taperStartMs, 0.0), max(taperEndMs, 0.0),
                                tpLinear if taperType == 1 else tpCos2, math.nan),
                     0.0, 1.0, 1.0, slLinear if sweepType == 1 else slExponential)
    try:
        spec.validate()
    except ValueError:
        return None
    return spec


class CorrelationPlan:
    """correlate.nim:66-160."""

    def __init__(self, T, pilot: Pilot, dtMs: float, recordSamples: int, outSamples: int = 0,
                 mode: int = A.CM_CORRELATE, epsPercent: float = 1.0, normalize: bool = True):
        from .plan import _dtype_code
        self.dtype = _dtype_code(T)
        ps = np.ascontiguousarray(pilot.samples)
        pdt = A.F32 if ps.dtype == np.float32 else A.F64
        if ps.dtype not in (np.float32, np.float64):
            ps = ps.astype(np.float64)
            pdt = A.F64
        h = C.c_void_p()
        A.check(A.lib().psg_corr_plan_create(ps.ctypes.data_as(C.c_void_p), pdt, ps.size, pilot.dtMs,
                                             pilot.t0Ms, self.dtype, dtMs, recordSamples, outSamples,
                                             mode, epsPercent, int(normalize), C.byref(h)))
        self.h = h
        self.dtMs = float(dtMs)
        self.recordSamples = int(recordSamples)
        self.pilotSamples = int(ps.size)

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and A._lib is not None:
            A._lib.psg_corr_plan_destroy(h)
            self.h = None

    @property
    def nfft(self) -> int:
        return A.lib().psg_corr_plan_nfft(self.h)

    @property
    def outSamples(self) -> int:
        return A.lib().psg_corr_plan_out_samples(self.h)

    @property
    def scale(self) -> float:
        return A.lib().psg_corr_plan_scale(self.h)

    def correlateInto(self, src, dst, meta: ChunkMeta, stack: "RecordStack" = None, rowMap=None):
        """correlate.nim:421-464 on CUDA tensors; with ``stack`` the
        correlated live rows are also added to it (vstack.nim:357-380) in the
        same launch, row r to stack row ``rowMap[r]`` (−1: not stacked; a host
        sequence, or a CUDA int32 tensor used as it is)."""
        import torch
        rows, cols = int(src.shape[0]), int(src.shape[1])
        meta.checkShape(rows)
        if dst is not None:
            meta.checkShape(int(dst.shape[0]))
            if int(dst.shape[1]) != self.outSamples:
                raise ValueError(f"dst must be {self.outSamples} samples wide, got {dst.shape[1]}")
        if meta.firstSample != 0:
            raise ValueError(f"correlation needs whole records from sample 0, got firstSample "
                             f"{meta.firstSample}")
        live, _ = meta.device(cols, 1, src.device.index)
        st = torch.cuda.current_stream(src.device).cuda_stream
        dptr = None if dst is None else dst.data_ptr()
        if stack is None:
            A.check(A.lib().psg_correlate(self.h, src.data_ptr(), dptr, rows, cols, live.data_ptr(),
                                          meta.dtMs, st))
        else:
            slive, _ = meta.device(self.outSamples, 0, src.device.index)
            rm = None
            if isinstance(rowMap, torch.Tensor) and rowMap.is_cuda:
                if rowMap.dtype != torch.int32 or rowMap.numel() != rows or not rowMap.is_contiguous():
                    raise ValueError(f"a device rowMap is {rows} contiguous int32 values")
                rm = rowMap
            elif rowMap is not None:
                rm = torch.as_tensor(np.asarray(rowMap, np.int32), device=src.device)
                if rm.numel() != rows:
                    raise ValueError(f"rowMap has {rm.numel()} entries for {rows} rows")
                self._rm = rm
            A.check(A.lib().psg_correlate_stack(self.h, stack.h, src.data_ptr(), dptr, rows, cols,
                                                live.data_ptr(), slive.data_ptr(),
                                                None if rm is None else rm.data_ptr(), meta.dtMs, st))


def initCorrelationPlan(T, pilot: Pilot, dtMs: float, recordSamples: int, outSamples: int = 0,
                        mode: int = A.CM_CORRELATE, epsPercent: float = 1.0,
                        normalize: bool = True) -> CorrelationPlan:
    return CorrelationPlan(T, pilot, dtMs, recordSamples, outSamples, mode, epsPercent, normalize)


class RecordStack:
    """A vertical record stack (vstack.nim:95-150, rsVertical): float64 sums
    and int32 counts on the device."""

    def __init__(self, rows: int, samples: int, dtMs: float):
        h = C.c_void_p()
        A.check(A.lib().psg_stack_create(rows, samples, dtMs, C.byref(h)))
        self.h = h
        self.rows, self.samples, self.dtMs = rows, samples, dtMs

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and A._lib is not None:
            A._lib.psg_stack_destroy(h)
            self.h = None

    def clear(self):
        import torch
        A.check(A.lib().psg_stack_clear(self.h, torch.cuda.current_stream().cuda_stream))

    def addRecord(self, b, meta: ChunkMeta, rowMap=None):
        """vstack.nim:357-380 on a CUDA tensor."""
        import torch
        rows, cols = int(b.shape[0]), int(b.shape[1])
        meta.checkShape(rows)
        if cols > self.samples:
            raise ValueError(f"the record has {cols} samples, the stack {self.samples}")
        live, _ = meta.device(cols, 0, b.device.index)
        rm = None
        if rowMap is not None:
            rm = torch.as_tensor(np.asarray(rowMap, np.int32), device=b.device)
            self._rm = rm
        dt = A.F32 if b.dtype == torch.float32 else A.F64
        A.check(A.lib().psg_stack_add(self.h, b.data_ptr(), dt, rows, cols, live.data_ptr(),
                                      None if rm is None else rm.data_ptr(),
                                      torch.cuda.current_stream(b.device).cuda_stream))

    def stackInto(self, dst, norm: int = A.FN_FOLD):
        import torch
        if tuple(dst.shape) != (self.rows, self.samples):
            raise ValueError(f"dst must be a [{self.rows}, {self.samples}] tensor, got {tuple(dst.shape)}")
        dt = A.F32 if dst.dtype == torch.float32 else A.F64
        A.check(A.lib().psg_stack_result(self.h, dst.data_ptr(), dt, norm,
                                         torch.cuda.current_stream(dst.device).cuda_stream))

    def foldInto(self, dst):
        import torch
        A.check(A.lib().psg_stack_fold(self.h, dst.data_ptr(),
                                       torch.cuda.current_stream(dst.device).cuda_stream))


def initRecordStack(rows: int, samples: int, dtMs: float) -> RecordStack:
    return RecordStack(rows, samples, dtMs)
