"""Ops and pipelines as plain data: the host side of
src/processSEG/pipeline.nim:92-380.

An ``Op`` holds its kind and the parameters of that kind; a ``Pipeline`` is an
ordered, editable list of them. Nothing is validated until ``compile``
(pipeline.nim:27-34), except what the reference's builders check themselves
(``bandPassOp`` checks its corners). Asking an op for the parameters of
another kind raises ``ValueError`` (pipeline.nim:222-254).
"""
from __future__ import annotations

import copy
import math
from dataclasses import dataclass, field
from typing import Iterable, List, Optional

from . import _abi as A
from .design import Corners, FilterSpec, GainCurve, bandPass
from .mute import MuteCurve


@dataclass
class FilterParams:
    spec: FilterSpec
    trend: int = A.TR_LINEAR


@dataclass
class IirParams:
    """An ``opIir``: a Butterworth spec, the phase and the trend removal
    (pipeline.nim:133-137)."""
    spec: FilterSpec
    phase: int = A.IP_ZERO
    trend: int = A.TR_LINEAR


@dataclass
class AgcParams:
    windowMs: float
    mode: int = A.AGC_RMS
    target: float = 1.0
    epsilon: float = 1e-9


@dataclass
class NormalizeParams:
    stat: int
    scope: int = A.PER_TRACE
    target: float = 1.0
    percentile: float = 99.0


@dataclass
class ClipParams:
    lo: float
    hi: float


@dataclass
class MuteParams:
    """An ``opMuteTop`` / ``opMuteBottom``: the mute time per offset and the
    taper on the muted side (pipeline.nim:121-125)."""
    curve: MuteCurve
    taperMs: float = 0.0


@dataclass
class GainCurveParams:
    curve: GainCurve
    tMinMs: float = 0.0
    tMaxMs: float = math.nan


class Op:
    """One operation of a ``Pipeline`` (pipeline.nim:158-174)."""

    __slots__ = ("_kind", "_p")

    def __init__(self, kind: int, params=None):
        self._kind = kind
        self._p = params

    @property
    def kind(self) -> int:
        return self._kind

    def _get(self, kinds, what):
        if self._kind not in kinds:
            raise ValueError(f"the op is {A.OP_NAMES[self._kind]}: it has no {what} "
                             "(check `op.kind` first)")
        return self._p

    @property
    def factor(self) -> float:
        return self._get((A.OP_SCALE,), "factor")

    @property
    def dB(self) -> float:
        return self._get((A.OP_GAIN_DB,), "gain in dB")

    @property
    def clip(self) -> ClipParams:
        return self._get((A.OP_CLIP,), "clip limits")

    @property
    def filter(self) -> FilterParams:
        return self._get((A.OP_FILTER,), "FFT filter")

    @property
    def iir(self) -> IirParams:
        return self._get((A.OP_IIR,), "IIR filter")

    @property
    def agc(self) -> AgcParams:
        return self._get((A.OP_AGC,), "AGC")

    @property
    def norm(self) -> NormalizeParams:
        return self._get((A.OP_NORMALIZE,), "normalization")

    @property
    def gainCurve(self) -> GainCurveParams:
        return self._get((A.OP_GAIN_CURVE,), "gain curve")

    @property
    def mute(self) -> MuteParams:
        return self._get((A.OP_MUTE_TOP, A.OP_MUTE_BOTTOM), "mute")

    def __repr__(self):
        return f"Op({A.OP_NAMES[self._kind]}, {self._p!r})"

    def __eq__(self, other):
        return isinstance(other, Op) and self._kind == other._kind and self._p == other._p

    def to_c(self) -> A.OpC:
        o = A.OpC()
        o.kind = self._kind
        o.trend = A.TR_LINEAR
        o.t_max_ms = math.nan
        p = self._p
        k = self._kind
        if k in (A.OP_SCALE, A.OP_GAIN_DB):
            o.factor = float(p)
        elif k == A.OP_CLIP:
            o.lo, o.hi = float(p.lo), float(p.hi)
        elif k == A.OP_FILTER:
            o.filter = p.spec.to_c()
            o.trend = int(p.trend)
        elif k == A.OP_IIR:
            o.filter = p.spec.to_c()
            o.trend = int(p.trend)
            o.iir_phase = int(p.phase)
        elif k == A.OP_AGC:
            o.window_ms, o.agc_mode, o.target, o.epsilon = p.windowMs, int(p.mode), p.target, p.epsilon
        elif k == A.OP_NORMALIZE:
            o.norm_stat, o.norm_scope = int(p.stat), int(p.scope)
            o.norm_target, o.percentile = p.target, p.percentile
        elif k == A.OP_GAIN_CURVE:
            o.curve = p.curve.to_c()
            o.t_min_ms, o.t_max_ms = p.tMinMs, p.tMaxMs
        elif k in (A.OP_MUTE_TOP, A.OP_MUTE_BOTTOM):
            o.mute = p.curve.to_c()
            o.taper_ms = p.taperMs
        return o


# ------------------------------------------------------------------ builders
def demeanOp() -> Op:
    return Op(A.OP_DEMEAN)


def detrendOp() -> Op:
    return Op(A.OP_DETREND)


def scaleOp(factor: float) -> Op:
    return Op(A.OP_SCALE, float(factor))


def gainDbOp(dB: float) -> Op:
    return Op(A.OP_GAIN_DB, float(dB))


def clipOp(lo: float, hi: float) -> Op:
    return Op(A.OP_CLIP, ClipParams(float(lo), float(hi)))


def polarityOp() -> Op:
    return Op(A.OP_POLARITY)


def muteTopOp(curve: MuteCurve, taperMs: float = 0.0) -> Op:
    """Zeroes each trace before its ``curve`` time, with a taper of
    ``taperMs`` on the muted side (pipeline.nim:282-285)."""
    return Op(A.OP_MUTE_TOP, MuteParams(curve, float(taperMs)))


def muteBottomOp(curve: MuteCurve, taperMs: float = 0.0) -> Op:
    """Zeroes each trace after its ``curve`` time (pipeline.nim:287-289)."""
    return Op(A.OP_MUTE_BOTTOM, MuteParams(curve, float(taperMs)))


def filterOp(spec: FilterSpec, trend: int = A.TR_LINEAR) -> Op:
    return Op(A.OP_FILTER, FilterParams(spec, trend))


def bandPassOp(corners: Corners, trend: int = A.TR_LINEAR) -> Op:
    """``filterOp(bandPass(corners))``; ``ValueError`` for bad corners
    (pipeline.nim:295-298)."""
    return filterOp(bandPass(corners), trend)


def iirOp(spec: FilterSpec, phase: int = A.IP_ZERO, trend: int = A.TR_LINEAR) -> Op:
    """A Butterworth biquad cascade (``IirPlan``, filter/iir.nim): zero phase
    (forward-backward) or minimum phase (one causal pass), with the edge
    handling of the FFT filters (pipeline.nim:300-303)."""
    return Op(A.OP_IIR, IirParams(spec, phase, trend))


def agcOp(windowMs: float, mode: int = A.AGC_RMS, target: float = 1.0,
          epsilon: float = 1e-9) -> Op:
    return Op(A.OP_AGC, AgcParams(float(windowMs), mode, float(target), float(epsilon)))


def normalizeOp(stat: int, scope: int = A.PER_TRACE, target: float = 1.0,
                percentile: float = 99.0) -> Op:
    return Op(A.OP_NORMALIZE, NormalizeParams(stat, scope, float(target), float(percentile)))


def gainCurveOp(curve: GainCurve, tMinMs: float = 0.0, tMaxMs: float = math.nan) -> Op:
    return Op(A.OP_GAIN_CURVE, GainCurveParams(curve, float(tMinMs), float(tMaxMs)))


# ------------------------------------------------------------------ pipeline
class Pipeline:
    """An ordered list of ``Op``s (pipeline.nim:176-380)."""

    def __init__(self, ops: Iterable[Op] = ()):
        self._ops: List[Op] = list(ops)

    def __len__(self):
        return len(self._ops)

    def __getitem__(self, i) -> Op:
        return self._ops[i]

    def __setitem__(self, i, op: Op):
        self._ops[i] = op

    def __iter__(self):
        return iter(self._ops)

    def add(self, op: Op):
        self._ops.append(op)

    def insert(self, op: Op, i: int):
        self._ops.insert(i, op)

    def delete(self, i: int):
        del self._ops[i]

    def clear(self):
        self._ops.clear()

    def copy(self) -> "Pipeline":
        return Pipeline(copy.deepcopy(self._ops))

    def c_ops(self):
        return A.ops_array(self._ops)

    def compile(self, T, dtMs: float, samples: int, recordSamples: int = 0):
        """Validates and precomputes the pipeline (pipeline.nim:466-523); see
        ``plan.compile``."""
        from .plan import compile as _compile
        return _compile(self, T, dtMs, samples, recordSamples)

    def requiredMargin(self, dtMs: float) -> int:
        """The plan's margin without compiling (pipeline.nim:525-548)."""
        import ctypes as C
        out = C.c_int32()
        arr = self.c_ops()
        A.check(A.lib().psg_required_margin(arr, len(self._ops), dtMs, C.byref(out)))
        return out.value

    def appliedResponseInto(self, T, dtMs: float, samples: int, hz, gain, ws) -> None:
        """The response of the flow as applied (pipeline.nim:840-880): a
        unit impulse at sample ``samples // 2`` of one live row at t0 = 0
        runs through the compiled plan on the device, with every filter's
        trend removal off (this pipeline is not changed), and ``gain[i]``
        receives ``|Σ x[j] exp(−2πi·hz[i]·j·dt)|`` of the output, in float64.
        ``ValueError`` when the flow does not compile; ``AssertionError``
        when ``hz`` and ``gain`` differ in length. Compiles a plan on every
        call; ``ws`` (a ``Workspace``) is grown to it when needed."""
        import numpy as np
        from .plan import _dtype_code
        hz_a = np.ascontiguousarray(np.asarray(hz, dtype=np.float64).reshape(-1))
        assert len(gain) == len(hz_a), "hz and gain need the same length"
        out = np.zeros(len(hz_a), dtype=np.float64)
        A.check(A.lib().psg_applied_response(self.c_ops(), len(self._ops), _dtype_code(T), float(dtMs),
                                             int(samples), hz_a.ctypes.data, len(hz_a), out.ctypes.data, ws.h))
        for i in range(len(out)):
            gain[i] = float(out[i])


def initPipeline(ops: Iterable[Op] = ()) -> Pipeline:
    return Pipeline(ops)


def decodeWindow(shown_first: int, shown_last: int, margin: int, traceLen: int):
    """``shown`` widened by ``margin`` on each side and clamped to
    ``0 ..< traceLen`` (pipeline.nim:550-560): returns ``(first, last)``."""
    m = min(max(margin, 0), max(traceLen, 0))
    return max(0, shown_first - m), min(traceLen - 1, shown_last + m)
