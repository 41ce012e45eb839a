"""Filter responses and gain curves as plain data: the host side of
src/processSEG/filter/design.nim and gain/curves.nim.

The builders check their arguments as the reference's builders do
(``checkCorners``, ``checkButter``, ``checkNotch``: design.nim:103-137;
``knotGain``/``powerGain``/``exponentialGain``: curves.nim:97-126) and raise
``ValueError``. Everything else (validation against an interval, responses,
impulse lengths) runs in the library at ``compile``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import List, Sequence

from . import _abi as A

INF = math.inf


@dataclass(frozen=True)
class Corners:
    """The corners of a cos² trapezoid in Hz, ``f1 < f2 ≤ f3 < f4``
    (design.nim:63-67). ``f2 = 0``: no low cut; ``f3 = Inf``: no high cut."""
    f1: float = 0.0
    f2: float = 0.0
    f3: float = INF
    f4: float = INF


@dataclass(frozen=True)
class Notch:
    freqHz: float
    widthHz: float


@dataclass(frozen=True)
class FilterSpec:
    """A zero-phase response (design.nim:78-91)."""
    kind: int = A.RK_TRAPEZOID
    corners: Corners = Corners()
    lowHz: float = 0.0
    lowSlope: float = 24.0
    highHz: float = INF
    highSlope: float = 24.0
    notches: tuple = ()
    zeroDc: bool = False

    def to_c(self) -> A.FilterSpecC:
        s = A.FilterSpecC()
        s.kind = self.kind
        s.zero_dc = 1 if self.zeroDc else 0
        if len(self.notches) > A.MAX_NOTCHES:
            raise ValueError(f"at most {A.MAX_NOTCHES} notches, got {len(self.notches)}")
        s.n_notches = len(self.notches)
        c = self.corners
        s.f1, s.f2, s.f3, s.f4 = c.f1, c.f2, c.f3, c.f4
        s.low_hz, s.low_slope = self.lowHz, self.lowSlope
        s.high_hz, s.high_slope = self.highHz, self.highSlope
        for i, n in enumerate(self.notches):
            s.notches[i].freq_hz = n.freqHz
            s.notches[i].width_hz = n.widthHz
        return s

    def withNotch(self, freqHz: float, widthHz: float) -> "FilterSpec":
        """``spec`` with a notch at ``freqHz`` (design.nim:212-218)."""
        _checkNotch(freqHz, widthHz)
        return replace(self, notches=self.notches + (Notch(freqHz, widthHz),))

    def withZeroDc(self) -> "FilterSpec":
        """``spec`` with bin 0 set to 0 when applied (design.nim:220-223)."""
        return replace(self, zeroDc=True)

    def response(self, f: float, dtMs: float) -> float:
        """The gain at ``f`` Hz (design.nim:236-255), computed by the library."""
        import ctypes as C
        out = C.c_double()
        A.check(A.lib().psg_response(C.byref(self.to_c()), f, dtMs, C.byref(out)))
        return out.value

    def impulseLength(self, dtMs: float) -> int:
        """The 99.9 %-energy half length L (design.nim:353-366)."""
        import ctypes as C
        out = C.c_int32()
        A.check(A.lib().psg_impulse_length(C.byref(self.to_c()), dtMs, C.byref(out)))
        return out.value


def _checkCorners(c: Corners):
    # design.nim:103-115
    for f in (c.f1, c.f2, c.f3, c.f4):
        if math.isnan(f):
            raise ValueError(f"a corner is NaN: {c}")
    hasLow, hasHigh = c.f2 > 0, c.f3 < INF
    if hasLow and not (c.f1 >= 0 and c.f1 < c.f2):
        raise ValueError(f"a low cut needs 0 ≤ f1 < f2 (a sloped ramp), got {c}")
    if not hasLow and (c.f1 != 0 or c.f2 != 0):
        raise ValueError(f"no low cut needs f1 = f2 = 0, got {c}")
    if hasHigh and not (c.f3 < c.f4 and c.f4 < INF):
        raise ValueError(f"a high cut needs f3 < f4 < Inf (a sloped ramp), got {c}")
    if not hasHigh and c.f4 != INF:
        raise ValueError(f"no high cut needs f3 = f4 = Inf, got {c}")
    if hasLow and hasHigh and not (c.f2 <= c.f3):
        raise ValueError(f"a band-pass needs f2 ≤ f3, got {c}")


def _checkSlope(s):
    if not (s > 0 and s < INF):
        raise ValueError(f"a slope must be finite and > 0 dB/octave, got {s}")


def _checkButter(lowHz, lowSlope, highHz, highSlope):
    # design.nim:121-131
    if not (lowHz >= 0 and lowHz < INF):
        raise ValueError(f"a low-cut corner must be finite and ≥ 0 (0: none), got {lowHz}")
    if not (highHz > 0):
        raise ValueError(f"a high-cut corner must be > 0 (Inf: none), got {highHz}")
    if lowHz > 0:
        _checkSlope(lowSlope)
    if highHz < INF:
        _checkSlope(highSlope)
    if not (lowHz < highHz):
        raise ValueError(f"the low-cut corner must be below the high-cut one, got {lowHz} and {highHz}")


def _checkNotch(freqHz, widthHz):
    if not (freqHz > 0 and freqHz < INF):
        raise ValueError(f"a notch frequency must be finite and > 0, got {freqHz}")
    if not (widthHz > 0 and widthHz < INF):
        raise ValueError(f"a notch width must be finite and > 0, got {widthHz}")


def bandPass(c: Corners) -> FilterSpec:
    """A cos² trapezoid band-pass, low-cut or high-cut (design.nim:177-181)."""
    _checkCorners(c)
    return FilterSpec(kind=A.RK_TRAPEZOID, corners=c)


def lowCut(f1: float, f2: float) -> FilterSpec:
    return bandPass(Corners(f1, f2, INF, INF))


def highCut(f3: float, f4: float) -> FilterSpec:
    return bandPass(Corners(0.0, 0.0, f3, f4))


def butterBandPass(lowHz: float, highHz: float, slopeDbPerOctave: float = 24.0,
                   highSlopeDbPerOctave: float = math.nan) -> FilterSpec:
    """A Butterworth band-pass with −6 dB corners (design.nim:191-200)."""
    hs = slopeDbPerOctave if math.isnan(highSlopeDbPerOctave) else highSlopeDbPerOctave
    _checkButter(lowHz, slopeDbPerOctave, highHz, hs)
    return FilterSpec(kind=A.RK_BUTTERWORTH, lowHz=lowHz, lowSlope=slopeDbPerOctave,
                      highHz=highHz, highSlope=hs)


def butterLowCut(hz: float, slopeDbPerOctave: float = 24.0) -> FilterSpec:
    if not (hz > 0):
        raise ValueError(f"a low-cut corner must be > 0, got {hz}")
    return butterBandPass(hz, INF, slopeDbPerOctave, slopeDbPerOctave)


def butterHighCut(hz: float, slopeDbPerOctave: float = 24.0) -> FilterSpec:
    if not (hz < INF):
        raise ValueError(f"a high-cut corner must be finite, got {hz}")
    return butterBandPass(0.0, hz, slopeDbPerOctave, slopeDbPerOctave)


# ---------------------------------------------------------------- gain curves

@dataclass(frozen=True)
class GainKnot:
    tMs: float
    dB: float


@dataclass(frozen=True)
class GainCurve:
    """A gain against time (curves.nim:71-80); build it with ``knotGain``,
    ``powerGain`` or ``exponentialGain``."""
    kind: int
    knots: tuple = ()
    power: float = 0.0
    refMs: float = 1000.0
    minMs: float = 1.0
    dbPerS: float = 0.0

    def to_c(self) -> A.GainCurveC:
        c = A.GainCurveC()
        c.kind = self.kind
        if len(self.knots) > A.MAX_KNOTS:
            raise ValueError(f"at most {A.MAX_KNOTS} knots, got {len(self.knots)}")
        c.n_knots = len(self.knots)
        for i, k in enumerate(self.knots):
            c.knots[i].t_ms = k.tMs
            c.knots[i].db = k.dB
        c.power, c.ref_ms, c.min_ms, c.db_per_s = self.power, self.refMs, self.minMs, self.dbPerS
        return c

    def gainDbAt(self, tMs: float) -> float:
        """curves.nim:132-152."""
        if math.isnan(tMs):
            return math.nan
        if self.kind == A.GC_KNOTS:
            k = self.knots
            if not k:
                return math.nan
            if tMs <= k[0].tMs:
                return k[0].dB
            if tMs >= k[-1].tMs:
                return k[-1].dB
            lo, hi = 0, len(k) - 1
            while hi - lo > 1:
                mid = (lo + hi) >> 1
                if k[mid].tMs <= tMs:
                    lo = mid
                else:
                    hi = mid
            f = (tMs - k[lo].tMs) / (k[hi].tMs - k[lo].tMs)
            return k[lo].dB + f * (k[hi].dB - k[lo].dB)
        if self.kind == A.GC_POWER:
            return 20 * self.power * math.log10(max(tMs, self.minMs) / self.refMs)
        return self.dbPerS * tMs / 1000

    def factorAt(self, tMs: float) -> float:
        """curves.nim:154-160."""
        if math.isnan(tMs):
            return math.nan
        if self.kind == A.GC_POWER:
            return math.pow(max(tMs, self.minMs) / self.refMs, self.power)
        return math.pow(10.0, self.gainDbAt(tMs) / 20)


def _fin(x):
    return math.isfinite(x)


def knotGain(knots: Sequence[GainKnot]) -> GainCurve:
    if len(knots) == 0:
        raise ValueError("a knot gain needs at least one knot")
    for i, k in enumerate(knots):
        if not (_fin(k.tMs) and _fin(k.dB)):
            raise ValueError(f"knot {i} is not finite: {k}")
        if i > 0 and not (k.tMs > knots[i - 1].tMs):
            raise ValueError(f"knot times must strictly increase: {knots[i - 1].tMs} ms is followed "
                             f"by {k.tMs} ms")
    return GainCurve(kind=A.GC_KNOTS, knots=tuple(knots))


def powerGain(power: float, refMs: float = 1000.0, minMs: float = 1.0) -> GainCurve:
    if not _fin(power):
        raise ValueError(f"a power must be finite, got {power}")
    if not (_fin(refMs) and refMs > 0):
        raise ValueError(f"refMs must be finite and positive, got {refMs}")
    if not (_fin(minMs) and minMs > 0):
        raise ValueError(f"minMs must be finite and positive, got {minMs}")
    return GainCurve(kind=A.GC_POWER, power=power, refMs=refMs, minMs=minMs)


def exponentialGain(dbPerS: float) -> GainCurve:
    if not _fin(dbPerS):
        raise ValueError(f"dbPerS must be finite, got {dbPerS}")
    return GainCurve(kind=A.GC_EXPONENTIAL, dbPerS=dbPerS)
