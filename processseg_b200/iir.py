"""``IirPlan`` (src/processSEG/filter/iir.nim): Butterworth biquad cascades,
zero phase (forward-backward, gain |H|² = the spec's response) or minimum
phase (one causal pass, gain |H|), with the FFT filters' edge handling. The
design (sections, margin, 0 Hz gain, magnitude) runs on the host in
``libpsgcuda.so``; applying one runs it as the ``iirOp`` step of a
one-op pipeline on the device."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A
from .design import FilterSpec


class IirPlan:
    """initIirPlan (filter/iir.nim:193-239): ``ValueError`` for a spec that is
    not Butterworth, has notches or 0 Hz suppression, or a slope that is not
    a multiple of 12 dB/octave (zero phase) or 6 (minimum phase)."""

    def __init__(self, T, spec: FilterSpec, dtMs: float, samples: int, phase: int = A.IP_ZERO,
                 trend: int = A.TR_LINEAR):
        from .plan import _dtype_code
        self.dtype = _dtype_code(T)
        self.spec, self.dtMs, self.samples = spec, float(dtMs), int(samples)
        self.phase, self.trend = int(phase), int(trend)
        order, margin, g = C.c_int32(), C.c_int32(), C.c_double()
        c = spec.to_c()
        A.check(A.lib().psg_iir_design(C.byref(c), self.dtMs, self.samples, self.phase, self.trend,
                                       C.byref(order), C.byref(margin), C.byref(g)))
        self.order, self.requiredMargin, self.dcGain = order.value, margin.value, g.value
        self._plan = None

    def magnitudeAt(self, f):
        """|H| (minimum phase) or |H|² (zero phase) at ``f`` Hz (a number or
        an array)."""
        fa = np.ascontiguousarray(np.atleast_1d(np.asarray(f, dtype=np.float64)))
        out = np.zeros(fa.size)
        c = self.spec.to_c()
        A.check(A.lib().psg_iir_magnitude(C.byref(c), self.dtMs, self.phase, fa.ctypes.data, fa.size,
                                          out.ctypes.data))
        return float(out[0]) if np.ndim(f) == 0 else out

    def applyFilter(self, b, meta, ws):
        """The filter on the live rows of ``b`` in place, each to its live
        length (filter/iir.nim:435-480), as a one-op plan on the device."""
        if self._plan is None:
            from .ops import iirOp, initPipeline
            self._plan = initPipeline([iirOp(self.spec, self.phase, self.trend)]).compile(
                self.dtype, self.dtMs, self.samples)
        ws.reserve(self._plan, rows=int(b.shape[0]), cols=int(b.shape[1]))
        self._plan.apply(b, meta, ws)


def initIirPlan(T, spec: FilterSpec, dtMs: float, samples: int, phase: int = A.IP_ZERO,
                trend: int = A.TR_LINEAR) -> IirPlan:
    return IirPlan(T, spec, dtMs, samples, phase, trend)
