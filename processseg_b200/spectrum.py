"""Amplitude spectra for display (src/processSEG/fft/spectrum.nim): a
``SpectrumPlan`` windows, demeans and tapers a trace window, zero-pads it to
``nfft`` and transforms it on the device (one CTA per trace); the panel form
averages the power of the live rows (``averageAmplitudeInto``), the trace
form gives amplitude and phase (``amplitudeInto``). The dB scale and the
phase helpers are host arithmetic on a few thousand bins."""
from __future__ import annotations

import ctypes as C
import math
from typing import Sequence

import numpy as np

from . import _abi as A
from .meta import same_interval

DB_PEAK, DB_ABSOLUTE = 0, 1
dbPeak, dbAbsolute = DB_PEAK, DB_ABSOLUTE


def _torch():
    import torch
    return torch


class SpectrumPlan:
    """initSpectrumPlan (fft/spectrum.nim:79-107): ``ValueError`` for
    ``windowLen < 1``, a ``dtMs`` that is not finite and positive, a taper
    fraction outside 0 .. 0.5, or an ``nfft`` shorter than the window or not
    2·3·5-smooth."""

    def __init__(self, T, dtMs: float, windowLen: int, taperFraction: float = 0.1, nfft: int = 0,
                 demean: bool = True):
        from .plan import _dtype_code
        self.dtype = _dtype_code(T)
        h = C.c_void_p()
        A.check(A.lib().psg_spectrum_plan_create(self.dtype, float(dtMs), int(windowLen), float(taperFraction),
                                                 int(nfft), int(bool(demean)), C.byref(h)))
        self.h = h
        self._dtMs = float(dtMs)
        n, b, w, ts = C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        A.check(A.lib().psg_spectrum_plan_info(h, C.byref(n), C.byref(b), C.byref(w), C.byref(ts)))
        self.nfft, self.bins, self.windowLen, self.taperSum = n.value, b.value, w.value, ts.value

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and A._lib is not None:
            A._lib.psg_spectrum_plan_destroy(h)
            self.h = None

    @property
    def dtMs(self) -> float:
        return self._dtMs

    def binHz(self, k: int) -> float:
        """The frequency of bin ``k``: ``k / (nfft·dt)``."""
        return float(k) * 1000 / (float(self.nfft) * self._dtMs)

    def sides(self, k: int) -> float:
        """1 at 0 Hz and at Nyquist, else 2."""
        return 1.0 if k == 0 or 2 * k == self.nfft else 2.0

    def _device_block(self, b):
        torch = _torch()
        want = torch.float32 if self.dtype == A.F32 else torch.float64
        if isinstance(b, torch.Tensor):
            if b.dtype != want or not b.is_cuda or not b.is_contiguous() or b.dim() != 2:
                raise ValueError("the block must be a C-contiguous [rows, cols] CUDA tensor of the plan's dtype")
            return b
        b = np.asarray(b)
        if b.ndim != 2 or b.dtype != np.dtype(np.float32 if self.dtype == A.F32 else np.float64):
            raise ValueError("the block must be a [rows, cols] array of the plan's dtype")
        return torch.from_numpy(np.ascontiguousarray(b)).cuda()

    def averageAmplitudeInto(self, b, meta, firstCol: int, amp, ws, rows=(0, 2 ** 62)) -> int:
        """The power-averaged amplitude spectrum of the window ``firstCol ..<
        firstCol + windowLen`` of the live rows ``rows`` (inclusive, clipped)
        of ``b`` into ``amp`` (``bins`` values); returns the rows averaged
        (fft/spectrum.nim:393-416). ``ValueError`` for a block that does not
        match the meta, another interval or a negative ``firstCol``;
        ``AssertionError`` for ``len(amp) != bins``."""
        torch = _torch()
        assert len(amp) == self.bins, "amp needs bins values"
        blk = self._device_block(b)
        meta.checkShape(int(blk.shape[0]))
        if not same_interval(meta.dtMs, self._dtMs):
            raise ValueError(f"the rows' interval {meta.dtMs} ms is not the plan's {self._dtMs} ms")
        live, _ = meta.device(int(blk.shape[1]), 0, blk.device.index)
        out = torch.empty(self.bins, dtype=torch.float64, device=blk.device)
        used = torch.zeros(1, dtype=torch.int64, device=blk.device)
        st = torch.cuda.current_stream(blk.device).cuda_stream
        A.check(A.lib().psg_spectrum_average(self.h, ws.h, blk.data_ptr(), int(blk.shape[0]), int(blk.shape[1]),
                                             live.data_ptr(), meta.dtMs, int(firstCol), int(rows[0]), int(rows[1]),
                                             out.data_ptr(), used.data_ptr(), st))
        vals = out.cpu().numpy()
        for k in range(self.bins):
            amp[k] = float(vals[k])
        return int(used.item())

    def amplitudes(self, b, meta, firstCol: int, ws):
        """amplitudeInto for every row of ``b``: (amp, phase) CUDA tensors of
        rows × bins values of the plan's dtype."""
        torch = _torch()
        blk = self._device_block(b)
        meta.checkShape(int(blk.shape[0]))
        if not same_interval(meta.dtMs, self._dtMs):
            raise ValueError(f"the rows' interval {meta.dtMs} ms is not the plan's {self._dtMs} ms")
        live, _ = meta.device(int(blk.shape[1]), 0, blk.device.index)
        amp = torch.empty(int(blk.shape[0]), self.bins, dtype=blk.dtype, device=blk.device)
        phase = torch.empty_like(amp)
        st = torch.cuda.current_stream(blk.device).cuda_stream
        A.check(A.lib().psg_spectrum_amplitude(self.h, ws.h, blk.data_ptr(), int(blk.shape[0]), int(blk.shape[1]),
                                               live.data_ptr(), meta.dtMs, int(firstCol), amp.data_ptr(),
                                               phase.data_ptr(), st))
        return amp, phase

    def amplitudeInto(self, x, amp, phase, ws):
        """The scaled amplitude and the phase (radians) of one window ``x``
        (up to ``windowLen`` samples; fft/spectrum.nim:283-300)."""
        from .meta import liveMeta
        assert len(amp) == self.bins and len(phase) == self.bins, "amp and phase need bins values"
        x = np.asarray(x, dtype=np.float32 if self.dtype == A.F32 else np.float64)[:self.windowLen]
        n = int(x.size)
        row = np.zeros((1, max(n, 1)), dtype=x.dtype)
        row[0, :n] = x
        meta = liveMeta(1, n, self._dtMs)
        a, p = self.amplitudes(row, meta, 0, ws)
        a, p = a.cpu().numpy()[0], p.cpu().numpy()[0]
        for k in range(self.bins):
            amp[k] = a[k]
            phase[k] = p[k]


def initSpectrumPlan(T, dtMs: float, windowLen: int, taperFraction: float = 0.1, nfft: int = 0,
                     demean: bool = True) -> SpectrumPlan:
    return SpectrumPlan(T, dtMs, windowLen, taperFraction, nfft, demean)


def amplitudePhaseInto(re, im, amp, phase):
    """Modulus and phase (atan2(im, re)) per bin (fft/spectrum.nim:125-136)."""
    n = len(re)
    assert len(im) == n and len(amp) == n and len(phase) == n, "re, im, amp and phase need the same length"
    for k in range(n):
        amp[k] = math.hypot(float(re[k]), float(im[k]))
        phase[k] = math.atan2(float(im[k]), float(re[k]))


def toDbInto(amp, db, reference: int = DB_PEAK, floorDb: float = -120.0, refAmplitude: float = 1.0):
    """20·log10(amp/ref) per bin, clamped below at ``floorDb``
    (fft/spectrum.nim:138-160)."""
    assert len(db) == len(amp), "amp and db need the same length"
    r = refAmplitude
    if reference == DB_PEAK:
        r = 0.0
        for a in amp:
            if a > r and a < math.inf:
                r = a
    for k, a in enumerate(amp):
        v = 20 * math.log10(a / r) if (r > 0 and a > 0) else -math.inf
        db[k] = max(v, floorDb)


def _wrap_step(d: float) -> float:
    while d > 180:
        d -= 360
    while d <= -180:
        d += 360
    return d


def unwrapPhaseInto(phaseDeg: Sequence[float], shown: Sequence[bool], dst):
    """Unwraps the shown finite bins, NaN elsewhere (fft/spectrum.nim:169-191)."""
    n = len(phaseDeg)
    assert len(shown) == n and len(dst) == n, "phase, shown and dst need the same length"
    last = math.nan
    for i in range(n):
        if not shown[i] or not math.isfinite(phaseDeg[i]):
            dst[i] = math.nan
        elif math.isnan(last):
            dst[i] = phaseDeg[i]
            last = dst[i]
        else:
            dst[i] = last + _wrap_step(phaseDeg[i] - last)
            last = dst[i]


def circularMeanDeg(angles: Sequence[float]):
    """(meanDeg, resultant) of angles in degrees (fft/spectrum.nim:193-216)."""
    sx = sy = 0.0
    n = 0
    for v in angles:
        if math.isfinite(v):
            sx += math.cos(math.radians(v))
            sy += math.sin(math.radians(v))
            n += 1
    if n == 0:
        return math.nan, 0.0
    res = min(math.hypot(sx, sy) / n, 1.0)
    if abs(sx) < 1e-12 and abs(sy) < 1e-12:
        return math.nan, res
    m = math.degrees(math.atan2(sy, sx))
    if m <= -180:
        m += 360
    return m, res


def removeDelayInto(unwrapped, hz, shown, dst) -> float:
    """Removes the least-squares line of the drawn finite bins; returns the
    delay in ms (fft/spectrum.nim:218-257)."""
    n = len(unwrapped)
    assert len(hz) == n and len(shown) == n and len(dst) == n, "phase, hz, shown and dst need the same length"
    cnt = 0
    sf = sf2 = sp = spf = 0.0
    ok = [bool(shown[i]) and math.isfinite(unwrapped[i]) and math.isfinite(hz[i]) for i in range(n)]
    for i in range(n):
        if ok[i]:
            f, p = hz[i], unwrapped[i]
            sf += f
            sf2 += f * f
            sp += p
            spf += p * f
            cnt += 1
    den = cnt * sf2 - sf * sf
    if cnt < 2 or abs(den) < 1e-12 * max(1.0, sf2):
        for i in range(n):
            dst[i] = math.nan
        return math.nan
    a = (sp * sf2 - sf * spf) / den
    b = (cnt * spf - sf * sp) / den
    for i in range(n):
        dst[i] = unwrapped[i] - (a + b * hz[i]) if ok[i] else math.nan
    return -b * 1000 / 360
