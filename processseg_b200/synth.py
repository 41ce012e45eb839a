"""Seeded synthetic gathers for tests and benchmarks, following the
generator semantics of src/processSEG/synth.nim: Ricker wavelets
``(1 − 2a)·e^(−a)``, ``a = (π f τ)²``, added within ±3000/f ms of their
centre (synth.nim:57-96), on hyperbolic moveout ``t = √(t0² + (x/v)²)``
(synth.nim:146-148), plus Gaussian noise, a DC offset and a sinusoid.

The reference's noise comes from Nim's ``std/random`` and is not
reproducible outside Nim (synth.nim:28-43); these generators use numpy's
PCG64 seeded per (workload, seed), identical for the oracle, the CPU
baseline and the GPU runs of one process.
"""
from __future__ import annotations

import math
from typing import Optional
from dataclasses import dataclass

import numpy as np

from . import _abi as A


def rng_for(workload: str, seed: int) -> np.random.Generator:
    tag = int.from_bytes(workload.encode()[:8].ljust(8, b"\0"), "little")
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence([tag, seed])))


def ricker(tau_ms, freq_hz):
    a = (math.pi * freq_hz * tau_ms / 1000.0) ** 2
    return (1 - 2 * a) * np.exp(-a)


def add_hyperbolas(x, dtMs, offsets, t0s, amps, freq=25.0, velocity=2000.0, live=None):
    """Adds one Ricker event per (t0, amp) on each row at its offset, within
    ±3000/f ms of the centre and inside the row's live length."""
    rows, cols = x.shape
    half = 3000.0 / freq
    hw = int(math.ceil(half / dtMs)) + 1
    r_idx = np.arange(rows)
    for t0, amp in zip(t0s, amps):
        centre = np.sqrt(t0 ** 2 + (np.abs(offsets) / velocity * 1000.0) ** 2)  # ms
        c0 = np.floor(centre / dtMs).astype(np.int64)
        j = c0[:, None] + np.arange(-hw, hw + 1)[None, :]
        tau = j * dtMs - centre[:, None]
        lim = cols if live is None else live[:, None]
        ok = (j >= 0) & (j < lim) & (np.abs(tau) <= half)
        vals = np.where(ok, amp * ricker(tau, freq), 0.0)
        jj = np.clip(j, 0, cols - 1)
        np.add.at(x, (np.repeat(r_idx, j.shape[1]).reshape(j.shape), jj), vals)


@dataclass
class Gather:
    data: np.ndarray        # [rows, cols]
    status: np.ndarray      # int32 per row
    numSamples: np.ndarray  # int32 per row
    t0Ms: np.ndarray        # float64 per row
    dtMs: float
    failed: np.ndarray      # ascending int64
    offsets: Optional[np.ndarray] = None  # float64 per row (NaN: unknown)

    def meta(self, firstSample=0):
        from .meta import initChunkMeta
        return initChunkMeta(self.status, self.numSamples, self.dtMs, self.t0Ms, firstSample,
                             self.failed, self.offsets)


def shot_gather(rows, cols, dtMs, seed, dtype=np.float32, live_range=None, sine_hz=None,
                sine_amp=0.3, noise=0.1, events=5, workload="gather", channels=240, row0=0):
    """A gather of ``rows`` traces: ``events`` Rickers (25 Hz) on hyperbolas,
    t0 ~ U(200, 3500) ms, amp ~ N(0, 1), offsets 25 m × ((row0 + row) mod channels);
    noise N(0, σ); a DC offset U(−0.5, 0.5) per trace; optional sinusoid;
    live lengths U{live_range} with zeros past them."""
    g = rng_for(workload, seed)
    t0s = g.uniform(200.0, 3500.0, events)
    amps = g.standard_normal(events)
    offsets = 25.0 * ((row0 + np.arange(rows)) % channels)
    if live_range is None:
        live = np.full(rows, cols, np.int64)
    else:
        live = g.integers(live_range[0], live_range[1] + 1, rows)
    x = np.zeros((rows, cols), np.float64)
    add_hyperbolas(x, dtMs, offsets, t0s, amps, live=live)
    x += g.standard_normal((rows, cols)) * noise
    x += g.uniform(-0.5, 0.5, rows)[:, None]
    if sine_hz is not None:
        t = np.arange(cols) * dtMs / 1000.0
        x += sine_amp * np.sin(2 * math.pi * sine_hz * t)[None, :]
    mask = np.arange(cols)[None, :] < live[:, None]
    x = np.where(mask, x, 0.0).astype(dtype)
    return Gather(np.ascontiguousarray(x), np.full(rows, A.TS_LIVE, np.int32),
                  live.astype(np.int32), np.zeros(rows), float(dtMs), np.zeros(0, np.int64),
                  offsets.astype(np.float64))


def c1(seed=1, dtype=np.float32):
    """48 traces × 2001 samples at 2 ms, all live."""
    return shot_gather(48, 2001, 2.0, seed, dtype, workload="c1")


def c2(seed=2, dtype=np.float32, rows=2000):
    """2000 traces × 3001 samples at 2 ms, live U{1500..3001}, 50 Hz sine."""
    return shot_gather(rows, 3001, 2.0, seed, dtype, live_range=(1500, 3001), sine_hz=50.0,
                       workload="c2")


def c5(seed=5, dtype=np.float32, rows=50000, shot=5000):
    """50000 traces × 6001 samples at 1 ms, live U{4000..6001}: consecutive
    shot gathers of ``shot`` traces, each with its own events and noise
    (seeded per shot), generated one at a time."""
    out = None
    for k, a in enumerate(range(0, rows, shot)):
        n = min(shot, rows - a)
        g = shot_gather(n, 6001, 1.0, seed * 65536 + k, dtype, live_range=(4000, 6001), workload="c5",
                        row0=a)
        if out is None:
            out = Gather(np.empty((rows, 6001), dtype), np.empty(rows, np.int32), np.empty(rows, np.int32),
                         np.zeros(rows), 1.0, np.zeros(0, np.int64))
        out.data[a:a + n] = g.data
        out.status[a:a + n] = g.status
        out.numSamples[a:a + n] = g.numSamples
    return out


def vibroseis_records(pilot, channels=240, samples=10001, sweeps=4, seed=3, p=0.02, noise=0.05,
                      dtype=np.float32):
    """Per channel a reflectivity series (Bernoulli(p) × N(0, 1)) convolved
    with the pilot (truncated to ``samples``), one record per sweep with
    independent N(0, noise) noise: an array [sweeps, channels, samples]."""
    g = rng_for("c3", seed)
    refl = (g.random((channels, samples)) < p) * g.standard_normal((channels, samples))
    n = 1
    while n < samples + pilot.size:
        n *= 2
    conv = np.fft.irfft(np.fft.rfft(refl, n) * np.fft.rfft(pilot.astype(np.float64), n)[None, :], n)
    conv = conv[:, :samples]
    out = np.empty((sweeps, channels, samples), dtype)
    for s in range(sweeps):
        out[s] = conv + noise * g.standard_normal((channels, samples))
    return out


# ------------------------------------------------------------ viewer load
def viewer_flows():
    """The three plans of the served viewer load: band-pass 4-8-60-80 + AGC
    500 ms; band-pass + RMS normalization per trace; Butterworth 5-100 Hz
    (24 dB/octave effective slope, 4 poles) + t² gain."""
    from . import (Corners, agcOp, bandPassOp, butterBandPass, filterOp, gainCurveOp,
                   normalizeOp, normRms, powerGain)
    bp = Corners(4, 8, 60, 80)
    return [[bandPassOp(bp), agcOp(500)],
            [bandPassOp(bp), normalizeOp(normRms)],
            [filterOp(butterBandPass(5, 100, 24)), gainCurveOp(powerGain(2))]]


@dataclass
class ViewerRequest:
    arrival_s: float
    flow: int        # index into viewer_flows()
    rows: int
    first: int       # decode window within the record
    cols: int


def viewer_requests(n, rate_hz=2000.0, record=6001, dtMs=2.0, seed=4, margins=None):
    """``n`` requests of the served viewer load: Poisson arrivals at
    ``rate_hz``, trace counts log-uniform in 48 .. 5000, shown windows
    log-uniform in 200 .. 4000 samples placed uniformly in the record, decoded
    with each plan's margin (decodeWindow), plans drawn uniformly."""
    from .ops import decodeWindow
    g = rng_for("c4", seed)
    t = np.cumsum(g.exponential(1.0 / rate_hz, n))
    out = []
    for i in range(n):
        flow = int(g.integers(0, 3))
        rows = int(round(math.exp(g.uniform(math.log(48), math.log(5000)))))
        width = int(round(math.exp(g.uniform(math.log(200), math.log(4000)))))
        a = int(g.integers(0, record - width + 1))
        m = margins[flow] if margins is not None else 0
        lo, hi = decodeWindow(a, a + width - 1, m, record)
        out.append(ViewerRequest(float(t[i]), flow, rows, lo, hi - lo + 1))
    return out
