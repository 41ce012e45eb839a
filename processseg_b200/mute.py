"""Mute curves (src/processSEG/core/mute.nim:29-123): the time of a top or
bottom mute per trace, as ``muteTopOp`` / ``muteBottomOp`` take it.

A time is in trace ms, on the axis of ``ChunkMeta`` (column ``j`` of row
``r`` is at ``t0Ms[r] + (firstSample + j)·dtMs``). ``timeMute``: one time for
every trace; ``tableMute``: linear in ``|offset|`` between knots, flat beyond
them; ``lmoMute``: ``t0Ms + |offset|/velocity + padMs``. The builders raise
``ValueError`` for what the reference's builders reject.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Sequence

from . import _abi as A


def _finite(x: float) -> bool:
    return math.isfinite(x)


@dataclass(frozen=True)
class MuteCurve:
    """MuteCurve (core/mute.nim:37-49). Build one with ``timeMute``,
    ``tableMute`` or ``lmoMute``."""
    kind: int
    tMs: float = 0.0
    offsets: tuple = ()
    timesMs: tuple = ()
    velocity: float = 0.0
    msPerDist: float = 0.0
    t0Ms: float = 0.0
    padMs: float = 0.0

    def muteTimeMs(self, offset: float) -> float:
        """The mute time in ms of a trace at ``offset`` (``|offset|`` is
        used); NaN when the curve needs the offset and it is NaN
        (core/mute.nim:103-123)."""
        if self.kind == A.MK_TIME:
            return self.tMs
        if self.kind == A.MK_LMO:
            return self.t0Ms + abs(offset) * self.msPerDist + self.padMs
        x = abs(offset)
        if math.isnan(x):
            return math.nan
        off, tm = self.offsets, self.timesMs
        last = len(off) - 1
        if x <= off[0]:
            return tm[0]
        if x >= off[last]:
            return tm[last]
        lo, hi = 0, last
        while hi - lo > 1:
            mid = (lo + hi) >> 1
            if off[mid] <= x:
                lo = mid
            else:
                hi = mid
        u = (x - off[lo]) / (off[hi] - off[lo])
        return tm[lo] + u * (tm[hi] - tm[lo])

    def to_c(self) -> A.MuteCurveC:
        c = A.MuteCurveC()
        c.kind = self.kind
        c.t_ms = self.tMs
        c.velocity, c.t0_ms, c.pad_ms = self.velocity, self.t0Ms, self.padMs
        c.n_knots = len(self.offsets)
        for i, (o, t) in enumerate(zip(self.offsets, self.timesMs)):
            c.offsets[i] = o
            c.times_ms[i] = t
        return c


def timeMute(tMs: float) -> MuteCurve:
    """A mute at ``tMs`` on every trace (core/mute.nim:55-59)."""
    if not _finite(tMs):
        raise ValueError(f"a mute time must be finite, got {tMs}")
    return MuteCurve(A.MK_TIME, tMs=float(tMs))


def tableMute(offsets: Sequence[float], timesMs: Sequence[float]) -> MuteCurve:
    """A mute interpolated linearly in ``|offset|`` between the knots, flat
    beyond them (core/mute.nim:61-82)."""
    offsets = [float(o) for o in offsets]
    timesMs = [float(t) for t in timesMs]
    if len(offsets) == 0:
        raise ValueError("a mute table needs at least one knot")
    if len(offsets) != len(timesMs):
        raise ValueError(f"a mute table has {len(offsets)} offsets and {len(timesMs)} times")
    if len(offsets) > A.MAX_MUTE_KNOTS:
        raise ValueError(f"a mute table takes at most {A.MAX_MUTE_KNOTS} knots on the device")
    for i, (o, t) in enumerate(zip(offsets, timesMs)):
        if not _finite(o) or o < 0:
            raise ValueError(f"mute table offsets must be finite and ≥ 0, got {o}")
        if i > 0 and o <= offsets[i - 1]:
            raise ValueError(f"mute table offsets must be strictly ascending: {offsets[i - 1]} is followed by {o}")
        if not _finite(t):
            raise ValueError(f"mute table times must be finite, got {t}")
    return MuteCurve(A.MK_TABLE, offsets=tuple(offsets), timesMs=tuple(timesMs))


def lmoMute(velocity: float, t0Ms: float = 0.0, padMs: float = 0.0) -> MuteCurve:
    """A mute at ``t0Ms + |offset|/velocity + padMs`` (velocity in distance
    units per second; core/mute.nim:84-97)."""
    if not _finite(velocity) or velocity <= 0:
        raise ValueError(f"an LMO mute velocity must be finite and positive, got {velocity}")
    if not _finite(t0Ms) or not _finite(padMs):
        raise ValueError(f"LMO mute times must be finite, got t0Ms {t0Ms}, padMs {padMs}")
    return MuteCurve(A.MK_LMO, velocity=float(velocity), msPerDist=1000 / float(velocity), t0Ms=float(t0Ms),
                     padMs=float(padMs))
