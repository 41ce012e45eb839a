"""``ChunkMeta``: the per-row metadata every kernel takes beside a block of
samples (src/processSEG/core/types.nim:69-288).

The reference wraps parseSEG's ``TraceRows`` view; parseSEG is not part of
this build, so a meta here holds the same facts as arrays: each row's trace
status, its trace length (``numSamples``), start time (``t0Ms``) and
source-receiver offset (``offset``, which mutes read; NaN when the headers
cannot give it), the block's interval, its window origin (``firstSample``)
and the rows that could not be decoded (``failed``, ascending).

For the device it is flattened once per block width into two arrays
(``isLive``/``liveSamples``/``sampleTimeMs`` per row) by the library's
``psg_rows_flatten``, and the device copies are cached per device.
"""
from __future__ import annotations

import bisect
import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

from . import _abi as A


def same_interval(dtMs: float, planDtMs: float) -> bool:
    """types.nim:136-145."""
    return abs(dtMs - planDtMs) <= 1e-9 * planDtMs


class ChunkMeta:
    """The metadata of a block of rows (types.nim:69-78); build it with
    ``initChunkMeta``."""

    def __init__(self, status, numSamples, t0Ms, dtMs, firstSample=0, failed=(), offsets=None):
        self.status = np.ascontiguousarray(status, dtype=np.int32)
        self.numSamples = np.ascontiguousarray(numSamples, dtype=np.int32)
        self.t0 = (np.full(self.status.size, math.nan) if t0Ms is None
                   else np.ascontiguousarray(t0Ms, dtype=np.float64))
        self.offsets = (np.full(self.status.size, math.nan) if offsets is None
                        else np.ascontiguousarray(offsets, dtype=np.float64))
        self.dtMs = float(dtMs)
        self.firstSample = int(firstSample)
        self.failed = np.ascontiguousarray(failed, dtype=np.int64)
        self._flat = {}
        self._dev = {}

    # ---------------------------------------------------------------- queries
    def __len__(self):
        return int(self.status.size)

    @property
    def len(self):
        return len(self)

    def isFailed(self, row: int) -> bool:
        i = bisect.bisect_left(self.failed.tolist(), row)
        return i < self.failed.size and int(self.failed[i]) == row

    def isLive(self, row: int) -> bool:
        """types.nim:221-224: live or unknown status, not failed."""
        return int(self.status[row]) in (A.TS_LIVE, A.TS_UNKNOWN) and not self.isFailed(row)

    def liveSamples(self, row: int, cols: int) -> int:
        """types.nim:226-230."""
        return min(max(int(self.numSamples[row]) - self.firstSample, 0), cols)

    def t0Ms(self, row: int) -> float:
        return float(self.t0[row])

    def offset(self, row: int) -> float:
        return float(self.offsets[row])

    def sampleTimeMs(self, row: int, col: int) -> float:
        """types.nim:237-240."""
        return float(self.t0[row]) + (self.firstSample + col) * self.dtMs

    def sub(self, first: int, last: int) -> "ChunkMeta":
        """The meta of rows ``first .. last`` (inclusive, types.nim:242-269)."""
        if first < 0 or last >= len(self) + 0 or last < first - 1:
            if not (first == len(self) and last == first - 1):
                raise ValueError(f"rows {first} .. {last} are outside 0 ..< {len(self)}")
        sl = slice(first, last + 1)
        f = self.failed[(self.failed >= first) & (self.failed <= last)] - first
        return ChunkMeta(self.status[sl], self.numSamples[sl], self.t0[sl], self.dtMs,
                         self.firstSample, f, self.offsets[sl])

    def checkShape(self, rows: int):
        if rows != len(self):
            raise ValueError(f"the block has {rows} rows, the meta {len(self)}")

    # ------------------------------------------------------------- flattening
    def flat(self, cols: int, mode: int = 0):
        """(live, startMs) host arrays for a block ``cols`` wide; mode 0 is the
        processing rule, 1 the correlation rule (not dead, not failed)."""
        key = (cols, mode)
        if key not in self._flat:
            rows = len(self)
            live = np.zeros(rows, np.int32)
            start = np.zeros(rows, np.float64)
            p = lambda a: a.ctypes.data_as(C.c_void_p)
            A.check(A.lib().psg_rows_flatten(p(self.status), p(self.numSamples), p(self.t0), rows,
                                             self.firstSample, self.dtMs, p(self.failed),
                                             self.failed.size, cols, mode, p(live), p(start)))
            self._flat[key] = (live, start)
        return self._flat[key]

    def keys(self):
        """(offset, t0Ms) host arrays: the trace keys a mute reads."""
        return self.offsets, self.t0

    def device_keys(self, device=None):
        """(offset, t0Ms) as CUDA tensors (cached per device)."""
        import torch
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        key = ("keys", dev.index)
        if key not in self._dev:
            self._dev[key] = (torch.from_numpy(self.offsets).to(dev), torch.from_numpy(self.t0).to(dev))
        return self._dev[key]

    def device(self, cols: int, mode: int = 0, device=None):
        """The flattened arrays as CUDA tensors (cached per device)."""
        import torch
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        key = (cols, mode, dev.index)
        if key not in self._dev:
            live, start = self.flat(cols, mode)
            self._dev[key] = (torch.from_numpy(live).to(dev), torch.from_numpy(start).to(dev))
        return self._dev[key]


def initChunkMeta(status: Sequence[int], numSamples: Sequence[int], dtMs: float,
                  t0Ms: Optional[Sequence[float]] = None, firstSample: int = 0,
                  failed: Sequence[int] = (), offsets: Optional[Sequence[float]] = None) -> ChunkMeta:
    """types.nim:80-122: validates once; raises ``ValueError``."""
    if not (math.isfinite(dtMs) and dtMs > 0) or (dtMs != 0 and abs(dtMs) < 2.2250738585072014e-308):
        raise ValueError(f"dtMs must be finite and positive, got {dtMs}")
    if firstSample < 0:
        raise ValueError(f"firstSample must be ≥ 0, got {firstSample}")
    rows = len(status)
    if len(numSamples) != rows:
        raise ValueError("need one numSamples per row")
    if offsets is not None and len(offsets) != rows:
        raise ValueError("need one offset per row")
    prev = None
    for r in failed:
        if r < 0 or r >= rows:
            raise ValueError(f"failed row {r} is outside 0 ..< {rows}")
        if prev is not None and r <= prev:
            raise ValueError(f"failed rows must be ascending and unique: {prev} is followed by {r}")
        prev = r
    return ChunkMeta(status, numSamples, t0Ms, dtMs, firstSample, failed, offsets)


def liveMeta(rows: int, samples: int, dtMs: float, t0Ms: float = 0.0) -> ChunkMeta:
    """A meta of ``rows`` live traces of ``samples`` samples starting at ``t0Ms``."""
    return initChunkMeta(np.full(rows, A.TS_LIVE, np.int32), np.full(rows, samples, np.int32),
                         dtMs, np.full(rows, t0Ms))
