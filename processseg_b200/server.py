"""The request loop for a viewer: continuous batching of zoom-window and
panel requests on the GPU (``psg_server_*`` in include/psg.h).

The reference's viewer loop (tests/utils/viewersim.nim:155-200) applies a
plan per stale buffer through its ``ProcessPool``, one call at a time. Here
requests from any thread are queued, admitted by their device footprint,
and run together: requests that arrive while others are on the GPU join the
next launch, and the copies of one overlap the kernels of others. Each
result is the plain ``apply``'s, bit for bit.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi as A
from .meta import ChunkMeta
from .plan import PipelinePlan


class CancelledError(Exception):
    """A served request cancelled before it started."""


class Server:
    def __init__(self, device: int = 0, arena_bytes: int = 2 << 30):
        h = C.c_void_p()
        A.check(A.lib().psg_server_create(device, arena_bytes, C.byref(h)))
        self.h = h
        self._keep = {}

    def close(self):
        if getattr(self, "h", None) is not None and A._lib is not None:
            A._lib.psg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, plan: PipelinePlan, src: np.ndarray, dst: np.ndarray, meta: ChunkMeta) -> int:
        """Queues ``plan`` on ``src`` into ``dst`` (host arrays of the same
        shape); returns a ticket for ``wait``."""
        rows, cols = src.shape
        meta.checkShape(rows)
        live, start = meta.flat(cols, 0)
        t = C.c_uint64()
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        A.check(A.lib().psg_submit(self.h, plan.h, p(src), p(dst), rows, cols, p(live), p(start),
                                   meta.dtMs, C.byref(t)))
        self._keep[t.value] = (plan, src, dst, live, start)
        return t.value

    def wait(self, ticket: int, timeout_ms: float = 10000.0):
        """Waits for a request; ``TimeoutError`` after ``timeout_ms``,
        ``CancelledError`` for a request cancelled before it started."""
        st = A.lib().psg_wait(self.h, ticket, timeout_ms)
        if st != A.ETIMEOUT:
            self._keep.pop(ticket, None)
        if st == A.ECANCELED:
            raise CancelledError(A.lib().psg_last_error().decode("utf-8", "replace"))
        A.check(st)

    def poll(self, ticket: int) -> bool:
        """True when the request has finished (or was cancelled)."""
        done = C.c_int32()
        A.check(A.lib().psg_poll(self.h, ticket, C.byref(done)))
        return bool(done.value)

    def cancel(self, ticket: int) -> bool:
        """Cancels a request that has not started: True; False when it has
        started or finished (wait for it). ``ValueError`` for an unknown
        ticket."""
        st = A.lib().psg_cancel(self.h, ticket)
        if st == A.OK:
            return True
        msg = A.lib().psg_last_error().decode("utf-8", "replace")
        if "unknown ticket" in msg:
            raise ValueError(msg)
        return False

    def stats(self, reset: bool = False) -> dict:
        out = (C.c_double * 8)()
        A.check(A.lib().psg_server_stats(self.h, out, 1 if reset else 0))
        keys = ["completed", "samples", "launches", "requests_per_launch", "p50_s", "p99_s",
                "msamples_per_s", "refused"]
        return dict(zip(keys, list(out)))
