"""The request loop for a viewer: continuous batching of zoom-window and
panel requests on the GPU (``psg_server_*`` in include/psg.h).

The reference's viewer loop (tests/utils/viewersim.nim:155-200) applies a
plan per stale buffer through its ``ProcessPool``, one call at a time. Here
requests from any thread are queued, admitted by their device footprint,
and run together: requests that arrive while others are on the GPU join the
next batch (or start one beside it when they can fill the device), and the
copies of one overlap the kernels of others. Requests whose buffers are
already on the device (CUDA tensors) skip the copies. Any plan the plain
apply takes is served: single-part float32 plans in batched launches, the
rest (per-panel normalizations, float64, IIR filters, mutes, long traces)
with the plain apply's own launches inside a batch. Each result is the
plain ``apply``'s, bit for bit.
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
        self.device = device
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

    def submit(self, plan: PipelinePlan, src, dst, meta: ChunkMeta) -> int:
        """Queues ``plan`` on ``src`` into ``dst`` (host arrays, or CUDA
        tensors on the server's device, of the same shape and the plan's
        dtype); returns a ticket for ``wait``. A plan that mutes reads the
        meta's offsets and t0Ms."""
        rows, cols = int(src.shape[0]), int(src.shape[1])
        meta.checkShape(rows)
        t = C.c_uint64()
        try:
            import torch
            on_device = isinstance(src, torch.Tensor)
        except ImportError:
            on_device = False
        if on_device:
            if not (src.is_cuda and dst.is_cuda and src.is_contiguous() and dst.is_contiguous()):
                raise ValueError("device requests take contiguous CUDA tensors")
            dev = src.device.index
            live, start = meta.device(cols, 0, dev)
            keys = plan._keys(meta, dev)
            st = torch.cuda.current_stream(dev).cuda_stream  # the caller's writes come first
            A.check(A.lib().psg_submit_device(self.h, plan.h, src.data_ptr(), dst.data_ptr(), rows, cols,
                                              live.data_ptr(), start.data_ptr(), keys, meta.dtMs, st,
                                              C.byref(t)))
            self._keep[t.value] = (plan, src, dst, live, start, keys)
            return t.value
        live, start = meta.flat(cols, 0)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        keys = plan._keys(meta, None)
        if keys is None:
            A.check(A.lib().psg_submit(self.h, plan.h, p(src), p(dst), rows, cols, p(live), p(start),
                                       meta.dtMs, C.byref(t)))
        else:
            A.check(A.lib().psg_submit_keyed(self.h, plan.h, p(src), p(dst), rows, cols, p(live), p(start), keys,
                                             meta.dtMs, C.byref(t)))
        self._keep[t.value] = (plan, src, dst, live, start, keys, meta)
        return t.value

    def wait(self, ticket: int, timeout_ms: float = 10000.0) -> float:
        """Waits for a request; ``TimeoutError`` after ``timeout_ms``,
        ``CancelledError`` for a request cancelled before it started.
        Returns when it finished, on ``time.perf_counter``'s clock."""
        done = C.c_double(0.0)
        st = A.lib().psg_wait_done(self.h, ticket, timeout_ms, C.byref(done))
        if st != A.ETIMEOUT:
            self._keep.pop(ticket, None)
        if st == A.ECANCELED:
            raise CancelledError(A.lib().psg_last_error().decode("utf-8", "replace"))
        A.check(st)
        return done.value

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

    def counters(self) -> dict:
        """Counters since the loop was created: batches, kernel launches,
        batches started beside running ones, requests completed."""
        out = (C.c_int64 * 4)()
        A.check(A.lib().psg_server_counters(self.h, out))
        return dict(zip(["batches", "kernels", "overlapped", "completed"], list(out)))

    def stats(self, reset: bool = False) -> dict:
        out = (C.c_double * 8)()
        A.check(A.lib().psg_server_stats(self.h, out, 1 if reset else 0))
        keys = ["completed", "samples", "launches", "requests_per_launch", "p50_s", "p99_s",
                "msamples_per_s", "refused"]
        return dict(zip(keys, list(out)))

    def load(self) -> tuple:
        """(requests, samples) outstanding: queued, staged or running."""
        out = (C.c_int64 * 2)()
        A.check(A.lib().psg_server_load(self.h, out))
        return int(out[0]), int(out[1])


def leastLoaded(loads) -> int:
    """The index of the least loaded of ``loads`` ((requests, samples) per
    loop): the fewest outstanding samples, then the fewest requests, then
    the lowest index."""
    loads = list(loads)
    if not loads:
        raise ValueError("no loops to choose from")
    return min(range(len(loads)), key=lambda i: (loads[i][1], loads[i][0], i))


class ServerPool:
    """One request loop per device, requests placed on the least loaded one
    (its outstanding samples). A request whose buffers are CUDA tensors runs
    on their device; host requests go where the load is least, with the plan
    compiled for that device once (``PipelinePlan.forDevice``). ``submit``
    returns a (loop index, ticket) pair for ``wait``, ``poll`` and
    ``cancel``."""

    def __init__(self, devices=None, arena_bytes: int = 2 << 30, loops=None):
        if loops is not None:
            self.loops = list(loops)       # loops made elsewhere (their device attribute set)
        else:
            import torch
            devs = list(range(torch.cuda.device_count())) if devices is None else list(devices)
            self.loops = []
            for d in devs:
                s = Server(d, arena_bytes)
                s.device = d
                self.loops.append(s)
        if not self.loops:
            raise ValueError("a pool needs at least one loop")

    def close(self):
        for s in self.loops:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def place(self, src) -> int:
        """The loop a request on ``src`` goes to."""
        dev = getattr(src, "device", None)
        if dev is not None and getattr(dev, "type", None) == "cuda":
            for i, s in enumerate(self.loops):
                if s.device == dev.index:
                    return i
            raise ValueError(f"no loop on cuda:{dev.index}")
        return leastLoaded(s.load() for s in self.loops)

    def submit(self, plan: PipelinePlan, src, dst, meta: ChunkMeta):
        i = self.place(src)
        s = self.loops[i]
        return i, s.submit(plan.forDevice(s.device), src, dst, meta)

    def wait(self, ticket, timeout_ms: float = 10000.0) -> float:
        i, t = ticket
        return self.loops[i].wait(t, timeout_ms)

    def poll(self, ticket) -> bool:
        i, t = ticket
        return self.loops[i].poll(t)

    def cancel(self, ticket) -> bool:
        i, t = ticket
        return self.loops[i].cancel(t)
