"""``ProcessPool`` (src/processSEG/core/pool.nim:89-347), the reference's
multi-threaded block apply, as a drop-in whose workers are the device's
SMs: ``apply`` and ``correlateInto`` take the pool's own workspace, run on
the device and return when the block is done, one call at a time (a second
caller waits, as on the reference's pool). Host (numpy) blocks go through
the library's chunked host-memory path; CUDA tensors stay on the device.
"""
from __future__ import annotations

import threading

from .plan import Workspace


class ProcessPool:
    """newProcessPool (pool.nim:145-166): ``ValueError`` for ``workers < 1``.
    ``workers`` is kept for the callers that read it; the rows of a block
    are spread over the device, not over host threads."""

    def __init__(self, workers: int = 4):
        if workers < 1:
            raise ValueError(f"a pool needs ≥ 1 worker, got {workers}")
        self._workers = int(workers)
        self._ws = Workspace()
        self._call = threading.Lock()

    @property
    def workers(self) -> int:
        return self._workers

    def ping(self):
        """An empty job: the pool's per-call overhead (pool.nim:189-197)."""
        with self._call:
            pass

    @staticmethod
    def _sync(x):
        try:
            import torch
            if isinstance(x, torch.Tensor):
                torch.cuda.current_stream(x.device).synchronize()
        except ImportError:
            pass

    def apply(self, plan, *args):
        """``apply(plan, b, meta)`` in place or ``apply(plan, src, dst, meta)``
        (pool.nim:277-302); blocks until the block is done. Raises
        ``ValueError`` before any sample changes, as ``PipelinePlan.apply``."""
        if len(args) == 2:
            b, meta = args
            blocks = (b,)
        elif len(args) == 3:
            src, dst, meta = args
            blocks = (src, dst)
        else:
            raise TypeError("apply(plan, b, meta) or apply(plan, src, dst, meta)")
        dst = blocks[-1]
        with self._call:
            self._ws.reserve(plan, rows=int(dst.shape[0]), cols=int(dst.shape[1]))
            plan.apply(*blocks, meta, self._ws)
            self._sync(dst)

    def correlateInto(self, plan, src, dst, meta):
        """Vibroseis correlation of ``src`` into ``dst`` (pool.nim:318-339);
        blocks until it is done."""
        with self._call:
            plan.correlateInto(src, dst, meta)
            self._sync(dst)


def newProcessPool(workers: int = 4) -> ProcessPool:
    return ProcessPool(workers)
