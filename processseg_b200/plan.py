"""``compile``, ``PipelinePlan``, ``Workspace`` and ``apply``: the host side
of src/processSEG/pipeline.nim:466-772 over the C ABI of libpsgcuda.so.

``apply`` takes either CUDA tensors (torch, C-contiguous ``[rows, cols]``;
the work is queued on the current torch stream and nothing is copied) or
numpy arrays (host memory: the library copies the block in, runs the plan
and copies it back before returning). Errors follow the reference:
``ValueError`` before any sample changes for a bad shape, width, interval
or overlap; ``AssertionError`` (the reference's AssertionDefect) for a
workspace that was not reserved for the plan.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np

from . import _abi as A
from .meta import ChunkMeta


def _dtype_code(T) -> int:
    if T in (A.F32, np.float32, "float32") or getattr(T, "__name__", "") == "float32":
        return A.F32
    if T in (A.F64, np.float64, float, "float64") or getattr(T, "__name__", "") == "float64":
        return A.F64
    try:
        import torch
        if T == torch.float32:
            return A.F32
        if T == torch.float64:
            return A.F64
    except ImportError:
        pass
    raise ValueError(f"a sample type must be float32 or float64, got {T!r}")


class Workspace:
    """The scratch of ``apply`` on the device (workspace.nim:50-96): a
    grow-only arena, one per thread or stream of callers."""

    def __init__(self):
        h = C.c_void_p()
        A.check(A.lib().psg_workspace_create(C.byref(h)))
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and A._lib is not None:
            A._lib.psg_workspace_destroy(h)
            self.h = None

    def reserve(self, plan: "PipelinePlan", rows: int = 65536, cols: int = 0):
        """Grows the arena to hold ``plan``'s scratch for up to ``rows`` rows,
        and, with ``cols``, the staging a host-memory ``apply`` of
        ``rows × cols`` needs. A no-op when it already fits."""
        A.check(A.lib().psg_workspace_reserve(self.h, plan.h, int(rows), int(cols)))

    @property
    def bytes(self) -> int:
        return A.lib().psg_workspace_bytes(self.h)

    def synchronize(self):
        """Waits for the host-memory applies queued with ``wait=False``."""
        A.check(A.lib().psg_workspace_sync(self.h))


def initWorkspace() -> Workspace:
    return Workspace()


def _is_torch(x) -> bool:
    try:
        import torch
        return isinstance(x, torch.Tensor)
    except ImportError:
        return False


class PipelinePlan:
    """A compiled pipeline (pipeline.nim:200-211): immutable, shared by any
    number of callers, each with its own ``Workspace``."""

    def __init__(self, h, dtype: int, dtMs: float, args=None, device: Optional[int] = None):
        self.h = h
        self.dtype = dtype
        self._dtMs = dtMs
        self._args = args      # what compile took, to compile a twin on another device
        self.device = device   # the device its tables live on
        self._twins = {}

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and A._lib is not None:
            A._lib.psg_plan_destroy(h)
            self.h = None

    # ------------------------------------------------------------ accessors
    @property
    def generation(self) -> int:
        return A.lib().psg_plan_generation(self.h)

    @property
    def requiredMargin(self) -> int:
        return A.lib().psg_plan_margin(self.h)

    @property
    def samples(self) -> int:
        return A.lib().psg_plan_samples(self.h)

    @property
    def recordSamples(self) -> int:
        return A.lib().psg_plan_record_samples(self.h)

    @property
    def dtMs(self) -> float:
        return self._dtMs

    @property
    def partCount(self) -> int:
        return A.lib().psg_plan_part_count(self.h)

    def __len__(self):
        return A.lib().psg_plan_len(self.h)

    def stepNfft(self, i: int) -> int:
        return A.lib().psg_plan_step_nfft(self.h, i)

    def stepMargin(self, i: int) -> int:
        return A.lib().psg_plan_step_margin(self.h, i)

    def workspaceSize(self, rows: int = 65536, cols: int = 0) -> int:
        """The device bytes ``Workspace.reserve(plan, rows, cols)`` holds
        for this plan (pipeline.nim ``workspaceSize``): the arena, plus the
        global work areas of a plan whose traces are too long for their FFT
        buffers to sit beside them in shared memory."""
        return A.lib().psg_plan_workspace_bytes(self.h, int(rows), int(cols))

    # ---------------------------------------------------------------- apply
    def _check_block(self, x, name):
        if x.ndim != 2:
            raise ValueError(f"{name} must be a [rows, cols] tensor, got rank {x.ndim}")
        want = np.float32 if self.dtype == A.F32 else np.float64
        if _is_torch(x):
            import torch
            tw = torch.float32 if self.dtype == A.F32 else torch.float64
            if x.dtype != tw:
                raise ValueError(f"{name} is {x.dtype}, the plan is for {tw}")
            if not x.is_contiguous():
                raise ValueError(f"{name} must be C-contiguous (row-major)")
            if not x.is_cuda:
                raise ValueError(f"{name} must be a CUDA tensor or a numpy array")
        else:
            if x.dtype != want:
                raise ValueError(f"{name} is {x.dtype}, the plan is for {np.dtype(want)}")
            if not x.flags.c_contiguous:
                raise ValueError(f"{name} must be C-contiguous (row-major)")

    def checkApply(self, src, dst, meta: ChunkMeta):
        """pipeline.nim:619-641: the checks ``apply`` makes before touching a
        sample (src None: in place), raising ``ValueError``: the shapes and
        sample types, the meta's rows, src and dst overlapping without being
        the same block, the interval and the width."""
        if self.h is None:
            raise ValueError("a PipelinePlan must come from compile")
        self._check_block(dst, "dst")
        rows, cols = int(dst.shape[0]), int(dst.shape[1])
        if src is not None:
            self._check_block(src, "src")
            if tuple(src.shape) != tuple(dst.shape):
                raise ValueError(f"src is {src.shape[0]} × {src.shape[1]}, dst {rows} × {cols}")
            if _is_torch(src) != _is_torch(dst):
                raise ValueError("src and dst must both be CUDA tensors or both numpy arrays")
        meta.checkShape(rows)
        ptr = (lambda a: a.data_ptr()) if _is_torch(dst) else (lambda a: a.ctypes.data)
        A.check(A.lib().psg_check_apply(self.h, None if src is None else ptr(src), ptr(dst), rows, cols,
                                        meta.dtMs))

    def apply(self, *args, stream=None, wait=True):
        """``apply(b, meta, ws)`` in place, or ``apply(src, dst, meta, ws)``
        from src into dst (pipeline.nim:736-772). With host arrays and
        ``wait=False`` the call returns once its copies and kernels are
        queued (``ws.synchronize()`` waits); consecutive calls then overlap,
        and the arrays must stay valid and unchanged until the wait."""
        if len(args) == 3:
            src, (dst, meta, ws) = None, args
        elif len(args) == 4:
            src, dst, meta, ws = args
        else:
            raise TypeError("apply(b, meta, ws) or apply(src, dst, meta, ws)")
        if self.h is None:
            raise ValueError("a PipelinePlan must come from compile")
        self._check_block(dst, "dst")
        rows, cols = int(dst.shape[0]), int(dst.shape[1])
        if src is not None:
            self._check_block(src, "src")
            if tuple(src.shape) != tuple(dst.shape):
                raise ValueError(f"src is {src.shape[0]} × {src.shape[1]}, dst {rows} × {cols}")
            if _is_torch(src) != _is_torch(dst):
                raise ValueError("src and dst must both be CUDA tensors or both numpy arrays")
        meta.checkShape(rows)
        if _is_torch(dst):
            import torch
            live, start = meta.device(cols, 0, dst.device.index)
            st = stream if stream is not None else torch.cuda.current_stream(dst.device).cuda_stream
            keys = self._keys(meta, dst.device.index)
            A.check(A.lib().psg_apply_keyed(self.h, ws.h, None if src is None else src.data_ptr(),
                                            dst.data_ptr(), rows, cols, live.data_ptr(), start.data_ptr(),
                                            keys, meta.dtMs, st))
        else:
            live, start = meta.flat(cols, 0)
            p = lambda a: a.ctypes.data_as(C.c_void_p)
            keys = self._keys(meta, None)
            fn = A.lib().psg_apply_host_keyed if wait else A.lib().psg_apply_host_async
            A.check(fn(self.h, ws.h, None if src is None else p(src), p(dst), rows, cols, p(live), p(start), keys,
                       meta.dtMs, stream if stream is not None else None))

    def capture(self, src, dst, meta: ChunkMeta, ws: Workspace) -> "ApplyGraph":
        """``apply(src, dst, meta, ws)`` on CUDA tensors (src None: in place)
        captured into a CUDA graph: ``replay()`` reruns it with one host
        call. The checks run here, once; the tensors, the meta's device
        arrays and the workspace must outlive the graph, and the workspace
        must not be grown while it lives."""
        import torch
        self._check_block(dst, "dst")
        if not _is_torch(dst):
            raise ValueError("capture takes CUDA tensors")
        rows, cols = int(dst.shape[0]), int(dst.shape[1])
        if src is not None:
            self._check_block(src, "src")
            if tuple(src.shape) != tuple(dst.shape):
                raise ValueError(f"src is {src.shape[0]} × {src.shape[1]}, dst {rows} × {cols}")
        meta.checkShape(rows)
        live, start = meta.device(cols, 0, dst.device.index)
        keys = self._keys(meta, dst.device.index)
        h = C.c_void_p()
        A.check(A.lib().psg_graph_capture(self.h, ws.h, None if src is None else src.data_ptr(), dst.data_ptr(),
                                          rows, cols, live.data_ptr(), start.data_ptr(), keys, meta.dtMs,
                                          C.byref(h)))
        return ApplyGraph(h, (self, ws, src, dst, live, start, keys))

    def forDevice(self, device: int) -> "PipelinePlan":
        """This plan compiled for ``device`` (itself when its tables are
        there; else a twin, compiled once and kept)."""
        if device == self.device:
            return self
        if device not in self._twins:
            if self._args is None:
                raise ValueError("the plan was not made by compile")
            import torch
            with torch.cuda.device(device):
                self._twins[device] = compile(*self._args)
        return self._twins[device]

    def traceShapes(self, part: int = 0) -> int:
        """How many launch shapes of the trace kernel part ``part`` can run
        on (0: the part runs on the general kernel). Every shape gives the
        same bits; the first apply at a new row-count class times them all
        and keeps the fastest (``PSG_TUNE=0`` keeps the first)."""
        return int(A.lib().psg_plan_trace_shapes(self.h, part))

    def pinTrace(self, part: int, shape: int):
        """Runs part ``part`` with launch shape ``shape`` whatever the row
        count (-1: back to the tuner's choices)."""
        A.check(A.lib().psg_plan_pin_trace(self.h, part, shape))

    def tuning(self) -> dict:
        """The launch shapes of each trace-kernel part and what the tuner
        measured: ``{"parts": [{"part", "pinned", "shapes": [...]}],
        "tuned": [{"part", "class", "rows", "us", "choice"}]}``."""
        import json
        need = C.c_int64(0)
        A.check(A.lib().psg_plan_tuning(self.h, None, 0, C.byref(need)))
        buf = C.create_string_buffer(int(need.value) + 64)
        A.check(A.lib().psg_plan_tuning(self.h, buf, len(buf), C.byref(need)))
        return json.loads(buf.value.decode())

    @property
    def needsKeys(self) -> bool:
        """The plan mutes: it reads each row's offset and t0Ms."""
        return bool(A.lib().psg_plan_needs_keys(self.h))

    def _keys(self, meta: ChunkMeta, device):
        """A ``psg_keys`` for a plan that mutes (device arrays for a device
        index, else the meta's host arrays); None for one that does not."""
        if not self.needsKeys:
            return None
        k = A.KeysC()
        if device is None:
            off, t0 = meta.keys()
            k.offset, k.t0_ms = off.ctypes.data, t0.ctypes.data
        else:
            off, t0 = meta.device_keys(device)
            k.offset, k.t0_ms = off.data_ptr(), t0.data_ptr()
        k.first_sample = meta.firstSample
        return C.pointer(k)

    def partNeedsPanel(self, part: int) -> bool:
        """Part ``part`` starts with a per-panel normalization
        (pipeline.nim:649-654)."""
        return bool(A.lib().psg_plan_part_needs_panel(self.h, int(part)))

    def _device_call(self, dst, meta, cols):
        import torch
        live, start = meta.device(cols, 0, dst.device.index)
        return live, start, torch.cuda.current_stream(dst.device).cuda_stream

    def runPart(self, src, dst, meta: ChunkMeta, part: int, factor, ws: Workspace):
        """runPart (pipeline.nim:690-723) on CUDA tensors: the steps of part
        ``part`` on ``dst`` (copied from ``src`` first unless it is None:
        the first part of a src → dst apply only). ``factor`` is a CUDA
        float64 tensor of one value (``panelFactorOf``/``panelFactorFrom``)
        or None; NaN or None leaves the rows alone."""
        self._check_block(dst, "dst")
        rows, cols = int(dst.shape[0]), int(dst.shape[1])
        if src is not None:
            self._check_block(src, "src")
            if tuple(src.shape) != tuple(dst.shape):
                raise ValueError(f"src is {src.shape[0]} × {src.shape[1]}, dst {rows} × {cols}")
        meta.checkShape(rows)
        live, start, st = self._device_call(dst, meta, cols)
        A.check(A.lib().psg_run_part_keyed(self.h, ws.h, int(part), None if src is None else src.data_ptr(),
                                           dst.data_ptr(), rows, cols, live.data_ptr(), start.data_ptr(),
                                           self._keys(meta, dst.device.index), meta.dtMs,
                                           None if factor is None else factor.data_ptr(), st))

    def panelPartials(self, b, meta: ChunkMeta, part: int, ws: Workspace):
        """The mergeable statistics of part ``part``'s per-panel
        normalization over this shard ``b`` of a panel: a CUDA float64
        tensor of ``PANEL_PARTIAL_DOUBLES`` values ([Σx², samples, rows,
        maxAbs] then 65536 histogram counts). Shards merge by summing every
        entry but maxAbs, which takes the maximum."""
        import torch
        self._check_block(b, "b")
        rows, cols = int(b.shape[0]), int(b.shape[1])
        meta.checkShape(rows)
        live, _, st = self._device_call(b, meta, cols)
        out = torch.empty(A.PANEL_PARTIAL_DOUBLES, dtype=torch.float64, device=b.device)
        A.check(A.lib().psg_panel_partials(self.h, ws.h, int(part), b.data_ptr(), rows, cols,
                                           live.data_ptr(), out.data_ptr(), st))
        return out

    def panelFactorFrom(self, partial, part: int, ws: Workspace):
        """The factor (a CUDA float64 tensor of one value, NaN when the
        normalization leaves the panel alone) of merged partials."""
        import torch
        out = torch.empty(1, dtype=torch.float64, device=partial.device)
        st = torch.cuda.current_stream(partial.device).cuda_stream
        A.check(A.lib().psg_panel_factor_from(self.h, ws.h, int(part), partial.data_ptr(),
                                              out.data_ptr(), st))
        return out

    def panelFactorOf(self, b, meta: ChunkMeta, part: int, ws: Workspace) -> float:
        """The per-panel factor of part ``part`` over the block ``b`` (a CUDA
        tensor), NaN when it leaves the block alone (pipeline.nim:656-669)."""
        import torch
        self._check_block(b, "b")
        rows, cols = int(b.shape[0]), int(b.shape[1])
        live, _ = meta.device(cols, 0, b.device.index)
        out = torch.empty(1, dtype=torch.float64, device=b.device)
        st = torch.cuda.current_stream(b.device).cuda_stream
        A.check(A.lib().psg_panel_factor(self.h, ws.h, part, b.data_ptr(), rows, cols,
                                         live.data_ptr(), out.data_ptr(), st))
        return float(out.item())


class ApplyGraph:
    """A captured apply (``PipelinePlan.capture``): ``replay(stream)`` runs it
    on ``stream`` (the current stream when None)."""

    def __init__(self, h, keep):
        self.h = h
        self._keep = keep  # what the graph points at stays alive with it

    def replay(self, stream=None):
        import torch
        st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        A.check(A.lib().psg_graph_launch(self.h, st))

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and A._lib is not None:
            A._lib.psg_graph_destroy(h)
            self.h = None


def compile(pipeline, T, dtMs: float, samples: int, recordSamples: int = 0) -> PipelinePlan:
    """Validates every op for blocks of up to ``samples`` samples at
    ``dtMs`` and uploads its tables to the current device
    (pipeline.nim:466-523). ``ValueError`` names the op:
    ``op 1 (opFilter): ...``."""
    dt = _dtype_code(T)
    ops = list(pipeline)
    arr = A.ops_array(ops)
    h = C.c_void_p()
    A.check(A.lib().psg_plan_compile(arr, len(ops), dt, float(dtMs), int(samples),
                                     int(recordSamples), C.byref(h)))
    dev = None
    try:
        import torch
        if torch.cuda.is_available():
            dev = torch.cuda.current_device()
    except ImportError:
        pass
    return PipelinePlan(h, dt, float(dtMs), (ops, T, dtMs, samples, recordSamples), dev)
