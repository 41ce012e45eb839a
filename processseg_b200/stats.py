"""The display-gain statistics of src/processSEG/gain/stats.nim on the device:
``traceStatsInto`` (:186-199), the RMS and max |x| of each row's live samples,
and ``panelStats`` (:253-304), the RMS, max |x| and clip percentile of a
panel's usable live rows. A viewer reads these every frame to set its gain.

Both take the reference's ChunkMeta: a row that is not live (dead, auxiliary
or failed) reads NaN in ``traceStatsInto`` and is left out of ``panelStats``;
a live row with no live samples (a zoom window past a short trace) reads
(0, 0) in ``traceStatsInto`` (``statsOf``, :124-127) and counts among the
panel's rows with no samples. The rows are flattened with
``psg_rows_flatten`` mode 3, which keeps those two apart.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _abi as A
from .meta import ChunkMeta
from .plan import Workspace


@dataclass
class TraceStats:
    """TraceStats (stats.nim:60-62)."""
    rms: float = 0.0
    maxAbs: float = 0.0


@dataclass
class PanelStats:
    """PanelStats (stats.nim:64-70): ``clip`` NaN when no percentile was asked
    for or no sample was usable."""
    rms: float = 0.0
    maxAbs: float = 0.0
    clip: float = math.nan
    rows: int = 0
    samples: int = 0


def _block(b):
    import torch
    if isinstance(b, torch.Tensor):
        if not b.is_cuda:
            b = b.cuda()
        t = b
    else:
        t = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    if t.dim() != 2 or not t.is_contiguous():
        raise ValueError("the block must be a C-contiguous [rows, cols] array")
    if t.dtype == torch.float32:
        return t, A.F32
    if t.dtype == torch.float64:
        return t, A.F64
    raise ValueError("the block must be float32 or float64")


def _check_percentile(p: float):
    """checkPercentile with NaN allowed (stats.nim:71-78)."""
    if not math.isnan(p) and not (0 <= p <= 100):
        raise ValueError(f"a percentile must be in 0 .. 100, got {p}")


def traceStatsInto(b, meta: ChunkMeta, stats: Optional[list] = None) -> list:
    """The statistics of each row of ``b`` (one TraceStats per row), of its live
    samples for a live row, NaN for a row that is not live. ``stats``, when
    given, must hold one entry per row (``ValueError`` otherwise) and is
    filled in place; the list is returned. ``ValueError`` when ``b`` does not
    match ``meta``."""
    import torch
    t, dtype = _block(b)
    rows, cols = int(t.shape[0]), int(t.shape[1])
    meta.checkShape(rows)
    if stats is not None and len(stats) != rows:
        raise ValueError(f"stats holds {len(stats)} values, the block has {rows} rows")
    live, _ = meta.device(cols, 3, t.device.index)
    rms = torch.empty(rows, dtype=torch.float64, device=t.device)
    mx = torch.empty(rows, dtype=torch.float64, device=t.device)
    st = torch.cuda.current_stream(t.device).cuda_stream
    A.check(A.lib().psg_trace_stats(t.data_ptr(), dtype, rows, cols, live.data_ptr(), rms.data_ptr(),
                                    mx.data_ptr(), st))
    r, m = rms.cpu().numpy(), mx.cpu().numpy()
    out = stats if stats is not None else [None] * rows
    for i in range(rows):
        out[i] = TraceStats(float(r[i]), float(m[i]))
    return out


def panelStats(b, meta: ChunkMeta, ws: Optional[Workspace] = None, clipPercentile: float = 99.0,
               rows: Optional[range] = None) -> PanelStats:
    """The statistics of the live rows of ``b`` in ``rows`` (clipped to the
    block; all rows when None) over their live samples, leaving out rows with
    a NaN or Inf; ``clip`` is the ``clipPercentile`` of |x| from the 65536-bin
    histogram, NaN to skip it. ``ValueError`` when ``b`` does not match
    ``meta`` or for a percentile outside 0 .. 100."""
    import torch
    t, dtype = _block(b)
    nrows, cols = int(t.shape[0]), int(t.shape[1])
    meta.checkShape(nrows)
    _check_percentile(clipPercentile)
    first, last = 0, nrows - 1
    if rows is not None:
        first, last = max(rows.start, 0), min(rows.stop - 1, nrows - 1)
    n = max(0, last - first + 1)
    live, _ = meta.device(cols, 3, t.device.index)
    ws = ws or Workspace()
    A.check(A.lib().psg_workspace_reserve(ws.h, None, max(n, 1), cols))
    out = torch.empty(5, dtype=torch.float64, device=t.device)
    st = torch.cuda.current_stream(t.device).cuda_stream
    esz = t.element_size()
    A.check(A.lib().psg_panel_stats(ws.h, t.data_ptr() + first * cols * esz if n else t.data_ptr(), dtype, n, cols,
                                    live.data_ptr() + first * 4 if n else live.data_ptr(), clipPercentile,
                                    out.data_ptr(), st))
    o = out.cpu().numpy()
    return PanelStats(float(o[0]), float(o[1]), float(o[2]), int(o[3]), int(o[4]))
