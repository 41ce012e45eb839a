"""The per-row scaling of src/processSEG/core/calibrate.nim (scaleRows,
scaleRowsInto: what ``calibrate`` does once it has resolved each row's
factor), on the device. Resolving the factors themselves (rules matched on
SEG-D sensor types, components, channel sets and stations, and the file's
descale headers) needs parseSEG's trace keys and file scales, which this
build does not have: a caller that has the factors (``RowCalibration.factor``:
1 for a kept row, NaN for an unresolved one) applies them here."""
from __future__ import annotations

import numpy as np

from . import _abi as A
from .plan import Workspace


def _on_device(x):
    import torch
    if isinstance(x, torch.Tensor):
        return x, False
    return torch.from_numpy(np.ascontiguousarray(x)).cuda(), True


def scaleRowsInto(src, dst, meta, factors, ws: Workspace = None):
    """Row r of ``src`` times ``factors[r]`` over its live length into ``dst``,
    failed rows and the samples past each live length copied
    (calibrate.nim:598-604). ``ValueError`` when the shapes do not match the
    meta, ``factors`` has not one factor per row or holds an infinite one."""
    import torch
    f = np.ascontiguousarray(factors, dtype=np.float64)
    if f.ndim != 1 or f.size != len(meta):
        raise ValueError(f"need one factor per row: {len(meta)} rows, {f.size} factors")
    d, d_host = _on_device(dst)
    s = None
    if src is not None:
        s, _ = _on_device(src)
        if tuple(s.shape) != tuple(d.shape) or s.dtype != d.dtype:
            raise ValueError("src and dst must have one shape and one dtype")
    if d.dim() != 2 or not d.is_contiguous():
        raise ValueError("the block must be a C-contiguous [rows, cols] array")
    meta.checkShape(int(d.shape[0]))
    dtype = A.F32 if d.dtype == torch.float32 else (A.F64 if d.dtype == torch.float64 else None)
    if dtype is None:
        raise ValueError("the block must be float32 or float64")
    live, _ = meta.device(int(d.shape[1]), 2, d.device.index)
    ws = ws or Workspace()
    st = torch.cuda.current_stream(d.device).cuda_stream
    A.check(A.lib().psg_scale_rows(ws.h, dtype, None if s is None else s.data_ptr(), d.data_ptr(), int(d.shape[0]),
                                   int(d.shape[1]), live.data_ptr(), f.ctypes.data, st))
    if d_host:
        np.copyto(dst, d.cpu().numpy())


def scaleRows(b, meta, factors, ws: Workspace = None):
    """``scaleRowsInto`` in place (calibrate.nim:583-590): every row that is
    not failed times its factor, up to its live length, whatever its status
    (pass 1 to keep a row); a NaN factor fills the row with NaN."""
    scaleRowsInto(None, b, meta, factors, ws)
