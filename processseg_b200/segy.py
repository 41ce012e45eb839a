"""SEG-Y trace records to a sample block and a ``ChunkMeta`` on the device:
the decode a reader does before the pipeline (the reference reads files
through parseSEG, which is not part of this build). Records are what a
prefetcher reads from a file: ``rows`` consecutive trace records of
``recordBytes`` bytes (a 240-byte trace header, then the samples), here a
CUDA uint8 tensor or a host uint8 array (copied to the device once).

Formats (SEG-Y rev 2 data sample format codes): 1 IBM float, 2 int32,
3 int16, 5 IEEE float32, 6 IEEE float64, 7 int24, 8 int8, 10 uint32,
11 uint16, 15 uint24, 16 uint8; big-endian unless ``littleEndian``."""
from __future__ import annotations

import numpy as np

from . import _abi as A
from .meta import initChunkMeta

SAMPLE_BYTES = {1: 4, 2: 4, 3: 2, 5: 4, 6: 8, 7: 3, 8: 1, 10: 4, 11: 2, 15: 3, 16: 1}


def _device_records(records):
    import torch
    if isinstance(records, torch.Tensor):
        if records.dtype != torch.uint8 or not records.is_cuda or records.dim() != 2 or not records.is_contiguous():
            raise ValueError("records must be a C-contiguous [rows, recordBytes] CUDA uint8 tensor")
        return records
    r = np.ascontiguousarray(records, dtype=np.uint8)
    if r.ndim != 2:
        raise ValueError("records must be [rows, recordBytes] bytes")
    return torch.from_numpy(r).cuda()


def decodeTraces(records, samples: int, format: int, T, littleEndian: bool = False, headerBytes: int = 240,
                 outCols: int = 0):
    """The samples of each record as a CUDA tensor [rows, outCols] of T
    (``outCols`` 0: ``samples``; zeros past ``samples``). ``ValueError`` for
    an unknown format or records too short for the samples."""
    import torch
    from .plan import _dtype_code
    dt = _dtype_code(T)
    rec = _device_records(records)
    rows, rb = int(rec.shape[0]), int(rec.shape[1])
    cols = int(outCols) or int(samples)
    out = torch.empty(rows, cols, dtype=torch.float32 if dt == A.F32 else torch.float64, device=rec.device)
    st = torch.cuda.current_stream(rec.device).cuda_stream
    A.check(A.lib().psg_segy_decode(rec.data_ptr(), rows, rb, int(headerBytes), int(samples), int(format),
                                    int(bool(littleEndian)), dt, out.data_ptr(), cols, st))
    return out


def traceKeys(records, littleEndian: bool = False):
    """The trace-header keys of each record as host arrays: ``status``,
    ``numSamples``, ``intervalUs``, ``offset``, ``t0Ms``."""
    import torch
    rec = _device_records(records)
    rows, rb = int(rec.shape[0]), int(rec.shape[1])
    dev = rec.device
    status = torch.empty(rows, dtype=torch.int32, device=dev)
    ns = torch.empty(rows, dtype=torch.int32, device=dev)
    dt = torch.empty(rows, dtype=torch.float64, device=dev)
    off = torch.empty(rows, dtype=torch.float64, device=dev)
    t0 = torch.empty(rows, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    A.check(A.lib().psg_segy_keys(rec.data_ptr(), rows, rb, int(bool(littleEndian)), status.data_ptr(),
                                  ns.data_ptr(), dt.data_ptr(), off.data_ptr(), t0.data_ptr(), st))
    return {"status": status.cpu().numpy(), "numSamples": ns.cpu().numpy(), "intervalUs": dt.cpu().numpy(),
            "offset": off.cpu().numpy(), "t0Ms": t0.cpu().numpy()}


def chunkMetaOf(keys, dtMs: float = float("nan"), firstSample: int = 0, failed=()):
    """The ``ChunkMeta`` of decoded records (adapters.nim:63-104): the sample
    interval from the keys' ``intervalUs`` unless ``dtMs`` is given;
    ``ValueError`` when it is unknown (0) or the rows disagree."""
    if dtMs != dtMs:  # NaN: from the keys
        us = keys["intervalUs"]
        if us.size == 0:
            raise ValueError("no rows to take the sample interval from")
        for r, x in enumerate(us):
            if not (0 < x < float("inf")):
                raise ValueError(f"row {r} has no sample interval in its headers ({x} µs): pass dtMs")
            if x != us[0]:
                raise ValueError(f"rows 0 and {r} have different sample intervals ({us[0]} and {x} µs)")
        dtMs = float(us[0]) / 1000
    return initChunkMeta(keys["status"], keys["numSamples"], dtMs, keys["t0Ms"], firstSample, failed, keys["offset"])
