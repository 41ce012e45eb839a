"""psg_panel_stats_static, the entry point for callers that cannot allocate
device memory (a viewer computing display-gain statistics every frame inside
a fixed memory budget, say): called through the C ABI twice in a row, each
time it must give what psg_panel_stats gives with a workspace on the same
block, and both must give the oracle's panelStats (gain/stats.nim:253-304):
float32 and float64, with a percentile, with none (NaN), with 100, and with
no rows. Named to run last: it holds a library-wide scratch array, and a run
stopping at its first failure has then already run every other test."""
import ctypes as C
import math

import numpy as np
import pytest

from processseg_b200 import _abi as A
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


def stats_with_workspace(lib, block, dtype, live, clip):
    ws = C.c_void_p()
    A.check(lib.psg_workspace_create(C.byref(ws)))
    try:
        A.check(lib.psg_workspace_reserve(ws, None, block.shape[0], 0))
        out = torch.zeros(5, dtype=torch.float64, device="cuda")
        st = torch.cuda.current_stream().cuda_stream
        A.check(lib.psg_panel_stats(ws, block.data_ptr(), dtype, block.shape[0], block.shape[1],
                                    live.data_ptr(), clip, out.data_ptr(), st))
        torch.cuda.synchronize()
        return out.cpu().numpy()
    finally:
        lib.psg_workspace_destroy(ws)


def stats_static(lib, block, dtype, live, clip):
    out = torch.full((5,), -7.0, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    A.check(lib.psg_panel_stats_static(block.data_ptr(), dtype, block.shape[0], block.shape[1],
                                       live.data_ptr(), clip, out.data_ptr(), st))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def close(got, want, rel):
    for x, y in zip(got, want):
        if math.isnan(y):
            assert math.isnan(x), (got, want)
        else:
            assert abs(x - y) <= rel * max(abs(y), 1e-300), (got, want)


def oracle_stats(data, live_np, clip):
    o = O.panel_stats(data, live_np, clip, signed=True)
    return np.array([o["rms"], o["maxAbs"], o["clip"], o["rows"], o["samples"]])


CASES = [
    (700, 1500, np.float32, 99.0),
    (333, 900, np.float32, 37.5),
    (257, 1201, np.float64, 99.0),
    (190, 640, np.float32, math.nan),
    (150, 333, np.float64, 100.0),
    (0, 64, np.float32, 99.0),
]


@pytest.mark.parametrize("rows,cols,dt,clip", CASES)
def test_static_panel_stats_match_oracle_and_workspace_form_on_two_calls(rows, cols, dt, clip):
    lib = A.lib()
    rng = np.random.default_rng(23 + rows)
    dtype = A.F32 if dt == np.float32 else A.F64
    for call in range(2):
        data = (rng.standard_normal((rows, cols)) * (1 + 3 * call)).astype(dt)
        live_np = rng.integers(0, cols + 1, rows).astype(np.int32)
        if rows > 10:
            live_np[5] = 0    # a live row with no samples: counted, no samples
            live_np[6] = -1   # a row that is not live: left out
            data[7, 3] = np.nan  # a row the statistics leave out
            live_np[7] = max(live_np[7], 4)
            data[8, 0] = np.inf
            live_np[8] = max(live_np[8], 1)
        block = torch.from_numpy(data).cuda() if rows else torch.zeros((0, cols), dtype=getattr(torch, dt.__name__),
                                                                       device="cuda")
        live = torch.from_numpy(live_np).cuda() if rows else torch.zeros(1, dtype=torch.int32, device="cuda")
        want = oracle_stats(data, live_np, clip)
        ws_form = stats_with_workspace(lib, block, dtype, live, clip)
        got = stats_static(lib, block, dtype, live, clip)
        close(got, ws_form, 1e-12)
        close(ws_form, want, 1e-12)
        close(got, want, 1e-12)
        if rows:
            assert got[3] > 0 and got[4] > 0
            if not math.isnan(clip):
                assert not math.isnan(got[2])
        else:
            assert got[3] == 0 and got[4] == 0 and math.isnan(got[2])


def test_static_panel_stats_reject_too_many_rows():
    lib = A.lib()
    rows = 65537
    block = torch.zeros(rows, 1, device="cuda")
    live = torch.ones(rows, dtype=torch.int32, device="cuda")
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    st = lib.psg_panel_stats_static(block.data_ptr(), A.F32, rows, 1, live.data_ptr(), 99.0,
                                    out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == A.EINVAL
    assert "at most 65536 rows" in lib.psg_last_error().decode()
