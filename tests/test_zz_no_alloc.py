"""psg_panel_stats_static, the entry point for callers that cannot allocate
device memory (a viewer computing display-gain statistics every frame inside
a fixed memory budget, say): called through the C ABI twice in a row, each
time it must give what psg_panel_stats gives with a workspace on the same
block. Named to run last: it holds a library-wide scratch array, and a run
stopping at its first failure has then already run every other test."""
import ctypes as C
import math

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


def stats_with_workspace(lib, block, live, clip):
    ws = C.c_void_p()
    A.check(lib.psg_workspace_create(C.byref(ws)))
    try:
        plan = C.c_void_p()
        ops = A.ops_array([])
        A.check(lib.psg_plan_compile(ops, 0, A.F32, 2.0, block.shape[1], 0, C.byref(plan)))
        A.check(lib.psg_workspace_reserve(ws, plan, block.shape[0], 0))
        out = torch.zeros(5, dtype=torch.float64, device="cuda")
        st = torch.cuda.current_stream().cuda_stream
        A.check(lib.psg_panel_stats(ws, block.data_ptr(), A.F32, block.shape[0], block.shape[1],
                                    live.data_ptr(), clip, out.data_ptr(), st))
        torch.cuda.synchronize()
        lib.psg_plan_destroy(plan)
        return out.cpu().numpy()
    finally:
        lib.psg_workspace_destroy(ws)


def stats_static(lib, block, live, clip):
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    A.check(lib.psg_panel_stats_static(block.data_ptr(), A.F32, block.shape[0], block.shape[1],
                                       live.data_ptr(), clip, out.data_ptr(), st))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def close(a, b, rel=1e-12):
    for x, y in zip(a, b):
        if math.isnan(y):
            assert math.isnan(x)
        else:
            assert abs(x - y) <= rel * max(abs(y), 1e-300), (a, b)


def test_static_panel_stats_match_workspace_form_on_two_calls():
    lib = A.lib()
    rng = np.random.default_rng(23)
    for call, (rows, cols, clip) in enumerate([(700, 1500, 99.0), (333, 900, 37.5)]):
        data = (rng.standard_normal((rows, cols)) * (1 + call)).astype(np.float32)
        live_np = rng.integers(0, cols + 1, rows).astype(np.int32)
        live_np[5] = 0
        data[7, 3] = np.nan  # a row the statistics leave out
        block = torch.from_numpy(data).cuda()
        live = torch.from_numpy(live_np).cuda()
        want = stats_with_workspace(lib, block, live, clip)
        got = stats_static(lib, block, live, clip)
        close(got, want)
        assert want[3] > 0 and not math.isnan(want[2])


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
