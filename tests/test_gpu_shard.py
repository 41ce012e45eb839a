"""The device side of a panel split by traces (psg_panel_partials,
psg_panel_factor_from, psg_run_part): shards of one panel, merged on one
GPU, give the factor of the whole panel, and running each shard with it
reproduces the whole panel's apply."""
import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import shard, synth

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]

BP = P.bandPass(P.Corners(3, 6, 70, 90))
FLOWS = {
    "pct": [P.demeanOp(), P.filterOp(BP), P.normalizeOp(P.normPercentile, P.perPanel, percentile=99.0),
            P.agcOp(300)],
    "max": [P.agcOp(200), P.normalizeOp(P.normMax, P.perPanel, target=2.0), P.scaleOp(0.5)],
    "rms": [P.demeanOp(), P.normalizeOp(P.normRms, P.perPanel, target=3.0),
            P.normalizeOp(P.normPercentile, P.perPanel, percentile=90.0)],
    # mutes read each shard's own rows' offsets and t0s (psg_run_part_keyed)
    "mutes": [P.muteTopOp(P.lmoMute(2000, t0Ms=40), taperMs=30), P.filterOp(BP),
              P.normalizeOp(P.normMax, P.perPanel), P.muteBottomOp(P.timeMute(4500), taperMs=50)],
}


def _sub_meta(g, a, b):
    return P.initChunkMeta(g.status[a:b], g.numSamples[a:b], g.dtMs, g.t0Ms[a:b], offsets=g.offsets[a:b])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("name", list(FLOWS))
def test_shards_reproduce_the_whole_panel(name, dtype):
    g = synth.c2(seed=21, rows=600, dtype=dtype)
    T = P.float32 if dtype == np.float32 else P.float64
    plan = P.initPipeline(FLOWS[name]).compile(T, 2.0, 3001)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=600, cols=3001)
    src = torch.from_numpy(g.data).cuda()
    want = torch.empty_like(src)
    plan.apply(src, want, g.meta(), ws)

    spans = [shard.shardRows(600, 3, r) for r in range(3)]
    outs = [torch.empty_like(src[a:b]) for a, b in spans]
    metas = [_sub_meta(g, a, b) for a, b in spans]
    srcs = [src[a:b].contiguous() for a, b in spans]
    for part in range(plan.partCount):
        factor = None
        if plan.partNeedsPanel(part):
            blocks = srcs if part == 0 else outs
            partials = [plan.panelPartials(blk, m, part, ws) for blk, m in zip(blocks, metas)]
            merged = shard.mergeLocal(partials)
            factor = plan.panelFactorFrom(merged, part, ws)
        for i in range(3):
            plan.runPart(srcs[i] if part == 0 else None, outs[i], metas[i], part, factor, ws)
    got = torch.cat(outs).cpu().numpy()
    w = want.cpu().numpy()
    if name in ("pct", "max", "mutes"):
        assert np.array_equal(got, w)
    else:
        # Σx² of the RMS statistic is summed in another order: the factor
        # differs by a few ulp at most.
        scale = np.sqrt(np.mean(w.astype(np.float64) ** 2))
        tol = 1e-6 if dtype == np.float32 else 1e-14
        assert np.max(np.abs(got.astype(np.float64) - w)) <= tol * scale


def test_one_shard_partials_give_the_panel_factor_bit_for_bit():
    g = synth.c2(seed=22, rows=300)
    for stat in (P.normMax, P.normRms, P.normPercentile):
        plan = P.initPipeline([P.normalizeOp(stat, P.perPanel)]).compile(P.float32, 2.0, 3001)
        ws = P.initWorkspace()
        ws.reserve(plan, rows=300, cols=3001)
        b = torch.from_numpy(g.data).cuda()
        f = plan.panelFactorOf(b, g.meta(), 0, ws)
        f2 = float(plan.panelFactorFrom(plan.panelPartials(b, g.meta(), 0, ws), 0, ws).item())
        assert f == f2


def test_apply_sharded_single_process_equals_apply():
    g = synth.c2(seed=23, rows=200)
    plan = P.initPipeline(FLOWS["pct"]).compile(P.float32, 2.0, 3001)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=200, cols=3001)
    src = torch.from_numpy(g.data).cuda()
    a, b = torch.empty_like(src), torch.empty_like(src)
    plan.apply(src, a, g.meta(), ws)
    shard.applySharded(plan, src, b, g.meta(), ws)
    assert torch.equal(a, b)


def test_parts_api_errors():
    plan = P.initPipeline(FLOWS["max"]).compile(P.float32, 2.0, 100)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=10, cols=100)
    b = torch.zeros(10, 100, device="cuda")
    m = P.liveMeta(10, 100, 2.0)
    assert not plan.partNeedsPanel(0) and plan.partNeedsPanel(1)
    with pytest.raises(AssertionError, match="no per-panel normalization"):
        plan.panelPartials(b, m, 0, ws)
    with pytest.raises(AssertionError, match="no part"):
        plan.runPart(None, b, m, 5, None, ws)
    with pytest.raises(ValueError):
        plan.runPart(None, torch.zeros(10, 101, device="cuda"), P.liveMeta(10, 101, 2.0), 0, None, ws)
