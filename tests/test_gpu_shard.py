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


def test_correlate_stack_by_channel_in_one_process_equals_the_whole_gather():
    """correlateStackSharded without a process group (one rank: every
    channel) gives correlateInto + stack over all records; and each channel
    block of two shards, stacked on its own, matches the whole stack's rows
    bit for bit (the rows a two-rank all-gather puts together)."""
    spec = P.linearSweep(8, 80, 4000, 2, P.initSweepTaper(200, 200, P.tpCos2))
    pilot = P.generatePilot(spec, np.float64)
    recs = synth.vibroseis_records(pilot.samples, channels=12, samples=4001, sweeps=3)
    sweeps, ch, ns = recs.shape
    block = recs.reshape(sweeps * ch, ns)
    rmap = (np.arange(sweeps * ch) % ch).astype(np.int32)
    meta = P.initChunkMeta(np.full(sweeps * ch, P.tsLive, np.int32), np.full(sweeps * ch, ns, np.int32), 2.0)
    cplan = P.initCorrelationPlan(P.float32, pilot, 2.0, ns, outSamples=1500)
    st = P.initRecordStack(ch, 1500, 2.0)
    cplan.correlateInto(torch.from_numpy(block).cuda(), None, meta, stack=st,
                        rowMap=torch.from_numpy(rmap).cuda())
    want = torch.empty(ch, 1500, device="cuda")
    st.stackInto(want)
    got = shard.correlateStackSharded(cplan, torch.from_numpy(block).cuda(), meta, rmap, ch)
    assert torch.equal(got, want)
    parts = []
    for r in range(2):
        idx, lmap, (c0, c1) = shard.channelShard(rmap, ch, 2, r)
        s2 = P.initRecordStack(c1 - c0, 1500, 2.0)
        sub = P.initChunkMeta(meta.status[idx], meta.numSamples[idx], 2.0)
        cplan.correlateInto(torch.from_numpy(np.ascontiguousarray(block[idx])).cuda(), None, sub, stack=s2,
                            rowMap=torch.from_numpy(lmap).cuda())
        o = torch.empty(c1 - c0, 1500, device="cuda")
        s2.stackInto(o)
        parts.append(o)
    assert torch.equal(torch.cat(parts), want)


def test_server_pool_places_requests_over_two_loops():
    """Two request loops (here both on device 0): host requests go to the
    less loaded one, each result the plain apply's."""
    plan = P.initPipeline(FLOWS["pct"]).compile(P.float32, 2.0, 3001)
    g = synth.c2(seed=22, rows=400)
    meta = g.meta()
    ws = P.initWorkspace()
    ws.reserve(plan, rows=400, cols=3001)
    want = np.zeros_like(g.data)
    plan.apply(g.data, want, meta, ws)
    loops = [P.Server(0, 256 << 20), P.Server(0, 256 << 20)]
    with P.ServerPool(loops=loops) as pool:
        outs = [np.zeros_like(g.data) for _ in range(8)]
        tickets = [pool.submit(plan, g.data, o, meta) for o in outs]
        for t in tickets:
            pool.wait(t, 30000)
    assert {i for i, _ in tickets} == {0, 1}
    for o in outs:
        assert np.array_equal(o, want)
