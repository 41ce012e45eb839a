"""The request loop (continuous batching): every request's result equals the
plain apply of its plan, bit for bit, whether it ran alone or batched with
others of different plans, widths and trace counts; admission refuses what
cannot fit; waits are bounded."""
import threading
import time

import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import synth, _abi as A

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


def test_results_are_the_same_alone_and_in_the_mix():
    flows = synth.viewer_flows()
    margins = [P.initPipeline(f).requiredMargin(2.0) for f in flows]
    reqs = synth.viewer_requests(24, seed=7, margins=margins)
    g = synth.shot_gather(5000, 6001, 2.0, seed=9, workload="c4", live_range=(3000, 6001))
    plans, jobs = {}, []
    for r in reqs:
        key = (r.flow, r.cols)
        if key not in plans:
            plans[key] = P.initPipeline(flows[r.flow]).compile(P.float32, 2.0, r.cols, recordSamples=6001)
        src = np.ascontiguousarray(g.data[:r.rows, r.first:r.first + r.cols])
        meta = P.initChunkMeta(g.status[:r.rows], g.numSamples[:r.rows], 2.0, g.t0Ms[:r.rows], r.first)
        jobs.append((plans[key], src, meta))
    # alone: the plain per-call apply
    want = []
    for plan, src, meta in jobs:
        ws = P.initWorkspace()
        ws.reserve(plan, rows=src.shape[0], cols=src.shape[1])
        dst = np.zeros_like(src)
        plan.apply(src, dst, meta, ws)
        want.append(dst)
    # in the mix: all submitted at once from two threads
    with P.Server(arena_bytes=1 << 30) as srv:
        outs = [np.zeros_like(src) for _, src, _ in jobs]
        tickets = [None] * len(jobs)

        def submit(idx):
            for i in idx:
                plan, src, meta = jobs[i]
                tickets[i] = srv.submit(plan, src, outs[i], meta)

        th = [threading.Thread(target=submit, args=(range(k, len(jobs), 2),)) for k in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for t in tickets:
            srv.wait(t)
        st = srv.stats()
    for got, w in zip(outs, want):
        assert np.array_equal(got, w)
    assert st["completed"] == len(jobs)
    assert st["requests_per_launch"] > 1  # requests were batched


def test_admission_and_bounded_waits():
    flow = synth.viewer_flows()[0]
    plan = P.initPipeline(flow).compile(P.float32, 2.0, 1000)
    with P.Server(arena_bytes=4 << 20) as srv:
        big = np.zeros((2000, 1000), np.float32)
        meta = P.liveMeta(2000, 1000, 2.0)
        with pytest.raises(MemoryError, match="admission refused"):
            srv.submit(plan, big, np.zeros_like(big), meta)
        small = np.ones((100, 1000), np.float32)
        t = srv.submit(plan, small, np.zeros_like(small), P.liveMeta(100, 1000, 2.0))
        srv.wait(t, 10000)
        with pytest.raises(ValueError, match="unknown ticket"):
            srv.wait(t, 10)
        assert srv.stats()["refused"] == 1
    # a muting plan needs its rows' keys: psg_submit without them refuses it
    import ctypes as C
    mute = P.initPipeline([P.muteTopOp(P.lmoMute(2000), taperMs=40), P.agcOp(500)]).compile(P.float32, 2.0, 1000)
    with P.Server(arena_bytes=4 << 20) as srv:
        x = np.ones((10, 1000), np.float32)
        y = np.zeros_like(x)
        live, start = P.liveMeta(10, 1000, 2.0).flat(1000, 0)
        t = C.c_uint64()
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        st = A.lib().psg_submit(srv.h, mute.h, p(x), p(y), 10, 1000, p(live), p(start), 2.0, C.byref(t))
        assert st == A.EINVAL and "mutes" in A.lib().psg_last_error().decode()


# every kind of plan the plain apply takes, each served as the plain apply
# gives it: the batched trace kernel (demean → band-pass → AGC at 3001
# samples), a per-panel normalization (two parts, the factor from the
# request's own rows), float64, an IIR filter, a mute (the rows' keys), and
# the batched generic kernel (the viewer's flows)
KIND_FLOWS = {
    "trace": ([P.demeanOp(), P.filterOp(P.bandPass(P.Corners(3, 6, 70, 90)).withNotch(50, 2)), P.agcOp(300)],
              P.float32),
    "panel": ([P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 60, 80)), P.normalizeOp(P.normRms, P.perPanel)],
              P.float32),
    "f64": ([P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 60, 80)), P.agcOp(500)], P.float64),
    "iir": ([P.iirOp(P.butterBandPass(4, 60, 24)), P.agcOp(500)], P.float32),
    "mute": ([P.muteTopOp(P.lmoMute(2000), taperMs=40), P.bandPassOp(P.Corners(4, 8, 60, 80)), P.agcOp(500)],
             P.float32),
    "generic": (synth.viewer_flows()[1], P.float32),
}


def kind_jobs(seed=11):
    g = synth.shot_gather(600, 3001, 2.0, seed=seed, workload="c4", live_range=(1500, 3001))
    offsets = np.linspace(-3000.0, 3000.0, 600)
    jobs = []
    rng = np.random.default_rng(seed)
    for k, (name, (flow, T)) in enumerate(sorted(KIND_FLOWS.items())):
        for j in range(2):
            rows = int(rng.integers(40, 600))
            plan = P.initPipeline(flow).compile(T, 2.0, 3001)
            dt = np.float32 if T == P.float32 else np.float64
            src = np.ascontiguousarray(g.data[:rows]).astype(dt)
            meta = P.initChunkMeta(g.status[:rows], g.numSamples[:rows], 2.0, g.t0Ms[:rows],
                                   offsets=offsets[:rows])
            jobs.append((name, plan, src, meta))
    return jobs


def plain(plan, src, meta):
    ws = P.initWorkspace()
    ws.reserve(plan, rows=src.shape[0], cols=src.shape[1])
    dst = np.zeros_like(src)
    plan.apply(src, dst, meta, ws)
    return dst


def test_every_plan_kind_is_served_as_the_plain_apply():
    jobs = kind_jobs()
    want = [plain(plan, src, meta) for _, plan, src, meta in jobs]
    with P.Server(arena_bytes=1 << 30) as srv:
        # each alone, then all at once (host buffers)
        for (name, plan, src, meta), w in zip(jobs, want):
            out = np.zeros_like(src)
            srv.wait(srv.submit(plan, src, out, meta), 30000)
            assert np.array_equal(out, w, equal_nan=True), name
        outs = [np.zeros_like(src) for _, _, src, _ in jobs]
        tickets = [srv.submit(plan, src, o, meta) for (_, plan, src, meta), o in zip(jobs, outs)]
        for t in tickets:
            srv.wait(t, 30000)
        st = srv.stats()
    for (name, *_), got, w in zip(jobs, outs, want):
        assert np.array_equal(got, w, equal_nan=True), name
    assert st["completed"] == 2 * len(jobs)  # each alone, then all at once


def test_device_requests_are_served_in_place_as_the_plain_apply():
    jobs = kind_jobs(seed=12)
    with P.Server(arena_bytes=64 << 20) as srv:
        srcs = [torch.from_numpy(src).cuda() for _, _, src, _ in jobs]
        want = []
        for (name, plan, src, meta), s in zip(jobs, srcs):
            ws = P.initWorkspace()
            ws.reserve(plan, rows=src.shape[0], cols=src.shape[1])
            d = torch.zeros_like(s)
            plan.apply(s, d, meta, ws)
            want.append(d)
        outs = [torch.full_like(s, float("nan")) for s in srcs]
        tickets = [srv.submit(plan, s, o, meta) for (_, plan, _, meta), s, o in zip(jobs, srcs, outs)]
        for t in tickets:
            srv.wait(t, 30000)
        torch.cuda.synchronize()
        for (name, *_), got, w in zip(jobs, outs, want):
            assert torch.equal(got.nan_to_num(7.0), w.nan_to_num(7.0)), name
        # the device form takes no arena bytes: a 64 MiB arena serves far more
        big = torch.from_numpy(np.ascontiguousarray(jobs[0][2])).cuda().repeat(40, 1)
        assert big.numel() * big.element_size() > 64 << 20
        name, plan, src, meta = jobs[0]
        reps = P.initChunkMeta(np.tile(meta.status, 40), np.tile(meta.numSamples, 40), 2.0,
                               np.tile(meta.t0, 40), offsets=np.tile(meta.offsets, 40))
        o = torch.empty_like(big)
        srv.wait(srv.submit(plan, big, o, reps), 30000)
        torch.cuda.synchronize()
        rows = src.shape[0]
        assert torch.equal(o[:rows].nan_to_num(7.0), want[0].nan_to_num(7.0))
        assert torch.equal(o[-rows:].nan_to_num(7.0), want[0].nan_to_num(7.0))


def test_large_ready_batches_run_beside_running_ones():
    """Requests that hold enough rows to fill the device start a batch while
    another batch's kernels run (psg_server_counters' overlapped), and every
    result is still the plain apply's."""
    flow, T = KIND_FLOWS["trace"]
    plan = P.initPipeline(flow).compile(T, 2.0, 3001)
    g = synth.c2(rows=2000)
    meta = g.meta()
    src = torch.from_numpy(g.data).cuda()
    ws = P.initWorkspace()
    ws.reserve(plan, rows=2000, cols=3001)
    want = torch.empty_like(src)
    plan.apply(src, want, meta, ws)
    with P.Server(arena_bytes=1 << 20) as srv:
        outs = [torch.empty_like(src) for _ in range(12)]
        tickets = []
        for o in outs:
            tickets.append(srv.submit(plan, src, o, meta))
            time.sleep(2e-5)  # the next request arrives while this one runs
        for t in tickets:
            srv.wait(t, 30000)
        c = srv.counters()
    torch.cuda.synchronize()
    for o in outs:
        assert torch.equal(o, want)
    assert c["batches"] >= 2 and c["kernels"] >= c["batches"]
    assert c["overlapped"] >= 1


def test_cancel_and_poll():
    """psg_cancel / psg_poll: requests still queued behind a small arena are
    cancelled (their buffers untouched, wait raises CancelledError); the
    rest complete with the plain apply's result; a started request is not
    cancelled."""
    from processseg_b200.server import CancelledError
    flow = synth.viewer_flows()[0]
    plan = P.initPipeline(flow).compile(P.float32, 2.0, 1000)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=2000, cols=1000)
    rng = np.random.default_rng(3)
    srcs = [rng.standard_normal((2000, 1000)).astype(np.float32) for _ in range(12)]
    meta = P.liveMeta(2000, 1000, 2.0)
    # an arena of one 8 MB request at a time: the later ones stay queued
    with P.Server(arena_bytes=9 << 20) as srv:
        dsts = [np.full((2000, 1000), 7.0, np.float32) for _ in srcs]
        tickets = [srv.submit(plan, s, d, meta) for s, d in zip(srcs, dsts)]
        cancelled = {t for t in tickets[-6:] if srv.cancel(t)}
        assert cancelled, "a one-request arena leaves requests queued"
        for i, t in enumerate(tickets):
            if t in cancelled:
                assert srv.poll(t)
                with pytest.raises(CancelledError):
                    srv.wait(t, 10000)
                assert np.all(dsts[i] == 7.0)
            else:
                srv.wait(t, 10000)
                want = np.zeros_like(srcs[i])
                plan.apply(srcs[i], want, meta, ws)
                assert np.array_equal(dsts[i], want)
        t = srv.submit(plan, srcs[0], dsts[0], meta)
        srv.wait(t, 10000)
        with pytest.raises(ValueError, match="unknown ticket"):
            srv.cancel(t)
