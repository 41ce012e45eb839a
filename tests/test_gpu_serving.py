"""The request loop (continuous batching): every request's result equals the
plain apply of its plan, bit for bit, whether it ran alone or batched with
others of different plans, widths and trace counts; admission refuses what
cannot fit; waits are bounded."""
import threading

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
    with pytest.raises(ValueError):
        plan64 = P.initPipeline(flow).compile(P.float64, 2.0, 1000)
        with P.Server(arena_bytes=4 << 20) as srv:
            x = np.ones((10, 1000))
            srv.submit(plan64, x, np.zeros_like(x), P.liveMeta(10, 1000, 2.0))


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
