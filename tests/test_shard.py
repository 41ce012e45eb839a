"""Trace sharding over ranks on the host: two gloo ranks on CPU.

The device side of a shard (psg_panel_partials / psg_panel_factor_from /
psg_run_part) is covered by tests/test_gpu_shard.py; here a numpy stand-in
computes each rank's partial statistics by the rules of panelStats
(gain/stats.nim:253-304), so that these tests check what crosses the ranks:
the partition, the merge (two all-reduces), the order of the collectives in
``applySharded``, and that a rank which fails before a collective makes the
others' collective fail within the process group's timeout.
"""
import datetime
import math
import multiprocessing as mp
import os
import socket
import time
import traceback

import numpy as np
import pytest

from processseg_b200 import _abi as A
from processseg_b200 import shard

torch = pytest.importorskip("torch")

HIST_SHIFT, MAX_KEY = 15, 0xFEFF


def np_partials(block, live):
    """[Σx², samples, rows, maxAbs] + 65536 counts of the usable rows."""
    out = np.zeros(A.PANEL_PARTIAL_DOUBLES)
    rows, cols = block.shape
    for r in range(rows):
        n = min(max(int(live[r]), 0), cols)
        if n == 0:
            continue
        x = block[r, :n]
        ss = float(np.sum(x.astype(np.float64) ** 2))
        m = float(np.max(np.abs(x.astype(np.float64))))
        if not math.isfinite(m) or ss == math.inf:
            continue
        out[0] += ss
        out[1] += n
        out[2] += 1
        out[3] = max(out[3], m)
        keys = np.minimum(np.abs(x.astype(np.float32)).view(np.uint32) >> HIST_SHIFT, MAX_KEY)
        np.add.at(out, A.PANEL_PARTIAL_HEAD + keys.astype(np.int64), 1.0)
    return out


def order_stat(h, j, mx):
    """orderStat (gain/stats.nim:237-251) over the counts ``h``."""
    below = 0
    for k in range(MAX_KEY + 1):
        c = int(h[k])
        if below + c > j:
            if k == 0:
                return 0.0
            lo = float(np.uint32(k << HIST_SHIFT).view(np.float32))
            hi = min(float(np.uint32((k + 1) << HIST_SHIFT).view(np.float32)), mx)
            return min(max(lo + (float(j - below) + 0.5) / float(c) * (hi - lo), lo), mx)
        below += c
    return mx


def clip_of(partial, p):
    """The clip percentile of merged partials (panelStats' last lines)."""
    samples, mx = int(partial[1]), float(partial[3])
    h = partial[A.PANEL_PARTIAL_HEAD:]
    rank = float(samples - 1) * p / 100
    k = min(int(math.floor(rank)), samples - 1)
    lower = order_stat(h, k, mx)
    f = rank - k
    if f == 0 or k + 1 >= samples:
        return lower
    return lower + f * (order_stat(h, k + 1, mx) - lower)


def panel(seed=11, rows=37, cols=300):
    g = np.random.default_rng(seed)
    b = (g.standard_normal((rows, cols)) * g.uniform(0.1, 10, rows)[:, None]).astype(np.float32)
    live = g.integers(0, cols + 1, rows).astype(np.int32)
    live[3] = 0
    b[5, 7] = np.nan  # a row a panel leaves out
    return b, live


class NumpyPlan:
    """Two parts: ×2, then a per-panel normalization to 1 of ``stat``
    followed by ×0.5 — the shape of a plan with a per-panel step, run on
    host arrays."""

    partCount = 2

    def __init__(self, stat, p=99.0, fail_rank=None, rank=0):
        self.stat, self.p, self.fail_rank, self.rank = stat, p, fail_rank, rank

    def partNeedsPanel(self, part):
        return part == 1

    def panelPartials(self, b, meta, part, ws):
        if self.fail_rank == self.rank:
            raise RuntimeError("planted failure before the exchange")
        return torch.from_numpy(np_partials(b, meta))

    def panelFactorFrom(self, partial, part, ws):
        q = partial.numpy()
        samples = q[1]
        if samples == 0:
            return torch.tensor([math.nan], dtype=torch.float64)
        level = {"max": q[3], "rms": math.sqrt(q[0] / samples), "pct": None}[self.stat]
        if level is None:
            level = clip_of(q, self.p)
        f = 1.0 / level if level > 0 and math.isfinite(level) else math.nan
        return torch.tensor([f], dtype=torch.float64)

    def runPart(self, src, dst, live, part, factor, ws):
        if src is not None:
            dst[...] = src
        for r in range(dst.shape[0]):
            n = min(max(int(live[r]), 0), dst.shape[1])
            if part == 0:
                dst[r, :n] *= np.float32(2)
            else:
                f = float(factor[0])
                if not math.isnan(f):
                    dst[r, :n] = (dst[r, :n] * np.float32(f)).astype(np.float32)
                dst[r, :n] *= np.float32(0.5)


def gather_case(channels=6, sweeps=4, samples=700, seed=21):
    """A small vibroseis gather: ``sweeps`` records per channel, in sweep
    order (record r on channel r % channels), with one dead record."""
    g = np.random.default_rng(seed)
    n = channels * sweeps
    recs = g.standard_normal((n, samples)).astype(np.float32)
    live = np.full(n, samples, np.int32)
    live[5] = 0
    return recs, live, (np.arange(n) % channels).astype(np.int32), channels


PILOT = np.random.default_rng(5).standard_normal(150)


def oracle_stack(recs, live, rmap, channels, out=400):
    """The oracle's correlateInto of ``recs`` with the vertical stack of each
    on its channel (vibroseis/vstack.nim:186-202, 439-471), float32."""
    from oracle import oracle as O
    num = np.zeros((channels, out))
    cnt = np.zeros((channels, out), np.int32)
    if len(recs):
        corr, _, _ = O.correlate(PILOT, 2.0, 0.0, recs, live, 2.0, recs.shape[1], out)
        O.stack_add(num, cnt, corr, np.where(live > 0, out, 0).astype(np.int32), rmap)
    return O.stack_result(num, cnt, np.float32)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, job, q):
    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                world_size=world, timeout=datetime.timedelta(seconds=job.get("timeout", 30)))
        b, live = panel()
        a0, a1 = shard.shardRows(b.shape[0], world, rank)
        mine, my_live = b[a0:a1].copy(), live[a0:a1].copy()
        if job["kind"] == "channels":
            recs, live, rmap, nch = gather_case()
            idx, lmap, (c0, c1) = shard.channelShard(rmap, nch, world, rank)
            local = oracle_stack(recs[idx], live[idx], lmap, c1 - c0)
            whole = shard.gatherChannels(torch.from_numpy(local), nch)
            q.put((rank, "ok", (idx, whole.numpy())))
        elif job["kind"] == "merge":
            part = torch.from_numpy(np_partials(mine, my_live))
            shard.mergePartials(part)
            q.put((rank, "ok", part.numpy()))
        else:
            plan = NumpyPlan(job["stat"], fail_rank=job.get("fail_rank"), rank=rank)
            dst = np.zeros_like(mine)
            t0 = time.monotonic()
            try:
                shard.applySharded(plan, mine, dst, my_live, None)
                q.put((rank, "ok", (a0, a1, dst)))
            except Exception as e:
                q.put((rank, "error", (repr(e), time.monotonic() - t0)))
                return
        dist.barrier()
        dist.destroy_process_group()
    except Exception:
        q.put((rank, "error", (traceback.format_exc(), 0.0)))


def run_ranks(job, world=2, limit=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, job, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    deadline = time.monotonic() + limit
    while len(out) < world and time.monotonic() < deadline:
        try:
            r, status, val = q.get(timeout=1)
            out[r] = (status, val)
        except Exception:
            if all(not p.is_alive() for p in procs) and q.empty():
                break
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return out


def test_shard_rows_partition():
    for rows in (0, 1, 7, 2000, 50001):
        for world in (1, 2, 3, 8):
            spans = [shard.shardRows(rows, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == rows
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.shardRows(10, 2, 2)


def test_merge_local_matches_whole_panel():
    b, live = panel()
    whole = np_partials(b, live)
    parts = [torch.from_numpy(np_partials(b[a:c], live[a:c]))
             for a, c in (shard.shardRows(b.shape[0], 3, r) for r in range(3))]
    m = shard.mergeLocal(parts).numpy()
    assert np.array_equal(m[1:], whole[1:])
    assert abs(m[0] - whole[0]) <= 1e-15 * whole[0]


def test_partials_pin_the_oracle_panel_stats():
    from oracle import oracle as O
    b, live = panel()
    st = O.panel_stats(b, live, 99.0)
    whole = np_partials(b, live)
    assert int(whole[1]) == st["samples"] and int(whole[2]) == st["rows"]
    assert whole[3] == st["maxAbs"]
    assert clip_of(whole, 99.0) == st["clip"]
    assert abs(math.sqrt(whole[0] / whole[1]) - st["rms"]) <= 1e-15 * st["rms"]


def test_merge_over_two_gloo_ranks():
    out = run_ranks({"kind": "merge"})
    assert set(out) == {0, 1}, out
    b, live = panel()
    whole = np_partials(b, live)
    for r in (0, 1):
        status, m = out[r]
        assert status == "ok", m
        assert np.array_equal(m[1:], whole[1:])
        assert abs(m[0] - whole[0]) <= 1e-15 * whole[0]


@pytest.mark.parametrize("stat", ["max", "pct"])
def test_apply_sharded_equals_whole_panel(stat):
    out = run_ranks({"kind": "apply", "stat": stat})
    assert set(out) == {0, 1}, out
    b, live = panel()
    want = np.zeros_like(b)
    shard.applySharded(NumpyPlan(stat), b, want, live, None)
    got = np.zeros_like(b)
    for r in (0, 1):
        status, val = out[r]
        assert status == "ok", val
        a0, a1, dst = val
        got[a0:a1] = dst
    assert np.array_equal(got, want, equal_nan=True)


def test_a_failed_rank_ends_the_others_collective():
    out = run_ranks({"kind": "apply", "stat": "max", "fail_rank": 1, "timeout": 5}, limit=90)
    assert out.get(1, ("", None))[0] == "error"
    status, val = out.get(0, ("missing", None))
    assert status == "error", (status, val)
    assert val[1] < 60


def test_channel_shards_cover_every_record_once():
    recs, live, rmap, nch = gather_case()
    for world in (1, 2, 3, 4):
        seen = []
        for r in range(world):
            idx, lmap, (c0, c1) = shard.channelShard(rmap, nch, world, r)
            assert np.all((rmap[idx] >= c0) & (rmap[idx] < c1))
            assert np.array_equal(lmap, rmap[idx] - c0)
            seen.extend(idx.tolist())
        assert sorted(seen) == list(range(len(rmap)))
    # a record mapped to no channel goes to no rank
    bad = rmap.copy()
    bad[0] = -1
    assert 0 not in shard.channelShard(bad, nch, 1, 0)[0]


def test_stack_by_channel_over_two_gloo_ranks():
    """Each rank correlates and stacks the records of its channels (every
    sweep of them); the all-gather of the stacked rows equals one stack of
    the whole gather, bit for bit."""
    out = run_ranks({"kind": "channels"})
    assert set(out) == {0, 1}, out
    recs, live, rmap, nch = gather_case()
    want = oracle_stack(recs, live, rmap, nch)
    for r in (0, 1):
        status, val = out[r]
        assert status == "ok", val
        idx, whole = val
        assert np.array_equal(whole, want)
    assert sorted(out[0][1][0].tolist() + out[1][1][0].tolist()) == list(range(len(rmap)))
