"""A panel split by traces over the ranks of a process group, one process
per GPU (torch.distributed: NCCL between GPUs, gloo on host tensors).

Traces are independent in every step of a plan (filter/apply.nim:81-84,
tests/tpipeline.nim:281-304), so each rank runs the plan on its own rows and
nothing crosses the ranks, with one exception: a per-panel normalization
takes one factor over the whole panel (gain/gain.nim:221-240, over
panelStats, gain/stats.nim:253-304). Its statistics merge: each rank
computes the partials of its rows (``PipelinePlan.panelPartials``: Σx²,
samples, rows, maxAbs and the 65536-bin histogram of |x|), the ranks sum
them and take the maximum of maxAbs (two all-reduces, the only collectives
of the path), and each rank derives the same factor from the merged
partials (``PipelinePlan.panelFactorFrom``). This is the parts API of
pipeline.nim:604-734 (``partNeedsPanel``, ``panelFactorOf``, ``runPart``)
with the factor's statistics reduced over ranks instead of read from one
block.

Every rank takes the same collectives in the same order, including ranks
whose shard has no rows; a rank that fails before a collective makes the
others' next collective fail when the process group's timeout runs out.
"""
from __future__ import annotations

from . import _abi as A


def shardRows(rows: int, world: int, rank: int) -> tuple[int, int]:
    """The contiguous rows ``[a, b)`` of ``rank`` among ``world`` ranks:
    sizes that differ by at most one, in rank order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    if rows < 0:
        raise ValueError(f"rows must be ≥ 0, got {rows}")
    base, extra = divmod(rows, world)
    a = rank * base + min(rank, extra)
    return a, a + base + (1 if rank < extra else 0)


def mergeLocal(partials):
    """The merge of partials held by one process (shards processed one after
    the other, or on one device): their sum, with the maximum of maxAbs."""
    partials = list(partials)
    if not partials:
        raise ValueError("no partials to merge")
    out = partials[0].clone()
    for p in partials[1:]:
        mx = max(float(out[3]), float(p[3]))
        out += p
        out[3] = mx
    return out


def mergePartials(partial, group=None):
    """Merges ``partial`` (a float64 tensor of ``PANEL_PARTIAL_DOUBLES``
    values, on the device for NCCL or on the host for gloo) over the ranks of
    ``group`` in place and returns it. Without an initialized process group
    (one process), it is returned unchanged."""
    import torch
    import torch.distributed as dist
    if partial.dtype != torch.float64 or partial.numel() != A.PANEL_PARTIAL_DOUBLES:
        raise ValueError(f"a partial is {A.PANEL_PARTIAL_DOUBLES} float64 values")
    if not dist.is_available() or not dist.is_initialized():
        return partial
    mx = partial[3:4].clone()
    partial[3] = 0.0
    dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX, group=group)
    partial[3:4] = mx
    return partial


def applySharded(plan, src, dst, meta, ws, group=None):
    """``apply`` (pipeline.nim:725-772) on this rank's shard of a panel:
    ``src``/``dst`` hold the rank's rows (``src`` None: in place) and
    ``meta`` describes them. Part by part: a part that starts with a
    per-panel normalization first merges the ranks' partial statistics
    (``mergePartials``) into one factor, which every rank applies. The
    result on each rank equals the rows of one ``apply`` over the whole
    panel (bit for bit for max and percentile statistics; the Σx² of an RMS
    statistic is summed in another order)."""
    for part in range(plan.partCount):
        from0 = part == 0 and src is not None
        factor = None
        if plan.partNeedsPanel(part):
            partial = plan.panelPartials(src if from0 else dst, meta, part, ws)
            mergePartials(partial, group)
            factor = plan.panelFactorFrom(partial, part, ws)
        plan.runPart(src if from0 else None, dst, meta, part, factor, ws)
    return dst


# ------------------------------------------------------------ by channel
# A vibroseis gather (vibroseis/vstack.nim:118-471, correlate.nim:421-464):
# every sweep of a channel stacks into that channel's output row, so the
# gather splits by channel with nothing crossing the ranks until the stacked
# rows are put together: each rank correlates and stacks the records of its
# channels (all their sweeps), and one all-gather assembles the stack.

def channelShard(rowMap, channels: int, world: int, rank: int):
    """The records of ``rank``'s channels: ``(records, localMap, (c0, c1))``
    with the channels ``[c0, c1)`` from ``shardRows`` over the channels, the
    ascending indices of the records whose channel (``rowMap[r]``) is one of
    them, and those records' output rows within the rank's stack
    (``rowMap − c0``). Records mapped outside ``[0, channels)`` go to no
    rank, as the stack skips them."""
    import numpy as np
    c0, c1 = shardRows(channels, world, rank)
    rm = np.asarray(rowMap, dtype=np.int64)
    idx = np.nonzero((rm >= c0) & (rm < c1))[0]
    return idx, (rm[idx] - c0).astype(np.int32), (c0, c1)


def gatherChannels(local, channels: int, group=None):
    """The ranks' stacked rows (``local``: this rank's ``[c1 − c0, samples]``
    tensor, on the device for NCCL or on the host for gloo) put together in
    channel order on every rank: one all-gather of equal-sized blocks (each
    rank's rows padded to the largest share). Without an initialized process
    group, ``local`` is the whole stack and is returned."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return local
    world = dist.get_world_size(group)
    per = -(-channels // world)
    buf = torch.zeros((per,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    buf[:local.shape[0]] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = []
    for r in range(world):
        a, b = shardRows(channels, world, r)
        out.append(parts[r][:b - a])
    return torch.cat(out)


class ChannelSplit:
    """``correlateInto`` with its vertical stack over a gather split by
    channel, set up once for a gather layout (``meta`` and ``rowMap`` over
    the gather's records, ``channels`` stacked rows) and run per gather:
    this rank correlates the records of its channels (every sweep of them),
    stacks each on its channel, and the stacked rows of every rank are
    gathered into the whole ``[channels, outSamples]`` float32 stack on this
    rank's device. ``norm`` is the stack's normalization (stackInto's; None:
    its default)."""

    def __init__(self, cplan, meta, rowMap, channels: int, group=None, norm=None):
        import numpy as np
        import torch
        import torch.distributed as dist
        from .meta import ChunkMeta
        from .vibroseis import initRecordStack
        self.cplan, self.channels, self.group, self.norm = cplan, channels, group, norm
        world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
        rank = dist.get_rank(group) if world > 1 else 0
        self.idx, lmap, (c0, c1) = channelShard(rowMap, channels, world, rank)
        self.dev = torch.device("cuda", torch.cuda.current_device())
        failed = np.nonzero(np.isin(self.idx, meta.failed))[0]
        self.meta = ChunkMeta(meta.status[self.idx], meta.numSamples[self.idx], meta.t0[self.idx], meta.dtMs,
                              meta.firstSample, failed, meta.offsets[self.idx])
        self.all = self.idx.size == len(rowMap) and bool(np.all(self.idx == np.arange(len(rowMap))))
        self.sel = torch.from_numpy(self.idx).to(self.dev)
        self.lmap = torch.from_numpy(lmap).to(self.dev)
        self.stack = initRecordStack(c1 - c0, cplan.outSamples, meta.dtMs)
        self.out = torch.empty((c1 - c0, cplan.outSamples), dtype=torch.float32, device=self.dev)
        self.mine = None

    def run(self, records, dst=None):
        """The whole stack of ``records`` (the gather's [records, samples]
        block: host or device; only this rank's records are read)."""
        import numpy as np
        import torch
        if isinstance(records, torch.Tensor) and records.device == self.dev and records.is_contiguous() and self.all:
            mine = records
        elif isinstance(records, torch.Tensor) and records.device == self.dev:
            shape = (self.idx.size,) + tuple(records.shape[1:])
            if self.mine is None or tuple(self.mine.shape) != shape or self.mine.dtype != records.dtype:
                self.mine = torch.empty(shape, dtype=records.dtype, device=self.dev)
            torch.index_select(records, 0, self.sel, out=self.mine)
            mine = self.mine
        else:
            mine = torch.from_numpy(np.ascontiguousarray(np.asarray(records)[self.idx])).to(self.dev)
        self.stack.clear()
        if self.idx.size:
            self.cplan.correlateInto(mine, None, self.meta, stack=self.stack, rowMap=self.lmap)
        if self.norm is None:
            self.stack.stackInto(self.out)
        else:
            self.stack.stackInto(self.out, self.norm)
        whole = gatherChannels(self.out, self.channels, self.group)
        if dst is not None:
            dst.copy_(whole)
        return whole


def correlateStackSharded(cplan, records, meta, rowMap, channels: int, dst=None, group=None, norm=None):
    """One gather through a ``ChannelSplit`` (set up for this call)."""
    return ChannelSplit(cplan, meta, rowMap, channels, group, norm).run(records, dst)
