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
