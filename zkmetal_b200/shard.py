"""Point-range sharding of one MSM across ranks (one process per GPU).

An MSM is a sum, so rank g of G computes the partial MSM of its contiguous
slice of points and scalars; the G partial results (one point each, in the
library's result layout) are all-gathered over the process group and added.
There is no other exchange.  The addition of the gathered points is passed in
(`add_results`): on GPUs it is the library's zkmsm_sum_results_device, which
runs on the device.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def shard_range(n_total: int, world: int, rank: int):
    """[start, stop) of `rank`'s points: contiguous, balanced, covering n_total."""
    if world <= 0 or not 0 <= rank < world or n_total < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(n_total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def gather_partials(partial: torch.Tensor, world: int, group=None) -> torch.Tensor:
    """All-gather one result per rank (uint8 tensor of equal size on every
    rank) into a [world * size] tensor, rank order."""
    out = torch.empty(world * partial.numel(), dtype=partial.dtype, device=partial.device)
    if world == 1:
        out.copy_(partial)
        return out
    dist.all_gather_into_tensor(out, partial.contiguous(), group=group)
    return out


def sharded_msm(n_total: int, world: int, rank: int, partial_msm, add_results, group=None):
    """Run this rank's shard through `partial_msm(start, stop) -> uint8 tensor`
    and combine all ranks' partials with `add_results(gathered, world)`."""
    start, stop = shard_range(n_total, world, rank)
    mine = partial_msm(start, stop)
    gathered = gather_partials(mine, world, group)
    return add_results(gathered, world)
