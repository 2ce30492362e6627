"""Data-parallel training over views (one process per GPU).

The path has exactly one exchange step: every rank renders and
back-propagates its own cameras with replicated parameters, the ranks' per-tet
gradient slots are summed (one all-reduce of 20 floats per tet over NCCL), and
every rank applies the same Adam update.  Views shard round-robin, so each rank
keeps the same number of cameras when the count divides evenly.
"""
from __future__ import annotations

from typing import Sequence


def shard_views(n_views: int, world: int, rank: int) -> list:
    """Indices of the views rank ``rank`` trains, round-robin over ``world`` ranks."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    return list(range(rank, n_views, world))


def allreduce_sum_(tensor, group=None, stream=None):
    """In-place sum of ``tensor`` over the process group (on ``stream`` if given)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return tensor
    if stream is not None:
        with torch.cuda.stream(stream):
            dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    else:
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor


class DataParallelStep:
    """accumulate (this rank's views) -> all-reduce of the gradient slots -> Adam."""

    def __init__(self, renderer, stream=None, group=None):
        self.r = renderer
        self.stream = stream
        self.group = group
        self._slots = None

    def __call__(self, cameras: Sequence, gt_images, lr_verts: float, lr_dens: float, lr_grads: float,
                 loss_type: int = 1, lr_base: float = 0.0, mode: str = "graph", lr_sh: float = 0.0):
        losses = self.r.accumulate_views(cameras, gt_images, loss_type=loss_type, mode=mode)
        if self._slots is None:
            self._slots = self.r.grad_slots()
        allreduce_sum_(self._slots, self.group, self.stream)
        self.r.apply_adam(lr_verts, lr_dens, lr_grads, lr_base, loss_type, lr_sh)
        return losses
