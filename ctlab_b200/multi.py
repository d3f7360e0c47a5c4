"""One scan across the ranks of a process group (one process per GPU).

The reference splits a scan over GPUs inside one process (`DD3Proj_multiGPU`,
`DD3Back_multiGPU`, src/DD3_GPU_Proj.h:138-141, src/DD3_GPU_Back.h; bodies not
published).  Here each rank owns a contiguous block of views:

* projection: every rank projects its views (views are independent), then the
  blocks are all-gathered so every rank holds the whole projection;
* backprojection: every rank backprojects its views into a whole volume, then
  the volumes are summed by an all-reduce (the backprojection is a sum over
  views; the in-plane mask is linear, so masked partial sums add up to the
  masked sum).

The collectives go through torch.distributed (NCCL on GPUs, gloo on CPU).  The
per-rank compute is any object with the Plan methods `proj_views` and
`back_views` (normally a `ctlab_b200.Plan` on this rank's GPU).
"""
from __future__ import annotations

import numpy as np


class ViewSplit:
    """Views [v0, v1) of `PN` belong to this rank: blocks of ceil(PN / world)."""

    def __init__(self, PN: int, world: int, rank: int):
        if world < 1 or not 0 <= rank < world:
            raise ValueError("bad world size or rank")
        self.PN, self.world, self.rank = PN, world, rank
        self.block = -(-PN // world)
        self.v0 = min(PN, rank * self.block)
        self.v1 = min(PN, self.v0 + self.block)

    @property
    def views(self) -> np.ndarray:
        return np.arange(self.v0, self.v1, dtype=np.int32)

    def owner(self, view: int) -> int:
        return view // self.block


class DistributedPlan:
    """Projects / backprojects one scan with its views split over the ranks."""

    def __init__(self, plan, PN: int, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.plan = plan
        self.split = ViewSplit(PN, dist.get_world_size(group), dist.get_rank(group))

    def proj(self, vol, out, mask=None, stream=None):
        """out [PN][DNU][DNV] (every rank) = the projection of vol."""
        import torch

        s = self.split
        per_view = out[0].numel()
        if s.PN % s.world == 0:
            full = out
        else:
            full = torch.zeros((s.world * s.block,) + tuple(out.shape[1:]), dtype=out.dtype, device=out.device)
        local = full[s.rank * s.block:(s.rank + 1) * s.block]
        if s.v1 > s.v0:
            self.plan.proj_views(s.views, vol, local[: s.v1 - s.v0], mask=mask, stream=stream)
        if s.v1 - s.v0 < s.block:
            local[s.v1 - s.v0:].zero_()
        if per_view:
            self.dist.all_gather_into_tensor(full, local.contiguous(), group=self.group)
        if full is not out:
            out.copy_(full[: s.PN])
        return out

    def back(self, prj, out, mask=None, stream=None):
        """out (every rank) = the backprojection of prj [PN][DNU][DNV]."""
        s = self.split
        if s.v1 > s.v0:
            self.plan.back_views(s.views, prj[s.v0:s.v1], out, mask=mask, stream=stream)
        else:
            out.zero_()
        self.dist.all_reduce(out, group=self.group)
        return out
