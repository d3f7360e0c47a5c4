"""One scan across the ranks of a process group (one process per GPU).

The reference splits a scan over GPUs: views for projection (`startPN`,
`DD3Proj_multiGPU`, src/DD3_GPU_Proj.h:138-141) and z slabs of the volume for
backprojection (`startVOL`, `DD3Back_multiGPU`, src/DD3_GPU_Back.h:138-142),
each slab seeing only the views whose rays reach it (`getPrjIdxPair`,
src/utilities.cuh:503-532) and the slabs put back together by
`combineVolume` (:538-589).  Here, with one process per GPU:

* projection: rank r projects its block of views of the whole (replicated)
  volume, then the blocks are all-gathered so every rank holds the whole
  projection;
* backprojection: rank r backprojects its z slab from the views that reach it
  (`slab_views`) into a volume of the slab's slices only, then the slabs are
  all-gathered (padded to the largest slab) and written into every rank's
  volume.  Slabs are disjoint, so nothing is summed across ranks and the result
  does not depend on the number of ranks' summation order.

The collectives go through torch.distributed (NCCL on GPUs, gloo on CPU) and,
when a CUDA stream is given, run on that stream after the rank's kernels.  The
per-rank compute comes from `make_plan(geometry)`: an object with the Plan
methods `proj_views(views, vol, out, mask, stream)` and `back(prj, out, mask,
stream)` (normally `lambda g: ctlab_b200.Plan(g, device=rank's GPU)`).
"""
from __future__ import annotations

import contextlib

import numpy as np


def _blocks(total: int, world: int, starts=None) -> list[tuple[int, int]]:
    """[lo, hi) per rank: the caller's start indices (one per rank, starting at 0,
    never decreasing, the last block ending at `total`) or even blocks."""
    if starts is None:
        b = -(-total // world) if world else 0
        return [(min(total, r * b), min(total, (r + 1) * b)) for r in range(world)]
    s = [int(v) for v in starts]
    if len(s) != world or s[0] != 0 or any(b < a for a, b in zip(s, s[1:])) or s[-1] > total:
        raise ValueError("starts must hold one index per rank, start at 0, never decrease and stay within the scan")
    return list(zip(s, s[1:] + [total]))


class ViewSplit:
    """Views [v0, v1) of `PN` belong to this rank (the reference's startPN, or
    blocks of ceil(PN / world))."""

    def __init__(self, PN: int, world: int, rank: int, starts=None):
        if world < 1 or not 0 <= rank < world:
            raise ValueError("bad world size or rank")
        self.PN, self.world, self.rank = PN, world, rank
        self.blocks = _blocks(PN, world, starts)
        self.v0, self.v1 = self.blocks[rank]
        self.block = max(b - a for a, b in self.blocks)

    @property
    def views(self) -> np.ndarray:
        return np.arange(self.v0, self.v1, dtype=np.int32)

    def owner(self, view: int) -> int:
        for r, (a, b) in enumerate(self.blocks):
            if a <= view < b:
                return r
        raise ValueError("view outside the scan")


class SlabSplit:
    """Slices [z0, z1) of `ZN` belong to this rank (the reference's startVOL, or
    blocks of ceil(ZN / world))."""

    def __init__(self, ZN: int, world: int, rank: int, starts=None):
        if world < 1 or not 0 <= rank < world:
            raise ValueError("bad world size or rank")
        self.ZN, self.world, self.rank = ZN, world, rank
        self.blocks = _blocks(ZN, world, starts)
        self.z0, self.z1 = self.blocks[rank]
        self.slab = max(b - a for a, b in self.blocks)


class DistributedPlan:
    """Projects (split by views) and backprojects (split by z slabs) one scan."""

    def __init__(self, g, make_plan, group=None, view_starts=None, slab_starts=None):
        import torch.distributed as dist

        from .dd3 import slab_geometry, slab_views

        self.dist = dist
        self.group = group
        self.g = g
        world, rank = dist.get_world_size(group), dist.get_rank(group)
        self.views = ViewSplit(g.PN, world, rank, view_starts)
        self.slabs = SlabSplit(g.ZN, world, rank, slab_starts)
        self.proj_plan = make_plan(g) if self.views.v1 > self.views.v0 else None
        z0, z1 = self.slabs.z0, self.slabs.z1
        self.slab_view_idx = slab_views(g, z0, z1) if z1 > z0 else np.zeros(0, np.int32)
        self.back_plan = None
        if self.slab_view_idx.size:
            self.back_plan = make_plan(slab_geometry(g, z0, z1, self.slab_view_idx))
        idx = self.slab_view_idx
        self._view_run = (int(idx[0]), int(idx[-1]) + 1) if idx.size and np.all(np.diff(idx) == 1) else None

    def close(self):
        for p in (self.proj_plan, self.back_plan):
            if p is not None and hasattr(p, "close"):
                p.close()

    @staticmethod
    def _on(stream, t):
        """Runs the torch ops and collectives that follow on the caller's stream."""
        if stream is None or not t.is_cuda:
            return contextlib.nullcontext()
        import torch
        return torch.cuda.stream(torch.cuda.ExternalStream(int(stream), device=t.device))

    def proj(self, vol, out, mask=None, stream=None):
        """out [PN][DNU][DNV] (every rank) = the projection of vol."""
        import torch

        s = self.views
        n = s.v1 - s.v0
        rest = tuple(out.shape[1:])
        with self._on(stream, out):
            local = torch.zeros((s.block,) + rest, dtype=out.dtype, device=out.device)
            if n:
                self.proj_plan.proj_views(s.views, vol, local[:n], mask=mask, stream=stream)
            full = torch.empty((s.world * s.block,) + rest, dtype=out.dtype, device=out.device)
            if out[0].numel():
                self.dist.all_gather_into_tensor(full, local, group=self.group)
            for r, (a, b) in enumerate(s.blocks):
                if b > a:
                    out[a:b].copy_(full[r * s.block:r * s.block + (b - a)])
        return out

    def back(self, prj, out, mask=None, stream=None):
        """out (every rank) = the backprojection of prj [PN][DNU][DNV]."""
        import torch

        g, s = self.g, self.slabs
        cols = g.YN * g.XN
        szn = s.z1 - s.z0
        with self._on(stream, out):
            local = torch.zeros((cols, s.slab), dtype=out.dtype, device=out.device)
            if self.back_plan is not None:
                if self._view_run is not None:
                    sub_prj = prj[self._view_run[0]:self._view_run[1]]
                else:
                    sel = torch.from_numpy(self.slab_view_idx.astype(np.int64)).to(prj.device)
                    sub_prj = prj.index_select(0, sel)
                sub = torch.empty((g.YN, g.XN, szn), dtype=out.dtype, device=out.device)
                self.back_plan.back(sub_prj.contiguous(), sub, mask=mask, stream=stream)
                local[:, :szn].copy_(sub.view(cols, szn))
            full = torch.empty((s.world * cols, s.slab), dtype=out.dtype, device=out.device)
            self.dist.all_gather_into_tensor(full, local, group=self.group)
            full = full.view(s.world, cols, s.slab)
            ov = out.view(cols, g.ZN)
            for r, (a, b) in enumerate(s.blocks):
                if b > a:
                    ov[:, a:b].copy_(full[r, :, : b - a])
        return out
