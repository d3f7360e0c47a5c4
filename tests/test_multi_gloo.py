"""Host logic of the view split over ranks (ctlab_b200.multi) on CPU: two gloo
ranks, an odd number of views (uneven blocks, one padded), the per-rank compute
stood in for by the FP64 oracle on each rank's views.  The gathered projection
must equal the one-process projection view for view, and the all-reduced
backprojection the one-process backprojection to summation order."""
import dataclasses
import os
import socket

import numpy as np
import pytest

from ctlab_b200.multi import ViewSplit


@pytest.mark.parametrize("PN,world", [(13, 2), (13, 4), (8, 2), (3, 4), (1, 2)])
def test_view_split_covers_every_view_once(PN, world):
    owned = []
    for r in range(world):
        s = ViewSplit(PN, world, r)
        assert 0 <= s.v0 <= s.v1 <= PN and s.v1 - s.v0 <= s.block
        owned += list(s.views)
        assert all(s.owner(v) == r for v in s.views)
    assert owned == list(range(PN))


class OracleViews:
    """Stand-in for a Plan on CPU: the oracle applied to a subset of views."""

    def __init__(self, g):
        self.g = g

    def _sub(self, views):
        return dataclasses.replace(self.g, hangs=self.g.hangs[views], hzPos=self.g.hzPos[views])

    def proj_views(self, views, vol, out, mask=None, stream=None):
        import oracle
        import torch
        out.copy_(torch.from_numpy(oracle.dd3_proj(self._sub(views), vol.numpy(), mask)))
        return out

    def back_views(self, views, prj, out, mask=None, stream=None):
        import oracle
        import torch
        out.copy_(torch.from_numpy(oracle.dd3_back(self._sub(views), prj.numpy(), mask)))
        return out


def _scan(PN):
    import oracle
    from ctlab_b200 import geometry as G
    import ctlab_b200 as cb
    g = G.small(PN=PN)
    hx, hy, hz = G.half_extents(g)
    vol = oracle.ellipsoid_phantom(g, cb.random_ellipsoids(3, hx, hy, hz, 4, 6))
    return g, vol


def _rank(rank, world, port, PN):
    import torch
    import torch.distributed as dist

    import oracle
    from ctlab_b200.multi import DistributedPlan

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, vol = _scan(PN)
        mask = (np.arange(g.XN * g.YN) % 7 != 0).astype(np.uint8)
        dp = DistributedPlan(OracleViews(g), g.PN)
        prj = torch.zeros(g.prj_shape, dtype=torch.float32)
        dp.proj(torch.from_numpy(vol), prj, mask=mask)
        ref = oracle.dd3_proj(g, vol, mask)
        assert np.array_equal(prj.numpy(), ref.astype(np.float32)), "gathered projection differs"
        back = torch.zeros(g.vol_shape, dtype=torch.float32)
        dp.back(prj, back, mask=mask)
        refb = oracle.dd3_back(g, prj.numpy(), mask)
        err = np.linalg.norm(back.numpy() - refb) / np.linalg.norm(refb)
        assert err < 1e-6, f"reduced backprojection rel L2 {err}"
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,PN", [(2, 13), (3, 13), (2, 12)])  # padded and direct gathers
def test_distributed_view_split_matches_one_process(world, PN):
    import torch.multiprocessing as mp
    mp.spawn(_rank, args=(world, _free_port(), PN), nprocs=world, join=True)
