"""Host logic of the multi-rank split (ctlab_b200.multi) on CPU with gloo ranks:
projection split by views (all-gather of the view blocks), backprojection split
by z slabs (each slab from the views that reach it, all-gather of the padded
slabs).  The per-rank compute is stood in for by the FP64 oracle on each rank's
sub-scan.  The gathered projection must equal the one-process projection view
for view; the gathered backprojection must equal the one-process backprojection
(the slab's own centre is rounded to float32, hence a 1e-5 bar), with uneven
and empty slabs and a helical scan whose slabs see only part of the views."""
import dataclasses
import os
import socket

import numpy as np
import pytest

from ctlab_b200.multi import SlabSplit, ViewSplit


@pytest.mark.parametrize("PN,world", [(13, 2), (13, 4), (8, 2), (3, 4), (1, 2)])
def test_view_split_covers_every_view_once(PN, world):
    owned = []
    for r in range(world):
        s = ViewSplit(PN, world, r)
        assert 0 <= s.v0 <= s.v1 <= PN and s.v1 - s.v0 <= s.block
        owned += list(s.views)
        assert all(s.owner(v) == r for v in s.views)
    assert owned == list(range(PN))


@pytest.mark.parametrize("ZN,world,starts", [(12, 2, None), (12, 2, [0, 5]), (12, 3, [0, 2, 9]), (12, 3, [0, 0, 7]),
                                             (5, 4, None)])
def test_slab_split_covers_every_slice_once(ZN, world, starts):
    owned = []
    for r in range(world):
        s = SlabSplit(ZN, world, r, starts)
        assert 0 <= s.z0 <= s.z1 <= ZN and s.z1 - s.z0 <= s.slab
        owned += list(range(s.z0, s.z1))
    assert owned == list(range(ZN))


@pytest.mark.parametrize("starts", [[1, 5], [0, 13], [0, 7, 3]])
def test_split_rejects_bad_starts(starts):
    with pytest.raises(ValueError):
        SlabSplit(12, len(starts), 0, starts)


class OracleScan:
    """Stand-in for a Plan on CPU: the oracle on a (sub-)scan."""

    def __init__(self, g):
        self.g = g

    def proj_views(self, views, vol, out, mask=None, stream=None):
        import oracle
        import torch
        sub = dataclasses.replace(self.g, hangs=self.g.hangs[views], hzPos=self.g.hzPos[views])
        out.copy_(torch.from_numpy(oracle.dd3_proj(sub, vol.numpy(), mask)))
        return out

    def back(self, prj, out, mask=None, stream=None):
        import oracle
        import torch
        out.copy_(torch.from_numpy(oracle.dd3_back(self.g, prj.numpy(), mask)))
        return out


SCANS = {
    "circular": dict(PN=13),
    # a long helical volume: each slab is reached by only part of the views
    "helical": dict(PN=30, ZN=300, dz=0.1, zpos=np.linspace(-14.0, 14.0, 30)),
}


def _scan(name):
    import oracle
    from ctlab_b200 import geometry as G
    g = G.small(**SCANS[name])
    hx, hy, hz = G.half_extents(g)
    vol = oracle.ellipsoid_phantom(g, oracle.random_ellipsoids(3, hx, hy, hz, 4, 6))
    return g, vol


def _rank(rank, world, port, name, view_starts, slab_starts):
    import torch
    import torch.distributed as dist

    import oracle
    from ctlab_b200.multi import DistributedPlan

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, vol = _scan(name)
        mask = (np.arange(g.XN * g.YN) % 7 != 0).astype(np.uint8)
        dp = DistributedPlan(g, OracleScan, view_starts=view_starts, slab_starts=slab_starts)
        if name == "helical" and dp.slabs.z1 > dp.slabs.z0:
            assert dp.slab_view_idx.size < g.PN, "a helical slab should not need every view"
        prj = torch.zeros(g.prj_shape, dtype=torch.float32)
        dp.proj(torch.from_numpy(vol), prj, mask=mask)
        ref = oracle.dd3_proj(g, vol, mask)
        assert np.array_equal(prj.numpy(), ref.astype(np.float32)), "gathered projection differs"
        back = torch.zeros(g.vol_shape, dtype=torch.float32)
        dp.back(prj, back, mask=mask)
        refb = oracle.dd3_back(g, prj.numpy(), mask)
        err = np.linalg.norm(back.numpy() - refb) / np.linalg.norm(refb)
        assert err < 1e-5, f"gathered slab backprojection rel L2 {err}"
        # every slab on its own, too
        for a, b in dp.slabs.blocks:
            if b > a:
                e = np.linalg.norm(back.numpy()[:, :, a:b] - refb[:, :, a:b]) / max(np.linalg.norm(refb[:, :, a:b]),
                                                                                   1e-30)
                assert e < 1e-5, (a, b, e)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("name,world,view_starts,slab_starts", [
    ("circular", 2, None, None),          # padded view blocks (13 = 7 + 6), even slabs
    ("circular", 3, [0, 2, 9], [0, 5, 6]),  # uneven views and slabs
    ("circular", 3, None, [0, 0, 7]),     # an empty slab
    ("helical", 2, None, [0, 110]),
    ("helical", 3, [0, 10, 20], [0, 80, 200]),
])
def test_distributed_split_matches_one_process(name, world, view_starts, slab_starts):
    import torch.multiprocessing as mp
    mp.spawn(_rank, args=(world, _free_port(), name, view_starts, slab_starts), nprocs=world, join=True)


def test_slab_views_on_the_host():
    """ctlab_slab_views (host only, no GPU): a circular scan's slabs need every view; a
    helical scan's slabs need a contiguous run that moves with the slab; an empty slab
    needs none; a slab outside the volume is an error."""
    import ctlab_b200 as cb
    from ctlab_b200 import geometry as G
    g = G.small(PN=16)
    assert cb.slab_views(g, 0, 5).tolist() == list(range(16))
    h = G.helical(XN=64, YN=64, ZN=256, dz=0.5, views_per_turn=64)
    runs = [cb.slab_views(h, z0, z0 + 32) for z0 in range(0, 256, 32)]
    for a, b in zip(runs, runs[1:]):
        assert np.all(np.diff(a) == 1) and 0 < a.size < h.PN
        assert b[0] >= a[0] and b[-1] >= a[-1]
    assert cb.slab_views(h, 7, 7).size == 0
    with pytest.raises(cb.CtlabError):
        cb.slab_views(h, 0, 257)
