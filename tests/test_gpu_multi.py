"""Multi-GPU splits on the GPU.

* ctlab_b200.multi.DistributedPlan with NCCL: a one-rank process group (this
  pool's calls have one GPU) must reproduce Plan.proj / Plan.back, also when the
  caller passes a side stream (the collectives must follow the rank's kernels on
  that stream).  The multi-rank host logic is covered by the gloo tests.
* DD3Proj_multiGPU / DD3Back_multiGPU (the reference's signatures): with one GPU,
  and with a three-part uneven split wrapped onto the one device
  (CTLAB_MULTIGPU_WRAP=1), against DD3Proj_gpu / DD3Back_gpu; on a helical scan
  the slabs see only part of the views and must still equal the whole
  backprojection.
"""
import os
import socket

import numpy as np
import pytest

import ctlab_b200 as cb
from ctlab_b200 import geometry as G

pytestmark = pytest.mark.gpu


def _rank(rank, world, port, out_path, side_stream):
    import torch
    import torch.distributed as dist

    from ctlab_b200.multi import DistributedPlan

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(rank)
    dist.init_process_group("nccl", rank=rank, world_size=world, device_id=torch.device("cuda", rank))
    try:
        g = G.small(PN=13, ZN=40, dz=0.2)
        hx, hy, hz = G.half_extents(g)
        vol = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        cb.ellipsoid_phantom(vol, g, cb.random_ellipsoids(3, hx, hy, hz, 4, 6))
        with cb.Plan(g) as plan:
            ref_p = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
            plan.proj(vol, ref_p)
            ref_b = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
            plan.back(ref_p, ref_b)
            torch.cuda.synchronize()
        dp = DistributedPlan(g, lambda geom: cb.Plan(geom, device=rank))
        s = torch.cuda.Stream() if side_stream else None
        h = None if s is None else s.cuda_stream
        p = torch.full_like(ref_p, float("nan"))
        b = torch.full_like(ref_b, float("nan"))
        torch.cuda.synchronize()
        dp.proj(vol, p, stream=h)
        dp.back(p, b, stream=h)
        if s is not None:
            s.synchronize()
        torch.cuda.synchronize()
        ep = float(torch.linalg.norm(p - ref_p) / torch.linalg.norm(ref_p))
        eb = float(torch.linalg.norm(b - ref_b) / torch.linalg.norm(ref_b))
        dp.close()
        with open(out_path, "w") as f:
            f.write("ok" if (ep <= 1e-6 and eb <= 1e-5) else f"mismatch proj {ep} back {eb}")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("side_stream", [False, True])
def test_distributed_split_one_rank_nccl_equals_plan(tmp_path, side_stream):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "result.txt")
    mp.spawn(_rank, args=(1, port, out, side_stream), nprocs=1, join=True)
    assert open(out).read() == "ok"


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


SCANS = {
    "circular": dict(PN=20, ZN=30, dz=0.3),
    "helical": dict(PN=40, ZN=400, dz=0.08, zpos=np.linspace(-14.0, 14.0, 40)),
}


@pytest.mark.parametrize("name", sorted(SCANS))
@pytest.mark.parametrize("parts", [1, 3])
def test_multigpu_entry_points_equal_single_gpu(name, parts, monkeypatch):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if parts > torch.cuda.device_count():
        monkeypatch.setenv("CTLAB_MULTIGPU_WRAP", "1")
    g = G.small(**SCANS[name])
    hx, hy, hz = G.half_extents(g)
    import oracle
    vol = oracle.ellipsoid_phantom(g, oracle.random_ellipsoids(5, hx, hy, hz, 5, 8))
    mask = (np.arange(g.XN * g.YN) % 5 != 0).astype(np.uint8)
    ref_p = np.zeros(g.prj_shape, np.float32)
    cb.DD3Proj_gpu(**g.args(), hvol=vol, hprj=ref_p, mask=mask, gpunum=0, prjMode=0)
    ref_b = np.zeros(g.vol_shape, np.float32)
    cb.DD3Back_gpu(**g.args(), hvol=ref_b, hprj=ref_p, mask=mask, gpunum=0, squared=0, prjMode=0)
    start_pn = [0, 3, 11][:parts]
    start_vol = [0, g.ZN // 5, g.ZN // 2][:parts]
    p = np.full(g.prj_shape, np.nan, np.float32)
    cb.DD3Proj_multiGPU(**g.args(), hvol=vol, hprj=p, mask=mask, prjMode=0, startPN=start_pn, gpuNum=parts)
    b = np.full(g.vol_shape, np.nan, np.float32)
    cb.DD3Back_multiGPU(**g.args(), hvol=b, hprj=ref_p, mask=mask, methodId=0, startVOL=start_vol, gpuNum=parts)
    assert np.all(np.isfinite(p)) and np.all(np.isfinite(b)), "a part was not written"
    assert _rel(p, ref_p) <= 1e-6, _rel(p, ref_p)
    assert _rel(b, ref_b) <= 1e-5, _rel(b, ref_b)
    if name == "helical" and parts == 3:
        # the slabs see only the views that reach them
        for z0, z1 in zip(start_vol, start_vol[1:] + [g.ZN]):
            assert 0 < cb.slab_views(g, z0, z1).size < g.PN


def test_multigpu_entry_points_reject_bad_splits():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    g = G.small()
    vol = np.zeros(g.vol_shape, np.float32)
    prj = np.zeros(g.prj_shape, np.float32)
    with pytest.raises(cb.CtlabError) as e:
        cb.DD3Proj_multiGPU(**g.args(), hvol=vol, hprj=prj, mask=None, prjMode=0, startPN=[2], gpuNum=1)
    assert e.value.code == cb.CTLAB_ERR_INVALID_ARG and "startPN" in e.value.message
    with pytest.raises(cb.CtlabError) as e:
        cb.DD3Back_multiGPU(**g.args(), hvol=vol, hprj=prj, mask=None, methodId=0, startVOL=[0], gpuNum=65)
    assert e.value.code == cb.CTLAB_ERR_INVALID_ARG
    with pytest.raises(cb.CtlabError) as e:
        cb.DD3Back_multiGPU(**g.args(), hvol=vol, hprj=prj, mask=None, methodId=2, startVOL=[0], gpuNum=1)
    assert e.value.code == cb.CTLAB_ERR_UNSUPPORTED
