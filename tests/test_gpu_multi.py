"""The view split (ctlab_b200.multi.DistributedPlan) on the GPU with NCCL: a one-rank
process group (this pool's calls have one GPU) must reproduce Plan.proj / Plan.back
(the multi-rank host logic is covered by the gloo tests)."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rank(rank, world, port, out_path):
    import torch
    import torch.distributed as dist

    import ctlab_b200 as cb
    from ctlab_b200 import geometry as G
    from ctlab_b200.multi import DistributedPlan

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(rank)
    dist.init_process_group("nccl", rank=rank, world_size=world, device_id=torch.device("cuda", rank))
    try:
        g = G.small(PN=13)
        hx, hy, hz = G.half_extents(g)
        vol = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        cb.ellipsoid_phantom(vol, g, cb.random_ellipsoids(3, hx, hy, hz, 4, 6))
        with cb.Plan(g) as plan:
            ref_p = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
            plan.proj(vol, ref_p)
            ref_b = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
            plan.back(ref_p, ref_b)
            dp = DistributedPlan(plan, g.PN)
            p = torch.zeros_like(ref_p)
            dp.proj(vol, p)
            b = torch.zeros_like(ref_b)
            dp.back(p, b)
            torch.cuda.synchronize()
            ok = bool(torch.equal(p, ref_p)) and float(torch.linalg.norm(b - ref_b) / torch.linalg.norm(ref_b)) < 1e-6
        with open(out_path, "w") as f:
            f.write("ok" if ok else "mismatch")
    finally:
        dist.destroy_process_group()


def test_view_split_one_rank_nccl_equals_plan(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "result.txt")
    mp.spawn(_rank, args=(1, port, out), nprocs=1, join=True)
    assert open(out).read() == "ok"
