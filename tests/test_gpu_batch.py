"""Batched projection (one persistent launch over uneven scans, optionally a
CUDA-graph replay) equals the per-scan projector bit for bit, and the
autotuner's choice keeps parity with the oracle and is cached."""
import json
import os

import numpy as np
import pytest

import ctlab_b200 as cb
import oracle
from ctlab_b200 import geometry as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def uneven_scans():
    f = G.DD3Geometry.flat
    return [f(sid=541.0, sdd=949.0, DNU=96, DNV=24, col_size=1.0, row_size=1.0, PN=40, XN=40, YN=36, ZN=20,
              dx=1.0, dz=1.0),
            f(sid=541.0, sdd=949.0, DNU=70, DNV=33, col_size=1.3, row_size=0.9, PN=17, XN=24, YN=24, ZN=30,
              dx=1.5, dz=0.7),
            G.small(PN=24, zpos=np.linspace(-1, 1, 24)),
            f(sid=541.0, sdd=949.0, DNU=130, DNV=16, col_size=0.8, row_size=1.0, PN=64, XN=64, YN=48, ZN=12,
              dx=1.0, dz=1.0)]


@pytest.mark.parametrize("warps", [None, "7", "mixed"])
def test_batched_projection_equals_per_scan_projection(torch_cuda, warps, monkeypatch):
    """Every case staged for 16-warp CTAs (the default), for 8-warp CTAs (CTLAB_PROJT_WARPS=7:
    the batch runs them in 256-thread CTAs, two per SM), or both kinds in one batch."""
    torch = torch_cuda
    geoms = uneven_scans()
    plans = []
    for i, g in enumerate(geoms):
        if warps == "7" or (warps == "mixed" and i % 2):
            monkeypatch.setenv("CTLAB_PROJT_WARPS", "7")
        else:
            monkeypatch.delenv("CTLAB_PROJT_WARPS", raising=False)
        plans.append(cb.Plan(g))
    monkeypatch.delenv("CTLAB_PROJT_WARPS", raising=False)
    vols, refs = [], []
    for i, (g, p) in enumerate(zip(geoms, plans)):
        hx, hy, hz = G.half_extents(g)
        v = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        cb.ellipsoid_phantom(v, g, cb.random_ellipsoids(30 + i, hx, hy, hz, 6, 10))
        vols.append(v)
        r = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        p.proj(v, r)
        refs.append(r)
    batch = cb.Batch(plans)
    assert batch.voxel_views == sum(g.voxel_views for g in geoms)
    stream = torch.cuda.Stream()
    for graph in (False, True, True):  # the second graph run replays
        outs = [torch.full(g.prj_shape, float("nan"), dtype=torch.float32, device="cuda") for g in geoms]
        with torch.cuda.stream(stream):
            batch.proj(vols, outs, graph=graph, stream=stream.cuda_stream)
        stream.synchronize()
        for o, r in zip(outs, refs):
            assert torch.equal(o, r)
    batch.close()
    for p in plans:
        p.close()


def test_autotuned_staging_keeps_parity_and_is_cached(torch_cuda, tmp_path):
    torch = torch_cuda
    g = uneven_scans()[0]
    hx, hy, hz = G.half_extents(g)
    vol = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
    cb.ellipsoid_phantom(vol, g, cb.random_ellipsoids(3, hx, hy, hz, 6, 10))
    ref = oracle.dd3_proj(g, vol.cpu().numpy())
    cache = str(tmp_path / "tiles.jsonl")
    out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
    with cb.Plan(g) as plan:
        ms = plan.autotune(vol, out, cache)
        assert ms > 0
        plan.proj(vol, out)
        torch.cuda.synchronize()
        err = float(np.linalg.norm(out.cpu().numpy() - ref) / np.linalg.norm(ref))
        assert err <= 1e-4
    rec = [json.loads(l) for l in open(cache)]
    assert len(rec) == 1 and rec[0]["gcap"] in (2, 4, 8, 16) and rec[0]["nstage"] in (2, 3, 4)
    with cb.Plan(g) as plan:
        assert plan.autotune(vol, out, cache) == -1.0  # from the cache
        plan.proj(vol, out)
        torch.cuda.synchronize()
        assert float(np.linalg.norm(out.cpu().numpy() - ref) / np.linalg.norm(ref)) <= 1e-4
    assert len(open(cache).readlines()) == 1
