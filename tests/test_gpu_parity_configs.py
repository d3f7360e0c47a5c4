"""The CUDA path against the FP64 oracle on the benchmark scans themselves.

* Config 1 (128x128x64, 360 views, 256x64): every view, projection and
  backprojection, in the z-prefix and the FP64 SAT modes, plus the committed raw
  oracle views of tests/golden/ (pinned by SHA-256, test_oracle_fixture.py).
* Config 2 (512x512x256, 888x64 detector): 24 evenly spaced views of the 984 and
  the views on and next to the x/y-driven hand-over angles pi/4, 3pi/4, 5pi/4,
  7pi/4 (+-1e-6 rad, and the float32 rounding of each), in both modes; the error is
  checked for the whole output and for every view.
* Config 3 (256x256x128, 720 views, 384x128): one full OS-SART iteration (24
  subsets, lambda 1) and two FISTA-TV iterations (lambda 1e-4) from noisy
  projections, against orc_os_sart / orc_fista_tv (marked slow: the oracle needs
  about a minute for each on 16 host cores).

Bar: relative L2 <= 1e-4 against the FP64 oracle for the operators' FP32 outputs.  The
iterated solver states get 5e-4: every subset update forms the residual b - Ax, which
cancels to about a tenth of b within the first subsets, so the FP32 operators' 1e-6
errors grow about tenfold per update (measured on the B200: 1.0e-4 after one OS-SART
iteration of 24 subsets, 1.6e-4 after two FISTA-TV iterations).
"""
import json
import math
import os

import numpy as np
import pytest

import ctlab_b200 as cb
import oracle
from ctlab_b200 import geometry as G
from conftest import record_error

pytestmark = pytest.mark.gpu

REL_L2 = 1e-4
REL_L2_SOLVER = 5e-4
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MODES = {"zprefix": cb.CTLAB_SAT_ZPREFIX, "fp64": cb.CTLAB_SAT_FP64}


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def config1_ref():
    g = G.config1()
    hx, hy, hz = G.half_extents(g)
    vol = oracle.ellipsoid_phantom(g, G.shepp_logan_ellipsoids(hx, hy, hz))
    prj = oracle.dd3_proj(g, vol)
    prj32 = prj.astype(np.float32)
    back = oracle.dd3_back(g, prj32)
    return g, vol, prj, prj32, back


@pytest.mark.parametrize("mode", sorted(MODES))
def test_config1_all_360_views_match_oracle(torch_cuda, config1_ref, mode):
    torch = torch_cuda
    g, vol, ref_p, prj32, ref_b = config1_ref
    with cb.Plan(g, sat_mode=MODES[mode]) as plan:
        out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(torch.from_numpy(vol).cuda(), out)
        vb = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.back(torch.from_numpy(prj32).cuda(), vb)
        torch.cuda.synchronize()
        got_p, got_b = out.cpu().numpy(), vb.cpu().numpy()
    ep, eb = rel_l2(got_p, ref_p), rel_l2(got_b, ref_b)
    worst = max(rel_l2(got_p[k], ref_p[k]) for k in range(g.PN))
    record_error(f"proj/config1_360views/{mode}", ep)
    record_error(f"proj/config1_360views/{mode}/worst_view", worst)
    record_error(f"back/config1_360views/{mode}", eb)
    assert ep <= REL_L2 and eb <= REL_L2 and worst <= REL_L2, (ep, eb, worst)
    # the committed, SHA-pinned oracle views (0: y-driven, 45: theta = pi/4, x-driven)
    meta = json.load(open(os.path.join(GOLD, "config1_oracle.json")))
    pinned = np.fromfile(os.path.join(GOLD, "config1_proj_views.f64"), "<f8").reshape(-1, g.DNU, g.DNV)
    for i, k in enumerate(meta["views"]):
        e = rel_l2(got_p[k], pinned[i])
        record_error(f"proj/config1_pinned_view{k}/{mode}", e)
        assert e <= REL_L2, (k, e)


def config2_switch_geometry():
    """Config 2 with 24 evenly spaced views of the 984 plus the hand-over angles."""
    g = G.config2()
    spread = g.hangs[np.linspace(0, g.PN - 1, 24).round().astype(int)].astype(np.float64)
    extra = []
    for q in (1, 3, 5, 7):
        a = q * math.pi / 4
        extra += [a - 1e-6, float(np.float32(a)), a + 1e-6]
    angles = np.concatenate([spread, extra])
    return G.DD3Geometry.flat(sid=G.SOD, sdd=G.SDD, DNU=g.DNU, DNV=g.DNV, col_size=1.0239, row_size=1.0960,
                              PN=angles.size, XN=g.XN, YN=g.YN, ZN=g.ZN, dx=g.dx, dz=g.dz, angles=angles)


@pytest.fixture(scope="module")
def config2_ref():
    g = config2_switch_geometry()
    hx, hy, hz = G.half_extents(g)
    vol = oracle.ellipsoid_phantom(g, oracle.random_ellipsoids(1, hx, hy, hz))
    prj = oracle.dd3_proj(g, vol)
    prj32 = prj.astype(np.float32)
    back = oracle.dd3_back(g, prj32)
    return g, vol, prj, prj32, back


@pytest.mark.parametrize("mode", sorted(MODES))
def test_config2_spread_and_switch_views_match_oracle(torch_cuda, config2_ref, mode):
    torch = torch_cuda
    g, vol, ref_p, prj32, ref_b = config2_ref
    with cb.Plan(g, sat_mode=MODES[mode]) as plan:
        out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(torch.from_numpy(vol).cuda(), out)
        vb = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.back(torch.from_numpy(prj32).cuda(), vb)
        torch.cuda.synchronize()
        got_p, got_b = out.cpu().numpy(), vb.cpu().numpy()
    ep, eb = rel_l2(got_p, ref_p), rel_l2(got_b, ref_b)
    per_view = [rel_l2(got_p[k], ref_p[k]) for k in range(g.PN)]
    record_error(f"proj/config2_24spread_12switch/{mode}", ep)
    record_error(f"proj/config2_24spread_12switch/{mode}/worst_view", max(per_view))
    record_error(f"proj/config2_switch_views_only/{mode}/worst_view", max(per_view[24:]))
    record_error(f"back/config2_24spread_12switch/{mode}", eb)
    assert ep <= REL_L2 and eb <= REL_L2, (ep, eb)
    assert max(per_view) <= REL_L2, per_view


@pytest.fixture(scope="module")
def config3_scan(torch_cuda):
    """Seeded random-ellipsoid phantom, its projection by the library, Poisson noise at
    I0 = 1e5 photons per ray (numpy, seeded): b = -ln(max(counts, 1) / I0)."""
    torch = torch_cuda
    g = G.config3()
    hx, hy, hz = G.half_extents(g)
    truth = oracle.ellipsoid_phantom(g, oracle.random_ellipsoids(11, hx, hy, hz))
    with cb.Plan(g) as plan:
        clean = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(torch.from_numpy(truth).cuda(), clean)
        torch.cuda.synchronize()
        clean = clean.cpu().numpy().astype(np.float64)
    counts = np.random.default_rng(5).poisson(1e5 * np.exp(-clean))
    meas = (-np.log(np.maximum(counts, 1) / 1e5)).astype(np.float32)
    return g, truth, meas


@pytest.mark.slow
def test_config3_one_os_sart_iteration_matches_oracle(torch_cuda, config3_scan):
    torch = torch_cuda
    g, truth, meas = config3_scan
    x0 = np.zeros(g.vol_shape, np.float32)
    ref = oracle.os_sart(g, x0, meas, None, os_num=24, iter_num=1, lam=1.0)
    with cb.Plan(g) as plan:
        x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.os_sart(x, torch.from_numpy(meas).cuda(), None, os_num=24, iter_num=1, lam=1.0)
        torch.cuda.synchronize()
        got = x.cpu().numpy()
    e = rel_l2(got, ref)
    record_error("os_sart/config3_24subsets_1iteration", e)
    assert e <= REL_L2_SOLVER, e


@pytest.mark.slow
def test_config3_two_fista_tv_iterations_match_oracle(torch_cuda, config3_scan):
    torch = torch_cuda
    g, truth, meas = config3_scan
    x0 = np.zeros(g.vol_shape, np.float32)
    ref = oracle.fista_tv(g, x0, meas, None, iter_num=2, tv_lambda=1e-4, tv_eps=1e-8)
    with cb.Plan(g) as plan:
        x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.fista_tv(x, torch.from_numpy(meas).cuda(), None, iter_num=2, tv_lambda=1e-4, tv_eps=1e-8)
        torch.cuda.synchronize()
        got = x.cpu().numpy()
    e = rel_l2(got, ref)
    record_error("fista_tv/config3_2iterations", e)
    assert e <= REL_L2_SOLVER, e
