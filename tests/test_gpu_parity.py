"""CUDA path (through the C ABI) against the FP64 CPU oracle.

Bar: relative L2 <= 1e-4 for projection and backprojection (the parity bar for
FP32 outputs against an FP64 oracle); FP64 SATs to 1e-12
relative.  Sizes are chosen so the oracle finishes in seconds.
"""
import math

import numpy as np
import pytest

import ctlab_b200 as cb
import oracle
from ctlab_b200 import geometry as G
from conftest import record_error

pytestmark = pytest.mark.gpu

REL_L2 = 1e-4


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def phantom(g, seed=0):
    hx, hy, hz = G.half_extents(g)
    rng = np.random.default_rng(seed)
    ell = cb.random_ellipsoids(seed + 1, hx, hy, hz, 6, 10)
    vol = oracle.ellipsoid_phantom(g, ell)
    vol += 0.002 * rng.random(g.vol_shape).astype(np.float32)  # texture everywhere
    return vol


CASES = {
    "small": dict(),
    "odd_offsets": dict(XN=23, YN=19, ZN=13, DNU=37, DNV=11, col_offset=0.37, row_offset=-0.21,
                        center=(1.3, -0.7, 0.4), start=0.05),
    "helical_shift": dict(PN=20, zpos=np.linspace(-1.5, 1.5, 20)),
    # a long helical volume: each view's cone meets only part of the z range,
    # so backprojector CTAs skip the views that miss their z slab
    "helical_long": dict(PN=40, ZN=600, dz=0.05, zpos=np.linspace(-14.0, 14.0, 40)),
    "wide_z": dict(XN=9, YN=8, ZN=300, DNU=20, DNV=40, dz=0.05, row_size=0.1),
    "single_row": dict(DNV=1, row_size=0.5),
    "coarse_det": dict(DNU=9, DNV=5, col_size=4.0, row_size=3.0),
}


def make_case(name):
    kw = dict(CASES[name])
    return G.small(**kw)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("sat_mode", [cb.CTLAB_SAT_FP64, cb.CTLAB_SAT_F32PAIR, cb.CTLAB_SAT_ZPREFIX])
def test_projection_matches_oracle(torch_cuda, name, sat_mode):
    torch = torch_cuda
    g = make_case(name)
    vol = phantom(g)
    rng = np.random.default_rng(7)
    mask = (rng.random(g.XN * g.YN) > 0.1).astype(np.uint8)
    ref = oracle.dd3_proj(g, vol, mask)
    with cb.Plan(g, sat_mode=sat_mode) as plan:
        out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(dev(torch, vol), out, mask=dev(torch, mask))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
    err = rel_l2(got, ref)
    record_error(f"proj/{name}/sat{sat_mode}", err)
    assert err <= REL_L2, f"{name}: rel L2 {err:.3e}"


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("sat_mode", [cb.CTLAB_SAT_FP64, cb.CTLAB_SAT_F32PAIR, cb.CTLAB_SAT_ZPREFIX])
def test_backprojection_matches_oracle(torch_cuda, name, sat_mode):
    torch = torch_cuda
    g = make_case(name)
    rng = np.random.default_rng(11)
    prj = oracle.dd3_proj(g, phantom(g)).astype(np.float32) + 0.01 * rng.random(g.prj_shape).astype(np.float32)
    mask = (rng.random(g.XN * g.YN) > 0.1).astype(np.uint8)
    ref = oracle.dd3_back(g, prj, mask)
    with cb.Plan(g, sat_mode=sat_mode) as plan:
        out = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.back(dev(torch, prj), out, mask=dev(torch, mask))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
    err = rel_l2(got, ref)
    record_error(f"back/{name}/sat{sat_mode}", err)
    assert err <= REL_L2, f"{name}: rel L2 {err:.3e}"


@pytest.mark.parametrize("name", ["small", "coarse_det", "odd_offsets"])
@pytest.mark.parametrize("env", [{"CTLAB_PROJT_CBMAX": "8"}, {"CTLAB_PROJT_GMAX": "1", "CTLAB_PROJT_NSTAGE": "2"},
                                 {"CTLAB_PROJT_GMAX": "2", "CTLAB_PROJT_NSTAGE": "4"}])
def test_zprefix_projector_staging_variants_match_oracle(torch_cuda, name, env, monkeypatch):
    """Stage capacities that force the global-memory fallback (8 staged columns)
    and other view-group sizes / stage depths of the z-prefix projector."""
    torch = torch_cuda
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    g = make_case(name)
    vol = phantom(g)
    ref = oracle.dd3_proj(g, vol)
    with cb.Plan(g, sat_mode=cb.CTLAB_SAT_ZPREFIX) as plan:
        out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(dev(torch, vol), out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
    err = rel_l2(got, ref)
    record_error(f"proj/{name}/zprefix/{'_'.join(env.values())}", err)
    assert err <= REL_L2, f"{name} {env}: rel L2 {err:.3e}"


def test_volume_sat_matches_oracle(torch_cuda):
    torch = torch_cuda
    g = G.small(PN=8, XN=70, YN=45, ZN=33, start=0.0)  # both orientations present
    vol = phantom(g)
    mask = (np.random.default_rng(2).random(g.XN * g.YN) > 0.2).astype(np.uint8)
    saty, satx = oracle.volume_sats(g, vol, mask)
    for mode, tol in ((cb.CTLAB_SAT_FP64, 1e-12), (cb.CTLAB_SAT_F32PAIR, 1e-9)):
        with cb.Plan(g, sat_mode=mode) as plan:
            plan.volume_sat(dev(torch, vol), dev(torch, mask))
            for o, ref in ((0, saty), (1, satx)):
                planes, rows, zp = plan.sat_layout(o)
                buf = torch.zeros(planes * rows * zp, dtype=torch.float64, device="cuda")
                plan.copy_volume_sat(o, buf)
                torch.cuda.synchronize()
                raw = buf.cpu().numpy()
                if mode == cb.CTLAB_SAT_FP64:
                    s = raw.reshape(planes, rows, zp)
                else:
                    f = raw.view(np.float32).reshape(planes, rows, zp, 2).astype(np.float64)
                    s = f[..., 0] + f[..., 1]
                s = s[:, :, : g.ZN + 1]
                assert s.shape == ref.shape
                np.testing.assert_allclose(s, ref, rtol=tol, atol=tol * np.abs(ref).max())
    # slice-major column z-prefixes (ZPREFIX plans): FP64 sums rounded to FP32,
    # [y][k][x] for y slices and [x][k][y] for x slices
    masked = vol.astype(np.float64) * mask.reshape(g.YN, g.XN, 1)
    zref = np.concatenate([np.zeros((g.YN, g.XN, 1)), np.cumsum(masked, axis=2)], axis=2)  # [y][x][k]
    with cb.Plan(g, sat_mode=cb.CTLAB_SAT_ZPREFIX) as plan:
        plan.volume_sat(dev(torch, vol), dev(torch, mask))
        for o, ref in ((0, zref.transpose(0, 2, 1)), (1, zref.transpose(1, 2, 0))):
            planes, rows, rs = plan.sat_layout(o)
            assert (planes, rows) == ref.shape[:2] and rs >= ref.shape[2] and rs % 4 == 0
            buf = torch.full((planes * rows * rs,), 7.0, dtype=torch.float32, device="cuda")
            plan.copy_volume_sat(o, buf)
            torch.cuda.synchronize()
            zs = buf.cpu().numpy().reshape(planes, rows, rs)
            np.testing.assert_allclose(zs[:, :, : ref.shape[2]], ref, rtol=1e-6, atol=1e-7 * np.abs(ref).max())
            assert not zs[:, :, ref.shape[2]:].any()  # pad columns are zero


def test_config1_views_match_oracle(torch_cuda):
    torch = torch_cuda
    g = G.config1()
    hx, hy, hz = G.half_extents(g)
    vol = oracle.ellipsoid_phantom(g, G.shepp_logan_ellipsoids(hx, hy, hz))
    views = np.arange(0, g.PN, 10)
    gs = g.with_views(views)
    ref_p = oracle.dd3_proj(gs, vol)
    with cb.Plan(g) as plan:
        out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(dev(torch, vol), out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()[views]
        record_error("proj/config1_36views", rel_l2(got, ref_p))
        assert rel_l2(got, ref_p) <= REL_L2
        prj = got.astype(np.float32)
        ref_b = oracle.dd3_back(gs, prj)
        vb = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.back_views(views, dev(torch, prj), vb)
        torch.cuda.synchronize()
        record_error("back/config1_36views", rel_l2(vb.cpu().numpy(), ref_b))
        assert rel_l2(vb.cpu().numpy(), ref_b) <= REL_L2


@pytest.mark.parametrize("sat_mode", [cb.CTLAB_SAT_FP64, cb.CTLAB_SAT_ZPREFIX])
def test_config2_views_match_oracle(torch_cuda, sat_mode):
    torch = torch_cuda
    g = G.config2()
    hx, hy, hz = G.half_extents(g)
    ell = cb.random_ellipsoids(1, hx, hy, hz)
    vol = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
    cb.ellipsoid_phantom(vol, g, ell)
    torch.cuda.synchronize()
    views = np.array([0, 101, 246, 500])  # y- and x-driven views
    gs = g.with_views(views)
    vol_h = vol.cpu().numpy()
    ref_p = oracle.dd3_proj(gs, vol_h)
    with cb.Plan(g, sat_mode=sat_mode) as plan:
        out = torch.zeros((len(views), g.DNU, g.DNV), dtype=torch.float32, device="cuda")
        plan.proj_views(views, vol, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        record_error(f"proj/config2_4views/sat{sat_mode}", rel_l2(got, ref_p))
        assert rel_l2(got, ref_p) <= REL_L2
        ref_b = oracle.dd3_back(gs, got)
        vb = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.back_views(views, out, vb)
        torch.cuda.synchronize()
        record_error(f"back/config2_4views/sat{sat_mode}", rel_l2(vb.cpu().numpy(), ref_b))
        assert rel_l2(vb.cpu().numpy(), ref_b) <= REL_L2


def test_gpu_phantom_matches_oracle_phantom(torch_cuda):
    torch = torch_cuda
    g = G.config1()
    hx, hy, hz = G.half_extents(g)
    ell = G.shepp_logan_ellipsoids(hx, hy, hz)
    ref = oracle.ellipsoid_phantom(g, ell)
    vol = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
    cb.ellipsoid_phantom(vol, g, ell)
    got = vol.cpu().numpy()
    bad = np.abs(got - ref) > 1e-6
    assert bad.mean() < 1e-4  # float vs double inside-tests on the surfaces only


@pytest.mark.parametrize("sat_mode", [cb.CTLAB_SAT_ZPREFIX, cb.CTLAB_SAT_FP64])
def test_legacy_host_entry_points_equal_plan_path(torch_cuda, sat_mode, monkeypatch):
    """DD3Proj_gpu / DD3Back_gpu (host pointers) equal the device plan path bit for
    bit; CTLAB_LEGACY_SAT selects the legacy calls' SAT arithmetic."""
    torch = torch_cuda
    monkeypatch.setenv("CTLAB_LEGACY_SAT", str(sat_mode))
    g = make_case("odd_offsets")
    vol = phantom(g)
    mask = (np.random.default_rng(4).random(g.XN * g.YN) > 0.3).astype(np.uint8)
    hp = np.zeros(g.prj_shape, np.float32)
    cb.DD3Proj_gpu(**g.args(), hvol=vol, hprj=hp, mask=mask, gpunum=0, prjMode=0)
    hb = np.zeros(g.vol_shape, np.float32)
    cb.DD3Back_gpu(**g.args(), hvol=hb, hprj=hp, mask=mask, gpunum=0, squared=1, prjMode=0)
    with cb.Plan(g, sat_mode=sat_mode) as plan:
        out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(dev(torch, vol), out, mask=dev(torch, mask))
        vb = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.back(dev(torch, hp), vb, mask=dev(torch, mask))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), hp)
        np.testing.assert_array_equal(vb.cpu().numpy(), hb)


def test_repeated_runs_are_bitwise_identical(torch_cuda):
    torch = torch_cuda
    g = G.config1()
    vol = dev(torch, phantom(G.config1(), 3))
    with cb.Plan(g) as plan:
        a = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        b = torch.zeros_like(a)
        plan.proj(vol, a)
        plan.proj(vol, b)
        va = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        vb = torch.zeros_like(va)
        plan.back(a, va)
        plan.back(a, vb)
        torch.cuda.synchronize()
        assert torch.equal(a, b) and torch.equal(va, vb)


def test_config2_adjointness_full_size(torch_cuda):
    torch = torch_cuda
    g = G.config2()
    gen = torch.Generator(device="cuda").manual_seed(5)
    x = torch.rand(g.vol_shape, dtype=torch.float32, device="cuda", generator=gen)
    y = torch.rand(g.prj_shape, dtype=torch.float32, device="cuda", generator=gen)
    with cb.Plan(g) as plan:
        ax = torch.zeros_like(y)
        plan.proj(x, ax)
        by = torch.zeros_like(x)
        plan.back(y, by)
        torch.cuda.synchronize()
        a = float((ax.double() * y.double()).sum())
        b = float((x.double() * by.double()).sum())
    record_error("adjoint_gap/config2", abs(a - b) / abs(a))
    assert abs(a - b) / abs(a) < 1e-4


def test_uniform_volume_central_rays_equal_chord_full_size(torch_cuda):
    torch = torch_cuda
    g = G.config2()
    with cb.Plan(g) as plan:
        ones = torch.ones(g.vol_shape, dtype=torch.float32, device="cuda")
        out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(ones, out)
        torch.cuda.synchronize()
        p = out.cpu().numpy()
    for k in (0, 130, 246, 400, 700):
        th = float(g.hangs[k]) % (2 * math.pi)
        c, s = math.cos(th), math.sin(th)
        S = np.array([-g.y0 * s, g.y0 * c, 0.0])
        xdrv = (math.pi / 4 <= th < 3 * math.pi / 4) or (5 * math.pi / 4 <= th < 7 * math.pi / 4)
        for u in (g.DNU // 2 - 1, g.DNU // 2):
            for v in (g.DNV // 2 - 1, g.DNV // 2):
                D = np.array([g.xds[u] * c - g.yds[u] * s, g.xds[u] * s + g.yds[u] * c, g.zds[v]])
                d = D - S
                chord = g.XN * g.dx * np.linalg.norm(d) / abs(d[0] if xdrv else d[1])
                assert abs(p[k, u, v] - chord) < 2e-5 * chord


def test_backprojection_rejects_curved_detector(torch_cuda):
    torch = torch_cuda
    g = G.small()
    ang = (np.arange(g.DNU) - (g.DNU - 1) / 2) * 0.002
    g.xds = (G.SDD * np.sin(ang)).astype(np.float32)
    g.yds = (G.SOD - G.SDD * np.cos(ang)).astype(np.float32)
    with cb.Plan(g) as plan:
        prj = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        vol = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.proj(vol, prj)  # projection accepts any detector
        with pytest.raises(cb.CtlabError) as e:
            plan.back(prj, vol)
        assert e.value.code == cb.CTLAB_ERR_UNSUPPORTED


def test_curved_detector_projection_matches_oracle(torch_cuda):
    torch = torch_cuda
    g = G.small()
    ang = (np.arange(g.DNU) - (g.DNU - 1) / 2) * 0.002
    g.xds = (G.SDD * np.sin(ang)).astype(np.float32)
    g.yds = (G.SOD - G.SDD * np.cos(ang)).astype(np.float32)
    vol = phantom(g)
    ref = oracle.dd3_proj(g, vol)
    with cb.Plan(g) as plan:
        out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(dev(torch, vol), out)
        torch.cuda.synchronize()
        assert rel_l2(out.cpu().numpy(), ref) <= REL_L2


def test_bounded_wait_times_out_and_context_survives(torch_cuda):
    torch = torch_cuda
    lib = cb.load()
    rc = lib.ctlab_debug_scan_stall(0, 2000)
    assert rc == cb.CTLAB_ERR_TIMEOUT, lib.ctlab_last_error()
    # the context is still usable
    g = G.small()
    with cb.Plan(g) as plan:
        out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(dev(torch, phantom(g)), out)
        torch.cuda.synchronize()
        assert float(out.abs().sum()) > 0


@pytest.mark.parametrize("zpos", [None, "helical"])
def test_zprefix_tall_volume_matches_oracle(torch_cuda, zpos):
    """A volume longer than the cone (ZN = 1200, several backprojector z blocks, beyond
    the FP64 projector's shared-memory columns): the z-prefix projector stages z ranges,
    and backprojector CTAs skip the views whose cone misses their z range."""
    torch = torch_cuda
    PN = 24
    zp = np.linspace(-10.0, 10.0, PN) if zpos else None
    g = G.small(PN=PN, XN=10, YN=9, ZN=1200, dz=0.02, DNU=24, DNV=40, row_size=0.1, zpos=zp)
    vol = phantom(g)
    rng = np.random.default_rng(5)
    prj = oracle.dd3_proj(g, vol).astype(np.float32) + 0.01 * rng.random(g.prj_shape).astype(np.float32)
    ref_p = oracle.dd3_proj(g, vol)
    ref_b = oracle.dd3_back(g, prj)
    with cb.Plan(g, sat_mode=cb.CTLAB_SAT_ZPREFIX) as plan:
        out_p = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(dev(torch, vol), out_p)
        out_b = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.back(dev(torch, prj), out_b)
        torch.cuda.synchronize()
        ep, eb = rel_l2(out_p.cpu().numpy(), ref_p), rel_l2(out_b.cpu().numpy(), ref_b)
    record_error(f"proj/tall_z_{zpos}/zprefix", ep)
    record_error(f"back/tall_z_{zpos}/zprefix", eb)
    assert ep <= REL_L2 and eb <= REL_L2, (ep, eb)


@pytest.mark.parametrize("sat_mode", [cb.CTLAB_SAT_ZPREFIX, cb.CTLAB_SAT_FP64])
@pytest.mark.parametrize("pinned", [False, True])
def test_legacy_overlapped_copies_equal_plan_path(torch_cuda, sat_mode, pinned, monkeypatch):
    """DD3Proj_gpu / DD3Back_gpu copy in chunks overlapped with the compute (the volume
    in y slabs, the projections in blocks of view groups, the backprojection in slabs of
    brick rows) from pinned or pageable host buffers: still bit for bit the plan path's
    results, on a scan large enough to split (config 1, 128x128x64, 360 views)."""
    torch = torch_cuda
    monkeypatch.setenv("CTLAB_LEGACY_SAT", str(sat_mode))
    g = G.config1()
    vol = phantom(g, 9)
    mask = (np.random.default_rng(6).random(g.XN * g.YN) > 0.2).astype(np.uint8)

    def host(shape):
        if pinned:
            return torch.zeros(shape, dtype=torch.float32, pin_memory=True).numpy()
        return np.zeros(shape, np.float32)

    hv = host(g.vol_shape)
    hv[...] = vol
    hp = host(g.prj_shape)
    cb.DD3Proj_gpu(**g.args(), hvol=hv, hprj=hp, mask=mask, gpunum=0, prjMode=0)
    hb = host(g.vol_shape)
    cb.DD3Back_gpu(**g.args(), hvol=hb, hprj=hp, mask=mask, gpunum=0, squared=0, prjMode=0)
    with cb.Plan(g, sat_mode=sat_mode) as plan:
        out = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
        plan.proj(dev(torch, vol), out, mask=dev(torch, mask))
        vb = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.back(dev(torch, hp), vb, mask=dev(torch, mask))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), hp)
        np.testing.assert_array_equal(vb.cpu().numpy(), hb)


_SHAPE_SCRIPT = r"""
import sys, json
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import ctlab_b200 as cb, oracle
from ctlab_b200 import geometry as G
out = {}
cases = {"small": dict(), "odd_offsets": dict(XN=23, YN=19, ZN=13, DNU=37, DNV=11, col_offset=0.37,
         row_offset=-0.21, center=(1.3, -0.7, 0.4), start=0.05),
         "helical_long": dict(PN=40, ZN=600, dz=0.05, zpos=np.linspace(-14.0, 14.0, 40)),
         "many_views": dict(PN=240, ZN=40, DNV=20)}
for name, kw in cases.items():
    g = G.small(**kw)
    rng = np.random.default_rng(3)
    prj = rng.random(g.prj_shape).astype(np.float32)
    ref = oracle.dd3_back(g, prj)
    with cb.Plan(g) as plan:
        v = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.back(torch.from_numpy(prj).cuda(), v)
        torch.cuda.synchronize()
        got = v.cpu().numpy()
    out[name] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
print(json.dumps(out))
"""


@pytest.mark.parametrize("zs", ["4", "8", "16"])
def test_backprojector_block_shapes_match_oracle(torch_cuda, zs):
    """Every block shape of the z-prefix backprojector (CTLAB_BACKT_ZS forces one for the
    whole process: 256, 512 or 1024 threads) on short and long view lists, odd sizes and a
    long helical volume (z blocks skipped per view)."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, CTLAB_BACKT_ZS=zs)
    r = subprocess.run([sys.executable, "-c", _SHAPE_SCRIPT, root], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    errs = json.loads(r.stdout.strip().splitlines()[-1])
    for name, e in errs.items():
        record_error(f"back/{name}/shape{zs}", e)
        assert e <= REL_L2, (name, zs, e)
