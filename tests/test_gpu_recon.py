"""Device reconstruction loops and elementwise kernels against the oracle and
against golden vectors from the reference's own compiled helpers."""
import os
import subprocess

import numpy as np
import pytest

import ctlab_b200 as cb
import oracle
from ctlab_b200 import geometry as G

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_helpers.npz"))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def scan(seed=0):
    g = G.small(PN=24, XN=22, YN=22, ZN=10, DNU=40, DNV=14, start=0.05)
    hx, hy, hz = G.half_extents(g)
    ell = cb.random_ellipsoids(seed + 3, hx, hy, hz, 5, 8)
    truth = oracle.ellipsoid_phantom(g, ell)
    prj = oracle.dd3_proj(g, truth).astype(np.float32)
    return g, truth, prj


def test_sart_weightings_match_reference_golden(torch_cuda):
    torch = torch_cuda
    lib = cb.load()
    # keep every device tensor alive until the stream has consumed it
    prj, real, rs = dev(torch, GOLD["sart_prj"]), dev(torch, GOLD["sart_real"]), dev(torch, GOLD["sart_rs"])
    vol, rec = dev(torch, GOLD["sart_vol"]), dev(torch, GOLD["sart_rec"])
    torch.cuda.synchronize()
    lib.ctlab_sart_proj_weight(prj.data_ptr(), real.data_ptr(), rs.data_ptr(), prj.numel(), None)
    lib.ctlab_sart_back_weight(vol.data_ptr(), rec.data_ptr(), rs.data_ptr(), vol.numel(), None)
    torch.cuda.synchronize()
    np.testing.assert_allclose(prj.cpu().numpy(), GOLD["sart_prj_out"], rtol=1e-6, atol=0)
    np.testing.assert_allclose(vol.cpu().numpy(), GOLD["sart_vol_out"], rtol=1e-6, atol=0)
    np.testing.assert_allclose(rec.cpu().numpy(), GOLD["sart_rec_out"], rtol=1e-6, atol=1e-6)


def test_fista_step_matches_reference_golden(torch_cuda):
    torch = torch_cuda
    lib = cb.load()
    t1, t2, lo, hi = GOLD["fista_t"]
    cur, las = dev(torch, GOLD["fista_cur"]), dev(torch, GOLD["fista_las"])
    torch.cuda.synchronize()
    lib.ctlab_fista_step(las.data_ptr(), cur.data_ptr(), t1, t2, cur.numel(), lo, hi, None)
    torch.cuda.synchronize()
    np.testing.assert_allclose(cur.cpu().numpy(), GOLD["fista_out"], rtol=2e-7, atol=1e-3)


def test_tv_gradient_matches_oracle(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(0)
    XN, YN, ZN = 17, 13, 9
    f = rng.random((YN, XN, ZN)).astype(np.float32)
    ref = oracle.tv_gradient(f, XN, YN, ZN, 1e-8)
    g = torch.zeros((YN, XN, ZN), dtype=torch.float32, device="cuda")
    fd = dev(torch, f)
    torch.cuda.synchronize()
    cb._lib.check(cb.load().ctlab_tv_gradient(fd.data_ptr(), g.data_ptr(), XN, YN, ZN, 1e-8, None))
    torch.cuda.synchronize()
    np.testing.assert_allclose(g.cpu().numpy(), ref, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("order", [None, "custom"])
def test_os_sart_matches_oracle(torch_cuda, order):
    torch = torch_cuda
    g, truth, prj = scan()
    mask = np.ones(g.XN * g.YN, np.uint8)
    x0 = np.zeros(g.vol_shape, np.float32)
    if order is None:
        ref = oracle.os_sart(g, x0, prj, mask, os_num=4, iter_num=2, lam=1.0)
        h_order = None
    else:
        # a custom subset-major order equal to the interleaved one
        h_order = np.concatenate([np.arange(s, g.PN, 4) for s in range(4)])
        ref = oracle.os_sart(g, x0, prj, mask, os_num=4, iter_num=2, lam=1.0)
    with cb.Plan(g) as plan:
        x = dev(torch, x0)
        res = plan.os_sart(x, dev(torch, prj), dev(torch, mask), os_num=4, iter_num=2, lam=1.0, order=h_order,
                           residuals=True)
        torch.cuda.synchronize()
        got = x.cpu().numpy()
    assert rel_l2(got, ref) < 1e-4
    assert res[1] < res[0] < 1.0


def test_os_sart_reduces_residual_and_error(torch_cuda):
    torch = torch_cuda
    g, truth, prj = scan(1)
    with cb.Plan(g) as plan:
        x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        res = plan.os_sart(x, dev(torch, prj), None, os_num=6, iter_num=6, lam=1.0, residuals=True)
        torch.cuda.synchronize()
        rmse0 = float(np.sqrt((truth ** 2).mean()))
        rmse = float(np.sqrt(((x.cpu().numpy() - truth) ** 2).mean()))
    assert np.all(np.diff(res) < 0)
    assert res[-1] < 0.1 and rmse < 0.6 * rmse0


def test_fista_tv_matches_oracle(torch_cuda):
    torch = torch_cuda
    g, truth, prj = scan(2)
    mask = np.ones(g.XN * g.YN, np.uint8)
    x0 = np.zeros(g.vol_shape, np.float32)
    ref = oracle.fista_tv(g, x0, prj, mask, iter_num=3, tv_lambda=1e-4, tv_eps=1e-8)
    with cb.Plan(g) as plan:
        x = dev(torch, x0)
        res = plan.fista_tv(x, dev(torch, prj), dev(torch, mask), iter_num=3, tv_lambda=1e-4, tv_eps=1e-8,
                            residuals=True)
        torch.cuda.synchronize()
        got = x.cpu().numpy()
    assert rel_l2(got, ref) < 1e-4
    assert res[-1] < res[0]


def test_os_sart_rejects_bad_order(torch_cuda):
    torch = torch_cuda
    g, truth, prj = scan()
    with cb.Plan(g) as plan:
        x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        with pytest.raises(cb.CtlabError) as e:
            plan.os_sart(x, dev(torch, prj), None, os_num=4, iter_num=1, order=np.zeros(g.PN, np.int32))
        assert e.value.code == cb.CTLAB_ERR_INVALID_ARG


@pytest.mark.parametrize("method", [0, 1, 2, 3, 4])
def test_cg_matches_oracle(torch_cuda, method):
    """ctlab_cg against the FP64 numpy CG (same exact line search and beta
    rule); after 3 iterations the images agree to 1e-3 relative L2 and the
    residual decreases every iteration."""
    torch = torch_cuda
    g = G.small(PN=16, XN=16, YN=14, ZN=10, DNU=28, DNV=12, start=0.1)
    hx, hy, hz = G.half_extents(g)
    truth = oracle.ellipsoid_phantom(g, G.shepp_logan_ellipsoids(hx, hy, hz))
    meas = oracle.dd3_proj(g, truth).astype(np.float32)
    x0 = np.zeros(g.vol_shape, np.float32)
    ref, ref_res = oracle.cg(g, x0, meas, iter_num=3, method=method)
    with cb.Plan(g) as plan:
        x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        res = plan.cg(x, torch.from_numpy(meas).cuda(), iter_num=3, method=method, residuals=True)
        torch.cuda.synchronize()
        got = x.cpu().numpy()
    err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    assert err <= 1e-3, err
    assert np.all(np.diff(res) < 0), res
    np.testing.assert_allclose(res, ref_res, rtol=1e-3)


def _write_scan(path, g, sid, sdd, col_size, row_size, os_num, iters, init, prj, mask):
    with open(path, "wb") as f:
        np.array([g.DNU, g.DNV, g.PN, g.XN, g.YN, g.ZN, os_num, iters], np.int32).tofile(f)
        np.array([sid, sdd, g.imgXCenter, g.imgYCenter, g.imgZCenter, g.dx, g.dz, col_size, row_size, 0.0, 0.0],
                 np.float32).tofile(f)
        np.asarray(g.hangs, np.float32).tofile(f)
        np.asarray(g.hzPos, np.float32).tofile(f)
        np.asarray(init, np.float32).tofile(f)
        np.asarray(prj, np.float32).tofile(f)
        np.asarray(mask, np.uint8).tofile(f)


@pytest.mark.parametrize("solver", ["os", "cg"])
def test_reference_signature_cxx_entry_points_equal_device_path(torch_cuda, solver, tmp_path):
    """OS_SART / CG called from a C++ program through the reference's
    thrust::host_vector signatures give the device solver's image."""
    import test_cxx_abi
    torch = torch_cuda
    sid, sdd, cs, rs = 541.0, 949.0, 1.0, 1.0
    g = G.DD3Geometry.flat(sid=sid, sdd=sdd, DNU=48, DNV=16, col_size=cs, row_size=rs, PN=24, XN=20, YN=18,
                           ZN=12, dx=0.8, dz=0.8)
    hx, hy, hz = G.half_extents(g)
    truth = oracle.ellipsoid_phantom(g, G.shepp_logan_ellipsoids(hx, hy, hz))
    meas = oracle.dd3_proj(g, truth).astype(np.float32)
    mask = (np.random.default_rng(3).random(g.XN * g.YN) > 0.1).astype(np.uint8)
    init = np.zeros(g.vol_shape, np.float32)
    inp, out = tmp_path / "in.bin", tmp_path / "out.raw"
    _write_scan(inp, g, sid, sdd, cs, rs, 4, 2, init, meas, mask)
    exe = str(tmp_path / "caller")
    test_cxx_abi.build_caller("host", exe)
    r = subprocess.run([exe, str(inp), str(out), solver, "1"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.float32).reshape(g.vol_shape)
    with cb.Plan(g) as plan:
        x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        m = torch.from_numpy(mask).cuda()
        if solver == "os":
            plan.os_sart(x, torch.from_numpy(meas).cuda(), mask=m, os_num=4, iter_num=2)
        else:
            plan.cg(x, torch.from_numpy(meas).cuda(), mask=m, iter_num=2, method=1)
        torch.cuda.synchronize()
        ref = x.cpu().numpy()
    err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    assert err <= 1e-6, err


def test_os_sart_calls_reuse_weights_only_for_the_same_subsets_and_mask(torch_cuda):
    """A plan keeps its OS-SART workspace and SART weights between calls: 2 + 2
    iterations equal 4 in one call bit for bit; a mask rewritten in place, other
    subsets or another order between calls give what a fresh plan gives."""
    torch = torch_cuda
    g, truth, prj = scan(2)
    meas = dev(torch, prj)
    mask_a = np.ones(g.XN * g.YN, np.uint8)
    mask_b = (np.random.default_rng(9).random(g.XN * g.YN) > 0.25).astype(np.uint8)
    with cb.Plan(g) as plan:
        one = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.os_sart(one, meas, dev(torch, mask_a), os_num=4, iter_num=4)
        two = torch.zeros_like(one)
        m = dev(torch, mask_a)
        plan.os_sart(two, meas, m, os_num=4, iter_num=2)
        plan.os_sart(two, meas, m, os_num=4, iter_num=2)
        torch.cuda.synchronize()
        assert torch.equal(one, two)
        # same device buffer, new mask bytes
        m.copy_(dev(torch, mask_b))
        x_b = torch.zeros_like(one)
        plan.os_sart(x_b, meas, m, os_num=4, iter_num=2)
        # other subsets, then a custom order
        x_c = torch.zeros_like(one)
        plan.os_sart(x_c, meas, m, os_num=3, iter_num=2)
        order = np.random.default_rng(1).permutation(g.PN)
        x_d = torch.zeros_like(one)
        plan.os_sart(x_d, meas, m, os_num=3, iter_num=2, order=order)
        torch.cuda.synchronize()
    with cb.Plan(g) as fresh:
        refs = []
        for os_num, o in ((4, None), (3, None), (3, order)):
            x = torch.zeros_like(one)
            fresh.os_sart(x, meas, dev(torch, mask_b), os_num=os_num, iter_num=2, order=o)
            refs.append(x)
        torch.cuda.synchronize()
    for got, want in zip((x_b, x_c, x_d), refs):
        assert torch.equal(got, want)


def test_fista_tv_and_cg_calls_reuse_their_workspace(torch_cuda):
    """FISTA-TV and CG keep their workspaces on the plan: a second call gives
    the first call's result bit for bit, and a mask rewritten in place between
    FISTA-TV calls gives what a fresh plan gives (its SART weights are rebuilt)."""
    torch = torch_cuda
    g, truth, prj = scan(4)
    meas = dev(torch, prj)
    mask_a = np.ones(g.XN * g.YN, np.uint8)
    mask_b = (np.random.default_rng(5).random(g.XN * g.YN) > 0.3).astype(np.uint8)
    with cb.Plan(g) as plan:
        m = dev(torch, mask_a)
        xs = []
        for _ in range(2):
            x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
            plan.fista_tv(x, meas, m, iter_num=3, tv_lambda=1e-3)
            xs.append(x)
        cgs = []
        for _ in range(2):
            x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
            plan.cg(x, meas, m, iter_num=3, method=1)
            cgs.append(x)
        m.copy_(dev(torch, mask_b))
        x_b = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plan.fista_tv(x_b, meas, m, iter_num=3, tv_lambda=1e-3)
        torch.cuda.synchronize()
    assert torch.equal(xs[0], xs[1]) and torch.equal(cgs[0], cgs[1])
    assert float(xs[0].abs().max()) > 0
    with cb.Plan(g) as fresh:
        want = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        fresh.fista_tv(want, meas, dev(torch, mask_b), iter_num=3, tv_lambda=1e-3)
        torch.cuda.synchronize()
    assert torch.equal(x_b, want)
