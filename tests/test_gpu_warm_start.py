"""What the trained warm-start network gains, measured by the data residual the
solver reports, ||Ax - b|| / ||b||.  Plain OS-SART runs 20 iterations from zero; the
warm start runs 2 iterations, the network, then OS-SART until its residual reaches the
plain solve's final one -- in fewer iterations in total, on a held-out phantom."""
import numpy as np
import pytest

import ctlab_b200 as cb
from ctlab_b200 import geometry as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def noisy_scan(torch, plan, g, seed):
    hx, hy, hz = G.half_extents(g)
    truth = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
    cb.ellipsoid_phantom(truth, g, cb.random_ellipsoids(100 + seed, hx, hy, hz))
    clean = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
    plan.proj(truth, clean)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    counts = torch.poisson(1e5 * torch.exp(-clean), generator=gen)
    return truth, -torch.log(torch.clamp(counts, min=1.0) / 1e5)


def test_warm_start_reaches_the_plain_residual_in_fewer_iterations(torch_cuda):
    torch = torch_cuda
    from ctlab_b200.learned import WarmStartNet
    g = G.DD3Geometry.flat(sid=541.0, sdd=949.0, DNU=96, DNV=24, col_size=1.0, row_size=1.0, PN=96, XN=48, YN=48,
                           ZN=16, dx=1.0, dz=1.0)
    its, os_num, scale = 20, 8, 1.0 / 0.03
    with cb.Plan(g) as plan:
        pairs = []
        for seed in range(5):
            _, meas = noisy_scan(torch, plan, g, seed)
            x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
            plan.os_sart(x, meas, os_num=os_num, iter_num=2)
            x2 = x.clone()
            plan.os_sart(x, meas, os_num=os_num, iter_num=its - 2)
            pairs.append((x2, x))
        net = WarmStartNet(seed=1)
        rng = np.random.default_rng(0)
        for step in range(400):
            x2, xt = pairs[step % len(pairs)]
            net.train_step(x2, xt, rng.integers(0, g.ZN, 8), scale, lr=1e-3)
        _, meas = noisy_scan(torch, plan, g, 5)  # held out
        x = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
        plain = plan.os_sart(x, meas, os_num=os_num, iter_num=its, residuals=True)
        xl = torch.zeros_like(x)
        first2 = plan.os_sart(xl, meas, os_num=os_num, iter_num=2, residuals=True)
        xw = torch.zeros_like(x)
        net.predict_volume(xl, scale, xw)
        net.check_kernels()
        cont = plan.os_sart(xw, meas, os_num=os_num, iter_num=its, residuals=True)
    assert np.all(np.diff(plain) < 0)
    assert abs(first2[-1] - plain[1]) <= 1e-5 * plain[1]  # the same 2-iteration start
    hits = [k + 1 for k, r in enumerate(cont) if r <= plain[-1]]
    assert hits, (plain[-1], cont)
    assert 2 + hits[0] < its, (hits[0], plain[-1], cont[:5])
