"""Warm-start CNN kernels (ctlab_cnn_*) against the FP64 numpy restatement
(oracle/cnn.py) on BF16-rounded operands, the network's gradients against a
numpy forward/backward with the same BF16 rounding points, and what training
gains: on held-out data the trained network's output is closer to the
30-iteration OS-SART image than its 2-iteration input."""
import numpy as np
import pytest

import ctlab_b200 as cb
import oracle
from ctlab_b200 import geometry as G
from oracle import cnn as ocnn

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def to_bf16_dev(torch, a):
    return torch.from_numpy(ocnn.bf16_bits(a).view(np.int16)).cuda().view(torch.bfloat16)


def from_bf16_dev(t):
    import torch
    return (t.view(torch.int16).cpu().numpy().astype(np.uint16).astype(np.uint32) << 16).view(np.float32)


# partial 8x16 tiles on purpose; the last shape gives every persistent CTA
# three or more tiles, so both halo buffers and accumulators are reused
SHAPES = [(2, 12, 20), (1, 9, 33), (8, 72, 200)]


@pytest.mark.parametrize("ci,co", [(16, 64), (64, 64), (64, 16)])
@pytest.mark.parametrize("shape", SHAPES)
def test_conv_forward_matches_numpy(torch_cuda, ci, co, shape):
    torch = torch_cuda
    lib = cb.load()
    B, H, W = shape
    rng = np.random.default_rng(ci + co + H)
    x = ocnn.bf16(rng.standard_normal((B, H, W, ci)))
    w = ocnn.bf16(rng.standard_normal((co, 9, ci)) * 0.1)
    b = rng.standard_normal(co).astype(np.float32)
    ref = ocnn.conv3x3(x, w, b)
    dx, dw, db = to_bf16_dev(torch, x), to_bf16_dev(torch, w), torch.from_numpy(b).cuda()
    if co == 16:  # output layer: channel 0 + bias + centre in FP32
        center = torch.from_numpy(rng.standard_normal((B, H, W)).astype(np.float32)).cuda()
        out = torch.zeros((B, H, W), dtype=torch.float32, device="cuda")
        assert lib.ctlab_cnn_conv(dx.data_ptr(), ci, dw.data_ptr(), db.data_ptr(), co, B, H, W, 2, None, None,
                                  out.data_ptr(), center.data_ptr(), None) == 0
        assert lib.ctlab_cnn_check(None) == 0  # no tensor-core wait ran out
        got = out.cpu().numpy()
        want = ref[..., 0] + center.cpu().numpy()
        assert rel(got, want) <= 1e-5
    else:
        out = torch.zeros((B, H, W, co), dtype=torch.bfloat16, device="cuda")
        assert lib.ctlab_cnn_conv(dx.data_ptr(), ci, dw.data_ptr(), db.data_ptr(), co, B, H, W, 0, out.data_ptr(),
                                  None, None, None, None) == 0
        assert lib.ctlab_cnn_check(None) == 0
        got = from_bf16_dev(out).reshape(B, H, W, co)
        want = np.maximum(ref, 0)
        assert rel(got, want) <= 6e-3  # BF16 output rounding (2^-9 relative)


@pytest.mark.parametrize("ci,co", [(16, 64), (64, 64), (64, 16)])
def test_conv_weight_gradient_matches_numpy(torch_cuda, ci, co):
    torch = torch_cuda
    lib = cb.load()
    B, H, W = 2, 11, 37
    rng = np.random.default_rng(3 * ci + co)
    act = ocnn.bf16(rng.standard_normal((B, H, W, ci)))
    dpre = ocnn.bf16(rng.standard_normal((B, H, W, co)))
    ref = ocnn.conv_wgrad(dpre, act)
    dw = torch.zeros(co * 9 * ci, dtype=torch.float32, device="cuda")
    db = torch.zeros(co, dtype=torch.float32, device="cuda")
    assert lib.ctlab_cnn_wgrad(to_bf16_dev(torch, dpre).data_ptr(), co, to_bf16_dev(torch, act).data_ptr(), ci, B, H,
                               W, dw.data_ptr(), db.data_ptr(), None) == 0
    assert rel(dw.cpu().numpy().reshape(co, 9, ci), ref) <= 1e-5
    assert rel(db.cpu().numpy(), dpre.astype(np.float64).sum(axis=(0, 1, 2))) <= 1e-5


def test_conv_data_gradient_is_flipped_transposed_convolution(torch_cuda):
    torch = torch_cuda
    lib = cb.load()
    B, H, W, ci, co = 2, 10, 18, 64, 64
    rng = np.random.default_rng(11)
    w = ocnn.bf16(rng.standard_normal((co, 9, ci)) * 0.1)
    dout = ocnn.bf16(rng.standard_normal((B, H, W, co)))
    mask = ocnn.bf16(rng.standard_normal((B, H, W, ci)))
    ref = ocnn.conv3x3(dout, ocnn.flip_transpose(w)) * (mask > 0)
    # the adjoint identity <conv(x, w), d> = <x, conv(d, flip_transpose(w))>
    x = rng.standard_normal((B, H, W, ci))
    lhs = float(np.sum(ocnn.conv3x3(x, w) * dout))
    rhs = float(np.sum(x * ocnn.conv3x3(dout, ocnn.flip_transpose(w))))
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs)
    out = torch.zeros((B, H, W, ci), dtype=torch.bfloat16, device="cuda")
    assert lib.ctlab_cnn_conv(to_bf16_dev(torch, dout).data_ptr(), co,
                              to_bf16_dev(torch, ocnn.flip_transpose(w)).data_ptr(), None, ci, B, H, W, 1,
                              out.data_ptr(), to_bf16_dev(torch, mask).data_ptr(), None, None, None) == 0
    assert rel(from_bf16_dev(out).reshape(B, H, W, ci), ref) <= 6e-3


def numpy_network(net, inp, center, target):
    """Forward + backward of the network in FP64 with the kernels' BF16
    rounding points (activations, data gradients, loss gradient)."""
    from ctlab_b200.learned import LAYERS
    ws, bs = [], []
    for li, (ci, co) in enumerate(LAYERS):
        p = net.params[li].cpu().numpy()
        ws.append(ocnn.bf16(p[: co * 9 * ci].reshape(co, 9, ci)))
        bs.append(p[co * 9 * ci:])
    acts = [inp]
    x = inp
    for li in range(len(LAYERS) - 1):
        x = ocnn.bf16(np.maximum(ocnn.conv3x3(x, ws[li], bs[li]), 0).astype(np.float32))
        acts.append(x)
    pred = ocnn.conv3x3(x, ws[-1], bs[-1])[..., 0] + center
    n = pred.size
    d = np.zeros(pred.shape + (16,))
    d[..., 0] = ocnn.bf16((2.0 / n * (pred - target)).astype(np.float32))
    grads = [None] * len(LAYERS)
    for li in range(len(LAYERS) - 1, -1, -1):
        grads[li] = ocnn.conv_wgrad(d, acts[li])
        if li:
            d = ocnn.bf16((ocnn.conv3x3(d, ocnn.flip_transpose(ws[li])) * (acts[li] > 0)).astype(np.float32))
    return pred, grads


def test_network_gradients_match_numpy(torch_cuda):
    torch = torch_cuda
    from ctlab_b200.learned import LAYERS, WarmStartNet
    net = WarmStartNet(seed=5)
    B, H, W = 2, 14, 22
    rng = np.random.default_rng(8)
    raw = np.zeros((B, H, W, 16), np.float32)
    raw[..., :5] = rng.random((B, H, W, 5))
    inp = ocnn.bf16(raw)
    center = inp[..., 2].copy()
    target = (center + 0.1 * rng.standard_normal((B, H, W))).astype(np.float32)
    pred = net.forward(to_bf16_dev(torch, inp), torch.from_numpy(center).cuda())
    net.backward(pred, torch.from_numpy(target).cuda())
    ref_pred, ref_grads = numpy_network(net, inp, center, target)
    # activations are re-rounded to BF16 after every layer from FP32 (GPU) or
    # FP64 (numpy) sums, so an occasional last-bit flip propagates: 1e-3
    assert rel(pred.cpu().numpy(), ref_pred) <= 1e-3
    for li, (ci, co) in enumerate(LAYERS):
        got = net.grad[li][: co * 9 * ci].cpu().numpy().reshape(co, 9, ci)
        err = rel(got, ref_grads[li])
        assert err <= 2e-2, (li, err)


def make_pairs(torch, g, seeds, iters_in=2, iters_out=30):
    """(2-iteration, 30-iteration) OS-SART images of noisy projections of random phantoms."""
    hx, hy, hz = G.half_extents(g)
    pairs = []
    with cb.Plan(g) as plan:
        for s in seeds:
            truth = torch.zeros(g.vol_shape, dtype=torch.float32, device="cuda")
            cb.ellipsoid_phantom(truth, g, cb.random_ellipsoids(100 + s, hx, hy, hz))
            clean = torch.zeros(g.prj_shape, dtype=torch.float32, device="cuda")
            plan.proj(truth, clean)
            gen = torch.Generator(device="cuda")
            gen.manual_seed(s)
            counts = torch.poisson(1e5 * torch.exp(-clean), generator=gen)
            meas = -torch.log(torch.clamp(counts, min=1.0) / 1e5)
            x = torch.zeros_like(truth)
            plan.os_sart(x, meas, os_num=8, iter_num=iters_in)
            x2 = x.clone()
            plan.os_sart(x, meas, os_num=8, iter_num=iters_out - iters_in)
            pairs.append((x2, x))
    return pairs


def test_trained_network_moves_the_warm_start_toward_the_converged_image(torch_cuda):
    torch = torch_cuda
    from ctlab_b200.learned import WarmStartNet
    g = G.DD3Geometry.flat(sid=541.0, sdd=949.0, DNU=96, DNV=24, col_size=1.0, row_size=1.0, PN=96, XN=48, YN=48,
                           ZN=16, dx=1.0, dz=1.0)
    pairs = make_pairs(torch, g, seeds=range(5))
    train, held = pairs[:4], pairs[4]
    scale = 1.0 / 0.03
    net = WarmStartNet(seed=1)
    rng = np.random.default_rng(0)
    losses = []
    for step in range(300):
        x2, x30 = train[step % len(train)]
        zs = rng.integers(0, g.ZN, 8)
        losses.append(net.train_step(x2, x30, zs, scale, lr=1e-3))
    assert np.mean(losses[-30:]) < 0.5 * np.mean(losses[:30])
    x2, x30 = held
    out = torch.zeros_like(x2)
    net.predict_volume(x2, scale, out)
    before = float(torch.linalg.norm(x2 - x30) / torch.linalg.norm(x30))
    after = float(torch.linalg.norm(out - x30) / torch.linalg.norm(x30))
    assert after < 0.8 * before, (before, after)
