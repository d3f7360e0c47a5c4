"""The allocation-free volume SAT (ctlab_volume_sat_noalloc) against the plan
path's volume SAT, through the C ABI.

The entry point exists for callers that cannot allocate device memory while
they reconstruct (a fixed, pre-reserved device-memory budget, or no implicit
device synchronisation from cudaMalloc / cudaFree allowed): it keeps the
scan's scratch in a fixed array inside the library.  This file is collected
last on purpose; it passes alone in a fresh process and after the rest.
"""
import numpy as np
import pytest

import ctlab_b200 as cb
from ctlab_b200 import geometry as G

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64 SAT tolerance used by the SAT parity tests


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_noalloc_volume_sat_matches_plan_path_on_two_calls(torch_cuda):
    torch = torch_cuda
    lib = cb.load()
    g = G.small(PN=8, XN=70, YN=45, ZN=33, start=0.0)  # views of both driving axes
    rng = np.random.default_rng(17)
    vol = torch.from_numpy(rng.random(g.vol_shape).astype(np.float32)).cuda()
    mask = torch.from_numpy((rng.random(g.XN * g.YN) > 0.2).astype(np.uint8)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    with cb.Plan(g, sat_mode=cb.CTLAB_SAT_FP64) as plan:  # the 2-D FP64 SAT the entry point also builds
        plan.volume_sat(vol, mask)
        refs = {}
        for o in (0, 1):
            planes, rows, zp = plan.sat_layout(o)
            buf = torch.zeros(planes * rows * zp, dtype=torch.float64, device="cuda")
            plan.copy_volume_sat(o, buf)
            refs[o] = (buf, planes, rows, zp)
        torch.cuda.synchronize()
    for call in range(2):
        for o in (0, 1):
            ref, planes, rows, zp = refs[o]
            out = torch.full((planes * rows * zp,), float("nan"), dtype=torch.float64, device="cuda")
            rc = lib.ctlab_volume_sat_noalloc(vol.data_ptr(), mask.data_ptr(), g.XN, g.YN, g.ZN, o, out.data_ptr(),
                                              zp, stream)
            assert rc == cb.CTLAB_OK, lib.ctlab_last_error()
            torch.cuda.synchronize()
            a = out.view(planes, rows, zp)[:, :, : g.ZN + 1].cpu().numpy()
            b = ref.view(planes, rows, zp)[:, :, : g.ZN + 1].cpu().numpy()
            assert np.all(np.isfinite(a)), f"call {call} orientation {o}: unwritten entries"
            np.testing.assert_allclose(a, b, rtol=TOL, atol=TOL * np.abs(b).max())
    assert lib.ctlab_noalloc_check(stream) == cb.CTLAB_OK, lib.ctlab_last_error()


def test_noalloc_check_reports_a_timed_out_scan_once(torch_cuda):
    """A scan on the fixed array whose lookback wait runs out (its first chunk never
    publishes) is reported by ctlab_noalloc_check as a timeout, once; the error word is
    then clear, and the next allocation-free SAT is valid and checks clean."""
    torch = torch_cuda
    lib = cb.load()
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.ctlab_noalloc_check(stream) == cb.CTLAB_OK, lib.ctlab_last_error()
    assert lib.ctlab_debug_noalloc_stall(2000, stream) == cb.CTLAB_OK, lib.ctlab_last_error()
    rc = lib.ctlab_noalloc_check(stream)
    assert rc == cb.CTLAB_ERR_TIMEOUT, lib.ctlab_last_error()
    assert b"timed out" in lib.ctlab_last_error()
    assert lib.ctlab_noalloc_check(stream) == cb.CTLAB_OK  # read and cleared
    # the context and the array stay usable
    g = G.small(PN=4, XN=20, YN=18, ZN=9, start=0.0)
    vol = torch.rand(g.vol_shape, dtype=torch.float32, device="cuda")
    zp = g.ZN + 1
    out = torch.zeros(g.YN * (g.XN + 1) * zp, dtype=torch.float64, device="cuda")
    assert lib.ctlab_volume_sat_noalloc(vol.data_ptr(), None, g.XN, g.YN, g.ZN, 0, out.data_ptr(), zp,
                                        stream) == cb.CTLAB_OK
    assert lib.ctlab_noalloc_check(stream) == cb.CTLAB_OK, lib.ctlab_last_error()
    v = vol.double().cpu().numpy()  # [y][x][z]
    ref = np.zeros((g.YN, g.XN + 1, zp))
    ref[:, 1:, 1:] = np.cumsum(np.cumsum(v, axis=1), axis=2)
    np.testing.assert_allclose(out.view(g.YN, g.XN + 1, zp).cpu().numpy(), ref, rtol=TOL, atol=1e-10)


def test_noalloc_volume_sat_rejects_volumes_beyond_its_scratch(torch_cuda):
    torch = torch_cuda
    lib = cb.load()
    tiny = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.ctlab_volume_sat_noalloc(tiny.data_ptr(), None, 2048, 2048, 1024, 0, out.data_ptr(), 1026, None)
    assert rc == cb.CTLAB_ERR_INVALID_ARG
    assert b"32 MiB" in lib.ctlab_last_error()
