"""The C-ABI library loads without a GPU, exports every entry point declared
in include/*.h, and rejects bad arguments on the host before touching CUDA."""
import ctypes as C
import glob
import os
import subprocess

import numpy as np
import pytest

import ctlab_b200 as cb
from ctlab_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    lib = cb.load()
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names += _lib.header_symbols(h)
    assert "DD3Proj_gpu" in names and "DD3Back_gpu" in names and "ctlab_os_sart" in names
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(lib, n)


def _geom(**kw):
    g = cb.small()
    for k, v in kw.items():
        setattr(g, k, v)
    return g


def _plan_create(g):
    lib = cb.load()
    keep = [g.xds, g.yds, g.zds, g.hangs, g.hzPos]
    fp = C.POINTER(C.c_float)
    geo = _lib.Geometry(g.x0, g.y0, g.z0, g.DNU, g.DNV, g.xds.ctypes.data_as(fp), g.yds.ctypes.data_as(fp),
                        g.zds.ctypes.data_as(fp), g.imgXCenter, g.imgYCenter, g.imgZCenter,
                        g.hangs.ctypes.data_as(fp), g.hzPos.ctypes.data_as(fp), g.PN, g.XN, g.YN, g.ZN, g.dx, g.dz)
    h = C.c_void_p()
    rc = lib.ctlab_plan_create(C.byref(geo), 0, 0, C.byref(h))
    del keep
    return rc, lib.ctlab_last_error().decode()


@pytest.mark.parametrize("field,value,needle", [
    ("XN", 0, "sizes"), ("dx", -1.0, "voxel"), ("dz", float("nan"), "voxel"),
])
def test_plan_rejects_bad_sizes_on_host(field, value, needle):
    rc, msg = _plan_create(_geom(**{field: value}))
    assert rc == cb.CTLAB_ERR_INVALID_ARG and needle in msg


def test_plan_rejects_nonfinite_geometry():
    g = cb.small()
    g.hangs[3] = np.inf
    rc, msg = _plan_create(g)
    assert rc == cb.CTLAB_ERR_INVALID_ARG and "non-finite" in msg


def test_plan_rejects_oversized_scans_on_host():
    g = cb.small()
    g.XN = g.YN = g.ZN = 8000  # 5.1e11 voxels: the size product is checked in FP64
    rc, msg = _plan_create(g)
    assert rc == cb.CTLAB_ERR_INVALID_ARG and "too large" in msg
    g = cb.small()
    g.zds = np.linspace(-40.0, 40.0, 5000).astype(np.float32)  # 5000 detector rows
    rc, msg = _plan_create(g)
    assert rc == cb.CTLAB_ERR_INVALID_ARG and "supported range" in msg


def test_plan_rejects_source_inside_volume_extent():
    g = cb.small()
    g.y0 = 2.0  # source inside the 10 mm volume
    rc, msg = _plan_create(g)
    assert rc == cb.CTLAB_ERR_INVALID_ARG and "source" in msg


def test_legacy_projection_rejects_other_models_without_touching_cuda():
    g = cb.small()
    vol = np.zeros(g.vol_shape, np.float32)
    prj = np.zeros(g.prj_shape, np.float32)
    with pytest.raises(cb.CtlabError) as e:
        cb.DD3Proj_gpu(**g.args(), hvol=vol, hprj=prj, mask=None, gpunum=0, prjMode=4)
    assert e.value.code == cb.CTLAB_ERR_UNSUPPORTED
    with pytest.raises(cb.CtlabError) as e:
        cb.DD3Back_gpu(**g.args(), hvol=vol, hprj=prj, mask=None, gpunum=0, squared=0, prjMode=2)
    assert e.value.code == cb.CTLAB_ERR_UNSUPPORTED


def test_legacy_wrappers_check_buffer_sizes():
    g = cb.small()
    with pytest.raises(cb.CtlabError):
        cb.DD3Proj_gpu(**g.args(), hvol=np.zeros(5, np.float32), hprj=np.zeros(g.prj_shape, np.float32),
                       mask=None, gpunum=0, prjMode=0)


def test_status_is_thread_local_and_cleared():
    lib = cb.load()
    _plan_create(_geom(XN=0))
    assert lib.ctlab_last_status() == cb.CTLAB_ERR_INVALID_ARG
    assert lib.ctlab_last_error()


def test_random_ellipsoids_are_seeded_and_in_range():
    a = cb.random_ellipsoids(1, 256, 256, 20)
    b = cb.random_ellipsoids(1, 256, 256, 20)
    c = cb.random_ellipsoids(2, 256, 256, 20)
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a[: min(len(a), len(c))], c[: min(len(a), len(c))])
    assert 20 <= len(a) <= 40
    assert np.all(np.abs(a[:, 1]) <= 0.8 * 256) and np.all(np.abs(a[:, 3]) <= 0.8 * 20)
    assert np.all((a[:, 4] >= 0.05 * 256) & (a[:, 4] <= 0.4 * 256))
    assert np.all((a[:, 0] >= 0) & (a[:, 0] <= 0.03))
    assert np.all((a[:, 7:] >= 0) & (a[:, 7:] <= np.pi))


def test_cnn_entry_points_reject_bad_arguments_on_host():
    # never dereferenced: every call below returns before any CUDA call
    lib, p = cb.load(), C.c_void_p(16)
    inv, uns = cb.CTLAB_ERR_INVALID_ARG, cb.CTLAB_ERR_UNSUPPORTED
    relu, mask, resid = 0, 1, 2
    assert lib.ctlab_cnn_conv(None, 64, p, p, 64, 1, 8, 8, relu, p, None, None, None, None) == inv
    assert lib.ctlab_cnn_conv(p, 64, p, p, 64, 0, 8, 8, relu, p, None, None, None, None) == inv
    assert lib.ctlab_cnn_conv(p, 64, p, None, 64, 1, 8, 8, relu, p, None, None, None, None) == inv  # no bias
    assert lib.ctlab_cnn_conv(p, 64, p, p, 64, 1, 8, 8, mask, p, None, None, None, None) == inv  # no mask
    assert lib.ctlab_cnn_conv(p, 64, p, p, 16, 1, 8, 8, resid, None, None, p, None, None) == inv  # no centre
    assert lib.ctlab_cnn_conv(p, 32, p, p, 64, 1, 8, 8, relu, p, None, None, None, None) == uns
    assert "channels" in lib.ctlab_last_error().decode()
    assert lib.ctlab_cnn_wgrad(p, 64, None, 64, 1, 8, 8, p, None, None) == inv
    assert lib.ctlab_cnn_wgrad(p, 64, p, 32, 1, 8, 8, p, None, None) == uns
