"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the FP64 CPU oracle.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs import this package.  See dd3_oracle.c for what is restated from where,
and what pins it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libdd3_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libctlab_ref_helpers.so")

_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_u8 = C.c_void_p
_lib = None


def build(ref: bool = False) -> None:
    subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    if ref:
        subprocess.run(["make", "-C", HERE, "ref"], check=True, capture_output=True)


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        geo = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, _fp, _fp, _fp, C.c_double, C.c_double,
               C.c_double, _fp, _fp, C.c_int, C.c_int, C.c_int, C.c_int]
        lib.orc_dd3_proj.argtypes = geo + [_fp, _dp, C.c_double, C.c_double, _u8]
        lib.orc_dd3_proj.restype = None
        lib.orc_dd3_back.argtypes = geo + [_dp, _fp, C.c_double, C.c_double, _u8]
        lib.orc_dd3_back.restype = C.c_int
        lib.orc_dd3_boundaries.argtypes = [C.c_int, _dp, _dp]
        lib.orc_regularize_angle.argtypes = [C.c_double]
        lib.orc_regularize_angle.restype = C.c_double
        lib.orc_view_is_xdriven.argtypes = [C.c_double]
        lib.orc_sat2d.argtypes = [_dp, C.c_long, C.c_long, C.c_int, C.c_int, _dp]
        lib.orc_volume_sats.argtypes = [C.c_int, C.c_int, C.c_int, _fp, _u8, _dp, _dp]
        lib.orc_detector_is_flat_uniform.argtypes = [C.c_int, C.c_int, _fp, _fp, _fp, C.c_double]
        lib.orc_sart_proj_weight.argtypes = [_fp, _fp, _fp, C.c_long]
        lib.orc_sart_back_weight.argtypes = [_fp, _fp, _fp, C.c_long]
        lib.orc_ossart_update.argtypes = [_fp, _fp, _fp, _u8, C.c_long, C.c_long, C.c_long, C.c_float,
                                          C.c_int, C.c_float, C.c_float]
        lib.orc_fista_step.argtypes = [_fp, _fp, C.c_float, C.c_float, C.c_long, C.c_float, C.c_float]
        lib.orc_tv_gradient.argtypes = [_fp, _fp, C.c_int, C.c_int, C.c_int, C.c_double]
        lib.orc_ellipsoid_phantom.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                              C.c_double, C.c_double, _dp, C.c_int, C.c_int, _fp]
        lib.orc_ellipsoid_line_integral.argtypes = [_dp, C.c_int, _dp, _dp]
        lib.orc_ellipsoid_line_integral.restype = C.c_double
        lib.orc_os_sart.argtypes = geo[:13] + [C.c_int, C.c_int, C.c_int, C.c_int, _fp, _fp, C.c_double,
                                               C.c_double, _u8, C.c_int, C.c_int, C.c_float, C.c_int,
                                               C.c_float, C.c_float]
        lib.orc_os_sart.restype = C.c_int
        lib.orc_fista_tv.argtypes = geo[:13] + [C.c_int, C.c_int, C.c_int, C.c_int, _fp, _fp, C.c_double,
                                                C.c_double, _u8, C.c_int, C.c_float, C.c_double, C.c_float,
                                                C.c_float]
        lib.orc_fista_tv.restype = C.c_int
        lib.orc_view_frame.argtypes = [C.c_double, C.c_double, C.c_double, C.c_float, C.c_float, _dp]
        lib.orc_view_to_world.argtypes = [C.c_float, C.c_float, _dp, _dp]
        lib.orc_random_ellipsoids.argtypes = [C.c_ulonglong, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                              C.c_float, _dp, C.c_int]
        lib.orc_random_ellipsoids.restype = C.c_int
        lib.orc_num_threads.restype = C.c_int
        lib.orc_set_num_threads.argtypes = [C.c_int]
        _lib = lib
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _geo(g):
    return [g.x0, g.y0, g.z0, g.DNU, g.DNV, _f(g.xds).ctypes.data_as(_fp), _f(g.yds).ctypes.data_as(_fp),
            _f(g.zds).ctypes.data_as(_fp), g.imgXCenter, g.imgYCenter, g.imgZCenter,
            _f(g.hangs).ctypes.data_as(_fp), _f(g.hzPos).ctypes.data_as(_fp), g.PN, g.XN, g.YN, g.ZN]


def _mask(mask):
    if mask is None:
        return None, None
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    return m, m.ctypes.data


def dd3_proj(g, vol, mask=None) -> np.ndarray:
    """FP64 branchless DD projection; returns [PN][DNU][DNV] float64."""
    lib = load()
    v = _f(vol)
    out = np.zeros((g.PN, g.DNU, g.DNV), np.float64)
    m, mp = _mask(mask)
    keep = [g.xds, g.yds, g.zds, g.hangs, g.hzPos]  # noqa: F841
    lib.orc_dd3_proj(*_geo(g), v.ctypes.data_as(_fp), out.ctypes.data_as(_dp), g.dx, g.dz, mp)
    return out


def dd3_back(g, prj, mask=None) -> np.ndarray:
    """FP64 branchless DD backprojection; returns a [YN][XN][ZN] float64 volume."""
    lib = load()
    p = _f(prj)
    out = np.zeros((g.YN, g.XN, g.ZN), np.float64)
    m, mp = _mask(mask)
    rc = lib.orc_dd3_back(*_geo(g), out.ctypes.data_as(_dp), p.ctypes.data_as(_fp), g.dx, g.dz, mp)
    if rc != 0:
        raise ValueError("oracle backprojection needs a flat detector with uniform pitch")
    return out


def boundaries(centers) -> np.ndarray:
    c = np.ascontiguousarray(centers, dtype=np.float64)
    out = np.zeros(c.size + 1)
    load().orc_dd3_boundaries(c.size + 1, c.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
    return out


def volume_sats(g, vol, mask=None):
    """Both FP64 volume SATs: (saty [YN][XN+1][ZN+1], satx [XN][YN+1][ZN+1])."""
    lib = load()
    v = _f(vol)
    saty = np.zeros((g.YN, g.XN + 1, g.ZN + 1))
    satx = np.zeros((g.XN, g.YN + 1, g.ZN + 1))
    m, mp = _mask(mask)
    lib.orc_volume_sats(g.XN, g.YN, g.ZN, v.ctypes.data_as(_fp), mp, saty.ctypes.data_as(_dp),
                        satx.ctypes.data_as(_dp))
    return saty, satx


def tv_gradient(vol, XN, YN, ZN, eps=1e-8) -> np.ndarray:
    f = _f(vol)
    g = np.zeros_like(f)
    load().orc_tv_gradient(f.ctypes.data_as(_fp), g.ctypes.data_as(_fp), XN, YN, ZN, eps)
    return g


def ellipsoid_phantom(g, ell, clamp_nonneg=True) -> np.ndarray:
    e = np.ascontiguousarray(ell, dtype=np.float64).reshape(-1, 10)
    out = np.zeros((g.YN, g.XN, g.ZN), np.float32)
    load().orc_ellipsoid_phantom(g.XN, g.YN, g.ZN, g.dx, g.dz, g.imgXCenter, g.imgYCenter, g.imgZCenter,
                                 e.ctypes.data_as(_dp), e.shape[0], 1 if clamp_nonneg else 0,
                                 out.ctypes.data_as(_fp))
    return out


def random_ellipsoids(seed: int, half_x: float, half_y: float, half_z: float, n_min: int = 20, n_max: int = 40,
                      v_max: float = 0.03) -> np.ndarray:
    """The seeded random-ellipsoid records of the synthetic workloads (phantom_rng.cpp)."""
    buf = np.zeros((n_max, 10), np.float64)
    n = load().orc_random_ellipsoids(seed, n_min, n_max, half_x, half_y, half_z, v_max, buf.ctypes.data_as(_dp),
                                     n_max)
    if n < 0:
        raise ValueError("bad random-ellipsoid arguments")
    return buf[:n].copy()


def ellipsoid_line_integral(ell, p0, p1) -> float:
    e = np.ascontiguousarray(ell, dtype=np.float64).reshape(-1, 10)
    a = np.ascontiguousarray(p0, dtype=np.float64)
    b = np.ascontiguousarray(p1, dtype=np.float64)
    return load().orc_ellipsoid_line_integral(e.ctypes.data_as(_dp), e.shape[0], a.ctypes.data_as(_dp),
                                              b.ctypes.data_as(_dp))


def os_sart(g, x0, prj, mask=None, os_num=4, iter_num=2, lam=1.0, clamp=False, min_v=-2000.0, max_v=6000.0):
    x = _f(x0).copy()
    p = _f(prj)
    m, mp = _mask(mask)
    rc = load().orc_os_sart(*_geo(g)[:13], g.PN, g.XN, g.YN, g.ZN, x.ctypes.data_as(_fp), p.ctypes.data_as(_fp),
                            g.dx, g.dz, mp, os_num, iter_num, lam, 1 if clamp else 0, min_v, max_v)
    if rc != 0:
        raise ValueError("oracle OS-SART needs a flat detector with uniform pitch")
    return x


def fista_tv(g, x0, prj, mask=None, iter_num=3, tv_lambda=1e-4, tv_eps=1e-8, min_v=-2000.0, max_v=6000.0):
    x = _f(x0).copy()
    p = _f(prj)
    m, mp = _mask(mask)
    rc = load().orc_fista_tv(*_geo(g)[:13], g.PN, g.XN, g.YN, g.ZN, x.ctypes.data_as(_fp), p.ctypes.data_as(_fp),
                             g.dx, g.dz, mp, iter_num, tv_lambda, tv_eps, min_v, max_v)
    if rc != 0:
        raise ValueError("oracle FISTA-TV needs a flat detector with uniform pitch")
    return x


def cg(g, x0, prj, mask=None, iter_num=3, method=0):
    """Nonlinear conjugate gradient for 1/2 ||A x - b||^2 with an exact line
    search along each direction (FP64 vectors; A, A^T = dd3_proj, dd3_back).
    method: 0 Fletcher-Reeves, 1 Polak-Ribiere-Polyak, 2 Crowder-Wolfe
    (Hestenes-Stiefel), 3 Dixon, 4 Dai-Yuan -- the beta rules named by
    CGMethod, src/DD3_GPU_recon.h:14-19, as published in the nonlinear CG
    literature.  Returns the image and ||A x_k - b|| / ||b|| per iteration."""
    A = lambda v: dd3_proj(g, v, mask).astype(np.float64)
    At = lambda r: dd3_back(g, r, mask).astype(np.float64)
    x = np.asarray(x0, np.float64).copy()
    b = np.asarray(prj, np.float64)
    r = A(x) - b
    gk = At(r)
    d = -gk
    gg = float(np.vdot(gk, gk))
    res = []
    for _ in range(iter_num):
        q = A(d)
        qq, gd = float(np.vdot(q, q)), float(np.vdot(gk, d))
        if qq <= 0 or gg <= 0:
            break
        alpha = -gd / qq
        x += alpha * d
        r += alpha * q
        gn = At(r)
        gng, gng_old, dgn = float(np.vdot(gn, gn)), float(np.vdot(gn, gk)), float(np.vdot(d, gn))
        yd = dgn - gd
        beta = [gng / gg, (gng - gng_old) / gg, (gng - gng_old) / yd if yd else 0.0,
                -gng / gd if gd else 0.0, gng / yd if yd else 0.0][method]
        d = -gn + beta * d
        gk, gg = gn, gng
        res.append(float(np.linalg.norm(r) / np.linalg.norm(b)))
    return x.astype(np.float32), np.array(res)


def set_threads(n: int) -> None:
    load().orc_set_num_threads(n)


def num_threads() -> int:
    return load().orc_num_threads()
