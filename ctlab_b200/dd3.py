"""Python mirror of CTLAB's DD3 entry points on top of libctlab_b200.

Host-array functions keep the reference's names, argument meaning and order
(``DD3Proj_gpu``, ``DD3Back_gpu``: src/DD3_GPU_Proj.h:41-44,
src/DD3_GPU_Back.h:40-44) and raise :class:`CtlabError` where the reference
would have ignored a CUDA error or exited.  :class:`Plan` is the
device-resident, stream-ordered interface over torch CUDA tensors (torch is
used only for device memory and streams).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import CtlabError, check, check_last, load
from .geometry import DD3Geometry

_fp = C.POINTER(C.c_float)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def DD3Proj_gpu(x0, y0, z0, DNU, DNV, xds, yds, zds, imgXCenter, imgYCenter, imgZCenter, hangs, hzPos,
                PN, XN, YN, ZN, hvol, hprj, dx, dz, mask, gpunum=0, prjMode=0):
    """Branchless DD projection of host ``hvol`` into host ``hprj`` (float32,
    written in place).  Same arguments as the reference's DD3Proj_gpu."""
    lib = load()
    xds, yds, zds, hangs, hzPos = map(_f32, (xds, yds, zds, hangs, hzPos))
    _require(hvol, np.float32, XN * YN * ZN, "hvol")
    _require(hprj, np.float32, PN * DNU * DNV, "hprj")
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    if m is not None and m.size != XN * YN:
        raise CtlabError(_lib.CTLAB_ERR_INVALID_ARG, "mask must hold XN*YN bytes")
    lib.DD3Proj_gpu(x0, y0, z0, DNU, DNV, _ptr(xds), _ptr(yds), _ptr(zds), imgXCenter, imgYCenter,
                    imgZCenter, _ptr(hangs), _ptr(hzPos), PN, XN, YN, ZN, _ptr(hvol), _ptr(hprj), dx, dz,
                    None if m is None else m.ctypes.data, gpunum, prjMode)
    check_last()


def DD3Back_gpu(x0, y0, z0, DNU, DNV, xds, yds, zds, imgXCenter, imgYCenter, imgZCenter, hangs, hzPos,
                PN, XN, YN, ZN, hvol, hprj, dx, dz, mask, gpunum=0, squared=0, prjMode=0):
    """Branchless DD backprojection of host ``hprj`` into host ``hvol``
    (float32, written in place).  Same arguments as DD3Back_gpu."""
    lib = load()
    xds, yds, zds, hangs, hzPos = map(_f32, (xds, yds, zds, hangs, hzPos))
    _require(hvol, np.float32, XN * YN * ZN, "hvol")
    _require(hprj, np.float32, PN * DNU * DNV, "hprj")
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    if m is not None and m.size != XN * YN:
        raise CtlabError(_lib.CTLAB_ERR_INVALID_ARG, "mask must hold XN*YN bytes")
    lib.DD3Back_gpu(x0, y0, z0, DNU, DNV, _ptr(xds), _ptr(yds), _ptr(zds), imgXCenter, imgYCenter,
                    imgZCenter, _ptr(hangs), _ptr(hzPos), PN, XN, YN, ZN, _ptr(hvol), _ptr(hprj), dx, dz,
                    None if m is None else m.ctypes.data, gpunum, squared, prjMode)
    check_last()


def DD3Proj_multiGPU(x0, y0, z0, DNU, DNV, xds, yds, zds, imgXCenter, imgYCenter, imgZCenter, hangs, hzPos,
                     PN, XN, YN, ZN, hvol, hprj, dx, dz, mask, prjMode, startPN, gpuNum):
    """One scan's views split over ``gpuNum`` GPUs: GPU i projects views
    [startPN[i], startPN[i+1]).  Same arguments as the reference's DD3Proj_multiGPU."""
    lib = load()
    xds, yds, zds, hangs, hzPos = map(_f32, (xds, yds, zds, hangs, hzPos))
    _require(hvol, np.float32, XN * YN * ZN, "hvol")
    _require(hprj, np.float32, PN * DNU * DNV, "hprj")
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    if m is not None and m.size != XN * YN:
        raise CtlabError(_lib.CTLAB_ERR_INVALID_ARG, "mask must hold XN*YN bytes")
    st = np.ascontiguousarray(startPN, dtype=np.int32)
    if st.size < gpuNum:
        raise CtlabError(_lib.CTLAB_ERR_INVALID_ARG, "startPN must hold gpuNum entries")
    lib.DD3Proj_multiGPU(x0, y0, z0, DNU, DNV, _ptr(xds), _ptr(yds), _ptr(zds), imgXCenter, imgYCenter,
                         imgZCenter, _ptr(hangs), _ptr(hzPos), PN, XN, YN, ZN, _ptr(hvol), _ptr(hprj), dx, dz,
                         None if m is None else m.ctypes.data, prjMode, st.ctypes.data_as(C.POINTER(C.c_int)),
                         gpuNum)
    check_last()


def DD3Back_multiGPU(x0, y0, z0, DNU, DNV, xds, yds, zds, imgXCenter, imgYCenter, imgZCenter, hangs, hzPos,
                     PN, XN, YN, ZN, hvol, hprj, dx, dz, mask, methodId, startVOL, gpuNum):
    """One scan's volume split into z slabs over ``gpuNum`` GPUs: GPU i backprojects
    slices [startVOL[i], startVOL[i+1]).  Same arguments as DD3Back_multiGPU."""
    lib = load()
    xds, yds, zds, hangs, hzPos = map(_f32, (xds, yds, zds, hangs, hzPos))
    _require(hvol, np.float32, XN * YN * ZN, "hvol")
    _require(hprj, np.float32, PN * DNU * DNV, "hprj")
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    if m is not None and m.size != XN * YN:
        raise CtlabError(_lib.CTLAB_ERR_INVALID_ARG, "mask must hold XN*YN bytes")
    st = np.ascontiguousarray(startVOL, dtype=np.int32)
    if st.size < gpuNum:
        raise CtlabError(_lib.CTLAB_ERR_INVALID_ARG, "startVOL must hold gpuNum entries")
    lib.DD3Back_multiGPU(x0, y0, z0, DNU, DNV, _ptr(xds), _ptr(yds), _ptr(zds), imgXCenter, imgYCenter,
                         imgZCenter, _ptr(hangs), _ptr(hzPos), PN, XN, YN, ZN, _ptr(hvol), _ptr(hprj), dx, dz,
                         None if m is None else m.ctypes.data, methodId, st.ctypes.data_as(C.POINTER(C.c_int)),
                         gpuNum)
    check_last()


def geometry_struct(g: DD3Geometry):
    """(ctypes ctlab_geometry, arrays kept alive) for a geometry record."""
    keep = [_f32(a) for a in (g.xds, g.yds, g.zds, g.hangs, g.hzPos)]
    geo = _lib.Geometry(g.x0, g.y0, g.z0, g.DNU, g.DNV, _ptr(keep[0]), _ptr(keep[1]), _ptr(keep[2]),
                        g.imgXCenter, g.imgYCenter, g.imgZCenter, _ptr(keep[3]), _ptr(keep[4]), g.PN, g.XN, g.YN,
                        g.ZN, g.dx, g.dz)
    return geo, keep


def slab_views(g: DD3Geometry, z0: int, z1: int) -> np.ndarray:
    """Views whose rays can reach slices [z0, z1) (ctlab_slab_views, host only); the
    others add exactly zero to the slab's backprojection."""
    lib = load()
    geo, keep = geometry_struct(g)
    out = np.zeros(max(g.PN, 1), np.int32)
    n = lib.ctlab_slab_views(C.byref(geo), z0, z1, out.ctypes.data_as(C.POINTER(C.c_int)), out.size)
    if n < 0:
        check(-n)
    return out[:n].copy()


def slab_geometry(g: DD3Geometry, z0: int, z1: int, views=None) -> DD3Geometry:
    """Slices [z0, z1) of g's volume as a volume of their own (same columns, its
    slices centred where they sit in g), seen by `views` (default: slab_views)."""
    import dataclasses
    if views is None:
        views = slab_views(g, z0, z1)
    szn = z1 - z0
    cz = float(np.float32(float(g.imgZCenter) + (z0 + 0.5 * szn - 0.5 * g.ZN) * float(g.dz)))
    return dataclasses.replace(g, ZN=szn, imgZCenter=cz, hangs=g.hangs[views].copy(), hzPos=g.hzPos[views].copy())


def _require(a, dtype, n, name):
    if not isinstance(a, np.ndarray) or a.dtype != dtype or not a.flags.c_contiguous or a.size != n:
        raise CtlabError(_lib.CTLAB_ERR_INVALID_ARG,
                         f"{name} must be a C-contiguous {np.dtype(dtype).name} array of {n} elements")


def proj(g: DD3Geometry, vol: np.ndarray, mask=None, gpunum: int = 0) -> np.ndarray:
    """Convenience host projection: returns [PN][DNU][DNV] float32."""
    out = np.zeros(g.prj_shape, np.float32)
    DD3Proj_gpu(**_legacy_args(g), hvol=_f32(vol), hprj=out, mask=mask, gpunum=gpunum, prjMode=0)
    return out


def back(g: DD3Geometry, prj: np.ndarray, mask=None, gpunum: int = 0) -> np.ndarray:
    """Convenience host backprojection: returns a (Z,X,Y) volume [YN][XN][ZN]."""
    out = np.zeros(g.vol_shape, np.float32)
    DD3Back_gpu(**_legacy_args(g), hvol=out, hprj=_f32(prj), mask=mask, gpunum=gpunum, squared=0,
                prjMode=0)
    return out


def _legacy_args(g: DD3Geometry) -> dict:
    a = g.args()
    return a


class Plan:
    """Device-resident plan (``ctlab_plan``): geometry tables and SAT
    workspaces on one GPU; calls are ordered on the given CUDA stream."""

    def __init__(self, g: DD3Geometry, device: int = 0, sat_mode: int = _lib.CTLAB_SAT_ZPREFIX):
        self.lib = load()
        self.g = g
        self.device = device
        self._keep = [g.xds, g.yds, g.zds, g.hangs, g.hzPos]
        geo = _lib.Geometry(g.x0, g.y0, g.z0, g.DNU, g.DNV, _ptr(g.xds), _ptr(g.yds), _ptr(g.zds),
                            g.imgXCenter, g.imgYCenter, g.imgZCenter, _ptr(g.hangs), _ptr(g.hzPos),
                            g.PN, g.XN, g.YN, g.ZN, g.dx, g.dz)
        h = C.c_void_p()
        check(self.lib.ctlab_plan_create(C.byref(geo), device, sat_mode, C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self.lib.ctlab_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def _stream(stream):
        if stream is None:
            import torch
            return torch.cuda.current_stream().cuda_stream
        return stream

    @staticmethod
    def _p(t):
        return None if t is None else t.data_ptr()

    def workspace_bytes(self) -> int:
        return int(self.lib.ctlab_plan_workspace_bytes(self.handle))

    def set_timing(self, on: bool = True):
        check(self.lib.ctlab_plan_set_timing(self.handle, 1 if on else 0))

    def last_times(self) -> tuple[float, float]:
        a, b = C.c_float(), C.c_float()
        check(self.lib.ctlab_plan_last_times(self.handle, C.byref(a), C.byref(b)))
        return a.value, b.value

    def last_launches(self) -> int:
        return int(self.lib.ctlab_plan_last_launches(self.handle))

    def autotune(self, vol, out, cache_path: str | None = None) -> float:
        """Picks the fastest projector staging for this scan (ctlab_plan_autotune);
        returns its time in ms, or -1 when it came from the cache."""
        ms = C.c_float()
        check(self.lib.ctlab_plan_autotune(self.handle, self._p(vol), self._p(out),
                                           None if cache_path is None else cache_path.encode(), C.byref(ms)))
        return ms.value

    def proj_tiles(self) -> dict:
        """The z-prefix projector's staging (views per CTA, rows per warp, ...)."""
        t = (C.c_int * 8)()
        check(self.lib.ctlab_plan_proj_tiles(self.handle, t))
        keys = ("views_per_cta", "rows_per_warp", "warps_per_view", "z_splits", "box_cols", "box_rows",
                "stages", "ctas")
        return dict(zip(keys, list(t)))

    def proj(self, vol, out, mask=None, stream=None):
        check(self.lib.ctlab_proj(self.handle, self._p(vol), self._p(mask), self._p(out), self._stream(stream)))
        return out

    def proj_views(self, views, vol, out, mask=None, stream=None):
        v = np.ascontiguousarray(views, dtype=np.int32)
        check(self.lib.ctlab_proj_views(self.handle, v.ctypes.data_as(C.POINTER(C.c_int)), int(v.size),
                                        self._p(vol), self._p(mask), self._p(out), self._stream(stream)))
        return out

    def back(self, prj, out, mask=None, stream=None):
        check(self.lib.ctlab_back(self.handle, self._p(prj), self._p(mask), self._p(out), self._stream(stream)))
        return out

    def back_views(self, views, prj, out, mask=None, stream=None):
        v = np.ascontiguousarray(views, dtype=np.int32)
        check(self.lib.ctlab_back_views(self.handle, v.ctypes.data_as(C.POINTER(C.c_int)), int(v.size),
                                        self._p(prj), self._p(mask), self._p(out), self._stream(stream)))
        return out

    def volume_sat(self, vol, mask=None, stream=None):
        check(self.lib.ctlab_volume_sat(self.handle, self._p(vol), self._p(mask), self._stream(stream)))

    def sat_layout(self, orientation: int) -> tuple[int, int, int]:
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(self.lib.ctlab_plan_sat_layout(self.handle, orientation, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def copy_volume_sat(self, orientation: int, out, stream=None):
        check(self.lib.ctlab_copy_volume_sat(self.handle, orientation, self._p(out), self._stream(stream)))
        return out

    def os_sart(self, x, meas, mask=None, os_num: int = 24, iter_num: int = 30, lam: float = 1.0,
                order=None, clamp: bool = False, min_v: float = -2000.0, max_v: float = 6000.0,
                residuals: bool = False, stream=None):
        res = np.zeros(max(iter_num, 1), np.float32) if residuals else None
        o = None if order is None else np.ascontiguousarray(order, dtype=np.int32)
        check(self.lib.ctlab_os_sart(
            self.handle, self._p(x), self._p(meas), self._p(mask), os_num, iter_num, lam,
            None if o is None else o.ctypes.data_as(C.POINTER(C.c_int)), 1 if clamp else 0, min_v, max_v,
            None if res is None else res.ctypes.data_as(_fp), self._stream(stream)))
        return None if res is None else res[:iter_num]

    def cg(self, x, meas, mask=None, iter_num: int = 10, method: int = 0, residuals: bool = False, stream=None):
        """Conjugate gradient for min ||A x - b||^2 (ctlab_cg); method is a CTLAB_CG_* beta rule."""
        res = np.zeros(max(iter_num, 1), np.float32) if residuals else None
        check(self.lib.ctlab_cg(self.handle, self._p(x), self._p(meas), self._p(mask), iter_num, method,
                                None if res is None else res.ctypes.data_as(_fp), self._stream(stream)))
        return None if res is None else res[:iter_num]

    def fista_tv(self, x, meas, mask=None, iter_num: int = 50, tv_lambda: float = 1e-4, tv_eps: float = 1e-8,
                 min_v: float = -2000.0, max_v: float = 6000.0, residuals: bool = False, stream=None):
        res = np.zeros(max(iter_num, 1), np.float32) if residuals else None
        check(self.lib.ctlab_fista_tv(self.handle, self._p(x), self._p(meas), self._p(mask), iter_num, tv_lambda,
                                      tv_eps, min_v, max_v, None if res is None else res.ctypes.data_as(_fp),
                                      self._stream(stream)))
        return None if res is None else res[:iter_num]


def ellipsoid_phantom(out, g: DD3Geometry, ell: np.ndarray, clamp_nonneg: bool = True, stream=None):
    """Fills the device volume ``out`` with the point-sampled ellipsoid sum."""
    lib = load()
    e = np.ascontiguousarray(ell, dtype=np.float64).reshape(-1, 10)
    check(lib.ctlab_ellipsoid_phantom(out.data_ptr(), g.XN, g.YN, g.ZN, g.dx, g.dz, g.imgXCenter, g.imgYCenter,
                                      g.imgZCenter, e.ctypes.data_as(C.POINTER(C.c_double)), e.shape[0],
                                      1 if clamp_nonneg else 0, Plan._stream(stream)))
    return out


def random_ellipsoids(seed: int, half_x: float, half_y: float, half_z: float, n_min: int = 20,
                      n_max: int = 40, v_max: float = 0.03) -> np.ndarray:
    """Random-ellipsoid records drawn by the library (std::mt19937_64)."""
    lib = load()
    buf = np.zeros((n_max, 10), np.float64)
    n = lib.ctlab_random_ellipsoids(seed, n_min, n_max, half_x, half_y, half_z, v_max,
                                    buf.ctypes.data_as(C.POINTER(C.c_double)), n_max)
    if n < 0:
        check(-n)
    return buf[:n].copy()


class Batch:
    """Projects the scans of several z-prefix plans with one persistent launch
    (ctlab_batch_*), optionally replayed from a CUDA graph."""

    def __init__(self, plans):
        self.lib = load()
        self.plans = list(plans)
        arr = (C.c_void_p * len(self.plans))(*[p.handle for p in self.plans])
        h = C.c_void_p()
        check(self.lib.ctlab_batch_create(arr, len(self.plans), C.byref(h)))
        self.handle = h

    @property
    def voxel_views(self) -> int:
        return int(self.lib.ctlab_batch_voxel_views(self.handle))

    def proj(self, vols, outs, masks=None, graph: bool = False, stream=None):
        n = len(self.plans)
        V = (C.c_void_p * n)(*[v.data_ptr() for v in vols])
        O = (C.c_void_p * n)(*[o.data_ptr() for o in outs])
        M = None if masks is None else (C.c_void_p * n)(*[None if m is None else m.data_ptr() for m in masks])
        check(self.lib.ctlab_batch_proj(self.handle, V, M, O, 1 if graph else 0, Plan._stream(stream)))
        return outs

    def close(self):
        if getattr(self, "handle", None):
            self.lib.ctlab_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
