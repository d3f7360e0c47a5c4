"""ctypes binding of libctlab_b200.so (the C ABI declared in include/ctlab_b200.h).

The shared library is built in-tree (``ctlab_b200/libctlab_b200.so``) by
``ctlab_b200/build.py``.  Loading fails loudly when it is missing: there is no
CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libctlab_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "ctlab_b200.h")

CTLAB_OK = 0
CTLAB_ERR_INVALID_ARG = 1
CTLAB_ERR_UNSUPPORTED = 2
CTLAB_ERR_CUDA = 3
CTLAB_ERR_OOM = 4
CTLAB_ERR_TIMEOUT = 5
CTLAB_ERR_INTERNAL = 6
CTLAB_SAT_FP64 = 0
CTLAB_SAT_F32PAIR = 1
CTLAB_SAT_ZPREFIX = 2
CTLAB_CG_FR, CTLAB_CG_PRP, CTLAB_CG_CW, CTLAB_CG_DI, CTLAB_CG_DY = range(5)

_ERR_NAMES = {
    CTLAB_ERR_INVALID_ARG: "invalid argument",
    CTLAB_ERR_UNSUPPORTED: "unsupported",
    CTLAB_ERR_CUDA: "CUDA error",
    CTLAB_ERR_OOM: "out of device memory",
    CTLAB_ERR_TIMEOUT: "device wait timed out",
    CTLAB_ERR_INTERNAL: "internal error",
}


class CtlabError(RuntimeError):
    """Raised for a non-zero status of a library call."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{_ERR_NAMES.get(code, 'error')} ({code}): {message}")
        self.code = code
        self.message = message


class Geometry(C.Structure):
    _fields_ = [
        ("x0", C.c_float), ("y0", C.c_float), ("z0", C.c_float),
        ("DNU", C.c_int), ("DNV", C.c_int),
        ("xds", C.POINTER(C.c_float)), ("yds", C.POINTER(C.c_float)), ("zds", C.POINTER(C.c_float)),
        ("imgXCenter", C.c_float), ("imgYCenter", C.c_float), ("imgZCenter", C.c_float),
        ("hangs", C.POINTER(C.c_float)), ("hzPos", C.POINTER(C.c_float)),
        ("PN", C.c_int),
        ("XN", C.c_int), ("YN", C.c_int), ("ZN", C.c_int),
        ("dx", C.c_float), ("dz", C.c_float),
    ]


_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p
_u8p = C.c_void_p

# name -> (restype, argtypes)
_SIGNATURES = {
    "DD3Proj_gpu": (None, [C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, _fp, _fp, _fp,
                           C.c_float, C.c_float, C.c_float, _fp, _fp, C.c_int, C.c_int, C.c_int,
                           C.c_int, _fp, _fp, C.c_float, C.c_float, _u8p, C.c_int, C.c_int]),
    "DD3Back_gpu": (None, [C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, _fp, _fp, _fp,
                           C.c_float, C.c_float, C.c_float, _fp, _fp, C.c_int, C.c_int, C.c_int,
                           C.c_int, _fp, _fp, C.c_float, C.c_float, _u8p, C.c_int, C.c_int, C.c_int]),
    "DD3Proj_multiGPU": (None, [C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, _fp, _fp, _fp,
                                C.c_float, C.c_float, C.c_float, _fp, _fp, C.c_int, C.c_int, C.c_int,
                                C.c_int, _fp, _fp, C.c_float, C.c_float, _u8p, C.c_int, _ip, C.c_int]),
    "DD3Back_multiGPU": (None, [C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, _fp, _fp, _fp,
                                C.c_float, C.c_float, C.c_float, _fp, _fp, C.c_int, C.c_int, C.c_int,
                                C.c_int, _fp, _fp, C.c_float, C.c_float, _u8p, C.c_int, _ip, C.c_int]),
    "ctlab_slab_views": (C.c_int, [C.POINTER(Geometry), C.c_int, C.c_int, _ip, C.c_int]),
    "ctlab_proj_multi": (C.c_int, [C.POINTER(Geometry), _vp, _vp, _vp, _ip, C.c_int]),
    "ctlab_back_multi": (C.c_int, [C.POINTER(Geometry), _vp, _vp, _vp, _ip, C.c_int]),
    "ctlab_last_status": (C.c_int, []),
    "ctlab_last_error": (C.c_char_p, []),
    "ctlab_plan_create": (C.c_int, [C.POINTER(Geometry), C.c_int, C.c_int, C.POINTER(_vp)]),
    "ctlab_plan_destroy": (C.c_int, [_vp]),
    "ctlab_plan_workspace_bytes": (C.c_longlong, [_vp]),
    "ctlab_proj": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "ctlab_proj_views": (C.c_int, [_vp, _ip, C.c_int, _vp, _vp, _vp, _vp]),
    "ctlab_back": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "ctlab_back_views": (C.c_int, [_vp, _ip, C.c_int, _vp, _vp, _vp, _vp]),
    "ctlab_volume_sat": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ctlab_plan_sat_layout": (C.c_int, [_vp, C.c_int, _ip, _ip, _ip]),
    "ctlab_copy_volume_sat": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "ctlab_plan_set_timing": (C.c_int, [_vp, C.c_int]),
    "ctlab_plan_last_times": (C.c_int, [_vp, _fp, _fp]),
    "ctlab_plan_last_launches": (C.c_int, [_vp]),
    "ctlab_os_sart": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_float, _ip, C.c_int,
                                C.c_float, C.c_float, _fp, _vp]),
    "ctlab_fista_tv": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_float, C.c_float, C.c_float,
                                 C.c_float, _fp, _vp]),
    "ctlab_cg": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, _fp, _vp]),
    "ctlab_plan_autotune": (C.c_int, [_vp, _vp, _vp, C.c_char_p, _fp]),
    "ctlab_cnn_check": (C.c_int, [_vp]),
    "ctlab_plan_proj_tiles": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "ctlab_batch_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.POINTER(_vp)]),
    "ctlab_batch_destroy": (C.c_int, [_vp]),
    "ctlab_batch_voxel_views": (C.c_longlong, [_vp]),
    "ctlab_batch_proj": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.c_int, _vp]),
    "ctlab_cnn_conv": (C.c_int, [_vp, C.c_int, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp,
                                 _vp, _vp, _vp]),
    "ctlab_cnn_wgrad": (C.c_int, [_vp, C.c_int, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp]),
    "ctlab_cnn_pack": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, C.c_float, _vp, _vp, _vp, _vp,
                                 _vp]),
    "ctlab_cnn_unpack": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, C.c_float, _vp, _vp]),
    "ctlab_cnn_loss_grad": (C.c_int, [_vp, _vp, C.c_longlong, _vp, _vp, _vp]),
    "ctlab_cnn_adam": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                 C.c_int, _vp, _vp, _vp]),
    "ctlab_tv_gradient": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_float, _vp]),
    "ctlab_fista_step": (C.c_int, [_vp, _vp, C.c_float, C.c_float, C.c_longlong, C.c_float,
                                   C.c_float, _vp]),
    "ctlab_sart_proj_weight": (C.c_int, [_vp, _vp, _vp, C.c_longlong, _vp]),
    "ctlab_sart_back_weight": (C.c_int, [_vp, _vp, _vp, C.c_longlong, _vp]),
    "ctlab_ellipsoid_phantom": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                          C.c_float, C.c_float, C.c_float,
                                          C.POINTER(C.c_double), C.c_int, C.c_int, _vp]),
    "ctlab_debug_scan_stall": (C.c_int, [C.c_int, C.c_uint]),
    "ctlab_volume_sat_noalloc": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp]),
    "ctlab_noalloc_check": (C.c_int, [_vp]),
    "ctlab_debug_noalloc_stall": (C.c_int, [C.c_uint, _vp]),
    "ctlab_random_ellipsoids": (C.c_int, [C.c_ulonglong, C.c_int, C.c_int, C.c_float, C.c_float,
                                          C.c_float, C.c_float, C.POINTER(C.c_double), C.c_int]),
}

_lib = None


def header_symbols(path: str = HEADER_PATH) -> list[str]:
    """Function names declared in the public header."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", text, flags=re.M)
    return sorted({n for n in names if n not in ("if", "while", "for", "return")})


def load(path: str | None = None) -> C.CDLL:
    """Loads the library once and binds every declared entry point."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"{p} is missing: build it with `python -m ctlab_b200.build` (nvcc, sm_100a). "
            "There is no CPU fallback.")
    lib = C.CDLL(p)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != CTLAB_OK:
        msg = load().ctlab_last_error()
        raise CtlabError(rc, msg.decode() if msg else "")


def check_last() -> None:
    lib = load()
    rc = lib.ctlab_last_status()
    if rc != CTLAB_OK:
        raise CtlabError(rc, lib.ctlab_last_error().decode())
