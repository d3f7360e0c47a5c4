"""ctlab_b200: CTLAB's branchless DD3 cone-beam projector, backprojector and
OS-SART / FISTA-TV loops on NVIDIA B200 (sm_100a).

The compute path is libctlab_b200.so (hand-written CUDA behind a C ABI,
include/ctlab_b200.h); this package is its Python host side.
"""
from ._lib import (CTLAB_ERR_CUDA, CTLAB_ERR_INTERNAL, CTLAB_ERR_INVALID_ARG, CTLAB_ERR_OOM,
                   CTLAB_ERR_TIMEOUT, CTLAB_ERR_UNSUPPORTED, CTLAB_OK, CTLAB_SAT_F32PAIR,
                   CTLAB_SAT_FP64, CTLAB_SAT_ZPREFIX, CtlabError, load)
from .dd3 import (Batch, DD3Back_gpu, DD3Back_multiGPU, DD3Proj_gpu, DD3Proj_multiGPU, Plan, back,
                  ellipsoid_phantom, proj, random_ellipsoids, slab_geometry, slab_views)
from .geometry import DD3Geometry, config1, config2, config3, shepp_logan_ellipsoids, small
from .multi import DistributedPlan, ViewSplit

__all__ = [
    "CTLAB_OK", "CTLAB_ERR_INVALID_ARG", "CTLAB_ERR_UNSUPPORTED", "CTLAB_ERR_CUDA", "CTLAB_ERR_OOM",
    "CTLAB_ERR_TIMEOUT", "CTLAB_ERR_INTERNAL", "CTLAB_SAT_FP64", "CTLAB_SAT_F32PAIR", "CTLAB_SAT_ZPREFIX",
    "CtlabError",
    "load", "DD3Proj_gpu", "DD3Back_gpu", "DD3Proj_multiGPU", "DD3Back_multiGPU", "slab_views", "slab_geometry", "Plan", "Batch", "proj", "back", "ellipsoid_phantom",
    "random_ellipsoids", "DD3Geometry", "config1", "config2", "config3", "small",
    "shepp_logan_ellipsoids", "DistributedPlan", "ViewSplit",
]
