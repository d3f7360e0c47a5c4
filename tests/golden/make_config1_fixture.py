"""Generates the pinned FP64 oracle fixture of the config-1 parity scan (128x128x64
volume at 0.5 mm holding the 3-D modified Shepp-Logan phantom, 360 views over 360
degrees, 256x64 detector of 1.0 mm cells, SOD 541 / SDD 949 mm):

  config1_oracle.json      SHA-256 of the raw little-endian float64 bytes of the whole
                           oracle projection [360][256][64] and of the oracle
                           backprojection [128][128][64] of that projection rounded to
                           float32, plus norms and sums
  config1_proj_views.f64   raw float64 projection of views 0 (y-driven) and 45
                           (theta = pi/4, the first x-driven angle) [2][256][64]
  config1_back_slice.f64   raw float64 backprojection, slice z = 32 [128][128]

The oracle's arithmetic is deterministic (every output is one thread's sequential
FP64 sum, compiled with -ffp-contract=off), so the hashes pin it exactly on this
image: tests/test_oracle_fixture.py regenerates both outputs and compares.

  python tests/golden/make_config1_fixture.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from ctlab_b200 import geometry as G  # noqa: E402  (pure Python: geometry records only)

VIEWS = (0, 45)
SLICE = 32


def config1_outputs():
    g = G.config1()
    hx, hy, hz = G.half_extents(g)
    vol = oracle.ellipsoid_phantom(g, G.shepp_logan_ellipsoids(hx, hy, hz))
    prj = oracle.dd3_proj(g, vol)
    back = oracle.dd3_back(g, prj.astype(np.float32))
    return g, vol, prj, back


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def summary(vol, prj, back) -> dict:
    return {
        "scan": "config1: 128x128x64 @0.5 mm, Shepp-Logan 3-D modified (0..0.02/mm), 360 views, 256x64 @1.0 mm",
        "volume_sha256_f32": hashlib.sha256(np.ascontiguousarray(vol, "<f4").tobytes()).hexdigest(),
        "proj_shape": list(prj.shape), "proj_sha256_f64": sha(prj),
        "proj_l2": float(np.linalg.norm(prj)), "proj_sum": float(prj.sum()),
        "back_shape": list(back.shape), "back_sha256_f64": sha(back),
        "back_l2": float(np.linalg.norm(back)), "back_sum": float(back.sum()),
        "views": list(VIEWS), "slice": SLICE,
    }


def main() -> None:
    _, vol, prj, back = config1_outputs()
    with open(os.path.join(HERE, "config1_oracle.json"), "w") as f:
        json.dump(summary(vol, prj, back), f, indent=1)
        f.write("\n")
    np.ascontiguousarray(prj[list(VIEWS)], "<f8").tofile(os.path.join(HERE, "config1_proj_views.f64"))
    np.ascontiguousarray(back[:, :, SLICE], "<f8").tofile(os.path.join(HERE, "config1_back_slice.f64"))


if __name__ == "__main__":
    main()
