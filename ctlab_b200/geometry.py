"""Scan geometries and phantoms used by the tests and the benchmark.

A :class:`DD3Geometry` carries exactly the scalar and array arguments of the
reference's ``DD3Proj_gpu`` / ``DD3Back_gpu`` (src/DD3_GPU_Proj.h:41-44):
source start (x0, y0, z0), detector cell centres (xds, yds, zds), image
centre, view angles and z positions, volume size and voxel sizes.

``flat`` builds the flat equal-distance detector of the reference's OS_SART
driver (src/DD3_GPU_recon.h:60-65): source at (0, sid, 0), detector plane at
y = sid - sdd, cells ``(u - (DNU-1)/2 - col_offset) * col_size`` and
``(v - (DNV-1)/2 - row_offset) * row_size`` -- the convention of calSVASVB,
src/utilities.hpp:3322-3348 (source at (0, S2O), detector at y = -O2D).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class DD3Geometry:
    x0: float
    y0: float
    z0: float
    xds: np.ndarray
    yds: np.ndarray
    zds: np.ndarray
    imgXCenter: float
    imgYCenter: float
    imgZCenter: float
    hangs: np.ndarray
    hzPos: np.ndarray
    XN: int
    YN: int
    ZN: int
    dx: float
    dz: float

    def __post_init__(self):
        for f in ("xds", "yds", "zds", "hangs", "hzPos"):
            setattr(self, f, np.ascontiguousarray(getattr(self, f), dtype=np.float32))

    @property
    def DNU(self) -> int:
        return int(self.xds.size)

    @property
    def DNV(self) -> int:
        return int(self.zds.size)

    @property
    def PN(self) -> int:
        return int(self.hangs.size)

    @property
    def vol_shape(self) -> tuple[int, int, int]:
        """numpy shape of a (Z,X,Y)-ordered volume: [YN][XN][ZN]."""
        return (self.YN, self.XN, self.ZN)

    @property
    def prj_shape(self) -> tuple[int, int, int]:
        return (self.PN, self.DNU, self.DNV)

    @property
    def voxel_views(self) -> int:
        return self.XN * self.YN * self.ZN * self.PN

    def args(self) -> dict:
        """Keyword arguments in the reference's names."""
        return dict(x0=self.x0, y0=self.y0, z0=self.z0, DNU=self.DNU, DNV=self.DNV,
                    xds=self.xds, yds=self.yds, zds=self.zds, imgXCenter=self.imgXCenter,
                    imgYCenter=self.imgYCenter, imgZCenter=self.imgZCenter, hangs=self.hangs,
                    hzPos=self.hzPos, PN=self.PN, XN=self.XN, YN=self.YN, ZN=self.ZN,
                    dx=self.dx, dz=self.dz)

    def with_views(self, idx) -> "DD3Geometry":
        idx = np.asarray(idx)
        return dataclasses.replace(self, hangs=self.hangs[idx].copy(), hzPos=self.hzPos[idx].copy())

    @staticmethod
    def flat(*, sid: float, sdd: float, DNU: int, DNV: int, col_size: float, row_size: float,
             PN: int, XN: int, YN: int, ZN: int, dx: float, dz: float, col_offset: float = 0.0,
             row_offset: float = 0.0, angles=None, zpos=None, center=(0.0, 0.0, 0.0)) -> "DD3Geometry":
        u = np.arange(DNU, dtype=np.float64)
        v = np.arange(DNV, dtype=np.float64)
        xds = (u - (DNU - 1) / 2.0 - col_offset) * col_size
        yds = np.full(DNU, sid - sdd)
        zds = (v - (DNV - 1) / 2.0 - row_offset) * row_size
        if angles is None:
            angles = 2.0 * math.pi * np.arange(PN) / PN
        if zpos is None:
            zpos = np.zeros(PN)
        return DD3Geometry(0.0, float(sid), 0.0, xds, yds, zds, float(center[0]), float(center[1]),
                           float(center[2]), np.asarray(angles), np.asarray(zpos), XN, YN, ZN,
                           float(dx), float(dz))


SOD = 541.0
SDD = 949.0


def config1() -> DD3Geometry:
    """128x128x64 at 0.5 mm, 360 views, 256x64 detector of 1.0 mm cells."""
    return DD3Geometry.flat(sid=SOD, sdd=SDD, DNU=256, DNV=64, col_size=1.0, row_size=1.0, PN=360,
                            XN=128, YN=128, ZN=64, dx=0.5, dz=0.5)


def config2() -> DD3Geometry:
    """512x512x256 (dx 1.0, dz 0.15625 mm), 984 views, 888x64 detector of 1.0239x1.0960 mm."""
    return DD3Geometry.flat(sid=SOD, sdd=SDD, DNU=888, DNV=64, col_size=1.0239, row_size=1.0960,
                            PN=984, XN=512, YN=512, ZN=256, dx=1.0, dz=0.15625)


def config3() -> DD3Geometry:
    """256x256x128 at 0.5 mm, 720 views, 384x128 detector of 1.0 mm cells."""
    return DD3Geometry.flat(sid=SOD, sdd=SDD, DNU=384, DNV=128, col_size=1.0, row_size=1.0, PN=720,
                            XN=256, YN=256, ZN=128, dx=0.5, dz=0.5)


def helical(XN: int = 512, YN: int = 512, ZN: int = 1024, dz: float = 0.5, views_per_turn: int = 984,
            pitch: float = 1.0) -> DD3Geometry:
    """Helical scan of a long volume (1 mm in-plane voxels, dz along z) with the 888x64
    detector of config 2: the source advances pitch x the detector's z coverage at the
    isocentre per turn, over the volume's z extent plus one coverage."""
    DNU, DNV, col, row = 888, 64, 1.0239, 1.0960
    coverage = DNV * row * SOD / SDD
    span = ZN * dz + coverage
    turns = math.ceil(span / (pitch * coverage))
    PN = turns * views_per_turn
    angles = 2.0 * math.pi * np.arange(PN) / views_per_turn
    zpos = np.linspace(-0.5 * span, 0.5 * span, PN)
    return DD3Geometry.flat(sid=SOD, sdd=SDD, DNU=DNU, DNV=DNV, col_size=col, row_size=row, PN=PN,
                            XN=XN, YN=YN, ZN=ZN, dx=1.0, dz=dz, angles=angles, zpos=zpos)


def config4(seed: int = 7, n: int = 48) -> list[DD3Geometry]:
    """The uneven batch: n scans with volumes from {128^3, 192x192x96, 256x256x64,
    384x384x32} (1 mm voxels), 180-720 views, detectors 256-768 cells wide and 32-64
    rows; cell sizes chosen so the detector covers the volume (10 % margin)."""
    rng = np.random.default_rng(seed)
    vols = [(128, 128, 128), (192, 192, 96), (256, 256, 64), (384, 384, 32)]
    out = []
    for _ in range(n):
        XN, YN, ZN = vols[int(rng.integers(len(vols)))]
        PN = int(rng.integers(180, 721))
        DNU = int(rng.integers(256, 769))
        DNV = int(rng.integers(32, 65))
        mag = SDD / SOD
        col = 1.1 * XN * math.sqrt(2.0) * mag / DNU
        row = 1.1 * ZN * mag / DNV
        out.append(DD3Geometry.flat(sid=SOD, sdd=SDD, DNU=DNU, DNV=DNV, col_size=col, row_size=row, PN=PN,
                                    XN=XN, YN=YN, ZN=ZN, dx=1.0, dz=1.0))
    return out


def small(PN: int = 24, XN: int = 24, YN: int = 20, ZN: int = 12, DNU: int = 40, DNV: int = 14,
          dx: float = 0.5, dz: float = 0.5, col_size: float = 0.9, row_size: float = 0.8,
          col_offset: float = 0.0, row_offset: float = 0.0, start: float = 0.0,
          zpos=None, center=(0.0, 0.0, 0.0)) -> DD3Geometry:
    """Small odd-sized scan for oracle-vs-GPU parity (seconds on the CPU)."""
    angles = start + 2.0 * math.pi * np.arange(PN) / PN
    return DD3Geometry.flat(sid=SOD, sdd=SDD, DNU=DNU, DNV=DNV, col_size=col_size,
                            row_size=row_size, PN=PN, XN=XN, YN=YN, ZN=ZN, dx=dx, dz=dz,
                            col_offset=col_offset, row_offset=row_offset, angles=angles,
                            zpos=zpos, center=center)


# 3-D modified Shepp-Logan head phantom, 10 ellipsoids, in units of the
# phantom half-extent: value, centre (x, y, z), semi-axes (a, b, c), rotation
# phi about z (degrees).  Intensities of the "modified" (contrast-enhanced)
# variant; literature values (Kak & Slaney's 3-D extension of Shepp-Logan).
_MODIFIED_SHEPP_LOGAN_3D = np.array([
    # val    x0      y0      z0      a       b       c      phi
    [1.0,   0.0,    0.0,    0.0,   0.69,   0.92,   0.81,    0.0],
    [-0.8,  0.0,  -0.0184,  0.0,   0.6624, 0.874,  0.78,    0.0],
    [-0.2,  0.22,   0.0,    0.0,   0.11,   0.31,   0.22,  -18.0],
    [-0.2, -0.22,   0.0,    0.0,   0.16,   0.41,   0.28,   18.0],
    [0.1,   0.0,    0.35,  -0.15,  0.21,   0.25,   0.41,    0.0],
    [0.1,   0.0,    0.1,    0.25,  0.046,  0.046,  0.05,    0.0],
    [0.1,   0.0,   -0.1,    0.25,  0.046,  0.046,  0.05,    0.0],
    [0.1,  -0.08,  -0.605,  0.0,   0.046,  0.023,  0.05,    0.0],
    [0.1,   0.0,   -0.606,  0.0,   0.023,  0.023,  0.02,    0.0],
    [0.1,   0.06,  -0.605,  0.0,   0.023,  0.046,  0.02,    0.0],
])


def shepp_logan_ellipsoids(half_x: float, half_y: float, half_z: float,
                           max_value: float = 0.02) -> np.ndarray:
    """Ellipsoid records (10 doubles each, see ctlab_ellipsoid_phantom) of
    the 3-D modified Shepp-Logan phantom scaled to the half extents, values
    scaled so the phantom lies in [0, max_value]."""
    t = _MODIFIED_SHEPP_LOGAN_3D
    out = np.zeros((t.shape[0], 10))
    out[:, 0] = t[:, 0] * max_value
    out[:, 1] = t[:, 1] * half_x
    out[:, 2] = t[:, 2] * half_y
    out[:, 3] = t[:, 3] * half_z
    out[:, 4] = t[:, 4] * half_x
    out[:, 5] = t[:, 5] * half_y
    out[:, 6] = t[:, 6] * half_z
    out[:, 7] = np.deg2rad(t[:, 7])
    return out


def half_extents(g: DD3Geometry) -> tuple[float, float, float]:
    return 0.5 * g.XN * g.dx, 0.5 * g.YN * g.dx, 0.5 * g.ZN * g.dz
