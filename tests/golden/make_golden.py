"""Generates tests/golden/ref_helpers.npz from the reference's own header-inline
helpers compiled where they lie (oracle/_ref/libctlab_ref_helpers.so, built by
`make -C oracle ref` from the reference tree).  Run in a container that has the
reference checkout; the committed .npz is what the tests read.

Covers: DD3Boundaries (float and double, src/utilities.cuh:413-433),
regularizeAngle (:279-286), invRotVox (:289-298), SART_Weighting::Proj_ptr /
Back_ptr (src/SARTWeighting.h:38-91), FISTA (src/FastIterativeShrinkageAlgorithm.h:44-48),
_Update (src/utilities.hpp:1062-1094) and prjWeight / bakWeight (:4304-4405).
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

fp = C.POINTER(C.c_float)
dp = C.POINTER(C.c_double)


def main() -> None:
    oracle.build(ref=True)
    lib = C.CDLL(oracle.REF_LIB)
    rng = np.random.default_rng(20240607)
    out = {}

    # DD3Boundaries: uniform, non-uniform, 2 cells, 1 cell
    cases = [np.linspace(-3.3, 4.1, 9), np.sort(rng.normal(size=13)) * 7.0, np.array([0.25, 1.5]),
             np.array([2.75])]
    for i, c in enumerate(cases):
        cf = c.astype(np.float32)
        bf = np.zeros(cf.size + 1, np.float32)
        lib.ref_dd3_boundaries_f(cf.size + 1, cf.ctypes.data_as(fp), bf.ctypes.data_as(fp))
        cd = c.astype(np.float64)
        bd = np.zeros(cd.size + 1)
        lib.ref_dd3_boundaries_d(cd.size + 1, cd.ctypes.data_as(dp), bd.ctypes.data_as(dp))
        out[f"bnd{i}_c"] = c
        out[f"bnd{i}_f"] = bf
        out[f"bnd{i}_d"] = bd

    # regularizeAngle
    angs = np.concatenate([rng.uniform(-20, 20, 64), [0.0, 6.283185307179586, -1e-9, 12.566370614359172]])
    lib.ref_regularize_angle_d.restype = C.c_double
    lib.ref_regularize_angle_d.argtypes = [C.c_double]
    lib.ref_regularize_angle_f.restype = C.c_float
    lib.ref_regularize_angle_f.argtypes = [C.c_float]
    out["ang_in"] = angs
    out["ang_d"] = np.array([lib.ref_regularize_angle_d(a) for a in angs])
    out["ang_f"] = np.array([lib.ref_regularize_angle_f(np.float32(a)) for a in angs], np.float32)

    # invRotVox
    vox = rng.normal(size=(16, 3)).astype(np.float32) * 50
    th = rng.uniform(0, 6.28, 16)
    zp = rng.normal(size=16).astype(np.float32)
    lib.ref_inv_rot_vox.argtypes = [fp, fp, C.c_float, C.c_float, C.c_float]
    rot = np.zeros_like(vox)
    for i in range(16):
        o = np.zeros(3, np.float32)
        lib.ref_inv_rot_vox(vox[i].ctypes.data_as(fp), o.ctypes.data_as(fp), np.float32(np.cos(th[i])),
                            np.float32(np.sin(th[i])), zp[i])
        rot[i] = o
    out.update(rot_in=vox, rot_th=th, rot_zp=zp, rot_out=rot)

    # SART weightings (epsilon 1e-7) with rowSum / colSum around the threshold
    n = 257
    prj = rng.normal(size=n).astype(np.float32)
    real = rng.normal(size=n).astype(np.float32)
    rs = np.abs(rng.normal(size=n)).astype(np.float32)
    rs[::7] = 0.0
    rs[3::11] = 1e-8
    rs[5::13] = 2e-7
    o_prj = prj.copy()
    lib.ref_sart_proj_ptr(o_prj.ctypes.data_as(fp), real.ctypes.data_as(fp), rs.ctypes.data_as(fp), n)
    vol = rng.normal(size=n).astype(np.float32)
    rec = rng.normal(size=n).astype(np.float32)
    o_vol, o_rec = vol.copy(), rec.copy()
    lib.ref_sart_back_ptr(o_vol.ctypes.data_as(fp), o_rec.ctypes.data_as(fp), rs.ctypes.data_as(fp), n)
    out.update(sart_prj=prj, sart_real=real, sart_rs=rs, sart_prj_out=o_prj, sart_vol=vol, sart_rec=rec,
               sart_vol_out=o_vol, sart_rec_out=o_rec)

    # prjWeight / bakWeight of utilities.hpp (epsilon 1e-9)
    o2 = prj.copy()
    lib.ref_prj_weight(o2.ctypes.data_as(fp), real.ctypes.data_as(fp), rs.ctypes.data_as(fp), n)
    v2, r2 = vol.copy(), rec.copy()
    lib.ref_bak_weight(v2.ctypes.data_as(fp), r2.ctypes.data_as(fp), rs.ctypes.data_as(fp), n)
    out.update(pw_out=o2, bw_vol_out=v2, bw_rec_out=r2)

    # FISTA with clamp
    las = rng.normal(size=n).astype(np.float32) * 3000
    cur = rng.normal(size=n).astype(np.float32) * 3000
    lib.ref_fista.argtypes = [fp, fp, C.c_float, C.c_float, C.c_int, C.c_float, C.c_float]
    fo = cur.copy()
    lib.ref_fista(las.ctypes.data_as(fp), fo.ctypes.data_as(fp), 2.3, 2.9, n, -2000.0, 6000.0)
    out.update(fista_las=las, fista_cur=cur, fista_out=fo, fista_t=np.array([2.3, 2.9, -2000.0, 6000.0]))

    # _Update (relaxation, mask, optional range)
    img = rng.normal(size=n).astype(np.float32)
    cor = rng.normal(size=n).astype(np.float32)
    weg = np.abs(rng.normal(size=n)).astype(np.float32) + 0.1
    msk = (rng.random(n) > 0.3).astype(np.float32)
    lib.ref_update.argtypes = [fp, fp, fp, fp, C.c_int, C.c_float, C.c_int, C.c_float, C.c_float]
    u0, u1 = img.copy(), img.copy()
    lib.ref_update(u0.ctypes.data_as(fp), cor.ctypes.data_as(fp), weg.ctypes.data_as(fp), msk.ctypes.data_as(fp),
                   n, 0.7, 0, 0.0, 0.0)
    lib.ref_update(u1.ctypes.data_as(fp), cor.ctypes.data_as(fp), weg.ctypes.data_as(fp), msk.ctypes.data_as(fp),
                   n, 0.7, 1, -0.5, 0.5)
    out.update(upd_img=img, upd_cor=cor, upd_weg=weg, upd_msk=msk, upd_out=u0, upd_out_clamp=u1)

    np.savez_compressed(os.path.join(HERE, "ref_helpers.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_helpers.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
