"""Known-answer and identity checks that pin the oracle's DD3 core, whose
reference bodies are absent (src/DD3_GPU_Proj.h:41-44 declares only)."""
import math

import numpy as np
import pytest

import oracle
from ctlab_b200 import geometry as G


def test_sat2d_matches_cumsum():
    rng = np.random.default_rng(1)
    a = rng.random((7, 5))
    s = oracle.volume_sats(G.small(XN=7, YN=1, ZN=5), a.astype(np.float32).reshape(1, 7, 5))[0][0]
    ref = np.zeros((8, 6))
    ref[1:, 1:] = np.cumsum(np.cumsum(a.astype(np.float32).astype(np.float64), 0), 1)
    np.testing.assert_allclose(s, ref, rtol=1e-13, atol=1e-13)


def _uniform_case(start):
    return G.small(PN=8, XN=20, YN=20, ZN=10, DNU=48, DNV=12, dx=1.0, dz=1.0, col_size=0.6,
                   row_size=0.5, start=start)


@pytest.mark.parametrize("start", [0.0, math.pi / 2 + 0.05, 0.3])
def test_uniform_box_central_rays_equal_chord_length(start):
    g = _uniform_case(start)
    vol = np.ones(g.vol_shape, np.float32)
    p = oracle.dd3_proj(g, vol)
    # rays whose footprint stays inside the box in b and z on every slice:
    # DD sums exactly NA slabs of length dx*|d|/|d_a|, the chord through the
    # two faces of the driving axis.
    for k in range(g.PN):
        th = float(g.hangs[k]) % (2 * math.pi)
        c, s = math.cos(th), math.sin(th)
        S = np.array([-g.y0 * s, g.y0 * c, 0.0])
        xdrv = (math.pi / 4 <= th < 3 * math.pi / 4) or (5 * math.pi / 4 <= th < 7 * math.pi / 4)
        for u in (g.DNU // 2 - 1, g.DNU // 2):
            for v in (g.DNV // 2 - 1, g.DNV // 2):
                D = np.array([g.xds[u] * c - g.yds[u] * s, g.xds[u] * s + g.yds[u] * c, g.zds[v]])
                d = D - S
                ext = g.XN * g.dx if xdrv else g.YN * g.dx
                chord = ext * np.linalg.norm(d) / abs(d[0] if xdrv else d[1])
                assert abs(p[k, u, v] - chord) < 1e-7 * chord


def test_projection_converges_to_analytic_ellipsoid_integrals():
    errs = []
    for fac in (1, 2):
        g = G.small(PN=4, XN=16 * fac, YN=14 * fac, ZN=8 * fac, DNU=40, DNV=12, dx=1.5 / fac, dz=1.5 / fac,
                    col_size=0.9, row_size=0.9, start=0.2)
        hx, hy, hz = G.half_extents(g)
        ell = np.array([[0.02, 0.5, -0.3, 0.2, 0.7 * hx, 0.6 * hy, 0.6 * hz, 0.3, 0.2, 0.1]])
        p = oracle.dd3_proj(g, oracle.ellipsoid_phantom(g, ell))
        an = np.zeros_like(p)
        for k in range(g.PN):
            th = float(g.hangs[k])
            c, s = math.cos(th), math.sin(th)
            S = np.array([-g.y0 * s, g.y0 * c, 0.0])
            for u in range(g.DNU):
                for v in range(g.DNV):
                    D = np.array([g.xds[u] * c - g.yds[u] * s, g.xds[u] * s + g.yds[u] * c, g.zds[v]])
                    an[k, u, v] = oracle.ellipsoid_line_integral(ell, S, D)
        errs.append(np.linalg.norm(p - an) / np.linalg.norm(an))
    assert errs[0] < 0.2 and errs[1] < 0.6 * errs[0], errs


def test_backprojector_is_adjoint_of_projector():
    g = G.small(PN=12, XN=26, YN=22, ZN=10, DNU=44, DNV=14, start=0.1)
    rng = np.random.default_rng(3)
    x = rng.random(g.vol_shape).astype(np.float32)
    y = rng.random(g.prj_shape).astype(np.float32)
    mask = (rng.random(g.XN * g.YN) > 0.2).astype(np.uint8)
    a = float((oracle.dd3_proj(g, x, mask) * y).sum())
    b = float((x * oracle.dd3_back(g, y, mask)).sum())
    assert abs(a - b) / abs(a) < 1e-5


def test_rotating_the_volume_by_90_degrees_shifts_the_view():
    # volume rotated by +90 deg about z seen at theta equals the original seen
    # at theta - 90 deg; exercises the x-driven and y-driven paths against
    # each other (the driving axis swaps between the two).
    n = 18
    base = G.small(PN=1, XN=n, YN=n, ZN=8, DNU=36, DNV=10, start=0.2)
    rng = np.random.default_rng(5)
    vol = rng.random(base.vol_shape).astype(np.float32)  # [y][x][z]
    # rotation by +90: new(x', y') = old(x, y) with x' = -y, y' = x
    # new[y'][x'] = old[y = -x'][x = y']
    rot = np.empty_like(vol)
    for yp in range(n):
        for xp in range(n):
            rot[yp, xp] = vol[n - 1 - xp, yp]
    g1 = base.with_views([0])
    g1.hangs[:] = 0.2 + math.pi / 2
    p_rot = oracle.dd3_proj(g1, rot)
    g0 = base.with_views([0])
    g0.hangs[:] = 0.2
    p0 = oracle.dd3_proj(g0, vol)
    # the two angles are float32 values 90 degrees apart only to ~1e-7 rad
    np.testing.assert_allclose(p_rot, p0, rtol=2e-5, atol=1e-6 * p0.max())


def test_row_and_column_sums_positive_inside_fov():
    g = G.small(PN=8, start=0.1)
    rows = oracle.dd3_proj(g, np.ones(g.vol_shape, np.float32))
    cols = oracle.dd3_back(g, np.ones(g.prj_shape, np.float32))
    assert rows.max() > 0 and np.all(rows >= 0)
    assert np.all(cols > 0)


def test_config2_switch_views_sit_on_both_sides_of_each_hand_over():
    """The hand-over views of the config-2 parity case (GPU test) straddle every
    x/y-driven switch angle after float32 rounding: just below, on, just above pi/4,
    3pi/4, 5pi/4, 7pi/4 (float32(5pi/4) and float32(7pi/4) round below the angle)."""
    from test_gpu_parity_configs import config2_switch_geometry
    lib = oracle.load()
    g = config2_switch_geometry()
    xd = [lib.orc_view_is_xdriven(lib.orc_regularize_angle(float(a))) for a in g.hangs]
    assert xd[24:] == [0, 1, 1, 1, 0, 0, 0, 0, 1, 1, 1, 0]
