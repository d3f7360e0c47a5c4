// Host-side geometry: validation, detector boundaries and per-view constants,
// all in FP64.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdarg>
#include <cstring>

#include "internal.h"

namespace ctlab {

namespace {

// Quadrant limits of the driving-axis choice (the PI_4 .. PI_7_4 constants
// of src/utilities.cuh:39-48).
constexpr double kPi4 = 0.785398163397448;
constexpr double kPi34 = 2.356194490192344;
constexpr double kPi54 = 3.926990816987241;
constexpr double kPi74 = 5.497787143782138;
constexpr double kTwoPi = 6.283185307179586;

// Angle into [0, 2pi); regularizeAngle, src/utilities.cuh:279-286.
double regularize(double a)
{
    while (a >= kTwoPi) a -= kTwoPi;
    while (a < 0) a += kTwoPi;
    return a;
}

// Cell centres -> N+1 boundaries; DD3Boundaries, src/utilities.cuh:413-433.
void boundaries(const std::vector<double> &c, std::vector<double> &b)
{
    const size_t n = c.size();
    b.resize(n + 1);
    if (n >= 2) {
        b[0] = 1.5 * c[0] - 0.5 * c[1];
        for (size_t i = 1; i < n; ++i) b[i] = 0.5 * c[i - 1] + 0.5 * c[i];
        b[n] = 1.5 * c[n - 1] - 0.5 * c[n - 2];
    } else {
        b[0] = c[0] - 0.5;
        b[1] = c[0] + 0.5;
    }
}

bool finite_all(const float *p, int n)
{
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

int bad(const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return set_status(CTLAB_ERR_INVALID_ARG, buf);
}

} // namespace

int build_geometry(const ctlab_geometry &g, HostGeometry &o)
{
    if (g.DNU < 1 || g.DNV < 1 || g.PN < 1 || g.XN < 1 || g.YN < 1 || g.ZN < 1)
        return bad("sizes must be >= 1 (DNU=%d DNV=%d PN=%d XN=%d YN=%d ZN=%d)", g.DNU, g.DNV,
                   g.PN, g.XN, g.YN, g.ZN);
    if (!(g.dx > 0) || !(g.dz > 0) || !std::isfinite(g.dx) || !std::isfinite(g.dz))
        return bad("voxel sizes must be finite and > 0 (dx=%g dz=%g)", g.dx, g.dz);
    if (!g.xds || !g.yds || !g.zds || !g.hangs || !g.hzPos)
        return bad("null geometry array (xds/yds/zds/hangs/hzPos)");
    const double nvox = (double)g.XN * g.YN * g.ZN;
    const double nbin = (double)g.PN * g.DNU * g.DNV;
    if (nvox > 4.0e11 || nbin > 4.0e11) return bad("volume or projection too large");
    if (g.DNU > 65536 || g.DNV > 4096 || g.ZN > 16384 || g.XN > 65536 || g.YN > 65536)
        return bad("dimension beyond the supported range (DNU<=65536, DNV<=4096, ZN<=16384)");
    if (!finite_all(g.xds, g.DNU) || !finite_all(g.yds, g.DNU) || !finite_all(g.zds, g.DNV) ||
        !finite_all(g.hangs, g.PN) || !finite_all(g.hzPos, g.PN))
        return bad("non-finite value in a geometry array");
    if (!std::isfinite(g.x0) || !std::isfinite(g.y0) || !std::isfinite(g.z0) ||
        !std::isfinite(g.imgXCenter) || !std::isfinite(g.imgYCenter) || !std::isfinite(g.imgZCenter))
        return bad("non-finite source position or image centre");

    o.x0 = g.x0; o.y0 = g.y0; o.z0 = g.z0;
    o.DNU = g.DNU; o.DNV = g.DNV; o.PN = g.PN;
    o.XN = g.XN; o.YN = g.YN; o.ZN = g.ZN;
    o.cx = g.imgXCenter; o.cy = g.imgYCenter; o.cz = g.imgZCenter;
    o.dx = g.dx; o.dz = g.dz;
    o.x_lo = o.cx - 0.5 * o.XN * o.dx;
    o.y_lo = o.cy - 0.5 * o.YN * o.dx;
    o.z_lo = o.cz - 0.5 * o.ZN * o.dz;

    o.ux.assign(g.xds, g.xds + g.DNU);
    o.uy.assign(g.yds, g.yds + g.DNU);
    o.vz.assign(g.zds, g.zds + g.DNV);
    boundaries(o.ux, o.bx);
    boundaries(o.uy, o.by);
    boundaries(o.vz, o.bz);

    // flat detector with uniform pitch?
    {
        const double ex = (o.bx[g.DNU] - o.bx[0]) / g.DNU, ey = (o.by[g.DNU] - o.by[0]) / g.DNU;
        const double pitch = std::hypot(ex, ey);
        const double ez = (o.bz[g.DNV] - o.bz[0]) / g.DNV;
        bool flat = pitch > 0 && ez != 0;
        for (int q = 0; q <= g.DNU && flat; ++q)
            if (std::hypot(o.bx[0] + q * ex - o.bx[q], o.by[0] + q * ey - o.by[q]) > 1e-4 * pitch)
                flat = false;
        for (int w = 0; w <= g.DNV && flat; ++w)
            if (std::fabs(o.bz[0] + w * ez - o.bz[w]) > 1e-4 * std::fabs(ez)) flat = false;
        o.flat_uniform = flat;
        o.dzb = ez;
    }

    o.views.resize(g.PN);
    o.angle.resize(g.PN);
    for (int p = 0; p < g.PN; ++p) o.angle[p] = (double)g.hangs[p];
    for (int p = 0; p < g.PN; ++p) {
        DevView &v = o.views[p];
        std::memset(&v, 0, sizeof v);
        const double th = regularize((double)g.hangs[p]);
        v.c = std::cos(th);
        v.s = std::sin(th);
        v.zP = g.hzPos[p];
        v.Sx = o.x0 * v.c - o.y0 * v.s;
        v.Sy = o.x0 * v.s + o.y0 * v.c;
        v.Sz = o.z0 + v.zP;
        v.xdrv = ((th >= kPi4 && th < kPi34) || (th >= kPi54 && th < kPi74)) ? 1 : 0;
        if (v.xdrv) {
            v.Sa = v.Sx; v.Sb = v.Sy;
            v.na = o.XN; v.nb = o.YN;
            v.a0 = o.cx - 0.5 * (o.XN - 1) * o.dx;
            v.b_lo = o.y_lo;
        } else {
            v.Sa = v.Sy; v.Sb = v.Sx;
            v.na = o.YN; v.nb = o.XN;
            v.a0 = o.cy - 0.5 * (o.YN - 1) * o.dx;
            v.b_lo = o.x_lo;
        }
        const double bx0 = o.bx[0], by0 = o.by[0];
        const double ex = (o.bx[g.DNU] - o.bx[0]) / g.DNU, ey = (o.by[g.DNU] - o.by[0]) / g.DNU;
        v.B0x = bx0 * v.c - by0 * v.s;
        v.B0y = bx0 * v.s + by0 * v.c;
        v.Ex = ex * v.c - ey * v.s;
        v.Ey = ex * v.s + ey * v.c;

        // The source must lie outside the volume's extent along the driving
        // axis, and every detector boundary / centre on a ray that crosses it.
        const double a_lo = v.a0 - 0.5 * o.dx, a_hi = a_lo + v.na * o.dx;
        if (v.Sa >= a_lo && v.Sa <= a_hi)
            return bad("view %d: source lies inside the volume's extent along the driving axis", p);
        for (int q = 0; q <= g.DNU; ++q) {
            const double wx = o.bx[q] * v.c - o.by[q] * v.s, wy = o.bx[q] * v.s + o.by[q] * v.c;
            const double wa = v.xdrv ? wx : wy;
            if ((wa - v.Sa) * (0.5 * (a_lo + a_hi) - v.Sa) <= 0)
                return bad("view %d: detector boundary %d is not across the volume from the source", p, q);
        }
    }
    return ok();
}

std::vector<double> det_table_host(const HostGeometry &g)
{
    DetTable t = det_table_layout(g.DNU, g.DNV);
    std::vector<double> h(t.total);
    std::copy(g.bx.begin(), g.bx.end(), h.begin() + t.off_bx);
    std::copy(g.by.begin(), g.by.end(), h.begin() + t.off_by);
    std::copy(g.ux.begin(), g.ux.end(), h.begin() + t.off_ux);
    std::copy(g.uy.begin(), g.uy.end(), h.begin() + t.off_uy);
    std::copy(g.bz.begin(), g.bz.end(), h.begin() + t.off_bz);
    std::copy(g.vz.begin(), g.vz.end(), h.begin() + t.off_vz);
    return h;
}

std::vector<std::vector<int>> view_runs(const HostGeometry &g, const std::vector<int> &list)
{
    std::vector<std::vector<int>> runs;
    for (int axis = 0; axis < 2; ++axis) {
        std::vector<std::pair<double, int>> ang;
        for (int pos = 0; pos < (int)list.size(); ++pos) {
            const DevView &V = g.views[list[pos]];
            if (V.xdrv != axis) continue;
            // the angle as given: views of different helical turns (different
            // source z) at the same angle mod 2 pi are not neighbours
            ang.push_back({g.angle[list[pos]], pos});
        }
        if (ang.empty()) continue;
        std::stable_sort(ang.begin(), ang.end(),
                         [](const std::pair<double, int> &a, const std::pair<double, int> &b) { return a.first < b.first; });
        // a gap wider than 4x the median spacing starts a new run
        std::vector<double> gaps;
        for (size_t i = 1; i < ang.size(); ++i) gaps.push_back(ang[i].first - ang[i - 1].first);
        double med = 0.0;
        if (!gaps.empty()) {
            std::vector<double> s2 = gaps;
            std::nth_element(s2.begin(), s2.begin() + s2.size() / 2, s2.end());
            med = s2[s2.size() / 2];
        }
        std::vector<int> cur{ang[0].second};
        for (size_t i = 1; i < ang.size(); ++i) {
            if (gaps[i - 1] > 4.0 * med + 1e-12) {
                runs.push_back(cur);
                cur.clear();
            }
            cur.push_back(ang[i].second);
        }
        runs.push_back(cur);
    }
    return runs;
}

} // namespace ctlab
