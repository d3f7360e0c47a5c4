/*
 * dd3_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement, in FP64, of CTLAB's branchless distance-driven (DD3)
 * cone-beam projector / backprojector and of the SART / OS-SART / FISTA-TV
 * loops that drive them.  It is the parity checker for the CUDA library in
 * ctlab_b200/ and the timed CPU baseline of bench.py.  Nothing in the
 * product links, loads or calls this file: only tests/, the smoke check in
 * __graft_entry__.py and bench.py's CPU-baseline / reference legs do.
 *
 * Parity status.  The reference ships the DD3 entry points as declarations
 * only (src/DD3_GPU_Proj.h:41-44, src/DD3_GPU_Back.h:40-44,
 * src/DD3_GPU_recon.h:60-65; their .cu bodies are absent, see
 * src/CMakeLists.txt:58-82).  What survives as compiled, header-inline code
 * -- DD3Boundaries, regularizeAngle, the SART weighting functors, the
 * ossart update functor and the FISTA functor -- is pinned against golden
 * vectors produced by the reference headers themselves (oracle/ref_helpers.cu,
 * tests/golden/).  The DD3 core (projection/backprojection) is a restatement
 * of the published branchless DD method (summed-area table of piecewise
 * constant slices, bilinear SAT interpolation, which is exact for axis
 * aligned rectangle integrals) and is pinned by analytic known answers
 * (uniform box chords, ellipsoid line integrals) and adjointness, not by
 * reference outputs, which cannot be produced.
 *
 * Conventions (shared with the CUDA library, stated once here):
 *   volume   float[XN*YN*ZN], (Z,X,Y) order: idx = (y*XN + x)*ZN + z
 *            (src/utilities.cuh:441, src/DD3_GPU_recon.h:37)
 *   mask     byte[XN*YN], idx = y*XN + x, applied to every z
 *   proj     float[PN*DNU*DNV], [view][u][v], v fastest
 *   geometry world = R(theta) * local, theta = regularizeAngle(hangs[p]),
 *            source (x0,y0,z0+zP), detector cells (xds,yds,zds+zP)
 *            (src/utilities.cuh:279-344)
 *   driving  a view is x-driven when theta lies in [pi/4,3pi/4) or
 *            [5pi/4,7pi/4), y-driven otherwise (constants of
 *            src/utilities.cuh:39-48).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI_4 0.785398163397448
#define ORC_PI_3_4 2.356194490192344
#define ORC_PI_5_4 3.926990816987241
#define ORC_PI_7_4 5.497787143782138
#define ORC_TWOPI 6.283185307179586

/* ------------------------------------------------------------------ */
/* helpers that restate header-inline reference code                   */
/* ------------------------------------------------------------------ */

/* Cell centres -> N+1 boundaries: midpoints, ends extrapolated
 * 1.5*c0 - 0.5*c1; a single cell gets centre -/+ 0.5.
 * Follows DD3Boundaries, src/utilities.cuh:413-433. */
void orc_dd3_boundaries(int n_boundaries, const double *c, double *b)
{
    if (n_boundaries >= 3) {
        int n = n_boundaries - 1;
        b[0] = 1.5 * c[0] - 0.5 * c[1];
        for (int i = 1; i < n; ++i) b[i] = 0.5 * c[i - 1] + 0.5 * c[i];
        b[n] = 1.5 * c[n - 1] - 0.5 * c[n - 2];
    } else {
        b[0] = c[0] - 0.5;
        b[1] = c[0] + 0.5;
    }
}

/* Angle into [0, 2pi).  Follows regularizeAngle, src/utilities.cuh:279-286. */
double orc_regularize_angle(double a)
{
    while (a >= ORC_TWOPI) a -= ORC_TWOPI;
    while (a < 0) a += ORC_TWOPI;
    return a;
}

int orc_view_is_xdriven(double theta_reg)
{
    return (theta_reg >= ORC_PI_4 && theta_reg < ORC_PI_3_4) ||
           (theta_reg >= ORC_PI_5_4 && theta_reg < ORC_PI_7_4);
}

/* ------------------------------------------------------------------ */
/* summed-area tables                                                  */
/* ------------------------------------------------------------------ */

/* Inclusive 2-D SAT with a zero first row/column:
 *   out[(i)*(nz+1) + k] = sum_{i'<i, k'<k} in[i'*in_stride_i + k'*in_stride_k]
 * for i in [0,ni], k in [0,nz]. */
void orc_sat2d(const double *in, long in_stride_i, long in_stride_k, int ni, int nz, double *out)
{
    long w = nz + 1;
    for (int k = 0; k <= nz; ++k) out[k] = 0.0;
    for (int i = 1; i <= ni; ++i) {
        double row = 0.0;
        out[(long)i * w] = 0.0;
        for (int k = 1; k <= nz; ++k) {
            row += in[(long)(i - 1) * in_stride_i + (long)(k - 1) * in_stride_k];
            out[(long)i * w + k] = out[(long)(i - 1) * w + k] + row;
        }
    }
}

/* Bilinear sample of a SAT of extent (ni+1) x (nz+1) at continuous boundary
 * coordinates (x, z), clamped to the table: exact rectangle integral of the
 * piecewise-constant field restricted to its support. */
static double sat_sample(const double *S, int ni, int nz, double x, double z)
{
    if (x < 0) x = 0;
    if (x > ni) x = ni;
    if (z < 0) z = 0;
    if (z > nz) z = nz;
    int i = (int)floor(x);
    if (i > ni - 1) i = ni - 1;
    int k = (int)floor(z);
    if (k > nz - 1) k = nz - 1;
    double fx = x - i, fz = z - k;
    long w = nz + 1;
    double s00 = S[(long)i * w + k], s01 = S[(long)i * w + k + 1];
    double s10 = S[(long)(i + 1) * w + k], s11 = S[(long)(i + 1) * w + k + 1];
    double a = s00 + fz * (s01 - s00);
    double b = s10 + fz * (s11 - s10);
    return a + fx * (b - a);
}

/* ------------------------------------------------------------------ */
/* per-view geometry                                                   */
/* ------------------------------------------------------------------ */

typedef struct {
    double c, s, zP;
    double Sx, Sy, Sz;
    int xdrv;
} orc_view;

static orc_view make_view(double x0, double y0, double z0, float ang, float zP)
{
    orc_view v;
    double th = orc_regularize_angle((double)ang);
    v.c = cos(th);
    v.s = sin(th);
    v.zP = (double)zP;
    v.Sx = x0 * v.c - y0 * v.s;
    v.Sy = x0 * v.s + y0 * v.c;
    v.Sz = z0 + v.zP;
    v.xdrv = orc_view_is_xdriven(th);
    return v;
}

/* A view's frame as make_view builds it: out = {cos, sin, zP, Sx, Sy, Sz,
 * x-driven}.  Exported so the tests can pin the oracle's rotation. */
void orc_view_frame(double x0, double y0, double z0, float ang, float zP, double *out)
{
    orc_view v = make_view(x0, y0, z0, ang, zP);
    out[0] = v.c; out[1] = v.s; out[2] = v.zP;
    out[3] = v.Sx; out[4] = v.Sy; out[5] = v.Sz;
    out[6] = (double)v.xdrv;
}

/* View-local point -> world with the rotation make_view uses (world =
 * R(theta) local + (0, 0, zP)); the inverse of the reference's invRotVox,
 * src/utilities.cuh:289-298, which the tests check it against. */
void orc_view_to_world(float ang, float zP, const double *local3, double *world3)
{
    orc_view v = make_view(0.0, 0.0, 0.0, ang, zP);
    world3[0] = local3[0] * v.c - local3[1] * v.s;
    world3[1] = local3[0] * v.s + local3[1] * v.c;
    world3[2] = local3[2] + v.zP;
}

static void boundaries_f(int n, const float *cf, double *b)
{
    if (n < 1) return;
    double *c = (double *)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) c[i] = (double)cf[i];
    orc_dd3_boundaries(n + 1, c, b);
    free(c);
}

/* Builds both volume SATs of the masked volume:
 *   saty[j][i'][k'] over (x,z) planes of y-slice j      (YN x (XN+1) x (ZN+1))
 *   satx[i][j'][k'] over (y,z) planes of x-slice i      (XN x (YN+1) x (ZN+1)) */
void orc_volume_sats(int XN, int YN, int ZN, const float *vol, const uint8_t *mask,
                     double *saty, double *satx)
{
    size_t nv = (size_t)XN * YN * ZN;
    double *f = (double *)malloc(sizeof(double) * nv);
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < (long)nv; ++idx) {
        long xy = idx / ZN;
        f[idx] = mask ? (double)vol[idx] * (double)(mask[xy] != 0) : (double)vol[idx];
    }
    long plane_y = (long)(XN + 1) * (ZN + 1);
    long plane_x = (long)(YN + 1) * (ZN + 1);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < YN; ++j)
        orc_sat2d(f + (long)j * XN * ZN, ZN, 1, XN, ZN, saty + (long)j * plane_y);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < XN; ++i)
        orc_sat2d(f + (long)i * ZN, (long)XN * ZN, 1, YN, ZN, satx + (long)i * plane_x);
    free(f);
}

/* Central-ray path length through one slab of the driving axis for the
 * detector cell centred at (cx, cy, cz): dx * |C - S| / |C_a - S_a|. */
static double path_weight(const orc_view *V, double dx, double cx, double cy, double cz)
{
    double ex = cx - V->Sx, ey = cy - V->Sy, ez = cz - V->Sz;
    double len = sqrt(ex * ex + ey * ey + ez * ez);
    double ea = V->xdrv ? ex : ey;
    return dx * len / fabs(ea);
}

/* ------------------------------------------------------------------ */
/* branchless DD projection                                            */
/* ------------------------------------------------------------------ */

/* Branchless DD cone-beam forward projection, FP64 throughout.
 * Same arguments as DD3Proj_gpu (src/DD3_GPU_Proj.h:41-44) minus the GPU
 * selectors; prj receives [PN][DNU][DNV] doubles.
 *
 * For each view and detector cell (u,v), for every slice j of the driving
 * axis a, the cell's two in-plane boundary rays and its two z boundaries
 * (taken along the cell's central in-plane ray) are intersected with the
 * slice plane a = a_j, giving an axis-aligned rectangle in slice index
 * units.  The rectangle integral of the masked slice is read from the
 * slice SAT by four clamped bilinear samples, divided by the rectangle's
 * signed area, summed over slices and multiplied by the central ray's path
 * length through one slab. */
void orc_dd3_proj(double x0, double y0, double z0, int DNU, int DNV,
                  const float *xds, const float *yds, const float *zds,
                  double imgXCenter, double imgYCenter, double imgZCenter,
                  const float *hangs, const float *hzPos, int PN,
                  int XN, int YN, int ZN, const float *vol, double *prj,
                  double dx, double dz, const uint8_t *mask)
{
    long plane_y = (long)(XN + 1) * (ZN + 1);
    long plane_x = (long)(YN + 1) * (ZN + 1);
    double *saty = (double *)malloc(sizeof(double) * (size_t)plane_y * YN);
    double *satx = (double *)malloc(sizeof(double) * (size_t)plane_x * XN);
    orc_volume_sats(XN, YN, ZN, vol, mask, saty, satx);

    double *bx = (double *)malloc(sizeof(double) * (DNU + 1));
    double *by = (double *)malloc(sizeof(double) * (DNU + 1));
    double *bz = (double *)malloc(sizeof(double) * (DNV + 1));
    boundaries_f(DNU, xds, bx);
    boundaries_f(DNU, yds, by);
    boundaries_f(DNV, zds, bz);

    const double x_lo = imgXCenter - 0.5 * XN * dx;
    const double y_lo = imgYCenter - 0.5 * YN * dx;
    const double z_lo = imgZCenter - 0.5 * ZN * dz;

#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int p = 0; p < PN; ++p) {
        for (int u = 0; u < DNU; ++u) {
            orc_view V = make_view(x0, y0, z0, hangs[p], hzPos[p]);
            /* world coordinates of the two boundaries and the centre */
            double B0x = bx[u] * V.c - by[u] * V.s, B0y = bx[u] * V.s + by[u] * V.c;
            double B1x = bx[u + 1] * V.c - by[u + 1] * V.s, B1y = bx[u + 1] * V.s + by[u + 1] * V.c;
            double Cx = (double)xds[u] * V.c - (double)yds[u] * V.s;
            double Cy = (double)xds[u] * V.s + (double)yds[u] * V.c;
            /* (b, a) = in-plane non-driving, driving coordinates */
            double Sa, Sb, B0a, B0b, B1a, B1b, Ca, a_c, b_lo;
            int NA, NB;
            const double *sat;
            long plane;
            if (V.xdrv) {
                Sa = V.Sx; Sb = V.Sy; B0a = B0x; B0b = B0y; B1a = B1x; B1b = B1y; Ca = Cx;
                NA = XN; NB = YN; a_c = imgXCenter; b_lo = y_lo; sat = satx; plane = plane_x;
            } else {
                Sa = V.Sy; Sb = V.Sx; B0a = B0y; B0b = B0x; B1a = B1y; B1b = B1x; Ca = Cy;
                NA = YN; NB = XN; a_c = imgYCenter; b_lo = x_lo; sat = saty; plane = plane_y;
            }
            (void)a_c;
            for (int v = 0; v < DNV; ++v) {
                double zc = (double)zds[v] + V.zP;
                double L = path_weight(&V, dx, Cx, Cy, zc);
                double zb0 = bz[v] + V.zP, zb1 = bz[v + 1] + V.zP;
                double acc = 0.0;
                for (int j = 0; j < NA; ++j) {
                    double aj = (V.xdrv ? imgXCenter : imgYCenter) + (j - 0.5 * (NA - 1)) * dx;
                    double da = aj - Sa;
                    double xa = (Sb + da / (B0a - Sa) * (B0b - Sb) - b_lo) / dx;
                    double xb = (Sb + da / (B1a - Sa) * (B1b - Sb) - b_lo) / dx;
                    double tc = da / (Ca - Sa);
                    double za = (V.Sz + tc * (zb0 - V.Sz) - z_lo) / dz;
                    double zb = (V.Sz + tc * (zb1 - V.Sz) - z_lo) / dz;
                    double area = (xb - xa) * (zb - za);
                    if (area == 0.0) continue;
                    const double *S = sat + (long)j * plane;
                    double R = sat_sample(S, NB, ZN, xb, zb) - sat_sample(S, NB, ZN, xa, zb) -
                               sat_sample(S, NB, ZN, xb, za) + sat_sample(S, NB, ZN, xa, za);
                    acc += R / area;
                }
                prj[((long)p * DNU + u) * DNV + v] = acc * L;
            }
        }
    }
    free(bx); free(by); free(bz);
    free(saty); free(satx);
}

/* ------------------------------------------------------------------ */
/* branchless DD backprojection                                        */
/* ------------------------------------------------------------------ */

/* Returns 0 when the detector is flat with uniform in-plane and z pitch
 * (relative tolerance tol), the only detector the voxel-driven
 * backprojector maps onto; -1 otherwise. */
int orc_detector_is_flat_uniform(int DNU, int DNV, const float *xds, const float *yds,
                                 const float *zds, double tol)
{
    double *bx = (double *)malloc(sizeof(double) * (DNU + 1));
    double *by = (double *)malloc(sizeof(double) * (DNU + 1));
    double *bz = (double *)malloc(sizeof(double) * (DNV + 1));
    boundaries_f(DNU, xds, bx);
    boundaries_f(DNU, yds, by);
    boundaries_f(DNV, zds, bz);
    int ok = 0;
    double ex = (bx[DNU] - bx[0]) / DNU, ey = (by[DNU] - by[0]) / DNU;
    double pitch = sqrt(ex * ex + ey * ey);
    double ez = (bz[DNV] - bz[0]) / DNV;
    if (pitch == 0.0 || ez == 0.0) ok = -1;
    for (int q = 0; q <= DNU && ok == 0; ++q) {
        double px = bx[0] + q * ex, py = by[0] + q * ey;
        if (hypot(px - bx[q], py - by[q]) > tol * pitch) ok = -1;
    }
    for (int w = 0; w <= DNV && ok == 0; ++w)
        if (fabs(bz[0] + w * ez - bz[w]) > tol * fabs(ez)) ok = -1;
    free(bx); free(by); free(bz);
    return ok;
}

static double cross2(double ax, double ay, double bx, double by) { return ax * by - ay * bx; }

/* Branchless DD cone-beam backprojection (voxel driven), FP64 throughout.
 * Same arguments as DD3Back_gpu (src/DD3_GPU_Back.h:40-44) minus the GPU
 * selectors; vol receives XN*YN*ZN doubles in (Z,X,Y) order.
 *
 * Each view's projection is first weighted by the same central-ray slab
 * path length the projector applies, W = prj * L, and summed into a SAT
 * over detector boundary indices.  For every voxel the footprint on the
 * detector is the image of the voxel's two boundaries across the driving
 * axis (in-plane, through the source) and of its two z boundaries (along
 * the ray through the voxel centre); the integral of W over that footprint,
 * in detector-index units, is four clamped bilinear SAT samples.  The sum
 * over views is multiplied by the in-plane mask.  With this weighting the
 * operator approximates the transpose of orc_dd3_proj. */
int orc_dd3_back(double x0, double y0, double z0, int DNU, int DNV,
                 const float *xds, const float *yds, const float *zds,
                 double imgXCenter, double imgYCenter, double imgZCenter,
                 const float *hangs, const float *hzPos, int PN,
                 int XN, int YN, int ZN, double *vol, const float *prj,
                 double dx, double dz, const uint8_t *mask)
{
    if (orc_detector_is_flat_uniform(DNU, DNV, xds, yds, zds, 1e-4) != 0) return -1;
    double *bx = (double *)malloc(sizeof(double) * (DNU + 1));
    double *by = (double *)malloc(sizeof(double) * (DNU + 1));
    double *bz = (double *)malloc(sizeof(double) * (DNV + 1));
    boundaries_f(DNU, xds, bx);
    boundaries_f(DNU, yds, by);
    boundaries_f(DNV, zds, bz);
    const double Ex_l = (bx[DNU] - bx[0]) / DNU, Ey_l = (by[DNU] - by[0]) / DNU;
    const double dzb = (bz[DNV] - bz[0]) / DNV;

    long qw = (long)(DNU + 1) * (DNV + 1);
    double *Q = (double *)malloc(sizeof(double) * (size_t)qw * PN);
    orc_view *views = (orc_view *)malloc(sizeof(orc_view) * (size_t)PN);
    for (int p = 0; p < PN; ++p) views[p] = make_view(x0, y0, z0, hangs[p], hzPos[p]);

#pragma omp parallel
    {
        double *W = (double *)malloc(sizeof(double) * (size_t)DNU * DNV);
#pragma omp for schedule(static)
        for (int p = 0; p < PN; ++p) {
            const orc_view *V = &views[p];
            for (int u = 0; u < DNU; ++u) {
                double Cx = (double)xds[u] * V->c - (double)yds[u] * V->s;
                double Cy = (double)xds[u] * V->s + (double)yds[u] * V->c;
                for (int v = 0; v < DNV; ++v) {
                    double L = path_weight(V, dx, Cx, Cy, (double)zds[v] + V->zP);
                    W[(long)u * DNV + v] = (double)prj[((long)p * DNU + u) * DNV + v] * L;
                }
            }
            orc_sat2d(W, DNV, 1, DNU, DNV, Q + (long)p * qw);
        }
        free(W);
    }

#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 0; j < YN; ++j) {
        for (int i = 0; i < XN; ++i) {
            double xc = imgXCenter + (i - 0.5 * (XN - 1)) * dx;
            double yc = imgYCenter + (j - 0.5 * (YN - 1)) * dx;
            double m = mask ? (double)(mask[(long)j * XN + i] != 0) : 1.0;
            for (int k = 0; k < ZN; ++k) {
                double zk = imgZCenter + (k - 0.5 * (ZN - 1)) * dz;
                double acc = 0.0;
                for (int p = 0; p < PN; ++p) {
                    const orc_view *V = &views[p];
                    double B0x = bx[0] * V->c - by[0] * V->s, B0y = bx[0] * V->s + by[0] * V->c;
                    double Ex = Ex_l * V->c - Ey_l * V->s, Ey = Ex_l * V->s + Ey_l * V->c;
                    double p1x, p1y, p2x, p2y;
                    if (V->xdrv) { p1x = xc; p1y = yc - 0.5 * dx; p2x = xc; p2y = yc + 0.5 * dx; }
                    else { p1x = xc - 0.5 * dx; p1y = yc; p2x = xc + 0.5 * dx; p2y = yc; }
                    double sbx = V->Sx - B0x, sby = V->Sy - B0y;
                    double ua = cross2(sbx, sby, p1x - V->Sx, p1y - V->Sy) /
                                cross2(Ex, Ey, p1x - V->Sx, p1y - V->Sy);
                    double ub = cross2(sbx, sby, p2x - V->Sx, p2y - V->Sy) /
                                cross2(Ex, Ey, p2x - V->Sx, p2y - V->Sy);
                    double tc = cross2(B0x - V->Sx, B0y - V->Sy, Ex, Ey) /
                                cross2(xc - V->Sx, yc - V->Sy, Ex, Ey);
                    double zb0 = bz[0] + V->zP;
                    double va = (V->Sz + tc * (zk - 0.5 * dz - V->Sz) - zb0) / dzb;
                    double vb = (V->Sz + tc * (zk + 0.5 * dz - V->Sz) - zb0) / dzb;
                    const double *S = Q + (long)p * qw;
                    double I = sat_sample(S, DNU, DNV, ub, vb) - sat_sample(S, DNU, DNV, ua, vb) -
                               sat_sample(S, DNU, DNV, ub, va) + sat_sample(S, DNU, DNV, ua, va);
                    double sg = ((ub > ua) ? 1.0 : -1.0) * ((vb > va) ? 1.0 : -1.0);
                    acc += I * sg;
                }
                vol[((long)j * XN + i) * ZN + k] = acc * m;
            }
        }
    }
    free(views); free(Q);
    free(bx); free(by); free(bz);
    return 0;
}

/* ------------------------------------------------------------------ */
/* SART weighting, updates, FISTA, TV                                  */
/* ------------------------------------------------------------------ */

/* r = (b - p)/rowSum where rowSum > 1e-7, else 0.
 * Follows SART_Weighting::Proj_ptr, src/SARTWeighting.h:38-53. */
void orc_sart_proj_weight(float *prj, const float *real_prj, const float *row_sum, long n)
{
    for (long i = 0; i < n; ++i)
        prj[i] = (row_sum[i] > 1.0e-7f) ? (real_prj[i] - prj[i]) / row_sum[i] : 0.0f;
}

/* vol = vol/colSum where colSum > 1e-7, else 0; recon += vol.
 * Follows SART_Weighting::Back_ptr, src/SARTWeighting.h:74-91. */
void orc_sart_back_weight(float *vol, float *recon, const float *col_sum, long n)
{
    for (long i = 0; i < n; ++i) {
        vol[i] = (col_sum[i] > 1.0e-7f) ? vol[i] / col_sum[i] : 0.0f;
        recon[i] += vol[i];
    }
}

/* OS-SART voxel update used by the drivers:
 *   x = (x + lambda * (colSum > 1e-7 ? q/colSum : 0)) * mask, optionally
 *   clamped to [minV, maxV].  Combines src/SARTWeighting.h:74-91 (epsilon
 *   test) with ossart_update_functor / _Update, src/utilities.hpp:1202-1225
 *   and :1062-1094 (relaxation, mask, range). */
void orc_ossart_update(float *x, const float *q, const float *col_sum, const uint8_t *mask,
                       long XN, long YN, long ZN, float lambda, int clamp, float minV, float maxV)
{
    long n = XN * YN * ZN;
    for (long i = 0; i < n; ++i) {
        float m = mask ? (float)(mask[i / ZN] != 0) : 1.0f;
        float upd = (col_sum[i] > 1.0e-7f) ? q[i] / col_sum[i] : 0.0f;
        float v = (x[i] + lambda * upd) * m;
        if (clamp) v = v < minV ? minV : (v > maxV ? maxV : v);
        x[i] = v;
    }
}

/* cur = clamp(cur + (t1-1)/t2 * (cur - las), minV, maxV).
 * Follows FISTA_functor, src/FastIterativeShrinkageAlgorithm.h:17-42. */
void orc_fista_step(const float *las, float *cur, float t1, float t2, long n, float minV, float maxV)
{
    for (long i = 0; i < n; ++i) {
        float r = cur[i] + (t1 - 1.0f) / t2 * (cur[i] - las[i]);
        cur[i] = r < minV ? minV : (r > maxV ? maxV : r);
    }
}

/* Gradient of the smoothed isotropic TV with forward differences and
 * replicated borders, on a (Z,X,Y) volume:
 *   TV(f) = sum_n sqrt(eps + sum_d (f[n+e_d] - f[n])^2)
 *   g[m]  = sum_d (f[m]-f[m+e_d]) / phi[m] + sum_d (f[m]-f[m-e_d]) / phi[m-e_d]
 * The 3-D TV gradient of GradientOfTV_GPU / descentDir_SHARED
 * (src/differentialFuncs.hpp:491-501, :599-612) restated in FP64. */
void orc_tv_gradient(const float *f, float *g, int XN, int YN, int ZN, double eps)
{
#define F_(x, y, z) ((double)f[(((long)(y)) * XN + (x)) * ZN + (z)])
#pragma omp parallel for collapse(2) schedule(static)
    for (int y = 0; y < YN; ++y)
        for (int x = 0; x < XN; ++x)
            for (int z = 0; z < ZN; ++z) {
                double c = F_(x, y, z);
                double fxp = x + 1 < XN ? F_(x + 1, y, z) : c;
                double fyp = y + 1 < YN ? F_(x, y + 1, z) : c;
                double fzp = z + 1 < ZN ? F_(x, y, z + 1) : c;
                double phi = sqrt(eps + (fxp - c) * (fxp - c) + (fyp - c) * (fyp - c) + (fzp - c) * (fzp - c));
                double gsum = ((c - fxp) + (c - fyp) + (c - fzp)) / phi;
                if (x > 0) {
                    double n = F_(x - 1, y, z);
                    double a = c, b = y + 1 < YN ? F_(x - 1, y + 1, z) : n, d = z + 1 < ZN ? F_(x - 1, y, z + 1) : n;
                    double ph = sqrt(eps + (a - n) * (a - n) + (b - n) * (b - n) + (d - n) * (d - n));
                    gsum += (c - n) / ph;
                }
                if (y > 0) {
                    double n = F_(x, y - 1, z);
                    double a = x + 1 < XN ? F_(x + 1, y - 1, z) : n, b = c, d = z + 1 < ZN ? F_(x, y - 1, z + 1) : n;
                    double ph = sqrt(eps + (a - n) * (a - n) + (b - n) * (b - n) + (d - n) * (d - n));
                    gsum += (c - n) / ph;
                }
                if (z > 0) {
                    double n = F_(x, y, z - 1);
                    double a = x + 1 < XN ? F_(x + 1, y, z - 1) : n, b = y + 1 < YN ? F_(x, y + 1, z - 1) : n, d = c;
                    double ph = sqrt(eps + (a - n) * (a - n) + (b - n) * (b - n) + (d - n) * (d - n));
                    gsum += (c - n) / ph;
                }
                g[((long)y * XN + x) * ZN + z] = (float)gsum;
            }
#undef F_
}

/* ------------------------------------------------------------------ */
/* phantoms                                                            */
/* ------------------------------------------------------------------ */

/* Point-sampled sum of rotated ellipsoids at voxel centres.
 * Each ellipsoid e has 10 doubles: value, cx, cy, cz, ax, ay, az (semi-axes,
 * mm), phi, theta, psi (ZYZ-free "z-x-z" Euler angles, radians).  A point p
 * is inside when |R^T (p - c) / a| <= 1 with R = Rz(phi) Rx(theta) Rz(psi).
 * The sum is clamped to >= 0 when clamp_nonneg is set. */
void orc_ellipsoid_phantom(int XN, int YN, int ZN, double dx, double dz,
                           double cxv, double cyv, double czv,
                           const double *ell, int n_ell, int clamp_nonneg, float *vol)
{
    double *R = (double *)malloc(sizeof(double) * 9 * (size_t)n_ell);
    for (int e = 0; e < n_ell; ++e) {
        const double *E = ell + 10 * e;
        double cf = cos(E[7]), sf = sin(E[7]), ct = cos(E[8]), st = sin(E[8]), cp = cos(E[9]), sp = sin(E[9]);
        double *r = R + 9 * e; /* row-major Rz(phi) Rx(theta) Rz(psi) */
        r[0] = cf * cp - sf * ct * sp; r[1] = -cf * sp - sf * ct * cp; r[2] = sf * st;
        r[3] = sf * cp + cf * ct * sp; r[4] = -sf * sp + cf * ct * cp; r[5] = -cf * st;
        r[6] = st * sp;                r[7] = st * cp;                 r[8] = ct;
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int y = 0; y < YN; ++y)
        for (int x = 0; x < XN; ++x)
            for (int z = 0; z < ZN; ++z) {
                double px = cxv + (x - 0.5 * (XN - 1)) * dx;
                double py = cyv + (y - 0.5 * (YN - 1)) * dx;
                double pz = czv + (z - 0.5 * (ZN - 1)) * dz;
                double acc = 0.0;
                for (int e = 0; e < n_ell; ++e) {
                    const double *E = ell + 10 * e;
                    const double *r = R + 9 * e;
                    double qx = px - E[1], qy = py - E[2], qz = pz - E[3];
                    /* local = R^T q */
                    double lx = r[0] * qx + r[3] * qy + r[6] * qz;
                    double ly = r[1] * qx + r[4] * qy + r[7] * qz;
                    double lz = r[2] * qx + r[5] * qy + r[8] * qz;
                    double s = (lx / E[4]) * (lx / E[4]) + (ly / E[5]) * (ly / E[5]) + (lz / E[6]) * (lz / E[6]);
                    if (s <= 1.0) acc += E[0];
                }
                if (clamp_nonneg && acc < 0) acc = 0;
                vol[((long)y * XN + x) * ZN + z] = (float)acc;
            }
    free(R);
}

/* Exact line integral of the ellipsoid sum along the segment P0 -> P1 (the
 * chord-length formula of Ellipsoid::intersectionLength,
 * src/Ellipsoid.h:209-247, extended to 3-D), clamped segment. */
double orc_ellipsoid_line_integral(const double *ell, int n_ell, const double *P0, const double *P1)
{
    double total = 0.0;
    for (int e = 0; e < n_ell; ++e) {
        const double *E = ell + 10 * e;
        double cf = cos(E[7]), sf = sin(E[7]), ct = cos(E[8]), st = sin(E[8]), cp = cos(E[9]), sp = sin(E[9]);
        double r[9] = {cf * cp - sf * ct * sp, -cf * sp - sf * ct * cp, sf * st,
                       sf * cp + cf * ct * sp, -sf * sp + cf * ct * cp, -cf * st,
                       st * sp, st * cp, ct};
        double s0[3] = {P0[0] - E[1], P0[1] - E[2], P0[2] - E[3]};
        double d[3] = {P1[0] - P0[0], P1[1] - P0[1], P1[2] - P0[2]};
        double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double o[3], w[3];
        for (int c = 0; c < 3; ++c) {
            o[c] = (r[0 + c] * s0[0] + r[3 + c] * s0[1] + r[6 + c] * s0[2]) / E[4 + c];
            w[c] = (r[0 + c] * d[0] + r[3 + c] * d[1] + r[6 + c] * d[2]) / (E[4 + c] * len);
        }
        double A = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
        double B = 2.0 * (w[0] * o[0] + w[1] * o[1] + w[2] * o[2]);
        double C = o[0] * o[0] + o[1] * o[1] + o[2] * o[2] - 1.0;
        double disc = B * B - 4.0 * A * C;
        if (disc <= 0) continue;
        double sq = sqrt(disc);
        double t1 = (-B - sq) / (2.0 * A), t2 = (-B + sq) / (2.0 * A);
        if (t1 < 0) t1 = 0;
        if (t2 > len) t2 = len;
        if (t2 > t1) total += E[0] * (t2 - t1);
    }
    return total;
}

/* ------------------------------------------------------------------ */
/* reconstruction loops (small sizes; FP32 state like the GPU drivers)  */
/* ------------------------------------------------------------------ */

static void proj_f(double x0, double y0, double z0, int DNU, int DNV, const float *xds,
                   const float *yds, const float *zds, double cx, double cy, double cz,
                   const float *angs, const float *zps, int PN, int XN, int YN, int ZN,
                   const float *vol, float *out, double dx, double dz, const uint8_t *mask)
{
    long n = (long)PN * DNU * DNV;
    double *tmp = (double *)malloc(sizeof(double) * (size_t)n);
    orc_dd3_proj(x0, y0, z0, DNU, DNV, xds, yds, zds, cx, cy, cz, angs, zps, PN, XN, YN, ZN,
                 vol, tmp, dx, dz, mask);
    for (long i = 0; i < n; ++i) out[i] = (float)tmp[i];
    free(tmp);
}

static void back_f(double x0, double y0, double z0, int DNU, int DNV, const float *xds,
                   const float *yds, const float *zds, double cx, double cy, double cz,
                   const float *angs, const float *zps, int PN, int XN, int YN, int ZN,
                   float *vol, const float *prj, double dx, double dz, const uint8_t *mask)
{
    long n = (long)XN * YN * ZN;
    double *tmp = (double *)malloc(sizeof(double) * (size_t)n);
    orc_dd3_back(x0, y0, z0, DNU, DNV, xds, yds, zds, cx, cy, cz, angs, zps, PN, XN, YN, ZN,
                 tmp, prj, dx, dz, mask);
    for (long i = 0; i < n; ++i) vol[i] = (float)tmp[i];
    free(tmp);
}

/* OS-SART with interleaved subsets {s, s+S, s+2S, ...}.  x holds the
 * initial image on entry and the result on exit.  Per subset:
 *   r = (b_s - A_s x)/rowSum_s  (0 where rowSum <= 1e-7)
 *   x = (x + lambda * B_s r / colSum_s) * mask   (0 where colSum <= 1e-7)
 * rowSum_s = A_s 1 and colSum_s = B_s 1 over the masked volume, the
 * all-ones evaluation of evalProjBack (src/DD3_GPU_recon.h:25-28).
 * Drives OS_SART, src/DD3_GPU_recon.h:60-65. */
int orc_os_sart(double x0, double y0, double z0, int DNU, int DNV, const float *xds,
                const float *yds, const float *zds, double cx, double cy, double cz,
                const float *hangs, const float *hzPos, int PN, int XN, int YN, int ZN,
                float *x, const float *prj, double dx, double dz, const uint8_t *mask,
                int osNum, int iterNum, float lambda, int clamp, float minV, float maxV)
{
    if (orc_detector_is_flat_uniform(DNU, DNV, xds, yds, zds, 1e-4) != 0) return -1;
    long nv = (long)XN * YN * ZN, nd = (long)DNU * DNV;
    int maxn = (PN + osNum - 1) / osNum;
    float *angs = (float *)malloc(sizeof(float) * maxn), *zps = (float *)malloc(sizeof(float) * maxn);
    float *bsub = (float *)malloc(sizeof(float) * maxn * nd), *p = (float *)malloc(sizeof(float) * maxn * nd);
    float *rs = (float *)malloc(sizeof(float) * maxn * nd), *ones_p = (float *)malloc(sizeof(float) * maxn * nd);
    float *ones_v = (float *)malloc(sizeof(float) * nv), *cs = (float *)malloc(sizeof(float) * nv);
    float *q = (float *)malloc(sizeof(float) * nv);
    for (long i = 0; i < nv; ++i) ones_v[i] = 1.0f;
    for (long i = 0; i < maxn * nd; ++i) ones_p[i] = 1.0f;
    for (int it = 0; it < iterNum; ++it) {
        for (int s = 0; s < osNum; ++s) {
            int n = 0;
            for (int v = s; v < PN; v += osNum) {
                angs[n] = hangs[v]; zps[n] = hzPos[v];
                memcpy(bsub + (long)n * nd, prj + (long)v * nd, sizeof(float) * nd);
                ++n;
            }
            if (n == 0) continue;
            proj_f(x0, y0, z0, DNU, DNV, xds, yds, zds, cx, cy, cz, angs, zps, n, XN, YN, ZN, ones_v, rs, dx, dz, mask);
            back_f(x0, y0, z0, DNU, DNV, xds, yds, zds, cx, cy, cz, angs, zps, n, XN, YN, ZN, cs, ones_p, dx, dz, mask);
            proj_f(x0, y0, z0, DNU, DNV, xds, yds, zds, cx, cy, cz, angs, zps, n, XN, YN, ZN, x, p, dx, dz, mask);
            orc_sart_proj_weight(p, bsub, rs, (long)n * nd);
            back_f(x0, y0, z0, DNU, DNV, xds, yds, zds, cx, cy, cz, angs, zps, n, XN, YN, ZN, q, p, dx, dz, mask);
            orc_ossart_update(x, q, cs, mask, XN, YN, ZN, lambda, clamp, minV, maxV);
        }
    }
    free(angs); free(zps); free(bsub); free(p); free(rs); free(ones_p); free(ones_v); free(cs); free(q);
    return 0;
}

/* FISTA-TV: SART-preconditioned gradient step over all views, one explicit
 * TV gradient step of weight tv_lambda, FISTA momentum with the clamp of
 * FISTA_functor (src/FastIterativeShrinkageAlgorithm.h:17-42):
 *   z   = (y + B((b - A y)/rowSum)/colSum) * mask   (epsilon tests as in SART)
 *   x_k = (z - tv_lambda * gradTV(z)) * mask
 *   t'  = (1 + sqrt(1 + 4 t^2))/2
 *   y   = clamp(x_k + (t-1)/t' (x_k - x_{k-1}), minV, maxV)
 * x holds the initial image on entry and x_k of the last iteration on exit. */
int orc_fista_tv(double x0, double y0, double z0, int DNU, int DNV, const float *xds,
                 const float *yds, const float *zds, double cx, double cy, double cz,
                 const float *hangs, const float *hzPos, int PN, int XN, int YN, int ZN,
                 float *x, const float *prj, double dx, double dz, const uint8_t *mask,
                 int iterNum, float tv_lambda, double tv_eps, float minV, float maxV)
{
    if (orc_detector_is_flat_uniform(DNU, DNV, xds, yds, zds, 1e-4) != 0) return -1;
    long nv = (long)XN * YN * ZN, nd = (long)PN * DNU * DNV;
    float *rs = (float *)malloc(sizeof(float) * nd), *cs = (float *)malloc(sizeof(float) * nv);
    float *ones_v = (float *)malloc(sizeof(float) * nv), *ones_p = (float *)malloc(sizeof(float) * nd);
    float *y = (float *)malloc(sizeof(float) * nv), *xp = (float *)malloc(sizeof(float) * nv);
    float *p = (float *)malloc(sizeof(float) * nd), *q = (float *)malloc(sizeof(float) * nv);
    float *g = (float *)malloc(sizeof(float) * nv);
    for (long i = 0; i < nv; ++i) ones_v[i] = 1.0f;
    for (long i = 0; i < nd; ++i) ones_p[i] = 1.0f;
    proj_f(x0, y0, z0, DNU, DNV, xds, yds, zds, cx, cy, cz, hangs, hzPos, PN, XN, YN, ZN, ones_v, rs, dx, dz, mask);
    back_f(x0, y0, z0, DNU, DNV, xds, yds, zds, cx, cy, cz, hangs, hzPos, PN, XN, YN, ZN, cs, ones_p, dx, dz, mask);
    memcpy(y, x, sizeof(float) * nv);
    memcpy(xp, x, sizeof(float) * nv);
    float t = 1.0f;
    for (int it = 0; it < iterNum; ++it) {
        proj_f(x0, y0, z0, DNU, DNV, xds, yds, zds, cx, cy, cz, hangs, hzPos, PN, XN, YN, ZN, y, p, dx, dz, mask);
        orc_sart_proj_weight(p, prj, rs, nd);
        back_f(x0, y0, z0, DNU, DNV, xds, yds, zds, cx, cy, cz, hangs, hzPos, PN, XN, YN, ZN, q, p, dx, dz, mask);
        for (long i = 0; i < nv; ++i) {
            float m = mask ? (float)(mask[i / ZN] != 0) : 1.0f;
            y[i] = (y[i] + ((cs[i] > 1.0e-7f) ? q[i] / cs[i] : 0.0f)) * m;
        }
        orc_tv_gradient(y, g, XN, YN, ZN, tv_eps);
        for (long i = 0; i < nv; ++i) {
            float m = mask ? (float)(mask[i / ZN] != 0) : 1.0f;
            x[i] = (y[i] - tv_lambda * g[i]) * m;
        }
        float tn = (1.0f + sqrtf(1.0f + 4.0f * t * t)) * 0.5f;
        memcpy(y, x, sizeof(float) * nv);
        orc_fista_step(xp, y, t, tn, nv, minV, maxV);
        memcpy(xp, x, sizeof(float) * nv);
        t = tn;
    }
    free(rs); free(cs); free(ones_v); free(ones_p); free(y); free(xp); free(p); free(q); free(g);
    return 0;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
