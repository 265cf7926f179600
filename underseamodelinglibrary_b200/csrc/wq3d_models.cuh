/*
 * wq3d_models.cuh -- ocean models and ray derivative terms, shared by the
 * propagation kernels and by host-side precomputation.
 *
 * Every function is __host__ __device__: quantities that depend only on
 * constants or targets (target sound speed, boundary slope terms, Thorp
 * coefficients) are evaluated once on the host; per-ray quantities are
 * evaluated in the kernels.  The arithmetic follows the reference's
 * operation order so that the FP64 form rounds the way the reference does
 * (the library is compiled with --fmad=false).
 */
#pragma once

#include <math.h>
#include <stdint.h>

#include "../../include/wq3d.h"

/* WQ3D_WITH_GRID=0 compiles the models without the gridded profile and
 * boundary kinds (they then read as the default kind); the host never
 * hands such a build an ocean that has a grid. */
#ifndef WQ3D_WITH_GRID
#define WQ3D_WITH_GRID 1
#endif

#ifdef __CUDACC__
#define WQ_HD __host__ __device__ __forceinline__
/* Out-of-line device functions: the per-dimension grid interpolation calls
 * the next dimension 1, 2 or 4 times per interpolation kind, so inlining
 * the chain would copy the innermost level hundreds of times into every
 * caller of sound_speed. */
#define WQ_NOINL __host__ __device__ __noinline__
#else
#define WQ_HD inline
#define WQ_NOINL inline
#endif

namespace wq3d {

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_PI_2
#define M_PI_2 1.57079632679489661923
#endif

/* reflect loss, with the constants of reflect_loss_rayleigh.cc:68-78 */
struct LossDev {
    int kind;
    double p[5];
    double rl_den, rl_spd, rl_att, rl_shr, rl_satt;
};

/* ------------------------------------------------------------------ */
/* rectilinear grids (types/gen_grid.h:83-520, gen_grid_utils.h)        */
/* ------------------------------------------------------------------ */
struct AxisDev {
    const double* x;
    const double* inc;
    int n;
    int kind;       /* WQ3D_AXIS_* */
    double sign;    /* seq_data: -1 for a decreasing axis */
};

struct GridDev {
    int ndim;
    int all_linear;  /* every axis interpolates linearly: unrolled path */
    int pchip0;      /* pchip on axis 0, linear on the others: unrolled path */
    AxisDev ax[3];
    int interp[3];
    int edge[3];
    const double* data;
};

/* seq_vector::increment clamps its index (seq_vector.h:140-143) */
WQ_HD double axis_inc(const AxisDev& a, long k) {
    /* a negative index wraps to a huge size_t there, so it clamps high too */
    if (k < 0 || k > a.n - 1) k = a.n - 1;
    return a.inc[k];
}

/* find_index of seq_linear (seq_linear.h:89-94), seq_log (seq_log.h:88-94)
 * and seq_data (seq_data.cc:15-36) */
WQ_HD int axis_find(const AxisDev& a, double v) {
    if (a.kind == WQ3D_AXIS_LINEAR) {
        const double f = floor((v - a.x[0]) / a.inc[0]);
        long k = (long)f;
        if (k > a.n - 2) k = a.n - 2;
        if (k < 0) k = 0;
        return (int)k;
    }
    if (a.kind == WQ3D_AXIS_LOG) {
        const double f = floor(log(v / a.x[0]) / log(a.inc[1] / a.inc[0]));
        long k = (long)f;
        if (k > a.n - 2) k = a.n - 2;
        if (k < 0) k = 0;
        return (int)k;
    }
    const double s = a.sign;
    v *= s;
    const int max_index = a.n - 1;
    if (max_index < 1) return 0;
    if (v <= s * a.x[0]) return 0;
    if (v >= s * a.x[max_index - 1]) return max_index - 1;
    /* first entry whose key exceeds v (std::map::upper_bound), minus one */
    int lo = 0, hi = a.n; /* keys s*x[] increase */
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (s * a.x[mid] > v) hi = mid; else lo = mid + 1;
    }
    return lo - 1;
}

template <int NDIM, int DIM>
struct GridInterp;

/* dim < 0: the data point at the corner index (data_grid_compute_offset) */
template <int NDIM>
struct GridInterp<NDIM, -1> {
    WQ_HD static double run(const GridDev& g, const int* index, const double*, double&, double*) {
        size_t off = (size_t)index[0];
        for (int d = 1; d < NDIM; ++d) off = (size_t)index[d] + (size_t)g.ax[d].n * off;
        return g.data[off];
    }
};

template <int NDIM, int DIM>
struct GridInterp {
    WQ_HD static double nearest(const GridDev& g, const int* index, const double* loc, double& deriv,
                                double* dv) {
        double result;
        double da = 0.0;
        const int k = index[DIM];
        const AxisDev& ax = g.ax[DIM];
        const double u = (loc[DIM] - ax.x[k]) / axis_inc(ax, k);
        if (u < 0.5) {
            result = GridInterp<NDIM, DIM - 1>::run(g, index, loc, da, dv);
        } else {
            int next[NDIM];
            for (int d = 0; d < NDIM; ++d) next[d] = index[d];
            ++next[DIM];
            result = GridInterp<NDIM, DIM - 1>::run(g, next, loc, da, dv);
        }
        if (dv) {
            dv[DIM] = deriv;
            if (DIM > 0) dv[DIM > 0 ? DIM - 1 : 0] = da;
        }
        return result;
    }

    WQ_HD static double linear(const GridDev& g, const int* index, const double* loc, double& deriv,
                               double* dv) {
        double da = 0.0, db = 0.0;
        const double a = GridInterp<NDIM, DIM - 1>::run(g, index, loc, da, dv);
        int next[NDIM];
        for (int d = 0; d < NDIM; ++d) next[d] = index[d];
        ++next[DIM];
        const double b = GridInterp<NDIM, DIM - 1>::run(g, next, loc, db, dv);
        const int k = index[DIM];
        const AxisDev& ax = g.ax[DIM];
        const double h = axis_inc(ax, k);
        const double u = (loc[DIM] - ax.x[k]) / h;
        const double result = a * (1.0 - u) + b * u;
        if (dv) {
            deriv = (b - a) / h;
            dv[DIM] = deriv;
            if (DIM > 0) dv[DIM > 0 ? DIM - 1 : 0] = da * (1.0 - u) + db * u;
        }
        return result;
    }

    /* harmonic mean slope (gen_grid_utils.h derivative<T>::compute) */
    WQ_HD static void harmonic(double d0, double d1, double dd0, double dd1, double w0, double w1,
                               bool deriv, double& m, double& dm) {
        if (d0 * d1 > 0.0) m = (w0 + w1) / (w0 / d0 + w1 / d1);
        if (deriv && dd0 * dd1 > 0.0) dm = (w0 + w1) / (w0 / dd0 + w1 / dd1);
    }
    /* end_point_derivative<T>::compute for scalars */
    WQ_HD static void end_point(double d0, double d1, double dd0, double dd1, bool deriv, double& m,
                                double& dm) {
        if (m * d0 < 0.0) {
            m = 0.0;
        } else if ((d0 * d1 < 0.0) && (fabs(m) > fabs(3.0 * d1))) {
            m = 3.0 * d1;
        }
        if (deriv) {
            if (dm * dd0 < 0.0) {
                dm = 0.0;
            } else if ((dd0 * dd1 < 0.0) && (fabs(dm) > fabs(3.0 * dd0))) {
                dm = 3.0 * dd0;
            }
        } else {
            dm = 0.0;
        }
    }

    /* gen_grid.h pchip, keeping the end-point slope "(2.0 + h1 + h2)" and
     * the slope2 weights built from h0 (gen_grid.h:458-488) */
    WQ_HD static double pchip(const GridDev& g, const int* index, const double* loc, double& deriv,
                              double* dv) {
        const AxisDev& ax = g.ax[DIM];
        const int kmin = 1;
        const int kmax = ax.n - 3;
        double y0, y1, y2, y3, dy0 = 0.0, dy1 = 0.0, dy2 = 0.0, dy3 = 0.0;
        const int k = index[DIM];
        y1 = GridInterp<NDIM, DIM - 1>::run(g, index, loc, dy1, dv);
        if (k >= kmin) {
            int prev[NDIM];
            for (int d = 0; d < NDIM; ++d) prev[d] = index[d];
            --prev[DIM];
            y0 = GridInterp<NDIM, DIM - 1>::run(g, prev, loc, dy0, dv);
        } else {
            y0 = y1;
            dy0 = dy1;
        }
        int next[NDIM];
        for (int d = 0; d < NDIM; ++d) next[d] = index[d];
        ++next[DIM];
        y2 = GridInterp<NDIM, DIM - 1>::run(g, next, loc, dy2, dv);
        if (k <= kmax) {
            int last[NDIM];
            for (int d = 0; d < NDIM; ++d) last[d] = next[d];
            ++last[DIM];
            y3 = GridInterp<NDIM, DIM - 1>::run(g, last, loc, dy3, dv);
        } else {
            y3 = y2;
            dy3 = dy2;
        }
        const double h0 = axis_inc(ax, (long)k - 1);
        const double h1 = axis_inc(ax, k);
        const double h2 = axis_inc(ax, (long)k + 1);
        const double h1_2 = h1 * h1;
        const double h1_3 = h1_2 * h1;
        const double s = loc[DIM] - ax.x[k];
        const double s_2 = s * s, s_3 = s_2 * s;
        const double sh_minus = s - h1;
        const double sh_term = 3.0 * h1 * s_2 - 2.0 * s_3;
        const double deriv0 = (y1 - y0) / h0;
        const double deriv1 = (y2 - y1) / h1;
        const double deriv2 = (y3 - y2) / h2;
        double dderiv0 = 0.0, dderiv1 = 0.0, dderiv2 = 0.0;
        if (dv) {
            dderiv0 = (dy1 - dy0) / h0;
            dderiv1 = (dy2 - dy1) / h1;
            dderiv2 = (dy3 - dy2) / h2;
        }
        double slope1 = 0.0, dslope1 = 0.0;
        if (k >= kmin) {
            const double w0 = 2.0 * h1 + h0;
            const double w1 = h1 + 2.0 * h0;
            harmonic(deriv0, deriv1, dderiv0, dderiv1, w0, w1, dv != nullptr, slope1, dslope1);
        } else {
            slope1 = ((2.0 + h1 + h2) * deriv1 - h1 * deriv2) / (h1 + h2);
            dslope1 = ((2.0 + h1 + h2) * dderiv1 - h1 * dderiv2) / (h1 + h2);
            end_point(deriv1, deriv2, dderiv1, dderiv2, dv != nullptr, slope1, dslope1);
        }
        double slope2 = 0.0, dslope2 = 0.0;
        if (k <= kmax) {
            const double w1 = 2.0 * h1 + h0;
            const double w2 = h1 + 2.0 * h0;
            harmonic(deriv1, deriv2, dderiv1, dderiv2, w1, w2, dv != nullptr, slope2, dslope2);
        } else {
            slope2 = ((2.0 + h1 + h2) * deriv1 - h1 * deriv0) / (h1 + h0);
            dslope2 = ((2.0 + h1 + h2) * dderiv1 - h1 * dderiv0) / (h1 + h0);
            end_point(deriv1, deriv0, dderiv1, dderiv0, dv != nullptr, slope2, dslope2);
        }
        const double result = y2 * sh_term / h1_3 + y1 * (h1_3 - sh_term) / h1_3 +
                              slope2 * s_2 * sh_minus / h1_2 +
                              slope1 * s * sh_minus * sh_minus / h1_2;
        if (dv) {
            const double v = s / h1;
            deriv = slope1 * (1.0 - v) + slope2 * v;
            dv[DIM] = deriv;
            if (DIM > 0)
                dv[DIM > 0 ? DIM - 1 : 0] = dy2 * sh_term / h1_3 + dy1 * (h1_3 - sh_term) / h1_3 +
                                            dslope2 * s_2 * sh_minus / h1_2 +
                                            dslope1 * s * sh_minus * sh_minus / h1_2;
        }
        return result;
    }

    WQ_NOINL static double run(const GridDev& g, const int* index, const double* loc, double& deriv,
                               double* dv) {
        switch (g.interp[DIM]) {
            case WQ3D_INTERP_NEAREST:
                return nearest(g, index, loc, deriv, dv);
            case WQ3D_INTERP_PCHIP:
                return pchip(g, index, loc, deriv, dv);
            default:
                return linear(g, index, loc, deriv, dv);
        }
    }
};

/* gen_grid::interpolate (gen_grid.h:83-123): edge limiting, find_index on
 * each axis, then the recursive interpolation.  dv may be null. */
template <int NDIM>
WQ_HD double grid_interpolate(const GridDev& g, const double* location, double* dv) {
    int index[NDIM];
    double loc[NDIM];
    for (int d = 0; d < NDIM; ++d) loc[d] = location[d];
    for (int d = 0; d < NDIM; ++d) {
        const AxisDev& ax = g.ax[d];
        if (g.edge[d]) {
            const double a = ax.x[0];
            const double b = ax.x[ax.n - 1];
            const double sign = (ax.inc[0] < 0) ? -1.0 : 1.0;
            const double dd = loc[d] * sign;
            if (dd <= a * sign) {
                loc[d] = a;
                index[d] = 0;
            } else if (dd >= b * sign) {
                loc[d] = b;
                index[d] = ax.n - 2;
            } else {
                index[d] = axis_find(ax, loc[d]);
            }
        } else {
            index[d] = axis_find(ax, loc[d]);
        }
    }
    double dresult = 0.0;
    return GridInterp<NDIM, NDIM - 1>::run(g, index, loc, dresult, dv);
}

/* The all-linear case of grid_interpolate, unrolled: the same expression
 * tree as the recursion of GridInterp (outermost over the last axis), and
 * the same writes to the shared derivative array, so results are
 * identical bit for bit while the evaluation stays inline in registers. */
WQ_HD double lin1(const GridDev& g, int d, const int* index, const double* loc, double a, double b,
                  double* u_out, double* h_out) {
    const AxisDev& ax = g.ax[d];
    const int k = index[d];
    const double h = axis_inc(ax, k);
    const double u = (loc[d] - ax.x[k]) / h;
    *u_out = u;
    *h_out = h;
    return a * (1.0 - u) + b * u;
}

template <int NDIM>
WQ_HD double grid_linear(const GridDev& g, const double* location, double* dv) {
    int index[NDIM];
    double loc[NDIM];
    for (int d = 0; d < NDIM; ++d) loc[d] = location[d];
    for (int d = 0; d < NDIM; ++d) {
        const AxisDev& ax = g.ax[d];
        if (g.edge[d]) {
            const double a = ax.x[0];
            const double b = ax.x[ax.n - 1];
            const double sign = (ax.inc[0] < 0) ? -1.0 : 1.0;
            const double dd = loc[d] * sign;
            if (dd <= a * sign) {
                loc[d] = a;
                index[d] = 0;
            } else if (dd >= b * sign) {
                loc[d] = b;
                index[d] = ax.n - 2;
            } else {
                index[d] = axis_find(ax, loc[d]);
            }
        } else {
            index[d] = axis_find(ax, loc[d]);
        }
    }
    const double* D = g.data;
    double u, h;
    if (NDIM == 1) {
        const double a = D[index[0]], b = D[index[0] + 1];
        const double r = lin1(g, 0, index, loc, a, b, &u, &h);
        if (dv) dv[0] = (b - a) / h;
        return r;
    }
    if (NDIM == 2) {
        const size_t n1 = (size_t)g.ax[1].n;
        const size_t o00 = (size_t)index[1] + n1 * (size_t)index[0];
        const size_t o10 = (size_t)index[1] + n1 * (size_t)(index[0] + 1);
        double u0, h0;
        /* outer axis 1; inner calls over axis 0 at index[1] and index[1]+1 */
        const double va = lin1(g, 0, index, loc, D[o00], D[o10], &u0, &h0);
        const double da = (D[o10] - D[o00]) / h0;
        const double vb = lin1(g, 0, index, loc, D[o00 + 1], D[o10 + 1], &u0, &h0);
        const double db = (D[o10 + 1] - D[o00 + 1]) / h0;
        const double r = lin1(g, 1, index, loc, va, vb, &u, &h);
        if (dv) {
            dv[1] = (vb - va) / h;
            dv[0] = da * (1.0 - u) + db * u;
        }
        return r;
    }
    /* NDIM == 3: outer axis 2, then axis 1, innermost axis 0 */
    const size_t n1 = (size_t)g.ax[1].n, n2 = (size_t)g.ax[2].n;
    auto off = [&](int i0, int i1, int i2) { return (size_t)i2 + n2 * ((size_t)i1 + n1 * (size_t)i0); };
    const int i0 = index[0], i1 = index[1], i2 = index[2];
    double u0, h0, u1, h1;
    double dv0_last = 0.0;
    /* one axis-1 interpolation at axis-2 index j: returns value, its axis-1
     * derivative, and the blended axis-0 derivative it leaves in dv[0] */
    auto plane = [&](int j, double* d1, double* d0) {
        const double a0 = D[off(i0, i1, j)], b0 = D[off(i0 + 1, i1, j)];
        const double va = lin1(g, 0, index, loc, a0, b0, &u0, &h0);
        const double da = (b0 - a0) / h0;
        const double a1 = D[off(i0, i1 + 1, j)], b1 = D[off(i0 + 1, i1 + 1, j)];
        const double vb = lin1(g, 0, index, loc, a1, b1, &u0, &h0);
        const double db = (b1 - a1) / h0;
        const double r = lin1(g, 1, index, loc, va, vb, &u1, &h1);
        *d1 = (vb - va) / h1;
        *d0 = da * (1.0 - u1) + db * u1;
        return r;
    };
    double d1a, d1b, d0a;
    const double pa = plane(i2, &d1a, &d0a);
    const double pb = plane(i2 + 1, &d1b, &dv0_last);
    const double r = lin1(g, 2, index, loc, pa, pb, &u, &h);
    if (dv) {
        dv[2] = (pb - pa) / h;
        dv[1] = d1a * (1.0 - u) + d1b * u;
        dv[0] = dv0_last;
    }
    return r;
}

/* pchip along axis 0 with every other axis linear (a profile grid's
 * usual form: pchip in depth, linear across), unrolled like grid_linear.
 * At axis 0 the recursion's corner values carry no derivative of their
 * own, so gen_grid.h's pchip (gen_grid.h:350-500) reduces to the value
 * and its axis-0 slope below; the spacing and offset terms depend only on
 * the axis-0 index and are computed once for every corner.  All corner
 * loads are issued before any arithmetic; the recursion instead fetched
 * them one out-of-line call at a time. */
struct Pchip0 {
    double h0, h1, h2, h1_2, h1_3, s, s_2, sh_minus, sh_term, v;
    bool lo_in;  /* k >= 1: a row below the cell */
    bool hi_in;  /* k <= n - 3: a row above the cell's upper row */
};

WQ_HD void pchip0_setup(const AxisDev& ax, int k, double x, Pchip0& P) {
    P.lo_in = k >= 1;
    P.hi_in = k <= ax.n - 3;
    P.h0 = axis_inc(ax, (long)k - 1);
    P.h1 = axis_inc(ax, k);
    P.h2 = axis_inc(ax, (long)k + 1);
    P.h1_2 = P.h1 * P.h1;
    P.h1_3 = P.h1_2 * P.h1;
    P.s = x - ax.x[k];
    P.s_2 = P.s * P.s;
    const double s_3 = P.s_2 * P.s;
    P.sh_minus = P.s - P.h1;
    P.sh_term = 3.0 * P.h1 * P.s_2 - 2.0 * s_3;
    P.v = P.s / P.h1;
}

/* one corner: rows k-1 .. k+2 of axis 0 (y0 / y3 already replaced by
 * y1 / y2 outside the axis); *deriv takes the axis-0 slope when want */
WQ_HD double pchip0_corner(const Pchip0& P, double y0, double y1, double y2, double y3, bool want,
                           double* deriv) {
    const double deriv0 = (y1 - y0) / P.h0;
    const double deriv1 = (y2 - y1) / P.h1;
    const double deriv2 = (y3 - y2) / P.h2;
    double slope1 = 0.0;
    if (P.lo_in) {
        const double w0 = 2.0 * P.h1 + P.h0;
        const double w1 = P.h1 + 2.0 * P.h0;
        if (deriv0 * deriv1 > 0.0) slope1 = (w0 + w1) / (w0 / deriv0 + w1 / deriv1);
    } else {
        slope1 = ((2.0 + P.h1 + P.h2) * deriv1 - P.h1 * deriv2) / (P.h1 + P.h2);
        if (slope1 * deriv1 < 0.0) {
            slope1 = 0.0;
        } else if ((deriv1 * deriv2 < 0.0) && (fabs(slope1) > fabs(3.0 * deriv2))) {
            slope1 = 3.0 * deriv2;
        }
    }
    double slope2 = 0.0;
    if (P.hi_in) {
        const double w1 = 2.0 * P.h1 + P.h0;
        const double w2 = P.h1 + 2.0 * P.h0;
        if (deriv1 * deriv2 > 0.0) slope2 = (w1 + w2) / (w1 / deriv1 + w2 / deriv2);
    } else {
        slope2 = ((2.0 + P.h1 + P.h2) * deriv1 - P.h1 * deriv0) / (P.h1 + P.h0);
        if (slope2 * deriv1 < 0.0) {
            slope2 = 0.0;
        } else if ((deriv1 * deriv0 < 0.0) && (fabs(slope2) > fabs(3.0 * deriv0))) {
            slope2 = 3.0 * deriv0;
        }
    }
    const double result = y2 * P.sh_term / P.h1_3 + y1 * (P.h1_3 - P.sh_term) / P.h1_3 +
                          slope2 * P.s_2 * P.sh_minus / P.h1_2 +
                          slope1 * P.s * P.sh_minus * P.sh_minus / P.h1_2;
    if (want) *deriv = slope1 * (1.0 - P.v) + slope2 * P.v;
    return result;
}

/* edge limiting and find_index on every axis (gen_grid.h:83-110) */
template <int NDIM>
WQ_HD void grid_locate(const GridDev& g, const double* location, int* index, double* loc) {
    for (int d = 0; d < NDIM; ++d) loc[d] = location[d];
    for (int d = 0; d < NDIM; ++d) {
        const AxisDev& ax = g.ax[d];
        if (g.edge[d]) {
            const double a = ax.x[0];
            const double b = ax.x[ax.n - 1];
            const double sign = (ax.inc[0] < 0) ? -1.0 : 1.0;
            const double dd = loc[d] * sign;
            if (dd <= a * sign) {
                loc[d] = a;
                index[d] = 0;
            } else if (dd >= b * sign) {
                loc[d] = b;
                index[d] = ax.n - 2;
            } else {
                index[d] = axis_find(ax, loc[d]);
            }
        } else {
            index[d] = axis_find(ax, loc[d]);
        }
    }
}

template <int NDIM>
WQ_HD double grid_pchip0(const GridDev& g, const double* location, double* dv) {
    int index[NDIM];
    double loc[NDIM];
    grid_locate<NDIM>(g, location, index, loc);
    const double* D = g.data;
    const AxisDev& a0 = g.ax[0];
    const int k = index[0];
    Pchip0 P;
    pchip0_setup(a0, k, loc[0], P);
    const int km = k >= 1 ? k - 1 : k;
    const int kp = k + 2 <= a0.n - 1 ? k + 2 : k + 1;
    const bool want = dv != nullptr;
    /* rows km, k, k+1, kp of axis 0 at axis-0 stride st, from offset o */
    auto corner = [&](size_t o, size_t st, double* d0) {
        double y0 = D[o + st * (size_t)km], y1 = D[o + st * (size_t)k];
        double y2 = D[o + st * (size_t)(k + 1)], y3 = D[o + st * (size_t)kp];
        if (!P.lo_in) y0 = y1;
        if (!P.hi_in) y3 = y2;
        return pchip0_corner(P, y0, y1, y2, y3, want, d0);
    };
    double u, h;
    if (NDIM == 1) {
        double d0 = 0.0;
        const double r = corner(0, 1, &d0);
        if (dv) dv[0] = d0;
        return r;
    }
    if (NDIM == 2) {
        const size_t n1 = (size_t)g.ax[1].n;
        double da = 0.0, db = 0.0;
        const double a = corner((size_t)index[1], n1, &da);
        const double b = corner((size_t)index[1] + 1, n1, &db);
        const double r = lin1(g, 1, index, loc, a, b, &u, &h);
        if (dv) {
            dv[1] = (b - a) / h;
            dv[0] = da * (1.0 - u) + db * u;
        }
        return r;
    }
    /* NDIM == 3: outer axis 2, then axis 1, innermost axis 0 (pchip) */
    const size_t n1 = (size_t)g.ax[1].n, n2 = (size_t)g.ax[2].n;
    const size_t st = n1 * n2;
    const int i1 = index[1], i2 = index[2];
    double u1, h1;
    auto plane = [&](int j, double* d1, double* d0) {
        double da = 0.0, db = 0.0;
        const double va = corner((size_t)j + n2 * (size_t)i1, st, &da);
        const double vb = corner((size_t)j + n2 * (size_t)(i1 + 1), st, &db);
        const double r = lin1(g, 1, index, loc, va, vb, &u1, &h1);
        *d1 = (vb - va) / h1;
        *d0 = da * (1.0 - u1) + db * u1;
        return r;
    };
    double d1a, d1b, d0a, d0b;
    const double pa = plane(i2, &d1a, &d0a);
    const double pb = plane(i2 + 1, &d1b, &d0b);
    const double r = lin1(g, 2, index, loc, pa, pb, &u, &h);
    if (dv) {
        dv[2] = (pb - pa) / h;
        dv[1] = d1a * (1.0 - u) + d1b * u;
        dv[0] = d0b;
    }
    return r;
}

#if WQ3D_WITH_GRID
/* grid evaluation: the unrolled linear and pchip-in-axis-0 paths inline,
 * others out of line */
WQ_HD double grid_value(const GridDev& g, const double* location, double* dv);

static WQ_NOINL double grid_eval(const GridDev& g, const double* location, double* dv) {
    switch (g.ndim) {
        case 1:
            return grid_interpolate<1>(g, location, dv);
        case 2:
            return grid_interpolate<2>(g, location, dv);
        default:
            return grid_interpolate<3>(g, location, dv);
    }
}

WQ_HD double grid_value(const GridDev& g, const double* location, double* dv) {
    if (g.all_linear) {
        switch (g.ndim) {
            case 1:
                return grid_linear<1>(g, location, dv);
            case 2:
                return grid_linear<2>(g, location, dv);
            default:
                return grid_linear<3>(g, location, dv);
        }
    }
    if (g.pchip0) {
        switch (g.ndim) {
            case 1:
                return grid_pchip0<1>(g, location, dv);
            case 2:
                return grid_pchip0<2>(g, location, dv);
            default:
                return grid_pchip0<3>(g, location, dv);
        }
    }
    return grid_eval(g, location, dv);
}
#endif  // WQ3D_WITH_GRID

struct BoundaryDev {
    int kind;
    double height;      /* flat and slope: _height */
    double normal[3];   /* rho, theta, phi */
    double loc_theta;   /* slope: _location */
    double loc_phi;
    double slope_a;     /* slope: sin(loc.theta) * tan(beta) (host precomputed) */
    double slope_b;     /* slope: tan(alpha)                 (host precomputed) */
    LossDev loss;
    GridDev grid;
};

struct ProfileDev {
    int kind;
    double p[4];
    double munk_k;      /* (-eps * speed * 2) / scale */
    double n2_factor;   /* 2 g0 / c0 */
    int flat_earth;
    int atten;
    double atten_coef;
    GridDev grid;
};

struct OceanDev {
    ProfileDev prof;
    BoundaryDev surf;
    BoundaryDev bot;
    int nvol;                        /* volume scattering layers          */
    double vol_rho[WQ3D_MAX_VOLUME]; /* volume_flat::_rho (volume_flat.h:32-37) */
};

/* to_radians / to_degrees of the reference's math_traits */
WQ_HD double deg2rad(double t) { return t * (M_PI / 180.0); }
WQ_HD double rad2deg(double t) { return t * (180.0 / M_PI); }

/* ------------------------------------------------------------------ */
/* sound speed: profile_{linear,munk,catenary,n2}.cc + adjust_speed     */
/* ------------------------------------------------------------------ */
WQ_HD void sound_speed(const ProfileDev& pr, double R, double rho, double theta,
                       double phi, double* c, double* g) {
    const double alt = rho - R;
    double cc, gr, gt = 0.0, gp = 0.0;
    switch (pr.kind) {
#if WQ3D_WITH_GRID
        case WQ3D_PROFILE_GRID: { /* profile_grid.h:68-130 */
            const double loc[3] = {rho, theta, phi};
            double dv[3] = {0.0, 0.0, 0.0};
            cc = grid_value(pr.grid, loc, dv);
            gr = dv[0];
            if (pr.grid.ndim >= 2) gt = dv[1];
            if (pr.grid.ndim >= 3) gp = dv[2];
            break;
        }
#endif
        case WQ3D_PROFILE_LINEAR: { /* profile_linear.cc:14-40 */
            const double z = -alt;
            if (z < pr.p[2]) {
                cc = pr.p[0] + pr.p[1] * z;
                gr = -pr.p[1];
            } else {
                cc = pr.p[0] + pr.p[1] * pr.p[2] + pr.p[3] * (z - pr.p[2]);
                gr = -pr.p[3];
            }
            break;
        }
        case WQ3D_PROFILE_MUNK: { /* profile_munk.cc:19-32 */
            const double z = 2.0 * (-alt - pr.p[0]) / pr.p[1];
            const double e = exp(-z);
            cc = (((z - 1.0) + e) * pr.p[3] + 1.0) * pr.p[2];
            gr = (1.0 - e) * pr.munk_k;
            break;
        }
        case WQ3D_PROFILE_CATENARY: { /* profile_catenary.cc:14-29 */
            const double x = (alt + pr.p[2]) / (-pr.p[1]);
            cc = pr.p[0] * cosh(x);
            gr = -sinh(x) * (pr.p[0] / pr.p[1]);
            break;
        }
        case WQ3D_PROFILE_N2: { /* profile_n2.cc:14-24 */
            cc = pr.p[0] / sqrt(1.0 - alt * pr.n2_factor);
            gr = pow(cc, 3.0) * pr.n2_factor / (2.0 * pr.p[0] * pr.p[0]);
            break;
        }
        default:
            cc = 1500.0;
            gr = 0.0;
    }
    if (pr.flat_earth) { /* profile_model.cc:14-26 */
        gr = (gr * rho + cc) / R;
        cc = cc * rho / R;
    }
    *c = cc;
    g[0] = gr;
    g[1] = gt;
    g[2] = gp;
}

/* ------------------------------------------------------------------ */
/* boundary height: boundary_flat.cc:39-63, boundary_slope.cc:55-68     */
/* ------------------------------------------------------------------ */
WQ_HD double boundary_height(const BoundaryDev& b, double theta, double phi) {
    if (b.kind == WQ3D_BOUNDARY_SLOPE) {
        return b.height * (1.0 + b.slope_a * (phi - b.loc_phi)) *
               (1.0 + b.slope_b * (theta - b.loc_theta));
    }
#if WQ3D_WITH_GRID
    if (b.kind == WQ3D_BOUNDARY_GRID) { /* boundary_grid.h:150-196 */
        const double loc[2] = {theta, phi};
        return grid_value(b.grid, loc, nullptr);
    }
#endif
    return b.height;
}

/* boundary height and unit normal (boundary_model::height with a normal):
 * flat and slope normals are constant; a grid's comes from the height
 * gradient (boundary_grid.h:150-196) */
WQ_HD double boundary_height_normal(const BoundaryDev& b, double theta, double phi, double* nrm) {
#if WQ3D_WITH_GRID
    if (b.kind == WQ3D_BOUNDARY_GRID) {
        const double loc[2] = {theta, phi};
        double grad[2] = {0.0, 0.0};
        const double rho = grid_value(b.grid, loc, grad);
        if (b.grid.ndim == 1) {
            const double t = -grad[0] / rho;
            const double N = sqrt(1 + t * t);
            nrm[0] = 1.0 / N;
            nrm[1] = t / N;
            nrm[2] = 0.0;
        } else {
            const double t = -grad[0] / rho;
            const double p = -grad[1] / (rho * sin(theta));
            const double N = sqrt(1 + t * t + p * p);
            nrm[0] = 1.0 / N;
            nrm[1] = t / N;
            nrm[2] = p / N;
        }
        return rho;
    }
#endif
    nrm[0] = b.normal[0];
    nrm[1] = b.normal[1];
    nrm[2] = b.normal[2];
    return boundary_height(b, theta, phi);
}

/* ------------------------------------------------------------------ */
/* small complex arithmetic for the Rayleigh model                      */
/* ------------------------------------------------------------------ */
struct cplx {
    double re, im;
};
WQ_HD cplx cmul(cplx a, cplx b) {
    return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
WQ_HD cplx cscale(cplx a, double s) { return cplx{a.re * s, a.im * s}; }
WQ_HD cplx csub_rc(double a, cplx b) { return cplx{a - b.re, -b.im}; }
/* complex division by Smith's method (R. L. Smith, CACM 5(8), 1962) */
WQ_HD cplx cdiv(cplx a, cplx b) {
    if (fabs(b.re) >= fabs(b.im)) {
        const double r = b.im / b.re;
        const double d = b.re + b.im * r;
        return cplx{(a.re + a.im * r) / d, (a.im - a.re * r) / d};
    }
    const double r = b.re / b.im;
    const double d = b.re * r + b.im;
    return cplx{(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}
/* principal square root (Kahan's formulation of the half-angle method) */
WQ_HD cplx csqrt_(cplx z) {
    if (z.re == 0.0 && z.im == 0.0) return cplx{0.0, z.im};
    const double t = sqrt(0.5 * (fabs(z.re) + hypot(z.re, z.im)));
    if (z.re >= 0.0) return cplx{t, z.im / (2.0 * t)};
    return cplx{fabs(z.im) / (2.0 * t), copysign(t, z.im)};
}

/* impedance (reflect_loss_rayleigh.cc:129-144) */
WQ_HD cplx rl_impedance(double density, double speed, double att,
                        double sin_angle, cplx* cosA, bool shear) {
    const cplx c{speed, -att * speed};
    const cplx sinA = cscale(c, sin_angle / 1.0);
    cplx sa{sinA.re / 1500.0, sinA.im / 1500.0};
    *cosA = csqrt_(csub_rc(1.0, cmul(sa, sa)));
    if (shear) return cdiv(cscale(c, density), *cosA);
    return cdiv(*cosA, cscale(c, density));
}

/* reflection loss in dB and phase (rad) at a grazing angle, frequency
 * independent part; Eckart is evaluated per frequency by the caller.
 * reflect_loss_constant.h:42-52, reflect_loss_rayleigh.cc:83-124 */
WQ_HD void reflect_loss_scalar(const LossDev& L, double angle, double* amp,
                               double* ph) {
    if (L.kind == WQ3D_LOSS_RAYLEIGH) {
        if (angle >= M_PI_2) angle = M_PI_2 - 1e-10;
        angle = M_PI_2 - angle;
        const double Zw = cos(angle) / (1500.0 * 1000.0);
        const double s = sin(angle);
        cplx cosAp, cosAs;
        cplx Zb = rl_impedance(L.rl_den, L.rl_spd, L.rl_att, s, &cosAp, false);
        if (L.rl_shr != 0.0 || L.rl_satt != 0.0) {
            const cplx Zs = rl_impedance(L.rl_den, L.rl_shr, L.rl_satt, s, &cosAs, true);
            const cplx sinAs = csqrt_(csub_rc(1.0, cmul(cosAs, cosAs)));
            const cplx cos2As = csub_rc(0.0, csub_rc(1.0, cscale(cmul(cosAs, cosAs), 2.0)));
            const cplx sin2As = cscale(cmul(sinAs, cosAs), 2.0);
            const cplx one{1.0, 0.0};
            const cplx a = cmul(cmul(cdiv(one, Zb), cos2As), cos2As);
            const cplx b = cmul(cmul(Zs, sin2As), sin2As);
            Zb = cdiv(one, cplx{a.re + b.re, a.im + b.im});
        }
        const cplx num{Zb.re - Zw, Zb.im};
        const cplx den{Zb.re + Zw, Zb.im};
        const cplx Rc = cdiv(num, den);
        *amp = -20.0 * log10(hypot(Rc.re, Rc.im));
        *ph = atan2(Rc.im, Rc.re);
        return;
    }
    *amp = L.p[0];
    *ph = L.p[1];
}

/* Derivatives of reflect_loss_scalar's Rayleigh loss (dB) with respect
 * to the bottom's density ratio, speed ratio and attenuation (dB per
 * wavelength) at a fixed grazing angle.  With R = (Zb - Zw)/(Zb + Zw) and
 * loss = -20 log10 |R|, d loss = -(20/ln 10) Re(2 Zw dZb / ((Zb + Zw)(Zb - Zw))),
 * where Zb = cos A / (c rho_b) gives dZb/d rho_b = -Zb / rho_b and
 * d ln Zb / d ln c = -1 / cos^2 A (sin A = sin(angle) c / c_water).  Other
 * loss models do not depend on these parameters (zero); a Rayleigh bottom
 * with shear is not differentiated here (NaN). */
WQ_HD void reflect_loss_rayleigh_grad(const LossDev& L, double angle, double* d) {
    d[0] = d[1] = d[2] = 0.0;
    if (L.kind != WQ3D_LOSS_RAYLEIGH) return;
    if (L.rl_shr != 0.0 || L.rl_satt != 0.0) {
        d[0] = d[1] = d[2] = NAN;
        return;
    }
    if (angle >= M_PI_2) angle = M_PI_2 - 1e-10;
    angle = M_PI_2 - angle;
    const double Zw = cos(angle) / (1500.0 * 1000.0);
    cplx cosA;
    const cplx Zb = rl_impedance(L.rl_den, L.rl_spd, L.rl_att, sin(angle), &cosA, false);
    const cplx base = cdiv(cscale(Zb, 2.0 * Zw), cmul(cplx{Zb.re + Zw, Zb.im}, cplx{Zb.re - Zw, Zb.im}));
    const double k = -20.0 * M_LOG10E;
    /* density ratio p0: rho_b = 1000 p0 */
    d[0] = k * (base.re * (-1000.0 / L.rl_den));
    /* speed ratio p1: c = 1500 p1 (1 - i att), d ln c / d p1 = 1 / p1 */
    const cplx g_c = cdiv(cplx{-1.0, 0.0}, cmul(cosA, cosA));
    const cplx gv = cscale(g_c, 1500.0 / L.rl_spd);
    d[1] = k * cmul(base, gv).re;
    /* attenuation p2: att = p2 K, d ln c / d p2 = -i K / (1 - i att) */
    const double K = 1.0 / (20.0 * M_LOG10E * (2.0 * M_PI));
    const cplx dlnc = cdiv(cplx{0.0, -K}, cplx{1.0, -L.rl_att});
    d[2] = k * cmul(base, cmul(g_c, dlnc)).re;
}

/* ------------------------------------------------------------------ */
/* wave_front::update derivative terms (wave_front.cc:133-171)          */
/* ------------------------------------------------------------------ */
WQ_HD void ray_derivs(double c, double sg_r, double sg_t, double sg_p,
                      const double* pos, const double* nd, double* pg,
                      double* ng, double* sin_out) {
    const double dcc_r = sg_r / c;
    const double dcc_t = sg_t / c;
    const double dcc_p = sg_p / c;
    const double st = sin(pos[1]);
    const double ct = cos(pos[1]) / st;
    const double c2 = c * c;
    pg[0] = c2 * nd[0];
    const double c2r = c2 / pos[0];
    pg[1] = c2r * nd[1];
    pg[2] = (c2r / st) * nd[2];
    ng[0] = c2r * (nd[1] * nd[1] + nd[2] * nd[2]) - dcc_r;
    ng[1] = (-c2r) * (nd[0] * nd[1] - (nd[2] * nd[2]) * ct) - dcc_t / pos[0];
    ng[2] = (-c2r) * (nd[2] * (nd[0] + nd[1] * ct)) - dcc_p / (pos[0] * st);
    *sin_out = st;
}

/* ------------------------------------------------------------------ */
/* the FP32 propagation form (WQ3D_FP32): sound speed, gradient and ray  */
/* derivatives of wave_front::update in single precision                */
/* ------------------------------------------------------------------ */
/* The analytic profiles at the altitude offset alt = rho - R (formed in
 * FP64, then rounded: 0.5 mm at 5 km), in single precision; a gridded
 * profile is interpolated in FP64 and rounded. */
WQ_HD void sound_speed_f32(const ProfileDev& pr, double R, double rho, double theta, double phi, float* c,
                           float* g) {
    const float alt = (float)(rho - R);
    float cc, gr, gt = 0.0f, gp = 0.0f;
    switch (pr.kind) {
#if WQ3D_WITH_GRID
        case WQ3D_PROFILE_GRID: {
            double c64, g64[3];
            sound_speed(pr, R, rho, theta, phi, &c64, g64);
            *c = (float)c64;
            g[0] = (float)g64[0];
            g[1] = (float)g64[1];
            g[2] = (float)g64[2];
            return;
        }
#endif
        case WQ3D_PROFILE_LINEAR: {
            const float z = -alt;
            if (z < (float)pr.p[2]) {
                cc = (float)pr.p[0] + (float)pr.p[1] * z;
                gr = -(float)pr.p[1];
            } else {
                cc = (float)(pr.p[0] + pr.p[1] * pr.p[2]) + (float)pr.p[3] * (z - (float)pr.p[2]);
                gr = -(float)pr.p[3];
            }
            break;
        }
        case WQ3D_PROFILE_MUNK: {
            const float z = 2.0f * (-alt - (float)pr.p[0]) / (float)pr.p[1];
            const float e = expf(-z);
            cc = (((z - 1.0f) + e) * (float)pr.p[3] + 1.0f) * (float)pr.p[2];
            gr = (1.0f - e) * (float)pr.munk_k;
            break;
        }
        case WQ3D_PROFILE_CATENARY: {
            const float x = (alt + (float)pr.p[2]) / (-(float)pr.p[1]);
            cc = (float)pr.p[0] * coshf(x);
            gr = -sinhf(x) * (float)(pr.p[0] / pr.p[1]);
            break;
        }
        case WQ3D_PROFILE_N2: {
            const float f = (float)pr.n2_factor;
            cc = (float)pr.p[0] / sqrtf(1.0f - alt * f);
            gr = cc * cc * cc * f / (float)(2.0 * pr.p[0] * pr.p[0]);
            break;
        }
        default:
            cc = 1500.0f;
            gr = 0.0f;
    }
    if (pr.flat_earth) {
        gr = gr * (float)(rho / R) + cc / (float)R;
        cc = cc * (float)(rho / R);
    }
    *c = cc;
    g[0] = gr;
    g[1] = gt;
    g[2] = gp;
}

/* ray_derivs in single precision (rho enters only as 1/rho factors, so its
 * rounding is relative) */
WQ_HD void ray_derivs_f32(float c, const float* sg, const double* pos, const double* nd, double* pg, double* ng) {
    const float rho = (float)pos[0];
    const float dcc_r = sg[0] / c;
    const float dcc_t = sg[1] / c;
    const float dcc_p = sg[2] / c;
    const float th = (float)pos[1];
    const float st = sinf(th);
    const float ct = cosf(th) / st;
    const float n0 = (float)nd[0], n1 = (float)nd[1], n2 = (float)nd[2];
    const float c2 = c * c;
    const float c2r = c2 / rho;
    pg[0] = (double)(c2 * n0);
    pg[1] = (double)(c2r * n1);
    pg[2] = (double)((c2r / st) * n2);
    ng[0] = (double)(c2r * (n1 * n1 + n2 * n2) - dcc_r);
    ng[1] = (double)((-c2r) * (n0 * n1 - (n2 * n2) * ct) - dcc_t / rho);
    ng[2] = (double)((-c2r) * (n2 * (n0 + n1 * ct)) - dcc_p / (rho * st));
}

/* wave_front::compute_target_distance for one (ray, target) pair
 * (wave_front.cc:222-236).  rho2 = rho*rho, two_R = 2*target rho,
 * R2 = target rho squared: the same values the reference forms. */
WQ_HD double target_distance2(double rho, double rho2, double theta,
                              double phi, double sin_t, double tgt_theta,
                              double tgt_phi, double tgt_sin, double R2,
                              double two_R) {
    const double a = 0.5 * (theta - tgt_theta);
    const double b = 0.5 * (phi - tgt_phi);
    const double inner = 1.0 - 2.0 * (a * a + tgt_sin * (sin_t * (b * b)));
    return fabs(rho2 + R2 - two_R * (rho * inner));
}

/* types/wvector1.cc distance2 */
WQ_HD double wdist2(double r1, double t1, double p1, double r2, double t2,
                    double p2) {
    const double st = sin(0.5 * (t1 - t2));
    const double sp = sin(0.5 * (p1 - p2));
    const double dn = 1.0 - 2.0 * (st * st + sin(t1) * sin(t2) * sp * sp);
    const double dot = r1 * r2 * dn;
    return fabs(r1 * r1 + r2 * r2 - 2.0 * dot);
}

}  // namespace wq3d
