/*
 * wq3d_adjoint.cuh -- reverse (adjoint) sweep of the propagation:
 * gradients of eigenray TL and travel time with respect to the nodes of a
 * piecewise-linear sound-speed profile (profile_grid<1>, linear in depth),
 * at the forward pass's frozen eigenray topology.
 *
 * Included at the end of wq3d_kernels.cu (its full build), so the recompute
 * calls the engine's own step functions and retraces the forward bit for
 * bit.
 *
 * Per ray, the state between two steps is S_m = (pos, ndir) of the prev,
 * curr and next fronts as the eigenray search of step m reads them (before
 * step m+1's reflections), plus the first frequency's attenuation on those
 * fronts.  Rays evolve independently: S_{m+1} = Phi_m(S_m; c), where Phi_m
 * is the reflection chain of wave_queue::detect_reflections (if the ray
 * reflects), the AB3 step (ode_integ.cc:131-186), wave_front::update and
 * the absorption of the new front.  An eigenray of step m is a function of
 * a few rays' S_m (beam-walk cell widths, the attenuation it interpolates)
 * and of the cpa terms of prev / curr / next, which are the next-front
 * positions of S_{m-2}, S_{m-1}, S_m (distance2 is never recomputed after a
 * reflection, wave_front.cc:222-236).
 *
 * Forward with recording:
 *   k_adj_checkpoint  S_m of every ray at m = 0, K, 2K, ...
 *   k_eigenray_jac    per eigenray record of the step: d TL / d (27 cube
 *                     values), d T / d cube, d TL / d (each beam-walk cell
 *                     width), d TL / d (the two attenuations), d TL / d
 *                     spread2 -- build_eigenray, compute_offsets and
 *                     spreading_hybrid_gaussian restated for one warp, the
 *                     walks differentiated by hand in reverse, the Taylor
 *                     fit by one dual-number lane per cube value.
 * Backward, per checkpoint segment [m0, m1), last segment first:
 *   k_adj_recompute   S_m0 .. S_m1-1 of every ray still seeded, from the
 *                     checkpoint, with the engine's step functions; each
 *                     step's reflection chain recorded
 *   k_adj_expand      each eigenray's partials times its weights, taken to
 *                     the rays' S_m (cube values through the target
 *                     distance, widths through the ray positions)
 *   k_adj_reverse     lambda_m = Phi_m^T lambda_{m+1} + seeds_m per ray; the
 *                     local Jacobian of Phi_m from dual numbers over S_m and
 *                     the profile nodes the step can reach (three passes of
 *                     eight directions); node gradients reduced per warp
 *   k_adj_startup     lambda_0 through the RK3 start-up (wave_queue.cc:
 *                     114-150) and init_wave's 1/c(source)
 */
#pragma once

#include "wq3d_dual.cuh"

namespace wq3d {

#ifdef WQ3D_ADJOINT_IMPL
namespace {

/* ------------------------------------------------------------------ */
/* state layout                                                        */
/* ------------------------------------------------------------------ */
/* component c of ray i in an [..][c][n] block */
__device__ __forceinline__ double& sref(double* base, int c, int n, int i) { return base[(size_t)c * n + i]; }

/* ------------------------------------------------------------------ */
/* templated restatements of the step functions                        */
/* (value parts follow the engine's operation order exactly)           */
/* ------------------------------------------------------------------ */
template <class T>
struct RayT {
    T pos[3], pg[3], nd[3], ng[3], c, sg[3], dist;
};

/* profile nodes [k0, k0 + w) carry dual directions base + (k - k0) */
struct ParamWin {
    int k0, w, base;
};

template <class T>
struct NodeOf;
template <>
struct NodeOf<double> {
    __device__ static double get(const double* data, int k, const ParamWin&, bool&) { return data[k]; }
};
template <int N>
struct NodeOf<Dual<N>> {
    __device__ static Dual<N> get(const double* data, int k, const ParamWin& pw, bool& ok) {
        const int j = k - pw.k0;
        if (j < 0 || j >= pw.w) {
            ok = false;
            return Dual<N>(data[k]);
        }
        return Dual<N>::var(data[k], pw.base + j);
    }
};

/* profile_grid<1>, linear in depth with edge limiting (grid_linear<1>),
 * and profile_model::adjust_speed's flat-earth correction */
template <class T>
__device__ void ssp_t(const QueueDev& q, const T& rho, const ParamWin& pw, bool& ok, T& c, T* g) {
    const ProfileDev& pr = q.oc.prof;
    const GridDev& gd = pr.grid;
    const AxisDev& ax = gd.ax[0];
    int k;
    T loc;
    const double r = val(rho);
    if (gd.edge[0]) {
        const double a = ax.x[0];
        const double b = ax.x[ax.n - 1];
        const double sign = (ax.inc[0] < 0) ? -1.0 : 1.0;
        const double dd = r * sign;
        if (dd <= a * sign) {
            loc = T(a);
            k = 0;
        } else if (dd >= b * sign) {
            loc = T(b);
            k = ax.n - 2;
        } else {
            k = axis_find(ax, r);
            loc = rho;
        }
    } else {
        k = axis_find(ax, r);
        loc = rho;
    }
    const T A = NodeOf<T>::get(gd.data, k, pw, ok);
    const T B = NodeOf<T>::get(gd.data, k + 1, pw, ok);
    const double h = axis_inc(ax, k);
    const T u = (loc - ax.x[k]) / h;
    T cc = A * (1.0 - u) + B * u;
    T gr = (B - A) / h;
    if (pr.flat_earth) {
        gr = (gr * rho + cc) / q.R;
        cc = cc * rho / q.R;
    }
    c = cc;
    g[0] = gr;
    g[1] = T(0.0);
    g[2] = T(0.0);
}

/* the interval index of a depth (the k of ssp_t) */
__device__ __forceinline__ int ssp_interval(const QueueDev& q, double r) {
    const GridDev& gd = q.oc.prof.grid;
    const AxisDev& ax = gd.ax[0];
    if (gd.edge[0]) {
        const double sign = (ax.inc[0] < 0) ? -1.0 : 1.0;
        if (r * sign <= ax.x[0] * sign) return 0;
        if (r * sign >= ax.x[ax.n - 1] * sign) return ax.n - 2;
    }
    return axis_find(ax, r);
}

__device__ __forceinline__ ParamWin window_at(const QueueDev& q, double r, int base) {
    const int np = q.oc.prof.grid.ax[0].n;
    ParamWin pw;
    pw.w = min(ADJ_W, np);
    pw.k0 = min(max(ssp_interval(q, r) - 2, 0), np - pw.w);
    pw.base = base;
    return pw;
}

template <class T>
__device__ __forceinline__ void ray_derivs_t(const T& c, const T& sg_r, const T& sg_t, const T& sg_p,
                                             const T* pos, const T* nd, T* pg, T* ng) {
    const T dcc_r = sg_r / c;
    const T dcc_t = sg_t / c;
    const T dcc_p = sg_p / c;
    const T st = sin(pos[1]);
    const T ct = cos(pos[1]) / st;
    const T c2 = c * c;
    pg[0] = c2 * nd[0];
    const T c2r = c2 / pos[0];
    pg[1] = c2r * nd[1];
    pg[2] = (c2r / st) * nd[2];
    ng[0] = c2r * (nd[1] * nd[1] + nd[2] * nd[2]) - dcc_r;
    ng[1] = (-c2r) * (nd[0] * nd[1] - (nd[2] * nd[2]) * ct) - dcc_t / pos[0];
    ng[2] = (-c2r) * (nd[2] * (nd[0] + nd[1] * ct)) - dcc_p / (pos[0] * st);
}

template <class T>
__device__ __forceinline__ void update_t(const QueueDev& q, RayT<T>& y, const ParamWin& pw, bool& ok) {
    ssp_t(q, y.pos[0], pw, ok, y.c, y.sg);
    ray_derivs_t(y.c, y.sg[0], y.sg[1], y.sg[2], y.pos, y.nd, y.pg, y.ng);
}

template <class T>
__device__ __forceinline__ void rk1_t(double h, const RayT<T>& y0, RayT<T>& y1) {
    for (int k = 0; k < 3; ++k) {
        y1.pos[k] = y0.pos[k] + 0.5 * h * y0.pg[k];
        y1.nd[k] = y0.nd[k] + 0.5 * h * y0.ng[k];
    }
}
template <class T>
__device__ __forceinline__ void rk2_t(double h, const RayT<T>& y0, const RayT<T>& y1, RayT<T>& y2) {
    for (int k = 0; k < 3; ++k) {
        y2.pos[k] = y0.pos[k] + h * (2.0 * y1.pg[k] - y0.pg[k]);
        y2.nd[k] = y0.nd[k] + h * (2.0 * y1.ng[k] - y0.ng[k]);
    }
}
template <class T>
__device__ __forceinline__ void rk3_t(double h, const RayT<T>& y0, const RayT<T>& y1, const RayT<T>& y2,
                                      RayT<T>& y3) {
    T p[3], d[3];
    for (int k = 0; k < 3; ++k) {
        p[k] = y0.pos[k] + h / 6.0 * (y0.pg[k] + 4.0 * y1.pg[k] + y2.pg[k]);
        d[k] = y0.nd[k] + h / 6.0 * (y0.ng[k] + 4.0 * y1.ng[k] + y2.ng[k]);
    }
    for (int k = 0; k < 3; ++k) {
        y3.pos[k] = p[k];
        y3.nd[k] = d[k];
    }
}
template <class T>
__device__ __forceinline__ void ab3_t(double h, const RayT<T>& y0, const RayT<T>& y1, const RayT<T>& y2,
                                      RayT<T>& y3) {
    const double A2 = 23.0 / 12.0, A1 = 16.0 / 12.0, A0 = 5.0 / 12.0;
    T d[3];
    for (int k = 0; k < 3; ++k) d[k] = h * (A2 * y2.pg[k] - A1 * y1.pg[k] + A0 * y0.pg[k]);
    const T b = y2.pos[0] * d[1];
    const T cc = y2.pos[0] * (sin(y2.pos[1]) * d[2]);
    y3.dist = sqrt(d[0] * d[0] + b * b + cc * cc);
    for (int k = 0; k < 3; ++k) {
        y3.pos[k] = y2.pos[k] + d[k];
        y3.nd[k] = y2.nd[k] + h * (A2 * y2.ng[k] - A1 * y1.ng[k] + A0 * y0.ng[k]);
    }
}

template <class T>
struct LocalT {
    RayT<T> v, c, x;
    T att; /* first frequency's loss added to the next front */
};

template <class T>
__device__ void collision_t(const QueueDev& q, const LocalT<T>& L, const T& tw, T* pos, T* nd, T& speed) {
    const double dt = q.dt;
    const double time1 = 2.0 * dt;
    const double time2 = dt * dt;
    const T dtime2 = tw * tw;
    const T drho = (L.x.c - L.v.c) / time1;
    const T d2rho = (L.x.c + L.v.c - 2.0 * L.c.c) / time2;
    speed = L.c.c + drho * tw + 0.5 * d2rho * dtime2;
    for (int k = 0; k < 3; ++k) {
        const T v1 = (L.x.pos[k] - L.v.pos[k]) / time1;
        const T v2 = (L.x.pos[k] + L.v.pos[k] - 2.0 * L.c.pos[k]) / time2;
        pos[k] = L.c.pos[k] + v1 * tw + 0.5 * v2 * dtime2;
    }
    for (int k = 0; k < 3; ++k) {
        const T v1 = (L.x.nd[k] - L.v.nd[k]) / time1;
        const T v2 = (L.x.nd[k] + L.v.nd[k] - 2.0 * L.c.nd[k]) / time2;
        nd[k] = L.c.nd[k] + v1 * tw + 0.5 * v2 * dtime2;
    }
}

/* reflection_model::reflection_reinit on the private state (reinit_local) */
template <class T>
__device__ void reinit_t(const QueueDev& q, LocalT<T>& L, const T& tw, const T* pos, const T* nd,
                         const ParamWin& pw, bool& ok) {
    RayT<T> past1, prev1, curr1, next1, temp;
    for (int k = 0; k < 3; ++k) {
        temp.pos[k] = pos[k];
        temp.nd[k] = nd[k];
    }
    update_t(q, temp, pw, ok);
    const T mtw = -tw;
    /* rk with a dual step: the same forms with h a T */
    auto rk1 = [&](const T& h, const RayT<T>& y0, RayT<T>& y1) {
        for (int k = 0; k < 3; ++k) {
            y1.pos[k] = y0.pos[k] + 0.5 * h * y0.pg[k];
            y1.nd[k] = y0.nd[k] + 0.5 * h * y0.ng[k];
        }
    };
    auto rk2 = [&](const T& h, const RayT<T>& y0, const RayT<T>& y1, RayT<T>& y2) {
        for (int k = 0; k < 3; ++k) {
            y2.pos[k] = y0.pos[k] + h * (2.0 * y1.pg[k] - y0.pg[k]);
            y2.nd[k] = y0.nd[k] + h * (2.0 * y1.ng[k] - y0.ng[k]);
        }
    };
    auto rk3 = [&](const T& h, const RayT<T>& y0, const RayT<T>& y1, const RayT<T>& y2, RayT<T>& y3) {
        T p[3], d[3];
        for (int k = 0; k < 3; ++k) {
            p[k] = y0.pos[k] + h / 6.0 * (y0.pg[k] + 4.0 * y1.pg[k] + y2.pg[k]);
            d[k] = y0.nd[k] + h / 6.0 * (y0.ng[k] + 4.0 * y1.ng[k] + y2.ng[k]);
        }
        for (int k = 0; k < 3; ++k) {
            y3.pos[k] = p[k];
            y3.nd[k] = d[k];
        }
    };
    rk1(mtw, temp, next1);
    update_t(q, next1, pw, ok);
    rk2(mtw, temp, next1, past1);
    update_t(q, past1, pw, ok);
    rk3(mtw, temp, next1, past1, curr1);
    update_t(q, curr1, pw, ok);

    const double h = q.dt;
    rk1_t(-h, curr1, next1);
    update_t(q, next1, pw, ok);
    rk2_t(-h, curr1, next1, past1);
    update_t(q, past1, pw, ok);
    rk3_t(-h, curr1, next1, past1, prev1);
    update_t(q, prev1, pw, ok);

    rk1_t(-h, prev1, next1);
    update_t(q, next1, pw, ok);
    rk2_t(-h, prev1, next1, temp);
    rk3_t(-h, prev1, next1, temp, past1);
    update_t(q, past1, pw, ok);

    ab3_t(h, past1, prev1, curr1, next1);
    update_t(q, next1, pw, ok);
    L.c = curr1;
    L.v = prev1;
    L.x = next1;
}

/* d loss / d grazing of reflect_loss_scalar's fluid Rayleigh model: with
 * A = pi/2 - grazing, Zw = cos A / (rho_w c_w), Zb = cos A_b / (c rho_b),
 * cos A_b = sqrt(1 - (sin A c / c_w)^2), R = (Zb - Zw)/(Zb + Zw),
 * d loss = -20 log10(e) Re(d ln R) */
__device__ double rayleigh_dloss_dgrazing(const LossDev& L, double grazing) {
    if (grazing >= M_PI_2) return 0.0;
    const double A = M_PI_2 - grazing;
    const double sA = sin(A), cA = cos(A);
    const double Zw = cA / (1500.0 * 1000.0);
    const double dZw = sA / (1500.0 * 1000.0);
    cplx cosA;
    const cplx Zb = rl_impedance(L.rl_den, L.rl_spd, L.rl_att, sA, &cosA, false);
    const cplx c{L.rl_spd, -L.rl_att * L.rl_spd};
    /* d cosA / d grazing = (sA c^2 / c_w^2) cA / cosA */
    const cplx c2 = cmul(c, c);
    const cplx dcos = cdiv(cscale(c2, sA * cA / (1500.0 * 1500.0)), cosA);
    const cplx dZb = cdiv(dcos, cscale(c, L.rl_den));
    const cplx num{dZb.re - dZw, dZb.im};
    const cplx den{Zb.re - Zw, Zb.im};
    const cplx num2{dZb.re + dZw, dZb.im};
    const cplx den2{Zb.re + Zw, Zb.im};
    const cplx a = cdiv(num, den), b = cdiv(num2, den2);
    return -20.0 * M_LOG10E * (a.re - b.re);
}

/* the first frequency's reflection loss at a dual grazing angle */
template <class T>
__device__ T loss_t(const QueueDev& q, const LossDev& Lo, const T& grazing) {
    if (Lo.kind == WQ3D_LOSS_ECKART) {
        const double w2 = Lo.p[0] * Lo.p[0];
        const T x = q.freq[0] * w2 * sin(grazing);
        return 8.6e-9 * (x * x);
    }
    double amp0 = 0.0, ph0 = 0.0;
    const double g = val(grazing);
    reflect_loss_scalar(Lo, g, &amp0, &ph0);
    const double d = (Lo.kind == WQ3D_LOSS_RAYLEIGH) ? rayleigh_dloss_dgrazing(Lo, g) : 0.0;
    return amp0 + d * (grazing - g);
}

/* boundary_height / boundary_height_normal for flat and sloped boundaries */
template <class T>
__device__ T bheight_t(const BoundaryDev& b, const T& theta, const T& phi) {
    if (b.kind == WQ3D_BOUNDARY_SLOPE)
        return b.height * (1.0 + b.slope_a * (phi - b.loc_phi)) * (1.0 + b.slope_b * (theta - b.loc_theta));
    return T(b.height);
}

/* surface_local without notices: returns whether the ray reflected */
template <class T>
__device__ bool surface_t(const QueueDev& q, LocalT<T>& L, const ParamWin& pw, bool& ok) {
    T c = L.c.c;
    const T d = c * c * L.c.nd[0];
    const T tw = (val(d) == 0.0) ? T(0.0) : -(L.c.pos[0] - q.R) / d;
    T pos[3], nd[3];
    collision_t(q, L, tw, pos, nd, c);
    const T n1 = L.c.nd[1], n2 = L.c.nd[2];
    const T grazing = atan2(L.c.nd[0], sqrt(n1 * n1 + n2 * n2));
    if (val(grazing) <= 0.0) return false;
    L.att = L.att + loss_t(q, q.oc.surf.loss, grazing);
    nd[0] = -nd[0];
    reinit_t(q, L, tw, pos, nd, pw, ok);
    return true;
}

/* bottom_local without notices (flat and sloped bottoms) */
template <class T>
__device__ void bottom_t(const QueueDev& q, LocalT<T>& L, const T& depth, const ParamWin& pw, bool& ok) {
    const BoundaryDev& B = q.oc.bot;
    bool shallow = false;
    T position[3] = {L.c.pos[0], L.c.pos[1], L.c.pos[2]};
    T ndir[3] = {L.c.nd[0], L.c.nd[1], L.c.nd[2]};
    T c = L.c.c;
    T c2 = c * c;
    double nrm[3] = {B.normal[0], B.normal[1], B.normal[2]};
    T bottom_rho = bheight_t(B, position[1], position[2]);
    T height_water = position[0] - bottom_rho;
    const double TOO_SHALLOW = 300.0 * q.dt;
    if ((q.R - val(bottom_rho)) < TOO_SHALLOW) shallow = true;
    double N;
    if (shallow) {
        N = ::sqrt(nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        nrm[0] = 0.0;
        nrm[1] = nrm[1] / N;
        nrm[2] = nrm[2] / N;
    }
    ndir[0] = c2 * ndir[0];
    ndir[1] = c2 * ndir[1];
    ndir[2] = c2 * ndir[2];
    T dot_full = nrm[0] * ndir[0] + nrm[1] * ndir[1] + nrm[2] * ndir[2];
    const double MIN_REFLECT = 6.0;
    T max_dot = -fmax((height_water + depth) * nrm[0], MIN_REFLECT);
    if (val(dot_full) >= val(max_dot)) dot_full = max_dot;
    const T dot_water = -height_water * nrm[0];
    const T time_water = fmax(dot_water / dot_full, 0.0);

    collision_t(q, L, time_water, position, ndir, c);
    bottom_rho = bheight_t(B, position[1], position[2]);
    nrm[0] = B.normal[0];
    nrm[1] = B.normal[1];
    nrm[2] = B.normal[2];
    if (shallow) {
        N = ::sqrt(nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        nrm[0] = 0.0;
        nrm[1] = nrm[1] / N;
        nrm[2] = nrm[2] / N;
    }
    c2 = c * c;
    height_water = position[0] - bottom_rho;
    ndir[0] = c2 * ndir[0];
    ndir[1] = c2 * ndir[1];
    ndir[2] = c2 * ndir[2];
    dot_full = nrm[0] * ndir[0] + nrm[1] * ndir[1] + nrm[2] * ndir[2];
    max_dot = -fmax((height_water + depth) * nrm[0], MIN_REFLECT);
    if (val(dot_full) >= val(max_dot)) dot_full = max_dot;

    T grazing;
    if (val(dot_full) / val(c) >= 1.0) {
        grazing = T(-M_PI_2);
    } else if (val(dot_full) / val(c) <= -1.0) {
        grazing = T(M_PI_2);
    } else {
        grazing = asin(-dot_full / c);
    }
    L.att = L.att + loss_t(q, B.loss, grazing);
    dot_full = dot_full * 2.0;
    ndir[0] = ndir[0] - dot_full * nrm[0];
    ndir[1] = ndir[1] - dot_full * nrm[1];
    ndir[2] = ndir[2] - dot_full * nrm[2];
    const T NN = sqrt(ndir[0] * ndir[0] + ndir[1] * ndir[1] + ndir[2] * ndir[2]) * c;
    ndir[0] = ndir[0] / NN;
    ndir[1] = ndir[1] / NN;
    ndir[2] = ndir[2] / NN;
    reinit_t(q, L, time_water, position, ndir, pw, ok);
}

/* chain codes: bits 0-7 event kinds (1 bottom), bits 16-19 event count */
__device__ __forceinline__ uint32_t chain_add(uint32_t code, bool bottom) {
    const uint32_t n = (code >> 16) & 0xf;
    return ((n + 1) << 16) | (code & 0xffffu) | (bottom ? (1u << n) : 0u);
}

/* the reflection chain of k_reflect (wave_queue.cc:197-256) on T values;
 * returns the chain code, bit 31 set when it ran past 8 events */
template <class T>
__device__ uint32_t chain_t(const QueueDev& q, LocalT<T>& L, const ParamWin& pw, bool& ok) {
    uint32_t code = 0;
    int next_try = -1;
    auto depth_at = [&](const LocalT<T>& l) { return bheight_t(q.oc.bot, l.x.pos[1], l.x.pos[2]) - l.x.pos[0]; };
    if (val(L.x.pos[0]) - q.R > 0.0 && surface_t(q, L, pw, ok)) {
        code = chain_add(code, false);
        next_try = 0;
    } else {
        const T depth = depth_at(L);
        if (val(depth) > 0.0) {
            bottom_t(q, L, depth, pw, ok);
            code = chain_add(code, true);
            next_try = 1;
        }
    }
    if (next_try >= 0) {
        for (int it = 0; it < MAX_BOUNCE; ++it) {
            if (((code >> 16) & 0xf) >= 8) return code | 0x80000000u;
            if (next_try == 0) {
                const T depth = depth_at(L);
                if (!(val(depth) > 0.0)) break;
                bottom_t(q, L, depth, pw, ok);
                code = chain_add(code, true);
                next_try = 1;
            } else {
                if (!(val(L.x.pos[0]) - q.R > 0.0 && surface_t(q, L, pw, ok))) break;
                code = chain_add(code, false);
                next_try = 0;
            }
        }
    }
    return code;
}

/* ------------------------------------------------------------------ */
/* compute_offsets (wave_queue.cc:708-924) on T cube values             */
/* ------------------------------------------------------------------ */
template <class T>
__device__ void taylor_t(const T* v, const double* delta, T& center, T* g, T h[3][3]) {
    /* v[m * 9 + nd * 3 + na], as make_taylor_coeff's v[m][nd][na] */
    auto V = [&](int m, int a, int b) -> const T& { return v[m * 9 + a * 3 + b]; };
    const double d0 = 2.0 * delta[0];
    const double d1 = 2.0 * delta[1];
    const double d2 = 2.0 * delta[2];
    center = V(1, 1, 1);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) h[r][c] = T(0.0);
    h[0][0] = (V(2, 1, 1) + V(0, 1, 1) - 2.0 * center) / (delta[0] * delta[0]);
    h[1][1] = (V(1, 2, 1) + V(1, 0, 1) - 2.0 * center) / (delta[1] * delta[1]);
    h[2][2] = (V(1, 1, 2) + V(1, 1, 0) - 2.0 * center) / (delta[2] * delta[2]);
    g[0] = (V(2, 0, 1) - V(0, 0, 1)) / d0;
    g[2] = (V(2, 2, 1) - V(0, 2, 1)) / d0;
    h[0][1] = (g[2] - g[0]) / d1;
    h[1][0] = h[0][1];
    g[0] = (V(2, 1, 0) - V(0, 1, 0)) / d0;
    g[2] = (V(2, 1, 2) - V(0, 1, 2)) / d0;
    h[0][2] = (g[2] - g[0]) / d2;
    h[2][0] = h[0][2];
    g[0] = (V(1, 2, 0) - V(1, 0, 0)) / d1;
    g[2] = (V(1, 2, 2) - V(1, 0, 2)) / d1;
    h[1][2] = (g[2] - g[0]) / d2;
    h[2][1] = h[1][2];
    g[0] = (V(2, 1, 1) - V(0, 1, 1)) / d0;
    g[1] = (V(1, 2, 1) - V(1, 0, 1)) / d1;
    g[2] = (V(1, 1, 2) - V(1, 1, 0)) / d2;
}

template <class T>
__device__ __forceinline__ double norm2_v(const T* g) {
    double t = 0.0;
    t += ::fabs(val(g[0])) * ::fabs(val(g[0]));
    t += ::fabs(val(g[1])) * ::fabs(val(g[1]));
    t += ::fabs(val(g[2])) * ::fabs(val(g[2]));
    return ::sqrt(t);
}

template <class T>
__device__ __forceinline__ void matvec_t(const T m[3][3], const T* x, T* y) {
    for (int r = 0; r < 3; ++r) {
        T t = T(0.0);
        t = t + m[r][0] * x[0];
        t = t + m[r][1] * x[1];
        t = t + m[r][2] * x[2];
        y[r] = t;
    }
}

/* The offsets and distances of build_eigenray for one CPA.  unstable_in is
 * the neighbour-count test; flip < 0 asks the double evaluation to make the
 * D/E sign test of the unstable branch (and return it), flip >= 0 applies
 * that decision. */
template <class T>
__device__ void offsets_t(const QueueDev& q, const FrontPtrs& V, const FrontPtrs& C, const FrontPtrs& X,
                          int t, int de0, int az0, const T* cube, const double* delta, bool unstable_in,
                          int& flip, T* offset, T* distance) {
    const int ic = de0 * q.naz + az0;
    bool unstable = unstable_in;
    T center, g[3], h[3][3], inv[3][3];
    taylor_t(cube, delta, center, g, h);
    T determinant = fmax(h[0][0] * (h[1][1] * h[2][2] - h[1][2] * h[2][1]) +
                             h[0][1] * (h[1][2] * h[2][0] - h[1][0] * h[2][2]) +
                             h[0][2] * (h[1][0] * h[2][1] - h[2][1] * h[2][0]),
                         1e-6);
    unstable = unstable || val(determinant) < norm2_v(g);
    for (int k = 0; k < 3; ++k) {
        const T hh = fmax(h[k][k], 1e-10);
        offset[k] = -g[k] / hh;
        if (::fabs(val(offset[k]) / delta[k]) > 0.5) {
            unstable = true;
            offset[k] = T((val(offset[k]) < 0.0) ? -(0.5 * delta[k]) : 0.5 * delta[k]);
        }
    }
    if (!unstable) {
        inv[0][0] = h[1][1] * h[2][2] - h[1][2] * h[2][1];
        inv[1][0] = h[1][2] * h[2][0] - h[1][0] * h[2][2];
        inv[2][0] = h[1][0] * h[2][1] - h[1][1] * h[2][0];
        inv[0][1] = inv[1][0];
        inv[1][1] = h[0][0] * h[2][2] - h[0][2] * h[2][0];
        inv[2][1] = h[2][0] * h[0][1] - h[0][0] * h[2][1];
        inv[0][2] = inv[2][0];
        inv[1][2] = inv[2][1];
        inv[2][2] = h[0][0] * h[1][1] - h[0][1] * h[1][0];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) inv[r][c] = inv[r][c] / determinant;
        const T ng[3] = {-g[0], -g[1], -g[2]};
        matvec_t(inv, ng, offset);
        unstable = unstable || ::fabs(val(offset[1])) >= 0.5 * ::fabs(delta[1]);
    } else {
        const T save_offset = offset[1];
        g[1] = T(0.0);
        determinant = h[0][0] * h[2][2] - h[0][2] * h[2][0];
        if (val(determinant) >= norm2_v(g)) {
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) inv[r][c] = T(0.0);
            inv[0][0] = h[2][2];
            inv[0][2] = -h[0][2];
            inv[1][1] = T(1.0);
            inv[2][0] = -h[2][0];
            inv[2][2] = h[0][0];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) inv[r][c] = inv[r][c] / determinant;
            const T ng[3] = {-g[0], -g[1], -g[2]};
            matvec_t(inv, ng, offset);
            offset[1] = save_offset;
        }
    }
    for (int k = 0; k < 3; ++k) {
        distance[k] = -g[k] * offset[k] - 0.5 * h[k][k] * offset[k] * offset[k];
        distance[k] = sqrt(fmax(distance[k], 0.0));
        if (val(offset[k]) < 0.0) distance[k] = distance[k] * -1.0;
    }
    if (unstable) {
        distance[1] = center - distance[0] * distance[0] - distance[2] * distance[2];
        if (val(distance[1]) <= 0.0) {
            distance[1] = T(0.0);
            offset[1] = T(0.0);
        } else {
            distance[1] = sqrt(distance[1]);
            offset[1] = fabs(offset[1]);
            if (flip < 0) {
                double cpa[3], nxt[3], prv[3], dir[3], speed;
                const double o0 = val(offset[0]);
                collision_location(q, V, C, X, ic, o0, cpa, dir, &speed);
                collision_location(q, V, C, X, ic + q.naz, o0, nxt, dir, &speed);
                collision_location(q, V, C, X, ic - q.naz, o0, prv, dir, &speed);
                double nxt_dir[3], tgt_dir[3];
                nxt_dir[0] = nxt[0] - cpa[0];
                nxt_dir[1] = (nxt[1] - prv[1]) * cpa[0];
                nxt_dir[2] = (nxt[2] - prv[2]) * cpa[0] * ::sin(cpa[1]);
                if (::fabs(nxt_dir[0]) < 0.01) nxt_dir[0] = 0.0;
                tgt_dir[0] = q.tgt[0][t] - cpa[0];
                tgt_dir[1] = (q.tgt[1][t] - cpa[1]) * cpa[0];
                tgt_dir[2] = (q.tgt[2][t] - cpa[2]) * cpa[0] * ::sin(cpa[1]);
                flip = (dot3(nxt_dir, tgt_dir) < 0.0) ? 1 : 0;
            }
            if (flip == 1) {
                distance[1] = distance[1] * -1.0;
                offset[1] = offset[1] * -1.0;
            }
        }
    }
    if (flip < 0) flip = 0;
}

/* ------------------------------------------------------------------ */
/* beam-walk cell widths (spreading_hybrid_gaussian.cc:430-571) with    */
/* their derivatives                                                   */
/* ------------------------------------------------------------------ */
/* positions of the live fronts (prev 0, curr 1, next 2) */
struct FrontAcc {
    const FrontPtrs* F[3];
    __device__ void pos(int role, int i, double* p) const {
        p[0] = F[role]->pos[0][i];
        p[1] = F[role]->pos[1][i];
        p[2] = F[role]->pos[2][i];
    }
};
/* positions of a recomputed state S_m */
struct SegAcc {
    const double* S; /* [18][n] of the state */
    int n;
    __device__ void pos(int role, int i, double* p) const {
        p[0] = S[(size_t)(role * 6 + 0) * n + i];
        p[1] = S[(size_t)(role * 6 + 1) * n + i];
        p[2] = S[(size_t)(role * 6 + 2) * n + i];
    }
};
/* stand-in positions for enumerating the rays a width reads */
struct IndexAcc {
    __device__ void pos(int, int i, double* p) const {
        p[0] = 6.4e6;
        p[1] = 0.7 + 1e-6 * (i & 1023);
        p[2] = 0.1 + 1e-6 * (i >> 10);
    }
};
struct NoSink {
    __device__ void operator()(int, int, const double*) const {}
};

/* wvector1 distance between rays i and j of a front, and its gradient
 * with respect to both positions times g, given to the sink */
template <class Acc, class Sink>
__device__ double fdist_vjp(const Acc& A, int role, int i, int j, double g, const Sink& sink) {
    double p[3], r[3];
    A.pos(role, i, p);
    A.pos(role, j, r);
    const double D = wdist2(p[0], p[1], p[2], r[0], r[1], r[2]);
    const double f = ::sqrt(D);
    if (g != 0.0 && f > 0.0) {
        const double ht = 0.5 * (p[1] - r[1]), hp = 0.5 * (p[2] - r[2]);
        const double st = ::sin(ht), ct = ::cos(ht), sp = ::sin(hp), cp = ::cos(hp);
        const double s1 = ::sin(p[1]), s2 = ::sin(r[1]), c1 = ::cos(p[1]), c2 = ::cos(r[1]);
        const double dn = 1.0 - 2.0 * (st * st + s1 * s2 * sp * sp);
        const double raw = p[0] * p[0] + r[0] * r[0] - 2.0 * p[0] * r[0] * dn;
        const double sg = (raw < 0.0) ? -1.0 : 1.0;
        const double k = sg * g / (2.0 * f);
        const double m = -2.0 * p[0] * r[0];
        const double gp[3] = {k * (2.0 * p[0] - 2.0 * r[0] * dn),
                              k * m * (-2.0 * (st * ct + c1 * s2 * sp * sp)),
                              k * m * (-2.0 * s1 * s2 * sp * cp)};
        const double gr[3] = {k * (2.0 * r[0] - 2.0 * p[0] * dn),
                              k * m * (-2.0 * (-st * ct + s1 * c2 * sp * sp)),
                              k * m * (2.0 * s1 * s2 * sp * cp)};
        sink(role, i, gp);
        sink(role, j, gr);
    }
    return f;
}

/* width_de (spreading_hybrid_gaussian.cc:430-495): value; with gw != 0 the
 * derivative times gw goes to g_no (offsets 0 and 2) and to the sink */
template <class Acc, class Sink>
__device__ double width_de_vjp(const QueueDev& q, const Acc& A, int d, int a, const double* no, double gw,
                               double* g_no, const Sink& sink) {
    const double ai = q.az_inc[min(max(a, 0), q.naz - 1)];
    const double u = ::fabs(no[0]) / q.dt;
    const double v = ::fabs(no[2]) / ai;
    const int max_az = q.naz - 1;
    const int az_wrap = (a + 1 >= max_az) ? 0 : a + 1;
    const int na = q.naz;
    const bool two = !(v < 1e-10);
    const bool tm = !(u < 1e-10);
    const int r2 = (no[0] < 0.0) ? 0 : 2;
    /* values first (the sink needs the blend weights) */
    const double L1 = fdist_vjp(A, 1, d * na + a, (d + 1) * na + a, 0.0, sink);
    double L2 = 0.0, length1 = L1;
    if (two) {
        L2 = fdist_vjp(A, 1, d * na + az_wrap, (d + 1) * na + az_wrap, 0.0, sink);
        length1 = (1.0 - v) * L1 + v * L2;
    }
    if (!tm) {
        if (gw != 0.0) {
            fdist_vjp(A, 1, d * na + a, (d + 1) * na + a, 0.5 * gw * (two ? 1.0 - v : 1.0), sink);
            if (two) {
                fdist_vjp(A, 1, d * na + az_wrap, (d + 1) * na + az_wrap, 0.5 * gw * v, sink);
                g_no[2] += 0.5 * gw * (L2 - L1) * ((no[2] < 0.0) ? -1.0 : 1.0) / ai;
            }
        }
        return 0.5 * length1;
    }
    const double M1 = fdist_vjp(A, r2, d * na + a, (d + 1) * na + a, 0.0, sink);
    double M2 = 0.0, length2 = M1;
    if (two) {
        M2 = fdist_vjp(A, r2, d * na + az_wrap + 1, (d + 1) * na + az_wrap + 1, 0.0, sink);
        length2 = (1.0 - v) * M1 + v * M2;
    }
    const double w = 0.5 * ((1.0 - u) * length1 + u * length2);
    if (gw != 0.0) {
        const double g1 = 0.5 * gw * (1.0 - u), g2 = 0.5 * gw * u;
        fdist_vjp(A, 1, d * na + a, (d + 1) * na + a, g1 * (two ? 1.0 - v : 1.0), sink);
        fdist_vjp(A, r2, d * na + a, (d + 1) * na + a, g2 * (two ? 1.0 - v : 1.0), sink);
        if (two) {
            fdist_vjp(A, 1, d * na + az_wrap, (d + 1) * na + az_wrap, g1 * v, sink);
            fdist_vjp(A, r2, d * na + az_wrap + 1, (d + 1) * na + az_wrap + 1, g2 * v, sink);
            g_no[2] += (g1 * (L2 - L1) + g2 * (M2 - M1)) * ((no[2] < 0.0) ? -1.0 : 1.0) / ai;
        }
        g_no[0] += 0.5 * gw * (length2 - length1) * ((no[0] < 0.0) ? -1.0 : 1.0) / q.dt;
    }
    return w;
}

/* width_az (spreading_hybrid_gaussian.cc:500-571), as width_de_vjp */
template <class Acc, class Sink>
__device__ double width_az_vjp(const QueueDev& q, const Acc& A, int d, int a, const double* no, double gw,
                               double* g_no, const Sink& sink) {
    const double di = q.de_inc[min(max(d, 0), q.nde - 1)];
    const double u = ::fabs(no[0]) / q.dt;
    const double v = ::fabs(no[1]) / di;
    const int max_az = q.naz - 1;
    const int max_de = q.nde - 1;
    const int de_upper = (d + 1 >= max_de) ? max_de - 2 : d;
    const int az_wrap = (a + 1 > max_az) ? 0 : a + 1;
    const int na = q.naz;
    const bool two = !(v < 1e-10 || ::fabs(v - 1.0) < 1e-10);
    const bool tm = !(u < 1e-10);
    const int r2 = (no[0] < 0.0) ? 0 : 2;
    const int du = de_upper + 1;
    const double L1 = fdist_vjp(A, 1, d * na + a, d * na + az_wrap, 0.0, sink);
    double L2 = 0.0, length1 = L1;
    if (two) {
        L2 = fdist_vjp(A, 1, du * na + a, du * na + az_wrap, 0.0, sink);
        length1 = (1.0 - v) * L1 + v * L2;
    }
    if (!tm) {
        if (gw != 0.0) {
            fdist_vjp(A, 1, d * na + a, d * na + az_wrap, 0.5 * gw * (two ? 1.0 - v : 1.0), sink);
            if (two) {
                fdist_vjp(A, 1, du * na + a, du * na + az_wrap, 0.5 * gw * v, sink);
                g_no[1] += 0.5 * gw * (L2 - L1) * ((no[1] < 0.0) ? -1.0 : 1.0) / di;
            }
        }
        return 0.5 * length1;
    }
    const double M1 = fdist_vjp(A, r2, d * na + a, d * na + az_wrap, 0.0, sink);
    double M2 = 0.0, length2 = M1;
    if (two) {
        M2 = fdist_vjp(A, r2, du * na + a, du * na + az_wrap, 0.0, sink);
        length2 = (1.0 - v) * M1 + v * M2;
    }
    const double w = 0.5 * ((1.0 - u) * length1 + u * length2);
    if (gw != 0.0) {
        const double g1 = 0.5 * gw * (1.0 - u), g2 = 0.5 * gw * u;
        fdist_vjp(A, 1, d * na + a, d * na + az_wrap, g1 * (two ? 1.0 - v : 1.0), sink);
        fdist_vjp(A, r2, d * na + a, d * na + az_wrap, g2 * (two ? 1.0 - v : 1.0), sink);
        if (two) {
            fdist_vjp(A, 1, du * na + a, du * na + az_wrap, g1 * v, sink);
            fdist_vjp(A, r2, du * na + a, du * na + az_wrap, g2 * v, sink);
            g_no[1] += (g1 * (L2 - L1) + g2 * (M2 - M1)) * ((no[1] < 0.0) ? -1.0 : 1.0) / di;
        }
        g_no[0] += 0.5 * gw * (length2 - length1) * ((no[0] < 0.0) ? -1.0 : 1.0) / q.dt;
    }
    return w;
}

/* ------------------------------------------------------------------ */
/* the hybrid Gaussian walks of one eigenray, first frequency, in the   */
/* order of spreading_hybrid_gaussian.cc:124-425, with their reverse    */
/* ------------------------------------------------------------------ */
constexpr int JAC_WARPS = 2;

struct WalkCells {
    double w[ADJ_MAX_CELLS];
    double nm[ADJ_MAX_CELLS];
    double cd[ADJ_MAX_CELLS];  /* cell distance, then d G / d distance   */
    double cw[ADJ_MAX_CELLS];  /* cell width, then d G / d width         */
    double p2[ADJ_MAX_CELLS];  /* d G / d spread2                        */
    int16_t d[ADJ_MAX_CELLS];
    int16_t a[ADJ_MAX_CELLS];
    uint8_t kind[ADJ_MAX_CELLS]; /* 0 width_de, 1 width_az */
    uint8_t virt[ADJ_MAX_CELLS];
};

/* one run of a walk: cells [b, e) after the start cell s0, sign +1 or -1 */
struct Run {
    int s0, b, e;
    double sign;
};

/* The pieces of one eigenray's beam walks (spreading_hybrid_gaussian.cc:
 * 124-425) the adjoint needs: the first frequency's Gaussian term and the
 * cell widths.  WarpWalker runs the walks with them. */
struct Walker {
    const QueueDev* q;
    FrontAcc A;
    WalkCells* wc;
    double s2;        /* spread2 of the first frequency */

    __device__ double gauss(double d, double w, double nm) const {
        const double bw = s2 + 2.0 * 2.0 * w * w;
        return ::exp((-0.5 * d * d) / bw) / ::sqrt(bw) * nm;
    }
    __device__ double wde(int d, int a, const double* no) {
        double g[3] = {0.0, 0.0, 0.0};
        return width_de_vjp(*q, A, d, a, no, 0.0, g, NoSink());
    }
    __device__ double waz(int d, int a, const double* no) {
        double g[3] = {0.0, 0.0, 0.0};
        return width_az_vjp(*q, A, d, a, no, 0.0, g, NoSink());
    }
};

/* One eigenray's beam walks (intensity_de / intensity_az,
 * spreading_hybrid_gaussian.cc:124-425, first frequency) on a whole warp,
 * as k_eigenray's WarpBuild runs them: the widths of up to 32 cells are
 * formed on the lanes at once, then the cell distances, the running
 * intensity and its threshold test follow in cell order (shuffles), so the
 * cells kept and every sum are those of the forward construction.  Cells
 * go to wc in walk order, each lane writing its own.  All lanes call every
 * member with the same arguments. */
struct WarpWalker {
    Walker W;
    int lane;
    int n;
    bool overflow;

    __device__ double sh(double v, int k) const { return __shfl_sync(0xffffffffu, v, k); }

    /* ncell prepared cells (lane j: width w_j, norm nm_j, virtual v_j) of a
     * run with sign s.  Advances cell_dist / cell_width and I in cell
     * order, records the cells up to the stop and returns whether the walk
     * stops here (threshold, a virtual cell or a full record).  "kstop" is
     * the cell (in this chunk) the threshold stopped on, or -1. */
    __device__ bool run(int ncell, int kind, int d_j, int a_j, double w_j, double nm_j, bool v_j,
                        double sign, double& cell_dist, double& cell_width, double& I, int& kstop) {
        kstop = -1;
        double my_cd = 0.0, my_cw = 0.0;
        int nend = ncell;
        bool stop = false;
        for (int k = 0; k < ncell; ++k) {
            const bool v = __shfl_sync(0xffffffffu, v_j, k);
            const double wk = sh(w_j, k);
            if (sign > 0.0) {
                cell_dist += cell_width;
                if (v) {
                    cell_dist += cell_width;
                } else {
                    cell_width = wk;
                    cell_dist += cell_width;
                }
            } else {
                cell_dist -= cell_width;
                if (v) {
                    cell_dist -= cell_width;
                } else {
                    cell_width = wk;
                    cell_dist -= cell_width;
                }
            }
            if (lane == k) {
                my_cd = cell_dist;
                my_cw = cell_width;
            }
            if (v) {
                nend = k + 1;
                stop = true;
                break;
            }
        }
        /* room in the record: a full record stops the walk (its eigenray is
         * then flagged and carries no gradient) */
        if (n + nend > ADJ_MAX_CELLS) {
            nend = ADJ_MAX_CELLS - n;
            overflow = true;
            stop = true;
        }
        const double g = (lane < nend) ? W.gauss(my_cd, my_cw, nm_j) : 0.0;
        int kstar = nend - 1;
        for (int k = 0; k < nend; ++k) {
            const double old = I;
            I = I + sh(g, k);
            if (I / old < 1.002305238) {
                kstar = k;
                kstop = k;
                stop = true;
                break;
            }
        }
        if (lane <= kstar && lane < nend) {
            const int c = n + lane;
            W.wc->w[c] = w_j;
            W.wc->nm[c] = nm_j;
            W.wc->cd[c] = my_cd;
            W.wc->cw[c] = my_cw;
            W.wc->d[c] = (int16_t)d_j;
            W.wc->a[c] = (int16_t)a_j;
            W.wc->kind[c] = (uint8_t)kind;
            W.wc->virt[c] = v_j ? 1 : 0;
        }
        n += (nend > 0) ? kstar + 1 : 0;
        return stop;
    }

    /* the start cells of a walk (center and lower neighbour) */
    __device__ void start(int kind, int dc, int ac, double wcv, double nmc, int dl, int al, double wlv, double nml) {
        if (n + 2 > ADJ_MAX_CELLS) {
            overflow = true;
            return;
        }
        if (lane == 0) {
            W.wc->w[n] = wcv;
            W.wc->nm[n] = nmc;
            W.wc->d[n] = (int16_t)dc;
            W.wc->a[n] = (int16_t)ac;
            W.wc->kind[n] = (uint8_t)kind;
            W.wc->virt[n] = 0;
            W.wc->w[n + 1] = wlv;
            W.wc->nm[n + 1] = nml;
            W.wc->d[n + 1] = (int16_t)dl;
            W.wc->a[n + 1] = (int16_t)al;
            W.wc->kind[n + 1] = (uint8_t)kind;
            W.wc->virt[n + 1] = 0;
        }
        n += 2;
    }

    /* intensity_de (spreading_hybrid_gaussian.cc:124-258) */
    __device__ double walk_de(int de0, int a, const double* no, double L, Run* runs) {
        const QueueDev& Q = *W.q;
        const FrontPtrs& C = *W.A.F[1];
        double wcv = 0.0, wlv = 0.0;
        if (lane == 0) wcv = W.wde(de0, a, no);
        if (lane == 1) wlv = W.wde(de0 - 1, a, no);
        wcv = sh(wcv, 0);
        wlv = sh(wlv, 1);
        const int i_c = n, i_l = n + 1;
        start(0, de0, a, wcv, Q.norm_de[de0], de0 - 1, a, wlv, Q.norm_de[de0 - 1]);
        double I = W.gauss(L - wcv, wcv, Q.norm_de[de0]);
        I = I + W.gauss(L + wlv, wlv, Q.norm_de[de0 - 1]);
        runs[0] = Run{i_l, n, n, 1.0};
        runs[1] = Run{i_c, n, n, -1.0};
        if (I < 1e-10) return I;
        double cell_width = wlv, cell_dist = L + wlv;
        int kst;
        for (int d0 = de0 - 2; d0 >= 0; d0 -= 32) {
            const int d = d0 - lane;
            const int ncell = min(32, d0 + 1);
            bool virt = false;
            double w = 0.0, nm = 0.0;
            if (lane < ncell) {
                virt = C.on_edge[(d + 1) * Q.naz + a] && C.on_edge[d * Q.naz + a];
                if (!virt) w = W.wde(d, a, no);
                nm = virt ? Q.norm_de[d + 1] : Q.norm_de[d];
            }
            if (run(ncell, 0, d, a, w, nm, virt, 1.0, cell_dist, cell_width, I, kst)) break;
        }
        runs[0].e = n;
        runs[1].b = runs[1].e = n;
        cell_width = wcv;
        cell_dist = L - wcv;
        const int size = Q.nde - 1;
        if (!overflow) {
            for (int d0 = de0 + 1; d0 < size; d0 += 32) {
                const int d = d0 + lane;
                const int ncell = min(32, size - d0);
                bool virt = false;
                double w = 0.0, nm = 0.0;
                if (lane < ncell) {
                    virt = C.on_edge[(d + 1) * Q.naz + a] && C.on_edge[d * Q.naz + a];
                    if (!virt) w = W.wde(d, a, no);
                    nm = virt ? Q.norm_de[d - 1] : Q.norm_de[d];
                }
                if (run(ncell, 0, d, a, w, nm, virt, -1.0, cell_dist, cell_width, I, kst)) break;
            }
        }
        runs[1].e = n;
        return I;
    }

    /* intensity_az (spreading_hybrid_gaussian.cc:264-425) */
    __device__ double walk_az(int d, int az0, const double* no, double L, Run* runs) {
        const QueueDev& Q = *W.q;
        const FrontPtrs& C = *W.A.F[1];
        const int max_de = Q.nde - 2;
        const int max_az = Q.naz - 1;
        const int az_lower = Q.az_boundary ? az0 : 0;
        const int az_upper = Q.az_boundary ? az0 : max_az - 1;
        auto norm = [&](int aa) { return (d >= max_de) ? Q.norm_az[1 * Q.naz + aa] : Q.norm_az[d * Q.naz + aa]; };
        const int a1 = (az0 < 1) ? max_az - 1 : az0 - 1;
        double wcv = 0.0, wlv = 0.0;
        if (lane == 0) wcv = W.waz(d, az0, no);
        if (lane == 1) wlv = W.waz(d, a1, no);
        wcv = sh(wcv, 0);
        wlv = sh(wlv, 1);
        const int i_c = n, i_l = n + 1;
        start(1, d, az0, wcv, norm(az0), d, a1, wlv, norm(a1));
        double I = W.gauss(L - wcv, wcv, norm(az0));
        I = I + W.gauss(L + wlv, wlv, norm(a1));
        runs[0] = Run{i_l, n, n, 1.0};
        runs[1] = Run{i_c, n, n, -1.0};
        if (I < 1e-10) return I;
        const int start_a = (a1 < 1) ? max_az - 1 : a1 - 1;
        double cell_width = wlv, cell_dist = L + wlv;
        int marked = -1;
        bool done = false;
        for (int k0 = 0; !done && k0 < max_az; k0 += 32) {
            const int kk = k0 + lane;
            int a = start_a - kk;
            a = ((a % max_az) + max_az) % max_az;
            int kind = 0; /* 0 process, 1 loop end (not marked), 2 marked stop */
            if (kk >= max_az || a == az_lower) {
                kind = 1;
            } else if (a == az0 || a == a1) {
                kind = 1;
            } else if (C.on_edge[d * Q.naz + a]) {
                kind = 2;
            }
            const unsigned stopmask = __ballot_sync(0xffffffffu, kind != 0);
            int first = 32, fk = 0;
            if (stopmask) {
                first = __ffs(stopmask) - 1;
                fk = __shfl_sync(0xffffffffu, kind, first);
            }
            const int ncell = first;
            double w = 0.0, nm = 0.0;
            if (lane < ncell) {
                w = W.waz(d, a, no);
                nm = norm(a);
            }
            int kst = -1;
            const bool brk = (ncell > 0) && run(ncell, 1, d, a, w, nm, false, 1.0, cell_dist, cell_width, I, kst);
            if (brk) {
                marked = (kst >= 0) ? k0 + kst : k0 + ncell - 1;
                done = true;
            } else {
                if (ncell > 0) marked = k0 + ncell - 1;
                if (stopmask) {
                    done = true;
                    if (fk == 2) marked = k0 + first;
                }
            }
        }
        runs[0].e = n;
        runs[1].b = runs[1].e = n;
        cell_width = wcv;
        cell_dist = L - wcv;
        done = overflow;
        for (int k0 = 0; !done && k0 < max_az; k0 += 32) {
            const int kk = k0 + lane;
            const int a = (az0 + 1 + kk) % max_az;
            int kind = 0;
            const int off = ((start_a - a) % max_az + max_az) % max_az;
            const bool dup = (a == az0) || (a == a1) || (marked >= 0 && off <= marked);
            if (kk >= max_az || a == az_upper || dup || C.on_edge[d * Q.naz + a]) kind = 1;
            const unsigned stopmask = __ballot_sync(0xffffffffu, kind != 0);
            int ncell = 32;
            if (stopmask) {
                ncell = __ffs(stopmask) - 1;
                done = true;
            }
            double w = 0.0, nm = 0.0;
            if (lane < ncell) {
                w = W.waz(d, a, no);
                nm = norm(a);
            }
            int kst = -1;
            if (ncell > 0 && run(ncell, 1, d, a, w, nm, false, -1.0, cell_dist, cell_width, I, kst)) done = true;
        }
        runs[1].e = n;
        return I;
    }

    /* reverse of one run: dI/d (cell widths) into gwid, dI/dL returned,
     * dI/d spread2 added to gs2, for gI = dTL/dI.  The Gaussian's partials
     * of every cell are formed on the lanes, then the adjoint recurrence
     * runs in cell order on lane 0 (gwid, gs2 and the returned value are
     * lane 0's) */
    __device__ double reverse_run(const Run& r, double L, double gI, double* gwid, double& gs2) {
        WalkCells* wc = W.wc;
        const double s = r.sign;
        for (int k = r.b + lane; k < r.e; k += 32) {
            const double cd = wc->cd[k], cw = wc->cw[k];
            const double bw = W.s2 + 2.0 * 2.0 * cw * cw;
            const double G = ::exp((-0.5 * cd * cd) / bw) / ::sqrt(bw) * wc->nm[k];
            const double gbw = G * (0.5 * cd * cd / (bw * bw) - 0.5 / bw);
            wc->cd[k] = -G * cd / bw;
            wc->cw[k] = gbw * 8.0 * cw;
            wc->p2[k] = gbw;
        }
        __syncwarp();
        double Acd = 0.0;
        if (lane == 0) {
            double Acw_next = 0.0;
            for (int k = r.e - 1; k >= r.b; --k) {
                Acd = gI * wc->cd[k] + Acd;
                const double Acw = gI * wc->cw[k] + Acw_next;
                gs2 += gI * wc->p2[k];
                if (wc->virt[k]) {
                    Acw_next = Acw + 2.0 * s * Acd;
                } else {
                    gwid[k] += Acw + s * Acd;
                    Acw_next = s * Acd;
                }
            }
            const double cw0 = wc->w[r.s0], cd0 = L + s * cw0;
            const double bw = W.s2 + 2.0 * 2.0 * cw0 * cw0;
            const double G = ::exp((-0.5 * cd0 * cd0) / bw) / ::sqrt(bw) * wc->nm[r.s0];
            const double gbw = G * (0.5 * cd0 * cd0 / (bw * bw) - 0.5 / bw);
            Acd = gI * (-G * cd0 / bw) + Acd;
            const double Acw = gI * gbw * 8.0 * cw0 + Acw_next;
            gs2 += gI * gbw;
            gwid[r.s0] += Acw + s * Acd;
        }
        __syncwarp();
        return Acd;
    }
};

}  // namespace

/* ------------------------------------------------------------------ */
/* forward recording kernels                                           */
/* ------------------------------------------------------------------ */

/* S_s of every ray when s is a multiple of the checkpoint interval;
 * launched before k_advance of step s (k_reflect of that step only writes
 * shadow slots, so the fronts hold S_s, except the prev and curr states of
 * rays that reflected at step s-1 while step s-1's commit is pending: those
 * come from that step's slots) */
__global__ void __launch_bounds__(128) k_adj_checkpoint(__grid_constant__ const QueueDev q, int k) {
    const int64_t s = *q.d_base + k;
    if (s % q.adj_K != 0) return;
    const int64_t slot = s / q.adj_K;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= q.adj_nckpt) {
        if (i == 0) set_err(q, ERR_ADJ_OVERFLOW);
        return;
    }
    if (i >= q.n) return;
    Roles R;
    roles_at(q, s, R);
    double* base = q.adj_ckpt + (size_t)slot * ADJ_S * q.n;
    const double* sp = prev_step_slot(q, s, i);
    const FrontPtrs* F[3] = {R.V, R.C, R.X};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            /* slot layout: pos at +0, nd at +6 of each 17-double state */
            const bool from_slot = sp && r < 2;
            base[(size_t)(r * 6 + c) * q.n + i] = from_slot ? sp[17 * (r + 1) + c] : F[r]->pos[c][i];
            base[(size_t)(r * 6 + 3 + c) * q.n + i] = from_slot ? sp[17 * (r + 1) + 6 + c] : F[r]->nd[c][i];
        }
}

/* the eigenray records of this chunk already given partials */
__global__ void k_adj_mark(__grid_constant__ const QueueDev q) {
    *q.adj_mark = min(*q.n_rec, q.cap_rec);
}

/* Partial derivatives of each eigenray record written in this step, on
 * the fronts it was built from (one warp per record). */
__global__ void __launch_bounds__(32 * JAC_WARPS) k_eigenray_jac(__grid_constant__ const QueueDev q, int k) {
    __shared__ double s_cube[JAC_WARPS][27];
    __shared__ double s_gth[JAC_WARPS][6];
    __shared__ WalkCells s_cells[JAC_WARPS];
    __shared__ double s_gw[JAC_WARPS][ADJ_MAX_CELLS];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t s = *q.d_base + k + 1;
    const double time = q.d_times[k + 1];
    const uint32_t lo = *q.adj_mark;
    const uint32_t hi = min(*q.n_rec, q.cap_rec);
    const FrontPtrs& V = q.F[ring_slot(s + 1)];
    const FrontPtrs& C = q.F[ring_slot(s + 2)];
    const FrontPtrs& X = q.F[ring_slot(s + 3)];
    for (uint32_t r = lo + blockIdx.x * JAC_WARPS + warp; r < hi; r += gridDim.x * JAC_WARPS) {
        __syncwarp();
        const wq3d_eigenray rec = q.rec[r];
        const int t = rec.t1 * q.nt2 + rec.t2;
        const int de0 = rec.de, az0 = rec.az;
        const int i = de0 * q.naz + az0;
        const TgtS tg{q.tgt[1][t], q.tgt[2][t], q.tgt_sin[t], q.tgt_R2[t], q.tgt_2R[t]};
        if (lane < 27) {
            const int m = lane / 9, nd_ = (lane / 3) % 3, na = lane % 3;
            const int j = (de0 + nd_ - 1) * q.naz + wrap_az(q, az0, na);
            const FrontPtrs& F = (m == 0) ? V : (m == 1) ? C : X;
            s_cube[warp][lane] = d2_at(F, j, tg);
        }
        __syncwarp();
        double cube[27];
        for (int j = 0; j < 27; ++j) cube[j] = s_cube[warp][j];
        bool bad = false;
        if (lane < 9) {
            const int surface = C.surface[i], bottom = C.bottom[i], caustic = C.caustic[i];
            const int j = (de0 + lane / 3 - 1) * q.naz + wrap_az(q, az0, lane % 3);
            bad = V.surface[j] != surface || C.surface[j] != surface || X.surface[j] != surface ||
                  V.bottom[j] != bottom || C.bottom[j] != bottom || X.bottom[j] != bottom ||
                  V.caustic[j] != caustic || C.caustic[j] != caustic || X.caustic[j] != caustic ||
                  V.on_edge[j];
        }
        const bool unstable_in = __any_sync(0xffffffffu, bad);
        const double delta[3] = {q.dt, q.de_inc[de0], q.az_inc[az0]};
        double off[3], dist[3];
        int flip = -1;
        offsets_t<double>(q, V, C, X, t, de0, az0, cube, delta, unstable_in, flip, off, dist);
        /* lane j: d (offset, distance) / d cube[j] */
        double dth[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (lane < 27) {
            Dual<1> cd[27];
            for (int j = 0; j < 27; ++j) cd[j] = Dual<1>::var(cube[j], j == lane ? 0 : -1);
            Dual<1> o[3], dd[3];
            int fl = flip;
            offsets_t<Dual<1>>(q, V, C, X, t, de0, az0, cd, delta, unstable_in, fl, o, dd);
            for (int m = 0; m < 3; ++m) {
                dth[m] = o[m].d[0];
                dth[3 + m] = dd[m].d[0];
            }
        }
        /* the walks forward and in reverse, on the whole warp */
        AdjRec* out = nullptr;
        uint32_t slot = 0;
        if (lane == 0) {
            slot = atomicAdd(q.adj_n, 1u);
            if (slot >= q.adj_cap) set_err(q, ERR_ADJ_OVERFLOW);
        }
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (slot >= q.adj_cap) continue;
        out = q.adj_rec + slot;
        WarpWalker WW;
        WW.W.q = &q;
        WW.W.A.F[0] = &V;
        WW.W.A.F[1] = &C;
        WW.W.A.F[2] = &X;
        WW.W.wc = &s_cells[warp];
        WW.W.s2 = q.tgt_spread2[(size_t)t * q.nf];
        WW.lane = lane;
        WW.n = 0;
        WW.overflow = false;
        /* spreading_hybrid_gaussian.cc:65-119 */
        int a = az0;
        double no_de[3] = {off[0], off[1], off[2]};
        if (off[2] < 0.0) {
            if (az0 > 0) {
                a = az0 - 1;
            } else if (q.az_boundary) {
                a = q.naz - 2;
            }
            no_de[2] = off[2] + q.az_inc[min(max(a, 0), q.naz - 1)];
        }
        double no_az[3] = {off[0], off[1], off[2]};
        int d = de0;
        if (off[1] < 0.0 && !C.on_edge[i - q.naz]) {
            d = de0 - 1;
            no_az[1] = off[1] + q.de_inc[min(max(d, 0), q.nde - 1)];
        }
        Run rde[2], raz[2];
        const double Ide = WW.walk_de(de0, a, no_de, dist[1], rde);
        const int n_de = WW.n;
        const double Iaz = WW.overflow ? 0.0 : WW.walk_az(d, az0, no_az, dist[2], raz);
        __syncwarp();
        const bool ovf = WW.overflow;
        const int ncells = min(WW.n, ADJ_MAX_CELLS);
        double* gw = s_gw[warp];
        for (int c = lane; c < ncells; c += 32) gw[c] = 0.0;
        __syncwarp();
        double gs2 = 0.0, gL_de = 0.0, gL_az = 0.0;
        double g_no_de[3] = {0.0, 0.0, 0.0}, g_no_az[3] = {0.0, 0.0, 0.0};
        if (!ovf) {
            const double si = Ide * Iaz;
            double gI_de = 0.0, gI_az = 0.0;
            if (si > 1e-30) {
                const double gsi = -10.0 / (si * 2.302585092994045684);
                gI_de = gsi * Iaz;
                gI_az = gsi * Ide;
            }
            gL_de = WW.reverse_run(rde[0], dist[1], gI_de, gw, gs2);
            gL_de = gL_de + WW.reverse_run(rde[1], dist[1], gI_de, gw, gs2);
            gL_az = WW.reverse_run(raz[0], dist[2], gI_az, gw, gs2);
            gL_az = gL_az + WW.reverse_run(raz[1], dist[2], gI_az, gw, gs2);
            /* width derivatives with respect to the offsets they blend
             * with, one cell per lane */
            for (int c = lane; c < ncells; c += 32) {
                if (WW.W.wc->virt[c] || gw[c] == 0.0) continue;
                if (c < n_de)
                    width_de_vjp(q, WW.W.A, WW.W.wc->d[c], WW.W.wc->a[c], no_de, gw[c], g_no_de, NoSink());
                else
                    width_az_vjp(q, WW.W.A, WW.W.wc->d[c], WW.W.wc->a[c], no_az, gw[c], g_no_az, NoSink());
            }
            for (int m = 0; m < 3; ++m)
                for (int o = 16; o > 0; o >>= 1) {
                    g_no_de[m] += __shfl_xor_sync(0xffffffffu, g_no_de[m], o);
                    g_no_az[m] += __shfl_xor_sync(0xffffffffu, g_no_az[m], o);
                }
        }
        /* the cells the walks used, in walk order */
        int nc = 0;
        {
            const unsigned lt = (1u << lane) - 1u;
            for (int c0 = 0; c0 < ncells; c0 += 32) {
                const int c = c0 + lane;
                const bool keep = !ovf && c < ncells && !WW.W.wc->virt[c] && gw[c] != 0.0;
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int o = nc + __popc(m & lt);
                    out->cell_d[o] = WW.W.wc->d[c];
                    out->cell_a[o] = WW.W.wc->a[c];
                    out->cell_kind[o] = WW.W.wc->kind[c];
                    out->cell_g[o] = gw[c];
                }
                nc += __popc(m);
            }
        }
        if (lane == 0) {
            /* attenuation interpolated in time (build_eigenray) */
            double ddt = off[0] / q.dt;
            const int ra0 = (ddt >= 0.0) ? 1 : 0, ra1 = (ddt >= 0.0) ? 2 : 1;
            if (ddt < 0.0) ddt = 1.0 + ddt;
            const FrontPtrs& A0 = (ra0 == 1) ? C : V;
            const FrontPtrs& A1 = (ra1 == 2) ? X : C;
            const double a0 = A0.atten[i], a1 = A1.atten[i];
            s_gth[warp][0] = (a1 - a0) / q.dt + g_no_de[0] + g_no_az[0];
            s_gth[warp][1] = g_no_az[1];
            s_gth[warp][2] = g_no_de[2];
            s_gth[warp][3] = 0.0;
            s_gth[warp][4] = gL_de;
            s_gth[warp][5] = gL_az;
            out->step = s;
            out->t = t;
            out->i = i;
            out->ncell = nc;
            out->flags = ovf ? ADJ_CELL_OVERFLOW : ADJ_VALID;
            out->a_de = a;
            out->d_az = d;
            out->role_a0 = ra0;
            out->role_a1 = ra1;
            for (int m = 0; m < 3; ++m) {
                out->no_de[m] = no_de[m];
                out->no_az[m] = no_az[m];
            }
            out->dTL_da0 = 1.0 - ddt;
            out->dTL_da1 = ddt;
            out->dTL_ds2 = gs2;
            (void)time;
        }
        __syncwarp();
        if (lane < 27) {
            double g = 0.0;
            for (int m = 0; m < 6; ++m) g += s_gth[warp][m] * dth[m];
            out->dTL[lane] = g;
            out->dT[lane] = dth[0];
        }
    }
}

/* ------------------------------------------------------------------ */
/* backward kernels                                                    */
/* ------------------------------------------------------------------ */
namespace {

/* the state index an eigenray's role-r cube entry belongs to */
__device__ __forceinline__ int64_t cube_state(int64_t m, int role) { return m - 2 + role; }

struct TouchSink {
    int64_t* last;
    int64_t m;
    __device__ void operator()(int, int i, const double*) const {
        atomicMax((unsigned long long*)(last + i), (unsigned long long)m);
    }
};

struct SeedSink {
    double* seed; /* [21][n] of the state */
    int n;
    __device__ void operator()(int role, int i, const double* g) const {
        for (int c = 0; c < 3; ++c) atomicAdd(seed + (size_t)(role * 6 + c) * n + i, g[c]);
    }
};

}  // namespace

/* the last state index at which each ray is seeded (last[] starts at -1,
 * stored as a biased unsigned maximum: value + 1) */
__global__ void k_adj_touch(AdjSweep a, __grid_constant__ const QueueDev q) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nrec) return;
    const AdjRec& R = q.adj_rec[r];
    if (!(R.flags & ADJ_VALID)) return;
    const int de0 = R.i / q.naz, az0 = R.i % q.naz;
    for (int lane = 0; lane < 27; ++lane) {
        const int m = lane / 9, nd_ = (lane / 3) % 3, na = lane % 3;
        const int j = (de0 + nd_ - 1) * q.naz + wrap_az(q, az0, na);
        const int64_t ms = cube_state(R.step, m);
        if (ms >= 0) atomicMax((unsigned long long*)(a.last + j), (unsigned long long)(ms + 1));
    }
    TouchSink ts{a.last, R.step + 1};
    ts(0, R.i, nullptr);
    IndexAcc A;
    double g[3];
    for (int c = 0; c < R.ncell; ++c) {
        if (R.cell_kind[c] == 0)
            width_de_vjp(q, A, R.cell_d[c], R.cell_a[c], R.no_de, 1.0, g, ts);
        else
            width_az_vjp(q, A, R.cell_d[c], R.cell_a[c], R.no_az, 1.0, g, ts);
    }
}

/* S_m0 .. S_m1-1 of each ray seeded at or after m0, and each step's
 * reflection chain, with the engine's own step functions */
__global__ void __launch_bounds__(128) k_adj_recompute(AdjSweep a, __grid_constant__ const QueueDev q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= q.n) return;
    if ((int64_t)a.last[i] - 1 < a.m0) return;
    const int n = q.n;
    const double* ck = q.adj_ckpt + (size_t)a.ckpt * ADJ_S * n;
    RayLocal L;
    RayS* Y[3] = {&L.v, &L.c, &L.x};
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            Y[r]->pos[c] = ck[(size_t)(r * 6 + c) * n + i];
            Y[r]->nd[c] = ck[(size_t)(r * 6 + 3 + c) * n + i];
        }
        Y[r]->dist = 0.0;
        update1(q, *Y[r]);
    }
    for (int f = 0; f < q.nf; ++f) {
        L.att[f] = 0.0;
        L.ph[f] = 0.0;
    }
    L.surface = L.bottom = L.caustic = 0;
    double dl[3] = {0.0, 0.0, 0.0};
    for (int64_t m = a.m0; m < a.m1; ++m) {
        const int64_t j = m - a.m0;
        double* S = a.seg + (size_t)j * ADJ_S * n;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                S[(size_t)(r * 6 + c) * n + i] = Y[r]->pos[c];
                S[(size_t)(r * 6 + 3 + c) * n + i] = Y[r]->nd[c];
            }
        /* k_reflect's chain (wave_queue.cc:197-256) */
        uint32_t code = 0;
        if (reflect_decision(q, L.x.pos, L.c.nd)) {
            int seq = 0;
            int next_try = -1;
            if (L.x.pos[0] - q.R > 0.0 && surface_local(q, q.F[0], L, i, m + 1, 0.0, seq)) {
                code = chain_add(code, false);
                next_try = 0;
            } else {
                const double depth = boundary_height(q.oc.bot, L.x.pos[1], L.x.pos[2]) - L.x.pos[0];
                if (depth > 0.0) {
                    bottom_local(q, q.F[0], L, i, depth, m + 1, 0.0, seq, dl);
                    code = chain_add(code, true);
                    next_try = 1;
                }
            }
            if (next_try >= 0) {
                for (int it = 0; it < MAX_BOUNCE; ++it) {
                    if (((code >> 16) & 0xf) >= 8) {
                        code |= 0x80000000u;
                        break;
                    }
                    if (next_try == 0) {
                        const double depth = boundary_height(q.oc.bot, L.x.pos[1], L.x.pos[2]) - L.x.pos[0];
                        if (!(depth > 0.0)) break;
                        bottom_local(q, q.F[0], L, i, depth, m + 1, 0.0, seq, dl);
                        code = chain_add(code, true);
                        next_try = 1;
                    } else {
                        if (!(L.x.pos[0] - q.R > 0.0 && surface_local(q, q.F[0], L, i, m + 1, 0.0, seq))) break;
                        code = chain_add(code, false);
                        next_try = 0;
                    }
                }
            }
        }
        if (code & 0x80000000u) atomicOr(a.err, ADJ_ERR_CHAIN);
        a.chain[(size_t)j * n + i] = code;
        if (m + 1 < a.m1) {
            RayS y3;
            ab3(q.dt, L.v, L.c, L.x, y3);
            update1(q, y3);
            L.v = L.c;
            L.c = L.x;
            L.x = y3;
        }
    }
}

/* each eigenray's partials times its weights, taken to its rays' states in
 * [m0, m1) */
__global__ void k_adj_expand(AdjSweep a, __grid_constant__ const QueueDev q) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nrec) return;
    const AdjRec& R = q.adj_rec[r];
    if (!(R.flags & ADJ_VALID)) return;
    const int64_t m = R.step;
    if (m < a.m0 || m - 2 >= a.m1) return;
    const double wtl = a.w_tl[r], wt = a.w_t[r];
    if (wtl == 0.0 && wt == 0.0) return;
    const int n = q.n;
    const int de0 = R.i / q.naz, az0 = R.i % q.naz;
    const int t = R.t;
    const double tth = q.tgt[1][t], tph = q.tgt[2][t], tsin = q.tgt_sin[t], twoR = q.tgt_2R[t];
    /* cube values: target distance2 at the next-front position of S_{m-2+role} */
    for (int lane = 0; lane < 27; ++lane) {
        const int role = lane / 9, nd_ = (lane / 3) % 3, na = lane % 3;
        const int64_t ms = cube_state(m, role);
        if (ms < a.m0 || ms >= a.m1 || ms < 0) continue;
        const double g = wtl * R.dTL[lane] + wt * R.dT[lane];
        if (g == 0.0) continue;
        const int j = (de0 + nd_ - 1) * q.naz + wrap_az(q, az0, na);
        const double* S = a.seg + (size_t)(ms - a.m0) * ADJ_S * n;
        const double rho = S[(size_t)12 * n + j], th = S[(size_t)13 * n + j], ph = S[(size_t)14 * n + j];
        const double st = ::sin(th), ct = ::cos(th);
        const double ha = 0.5 * (th - tth), hb = 0.5 * (ph - tph);
        const double inner = 1.0 - 2.0 * (ha * ha + tsin * (st * (hb * hb)));
        const double raw = rho * rho + q.tgt_R2[t] - twoR * (rho * inner);
        const double sg = (raw < 0.0) ? -g : g;
        const double d_in_th = -2.0 * (ha + tsin * ct * hb * hb);
        const double d_in_ph = -2.0 * (tsin * st * hb);
        double* sd = a.seed + (size_t)(ms - a.m0) * ADJ_L * n;
        atomicAdd(sd + (size_t)12 * n + j, sg * (2.0 * rho - twoR * inner));
        atomicAdd(sd + (size_t)13 * n + j, sg * (-twoR * rho * d_in_th));
        atomicAdd(sd + (size_t)14 * n + j, sg * (-twoR * rho * d_in_ph));
    }
    if (m >= a.m1 || wtl == 0.0) return;
    /* widths and attenuation at S_m */
    SegAcc A{a.seg + (size_t)(m - a.m0) * ADJ_S * n, n};
    double* sd = a.seed + (size_t)(m - a.m0) * ADJ_L * n;
    SeedSink sink{sd, n};
    double gno[3];
    for (int c = 0; c < R.ncell; ++c) {
        const double gw = wtl * R.cell_g[c];
        if (R.cell_kind[c] == 0)
            width_de_vjp(q, A, R.cell_d[c], R.cell_a[c], R.no_de, gw, gno, sink);
        else
            width_az_vjp(q, A, R.cell_d[c], R.cell_a[c], R.no_az, gw, gno, sink);
    }
    atomicAdd(sd + (size_t)(18 + R.role_a0) * n + R.i, wtl * R.dTL_da0);
    atomicAdd(sd + (size_t)(18 + R.role_a1) * n + R.i, wtl * R.dTL_da1);
}

namespace {

/* lambda contribution of one pass of NB dual directions over the inputs
 * [off, off + NB) of Phi_m (18 state values, then the window's nodes) */
template <int NB>
__device__ __noinline__ uint32_t step_vjp_pass(const QueueDev& q, const AdjSweep& a, const double* S,
                                               uint32_t code, ParamWin pw, int off, const double* lam1,
                                               double* lam0, double* gnode) {
    using D = Dual<NB>;
    bool ok = true;
    LocalT<D> L;
    RayT<D>* Y[3] = {&L.v, &L.c, &L.x};
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            Y[r]->pos[c] = D::var(S[r * 6 + c], r * 6 + c - off);
            Y[r]->nd[c] = D::var(S[r * 6 + 3 + c], r * 6 + 3 + c - off);
        }
        Y[r]->dist = D(0.0);
    }
    pw.base = ADJ_S - off;
    for (int r = 0; r < 3; ++r) update_t(q, *Y[r], pw, ok);
    L.att = D(0.0);
    uint32_t err = 0;
    if (code) {
        const uint32_t c2 = chain_t(q, L, pw, ok);
        if (c2 != code) err |= ADJ_ERR_TOPOLOGY;
    }
    RayT<D> y3;
    ab3_t(q.dt, L.v, L.c, L.x, y3);
    D inc;
    if (q.oc.prof.atten == WQ3D_ATTEN_CONSTANT)
        inc = q.oc.prof.atten_coef * y3.dist * q.freq[0];
    else
        inc = y3.dist * a.alpha0 * (1.0 + 5.88264e-6 * (y3.pos[0] - q.R));
    if (!ok) err |= ADJ_ERR_WINDOW;
    const D* outs[18] = {&L.c.pos[0], &L.c.pos[1], &L.c.pos[2], &L.c.nd[0], &L.c.nd[1], &L.c.nd[2],
                         &L.x.pos[0], &L.x.pos[1], &L.x.pos[2], &L.x.nd[0], &L.x.nd[1], &L.x.nd[2],
                         &y3.pos[0],  &y3.pos[1],  &y3.pos[2],  &y3.nd[0],  &y3.nd[1],  &y3.nd[2]};
    const double l_att = lam1[19] + lam1[20];
    const double l_inc = lam1[20];
    for (int j = 0; j < NB; ++j) {
        const int J = off + j;
        if (J >= ADJ_S + pw.w) break;
        double g = 0.0;
        for (int o = 0; o < 18; ++o) g += lam1[o] * outs[o]->d[j];
        g += l_att * L.att.d[j] + l_inc * inc.d[j];
        if (J < ADJ_S)
            lam0[J] += g;
        else
            gnode[J - ADJ_S] += g;
    }
    return err;
}

/* lambda contribution of Phi_m for a step without reflections, front by
 * front.  Without a reflection chain, Phi_m passes the curr and next
 * states through and forms the new front from the three fronts'
 * derivatives (AB3): each front's (pg, ng) depends only on its own six
 * state values and the two profile nodes around its depth, so one dual
 * pass of eight directions per front gives its block of the Jacobian, and
 * AB3, the step length and the absorption increment are transposed by
 * hand.  Equal to step_vjp_pass's three passes over all 24 inputs. */
__device__ __noinline__ uint32_t step_vjp_blocked(const QueueDev& q, const AdjSweep& a, const double* S,
                                                  const ParamWin& pw, const double* lam1, double* lam0,
                                                  double* gnode) {
    using D = Dual<8>;
    const double h = q.dt;
    const double A2 = 23.0 / 12.0, A1 = 16.0 / 12.0, A0 = 5.0 / 12.0;
    const double coef[3] = {h * A0, -h * A1, h * A2}; /* V, C, X */
    uint32_t err = 0;
    /* the three fronts' derivatives (values) and Jacobian blocks */
    double pg[3][3];
    double J[3][6][8]; /* [front][pg0..2, ng0..2][pos0..2, nd0..2, node k, node k+1] */
    int knode[3];
    for (int r = 0; r < 3; ++r) {
        bool ok = true;
        RayT<D> Y;
        for (int c = 0; c < 3; ++c) {
            Y.pos[c] = D::var(S[r * 6 + c], c);
            Y.nd[c] = D::var(S[r * 6 + 3 + c], 3 + c);
        }
        Y.dist = D(0.0);
        ParamWin pr;
        pr.k0 = ssp_interval(q, S[r * 6]);
        pr.w = 2;
        pr.base = 6;
        knode[r] = pr.k0;
        update_t(q, Y, pr, ok);
        if (!ok) err |= ADJ_ERR_WINDOW;
        for (int k = 0; k < 3; ++k) {
            pg[r][k] = Y.pg[k].v;
            for (int j = 0; j < 8; ++j) {
                J[r][k][j] = Y.pg[k].d[j];
                J[r][3 + k][j] = Y.ng[k].d[j];
            }
        }
    }
    /* AB3 step values (ab3_t): d_k and the step length */
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = h * (A2 * pg[2][k] - A1 * pg[1][k] + A0 * pg[0][k]);
    const double rx = S[12], tx = S[13];
    const double sx = ::sin(tx), cx = ::cos(tx);
    const double b = rx * d[1];
    const double cc = rx * (sx * d[2]);
    const double dist = ::sqrt(d[0] * d[0] + b * b + cc * cc);
    /* the absorption increment of the first frequency */
    const double l_inc = lam1[20];
    double l_dist = 0.0, l_y3r = 0.0;
    if (q.oc.prof.atten == WQ3D_ATTEN_CONSTANT) {
        l_dist = l_inc * (q.oc.prof.atten_coef * q.freq[0]);
    } else {
        const double y3r = S[12] + d[0];
        l_dist = l_inc * (a.alpha0 * (1.0 + 5.88264e-6 * (y3r - q.R)));
        l_y3r = l_inc * (dist * a.alpha0 * 5.88264e-6);
    }
    /* curr and next pass through; the new front's position and direction
     * add to the next front's */
    for (int c = 0; c < 6; ++c) {
        lam0[6 + c] += lam1[c];
        lam0[12 + c] += lam1[6 + c];
    }
    double L3p[3] = {lam1[12] + l_y3r, lam1[13], lam1[14]};
    for (int k = 0; k < 3; ++k) {
        lam0[12 + k] += L3p[k];
        lam0[15 + k] += lam1[15 + k];
    }
    /* through the step length: d dist / d (d, rho_X, theta_X) */
    double ld[3] = {L3p[0], L3p[1], L3p[2]};
    if (dist > 0.0 && l_dist != 0.0) {
        const double gdist = l_dist / dist;
        ld[0] += gdist * d[0];
        ld[1] += gdist * (b * rx);
        ld[2] += gdist * (cc * rx * sx);
        lam0[12] += gdist * (b * d[1] + cc * sx * d[2]);
        lam0[13] += gdist * (cc * rx * cx * d[2]);
    }
    /* through AB3 into each front's derivatives, then its block */
    for (int r = 0; r < 3; ++r) {
        double lo[6];
        for (int k = 0; k < 3; ++k) {
            lo[k] = coef[r] * ld[k];
            lo[3 + k] = coef[r] * lam1[15 + k];
        }
        for (int j = 0; j < 6; ++j) {
            double g = 0.0;
            for (int o = 0; o < 6; ++o) g += lo[o] * J[r][o][j];
            lam0[r * 6 + j] += g;
        }
        for (int t = 0; t < 2; ++t) {
            double g = 0.0;
            for (int o = 0; o < 6; ++o) g += lo[o] * J[r][o][6 + t];
            const int w = knode[r] + t - pw.k0;
            if (w < 0 || w >= pw.w) {
                if (g != 0.0) err |= ADJ_ERR_WINDOW;
            } else {
                gnode[w] += g;
            }
        }
    }
    return err;
}

/* init_wave and the RK3 start-up of one ray (k_startup) on dual node
 * values: lambda_0 . d S_0 / d nodes into gnode */
__device__ __noinline__ uint32_t startup_vjp(const QueueDev& q, const AdjSweep& a, int i, ParamWin pw,
                                             const double* lam, double* gnode) {
    using D = Dual<ADJ_W>;
    bool ok = true;
    const int d = i / q.naz, az = i % q.naz;
    pw.base = 0;
    D cs, gs[3];
    ssp_t(q, D(q.source[0]), pw, ok, cs, gs);
    RayT<D> c0;
    c0.nd[0] = q.sin_de[d] / cs;
    c0.nd[1] = (-q.cos_de[d] * q.cos_az[az]) / cs;
    c0.nd[2] = (q.cos_de[d] * q.sin_az[az]) / cs;
    c0.pos[0] = D(q.source[0]);
    c0.pos[1] = D(q.source[1]);
    c0.pos[2] = D(q.source[2]);
    c0.dist = D(0.0);
    update_t(q, c0, pw, ok);
    const double h = -q.dt;
    RayT<D> n1, p1, v1;
    rk1_t(h, c0, n1);
    update_t(q, n1, pw, ok);
    rk2_t(h, c0, n1, p1);
    update_t(q, p1, pw, ok);
    rk3_t(h, c0, n1, p1, v1);
    update_t(q, v1, pw, ok);
    rk1_t(h, v1, n1);
    update_t(q, n1, pw, ok);
    rk2_t(h, v1, n1, p1);
    update_t(q, p1, pw, ok);
    rk3_t(h, v1, n1, p1, p1);
    update_t(q, p1, pw, ok);
    RayT<D> x;
    ab3_t(q.dt, p1, v1, c0, x);
    D inc;
    if (q.oc.prof.atten == WQ3D_ATTEN_CONSTANT)
        inc = q.oc.prof.atten_coef * x.dist * q.freq[0];
    else
        inc = x.dist * a.alpha0 * (1.0 + 5.88264e-6 * (x.pos[0] - q.R));
    const D* outs[18] = {&v1.pos[0], &v1.pos[1], &v1.pos[2], &v1.nd[0], &v1.nd[1], &v1.nd[2],
                         &c0.pos[0], &c0.pos[1], &c0.pos[2], &c0.nd[0], &c0.nd[1], &c0.nd[2],
                         &x.pos[0],  &x.pos[1],  &x.pos[2],  &x.nd[0],  &x.nd[1],  &x.nd[2]};
    for (int j = 0; j < pw.w; ++j) {
        double g = 0.0;
        for (int o = 0; o < 18; ++o) g += lam[o] * outs[o]->d[j];
        g += lam[20] * inc.d[j];
        gnode[j] += g;
    }
    return ok ? 0u : ADJ_ERR_WINDOW;
}

/* adds a thread's node gradients into a.grad: warp sums, one atomic per
 * node and warp */
__device__ void reduce_nodes(const AdjSweep& a, const double* gacc) {
    const int lane = threadIdx.x & 31;
    for (int k = 0; k < a.nodes; ++k) {
        double v = gacc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0 && v != 0.0) atomicAdd(a.grad + k, v);
    }
}

}  // namespace

/* lambda_m = Phi_m^T lambda_{m+1} + seeds_m for m = m1-1 .. m0 */
__global__ void __launch_bounds__(128) k_adj_reverse(AdjSweep a, __grid_constant__ const QueueDev q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double gacc[ADJ_MAX_NODES];
    for (int k = 0; k < a.nodes; ++k) gacc[k] = 0.0;
    const int n = q.n;
    const bool active = i < n && (int64_t)a.last[i] - 1 >= a.m0;
    if (active) {
        double lam[ADJ_L];
        for (int c = 0; c < ADJ_L; ++c) lam[c] = a.lam[(size_t)c * n + i];
        uint32_t err = 0;
        for (int64_t m = a.m1 - 1; m >= a.m0; --m) {
            const int64_t j = m - a.m0;
            bool any = false;
            for (int c = 0; c < ADJ_L; ++c) any |= lam[c] != 0.0;
            if (any && m < a.m_end) {
                const double* Sb = a.seg + (size_t)j * ADJ_S * n;
                double S[ADJ_S];
                for (int c = 0; c < ADJ_S; ++c) S[c] = Sb[(size_t)c * n + i];
                const uint32_t code = a.chain[(size_t)j * n + i];
                ParamWin pw = window_at(q, S[12], 0);
                double lam0[ADJ_S], gnode[ADJ_W];
                for (int c = 0; c < ADJ_S; ++c) lam0[c] = 0.0;
                for (int c = 0; c < ADJ_W; ++c) gnode[c] = 0.0;
                if (code == 0) {
                    err |= step_vjp_blocked(q, a, S, pw, lam, lam0, gnode);
                } else {
                    for (int off = 0; off < ADJ_S + pw.w; off += ADJ_NB)
                        err |= step_vjp_pass<ADJ_NB>(q, a, S, code, pw, off, lam, lam0, gnode);
                }
                for (int c = 0; c < pw.w; ++c) gacc[pw.k0 + c] += gnode[c];
                const double la_v = lam[18], la_c = lam[19], la_x = lam[20];
                for (int c = 0; c < ADJ_S; ++c) lam[c] = lam0[c];
                lam[18] = 0.0;
                lam[19] = la_v;
                lam[20] = la_c + la_x;
            } else if (m < a.m_end) {
                for (int c = 0; c < ADJ_L; ++c) lam[c] = 0.0;
            }
            const double* sd = a.seed + (size_t)j * ADJ_L * n;
            for (int c = 0; c < ADJ_L; ++c) lam[c] += sd[(size_t)c * n + i];
        }
        for (int c = 0; c < ADJ_L; ++c) a.lam[(size_t)c * n + i] = lam[c];
        if (err) atomicOr(a.err, err);
    }
    reduce_nodes(a, gacc);
}

/* lambda_0 through the start-up */
__global__ void __launch_bounds__(128) k_adj_startup(AdjSweep a, __grid_constant__ const QueueDev q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double gacc[ADJ_MAX_NODES];
    for (int k = 0; k < a.nodes; ++k) gacc[k] = 0.0;
    if (i < q.n && a.last[i] > 0) {
        double lam[ADJ_L];
        bool any = false;
        for (int c = 0; c < ADJ_L; ++c) {
            lam[c] = a.lam[(size_t)c * q.n + i];
            any |= lam[c] != 0.0;
        }
        if (any) {
            const ParamWin pw = window_at(q, q.source[0], 0);
            double gnode[ADJ_W];
            for (int c = 0; c < ADJ_W; ++c) gnode[c] = 0.0;
            const uint32_t err = startup_vjp(q, a, i, pw, lam, gnode);
            if (err) atomicOr(a.err, err);
            for (int c = 0; c < pw.w; ++c) gacc[pw.k0 + c] += gnode[c];
        }
    }
    reduce_nodes(a, gacc);
}

#endif  // WQ3D_ADJOINT_IMPL

}  // namespace wq3d
