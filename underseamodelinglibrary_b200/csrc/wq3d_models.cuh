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

#ifdef __CUDACC__
#define WQ_HD __host__ __device__ __forceinline__
#else
#define WQ_HD inline
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

/* rectilinear grid with up to 3 axes (types/gen_grid.h) */
struct GridDev {
    int ndim;
    const double* axis[3];
    int n[3];
    int interp[3];
    int edge[3];
    const double* data;
};

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
};

/* ------------------------------------------------------------------ */
/* sound speed: profile_{linear,munk,catenary,n2}.cc + adjust_speed     */
/* ------------------------------------------------------------------ */
WQ_HD void sound_speed(const ProfileDev& pr, double R, double rho,
                       double* c, double* g_rho) {
    const double alt = rho - R;
    double cc, gr;
    switch (pr.kind) {
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
    *g_rho = gr;
}

/* ------------------------------------------------------------------ */
/* boundary height: boundary_flat.cc:39-63, boundary_slope.cc:55-68     */
/* ------------------------------------------------------------------ */
WQ_HD double boundary_height(const BoundaryDev& b, double theta, double phi) {
    if (b.kind == WQ3D_BOUNDARY_SLOPE) {
        return b.height * (1.0 + b.slope_a * (phi - b.loc_phi)) *
               (1.0 + b.slope_b * (theta - b.loc_theta));
    }
    return b.height;
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
