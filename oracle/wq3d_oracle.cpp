/*
 * wq3d_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the USML WaveQ3D propagation path, used by tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py as the
 * checker for the CUDA engine.  It is never linked into the product.
 *
 * It restates, with plain std::vector storage instead of Boost uBLAS, the
 * reference's arithmetic in the reference's operation order (build with
 * -ffp-contract=off so no FMA contraction changes a rounding):
 *   waveq3d/wave_queue.cc        ctor, init_wavefronts, step, reflections,
 *                                caustics, eigenray detection and build
 *   waveq3d/wave_front.cc        init_wave, update, find_edges,
 *                                compute_target_distance
 *   waveq3d/ode_integ.cc         RK3 stages and AB3
 *   waveq3d/reflection_model.cc  bottom/surface reflection and re-init
 *   waveq3d/spreading_hybrid_gaussian.cc, waveq3d/spreading_ray.cc
 *   ocean/profile_*.cc, boundary_{flat,slope}.cc, reflect_loss_*.{h,cc},
 *   attenuation_{thorp,constant}.cc, types/wvector1.cc
 *   biverbs/biverb_generator.cc, biverbs/biverb_collection.cc,
 *   eigenverbs/eigenverb_collection.cc (find_eigenverbs),
 *   ocean/scattering_{constant,lambert,chapman}.h, types/wposition1.cc
 * Each function cites the file:line it follows.  Reference quirks are kept
 * on purpose (they are listed where they occur).
 *
 * Parity pin: tests/test_oracle_kats.py checks this code against the
 * analytic known-answer values of the reference's own tests
 * (waveq3d/test/eigenray_test.cc, refraction_test.cc, reflection_test.cc,
 * proploss_test.cc).  The reference itself cannot be built here (it needs
 * Boost uBLAS and netCDF, neither of which is installed).
 *
 * The C entry points mirror include/wq3d.h with an "oracle_" prefix.
 */
#include "../include/wq3d.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#ifndef ORACLE_OPCOUNT
/* the Rayleigh loss's complex arithmetic and the C-ABI arrays (plain
 * double also in the op-counting build, opcount.cpp) */
typedef double oracle_plain_double;
#endif
/* the op-counting build (opcount.cpp) attributes the operations of a
 * scope to a phase of the step: 1 target distances, 2 CPA search, 3
 * eigenray construction (everything else is 0, the ray step itself) */
#ifdef ORACLE_OPCOUNT
#define ORACLE_PHASE(p) wq3d_opcount::Phase oracle_phase_scope_(p)
#else
#define ORACLE_PHASE(p)
#endif
/* C-ABI double arrays seen as the oracle's scalar type and back (casts
 * that change nothing except in the op-counting build) */
template <class T>
inline const double* abi_in(const T* p) { return reinterpret_cast<const double*>(p); }
template <class T>
inline oracle_plain_double* abi_out(T* p) { return reinterpret_cast<oracle_plain_double*>(p); }
template <class T>
inline const oracle_plain_double* abi_out(const T* p) { return reinterpret_cast<const oracle_plain_double*>(p); }

namespace {

const double PI = M_PI;
const double TWO_PI = 2.0 * M_PI;
inline double to_radians(double t) { return t * (M_PI / 180.0); }
inline double to_degrees(double t) { return t * (180.0 / M_PI); }
/* usml copysign (ublas/math_traits.h:176): sign taken from "v < 0" only */
inline double usml_copysign(double t, double v) { return (v < 0.0) ? -t : t; }

std::string g_err;

/* ------------------------------------------------------------------ */
/* ocean models                                                        */
/* ------------------------------------------------------------------ */

/* seq_vector axis used by a grid (types/seq_vector.h) */
struct Axis {
    std::vector<double> x, inc;
    int kind = WQ3D_AXIS_LINEAR;
    double sign = 1.0;
    size_t size() const { return x.size(); }
    /* seq_vector::increment clamps (seq_vector.h:140-143) */
    double increment(size_t i) const { return inc[std::max((size_t)0, std::min(x.size() - 1, i))]; }
    /* seq_linear.h:89-94, seq_log.h:88-94, seq_data.cc:15-36 */
    size_t find_index(double value) const {
        if (kind == WQ3D_AXIS_LINEAR) {
            return (size_t)std::max((long)0, std::min((long)size() - 2, (long)std::floor((value - x[0]) / inc[0])));
        }
        if (kind == WQ3D_AXIS_LOG) {
            return (size_t)std::max((long)0, std::min((long)size() - 2,
                                                      (long)std::floor(std::log(value / x[0]) / std::log(inc[1] / inc[0]))));
        }
        value *= sign;
        const size_t max_index = size() - 1;
        if (max_index < 1) return 0;
        if (value <= sign * x[0]) return 0;
        if (value >= sign * x[max_index - 1]) return max_index - 1;
        /* std::map<key, index>::upper_bound over keys sign*x[n] */
        size_t n = 0;
        while (n < size() && !(sign * x[n] > value)) ++n;
        return n - 1;
    }
};

/* gen_grid<N, double> (types/gen_grid.h:83-520) */
struct Grid {
    int ndim = 0;
    Axis axis[3];
    std::vector<double> data;
    int interp[3] = {0, 0, 0};
    int edge[3] = {1, 1, 1};

    double at(const size_t* index) const {
        size_t off = index[0];
        for (int d = 1; d < ndim; ++d) off = index[d] + axis[d].size() * off;
        return data[off];
    }
    double interp_dim(int dim, const size_t* index, const double* loc, double& deriv, double* dv) const {
        if (dim < 0) return at(index);
        if (axis[dim].size() < 2) return nearest(dim, index, loc, deriv, dv);
        switch (interp[dim]) {
            case WQ3D_INTERP_NEAREST:
                return nearest(dim, index, loc, deriv, dv);
            case WQ3D_INTERP_PCHIP:
                return pchip(dim, index, loc, deriv, dv);
            default:
                return linear(dim, index, loc, deriv, dv);
        }
    }
    double nearest(int dim, const size_t* index, const double* loc, double& deriv, double* dv) const {
        double result, da = 0.0;
        const size_t k = index[dim];
        const Axis& ax = axis[dim];
        const double u = (loc[dim] - ax.x[k]) / ax.increment(k);
        if (u < 0.5) {
            result = interp_dim(dim - 1, index, loc, da, dv);
        } else {
            size_t next[3] = {index[0], index[1], index[2]};
            ++next[dim];
            result = interp_dim(dim - 1, next, loc, da, dv);
        }
        if (dv) {
            dv[dim] = deriv;
            if (dim > 0) dv[dim - 1] = da;
        }
        return result;
    }
    double linear(int dim, const size_t* index, const double* loc, double& deriv, double* dv) const {
        double da = 0.0, db = 0.0;
        const double a = interp_dim(dim - 1, index, loc, da, dv);
        size_t next[3] = {index[0], index[1], index[2]};
        ++next[dim];
        const double b = interp_dim(dim - 1, next, loc, db, dv);
        const size_t k = index[dim];
        const Axis& ax = axis[dim];
        const double h = ax.increment(k);
        const double u = (loc[dim] - ax.x[k]) / h;
        const double result = a * (1.0 - u) + b * u;
        if (dv) {
            deriv = (b - a) / h;
            dv[dim] = deriv;
            if (dim > 0) dv[dim - 1] = da * (1.0 - u) + db * u;
        }
        return result;
    }
    /* gen_grid_utils.h derivative<double> / end_point_derivative<double> */
    static void harmonic(double d0, double d1, double dd0, double dd1, double w0, double w1, bool deriv,
                         double& m, double& dm) {
        if (d0 * d1 > 0.0) m = (w0 + w1) / (w0 / d0 + w1 / d1);
        if (deriv && dd0 * dd1 > 0.0) dm = (w0 + w1) / (w0 / dd0 + w1 / dd1);
    }
    static void end_point(double d0, double d1, double dd0, double dd1, bool deriv, double& m, double& dm) {
        if (m * d0 < 0.0) {
            m = 0.0;
        } else if ((d0 * d1 < 0.0) && (std::abs(m) > std::abs(3.0 * d1))) {
            m = 3.0 * d1;
        }
        if (deriv) {
            if (dm * dd0 < 0.0) {
                dm = 0.0;
            } else if ((dd0 * dd1 < 0.0) && (std::abs(dm) > std::abs(3.0 * dd0))) {
                dm = 3.0 * dd0;
            }
        } else {
            dm = 0.0;
        }
    }
    /* gen_grid.h pchip, with its end-point formulas as written */
    double pchip(int dim, const size_t* index, const double* loc, double& deriv, double* dv) const {
        const Axis& ax = axis[dim];
        const size_t kmin = 1u;
        const size_t kmax = ax.size() - 3u;
        double y0, y1, y2, y3, dy0 = 0.0, dy1 = 0.0, dy2 = 0.0, dy3 = 0.0;
        const size_t k = index[dim];
        y1 = interp_dim(dim - 1, index, loc, dy1, dv);
        if (k >= kmin) {
            size_t prev[3] = {index[0], index[1], index[2]};
            --prev[dim];
            y0 = interp_dim(dim - 1, prev, loc, dy0, dv);
        } else {
            y0 = y1;
            dy0 = dy1;
        }
        size_t next[3] = {index[0], index[1], index[2]};
        ++next[dim];
        y2 = interp_dim(dim - 1, next, loc, dy2, dv);
        if (k <= kmax) {
            size_t last[3] = {next[0], next[1], next[2]};
            ++last[dim];
            y3 = interp_dim(dim - 1, last, loc, dy3, dv);
        } else {
            y3 = y2;
            dy3 = dy2;
        }
        const double h0 = ax.increment(k - 1);
        const double h1 = ax.increment(k);
        const double h2 = ax.increment(k + 1);
        const double h1_2 = h1 * h1;
        const double h1_3 = h1_2 * h1;
        const double s = loc[dim] - ax.x[k];
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
                              slope2 * s_2 * sh_minus / h1_2 + slope1 * s * sh_minus * sh_minus / h1_2;
        if (dv) {
            const double v = s / h1;
            deriv = slope1 * (1.0 - v) + slope2 * v;
            dv[dim] = deriv;
            if (dim > 0)
                dv[dim - 1] = dy2 * sh_term / h1_3 + dy1 * (h1_3 - sh_term) / h1_3 +
                              dslope2 * s_2 * sh_minus / h1_2 + dslope1 * s * sh_minus * sh_minus / h1_2;
        }
        return result;
    }
    /* gen_grid::interpolate (gen_grid.h:83-123) */
    double interpolate(const double* location, double* dv) const {
        size_t index[3] = {0, 0, 0};
        double loc[3] = {0, 0, 0};
        for (int d = 0; d < ndim; ++d) loc[d] = location[d];
        for (int d = 0; d < ndim; ++d) {
            const Axis& ax = axis[d];
            if (ax.size() < 2) {
                loc[d] = ax.x[0];
                index[d] = 0;
            } else if (edge[d]) {
                const double a = ax.x[0];
                const double b = ax.x[ax.size() - 1];
                const double sign = (ax.increment(0) < 0) ? -1.0 : 1.0;
                const double dd = loc[d] * sign;
                if (dd <= a * sign) {
                    loc[d] = a;
                    index[d] = 0;
                } else if (dd >= b * sign) {
                    loc[d] = b;
                    index[d] = ax.size() - 2;
                } else {
                    index[d] = ax.find_index(loc[d]);
                }
            } else {
                index[d] = ax.find_index(loc[d]);
            }
        }
        double dresult = 0.0;
        return interp_dim(ndim - 1, index, loc, dresult, dv);
    }
};

void load_grid(Grid& g, const wq3d_grid_desc& d) {
    g.ndim = d.ndim;
    size_t total = 1;
    for (int k = 0; k < d.ndim; ++k) {
        const size_t n = d.axis_size[k];
        g.axis[k].x.assign(d.axis[k], d.axis[k] + n);
        g.axis[k].inc.assign(d.axis_inc[k], d.axis_inc[k] + n);
        g.axis[k].kind = d.axis_kind[k];
        g.axis[k].sign = (n > 1 && d.axis[k][1] - d.axis[k][0] < 0) ? -1.0 : 1.0;
        int it = d.interp[k];
        /* data_grid::interp_type (data_grid.h:137-145) */
        if (it > WQ3D_INTERP_NEAREST && n < 2) {
            it = WQ3D_INTERP_NEAREST;
        } else if (it > WQ3D_INTERP_LINEAR && n < 4) {
            it = WQ3D_INTERP_LINEAR;
        }
        g.interp[k] = it;
        g.edge[k] = d.edge_limit[k] ? 1 : 0;
        total *= n;
    }
    g.data.assign(d.data, d.data + total);
}

struct Boundary {
    int kind = WQ3D_BOUNDARY_FLAT;
    double height = 0.0;      /* flat/slope: _height */
    double normal_rho = 1.0;  /* flat */
    double loc[3] = {0, 0, 0};/* slope: _location (copied, see quirk note) */
    double nrm[3] = {0, 0, 0};/* slope: _normal (rho, theta, phi) */
    Grid grid;
    wq3d_reflect_loss_desc loss{};
    /* rayleigh derived constants (reflect_loss_rayleigh.cc:68-78) */
    double rl_den = 0, rl_spd = 0, rl_att = 0, rl_shr = 0, rl_satt = 0;
};

struct Ocean {
    wq3d_profile_desc prof{};
    Grid pgrid;
    Boundary surf, bot;
    double build_radius = 6371000.0;
    std::vector<double> vol_rho; /* volume_flat::_rho per layer (volume_flat.h:32-37) */
};

/* profile_munk.cc:19-32, profile_linear.cc:14-40, profile_catenary.cc:14-29,
 * profile_n2.cc:14-24, with profile_model::adjust_speed (profile_model.cc:14-26) */
void sound_speed(const Ocean& oc, double R, double rho, double theta,
                 double phi, double* c, double* g) {
    const double* p = abi_in(oc.prof.p);
    const double alt = rho - R;
    double gr = 0.0, gt = 0.0, gp = 0.0;
    double cc = 0.0;
    switch (oc.prof.kind) {
        case WQ3D_PROFILE_LINEAR: {
            const double z = -alt;
            if (z < p[2]) {
                cc = p[0] + p[1] * z;
                gr = -p[1];
            } else {
                cc = p[0] + p[1] * p[2] + p[3] * (z - p[2]);
                gr = -p[3];
            }
            break;
        }
        case WQ3D_PROFILE_MUNK: {
            const double z = 2.0 * (-alt - p[0]) / p[1];
            cc = (((z - 1.0) + std::exp(-z)) * p[3] + 1.0) * p[2];
            gr = (1.0 - std::exp(-z)) * (-p[3] * p[2] * 2.0 / p[1]);
            break;
        }
        case WQ3D_PROFILE_CATENARY: {
            cc = p[0] * std::cosh((alt + p[2]) / (-p[1]));
            gr = -std::sinh((alt + p[2]) / (-p[1])) * (p[0] / p[1]);
            break;
        }
        case WQ3D_PROFILE_N2: {
            const double factor = 2.0 * p[1] / p[0];
            cc = p[0] / std::sqrt(1.0 - alt * factor);
            gr = std::pow(cc, 3.0) * factor / (2.0 * p[0] * p[0]);
            break;
        }
        case WQ3D_PROFILE_GRID: {
            /* profile_grid.h:68-130 */
            const double loc[3] = {rho, theta, phi};
            double dv[3] = {0.0, 0.0, 0.0};
            cc = oc.pgrid.interpolate(loc, dv);
            gr = dv[0];
            if (oc.pgrid.ndim >= 2) gt = dv[1];
            if (oc.pgrid.ndim >= 3) gp = dv[2];
            break;
        }
        default:
            cc = 1500.0;
    }
    if (oc.prof.flat_earth) {
        gr = (gr * rho + cc) / R;
        cc = cc * rho / R;
    }
    *c = cc;
    if (g) {
        g[0] = gr;
        g[1] = gt;
        g[2] = gp;
    }
}

/* boundary_flat.cc:39-63, boundary_slope.cc:31-68 */
void height(const Boundary& b, double rho, double theta, double phi,
            double* h, double* n) {
    (void)rho;
    if (b.kind == WQ3D_BOUNDARY_GRID) {
        /* boundary_grid.h:150-196 */
        const double loc[2] = {theta, phi};
        double grad[2] = {0.0, 0.0};
        *h = b.grid.interpolate(loc, n ? grad : nullptr);
        if (n) {
            if (b.grid.ndim == 1) {
                const double t = -grad[0] / (*h);
                const double N = std::sqrt(1 + t * t);
                n[0] = 1.0 / N;
                n[1] = t / N;
                n[2] = 0.0;
            } else {
                const double t = -grad[0] / (*h);
                const double pp = -grad[1] / ((*h) * std::sin(theta));
                const double N = std::sqrt(1 + t * t + pp * pp);
                n[0] = 1.0 / N;
                n[1] = t / N;
                n[2] = pp / N;
            }
        }
        return;
    }
    if (b.kind == WQ3D_BOUNDARY_SLOPE) {
        const double alpha = -std::asin(b.nrm[1]);
        const double beta = -std::asin(b.nrm[2]);
        *h = b.height *
             (1.0 + std::sin(b.loc[1]) * std::tan(beta) * (phi - b.loc[2])) *
             (1.0 + std::tan(alpha) * (theta - b.loc[1]));
        if (n) {
            n[0] = b.nrm[0];
            n[1] = b.nrm[1];
            n[2] = b.nrm[2];
        }
        return;
    }
    *h = b.height;
    if (n) {
        n[0] = b.normal_rho;
        n[1] = 0.0;
        n[2] = 0.0;
    }
}

/* reflect_loss_constant.h:42-52, reflect_loss_rayleigh.cc:83-144,
 * reflect_loss_eckart.h:76-85.  amplitude/phase are per frequency. */
void reflect_loss(const Boundary& b, const std::vector<double>& freq,
                  double angle, double* amp, double* ph) {
    const size_t nf = freq.size();
    switch (b.loss.kind) {
        case WQ3D_LOSS_RAYLEIGH: {
            typedef std::complex<oracle_plain_double> cd;
            const double dw = 1000.0, sw = 1500.0;
            if (angle >= M_PI_2) angle = M_PI_2 - 1e-10;
            angle = M_PI_2 - angle;
            const double Zw = std::cos(angle) / (sw * dw);
            auto impedance = [&](double density, double speed, double att,
                                 cd* cosA, bool shear) {
                const cd c(speed, -att * speed);
                cd sinA = std::sin(angle) * c / sw;
                *cosA = std::sqrt(1.0 - sinA * sinA);
                cd value;
                if (shear) {
                    value = c * density / *cosA;
                } else {
                    value = *cosA / (c * density);
                }
                return value;
            };
            cd cosAp, cosAs;
            cd Zb = impedance(b.rl_den, b.rl_spd, b.rl_att, &cosAp, false);
            if (b.rl_shr != 0.0 || b.rl_satt != 0.0) {
                const cd Zs = impedance(b.rl_den, b.rl_shr, b.rl_satt, &cosAs, true);
                const cd sinAs = std::sqrt(1.0 - cosAs * cosAs);
                const cd cos2As = 2.0 * cosAs * cosAs - 1.0;
                const cd sin2As = 2.0 * sinAs * cosAs;
                Zb = 1.0 / ((1.0 / Zb) * cos2As * cos2As + Zs * sin2As * sin2As);
            }
            const cd R = (Zb - Zw) / (Zb + Zw);
            const double a = -20.0 * std::log10(std::abs(R));
            const double p = std::arg(R);
            for (size_t f = 0; f < nf; ++f) {
                amp[f] = a * 1.0;
                if (ph) ph[f] = p * 1.0;
            }
            break;
        }
        case WQ3D_LOSS_ECKART: {
            const double w2 = b.loss.p[0] * b.loss.p[0];
            for (size_t f = 0; f < nf; ++f) {
                const double x = freq[f] * w2 * std::sin(angle);
                amp[f] = 8.6e-9 * (x * x);
                if (ph) ph[f] = M_PI;
            }
            break;
        }
        default:
            for (size_t f = 0; f < nf; ++f) {
                amp[f] = b.loss.p[0];
                if (ph) ph[f] = b.loss.p[1];
            }
    }
}

void setup_boundary(Boundary& b, const wq3d_boundary_desc& d, double R,
                    bool is_surface) {
    b.kind = d.kind;
    b.loss = d.loss;
    if (d.kind == WQ3D_BOUNDARY_SLOPE) {
        /* boundary_slope.cc:13-24; the reference keeps a reference to the
         * caller's wposition1 (boundary_slope.h:84); here it is copied. */
        b.loc[0] = d.location[0];
        b.loc[1] = d.location[1];
        b.loc[2] = d.location[2];
        b.height = R - d.depth;
        b.nrm[1] = std::sin(d.lat_slope);
        b.nrm[2] = -std::sin(d.lng_slope);
        b.nrm[0] = std::sqrt(1.0 - b.nrm[1] * b.nrm[1] - b.nrm[2] * b.nrm[2]);
        if (d.loss.kind == WQ3D_LOSS_DEFAULT) {
            b.loss.kind = WQ3D_LOSS_CONSTANT;
            b.loss.p[0] = 0.0;
            b.loss.p[1] = 0.0;
        }
    } else if (d.kind == WQ3D_BOUNDARY_GRID) {
        load_grid(b.grid, d.grid);
        /* boundary_grid.h:56-59 */
        if (d.loss.kind == WQ3D_LOSS_DEFAULT) {
            b.loss.kind = WQ3D_LOSS_RAYLEIGH;
            const double sand[5] = {1.9, 1.10, 0.8, 0.00, 2.5};
            for (int k = 0; k < 5; ++k) b.loss.p[k] = sand[k];
        }
    } else {
        /* boundary_flat.cc:19-31 */
        b.kind = WQ3D_BOUNDARY_FLAT;
        b.height = R - std::abs(d.depth);
        if (std::abs(d.depth) < 1e-6) {
            b.normal_rho = -1.0;
            if (d.loss.kind == WQ3D_LOSS_DEFAULT) {
                b.loss.kind = WQ3D_LOSS_CONSTANT;
                b.loss.p[0] = 0.0;
                b.loss.p[1] = M_PI;
            }
        } else {
            b.normal_rho = 1.0;
        }
        if (b.loss.kind == WQ3D_LOSS_DEFAULT) {
            b.loss.kind = WQ3D_LOSS_CONSTANT;
            b.loss.p[0] = 0.0;
            b.loss.p[1] = 0.0;
        }
    }
    (void)is_surface;
    if (b.loss.kind == WQ3D_LOSS_RAYLEIGH) {
        /* reflect_loss_rayleigh.cc:17,68-78 */
        const double ATT_CONVERT = 1.0 / (20.0 * M_LOG10E * TWO_PI);
        b.rl_den = 1000.0 * b.loss.p[0];
        b.rl_spd = 1500.0 * b.loss.p[1];
        b.rl_att = b.loss.p[2] * ATT_CONVERT;
        b.rl_shr = 1500.0 * b.loss.p[3];
        b.rl_satt = b.loss.p[4] * ATT_CONVERT;
    }
}

/* ------------------------------------------------------------------ */
/* wavefronts                                                          */
/* ------------------------------------------------------------------ */

/* one ray of a 1x1 wave_front, used by reflection_reinit */
struct Ray {
    double pos[3] = {0, 0, 0};
    double pg[3] = {0, 0, 0};
    double nd[3] = {0, 0, 0};
    double ng[3] = {0, 0, 0};
    double c = 0.0;
    double sg[3] = {0, 0, 0};
    double dist = 0.0;
};

/* wave_front.cc:133-171 (Reilly eqs. 36-41) for one ray */
inline void derivs(double c, const double* sg, const double* pos,
                   const double* nd, double* pg, double* ng, double* sin_t) {
    const double dcc_r = sg[0] / c;
    const double dcc_t = sg[1] / c;
    const double dcc_p = sg[2] / c;
    const double st = std::sin(pos[1]);
    const double ct = std::cos(pos[1]) / st;
    const double c2 = c * c;
    pg[0] = c2 * nd[0];
    const double c2r = c2 / pos[0];
    pg[1] = c2r * nd[1];
    pg[2] = (c2r / st) * nd[2];
    ng[0] = c2r * (nd[1] * nd[1] + nd[2] * nd[2]) - dcc_r;
    ng[1] = (-c2r) * (nd[0] * nd[1] - (nd[2] * nd[2]) * ct) - dcc_t / pos[0];
    ng[2] = (-c2r) * (nd[2] * (nd[0] + nd[1] * ct)) - dcc_p / (pos[0] * st);
    if (sin_t) *sin_t = st;
}

struct Front {
    size_t n = 0, nf = 0, nt = 0;
    std::vector<double> pos[3], pg[3], nd[3], ng[3], c, sg[3], dist, plen;
    std::vector<double> atten, phase; /* n*nf */
    std::vector<int> surface, bottom, caustic, upper, lower;
    std::vector<unsigned char> on_edge;
    std::vector<double> sin_t; /* wave_front::_sin_theta */
    std::vector<double> d2;    /* nt*n, distance2(t1,t2)(de,az) */

    void alloc(size_t n_, size_t nf_, size_t nt_) {
        n = n_;
        nf = nf_;
        nt = nt_;
        for (int k = 0; k < 3; ++k) {
            pos[k].assign(n, 0.0);
            pg[k].assign(n, 0.0);
            nd[k].assign(n, 0.0);
            ng[k].assign(n, 0.0);
            sg[k].assign(n, 0.0);
        }
        c.assign(n, 0.0);
        dist.assign(n, 0.0);
        plen.assign(n, 0.0);
        atten.assign(n * nf, 0.0);
        phase.assign(n * nf, 0.0);
        surface.assign(n, 0);
        bottom.assign(n, 0);
        caustic.assign(n, 0);
        upper.assign(n, 0);
        lower.assign(n, 0);
        on_edge.assign(n, 0);
        sin_t.assign(n, 0.0);
        d2.assign(nt * n, 0.0);
    }
    void get(size_t r, Ray& y) const {
        for (int k = 0; k < 3; ++k) {
            y.pos[k] = pos[k][r];
            y.pg[k] = pg[k][r];
            y.nd[k] = nd[k][r];
            y.ng[k] = ng[k][r];
            y.sg[k] = sg[k][r];
        }
        y.c = c[r];
        y.dist = dist[r];
    }
};

struct Eig {
    wq3d_eigenray rec;
    std::vector<double> inten, phase;
};

struct Queue {
    Ocean oc;
    double R = 6371000.0;
    std::vector<double> freq, de, de_inc, az, az_inc;
    size_t nde = 0, naz = 0, nf = 0, n = 0, nt1 = 0, nt2 = 0, nt = 0;
    double src[3] = {0, 0, 0};      /* _source_pos (clamped) */
    double src_in[3] = {0, 0, 0};   /* pos passed to ctor */
    double dt = 0.1, time = 0.0;
    int64_t steps = 0;
    std::vector<double> tgt[3], tgt_sin;
    bool has_targets = false;
    bool az_boundary = false, de_branch = false;
    int spreading = WQ3D_HYBRID_GAUSSIAN;
    bool has_spreading = false;
    wq3d_thresholds th{300.0, 300.0, 999, 999, 999, 999, 999};
    double eigenverb_thresh = 1e-30;
    std::vector<double> alpha; /* thorp coefficients */
    Front F[4];
    Front *past, *prev, *curr, *next;
    /* spreading_hybrid_gaussian / spreading_ray members */
    std::vector<double> norm_de, norm_az, init_area;
    std::vector<double> spread, beam_width, int_de, int_az;
    std::vector<unsigned char> dup;
    double init_sound_speed = 0.0;
    std::vector<Eig> found;
    std::vector<wq3d_reflection> refl;
    bool want_refl = false;
    bool want_verbs = false;
    std::vector<wq3d_eigenverb> verbs;
    std::vector<double> verb_power;
    int32_t ev_seq = 0;  /* events of the ray being processed this step */
    wq3d_callbacks cb{};
    void* cb_ctx = nullptr;
    uint64_t run_id = 0;

    size_t idx(size_t d, size_t a) const { return d * naz + a; }

    /* attenuation_thorp.cc:14-36 / attenuation_constant.cc:14-25 */
    void attenuation(Front& f, size_t r) {
        const double alt = f.pos[0][r] - R;
        for (size_t k = 0; k < nf; ++k) {
            if (oc.prof.attenuation == WQ3D_ATTEN_CONSTANT) {
                f.atten[r * nf + k] = oc.prof.attenuation_coef * f.dist[r] * freq[k];
            } else {
                f.atten[r * nf + k] = f.dist[r] * alpha[k] * (1.0 + 5.88264e-6 * alt);
            }
        }
    }

    /* wave_front::update (wave_front.cc:125-178) over a whole front */
    void update(Front& f) {
        for (size_t r = 0; r < n; ++r) {
            double p3[3] = {f.pos[0][r], f.pos[1][r], f.pos[2][r]};
            double nd3[3] = {f.nd[0][r], f.nd[1][r], f.nd[2][r]};
            double sg3[3];
            sound_speed(oc, R, p3[0], p3[1], p3[2], &f.c[r], sg3);
            for (int k = 0; k < 3; ++k) f.sg[k][r] = sg3[k];
            attenuation(f, r);
            for (size_t k = 0; k < nf; ++k) f.phase[r * nf + k] = 0.0;
            double pg3[3], ng3[3];
            derivs(f.c[r], sg3, p3, nd3, pg3, ng3, &f.sin_t[r]);
            for (int k = 0; k < 3; ++k) {
                f.pg[k][r] = pg3[k];
                f.ng[k][r] = ng3[k];
            }
        }
        if (has_targets) compute_target_distance(f);
    }

    /* wave_front::compute_target_distance (wave_front.cc:222-236) */
    void compute_target_distance(Front& f) {
        ORACLE_PHASE(1);
        for (size_t t = 0; t < nt; ++t) {
            const double R2 = tgt[0][t], TH = tgt[1][t], PH = tgt[2][t];
            const double S = tgt_sin[t];
            double* out = &f.d2[t * n];
            for (size_t r = 0; r < n; ++r) {
                const double rr = f.pos[0][r];
                const double a = 0.5 * (f.pos[1][r] - TH);
                const double b = 0.5 * (f.pos[2][r] - PH);
                const double inner = 1.0 - 2.0 * (a * a + S * (f.sin_t[r] * (b * b)));
                out[r] = std::abs(rr * rr + R2 * R2 - 2.0 * R2 * (rr * inner));
            }
        }
    }

    /* wave_front::update for a 1x1 front without targets */
    void update1(Ray& y) {
        sound_speed(oc, R, y.pos[0], y.pos[1], y.pos[2], &y.c, y.sg);
        derivs(y.c, y.sg, y.pos, y.nd, y.pg, y.ng, nullptr);
    }

    /* ode_integ.cc:20-126 on single rays */
    static void rk1(double h, const Ray& y0, Ray& y1) {
        for (int k = 0; k < 3; ++k) {
            y1.pos[k] = y0.pos[k] + 0.5 * h * y0.pg[k];
            y1.nd[k] = y0.nd[k] + 0.5 * h * y0.ng[k];
        }
    }
    static void rk2(double h, const Ray& y0, const Ray& y1, Ray& y2) {
        for (int k = 0; k < 3; ++k) {
            y2.pos[k] = y0.pos[k] + h * (2.0 * y1.pg[k] - y0.pg[k]);
            y2.nd[k] = y0.nd[k] + h * (2.0 * y1.ng[k] - y0.ng[k]);
        }
    }
    static void rk3(double h, const Ray& y0, const Ray& y1, const Ray& y2,
                    Ray& y3) {
        double p[3], q[3];
        for (int k = 0; k < 3; ++k) {
            p[k] = y0.pos[k] + h / 6.0 * (y0.pg[k] + 4.0 * y1.pg[k] + y2.pg[k]);
            q[k] = y0.nd[k] + h / 6.0 * (y0.ng[k] + 4.0 * y1.ng[k] + y2.ng[k]);
        }
        for (int k = 0; k < 3; ++k) {
            y3.pos[k] = p[k];
            y3.nd[k] = q[k];
        }
    }
    /* ode_integ.cc:131-186 */
    static void ab3(double h, const Ray& y0, const Ray& y1, const Ray& y2,
                    Ray& y3) {
        const double A2 = 23.0 / 12.0, A1 = 16.0 / 12.0, A0 = 5.0 / 12.0;
        double d[3];
        for (int k = 0; k < 3; ++k)
            d[k] = h * (A2 * y2.pg[k] - A1 * y1.pg[k] + A0 * y0.pg[k]);
        const double b = y2.pos[0] * d[1];
        const double cc = y2.pos[0] * (std::sin(y2.pos[1]) * d[2]);
        y3.dist = std::sqrt(d[0] * d[0] + b * b + cc * cc);
        for (int k = 0; k < 3; ++k) y3.pos[k] = y2.pos[k] + d[k];
        for (int k = 0; k < 3; ++k)
            y3.nd[k] = y2.nd[k] + h * (A2 * y2.ng[k] - A1 * y1.ng[k] + A0 * y0.ng[k]);
    }

    /* whole-front versions of the RK3 / AB3 stages (wave_queue.cc:114-150) */
    void front_rk(int stage, double h, Front* y0, Front* y1, Front* y2,
                  Front* y3) {
        for (size_t r = 0; r < n; ++r) {
            Ray a, b, c, d;
            y0->get(r, a);
            if (y1) y1->get(r, b);
            if (y2) y2->get(r, c);
            if (stage == 1) {
                rk1(h, a, d);
                for (int k = 0; k < 3; ++k) {
                    y1->pos[k][r] = d.pos[k];
                    y1->nd[k][r] = d.nd[k];
                }
            } else if (stage == 2) {
                rk2(h, a, b, d);
                for (int k = 0; k < 3; ++k) {
                    y2->pos[k][r] = d.pos[k];
                    y2->nd[k][r] = d.nd[k];
                }
            } else {
                rk3(h, a, b, c, d);
                for (int k = 0; k < 3; ++k) {
                    y3->pos[k][r] = d.pos[k];
                    y3->nd[k][r] = d.nd[k];
                }
            }
        }
    }
    void front_ab3(double h, Front* y0, Front* y1, Front* y2, Front* y3) {
        for (size_t r = 0; r < n; ++r) {
            Ray a, b, c, d;
            y0->get(r, a);
            y1->get(r, b);
            y2->get(r, c);
            ab3(h, a, b, c, d);
            y3->dist[r] = d.dist;
            for (int k = 0; k < 3; ++k) {
                y3->pos[k][r] = d.pos[k];
                y3->nd[k][r] = d.nd[k];
            }
        }
    }

    /* ------------------------------------------------------------ */
    int create(const wq3d_ocean_desc* od, const wq3d_queue_desc* qd) {
        oc.prof = od->profile;
        oc.build_radius = od->earth_radius;
        setup_boundary(oc.surf, od->surface, od->earth_radius, true);
        setup_boundary(oc.bot, od->bottom, od->earth_radius, false);
        if (oc.prof.kind == WQ3D_PROFILE_GRID) load_grid(oc.pgrid, od->profile.grid);
        if (od->num_volume < 0 || od->num_volume > WQ3D_MAX_VOLUME) {
            g_err = "oracle: bad number of volume layers";
            return WQ3D_ERR_INVALID;
        }
        for (int k = 0; k < od->num_volume; ++k)
            oc.vol_rho.push_back(od->earth_radius - std::abs(od->volume[k].depth));
        R = qd->earth_radius;
        nde = qd->num_de;
        naz = qd->num_az;
        nf = qd->num_freq;
        n = nde * naz;
        if (nde < 1 || naz < 1 || nf < 1) {
            g_err = "oracle: empty fan";
            return WQ3D_ERR_INVALID;
        }
        freq.assign(qd->freq, qd->freq + nf);
        de.assign(qd->de, qd->de + nde);
        de_inc.assign(qd->de_inc, qd->de_inc + nde);
        az.assign(qd->az, qd->az + naz);
        az_inc.assign(qd->az_inc, qd->az_inc + naz);
        dt = qd->time_step;
        spreading = qd->spreading;
        run_id = qd->run_id;
        has_targets = qd->targets != nullptr &&
                      qd->num_targets1 * qd->num_targets2 > 0;
        nt1 = has_targets ? qd->num_targets1 : 0;
        nt2 = has_targets ? qd->num_targets2 : 0;
        nt = nt1 * nt2;
        for (int k = 0; k < 3; ++k) {
            tgt[k].assign(nt, 0.0);
            for (size_t t = 0; t < nt; ++t) tgt[k][t] = qd->targets[k * nt + t];
        }
        tgt_sin.assign(nt, 0.0);
        for (size_t t = 0; t < nt; ++t) tgt_sin[t] = std::sin(tgt[1][t]);
        alpha.assign(nf, 0.0);
        for (size_t k = 0; k < nf; ++k) {
            double F2 = freq[k];
            F2 = 1e-6 * F2 * F2;
            alpha[k] = 1e-3 *
                       (3.3e-3 + F2 * (0.11 / (1.0 + F2) + 44.0 / (4100.0 + F2) + 3.0e-4)) /
                       (1.0 - 5.88264e-6 * 1000.0);
        }

        /* wave_queue.cc:47-53 */
        az_boundary = false;
        if (naz > 1) {
            const double az_first = std::abs(az[0]);
            const double az_last = std::abs(az[naz - 1]);
            az_boundary = (std::fmod(az_first + 360.0, 360.0) ==
                           std::fmod(az_last + 360.0, 360.0));
        }
        /* wave_queue.cc:58-68 source clamp (applies to _source_pos only) */
        for (int k = 0; k < 3; ++k) src[k] = src_in[k] = qd->source[k];
        {
            const double offset = 0.1;
            double bottom_rho = 0.0;
            height(oc.bot, src[0], src[1], src[2], &bottom_rho, nullptr);
            bottom_rho += offset;
            if (src[0] - R > -offset) {
                src[0] = -offset + R;
            } else if (src[0] < bottom_rho) {
                src[0] = bottom_rho;
            }
        }
        for (auto& f : F) f.alloc(n, nf, nt);
        past = &F[0];
        prev = &F[1];
        curr = &F[2];
        next = &F[3];

        init_wave();
        update(*curr);
        init_wavefronts();

        has_spreading = (nde >= 3 && naz >= 3);
        if (has_spreading) {
            if (spreading == WQ3D_HYBRID_GAUSSIAN)
                init_hybrid();
            else
                init_classic();
        }
        return WQ3D_OK;
    }

    /* wave_front::init_wave (wave_front.cc:84-121), called with the
     * ctor's unclamped pos (wave_queue.cc:83) */
    void init_wave() {
        for (size_t r = 0; r < nde; ++r) {
            const double cos_de = std::cos(to_radians(de[r]));
            const double sin_de = std::sin(to_radians(de[r]));
            for (size_t a = 0; a < naz; ++a) {
                const double cos_az = std::cos(to_radians(az[a]));
                const double sin_az = std::sin(to_radians(az[a]));
                const size_t i = idx(r, a);
                curr->nd[0][i] = sin_de;
                curr->nd[1][i] = -cos_de * cos_az;
                curr->nd[2][i] = cos_de * sin_az;
                curr->pos[0][i] = src_in[0];
                curr->pos[1][i] = src_in[1];
                curr->pos[2][i] = src_in[2];
            }
        }
        double c0;
        sound_speed(oc, R, src_in[0], src_in[1], src_in[2], &c0, nullptr);
        for (int k = 0; k < 3; ++k)
            for (size_t i = 0; i < n; ++i) curr->nd[k][i] = curr->nd[k][i] / c0;
    }

    /* wave_queue.cc:114-150 */
    void init_wavefronts() {
        const double h = -dt;
        front_rk(1, h, curr, next, nullptr, nullptr);
        update(*next);
        front_rk(2, h, curr, next, past, nullptr);
        update(*past);
        front_rk(3, h, curr, next, past, prev);
        update(*prev);

        front_rk(1, h, prev, next, nullptr, nullptr);
        update(*next);
        front_rk(2, h, prev, next, past, nullptr);
        update(*past);
        front_rk(3, h, prev, next, past, past);
        update(*past);

        front_ab3(dt, past, prev, curr, next);
        update(*next);
        for (size_t r = 0; r < n; ++r) next->plen[r] = next->dist[r] + curr->plen[r];
    }

    /* wave_queue.cc:155-192 */
    void step() {
        ++steps;
        detect_reflections();
        Front* save = past;
        past = prev;
        prev = curr;
        curr = next;
        next = save;
        time += dt;

        front_ab3(dt, past, prev, curr, next);
        update(*next);
        for (size_t r = 0; r < n; ++r) {
            next->plen[r] = next->dist[r] + curr->plen[r];
            for (size_t k = 0; k < nf; ++k) {
                next->atten[r * nf + k] += curr->atten[r * nf + k];
                next->phase[r * nf + k] += curr->phase[r * nf + k];
            }
            next->surface[r] = curr->surface[r];
            next->bottom[r] = curr->bottom[r];
            next->upper[r] = curr->upper[r];
            next->lower[r] = curr->lower[r];
            next->caustic[r] = curr->caustic[r];
        }
        detect_eigenrays();
        deliver();
        if (cb.check_eigenrays) cb.check_eigenrays(cb_ctx, time, run_id);
    }

    /* wave_queue.cc:197-216 */
    void detect_reflections() {
        for (size_t d = 0; d < nde; ++d) {
            for (size_t a = 0; a < naz; ++a) {
                ev_seq = 0;
                detect_volume_scattering(d, a);
                if (!detect_surface(d, a)) {
                    if (!detect_bottom(d, a)) {
                        detect_vertices(d, a);
                        detect_caustics(d, a);
                    }
                }
            }
        }
        find_edges(*next);
    }

    /* wave_queue.cc:222-234 */
    bool detect_surface(size_t d, size_t a) {
        const size_t i = idx(d, a);
        if (next->pos[0][i] - R > 0.0) {
            if (surface_reflection(d, a)) {
                next->surface[i] += 1;
                curr->surface[i] = prev->surface[i] = past->surface[i] = next->surface[i];
                detect_volume_scattering(d, a);
                detect_bottom(d, a);
                return true;
            }
        }
        return false;
    }

    /* wave_queue.cc:240-256 */
    bool detect_bottom(size_t d, size_t a) {
        const size_t i = idx(d, a);
        double h;
        height(oc.bot, next->pos[0][i], next->pos[1][i], next->pos[2][i], &h, nullptr);
        const double depth = h - next->pos[0][i];
        if (depth > 0.0) {
            if (bottom_reflection(d, a, depth)) {
                next->bottom[i] += 1;
                curr->bottom[i] = prev->bottom[i] = past->bottom[i] = next->bottom[i];
                detect_volume_scattering(d, a);
                detect_surface(d, a);
                return true;
            }
        }
        return false;
    }

    /* wave_queue::detect_volume_scattering (wave_queue.cc:297-345).  The
     * collision time is measured to the ocean surface, not to the layer,
     * as in the reference. */
    void detect_volume_scattering(size_t d, size_t a) {
        if (!want_verbs) return;
        const size_t i = idx(d, a);
        if (above_bounce(curr, i)) return;
        for (size_t k = 0; k < oc.vol_rho.size(); ++k) {
            const double height = oc.vol_rho[k];
            const double d1 = height - next->pos[0][i];
            const double d2 = height - curr->pos[0][i];
            if (d1 * d2 >= 0) continue;
            double c = curr->c[i];
            const double dd = c * c * curr->nd[0][i];
            const double time_water = (dd == 0.0) ? double(0.0) : -(curr->pos[0][i] - R) / dd;
            double position[3], ndir[3];
            collision_location(d, a, time_water, position, ndir, &c);
            const double grazing =
                std::atan2(curr->nd[0][i], std::sqrt(curr->nd[1][i] * curr->nd[1][i] +
                                                     curr->nd[2][i] * curr->nd[2][i]));
            const int type = (d1 > 0) ? WQ3D_VERB_VOLUME_LOWER + 2 * (int)k : WQ3D_VERB_VOLUME_UPPER + 2 * (int)k;
            build_eigenverb(d, a, time_water, grazing, c, position, ndir, type);
        }
    }

    /* wave_queue::build_eigenverb (wave_queue.cc:1063-1164) */
    void build_eigenverb(size_t d, size_t a, double tw, double grazing, double speed,
                         const double* position, const double* ndir, int type) {
        const int32_t seq = ev_seq++;
        const size_t i = idx(d, a);
        grazing = std::abs(grazing);
        if (!want_verbs || above_bounce(curr, i) || time <= 0.0 || grazing < 1e-6 ||
            (az_boundary && a == naz - 1) || std::abs(de[d]) > 89.9)
            return;
        /* seq_vector::increment clamps, and an index of -1 wraps to the end
         * (seq_vector.h:140-143) */
        auto inc = [](const std::vector<double>& v, size_t k) { return v[std::min(v.size() - 1, k)]; };
        const double de_angle = to_radians(de[d]);
        const double de_plus = de_angle + 0.5 * to_radians(inc(de_inc, d));
        const double de_minus = de_angle - 0.5 * to_radians(inc(de_inc, d - 1));
        const double az_angle = to_radians(az[a]);
        const double az_plus = az_angle + 0.5 * to_radians(inc(az_inc, a));
        const size_t az_index = (a == 0 && az_boundary) ? naz - 1 : a;
        const double az_minus = az_angle - 0.5 * to_radians(inc(az_inc, az_index - 1));
        const double area = (std::sin(de_plus) - std::sin(de_minus)) * (az_plus - az_minus);
        const double de_delta = de_plus - de_minus;
        const double az_delta = area / de_delta;
        const double path_length = curr->plen[i] + curr->c[i] * tw;
        if (path_length <= 0) return;
        const double sin_grazing = std::sin(grazing);
        wq3d_eigenverb v{};
        v.length = 0.5 * path_length * de_delta / sin_grazing;
        v.width = 0.5 * path_length * az_delta;
        std::vector<double> power(nf);
        bool above = false;
        for (size_t k = 0; k < nf; ++k) {
            power[k] = std::pow(10.0, -0.1 * curr->atten[i * nf + k]) * area / sin_grazing;
            if (power[k] >= eigenverb_thresh) above = true;
        }
        if (!above) return;
        /* wvector1::direction (wvector1.cc:79-82) */
        v.direction = to_radians(to_degrees(std::atan2(ndir[2], -ndir[1])));
        v.travel_time = time + tw;
        v.grazing = grazing;
        v.sound_speed = speed;
        for (int k = 0; k < 3; ++k) v.position[k] = position[k];
        v.de = (int32_t)d;
        v.az = (int32_t)a;
        v.source_de = to_radians(de[d]);
        v.source_az = to_radians(az[a]);
        v.surface = curr->surface[i];
        v.bottom = curr->bottom[i];
        v.caustic = curr->caustic[i];
        v.upper = curr->upper[i];
        v.lower = curr->lower[i];
        v.interface_num = type;
        v.step = (int64_t)steps;
        v.seq = seq;
        verbs.push_back(v);
        verb_power.insert(verb_power.end(), power.begin(), power.end());
        if (cb.add_eigenverb) cb.add_eigenverb(cb_ctx, &v, abi_out(power.data()), nf, type);
    }

    /* wave_queue.cc:261-269 */
    void detect_vertices(size_t d, size_t a) {
        const size_t i = idx(d, a);
        const double L = curr->nd[0][i];
        const double Rr = next->nd[0][i];
        if (L * Rr < 0.0 && Rr < 0.0) {
            next->upper[i]++;
        } else if (L * Rr < 0.0 && 0.0 < Rr) {
            next->lower[i]++;
        }
    }

    /* wave_queue.cc:274-292 */
    void detect_caustics(size_t d, size_t a) {
        if (d < nde - 1) {
            const size_t i = idx(d, a), j = idx(d + 1, a);
            const double A = curr->pos[0][j];
            const double B = curr->pos[0][i];
            const double C = next->pos[0][j];
            const double D = next->pos[0][i];
            bool fold = false;
            if (next->surface[j] == next->surface[i] && next->bottom[j] == next->bottom[i]) fold = true;
            if ((C - D) * (A - B) < 0 && fold) {
                next->caustic[j]++;
                for (size_t k = 0; k < nf; ++k) next->phase[j * nf + k] -= M_PI_2;
            }
        }
    }

    /* wave_front::find_edges (wave_front.cc:184-216) */
    void find_edges(Front& f) {
        std::fill(f.on_edge.begin(), f.on_edge.end(), 0);
        const size_t max_de = nde - 1;
        for (size_t a = 0; a < naz; ++a) {
            f.on_edge[idx(0, a)] = 1;
            f.on_edge[idx(max_de, a)] = 1;
        }
        for (size_t a = 0; a < naz; ++a) {
            for (size_t d = 1; d < max_de; ++d) {
                const double r0 = f.pos[0][idx(d, a)];
                const double rp = f.pos[0][idx(d + 1, a)];
                const double rm = f.pos[0][idx(d - 1, a)];
                if ((r0 < rp && r0 < rm) || (r0 > rp && r0 > rm)) {
                    f.on_edge[idx(d, a)] = 1;
                    const double n0 = f.nd[0][idx(d, a)];
                    if (std::abs(n0 - f.nd[0][idx(d - 1, a)]) >
                        std::abs(n0 - f.nd[0][idx(d + 1, a)])) {
                        f.on_edge[idx(d - 1, a)] = 1;
                    } else {
                        f.on_edge[idx(d + 1, a)] = 1;
                    }
                }
            }
        }
    }

    /* wave_queue.cc:982-1057 */
    void collision_location(size_t d, size_t a, double tw, double* pos,
                            double* nd, double* speed) const {
        const size_t i = idx(d, a);
        const double time1 = 2.0 * dt;
        const double time2 = dt * dt;
        const double dtime2 = tw * tw;
        double drho = (next->c[i] - prev->c[i]) / time1;
        double d2rho = (next->c[i] + prev->c[i] - 2.0 * curr->c[i]) / time2;
        *speed = curr->c[i] + drho * tw + 0.5 * d2rho * dtime2;
        for (int k = 0; k < 3; ++k) {
            const double v1 = (next->pos[k][i] - prev->pos[k][i]) / time1;
            const double v2 = (next->pos[k][i] + prev->pos[k][i] - 2.0 * curr->pos[k][i]) / time2;
            pos[k] = curr->pos[k][i] + v1 * tw + 0.5 * v2 * dtime2;
        }
        for (int k = 0; k < 3; ++k) {
            const double v1 = (next->nd[k][i] - prev->nd[k][i]) / time1;
            const double v2 = (next->nd[k][i] + prev->nd[k][i] - 2.0 * curr->nd[k][i]) / time2;
            nd[k] = curr->nd[k][i] + v1 * tw + 0.5 * v2 * dtime2;
        }
    }

    void record_reflection(size_t d, size_t a, double tw, double grazing,
                           double c, const double* pos, const double* nd,
                           int type) {
        if (!want_refl) return;
        wq3d_reflection r{};
        r.time = time + tw;
        r.dt = tw;
        r.grazing = grazing;
        r.speed = c;
        for (int k = 0; k < 3; ++k) {
            r.position[k] = pos[k];
            r.ndirection[k] = nd[k];
        }
        r.de = (int32_t)d;
        r.az = (int32_t)a;
        r.type = type;
        r.step = steps;
        refl.push_back(r);
        if (cb.reflect) cb.reflect(cb_ctx, &r);
    }

    /* reflection_model.cc:33-182 */
    bool bottom_reflection(size_t d, size_t a, double depth) {
        const size_t i = idx(d, a);
        double N;
        bool shallow = false;
        double position[3] = {curr->pos[0][i], curr->pos[1][i], curr->pos[2][i]};
        double ndir[3] = {curr->nd[0][i], curr->nd[1][i], curr->nd[2][i]};
        double c = curr->c[i];
        double c2 = c * c;
        double bottom_rho, nrm[3];
        height(oc.bot, position[0], position[1], position[2], &bottom_rho, nrm);
        double height_water = position[0] - bottom_rho;
        const double TOO_SHALLOW = 300.0 * dt;
        if ((R - bottom_rho) < TOO_SHALLOW) shallow = true;
        if (shallow) {
            N = std::sqrt(nrm[1] * nrm[1] + nrm[2] * nrm[2]);
            nrm[0] = 0.0;
            nrm[1] = nrm[1] / N;
            nrm[2] = nrm[2] / N;
        }
        ndir[0] = c2 * ndir[0];
        ndir[1] = c2 * ndir[1];
        ndir[2] = c2 * ndir[2];
        double dot_full = nrm[0] * ndir[0] + nrm[1] * ndir[1] + nrm[2] * ndir[2];
        const double MIN_REFLECT = 6.0;
        double max_dot = -std::max(MIN_REFLECT, (height_water + depth) * nrm[0]);
        if (dot_full >= max_dot) dot_full = max_dot;
        const double dot_water = -height_water * nrm[0];
        const double time_water = std::max<double>(0.0, dot_water / dot_full);

        collision_location(d, a, time_water, position, ndir, &c);
        height(oc.bot, position[0], position[1], position[2], &bottom_rho, nrm);
        if (shallow) {
            N = std::sqrt(nrm[1] * nrm[1] + nrm[2] * nrm[2]);
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
        max_dot = -std::max(MIN_REFLECT, (height_water + depth) * nrm[0]);
        if (dot_full >= max_dot) dot_full = max_dot;

        double grazing = 0.0;
        if (dot_full / c >= 1.0) {
            grazing = -M_PI_2;
        } else if (dot_full / c <= -1.0) {
            grazing = M_PI_2;
        } else {
            grazing = std::asin(-dot_full / c);
        }
        record_reflection(d, a, time_water, grazing, c, position, ndir, 0);
        if (want_verbs) build_eigenverb(d, a, time_water, grazing, c, position, ndir, WQ3D_VERB_BOTTOM);

        std::vector<double> amp(nf), ph(nf);
        reflect_loss(oc.bot, freq, grazing, amp.data(), ph.data());
        for (size_t k = 0; k < nf; ++k) {
            next->atten[i * nf + k] += amp[k];
            next->phase[i * nf + k] += ph[k];
        }
        dot_full *= 2.0;
        ndir[0] = ndir[0] - dot_full * nrm[0];
        ndir[1] = ndir[1] - dot_full * nrm[1];
        ndir[2] = ndir[2] - dot_full * nrm[2];
        N = std::sqrt(ndir[0] * ndir[0] + ndir[1] * ndir[1] + ndir[2] * ndir[2]) * c;
        ndir[0] = ndir[0] / N;
        ndir[1] = ndir[1] / N;
        ndir[2] = ndir[2] / N;
        reflection_reinit(d, a, time_water, position, ndir);
        return true;
    }

    /* reflection_model.cc:187-243 */
    bool surface_reflection(size_t d, size_t a) {
        const size_t i = idx(d, a);
        double c = curr->c[i];
        const double dd = c * c * curr->nd[0][i];
        const double time_water = (dd == 0.0) ? double(0.0) : -(curr->pos[0][i] - R) / dd;
        double position[3], ndir[3];
        collision_location(d, a, time_water, position, ndir, &c);
        const double grazing =
            std::atan2(curr->nd[0][i], std::sqrt(curr->nd[1][i] * curr->nd[1][i] +
                                                 curr->nd[2][i] * curr->nd[2][i]));
        if (grazing <= 0.0) return false;
        record_reflection(d, a, time_water, grazing, c, position, ndir, 1);
        if (want_verbs) build_eigenverb(d, a, time_water, grazing, c, position, ndir, WQ3D_VERB_SURFACE);
        std::vector<double> amp(nf);
        reflect_loss(oc.surf, freq, grazing, amp.data(), nullptr);
        for (size_t k = 0; k < nf; ++k) {
            next->atten[i * nf + k] += amp[k];
            next->phase[i * nf + k] -= M_PI;
        }
        ndir[0] = -ndir[0];
        reflection_reinit(d, a, time_water, position, ndir);
        return true;
    }

    /* reflection_model::reflection_copy (reflection_model.cc:335-360) */
    void reflection_copy(Front* f, size_t i, const Ray& y) {
        for (int k = 0; k < 3; ++k) {
            f->pos[k][i] = y.pos[k];
            f->pg[k][i] = y.pg[k];
            f->nd[k][i] = y.nd[k];
            f->ng[k][i] = y.ng[k];
            f->sg[k][i] = y.sg[k];
        }
        f->c[i] = y.c;
        f->dist[i] = y.dist;
        f->plen[i] += 0.0; /* results.path_length of a fresh 1x1 front is 0 */
    }

    /* reflection_model.cc:248-330.  Keeps the reference's "past.update()"
     * at :315, which leaves temp's derivatives from its first update. */
    void reflection_reinit(size_t d, size_t a, double tw, const double* pos,
                           const double* nd) {
        const size_t i = idx(d, a);
        Ray past1, prev1, curr1, next1, temp;
        for (int k = 0; k < 3; ++k) {
            temp.pos[k] = pos[k];
            temp.nd[k] = nd[k];
        }
        update1(temp);
        rk1(-tw, temp, next1);
        update1(next1);
        rk2(-tw, temp, next1, past1);
        update1(past1);
        rk3(-tw, temp, next1, past1, curr1);
        update1(curr1);
        reflection_copy(curr, i, curr1);

        const double h = dt;
        rk1(-h, curr1, next1);
        update1(next1);
        rk2(-h, curr1, next1, past1);
        update1(past1);
        rk3(-h, curr1, next1, past1, prev1);
        update1(prev1);
        reflection_copy(prev, i, prev1);

        rk1(-h, prev1, next1);
        update1(next1);
        rk2(-h, prev1, next1, temp);
        update1(past1);
        rk3(-h, prev1, next1, temp, past1);
        update1(past1);
        reflection_copy(past, i, past1);

        ab3(h, past1, prev1, curr1, next1);
        update1(next1);
        reflection_copy(next, i, next1);
    }

    bool above_bounce(const Front* f, size_t i) const {
        return f->bottom[i] > th.max_bottom || f->surface[i] > th.max_surface ||
               f->caustic[i] > th.max_caustic || f->upper[i] > th.max_upper ||
               f->lower[i] > th.max_lower;
    }

    /* wave_queue.cc:351-404 */
    void detect_eigenrays() {
        if (!has_targets) return;
        ORACLE_PHASE(2);
        double cube[3][3][3];
        const size_t az_start = az_boundary ? 0 : 1;
        for (size_t t1 = 0; t1 < nt1; ++t1) {
            for (size_t t2 = 0; t2 < nt2; ++t2) {
                const size_t t = t1 * nt2 + t2;
                de_branch = false;
                const double slat = 90.0 - to_degrees(src[1]);
                const double slng = to_degrees(src[2]);
                const double tlat = 90.0 - to_degrees(tgt[1][t]);
                const double tlng = to_degrees(tgt[2][t]);
                if (std::abs(slat - tlat) < 1e-4 && std::abs(slng - tlng) < 1e-4)
                    de_branch = true;
                const double* dp = &prev->d2[t * n];
                const double* dc = &curr->d2[t * n];
                const double* dn = &next->d2[t * n];
                for (size_t d = 1; d < nde - 1; ++d) {
                    for (size_t a = az_start; a < naz - 1; ++a) {
                        const size_t i = idx(d, a);
                        if (curr->on_edge[i]) continue;
                        cube[1][1][1] = dc[i];
                        cube[2][1][1] = dn[i];
                        if (cube[2][1][1] <= cube[1][1][1]) continue;
                        cube[0][1][1] = dp[i];
                        if (cube[0][1][1] < cube[1][1][1]) continue;
                        if (is_closest_ray(t, d, a, cube)) build_eigenray(t1, t2, d, a, cube);
                    }
                }
            }
        }
    }

    /* wave_queue.cc:411-488 */
    bool is_closest_ray(size_t t, size_t de0, size_t az0, double cube[3][3][3]) {
        const double center = cube[1][1][1];
        const size_t max_az = naz - 1;
        for (size_t nd_ = 0; nd_ < 3; ++nd_) {
            for (size_t na = 0; na < 3; ++na) {
                if (nd_ == 1 && na == 1) continue;
                const size_t d = de0 + nd_ - 1;
                size_t a = az0 + na - 1;
                if (az_boundary) {
                    if (az0 + na == 0) {
                        a = naz - 2;
                    } else if (a >= max_az) {
                        a = 0;
                    }
                }
                const size_t i = idx(d, a);
                cube[0][nd_][na] = prev->d2[t * n + i];
                cube[1][nd_][na] = curr->d2[t * n + i];
                cube[2][nd_][na] = next->d2[t * n + i];
                if (a == 0 && !az_boundary) continue;
                if (a == max_az) continue;
                if (de_branch) {
                    if (curr->on_edge[i]) continue;
                } else {
                    if (nd_ != 1) {
                        if (curr->on_edge[i]) continue;
                    }
                }
                if (nd_ == 2 || na == 2) {
                    if (de_branch) {
                        if (az0 == 0) {
                            if (cube[1][nd_][na] < center) return false;
                        } else {
                            return false;
                        }
                    } else {
                        if (cube[1][nd_][na] <= center) return false;
                    }
                } else {
                    if (cube[1][nd_][na] < center) return false;
                }
                if (cube[2][nd_][na] <= center) return false;
                if (cube[0][nd_][na] < center) return false;
            }
        }
        return true;
    }

    /* wave_queue.cc:929-977 */
    static void make_taylor_coeff(const double v[3][3][3], const double* delta,
                                  double& center, double* g, double h[3][3]) {
        const double d0 = 2.0 * delta[0];
        const double d1 = 2.0 * delta[1];
        const double d2 = 2.0 * delta[2];
        center = v[1][1][1];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) h[r][c] = 0.0;
        h[0][0] = (v[2][1][1] + v[0][1][1] - 2.0 * center) / (delta[0] * delta[0]);
        h[1][1] = (v[1][2][1] + v[1][0][1] - 2.0 * center) / (delta[1] * delta[1]);
        h[2][2] = (v[1][1][2] + v[1][1][0] - 2.0 * center) / (delta[2] * delta[2]);
        g[0] = (v[2][0][1] - v[0][0][1]) / d0;
        g[2] = (v[2][2][1] - v[0][2][1]) / d0;
        h[0][1] = (g[2] - g[0]) / d1;
        h[1][0] = h[0][1];
        g[0] = (v[2][1][0] - v[0][1][0]) / d0;
        g[2] = (v[2][1][2] - v[0][1][2]) / d0;
        h[0][2] = (g[2] - g[0]) / d2;
        h[2][0] = h[0][2];
        g[0] = (v[1][2][0] - v[1][0][0]) / d1;
        g[2] = (v[1][2][2] - v[1][0][2]) / d1;
        h[1][2] = (g[2] - g[0]) / d2;
        h[2][1] = h[1][2];
        g[0] = (v[2][1][1] - v[0][1][1]) / d0;
        g[1] = (v[1][2][1] - v[1][0][1]) / d1;
        g[2] = (v[1][1][2] - v[1][1][0]) / d2;
    }

    static double dot3(const double* a, const double* b) {
        double t = 0.0;
        t += a[0] * b[0];
        t += a[1] * b[1];
        t += a[2] * b[2];
        return t;
    }
    static void matvec(const double m[3][3], const double* x, double* y) {
        for (int r = 0; r < 3; ++r) {
            double t = 0.0;
            t += m[r][0] * x[0];
            t += m[r][1] * x[1];
            t += m[r][2] * x[2];
            y[r] = t;
        }
    }
    static double norm2(const double* g) {
        double t = 0.0;
        t += std::abs(g[0]) * std::abs(g[0]);
        t += std::abs(g[1]) * std::abs(g[1]);
        t += std::abs(g[2]) * std::abs(g[2]);
        return std::sqrt(t);
    }

    size_t wrap_az(size_t az0, size_t na) const {
        size_t a = az0 + na - 1;
        if (az_boundary) {
            if (az0 + na == 0) {
                a = naz - 2;
            } else if (a >= naz - 1) {
                a = 0;
            }
        }
        return a;
    }

    /* wave_queue.cc:708-924 */
    void compute_offsets(size_t t, size_t de0, size_t az0, const double cube[3][3][3],
                         const double* delta, double* offset, double* distance) {
        bool unstable = false;
        const size_t ic = idx(de0, az0);
        const int surface = curr->surface[ic];
        const int bottom = curr->bottom[ic];
        const int caustic = curr->caustic[ic];
        for (size_t nd_ = 0; nd_ < 3 && !unstable; ++nd_) {
            const size_t d = de0 + nd_ - 1;
            for (size_t na = 0; na < 3 && !unstable; ++na) {
                const size_t a = wrap_az(az0, na);
                const size_t i = idx(d, a);
                if (prev->surface[i] != surface || curr->surface[i] != surface ||
                    next->surface[i] != surface || prev->bottom[i] != bottom ||
                    curr->bottom[i] != bottom || next->bottom[i] != bottom ||
                    prev->caustic[i] != caustic || curr->caustic[i] != caustic ||
                    next->caustic[i] != caustic || prev->on_edge[i] ||
                    prev->on_edge[i] || prev->on_edge[i]) {
                    unstable = true;
                }
            }
        }
        double center, g[3], h[3][3], inv[3][3];
        make_taylor_coeff(cube, delta, center, g, h);
        /* quirk kept: hessian(2,1)*hessian(2,0) (wave_queue.cc:762-763) */
        double determinant =
            std::max<double>(1e-6, h[0][0] * (h[1][1] * h[2][2] - h[1][2] * h[2][1]) +
                               h[0][1] * (h[1][2] * h[2][0] - h[1][0] * h[2][2]) +
                               h[0][2] * (h[1][0] * h[2][1] - h[2][1] * h[2][0]));
        unstable = unstable || determinant < norm2(g);
        for (int k = 0; k < 3; ++k) {
            const double hh = std::max<double>(1e-10, h[k][k]);
            offset[k] = -g[k] / hh;
            if (std::abs(offset[k] / delta[k]) > 0.5) {
                unstable = true;
                offset[k] = usml_copysign(0.5 * delta[k], offset[k]);
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
                for (int c = 0; c < 3; ++c) inv[r][c] /= determinant;
            const double ng[3] = {-g[0], -g[1], -g[2]};
            matvec(inv, ng, offset);
            unstable = unstable || std::abs(offset[1]) >= 0.5 * std::abs(delta[1]);
        } else {
            const double save_offset = offset[1];
            g[1] = 0.0;
            determinant = h[0][0] * h[2][2] - h[0][2] * h[2][0];
            if (determinant >= norm2(g)) {
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) inv[r][c] = 0.0;
                inv[0][0] = h[2][2];
                inv[0][2] = -h[0][2];
                inv[1][1] = 1.0;
                inv[2][0] = -h[2][0];
                inv[2][2] = h[0][0];
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) inv[r][c] /= determinant;
                const double ng[3] = {-g[0], -g[1], -g[2]};
                matvec(inv, ng, offset);
                offset[1] = save_offset;
            }
        }
        for (int k = 0; k < 3; ++k) {
            distance[k] = -g[k] * offset[k] - 0.5 * h[k][k] * offset[k] * offset[k];
            distance[k] = std::sqrt(std::max<double>(0.0, distance[k]));
            if (offset[k] < 0.0) distance[k] *= -1.0;
        }
        if (unstable) {
            distance[1] = center - distance[0] * distance[0] - distance[2] * distance[2];
            if (distance[1] <= 0.0) {
                distance[1] = 0.0;
                offset[1] = 0.0;
            } else {
                distance[1] = std::sqrt(distance[1]);
                offset[1] = std::abs(offset[1]);
                double cpa[3], nxt[3], prv[3], dir[3], speed;
                collision_location(de0, az0, offset[0], cpa, dir, &speed);
                collision_location(de0 + 1, az0, offset[0], nxt, dir, &speed);
                collision_location(de0 - 1, az0, offset[0], prv, dir, &speed);
                double nxt_dir[3], tgt_dir[3];
                nxt_dir[0] = nxt[0] - cpa[0];
                nxt_dir[1] = (nxt[1] - prv[1]) * cpa[0];
                nxt_dir[2] = (nxt[2] - prv[2]) * cpa[0] * std::sin(cpa[1]);
                if (std::abs(nxt_dir[0]) < 0.01) nxt_dir[0] = 0.0;
                tgt_dir[0] = tgt[0][t] - cpa[0];
                tgt_dir[1] = (tgt[1][t] - cpa[1]) * cpa[0];
                tgt_dir[2] = (tgt[2][t] - cpa[2]) * cpa[0] * std::sin(cpa[1]);
                const double dot = dot3(nxt_dir, tgt_dir);
                if (dot < 0.0) {
                    distance[1] *= -1.0;
                    offset[1] *= -1.0;
                }
            }
        }
    }

    /* types/wvector1.cc distance2/distance between two front points */
    static double wdist2(double r1, double t1, double p1, double r2, double t2,
                         double p2) {
        const double st = std::sin(0.5 * (t1 - t2));
        const double sp = std::sin(0.5 * (p1 - p2));
        const double dn = 1.0 - 2.0 * (st * st + std::sin(t1) * std::sin(t2) * sp * sp);
        const double dot = r1 * r2 * dn;
        return std::abs(r1 * r1 + r2 * r2 - 2.0 * dot);
    }
    double fdist(const Front* f, size_t d1, size_t a1, size_t d2, size_t a2) const {
        const size_t i = idx(d1, a1), j = idx(d2, a2);
        return std::sqrt(wdist2(f->pos[0][i], f->pos[1][i], f->pos[2][i],
                                f->pos[0][j], f->pos[1][j], f->pos[2][j]));
    }

    /* spreading_hybrid_gaussian.cc:28-59 */
    void init_hybrid() {
        norm_de.assign(nde, 0.0);
        norm_az.assign(n, 0.0);
        init_area.assign(n, 0.0);
        spread.assign(nf, 0.0);
        beam_width.assign(nf, 0.0);
        int_de.assign(nf, 0.0);
        int_az.assign(nf, 0.0);
        dup.assign(naz, 0);
        for (size_t d = 0; d < nde - 1; ++d) {
            const double de1 = to_radians(de[d]);
            const double de2 = to_radians(de[d + 1]);
            norm_de[d] = de2 - de1;
            for (size_t a = 0; a < naz - 1; ++a) {
                const double az1 = to_radians(az[a]);
                const double az2 = to_radians(az[a + 1]);
                init_area[idx(d, a)] = (std::sin(de2) - std::sin(de1)) * (az2 - az1);
                norm_az[idx(d, a)] = init_area[idx(d, a)] / norm_de[d];
            }
            norm_az[idx(d, naz - 1)] = norm_az[idx(d, naz - 2)];
        }
        norm_de[nde - 1] = norm_de[nde - 2];
        for (size_t a = 0; a < naz - 1; ++a) {
            init_area[idx(nde - 1, a)] = init_area[idx(nde - 2, a)];
            norm_az[idx(nde - 1, a)] = norm_az[idx(nde - 2, a)];
        }
        const double s = std::sqrt(TWO_PI);
        for (auto& v : norm_de) v /= s;
        for (auto& v : norm_az) v /= s;
    }

    /* spreading_ray.cc:26-45 */
    void init_classic() {
        init_area.assign(n, 0.0);
        spread.assign(nf, 0.0);
        for (size_t d = 0; d < nde - 1; ++d) {
            for (size_t a = 0; a < naz - 1; ++a) {
                const double de1 = to_radians(de[d]);
                const double de2 = to_radians(de[d + 1]);
                const double az1 = to_radians(az[a]);
                const double az2 = to_radians(az[a + 1]);
                init_area[idx(d, a)] = (std::sin(de2) - std::sin(de1)) * (az2 - az1);
            }
            init_area[idx(d, naz - 1)] = init_area[idx(d, naz - 2)];
        }
        for (size_t a = 0; a < naz - 1; ++a)
            init_area[idx(nde - 1, a)] = init_area[idx(nde - 2, a)];
        init_sound_speed = curr->c[0];
    }

    /* spreading_hybrid_gaussian.h:148-153 */
    void gaussian(double d, double w, double A, double* out) {
        for (size_t k = 0; k < nf; ++k) {
            beam_width[k] = spread[k] + 2.0 * 2.0 * w * w;
            out[k] = std::exp((-0.5 * d * d) / beam_width[k]) / std::sqrt(beam_width[k]) * A;
        }
    }
    void gadd(double d, double w, double A, std::vector<double>& acc) {
        std::vector<double> g(nf);
        gaussian(d, w, A, g.data());
        for (size_t k = 0; k < nf; ++k) acc[k] += g[k];
    }

    /* spreading_hybrid_gaussian.cc:430-495 (quirk: az_wrap + 1 at :487) */
    double width_de(size_t d, size_t a, const double* offset) {
        const double u = std::fabs(offset[0]) / dt;
        const double v = std::fabs(offset[2]) / az_inc[std::min(a, naz - 1)];
        const size_t max_az = naz - 1;
        const size_t az_wrap = (a + 1 >= max_az) ? 0 : a + 1;
        double L1 = fdist(curr, d, a, d + 1, a), L2, length1, length2;
        if (v < 1e-10) {
            length1 = L1;
        } else {
            L2 = fdist(curr, d, az_wrap, d + 1, az_wrap);
            length1 = (1.0 - v) * L1 + v * L2;
        }
        if (u < 1e-10) return 0.5 * length1;
        const Front* p2 = (offset[0] < 0.0) ? prev : next;
        L1 = fdist(p2, d, a, d + 1, a);
        if (v < 1e-10) {
            length2 = L1;
        } else {
            L2 = fdist(p2, d, az_wrap + 1, d + 1, az_wrap + 1);
            length2 = (1.0 - v) * L1 + v * L2;
        }
        return 0.5 * ((1.0 - u) * length1 + u * length2);
    }

    /* spreading_hybrid_gaussian.cc:500-571 */
    double width_az(size_t d, size_t a, const double* offset) {
        const double u = std::fabs(offset[0]) / dt;
        const double v = std::fabs(offset[1]) / de_inc[std::min(d, nde - 1)];
        const size_t max_az = naz - 1;
        const size_t max_de = nde - 1;
        const size_t de_upper = (d + 1 >= max_de) ? max_de - 2 : d;
        const size_t az_wrap = (a + 1 > max_az) ? 0 : a + 1;
        double L1 = fdist(curr, d, a, d, az_wrap), L2, length1, length2;
        if (v < 1e-10 || std::abs(v - 1.0) < 1e-10) {
            length1 = L1;
        } else {
            L2 = fdist(curr, de_upper + 1, a, de_upper + 1, az_wrap);
            length1 = (1.0 - v) * L1 + v * L2;
        }
        if (u < 1e-10) return 0.5 * length1;
        const Front* p2 = (offset[0] < 0.0) ? prev : next;
        L1 = fdist(p2, d, a, d, az_wrap);
        if (v < 1e-10 || std::abs(v - 1.0) < 1e-10) {
            length2 = L1;
        } else {
            L2 = fdist(p2, de_upper + 1, a, de_upper + 1, az_wrap);
            length2 = (1.0 - v) * L1 + v * L2;
        }
        return 0.5 * ((1.0 - u) * length1 + u * length2);
    }

    /* spreading_hybrid_gaussian.cc:124-258 */
    void intensity_de(size_t de0, size_t a, const double* offset, const double* distance) {
        const size_t ic = 0;
        (void)ic;
        int d = (int)de0;
        double cell_width = width_de(d, a, offset);
        const double initial_width = cell_width;
        const double L = distance[1];
        double cell_dist = L - cell_width;
        gaussian(cell_dist, cell_width, norm_de[d], int_de.data());
        d = (int)de0 - 1;
        cell_width = width_de(d, a, offset);
        cell_dist = L + cell_width;
        gadd(cell_dist, cell_width, norm_de[d], int_de);
        if (int_de[0] < 1e-10) return;
        for (d = (int)de0 - 2; d >= 0; --d) {
            const bool virtual_ray = curr->on_edge[idx(d + 1, a)] && curr->on_edge[idx(d, a)];
            double new_norm;
            cell_dist += cell_width;
            if (virtual_ray) {
                cell_dist += cell_width;
                new_norm = norm_de[d + 1];
            } else {
                cell_width = width_de(d, a, offset);
                cell_dist += cell_width;
                new_norm = norm_de[d];
            }
            const double old_tl = int_de[0];
            gadd(cell_dist, cell_width, new_norm, int_de);
            if (int_de[0] / old_tl < 1.002305238) break;
            if (virtual_ray) break;
        }
        cell_width = initial_width;
        cell_dist = L - cell_width;
        const int size = (int)nde - 1;
        for (d = (int)de0 + 1; d < size; ++d) {
            const bool virtual_ray = curr->on_edge[idx(d + 1, a)] && curr->on_edge[idx(d, a)];
            double new_norm;
            cell_dist -= cell_width;
            if (virtual_ray) {
                cell_dist -= cell_width;
                new_norm = norm_de[d - 1];
            } else {
                cell_width = width_de(d, a, offset);
                cell_dist -= cell_width;
                new_norm = norm_de[d];
            }
            const double old_tl = int_de[0];
            gadd(cell_dist, cell_width, new_norm, int_de);
            if (int_de[0] / old_tl < 1.002305238) break;
            if (virtual_ray) break;
        }
    }

    /* spreading_hybrid_gaussian.cc:264-425 (quirk: _norm_az(1,a) near the
     * D/E fan ends, :298-302) */
    void intensity_az(size_t d, size_t az0, const double* offset, const double* distance) {
        const size_t max_de = nde - 2;
        const size_t max_az = naz - 1;
        size_t az_upper, az_lower;
        if (az_boundary) {
            az_lower = az_upper = az0;
        } else {
            az_lower = 0;
            az_upper = max_az - 1;
        }
        std::fill(dup.begin(), dup.end(), 0);
        size_t a = az0;
        dup[a] = 1;
        double cell_width = width_az(d, a, offset);
        const double initial_width = cell_width;
        const double L = distance[2];
        double cell_dist = L - cell_width;
        double new_norm = (d >= max_de) ? norm_az[idx(1, a)] : norm_az[idx(d, a)];
        gaussian(cell_dist, cell_width, new_norm, int_az.data());
        a = (az0 < 1) ? max_az - 1 : az0 - 1;
        dup[a] = 1;
        cell_width = width_az(d, a, offset);
        cell_dist = L + cell_width;
        new_norm = (d >= max_de) ? norm_az[idx(1, a)] : norm_az[idx(d, a)];
        gadd(cell_dist, cell_width, new_norm, int_az);
        if (int_az[0] < 1e-10) return;
        if (a < 1) {
            a = max_az - 1;
        } else {
            --a;
        }
        while ((a % max_az) != az_lower) {
            if (dup[a]) break;
            dup[a] = 1;
            if (curr->on_edge[idx(d, a)]) break;
            cell_dist += cell_width;
            cell_width = width_az(d, a, offset);
            cell_dist += cell_width;
            const double old_tl = int_az[0];
            new_norm = (d >= max_de) ? norm_az[idx(1, a)] : norm_az[idx(d, a)];
            gadd(cell_dist, cell_width, new_norm, int_az);
            if (int_az[0] / old_tl < 1.002305238) break;
            if (a == 0) {
                a += max_az - 1;
            } else {
                --a;
            }
        }
        cell_width = initial_width;
        cell_dist = L - cell_width;
        a = az0 + 1;
        while ((a % max_az) != az_upper) {
            if (a == max_az) a = 0;
            if (dup[a]) break;
            dup[a] = 1;
            if (curr->on_edge[idx(d, a)]) break;
            cell_dist -= cell_width;
            cell_width = width_az(d, a, offset);
            cell_dist -= cell_width;
            const double old_tl = int_az[0];
            new_norm = (d >= max_de) ? norm_az[idx(1, a)] : norm_az[idx(d, a)];
            gadd(cell_dist, cell_width, new_norm, int_az);
            if (int_az[0] / old_tl < 1.002305238) break;
            ++a;
        }
    }

    /* spreading_hybrid_gaussian.cc:65-119 */
    void intensity_hybrid(size_t t, size_t de0, size_t az0, const double* offset,
                          const double* distance, double* out) {
        double c;
        sound_speed(oc, R, tgt[0][t], tgt[1][t], tgt[2][t], &c, nullptr);
        for (size_t k = 0; k < nf; ++k) spread[k] = TWO_PI * c / freq[k];
        for (size_t k = 0; k < nf; ++k) spread[k] = spread[k] * spread[k];
        size_t d = de0, a = az0;
        double no[3] = {offset[0], offset[1], offset[2]};
        if (offset[2] < 0.0) {
            if (az0 > 0) {
                a = az0 - 1;
            } else if (az_boundary) {
                a = naz - 2;
            }
            no[2] = offset[2] + az_inc[std::min(a, naz - 1)];
        }
        intensity_de(de0, a, no, distance);
        no[0] = offset[0];
        no[1] = offset[1];
        no[2] = offset[2];
        if (offset[1] < 0.0 && !curr->on_edge[idx(de0 - 1, az0)]) {
            d = de0 - 1;
            no[1] = offset[1] + de_inc[std::min(d, nde - 1)];
        }
        intensity_az(d, az0, no, distance);
        for (size_t k = 0; k < nf; ++k) out[k] = int_de[k] * int_az[k];
    }

    /* wvector1::area (types/wvector1.cc) on four front points */
    double area4(const Front* f, size_t d, size_t a) const {
        auto P = [&](size_t dd, size_t aa, double* p) {
            const size_t i = idx(dd, aa);
            p[0] = f->pos[0][i];
            p[1] = f->pos[1][i];
            p[2] = f->pos[2][i];
        };
        double p1[3], p2[3], p3[3], p4[3];
        P(d, a, p1);
        P(d + 1, a, p2);
        P(d + 1, a + 1, p3);
        P(d, a + 1, p4);
        auto dist = [](const double* x, const double* y) {
            return std::sqrt(wdist2(x[0], x[1], x[2], y[0], y[1], y[2]));
        };
        double aa = dist(p1, p2);
        const double b = dist(p1, p3);
        double c = dist(p2, p3);
        const double area1 = 0.25 * std::sqrt((aa + b + c) * (b + c - aa) * (c + aa - b) * (aa + b - c));
        aa = dist(p1, p4);
        c = dist(p4, p3);
        const double area2 = 0.25 * std::sqrt((aa + b + c) * (b + c - aa) * (c + aa - b) * (aa + b - c));
        return area1 + area2;
    }

    /* spreading_ray.cc:47-133 */
    void intensity_classic(size_t t, size_t de0, size_t az0, const double* offset, double* out) {
        size_t d = de0, a = az0;
        if (offset[1] < 0.0) --d;
        /* the reference decrements an unsigned index here, which leaves the
         * array when az == 0 on a wrapped fan; wrap it instead */
        if (offset[2] < 0.0) a = (a == 0) ? naz - 2 : a - 1;
        double c;
        sound_speed(oc, R, tgt[0][t], tgt[1][t], tgt[2][t], &c, nullptr);
        const double area1 = area4(curr, d, a);
        const double area2 = (offset[0] < 0.0) ? area4(prev, d, a) : area4(next, d, a);
        double u = std::fabs(offset[0]) / dt;
        const double area = (1.0 - u) * area1 + u * area2;
        const double loss = init_area[idx(d, a)] * c / (area * init_sound_speed);
        for (size_t k = 0; k < nf; ++k) out[k] = loss;
        u = std::fabs(offset[1]) / de_inc[std::min(d, nde - 1)] - 1.0;
        if (u > 4.0)
            for (size_t k = 0; k < nf; ++k) out[k] *= 0.0;
        u = std::fabs(offset[2]) / az_inc[std::min(a, naz - 1)] - 1.0;
        if (u > 4.0)
            for (size_t k = 0; k < nf; ++k) out[k] *= 0.0;
    }

    static void direction(const double* nd, double* dde, double* daz) {
        *dde = to_degrees(std::atan2(nd[0], std::sqrt(nd[1] * nd[1] + nd[2] * nd[2])));
        *daz = to_degrees(std::atan2(nd[2], -nd[1]));
    }

    /* wave_queue.cc:495-702 */
    void build_eigenray(size_t t1, size_t t2, size_t de0, size_t az0, double cube[3][3][3]) {
        ORACLE_PHASE(3);
        const size_t ic = idx(de0, az0);
        const size_t t = t1 * nt2 + t2;
        if (above_bounce(curr, ic)) return;
        double delta[3], offset[3], distance[3];
        delta[0] = dt;
        delta[1] = de_inc[std::min(de0, nde - 1)];
        delta[2] = az_inc[std::min(az0, naz - 1)];
        /* the "unstable" loop at wave_queue.cc:534-562 has no effect */
        compute_offsets(t, de0, az0, cube, delta, offset, distance);

        Eig e;
        wq3d_eigenray& r = e.rec;
        std::memset(&r, 0, sizeof(r));
        r.time = time + offset[0];
        r.source_de = de[de0] + offset[1];
        r.source_az = az[az0] + offset[2];
        r.surface = curr->surface[ic];
        r.bottom = curr->bottom[ic];
        r.caustic = curr->caustic[ic];
        r.upper = curr->upper[ic];
        r.lower = curr->lower[ic];
        r.t1 = (int32_t)t1;
        r.t2 = (int32_t)t2;
        r.de = (int32_t)de0;
        r.az = (int32_t)az0;
        r.step = steps;
        e.phase.assign(&curr->phase[ic * nf], &curr->phase[ic * nf] + nf);

        std::vector<double> si(nf);
        if (spreading == WQ3D_HYBRID_GAUSSIAN)
            intensity_hybrid(t, de0, az0, offset, distance, si.data());
        else
            intensity_classic(t, de0, az0, offset, si.data());
        for (size_t k = 0; k < nf; ++k)
            if (std::isnan(si[k])) return;
        e.inten.assign(nf, 0.0);
        for (size_t k = 0; k < nf; ++k) e.inten[k] = -10.0 * std::log10(std::max<double>(si[k], 1e-30));
        double ddt = offset[0] / dt;
        if (ddt >= 0.0) {
            for (size_t k = 0; k < nf; ++k)
                e.inten[k] = e.inten[k] + curr->atten[ic * nf + k] * (1.0 - ddt) +
                             next->atten[ic * nf + k] * ddt;
        } else {
            ddt = 1.0 + ddt;
            for (size_t k = 0; k < nf; ++k)
                e.inten[k] = e.inten[k] + prev->atten[ic * nf + k] * (1.0 - ddt) +
                             curr->atten[ic * nf + k] * ddt;
        }
        bool above = false;
        for (size_t k = 0; k < nf; ++k)
            if (e.inten[k] < th.intensity) above = true;
        if (!above) return;

        double ang[3][3][3], center, g[3], h[3][3], hv[3];
        for (int which = 0; which < 2; ++which) {
            for (size_t nd_ = 0; nd_ < 3; ++nd_) {
                for (size_t na = 0; na < 3; ++na) {
                    const size_t d = de0 + nd_ - 1;
                    const size_t a = wrap_az(az0, na);
                    const size_t i = idx(d, a);
                    const Front* fs[3] = {prev, curr, next};
                    for (int k = 0; k < 3; ++k) {
                        const double v[3] = {fs[k]->nd[0][i], fs[k]->nd[1][i], fs[k]->nd[2][i]};
                        double x, y;
                        direction(v, &x, &y);
                        ang[k][nd_][na] = (which == 0) ? x : y;
                    }
                }
            }
            make_taylor_coeff(ang, delta, center, g, h);
            matvec(h, offset, hv);
            const double val = center + dot3(g, offset) + 0.5 * dot3(offset, hv);
            if (which == 0)
                r.target_de = val;
            else
                r.target_az = val;
        }
        found.push_back(std::move(e));
    }

    void deliver() {
        if (!cb.add_eigenray) return;
        for (const Eig& e : found) {
            if (e.rec.step != steps) continue;
            cb.add_eigenray(cb_ctx, (size_t)e.rec.t1, (size_t)e.rec.t2, &e.rec,
                            abi_out(e.inten.data()), abi_out(e.phase.data()), nf, run_id);
        }
    }
};

}  // namespace

/* ------------------------------------------------------------------ */
/* C entry points (oracle_ prefix; same meaning as include/wq3d.h)     */
/* ------------------------------------------------------------------ */
extern "C" {

const char* oracle_last_error_string(void) { return g_err.c_str(); }

int oracle_queue_create(const wq3d_ocean_desc* od, const wq3d_queue_desc* qd,
                        void** out) {
    if (!od || !qd || !out) return WQ3D_ERR_INVALID;
    Queue* q = new Queue();
    const int rc = q->create(od, qd);
    if (rc != WQ3D_OK) {
        delete q;
        return rc;
    }
    *out = q;
    return WQ3D_OK;
}

int oracle_queue_destroy(void* q) {
    delete static_cast<Queue*>(q);
    return WQ3D_OK;
}

int oracle_queue_set_thresholds(void* qv, const wq3d_thresholds* t) {
    Queue* q = static_cast<Queue*>(qv);
    q->th = *t;
    q->th.intensity = std::abs(t->intensity);
    q->eigenverb_thresh = std::pow(10.0, -0.1 * std::abs(t->eigenverb));
    return WQ3D_OK;
}

int oracle_queue_set_reflections(void* qv, int on) {
    static_cast<Queue*>(qv)->want_refl = on != 0;
    return WQ3D_OK;
}

int oracle_queue_step(void* qv, size_t nsteps) {
    Queue* q = static_cast<Queue*>(qv);
    for (size_t s = 0; s < nsteps; ++s) q->step();
    return WQ3D_OK;
}

int oracle_queue_run(void* qv, double time_max, size_t* steps_done) {
    Queue* q = static_cast<Queue*>(qv);
    size_t k = 0;
    while (q->time < time_max) {
        q->step();
        ++k;
    }
    if (steps_done) *steps_done = k;
    return WQ3D_OK;
}

int oracle_queue_time(void* qv, double* t) {
    *t = static_cast<Queue*>(qv)->time;
    return WQ3D_OK;
}

int oracle_queue_source(void* qv, double* s) {
    Queue* q = static_cast<Queue*>(qv);
    for (int k = 0; k < 3; ++k) s[k] = q->src[k];
    return WQ3D_OK;
}

int oracle_queue_get_front(void* qv, int which, const wq3d_front_view* v) {
    Queue* q = static_cast<Queue*>(qv);
    const Front* f = which == WQ3D_FRONT_PAST   ? q->past
                     : which == WQ3D_FRONT_PREV ? q->prev
                     : which == WQ3D_FRONT_CURR ? q->curr
                                                : q->next;
    const size_t n = q->n, nf = q->nf;
    auto cp = [n](oracle_plain_double* dst, const std::vector<double>& src) {
        if (dst) std::memcpy(dst, src.data(), n * sizeof(double));
    };
    auto cpi = [n](int32_t* dst, const std::vector<int>& src) {
        if (dst)
            for (size_t i = 0; i < n; ++i) dst[i] = src[i];
    };
    cp(v->rho, f->pos[0]);
    cp(v->theta, f->pos[1]);
    cp(v->phi, f->pos[2]);
    for (int k = 0; k < 3; ++k) {
        cp(v->pos_grad[k], f->pg[k]);
        cp(v->ndir[k], f->nd[k]);
        cp(v->ndir_grad[k], f->ng[k]);
        cp(v->sound_grad[k], f->sg[k]);
    }
    cp(v->sound_speed, f->c);
    cp(v->distance, f->dist);
    cp(v->path_length, f->plen);
    if (v->attenuation) std::memcpy(v->attenuation, f->atten.data(), n * nf * sizeof(double));
    if (v->phase) std::memcpy(v->phase, f->phase.data(), n * nf * sizeof(double));
    cpi(v->surface, f->surface);
    cpi(v->bottom, f->bottom);
    cpi(v->caustic, f->caustic);
    cpi(v->upper, f->upper);
    cpi(v->lower, f->lower);
    if (v->on_edge) std::memcpy(v->on_edge, f->on_edge.data(), n);
    return WQ3D_OK;
}

/* all eigenrays found so far, in the order the reference notifies them */
int oracle_queue_take_eigenrays(void* qv, wq3d_eigenray* rays, double* inten,
                                double* phase, size_t capacity, size_t* count) {
    Queue* q = static_cast<Queue*>(qv);
    *count = q->found.size();
    if (!rays) return WQ3D_OK;
    if (capacity < q->found.size()) return WQ3D_ERR_OVERFLOW;
    const size_t nf = q->nf;
    for (size_t i = 0; i < q->found.size(); ++i) {
        rays[i] = q->found[i].rec;
        if (inten) std::memcpy(inten + i * nf, q->found[i].inten.data(), nf * sizeof(double));
        if (phase) std::memcpy(phase + i * nf, q->found[i].phase.data(), nf * sizeof(double));
    }
    q->found.clear();
    return WQ3D_OK;
}

int oracle_queue_set_eigenverbs(void* qv, int on) {
    static_cast<Queue*>(qv)->want_verbs = on != 0;
    return WQ3D_OK;
}

/* eigenverbs made so far, in the order the listener saw them; power holds
 * num_freq values per eigenverb */
int oracle_queue_take_eigenverbs(void* qv, wq3d_eigenverb* out, double* power, size_t capacity,
                                 size_t* count) {
    Queue* q = static_cast<Queue*>(qv);
    *count = q->verbs.size();
    if (!out) return WQ3D_OK;
    if (capacity < q->verbs.size()) return WQ3D_ERR_OVERFLOW;
    std::memcpy(out, q->verbs.data(), q->verbs.size() * sizeof(wq3d_eigenverb));
    if (power) std::memcpy(power, q->verb_power.data(), q->verb_power.size() * sizeof(double));
    q->verbs.clear();
    q->verb_power.clear();
    return WQ3D_OK;
}

int oracle_queue_take_reflections(void* qv, wq3d_reflection* out, size_t capacity,
                                  size_t* count) {
    Queue* q = static_cast<Queue*>(qv);
    *count = q->refl.size();
    if (!out) return WQ3D_OK;
    if (capacity < q->refl.size()) return WQ3D_ERR_OVERFLOW;
    std::memcpy(out, q->refl.data(), q->refl.size() * sizeof(wq3d_reflection));
    q->refl.clear();
    return WQ3D_OK;
}

int oracle_queue_set_callbacks(void* qv, const wq3d_callbacks* cb, void* ctx) {
    Queue* q = static_cast<Queue*>(qv);
    if (cb)
        q->cb = *cb;
    else
        q->cb = wq3d_callbacks{};
    q->cb_ctx = ctx;
    return WQ3D_OK;
}

/* single-point ocean evaluations, for model-level parity tests */
int oracle_sound_speed(const wq3d_ocean_desc* od, double R, size_t n,
                       const double* rho, const double* theta, const double* phi,
                       double* speed, double* grad) {
    Ocean oc;
    oc.prof = od->profile;
    if (oc.prof.kind == WQ3D_PROFILE_GRID) load_grid(oc.pgrid, od->profile.grid);
    for (size_t i = 0; i < n; ++i) {
        double g[3];
        sound_speed(oc, R, rho[i], theta[i], phi[i], &speed[i], g);
        if (grad)
            for (int k = 0; k < 3; ++k) grad[k * n + i] = g[k];
    }
    return WQ3D_OK;
}

int oracle_height(const wq3d_ocean_desc* od, int which, size_t n,
                  const double* rho, const double* theta, const double* phi,
                  double* h, double* nrm) {
    Boundary b;
    setup_boundary(b, which == 0 ? od->surface : od->bottom, od->earth_radius, which == 0);
    for (size_t i = 0; i < n; ++i) {
        double nn[3];
        height(b, rho[i], theta[i], phi[i], &h[i], nn);
        if (nrm)
            for (int k = 0; k < 3; ++k) nrm[k * n + i] = nn[k];
    }
    return WQ3D_OK;
}

/* attenuation_model::attenuation (attenuation_thorp.cc:14-36,
 * attenuation_constant.cc:14-25) at n points, point-major output */
int oracle_attenuation(const wq3d_ocean_desc* od, double R, size_t n, const double* rho,
                       const double* distance, size_t nf, const double* freq, double* atten) {
    for (size_t k = 0; k < nf; ++k) {
        double alpha = 0.0;
        if (od->profile.attenuation != WQ3D_ATTEN_CONSTANT) {
            double F2 = freq[k];
            F2 = 1e-6 * F2 * F2;
            alpha = 1e-3 * (3.3e-3 + F2 * (0.11 / (1.0 + F2) + 44.0 / (4100.0 + F2) + 3.0e-4)) /
                    (1.0 - 5.88264e-6 * 1000.0);
        }
        for (size_t i = 0; i < n; ++i) {
            atten[i * nf + k] = (od->profile.attenuation == WQ3D_ATTEN_CONSTANT)
                                    ? od->profile.attenuation_coef * distance[i] * freq[k]
                                    : distance[i] * alpha * (1.0 + 5.88264e-6 * (rho[i] - R));
        }
    }
    return WQ3D_OK;
}

int oracle_reflect_loss(const wq3d_ocean_desc* od, int which, size_t n,
                        const double* grazing, size_t nf, const double* freq,
                        double* amp, double* phase) {
    Boundary b;
    setup_boundary(b, which == 0 ? od->surface : od->bottom, od->earth_radius, which == 0);
    std::vector<double> fv(freq, freq + nf);
    for (size_t i = 0; i < n; ++i)
        reflect_loss(b, fv, grazing[i], amp + i * nf, phase ? phase + i * nf : nullptr);
    return WQ3D_OK;
}

}  // extern "C"

/* ------------------------------------------------------------------ */
/* bistatic eigenverbs                                                 */
/* ------------------------------------------------------------------ */
namespace {

double bv_to_degrees(double t) { return t * (180.0 / M_PI); }
double bv_to_radians(double t) { return t * (M_PI / 180.0); }

/* wposition1 with the reference's getters and setters (types/wposition1.h) */
struct BvPos {
    double rho, theta, phi, R0;
    double latitude() const { return 90.0 - bv_to_degrees(theta); }
    double longitude() const { return bv_to_degrees(phi); }
    double altitude() const { return rho - R0; }
    void latitude(double v) { theta = bv_to_radians(90.0 - v); }
    void longitude(double v) { phi = bv_to_radians(v); }
    void altitude(double v) { rho = v + R0; }
};

/* wposition1(location, range, bearing) (types/wposition1.cc:23-37) */
BvPos bv_move(const BvPos& location, double range, double bearing) {
    const double lat1 = bv_to_radians(location.latitude());
    const double lng1 = bv_to_radians(location.longitude());
    const double R = location.R0 + location.altitude();
    range /= R;
    const double lat2 = std::asin(std::sin(lat1) * std::cos(range) + std::cos(lat1) * std::sin(range) * std::cos(bearing));
    const double lng2 = lng1 + std::atan2(std::sin(bearing) * std::sin(range) * std::cos(lat1),
                                          std::cos(range) - std::sin(lat1) * std::sin(lat2));
    BvPos p = location;
    p.latitude(bv_to_degrees(lat2));
    p.longitude(bv_to_degrees(lng2));
    p.altitude(location.altitude());
    return p;
}

/* wposition1::gc_range (types/wposition1.cc:57-92) */
double bv_gc_range(const BvPos& self, const BvPos& location, double* bearing) {
    const double lat1 = bv_to_radians(self.latitude());
    const double lng1 = bv_to_radians(self.longitude());
    const double R = self.R0 + self.altitude();
    const double lat2 = bv_to_radians(location.latitude());
    const double lng2 = bv_to_radians(location.longitude());
    double hav1at = std::sin(0.5 * (lat1 - lat2));
    hav1at *= hav1at;
    double havlng = std::sin(0.5 * (lng1 - lng2));
    havlng *= havlng;
    const double range = 2.0 * std::asin(std::sqrt(hav1at + std::cos(lat1) * std::cos(lat2) * havlng));
    if (std::abs(range) < 1e-6 || std::abs(lat1) < 1e-10) {
        *bearing = (lat1 > 0) ? M_PI : 0.0;
    } else {
        *bearing = std::atan2(std::sin(lng1 - lng2) * std::cos(lat2),
                              std::cos(lat1) * std::sin(lat2) - std::sin(lat1) * std::cos(lat2) * std::cos(lng1 - lng2));
        *bearing = std::fmod(2.0 * M_PI - *bearing, 2.0 * M_PI);
    }
    return range * R;
}

BvPos bv_pos(const wq3d_eigenverb& v, double R0) { return BvPos{v.position[0], v.position[1], v.position[2], R0}; }

/* eigenverb_collection::find_eigenverbs (eigenverb_collection.cc:60-93):
 * the search quadrilateral A-B-C-D of a bounding eigenverb, as (latitude,
 * longitude) corners */
struct BvQuad {
    double x[4], y[4];
};

BvQuad bv_quad(const wq3d_eigenverb& bounding, double R0, double search_scale) {
    const BvPos pos = bv_pos(bounding, R0);
    const double d = bounding.direction;
    const BvPos c[4] = {bv_move(pos, search_scale * bounding.length, d),
                        bv_move(pos, search_scale * bounding.width, d + M_PI_2),
                        bv_move(pos, search_scale * bounding.length, d + M_PI),
                        bv_move(pos, search_scale * bounding.width, d + M_PI + M_PI_2)};
    BvQuad q;
    for (int k = 0; k < 4; ++k) {
        q.x[k] = c[k].latitude();
        q.y[k] = c[k].longitude();
    }
    return q;
}

/* a centre strictly inside the quadrilateral (bgi::within); the sources
 * are tested in index order */
bool bv_found(const BvQuad& q, const wq3d_eigenverb& v, double R0) {
    const BvPos p = bv_pos(v, R0);
    const double x = p.latitude(), y = p.longitude();
    int pos_n = 0, neg_n = 0;
    for (int k = 0; k < 4; ++k) {
        const int k2 = (k + 1) % 4;
        const double cr = (q.x[k2] - q.x[k]) * (y - q.y[k]) - (q.y[k2] - q.y[k]) * (x - q.x[k]);
        pos_n += cr > 0.0;
        neg_n += cr < 0.0;
    }
    return pos_n == 4 || neg_n == 4;
}

/* ocean/scattering_{constant,lambert,chapman}.h, single-point forms */
void bv_scattering(const wq3d_scattering_desc& m, const std::vector<double>& freq, double de_incident,
                   double de_scattered, std::vector<double>& amp) {
    amp.assign(freq.size(), 0.0);
    if (m.kind == WQ3D_SCATTER_CONSTANT) {
        const double a = std::pow(10.0, m.p / 10.0);
        for (auto& v : amp) v = a;
    } else if (m.kind == WQ3D_SCATTER_LAMBERT) {
        const double coeff = std::pow(10.0, m.p / 10.0);
        for (auto& v : amp) v = std::abs(coeff * std::sin(de_incident) * std::sin(de_scattered));
    } else {
        const double grazing = 0.5 * (de_incident + de_scattered) * 180.0 / M_PI;
        const double speed = m.p * 1.94384449;
        for (size_t f = 0; f < freq.size(); ++f) {
            const double beta = 158.0 * std::pow(speed * std::pow(freq[f], 1.0 / 3.0), -0.58);
            const double a = 2.6 - 42.4 * std::log10(beta) + 3.3 * beta * std::log10(grazing / 30.0 + 1e-6);
            amp[f] = std::pow(10.0, a / 10.0);
        }
    }
}

}  // namespace

extern "C" {

/* biverb_generator::run for one interface (biverb_generator.cc:50-72)
 * with biverb_collection::add_biverb (biverb_collection.cc:44-172);
 * records in (receiver, source) order, as wq3d_biverbs returns them */
int oracle_biverbs(const wq3d_eigenverb* src, const double* src_power, size_t num_src,
                   const wq3d_eigenverb* rcv, const double* rcv_power, size_t num_rcv,
                   const double* freq, size_t num_freq, const wq3d_scattering_desc* scattering,
                   double earth_radius, double search_scale, double power_threshold,
                   wq3d_biverb* out, double* out_power, size_t capacity, size_t* count) {
    const std::vector<double> fv(freq, freq + num_freq);
    std::vector<double> scatter, power(num_freq);
    size_t n = 0;
    for (size_t ri = 0; ri < num_rcv; ++ri) {
        const wq3d_eigenverb& r = rcv[ri];
        const BvQuad quad = bv_quad(r, earth_radius, search_scale);
        for (size_t si = 0; si < num_src; ++si) {
            const wq3d_eigenverb& s = src[si];
            if (!bv_found(quad, s, earth_radius)) continue;
            bv_scattering(*scattering, fv, s.grazing, r.grazing, scatter);

            double bearing;
            const double range = bv_gc_range(bv_pos(r, earth_radius), bv_pos(s, earth_radius), &bearing);
            if (range < 1e-6) bearing = 0;
            bearing -= r.direction;
            const double ys = range * std::cos(bearing);
            const double ys2 = ys * ys;
            const double xs = range * std::sin(bearing);
            const double xs2 = xs * xs;

            const double alpha = s.direction - r.direction;
            const double cos2alpha = std::cos(2.0 * alpha);
            const double sin2alpha = std::sin(2.0 * alpha);
            const double src_length2 = s.length * s.length;
            const double src_width2 = s.width * s.width;
            const double src_sum = src_length2 + src_width2;
            const double src_diff = src_length2 - src_width2;
            const double src_prod = src_length2 * src_width2;
            const double rcv_length2 = r.length * r.length;
            const double rcv_width2 = r.width * r.width;
            const double rcv_sum = rcv_length2 + rcv_width2;
            const double rcv_diff = rcv_length2 - rcv_width2;
            const double rcv_prod = rcv_length2 * rcv_width2;

            double det_sr = 0.5 * (2.0 * (src_prod + rcv_prod) + (src_sum * rcv_sum) - (src_diff * rcv_diff) * cos2alpha);
            for (size_t f = 0; f < num_freq; ++f)
                power[f] = 0.25 * 0.5 * src_power[si * num_freq + f] * rcv_power[ri * num_freq + f] * scatter[f];
            const double new_prod = src_diff * cos2alpha;
            const double kappa = -0.25 *
                                 (xs2 * (src_sum + new_prod + 2.0 * rcv_length2) +
                                  ys2 * (src_sum - new_prod + 2.0 * rcv_width2) -
                                  2.0 * std::sqrt(xs2 * ys2) * src_diff * sin2alpha) /
                                 det_sr;
            const double overlap_scale = std::exp(kappa) / std::sqrt(det_sr);
            double pmax = 0.0;
            for (size_t f = 0; f < num_freq; ++f) {
                power[f] *= overlap_scale;
                pmax = std::max(pmax, std::abs(power[f]));
            }
            det_sr = det_sr / (src_prod * rcv_prod);
            const double sigma = 0.5 *
                                 ((1.0 / src_width2 + 1.0 / src_length2) +
                                  (1.0 / src_width2 - 1.0 / src_length2) * cos2alpha + 2.0 / rcv_width2) /
                                 det_sr;
            const double factor = std::cos(r.grazing) / r.sound_speed;
            if (!(pmax >= power_threshold)) continue;
            if (out && n < capacity) {
                wq3d_biverb& v = out[n];
                v.travel_time = s.travel_time + r.travel_time;
                v.duration = 0.5 * factor * std::sqrt(sigma);
                v.source_de = s.source_de;
                v.source_az = s.source_az;
                v.receiver_de = r.source_de;
                v.receiver_az = r.source_az;
                v.de_index = r.de;
                v.az_index = r.az;
                v.source_surface = s.surface;
                v.source_bottom = s.bottom;
                v.source_caustic = s.caustic;
                v.source_upper = s.upper;
                v.source_lower = s.lower;
                v.receiver_surface = r.surface;
                v.receiver_bottom = r.bottom;
                v.receiver_caustic = r.caustic;
                v.receiver_upper = r.upper;
                v.receiver_lower = r.lower;
                v.source = (int32_t)si;
                v.receiver = (int32_t)ri;
                for (size_t f = 0; f < num_freq; ++f) out_power[n * num_freq + f] = power[f];
            }
            ++n;
        }
    }
    *count = n;
    return (out && n > capacity) ? WQ3D_ERR_OVERFLOW : WQ3D_OK;
}

}  // extern "C"
