/*
 * wq3d_kernels.cu -- FP64 WaveQ3D propagation kernels for sm_100a.
 *
 * One step of wave_queue::step() (waveq3d/wave_queue.cc:155-192) is five
 * launches (four under the inline reflection schedule):
 *   k_reflect   one thread per ray on the worklist of rays that reflect in
 *               this step: the surface/bottom reflection chain with the RK3
 *               re-initialisation (reflect_chain), on a private copy of the
 *               ray written to its shadow slot.  It only reads the fronts,
 *               so it runs on a side stream beside the previous step's
 *               k_cpa / k_eigenray.
 *   k_advance   one thread per ray: caustic hand-off (for a reflecting ray
 *               on its states before the reflection) and vertices,
 *               wave_front::find_edges (reflecting rays read from their
 *               shadow slots), the queue rotation, the AB3 step and
 *               wave_front::update of the new front, and the next step's
 *               reflection worklist; k_advance_inline runs the next step's
 *               reflection chains itself instead.
 *   k_commit    writes the reflected rays' slots and the caustic and vertex
 *               counts into the fronts, on the eigenray stream.
 *   k_cpa       closest-point-of-approach test (detect_eigenrays +
 *               is_closest_ray) over patches of neighbouring rays x tiles
 *               of targets, with distance2 recomputed from per-front terms
 *               and targets no ray of a patch can keep dropped first;
 *               k_cpa_f32 screens each pair in FP32 before the FP64
 *               comparisons.
 *   k_eigenray  one warp per CPA found: build_eigenray, compute_offsets,
 *               hybrid Gaussian or classic spreading, target angles.
 *
 * Compiled with --fmad=false: every add and multiply rounds as in the
 * reference, so the FP64 form differs from the CPU oracle only through the
 * last-place differences between CUDA's and the host's sin/cos/exp.
 *
 * The file is compiled twice.  The full build defines every kernel, with
 * the stepping kernels in namespace "gridded" (all ocean model kinds).  The
 * second build (WQ3D_WITH_GRID=0, WQ3D_KERNEL_NS=analytic,
 * WQ3D_STEP_KERNELS_ONLY=1) defines only the stepping kernels, in
 * namespace "analytic", without the gridded models.
 */
#ifndef WQ3D_KERNEL_NS
#define WQ3D_KERNEL_NS gridded
#endif
#ifndef WQ3D_STEP_KERNELS_ONLY
#define WQ3D_STEP_KERNELS_ONLY 0
#endif
#include <cuda_runtime.h>
#include <stdint.h>

#include "wq3d_engine.cuh"

namespace wq3d {

namespace {

struct RayS {
    double pos[3];
    double pg[3];
    double nd[3];
    double ng[3];
    double c;
    double sg[3];
    double dist;
};

struct Roles {
    const FrontPtrs* P;
    const FrontPtrs* V;
    const FrontPtrs* C;
    const FrontPtrs* X;
};

__device__ __forceinline__ void roles_at(const QueueDev& q, int64_t s,
                                         Roles& r) {
    r.P = &q.F[ring_slot(s + 4)];
    r.V = &q.F[ring_slot(s + 1)];
    r.C = &q.F[ring_slot(s + 2)];
    r.X = &q.F[ring_slot(s + 3)];
}

__device__ __forceinline__ void set_err(const QueueDev& q, uint32_t bit) {
    atomicOr(q.err, bit);
}

/* profile evaluation for one point (profile_model::sound_speed) */
__device__ __forceinline__ void profile_at(const QueueDev& q, const double* pos,
                                           double* c, double* sg) {
    sound_speed(q.oc.prof, q.R, pos[0], pos[1], pos[2], c, sg);
}

/* wave_front::update on a 1x1 front without targets */
__device__ __forceinline__ void update1(const QueueDev& q, RayS& y) {
    profile_at(q, y.pos, &y.c, y.sg);
    double st;
    ray_derivs(y.c, y.sg[0], y.sg[1], y.sg[2], y.pos, y.nd, y.pg, y.ng, &st);
}

/* wave_front::update of the FP32 propagation form (no distance terms) */
__device__ __forceinline__ void update1_f32(const QueueDev& q, RayS& y) {
    float c, g[3];
    sound_speed_f32(q.oc.prof, q.R, y.pos[0], y.pos[1], y.pos[2], &c, g);
    y.c = (double)c;
    y.sg[0] = (double)g[0];
    y.sg[1] = (double)g[1];
    y.sg[2] = (double)g[2];
    ray_derivs_f32(c, g, y.pos, y.nd, y.pg, y.ng);
}

/* ode_integ.cc:20-126 */
__device__ __forceinline__ void rk1(double h, const RayS& y0, RayS& y1) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        y1.pos[k] = y0.pos[k] + 0.5 * h * y0.pg[k];
        y1.nd[k] = y0.nd[k] + 0.5 * h * y0.ng[k];
    }
}
__device__ __forceinline__ void rk2(double h, const RayS& y0, const RayS& y1,
                                    RayS& y2) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        y2.pos[k] = y0.pos[k] + h * (2.0 * y1.pg[k] - y0.pg[k]);
        y2.nd[k] = y0.nd[k] + h * (2.0 * y1.ng[k] - y0.ng[k]);
    }
}
__device__ __forceinline__ void rk3(double h, const RayS& y0, const RayS& y1,
                                    const RayS& y2, RayS& y3) {
    double p[3], d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        p[k] = y0.pos[k] + h / 6.0 * (y0.pg[k] + 4.0 * y1.pg[k] + y2.pg[k]);
        d[k] = y0.nd[k] + h / 6.0 * (y0.ng[k] + 4.0 * y1.ng[k] + y2.ng[k]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        y3.pos[k] = p[k];
        y3.nd[k] = d[k];
    }
}
/* ode_integ.cc:131-186, including the step distance of ab3_pos */
__device__ __forceinline__ void ab3(double h, const RayS& y0, const RayS& y1,
                                    const RayS& y2, RayS& y3) {
    const double A2 = 23.0 / 12.0, A1 = 16.0 / 12.0, A0 = 5.0 / 12.0;
    double d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        d[k] = h * (A2 * y2.pg[k] - A1 * y1.pg[k] + A0 * y0.pg[k]);
    const double b = y2.pos[0] * d[1];
    const double cc = y2.pos[0] * (sin(y2.pos[1]) * d[2]);
    y3.dist = sqrt(d[0] * d[0] + b * b + cc * cc);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        y3.pos[k] = y2.pos[k] + d[k];
        y3.nd[k] = y2.nd[k] + h * (A2 * y2.ng[k] - A1 * y1.ng[k] + A0 * y0.ng[k]);
    }
}

#if !WQ3D_STEP_KERNELS_ONLY
/* one ray's state (k_volume) */
__device__ __forceinline__ void load_ray(const FrontPtrs& f, int r, RayS& y) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        y.pos[k] = f.pos[k][r];
        y.pg[k] = f.pg[k][r];
        y.nd[k] = f.nd[k][r];
        y.ng[k] = f.ng[k][r];
        y.sg[k] = f.sg[k][r];
    }
    y.c = f.c[r];
    y.dist = f.dist[r];
}
#endif

/* load_ray through the read-only data cache, for kernels that never write
 * the arrays they read this way: the loads may then all be in flight at
 * once instead of waiting behind stores to the caller's copy */
__device__ __forceinline__ void load_ray_ro(const FrontPtrs& f, int r, RayS& y) {
    double v[17];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v[k] = __ldg(f.pos[k] + r);
        v[3 + k] = __ldg(f.pg[k] + r);
        v[6 + k] = __ldg(f.nd[k] + r);
        v[9 + k] = __ldg(f.ng[k] + r);
        v[12 + k] = __ldg(f.sg[k] + r);
    }
    v[15] = __ldg(f.c + r);
    v[16] = __ldg(f.dist + r);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        y.pos[k] = v[k];
        y.pg[k] = v[3 + k];
        y.nd[k] = v[6 + k];
        y.ng[k] = v[9 + k];
        y.sg[k] = v[12 + k];
    }
    y.c = v[15];
    y.dist = v[16];
}

/* reflection_model::reflection_copy (reflection_model.cc:335-360); the
 * copied path_length of a fresh 1x1 front is zero, so it is left alone */
__device__ __forceinline__ void copy_ray(const FrontPtrs& f, int r, const RayS& y) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        f.pos[k][r] = y.pos[k];
        f.pg[k][r] = y.pg[k];
        f.nd[k][r] = y.nd[k];
        f.ng[k][r] = y.ng[k];
        f.sg[k][r] = y.sg[k];
    }
    f.c[r] = y.c;
    f.dist[r] = y.dist;
}

/* wave_front::update of the main front for one ray: profile, attenuation
 * (attenuation_thorp.cc:14-36 / attenuation_constant.cc:14-25), cleared
 * phase, derivatives and the distance2 terms */
__device__ __forceinline__ void update_main(const QueueDev& q, const FrontPtrs& f,
                                            int r, RayS& y, bool accumulate,
                                            const FrontPtrs* src) {
    profile_at(q, y.pos, &y.c, y.sg);
    double st;
    ray_derivs(y.c, y.sg[0], y.sg[1], y.sg[2], y.pos, y.nd, y.pg, y.ng, &st);
    copy_ray(f, r, y);
    f.cpa[0][r] = y.pos[0];
    f.cpa[1][r] = y.pos[1];
    f.cpa[2][r] = y.pos[2];
    f.cpa[3][r] = st;
    const double alt = y.pos[0] - q.R;
    for (int k = 0; k < q.nf; ++k) {
        double a;
        if (q.oc.prof.atten == WQ3D_ATTEN_CONSTANT) {
            a = q.oc.prof.atten_coef * y.dist * q.freq[k];
        } else {
            a = y.dist * q.alpha[k] * (1.0 + 5.88264e-6 * alt);
        }
        double p = 0.0;
        if (accumulate) {
            a += src->atten[(size_t)k * q.n + r];
            p += src->phase[(size_t)k * q.n + r];
        }
        f.atten[(size_t)k * q.n + r] = a;
        f.phase[(size_t)k * q.n + r] = p;
    }
}

#if !WQ3D_STEP_KERNELS_ONLY
/* wave_queue::collision_location (wave_queue.cc:982-1057) */
__device__ void collision_location(const QueueDev& q, const FrontPtrs& V,
                                   const FrontPtrs& C, const FrontPtrs& X, int i,
                                   double tw, double* pos, double* nd,
                                   double* speed) {
    const double dt = q.dt;
    const double time1 = 2.0 * dt;
    const double time2 = dt * dt;
    const double dtime2 = tw * tw;
    const double drho = (X.c[i] - V.c[i]) / time1;
    const double d2rho = (X.c[i] + V.c[i] - 2.0 * C.c[i]) / time2;
    *speed = C.c[i] + drho * tw + 0.5 * d2rho * dtime2;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double v1 = (X.pos[k][i] - V.pos[k][i]) / time1;
        const double v2 = (X.pos[k][i] + V.pos[k][i] - 2.0 * C.pos[k][i]) / time2;
        pos[k] = C.pos[k][i] + v1 * tw + 0.5 * v2 * dtime2;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double v1 = (X.nd[k][i] - V.nd[k][i]) / time1;
        const double v2 = (X.nd[k][i] + V.nd[k][i] - 2.0 * C.nd[k][i]) / time2;
        nd[k] = C.nd[k][i] + v1 * tw + 0.5 * v2 * dtime2;
    }
}
#endif

/* One reflecting ray's prev/curr/next state and next-front losses, held
 * privately while k_reflect works on it.  The results go to a shadow slot
 * that k_advance commits, so k_cpa / k_eigenray of the previous step can
 * read the fronts at the same time.  (The reference also rewrites the
 * ray's "past" entry, reflection_model.cc:320, but the AB3 step of the
 * same wave_queue::step overwrites that entry before anything reads it.) */
struct RayLocal {
    RayS v, c, x;
    double att[MAX_FREQ];
    double ph[MAX_FREQ];
    double phf[MAX_FREQ];  /* the phases had the caustic hand-off shifted them first */
    int surface, bottom, caustic;
};

/* collision_location (wave_queue.cc:982-1057) from one ray's prev, curr
 * and next states */
__device__ void collision_rays(const QueueDev& q, const RayS& V, const RayS& Cr, const RayS& X,
                               double tw, double* pos, double* nd, double* speed) {
    const double dt = q.dt;
    const double time1 = 2.0 * dt;
    const double time2 = dt * dt;
    const double dtime2 = tw * tw;
    const double drho = (X.c - V.c) / time1;
    const double d2rho = (X.c + V.c - 2.0 * Cr.c) / time2;
    *speed = Cr.c + drho * tw + 0.5 * d2rho * dtime2;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double v1 = (X.pos[k] - V.pos[k]) / time1;
        const double v2 = (X.pos[k] + V.pos[k] - 2.0 * Cr.pos[k]) / time2;
        pos[k] = Cr.pos[k] + v1 * tw + 0.5 * v2 * dtime2;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double v1 = (X.nd[k] - V.nd[k]) / time1;
        const double v2 = (X.nd[k] + V.nd[k] - 2.0 * Cr.nd[k]) / time2;
        nd[k] = Cr.nd[k] + v1 * tw + 0.5 * v2 * dtime2;
    }
}

/* collision_location on the private state */
__device__ __forceinline__ void collision_local(const QueueDev& q, const RayLocal& L, double tw,
                                                double* pos, double* nd, double* speed) {
    collision_rays(q, L.v, L.c, L.x, tw, pos, nd, speed);
}

/* seq_vector::increment: the index clamps to the last element, and -1
 * (an unsigned index in the reference) clamps there too */
__device__ __forceinline__ double seq_inc(const double* inc, int n, int k) {
    return inc[(k < 0 || k > n - 1) ? n - 1 : k];
}

/* wave_queue::build_eigenverb (wave_queue.cc:1063-1164) for ray i.  C is
 * the stored "curr" front: its path length, attenuation and caustic /
 * upper / lower counts are not changed by reflections.  curr_c is curr's
 * sound speed (re-initialised by an earlier reflection of this step) and
 * surface / bottom the counts at this point of the reflection chain. */
__device__ __noinline__ void build_eigenverb(const QueueDev& q, const FrontPtrs& C, int i, int64_t step,
                                double t_old, double tw, double grazing, double speed,
                                const double* pos, const double* nd, int type, double curr_c,
                                int surface, int bottom, int seq) {
    grazing = fabs(grazing);
    const int d = i / q.naz, a = i % q.naz;
    if (bottom > q.max_bottom || surface > q.max_surface || C.caustic[i] > q.max_caustic ||
        C.upper[i] > q.max_upper || C.lower[i] > q.max_lower)
        return;
    if (t_old <= 0.0 || grazing < 1e-6 || (q.az_boundary && a == q.naz - 1) || fabs(q.de[d]) > 89.9)
        return;
    /* footprint of the ray's share of the fan, half-way to its neighbours */
    const double de_angle = deg2rad(q.de[d]);
    const double de_plus = de_angle + 0.5 * deg2rad(seq_inc(q.de_inc, q.nde, d));
    const double de_minus = de_angle - 0.5 * deg2rad(seq_inc(q.de_inc, q.nde, d - 1));
    const double az_angle = deg2rad(q.az[a]);
    const double az_plus = az_angle + 0.5 * deg2rad(seq_inc(q.az_inc, q.naz, a));
    const int az_index = (a == 0 && q.az_boundary) ? q.naz - 1 : a;
    const double az_minus = az_angle - 0.5 * deg2rad(seq_inc(q.az_inc, q.naz, az_index - 1));
    const double area = (sin(de_plus) - sin(de_minus)) * (az_plus - az_minus);
    const double de_delta = de_plus - de_minus;
    const double az_delta = area / de_delta;
    const double path_length = C.plen[i] + curr_c * tw;
    if (path_length <= 0) return;
    const double sin_grazing = sin(grazing);
    bool above = false;
    for (int f = 0; f < q.nf && !above; ++f)
        above = pow(10.0, -0.1 * C.atten[(size_t)f * q.n + i]) * area / sin_grazing >= q.verb_threshold;
    if (!above) return;
    const uint32_t slot = atomicAdd(q.n_verb, 1u);
    if (slot >= q.cap_verb) {
        set_err(q, ERR_VERB_OVERFLOW);
        return;
    }
    wq3d_eigenverb v;
    v.travel_time = t_old + tw;
    v.length = 0.5 * path_length * de_delta / sin_grazing;
    v.width = 0.5 * path_length * az_delta;
    for (int k = 0; k < 3; ++k) v.position[k] = pos[k];
    /* wvector1::direction (wvector1.cc:79-82), degrees and back */
    v.direction = deg2rad(rad2deg(atan2(nd[2], -nd[1])));
    v.grazing = grazing;
    v.sound_speed = speed;
    v.source_de = deg2rad(q.de[d]);
    v.source_az = deg2rad(q.az[a]);
    v.de = d;
    v.az = a;
    v.surface = surface;
    v.bottom = bottom;
    v.caustic = C.caustic[i];
    v.upper = C.upper[i];
    v.lower = C.lower[i];
    v.interface_num = type;
    v.step = step;
    v.seq = seq;
    v.pad = 0;
    q.verb[slot] = v;
    for (int f = 0; f < q.nf; ++f)
        q.verb_power[(size_t)slot * q.nf + f] =
            pow(10.0, -0.1 * C.atten[(size_t)f * q.n + i]) * area / sin_grazing;
}

/* wave_queue::detect_volume_scattering (wave_queue.cc:297-345) with the
 * ray's prev / curr / next states V, Cr, X.  The collision time is
 * measured to the ocean surface, not to the layer, as in the reference. */
__device__ __noinline__ void volume_scatter(const QueueDev& q, const FrontPtrs& C, int i, int64_t step,
                               double t_old, const RayS& V, const RayS& Cr, const RayS& X,
                               int surface, int bottom, int& seq) {
    if (bottom > q.max_bottom || surface > q.max_surface || C.caustic[i] > q.max_caustic ||
        C.upper[i] > q.max_upper || C.lower[i] > q.max_lower)
        return;
    for (int k = 0; k < q.oc.nvol; ++k) {
        const double height = q.oc.vol_rho[k];
        const double d1 = height - X.pos[0];
        const double d2 = height - Cr.pos[0];
        if (d1 * d2 >= 0) continue;
        double c = Cr.c;
        const double dd = c * c * Cr.nd[0];
        const double tw = (dd == 0.0) ? 0.0 : -(Cr.pos[0] - q.R) / dd;
        double pos[3], nd[3];
        collision_rays(q, V, Cr, X, tw, pos, nd, &c);
        const double grazing = atan2(Cr.nd[0], sqrt(Cr.nd[1] * Cr.nd[1] + Cr.nd[2] * Cr.nd[2]));
        const int type = (d1 > 0) ? WQ3D_VERB_VOLUME_LOWER + 2 * k : WQ3D_VERB_VOLUME_UPPER + 2 * k;
        build_eigenverb(q, C, i, step, t_old, tw, grazing, c, pos, nd, type, Cr.c, surface, bottom, seq++);
    }
}

/* The updates of the re-initialisation, out of line: inlined, they keep
 * the temporary rays in registers, but the larger code made k_reflect
 * wait on instruction fetch (90.6 instead of 58.4 us per launch on the
 * sloped workload, ncu: "no instruction" stalls 2.9 -> 10.1 per issue). */
__device__ __noinline__ void reinit_update(const QueueDev& q, RayS& y) {
    if (q.precision == WQ3D_FP32)
        update1_f32(q, y);
    else
        update1(q, y);
}

/* reflection_model::reflection_reinit on the private state */
__device__ __noinline__ void reinit_local(const QueueDev& q, RayLocal& L, double tw, const double* pos,
                             const double* nd) {
    RayS past1, prev1, curr1, next1, temp;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        temp.pos[k] = pos[k];
        temp.nd[k] = nd[k];
    }
    next1.dist = 0.0;
    past1.dist = 0.0;
    prev1.dist = 0.0;
    curr1.dist = 0.0;
    temp.dist = 0.0;
    reinit_update(q, temp);
    rk1(-tw, temp, next1);
    reinit_update(q, next1);
    rk2(-tw, temp, next1, past1);
    reinit_update(q, past1);
    rk3(-tw, temp, next1, past1, curr1);
    reinit_update(q, curr1);

    const double h = q.dt;
    rk1(-h, curr1, next1);
    reinit_update(q, next1);
    rk2(-h, curr1, next1, past1);
    reinit_update(q, past1);
    rk3(-h, curr1, next1, past1, prev1);
    reinit_update(q, prev1);

    rk1(-h, prev1, next1);
    reinit_update(q, next1);
    rk2(-h, prev1, next1, temp);
    rk3(-h, prev1, next1, temp, past1);
    reinit_update(q, past1);

    ab3(h, past1, prev1, curr1, next1);
    reinit_update(q, next1);
    L.c = curr1;
    L.v = prev1;
    L.x = next1;
}

__device__ void record_reflection(const QueueDev& q, int64_t step, double t_old,
                                  int i, double tw, double grazing, double c,
                                  const double* pos, const double* nd, int type,
                                  int seq) {
    if (!q.want_refl) return;
    const uint32_t slot = atomicAdd(q.n_refl, 1u);
    if (slot >= q.cap_refl) {
        set_err(q, ERR_REFL_OVERFLOW);
        return;
    }
    wq3d_reflection r;
    r.time = t_old + tw;
    r.dt = tw;
    r.grazing = grazing;
    r.speed = c;
    for (int k = 0; k < 3; ++k) {
        r.position[k] = pos[k];
        r.ndirection[k] = nd[k];
    }
    r.de = i / q.naz;
    r.az = i % q.naz;
    r.type = type;
    r.pad = seq;
    r.step = step;
    q.refl[slot] = r;
}

/* reflection_model::surface_reflection (reflection_model.cc:187-243) */
__device__ __noinline__ bool surface_local(const QueueDev& q, const FrontPtrs& C, RayLocal& L, int i, int64_t step,
                              double t_old, int& seq) {
    double c = L.c.c;
    const double d = c * c * L.c.nd[0];
    const double tw = (d == 0.0) ? 0.0 : -(L.c.pos[0] - q.R) / d;
    double pos[3], nd[3];
    collision_local(q, L, tw, pos, nd, &c);
    const double n1 = L.c.nd[1], n2 = L.c.nd[2];
    const double grazing = atan2(L.c.nd[0], sqrt(n1 * n1 + n2 * n2));
    if (grazing <= 0.0) return false;
    record_reflection(q, step, t_old, i, tw, grazing, c, pos, nd, 1, seq);
    if (q.want_verbs)
        build_eigenverb(q, C, i, step, t_old, tw, grazing, c, pos, nd, WQ3D_VERB_SURFACE, L.c.c, L.surface,
                        L.bottom, seq);
    ++seq;
    const LossDev& Lo = q.oc.surf.loss;
    double amp0 = 0.0, ph0 = 0.0;
    if (Lo.kind != WQ3D_LOSS_ECKART) reflect_loss_scalar(Lo, grazing, &amp0, &ph0);
    const double w2 = Lo.p[0] * Lo.p[0];
    const double sg = sin(grazing);
    for (int k = 0; k < q.nf; ++k) {
        double a = amp0;
        if (Lo.kind == WQ3D_LOSS_ECKART) {
            const double x = q.freq[k] * w2 * sg;
            a = 8.6e-9 * (x * x);
        }
        L.att[k] += a;
        L.ph[k] -= M_PI;
        L.phf[k] -= M_PI;
    }
    nd[0] = -nd[0];
    reinit_local(q, L, tw, pos, nd);
    return true;
}

/* reflection_model::bottom_reflection (reflection_model.cc:33-182) */
__device__ __noinline__ void bottom_local(const QueueDev& q, const FrontPtrs& C, RayLocal& L, int i, double depth,
                             int64_t step, double t_old, int& seq, double* dl) {
    const BoundaryDev& B = q.oc.bot;
    bool shallow = false;
    double position[3] = {L.c.pos[0], L.c.pos[1], L.c.pos[2]};
    double ndir[3] = {L.c.nd[0], L.c.nd[1], L.c.nd[2]};
    double c = L.c.c;
    double c2 = c * c;
    double nrm[3];
    double bottom_rho = boundary_height_normal(B, position[1], position[2], nrm);
    double height_water = position[0] - bottom_rho;
    const double TOO_SHALLOW = 300.0 * q.dt;
    if ((q.R - bottom_rho) < TOO_SHALLOW) shallow = true;
    double N;
    if (shallow) {
        N = sqrt(nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        nrm[0] = 0.0;
        nrm[1] = nrm[1] / N;
        nrm[2] = nrm[2] / N;
    }
    ndir[0] = c2 * ndir[0];
    ndir[1] = c2 * ndir[1];
    ndir[2] = c2 * ndir[2];
    double dot_full = nrm[0] * ndir[0] + nrm[1] * ndir[1] + nrm[2] * ndir[2];
    const double MIN_REFLECT = 6.0;
    double max_dot = -fmax(MIN_REFLECT, (height_water + depth) * nrm[0]);
    if (dot_full >= max_dot) dot_full = max_dot;
    const double dot_water = -height_water * nrm[0];
    const double time_water = fmax(0.0, dot_water / dot_full);

    collision_local(q, L, time_water, position, ndir, &c);
    bottom_rho = boundary_height_normal(B, position[1], position[2], nrm);
    if (shallow) {
        N = sqrt(nrm[1] * nrm[1] + nrm[2] * nrm[2]);
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
    max_dot = -fmax(MIN_REFLECT, (height_water + depth) * nrm[0]);
    if (dot_full >= max_dot) dot_full = max_dot;

    double grazing;
    if (dot_full / c >= 1.0) {
        grazing = -M_PI_2;
    } else if (dot_full / c <= -1.0) {
        grazing = M_PI_2;
    } else {
        grazing = asin(-dot_full / c);
    }
    record_reflection(q, step, t_old, i, time_water, grazing, c, position, ndir, 0, seq);
    if (q.want_verbs)
        build_eigenverb(q, C, i, step, t_old, time_water, grazing, c, position, ndir, WQ3D_VERB_BOTTOM, L.c.c,
                        L.surface, L.bottom, seq);
    ++seq;

    const LossDev& Lo = B.loss;
    double amp0 = 0.0, ph0 = 0.0;
    if (Lo.kind != WQ3D_LOSS_ECKART) reflect_loss_scalar(Lo, grazing, &amp0, &ph0);
    if (q.sens) {
        double g[3];
        reflect_loss_rayleigh_grad(Lo, grazing, g);
        for (int j = 0; j < 3; ++j) dl[j] += g[j];
    }
    const double w2 = Lo.p[0] * Lo.p[0];
    const double sgz = sin(grazing);
    for (int k = 0; k < q.nf; ++k) {
        double a = amp0, p = ph0;
        if (Lo.kind == WQ3D_LOSS_ECKART) {
            const double x = q.freq[k] * w2 * sgz;
            a = 8.6e-9 * (x * x);
            p = M_PI;
        }
        L.att[k] += a;
        L.ph[k] += p;
        L.phf[k] += p;
    }
    dot_full *= 2.0;
    ndir[0] = ndir[0] - dot_full * nrm[0];
    ndir[1] = ndir[1] - dot_full * nrm[1];
    ndir[2] = ndir[2] - dot_full * nrm[2];
    N = sqrt(ndir[0] * ndir[0] + ndir[1] * ndir[1] + ndir[2] * ndir[2]) * c;
    ndir[0] = ndir[0] / N;
    ndir[1] = ndir[1] / N;
    ndir[2] = ndir[2] / N;
    reinit_local(q, L, time_water, position, ndir);
}

/* whether the "next" ray reflects at the start of the following step:
 * 1 = surface if above the surface and heading up (surface_reflection's
 * grazing > 0), else 2 = bottom if below the bottom (wave_queue.cc:222-256) */
__device__ __forceinline__ uint8_t reflect_decision(const QueueDev& q,
                                                    const double* xpos,
                                                    const double* cnd) {
    if (xpos[0] - q.R > 0.0) {
        const double grazing = atan2(cnd[0], sqrt(cnd[1] * cnd[1] + cnd[2] * cnd[2]));
        if (grazing > 0.0) return 1;
    }
    const double h = boundary_height(q.oc.bot, xpos[1], xpos[2]);
    return (h - xpos[0] > 0.0) ? 2 : 0;
}

/* appends a reflecting ray to worklist p: surface reflections fill it
 * from the front, bottom reflections from the back, so the warps of
 * k_reflect mostly take one path */
__device__ __forceinline__ void work_append(const QueueDev& q, int p, uint8_t kind, int i) {
    if (kind == 1) {
        const uint32_t slot = atomicAdd(q.n_work[p], 1u);
        if (slot < (uint32_t)q.n) q.work[p][slot] = (uint32_t)i;
    } else {
        const uint32_t slot = atomicAdd(q.n_work_b[p], 1u);
        if (slot < (uint32_t)q.n) q.work[p][q.n - 1 - slot] = (uint32_t)i;
    }
}

/* shadow slot of a reflecting ray: prev, curr, next (17 doubles each), the
 * next front's attenuation and phase (nf each), and the three loss
 * tangents its bottom bounces add; counts in shadow_cnt */
/* a shadow slot: prev, curr and next states (17 doubles each), the next
 * front's attenuation and phase (nf each), the three loss tangents of the
 * step's bottom bounces, and the phases again as they are when the caustic
 * hand-off of the neighbour below shifted them by -pi/2 before the
 * reflection (nf) */
__device__ __forceinline__ size_t shadow_stride(const QueueDev& q) { return 54 + 3 * (size_t)q.nf; }

__device__ __forceinline__ void ray_to(double* dst, const RayS& y) {
    for (int k = 0; k < 3; ++k) {
        dst[k] = y.pos[k];
        dst[3 + k] = y.pg[k];
        dst[6 + k] = y.nd[k];
        dst[9 + k] = y.ng[k];
        dst[13 + k] = y.sg[k];
    }
    dst[12] = y.c;
    dst[16] = y.dist;
}

__device__ __forceinline__ void ray_from(const double* src, RayS& y) {
    for (int k = 0; k < 3; ++k) {
        y.pos[k] = src[k];
        y.pg[k] = src[3 + k];
        y.nd[k] = src[6 + k];
        y.ng[k] = src[9 + k];
        y.sg[k] = src[13 + k];
    }
    y.c = src[12];
    y.dist = src[16];
}

/* A ray that reflected at step s-1 keeps its post-reflection states in
 * that step's shadow slot until k_commit of step s-1, which runs on its
 * own stream behind the eigenray construction of step s-2, has written
 * them into the fronts.  At step s those are its prev state (the slot's
 * curr, at +17) and its curr state (the slot's next, at +34), with the
 * slot's counts.  Returns the slot, or null when the ray did not reflect
 * at step s-1 and the fronts hold its states. */
__device__ __forceinline__ const double* prev_step_slot(const QueueDev& q, int64_t s, int i,
                                                        const int32_t** cnt = nullptr) {
    const int p = shadow_set(s + SHADOW_SETS - 1); /* the set of step s-1 */
    if (!(__ldg(q.commit_flag[p] + i) & COMMIT_REFLECT)) return nullptr;
    const int32_t w = __ldg(q.shadow_slot[p] + i);
    WQ_CHECKED_OR(q, w >= 0 && w < q.n, return nullptr);
    if (cnt) *cnt = q.shadow_cnt[p] + 3 * (size_t)w;
    return q.shadow[p] + (size_t)w * shadow_stride(q);
}

/* the prev and curr states of ray i at step s (fronts V and C, or the
 * previous step's shadow slot) */
__device__ __forceinline__ void load_prev_curr(const QueueDev& q, int64_t s, const Roles& R, int i,
                                               RayS& v, RayS& c) {
    const double* sp = prev_step_slot(q, s, i);
    if (sp) {
        ray_from(sp + 17, v);
        ray_from(sp + 34, c);
    } else {
        load_ray_ro(*R.V, i, v);
        load_ray_ro(*R.C, i, c);
    }
}

/* rho of ray j on the curr front at step s */
__device__ __forceinline__ double curr_rho(const QueueDev& q, int64_t s, const Roles& R, int j) {
    const double* sp = prev_step_slot(q, s, j);
    return sp ? __ldg(sp + 34) : __ldg(R.C->pos[0] + j);
}

}  // namespace

namespace WQ3D_KERNEL_NS {

/* ------------------------------------------------------------------ */
/* start-up: wave_queue ctor (wave_queue.cc:83-85) for one ray         */
/* ------------------------------------------------------------------ */
__global__ void __launch_bounds__(128) k_startup(__grid_constant__ const QueueDev q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= q.n) return;
    const int d = i / q.naz, a = i % q.naz;
    const FrontPtrs& past = q.F[0];
    const FrontPtrs& prev = q.F[1];
    const FrontPtrs& curr = q.F[2];
    const FrontPtrs& next = q.F[3];
    /* wave_front::init_wave (wave_front.cc:84-121) */
    RayS c0;
    c0.nd[0] = q.sin_de[d] / q.c_source;
    c0.nd[1] = (-q.cos_de[d] * q.cos_az[a]) / q.c_source;
    c0.nd[2] = (q.cos_de[d] * q.sin_az[a]) / q.c_source;
    c0.pos[0] = q.source[0];
    c0.pos[1] = q.source[1];
    c0.pos[2] = q.source[2];
    c0.dist = 0.0;
    update_main(q, curr, i, c0, false, nullptr);
    /* init_wavefronts (wave_queue.cc:114-150); intermediate updates of the
     * reference's _next land in registers, only final values are stored */
    const double h = -q.dt;
    RayS n1, p1, v1;
    n1.dist = 0.0;
    p1.dist = 0.0;
    v1.dist = 0.0;
    rk1(h, c0, n1);
    update1(q, n1);
    rk2(h, c0, n1, p1);
    update1(q, p1);
    rk3(h, c0, n1, p1, v1);
    update_main(q, prev, i, v1, false, nullptr);
    rk1(h, v1, n1);
    update1(q, n1);
    rk2(h, v1, n1, p1);
    update1(q, p1);
    rk3(h, v1, n1, p1, p1);
    update_main(q, past, i, p1, false, nullptr);
    RayS x;
    ab3(q.dt, p1, v1, c0, x);
    update_main(q, next, i, x, false, nullptr);
    next.plen[i] = x.dist + 0.0;
    curr.plen[i] = 0.0;
    prev.plen[i] = 0.0;
    past.plen[i] = 0.0;
    for (int f = 0; f < RING; ++f) {
        const FrontPtrs& F = q.F[f];
        F.surface[i] = 0;
        F.bottom[i] = 0;
        F.caustic[i] = 0;
        F.upper[i] = 0;
        F.lower[i] = 0;
        F.on_edge[i] = 0;
    }
    const uint8_t f = reflect_decision(q, x.pos, c0.nd);
    q.flag[0][i] = f;
    if (f) work_append(q, 0, f, i);
    (void)a;
}

/* ------------------------------------------------------------------ */
/* one step: reflections (overlapping the previous step's CPA work),   */
/* then every ray advances                                             */
/* ------------------------------------------------------------------ */

/* The reflection chain of ray i at the start of step s (wave_queue.cc:
 * 197-256) on L: the ray's prev, curr and next states, counts and next-front
 * losses before the step's reflections.  The result goes to slot w of set
 * shadow_set(s); k_advance of step s takes it from there.  The caustic
 * hand-off from the D/E neighbour below (wave_queue.cc:274-292), which the
 * reference runs before the ray reflects, is decided by k_advance of step
 * s, when that neighbour's next front is complete; the slot carries the
 * phases both without and with its -pi/2 shift. */
__device__ __forceinline__ void reflect_chain_body(const QueueDev& q, int64_t s, int i, uint32_t w,
                                                   RayLocal& L, double t_old) {
    Roles R;
    roles_at(q, s, R);
    for (int f = 0; f < q.nf; ++f) L.phf[f] = L.ph[f] - M_PI_2;
    /* the reference's detect_reflections for this ray: volume layers,
     * then the surface / bottom chain, volume layers after each
     * reflection (wave_queue.cc:202-256); seq orders the ray's events */
    const bool vol = q.want_verbs && q.oc.nvol > 0;
    double dl[3] = {0.0, 0.0, 0.0};
    bool reflected = false;
    int seq = 0;
    int next_try = -1; /* 0: try bottom next, 1: try surface next */
    if (vol) volume_scatter(q, *R.C, i, s + 1, t_old, L.v, L.c, L.x, L.surface, L.bottom, seq);
    if (L.x.pos[0] - q.R > 0.0 && surface_local(q, *R.C, L, i, s + 1, t_old, seq)) {
        L.surface += 1;
        reflected = true;
        next_try = 0;
    } else {
        const double depth = boundary_height(q.oc.bot, L.x.pos[1], L.x.pos[2]) - L.x.pos[0];
        if (depth > 0.0) {
            bottom_local(q, *R.C, L, i, depth, s + 1, t_old, seq, dl);
            L.bottom += 1;
            reflected = true;
            next_try = 1;
        }
    }
    if (reflected) {
        if (vol) volume_scatter(q, *R.C, i, s + 1, t_old, L.v, L.c, L.x, L.surface, L.bottom, seq);
        int it = 0;
        for (; it < MAX_BOUNCE; ++it) {
            if (next_try == 0) {
                const double depth = boundary_height(q.oc.bot, L.x.pos[1], L.x.pos[2]) - L.x.pos[0];
                if (!(depth > 0.0)) break;
                bottom_local(q, *R.C, L, i, depth, s + 1, t_old, seq, dl);
                L.bottom += 1;
                next_try = 1;
            } else {
                if (!(L.x.pos[0] - q.R > 0.0 && surface_local(q, *R.C, L, i, s + 1, t_old, seq))) break;
                L.surface += 1;
                next_try = 0;
            }
            if (vol) volume_scatter(q, *R.C, i, s + 1, t_old, L.v, L.c, L.x, L.surface, L.bottom, seq);
        }
        if (it == MAX_BOUNCE) set_err(q, ERR_BOUNCE_LIMIT);
    }
    const int set = shadow_set(s);
    const size_t stride = shadow_stride(q);
    double* sh = q.shadow[set] + (size_t)w * stride;
    ray_to(sh, L.v);
    ray_to(sh + 17, L.c);
    ray_to(sh + 34, L.x);
    for (int f = 0; f < q.nf; ++f) {
        sh[51 + f] = L.att[f];
        sh[51 + q.nf + f] = L.ph[f];
        sh[54 + 2 * q.nf + f] = L.phf[f];
    }
    /* the next front's loss tangents take this step's bottom bounces
     * when k_commit applies the slot; the previous step's eigenray
     * construction may still be reading them */
    if (q.sens)
        for (int j = 0; j < 3; ++j) sh[51 + 2 * q.nf + j] = dl[j];
    q.shadow_cnt[set][3 * (size_t)w] = L.surface;
    q.shadow_cnt[set][3 * (size_t)w + 1] = L.bottom;
    q.shadow_cnt[set][3 * (size_t)w + 2] = L.caustic;
    q.shadow_slot[set][i] = (int32_t)w;
}

/* out of line for the inline schedule's advance, whose other rays need
 * none of its registers */
__device__ __noinline__ void reflect_chain(const QueueDev& q, int64_t s, int i, uint32_t w, RayLocal& L,
                                           double t_old) {
    reflect_chain_body(q, s, i, w, L, t_old);
}

/* Reflecting rays of step s listed by the launch that produced the "next"
 * front: the reflection chain on a private copy of each ray.  The fronts
 * are only read here, so this kernel runs concurrently with k_cpa /
 * k_eigenray of step s-1.  (k_advance reflects the following step's rays
 * itself where nothing in between needs the committed fronts; this kernel
 * then finds an empty list.) */
__global__ void __launch_bounds__(64) k_reflect(__grid_constant__ const QueueDev q, int k) {
    const int64_t s = *q.d_base + k;
    const uint32_t nsurf = min(*q.n_work[s & 1], (uint32_t)q.n);
    const uint32_t nwork = nsurf + min(*q.n_work_b[s & 1], (uint32_t)q.n - nsurf);
    const uint32_t* work = q.work[s & 1];
    const double t_old = q.d_times[k];
    Roles R;
    roles_at(q, s, R);
    for (uint32_t ww = blockIdx.x * blockDim.x + threadIdx.x; ww < nwork; ww += gridDim.x * blockDim.x) {
        /* list slot: surface part at the front, bottom part at the back */
        const uint32_t w = ww < nsurf ? ww : (uint32_t)q.n - 1 - (ww - nsurf);
        const int i = (int)work[w];
        WQ_CHECKED_OR(q, i >= 0 && i < q.n, continue);
        RayLocal L;
        {
            /* the fronts are read-only here */
            RayS v, c, x;
            load_prev_curr(q, s, R, i, v, c);
            load_ray_ro(*R.X, i, x);
            L.v = v;
            L.c = c;
            L.x = x;
            L.surface = __ldg(R.X->surface + i);
            L.bottom = __ldg(R.X->bottom + i);
            L.caustic = __ldg(R.X->caustic + i);
        }
        for (int f = 0; f < q.nf; ++f) {
            L.att[f] = __ldg(R.X->atten + (size_t)f * q.n + i);
            L.ph[f] = __ldg(R.X->phase + (size_t)f * q.n + i);
        }
        reflect_chain_body(q, s, i, w, L, t_old);
    }
    /* the last block to finish empties this step's worklist, which the
     * advance of step s+1 refills (every block has read the count by then;
     * the advance of step s fills the other list) */
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t prev = atomicAdd(q.n_done, 1u);
        if (prev == gridDim.x - 1) {
            *q.n_work[s & 1] = 0;
            *q.n_work_b[s & 1] = 0;
            *q.n_done = 0;
        }
    }
}

/* Every ray: commit of a reflected ray's shadow slot, caustic hand-off and
 * vertices for rays that did not reflect, find_edges of the front that
 * becomes "curr" (wave_front.cc:184-216; reflecting neighbours are read
 * from their shadow slots), the rotation, AB3 and update of the new front
 * (wave_queue.cc:162-183), and the reflection decision of the next step. */
/* five blocks per SM for the analytic build (96 registers, spills to L1
 * that cost less than the lost occupancy); the gridded build calls the
 * out-of-line grid interpolation and keeps its full register budget */
#if WQ3D_WITH_GRID
#define WQ_ADVANCE_BOUNDS __launch_bounds__(128)
#else
#define WQ_ADVANCE_BOUNDS __launch_bounds__(128, 5)
#endif
template <bool INLINE>
__device__ __forceinline__ void advance_body(const QueueDev& q, int k) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t s = *q.d_base + k;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        q.n_cand[cand_list(s + 1)] = 0;
        /* the slot count the next step's inline reflections start from */
        q.n_slot[shadow_set(s + 2)] = 0;
    }
    if (i >= q.n) return;
    Roles R;
    roles_at(q, s, R);
    const uint8_t* flag_in = q.flag[s & 1];
    uint8_t* flag_out = q.flag[(s + 1) & 1];
    const int naz = q.naz;
    const int d = i / naz;
    const size_t stride = shadow_stride(q);
    const int max_de = q.nde - 1;
    int jrow[4];
    jrow[0] = i + (max(d - 2, 0) - d) * naz;
    jrow[1] = i + (max(d - 1, 0) - d) * naz;
    jrow[2] = i + (min(d + 1, max_de) - d) * naz;
    jrow[3] = i + (min(d + 2, max_de) - d) * naz;
    const bool refl = __ldg(flag_in + i) != 0;
    bool fl[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) fl[t] = __ldg(flag_in + jrow[t]) != 0;
    /* Reads go through the read-only path: in this launch no ray reads an
     * element that another ray writes (neighbours are read only where they
     * do not reflect, and a reflecting ray's entries come from its shadow
     * slot), and a ray's own updated counters and phases stay in
     * registers, so the loads need not wait behind the stores. */
    RayS y0, y1, y2, y3;
    /* one round of loads: this ray on the three fronts, and the rows
     * d-2 .. d+2 that detect_caustics and find_edges may read (rows
     * clamped to the fan; a clamped row is never used) */
    const int set = shadow_set(s);
    if (!refl) load_prev_curr(q, s, R, i, y0, y1);
    load_ray_ro(*R.X, i, y2);
    int32_t sf = __ldg(R.X->surface + i);
    int32_t bt = __ldg(R.X->bottom + i);
    int32_t cs = __ldg(R.X->caustic + i);
    int32_t up = __ldg(R.X->upper + i);
    int32_t lo = __ldg(R.X->lower + i);
    double rr[4], nn[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        rr[t] = __ldg(R.X->pos[0] + jrow[t]);
        nn[t] = __ldg(R.X->nd[0] + jrow[t]);
    }
    const double c_below = curr_rho(q, s, R, jrow[1]);
    const int32_t sf_below = __ldg(R.X->surface + jrow[1]);
    const int32_t bt_below = __ldg(R.X->bottom + jrow[1]);
    const double x_below = rr[1];
    /* reflecting neighbours: their post-reflection entries */
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        if (fl[t]) {
            const int32_t wj = __ldg(q.shadow_slot[set] + jrow[t]);
            WQ_CHECKED_OR(q, wj >= 0 && wj < q.n, return);
            const double* shj = q.shadow[set] + (size_t)wj * stride;
            rr[t] = __ldg(shj + 34);
            nn[t] = __ldg(shj + 34 + 6);
        }
    }
    const double* sh = nullptr;
    bool fold_hit = false, vtx_up = false, vtx_lo = false;
    if (refl) {
        /* the reflected ray's states come from its shadow slot; k_commit
         * writes them into the curr and next fronts once the previous
         * step's eigenray construction no longer reads those fronts */
        const int32_t w = __ldg(q.shadow_slot[set] + i);
        WQ_CHECKED_OR(q, w >= 0 && w < q.n, return);
        sh = q.shadow[set] + (size_t)w * stride;
        ray_from(sh, y0);
        ray_from(sh + 17, y1);
        ray_from(sh + 34, y2);
        sf = __ldg(q.shadow_cnt[set] + 3 * (size_t)w);
        bt = __ldg(q.shadow_cnt[set] + 3 * (size_t)w + 1);
        cs = __ldg(q.shadow_cnt[set] + 3 * (size_t)w + 2);
        /* detect_caustics of the neighbour below on this ray's states
         * before its reflection (wave_queue.cc:274-292: the reference runs
         * it first); the fronts still hold them until k_commit */
        if (d >= 1 && !fl[1]) {
            const double A = curr_rho(q, s, R, i), B = c_below;
            const double Cc = __ldg(R.X->pos[0] + i), D = x_below;
            const bool fold = (__ldg(R.X->surface + i) == sf_below) && (__ldg(R.X->bottom + i) == bt_below);
            if ((Cc - D) * (A - B) < 0 && fold) {
                fold_hit = true;
                cs += 1;
            }
        }
    } else {
        /* detect_caustics of the neighbour below (wave_queue.cc:274-292) */
        if (d >= 1 && !fl[1]) {
            const double A = y1.pos[0], B = c_below;
            const double Cc = y2.pos[0], D = x_below;
            const bool fold = (sf == sf_below) && (bt == bt_below);
            if ((Cc - D) * (A - B) < 0 && fold) {
                fold_hit = true;
                cs += 1;
            }
        }
        /* detect_vertices (wave_queue.cc:261-269) */
        const double L = y1.nd[0];
        const double Rn = y2.nd[0];
        if (L * Rn < 0.0 && Rn < 0.0) {
            vtx_up = true;
            up += 1;
        } else if (L * Rn < 0.0 && 0.0 < Rn) {
            vtx_lo = true;
            lo += 1;
        }
    }
    /* find_edges on the post-reflection "next" front (wave_front.cc:
     * 184-216): a row is an extremum when its rho is below or above both
     * neighbour rows */
    bool edge;
    {
        auto ext = [](double r0, double rp, double rm) {
            return (r0 < rp && r0 < rm) || (r0 > rp && r0 > rm);
        };
        const double r_here = y2.pos[0], n_here = y2.nd[0];
        const bool ext_d = d >= 1 && d <= max_de - 1 && ext(r_here, rr[2], rr[1]);
        const bool ext_up = d + 1 >= 1 && d + 1 <= max_de - 1 && ext(rr[2], rr[3], r_here);
        const bool ext_dn = d - 1 >= 1 && d - 1 <= max_de - 1 && ext(rr[1], r_here, rr[0]);
        edge = (d == 0) || (d == max_de) || ext_d;
        if (!edge && ext_up) {
            const double n0 = nn[2];
            if (fabs(n0 - n_here) > fabs(n0 - nn[3])) edge = true;
        }
        if (!edge && ext_dn) {
            const double n0 = nn[1];
            if (!(fabs(n0 - nn[0]) > fabs(n0 - n_here))) edge = true;
        }
    }
    const double plen_x = __ldg(R.X->plen + i);
    /* rotate and take the AB3 step; wave_front::update of the new front
     * (the distance terms' sin(theta) is FP64 in every form) */
    ab3(q.dt, y0, y1, y2, y3);
    double st;
    if (q.precision == WQ3D_FP32) {
        update1_f32(q, y3);
        st = sin(y3.pos[1]);
    } else {
        profile_at(q, y3.pos, &y3.c, y3.sg);
        ray_derivs(y3.c, y3.sg[0], y3.sg[1], y3.sg[2], y3.pos, y3.nd, y3.pg, y3.ng, &st);
    }
    const uint8_t f_next = reflect_decision(q, y3.pos, y2.nd);
    /* the per-step finiteness check: a NaN or Inf in the environment (a
     * bad profile node, a zero sound speed) reaches the new front here */
    if (!isfinite(y3.pos[0] + y3.pos[1] + y3.pos[2] + y3.nd[0] + y3.nd[1] + y3.nd[2])) set_err(q, ERR_NONFINITE);
    /* stores: the new front, the next front's edge flag (not read by the
     * previous step's eigenray construction) and what k_commit changes on
     * the prev / curr / next fronts */
    q.commit_flag[set][i] = (uint8_t)((refl ? COMMIT_REFLECT : 0) | (fold_hit ? COMMIT_FOLD : 0) |
                                 (vtx_up ? COMMIT_UPPER : 0) | (vtx_lo ? COMMIT_LOWER : 0));
    R.X->on_edge[i] = edge ? 1 : 0;
    const FrontPtrs& P = *R.P;
    copy_ray(P, i, y3);
    P.cpa[0][i] = y3.pos[0];
    P.cpa[1][i] = y3.pos[1];
    P.cpa[2][i] = y3.pos[2];
    P.cpa[3][i] = st;
    P.plen[i] = y3.dist + plen_x;
    P.surface[i] = sf;
    P.bottom[i] = bt;
    P.upper[i] = up;
    P.lower[i] = lo;
    P.caustic[i] = cs;
    if (q.sens)
        for (int j = 0; j < 3; ++j)
            P.dA[(size_t)j * q.n + i] = __ldg(R.X->dA + (size_t)j * q.n + i) + (refl ? __ldg(sh + 51 + 2 * q.nf + j) : 0.0);
    /* attenuation (attenuation_thorp.cc:14-36 / attenuation_constant.cc:
     * 14-25) added to the next front's, phase carried over; the next
     * front's own entries take the reflection's values or the caustic's
     * phase shift first */
    const double alt = y3.pos[0] - q.R;
#pragma unroll 5
    for (int f = 0; f < q.nf; ++f) {
        const size_t o = (size_t)f * q.n + i;
        double ax, px;
        if (refl) {
            ax = __ldg(sh + 51 + f);
            px = __ldg(sh + (fold_hit ? 54 + 2 * q.nf : 51 + q.nf) + f);
        } else {
            ax = __ldg(R.X->atten + o);
            px = __ldg(R.X->phase + o);
            if (fold_hit) px -= M_PI_2;
        }
        double a;
        if (q.oc.prof.atten == WQ3D_ATTEN_CONSTANT) {
            a = q.oc.prof.atten_coef * y3.dist * q.freq[f];
        } else {
            a = y3.dist * q.alpha[f] * (1.0 + 5.88264e-6 * alt);
        }
        a += ax;
        double p = 0.0;
        p += px;
        P.atten[o] = a;
        P.phase[o] = p;
    }
    flag_out[i] = f_next;
    if (!f_next) return;
    if (!INLINE) {
        work_append(q, (int)((s + 1) & 1), f_next, i);
        return;
    }
    /* the reflections of step s+1 right here: this ray's prev and curr
     * states at step s+1 are its curr and next at step s, its next the
     * front just written (read back by this thread) */
    RayLocal L;
    if (refl) {
        ray_from(sh + 17, L.v);
        ray_from(sh + 34, L.c);
    } else {
        const double* sp = prev_step_slot(q, s, i);
        if (sp)
            ray_from(sp + 34, L.v);
        else
            load_ray_ro(*R.C, i, L.v);
        load_ray_ro(*R.X, i, L.c);
    }
    L.x = y3;
    L.surface = sf;
    L.bottom = bt;
    L.caustic = cs;
    for (int f = 0; f < q.nf; ++f) {
        L.att[f] = P.atten[(size_t)f * q.n + i];
        L.ph[f] = P.phase[(size_t)f * q.n + i];
    }
    const uint32_t w = atomicAdd(q.n_slot + shadow_set(s + 1), 1u);
    if (w >= (uint32_t)q.n) {
        set_err(q, ERR_SLOT_OVERFLOW);
        return;
    }
    reflect_chain(q, s + 1, i, w, L, q.d_times[k + 1]);
}

/* the side schedule: the reflecting rays of step s+1 go to the worklist
 * of k_reflect */
__global__ void WQ_ADVANCE_BOUNDS k_advance(__grid_constant__ const QueueDev q, int k) {
    advance_body<false>(q, k);
}

/* the inline schedule: each thread runs step s+1's reflection chain of
 * its ray itself */
__global__ void WQ_ADVANCE_BOUNDS k_advance_inline(__grid_constant__ const QueueDev q, int k) {
    advance_body<true>(q, k);
}

}  // namespace WQ3D_KERNEL_NS

#if !WQ3D_STEP_KERNELS_ONLY
/* What k_advance of step s decided for the prev / curr / next fronts, done
 * after the eigenray construction of step s-1 has read them: a reflected ray's
 * states, counts and next-front losses from its shadow slot
 * (reflection_model::reflection_copy, reflection_model.cc:335-360), and for
 * the other rays the caustic hand-off (count, and phase - pi/2 on every
 * frequency, wave_queue.cc:274-292) and the vertex counts (:261-269).
 * Until it has run, step s+1 reads a reflected ray's states from the slot
 * (prev_step_slot); the eigenray construction of step s, the eigenverbs of
 * step s+1 and the commit of step s+2 (which reuses this step's slot set)
 * wait for it. */
__global__ void __launch_bounds__(128) k_commit(__grid_constant__ const QueueDev q, int k) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= q.n) return;
    const int64_t s = *q.d_base + k;
    const int set = shadow_set(s);
    const uint8_t b = q.commit_flag[set][i];
    if (!b) return;
    Roles R;
    roles_at(q, s, R);
    if (b & COMMIT_REFLECT) {
        /* the prev front is read by no later kernel (this step's AB3 took
         * the reflected prev state from the slot) but is the "past" front
         * a caller may look at after the step */
        const int32_t w = q.shadow_slot[set][i];
        WQ_CHECKED_OR(q, w >= 0 && w < q.n, return);
        const double* sh = q.shadow[set] + (size_t)w * shadow_stride(q);
        const int32_t* cnt = q.shadow_cnt[set] + 3 * (size_t)w;
        RayS y;
        ray_from(sh, y);
        copy_ray(*R.V, i, y);
        ray_from(sh + 17, y);
        copy_ray(*R.C, i, y);
        ray_from(sh + 34, y);
        copy_ray(*R.X, i, y);
        R.V->surface[i] = R.C->surface[i] = R.X->surface[i] = cnt[0];
        R.V->bottom[i] = R.C->bottom[i] = R.X->bottom[i] = cnt[1];
        /* with the caustic hand-off k_advance found before the reflection */
        const bool fold = (b & COMMIT_FOLD) != 0;
        R.X->caustic[i] = cnt[2] + (fold ? 1 : 0);
        const double* ph = sh + (fold ? 54 + 2 * q.nf : 51 + q.nf);
        for (int f = 0; f < q.nf; ++f) {
            R.X->atten[(size_t)f * q.n + i] = sh[51 + f];
            R.X->phase[(size_t)f * q.n + i] = ph[f];
        }
        if (q.sens)
            for (int j = 0; j < 3; ++j) R.X->dA[(size_t)j * q.n + i] += sh[51 + 2 * q.nf + j];
        return;
    }
    if (b & COMMIT_FOLD) {
        R.X->caustic[i] += 1;
        for (int f = 0; f < q.nf; ++f) R.X->phase[(size_t)f * q.n + i] -= M_PI_2;
    }
    if (b & COMMIT_UPPER) R.X->upper[i] += 1;
    if (b & COMMIT_LOWER) R.X->lower[i] += 1;
}

/* Volume-layer eigenverbs of the rays that do not reflect in step s
 * (wave_queue.cc:202; k_reflect handles the reflecting ones).  Launched
 * before k_advance of the same step, only when an eigenverb listener is
 * installed and the ocean has volume layers. */
__global__ void __launch_bounds__(128) k_volume(__grid_constant__ const QueueDev q, int k) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= q.n) return;
    const int64_t s = *q.d_base + k;
    if (q.flag[s & 1][i]) return;
    Roles R;
    roles_at(q, s, R);
    const double rc = R.C->pos[0][i], rx = R.X->pos[0][i];
    bool cross = false;
    for (int v = 0; v < q.oc.nvol; ++v) cross |= (q.oc.vol_rho[v] - rx) * (q.oc.vol_rho[v] - rc) < 0;
    if (!cross) return;
    RayS y0, y1, y2;
    load_ray(*R.V, i, y0);
    load_ray(*R.C, i, y1);
    load_ray(*R.X, i, y2);
    int seq = 0;
    volume_scatter(q, *R.C, i, s + 1, q.d_times[k], y0, y1, y2, R.C->surface[i], R.C->bottom[i], seq);
}

/* ------------------------------------------------------------------ */
/* CPA search (wave_queue.cc:351-488)                                  */
/* ------------------------------------------------------------------ */
namespace {

struct TgtS {
    double th, ph, sn, R2, twoR;
};

__device__ __forceinline__ double d2_at(const FrontPtrs& f, int i, const TgtS& t) {
    const double rho = f.cpa[0][i];
    return target_distance2(rho, rho * rho, f.cpa[1][i], f.cpa[2][i], f.cpa[3][i],
                            t.th, t.ph, t.sn, t.R2, t.twoR);
}

/* appends (target, ray) to the candidate list of the step at s */
__device__ __forceinline__ void cand_push(const QueueDev& q, int64_t s, uint32_t t, uint32_t i) {
    const int l = cand_list(s);
    const uint32_t slot = atomicAdd(q.n_cand + l, 1u);
    if (slot < q.cap_cand) {
        uint32_t* c = q.cand + (size_t)l * 2 * q.cap_cand;
        c[2 * slot] = t;
        c[2 * slot + 1] = i;
    } else {
        set_err(q, ERR_CAND_OVERFLOW);
    }
}

__device__ __forceinline__ int wrap_az(const QueueDev& q, int az, int na) {
    int a = az + na - 1;
    if (q.az_boundary) {
        if (az + na == 0) {
            a = q.naz - 2;
        } else if (a >= q.naz - 1) {
            a = 0;
        }
    }
    return a;
}

/* is_closest_ray (wave_queue.cc:411-488); also fills the cube */
__device__ bool is_closest(const QueueDev& q, const FrontPtrs& V, const FrontPtrs& C,
                           const FrontPtrs& X, const TgtS& t, bool de_branch, int de,
                           int az, double center, double cube[3][3][3]) {
    const int max_az = q.naz - 1;
    for (int nd_ = 0; nd_ < 3; ++nd_) {
        for (int na = 0; na < 3; ++na) {
            if (nd_ == 1 && na == 1) continue;
            const int d = de + nd_ - 1;
            const int a = wrap_az(q, az, na);
            const int i = d * q.naz + a;
            cube[0][nd_][na] = d2_at(V, i, t);
            cube[1][nd_][na] = d2_at(C, i, t);
            cube[2][nd_][na] = d2_at(X, i, t);
            if (a == 0 && !q.az_boundary) continue;
            if (a == max_az) continue;
            if (de_branch) {
                if (C.on_edge[i]) continue;
            } else {
                if (nd_ != 1 && C.on_edge[i]) continue;
            }
            if (nd_ == 2 || na == 2) {
                if (de_branch) {
                    if (az == 0) {
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

}  // namespace

/* ------------------------------------------------------------------ */
/* CPA search over ray patches, with an FP32 screen in the FP32C form     */
/* ------------------------------------------------------------------ */
/* The comparisons that reject almost every (ray, target) pair -- "next <=
 * curr" and "prev < curr" on distance2 (wave_queue.cc:386-393) -- are
 * decided from the sign of a distance2 difference.  With coordinates
 * relative to a reference ray of the block (r = rho - rho0, x = theta -
 * theta0, y = phi - phi0; target Rr, X, Y likewise) the reference's
 * distance2 is, in exact arithmetic,
 *     Rr^2 + sum_k w_k(target) q_k(ray)
 *     q = (r^2, r, rho x^2, rho x, rho, rho s y^2, rho s y, rho s)
 *     w = (1, -2 Rr, R, -2 R X, R X^2, R S, -2 R S Y, R S Y^2)
 * (s = sin theta, S = sin Theta), so a difference of two fronts is
 * sum_k w_k dq_k: the per-ray feature differences dq_k are formed once in
 * FP64, and each pair costs 8 FP32 FMAs per comparison.  A comparison is
 * accepted in FP32 only when the difference exceeds 32 u sum_k W_k |dq_k|
 * (W_k = largest |w_k| of the target tile, u = 2^-24; the FP32 evaluation
 * error is below 12 u of that sum) plus max(1 m^2, 4e-15 (rho^2 + R^2))
 * for the rounding of the reference's FP64 expression on the two fronts
 * (each within 5 x 2^-53 (rho^2 + R^2), 0.05 m^2 at earth radius).  The
 * screen only rejects; every pair it does not reject is queued per warp and
 * finished with the FP64 comparisons, 32 at a time so the lanes stay
 * converged.  Hence the eigenrays equal the FP64 form's, which runs the
 * same patch search with every surviving pair going to those comparisons
 * (k_cpa).
 *
 * A block holds a patch of CPA_PATCH_DE x CPA_PATCH_AZ neighbouring rays,
 * whose positions and directions are close, so for a given target the
 * screen's value sum_k w_k dq_k varies little across the patch.  Before
 * the per-ray loop, each target is tested once for the whole patch: with
 * lo_k <= dq_k <= hi_k over the patch's rays, sum_k max(w_k lo_k, w_k hi_k)
 * (exact products of FP32 values, summed in FP64) bounds every ray's exact
 * value; adding the FP32 evaluation error (8 u sum W_k M_k, M_k = max
 * |dq_k|) and the largest guard of the patch (33 u sum W_k M_k + c0), a
 * negative bound means every ray of the patch would reject the target, so
 * it is dropped before the loop.  Only the targets that survive for the
 * "next" and the "prev" comparison reach the per-ray loop. */
namespace {
constexpr int F32_TARGETS = CPA_F32_TARGETS;
struct TgtW {
    float w[8];
};
struct WarpQueue {
    uint32_t e[64];
};

/* finishes queued pairs in FP64: entry = (thread of the ray << 16) | target */
__device__ __noinline__ void cpa_finish(const QueueDev& q, int64_t s, const FrontPtrs& V, const FrontPtrs& C,
                           const FrontPtrs& X, const TgtS* tile, int t0, int de0, int az0,
                           const uint32_t* e, int count, int lane) {
    if (lane >= count) return;
    const uint32_t v = e[lane];
    const int j = (int)(v & 0xffffu);
    const int th = (int)(v >> 16);
    WQ_CHECKED_OR(q, j < CPA_F32_TARGETS && th < CPA_THREADS, return);
    const int de = de0 + th / CPA_PATCH_AZ, az = az0 + th % CPA_PATCH_AZ;
    const int i = de * q.naz + az;
    WQ_CHECKED_OR(q, de < q.nde && az < q.naz, return);
    const TgtS t = tile[j];
    const double center = d2_at(C, i, t);
    if (d2_at(X, i, t) <= center) return;
    if (d2_at(V, i, t) < center) return;
    double cube[3][3][3];
    if (!is_closest(q, V, C, X, t, q.de_branch[t0 + j] != 0, de, az, center, cube)) return;
    cand_push(q, s, (uint32_t)(t0 + j), (uint32_t)i);
}

/* order-preserving keys of floats, for the warp's unsigned min / max
 * reductions (non-NaN values; -0 orders below +0) */
__device__ __forceinline__ unsigned f2key(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key2f(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

/* whether every ray of the patch rejects a target on one comparison.  In
 * FP32: each product and the 8-term sums carry at most about 8u of mag
 * (u = 2^-24), the weight sum about 9u of wm, the last three additions
 * about 3u of mag + c0; the 14u, 43u (41u of the per-ray screen plus its
 * own rounding) and 1.0003 factors cover them, so a rejection implies that
 * every ray's FP32 screen rejects the pair. */
struct PatchGuard {
    float M[8]; /* max(|lo_k|, |hi_k|) of the patch's feature ranges      */
    float K;    /* 43u * sum_k W_k M_k (W: the tile's largest weights)     */
    float Cc;   /* 1.0003 c0                                               */
};

/* the parts of the bound that are the same for every target of the tile */
__device__ __forceinline__ PatchGuard patch_guard(const float* lo, const float* hi, const float* W, float c0) {
    PatchGuard p;
    float wm = 0.0f;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        p.M[m] = fmaxf(fabsf(lo[m]), fabsf(hi[m]));
        wm += W[m] * p.M[m];
    }
    const float u = 5.9604645e-8f; /* 2^-24 */
    p.K = (43.0f * u) * wm;
    p.Cc = 1.0003f * c0;
    return p;
}

/* The sum above with one product per term: rounding is monotone, so
 * max(fl(w lo), fl(w hi)) is fl(w hi) for w >= 0 and fl(w lo) otherwise,
 * and max(|fl(w lo)|, |fl(w hi)|) is fl(|w| max(|lo|, |hi|)); the
 * additions keep their order, so the decisions are those of the full
 * form. */
__device__ __forceinline__ bool patch_rejects(const TgtW& g, const float* lo, const float* hi,
                                              const PatchGuard& p) {
    float ub = 0.0f, mag = 0.0f;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const float w = g.w[m];
        ub += w * (w >= 0.0f ? hi[m] : lo[m]);
        mag += fabsf(w) * p.M[m];
    }
    const float u = 5.9604645e-8f; /* 2^-24 */
    return ub + (14.0f * u) * mag + p.K + p.Cc < 0.0f;
}
}  // namespace

/* FP32 screen value sum_k w_k dq_k as two 4-term chains (any summation
 * order stays within the guard's 8 u bound) */
__device__ __forceinline__ float screen_dot(const TgtW& g, const float* d) {
    float a = fmaf(g.w[3], d[3], fmaf(g.w[2], d[2], fmaf(g.w[1], d[1], d[0])));
    float b = fmaf(g.w[7], d[7], fmaf(g.w[6], d[6], fmaf(g.w[5], d[5], g.w[4] * d[4])));
    return a + b;
}

/* The patch search; SCREEN decides the per-pair comparisons in FP32 first
 * (FP32C form), otherwise every pair of the patch's surviving targets goes
 * to the FP64 comparisons (FP64 form) */
template <bool SCREEN>
__device__ __forceinline__ void cpa_patch(const QueueDev& q, int k) {
    __shared__ TgtS tile[F32_TARGETS];
    __shared__ TgtW tw[F32_TARGETS];
    __shared__ float wmax[CPA_THREADS / 32][8];
    __shared__ float red[CPA_THREADS / 32][32];
    __shared__ float bound[32];
    __shared__ uint16_t surv[F32_TARGETS];
    __shared__ int nsurv;
    __shared__ WarpQueue wq[CPA_THREADS / 32];
    const int64_t s = *q.d_base + k + 1;
    const FrontPtrs& V = q.F[ring_slot(s + 1)];
    const FrontPtrs& C = q.F[ring_slot(s + 2)];
    const FrontPtrs& X = q.F[ring_slot(s + 3)];
    if (q.nde < 3 || q.naz < 3 || q.nt <= 0) return;
    const int n_pa = (q.naz + CPA_PATCH_AZ - 1) / CPA_PATCH_AZ;
    const int de0 = (blockIdx.x / n_pa) * CPA_PATCH_DE;
    const int az0 = (blockIdx.x % n_pa) * CPA_PATCH_AZ;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int de = de0 + threadIdx.x / CPA_PATCH_AZ, az = az0 + threadIdx.x % CPA_PATCH_AZ;
    bool active = de < q.nde && az < q.naz;
    const int i = active ? de * q.naz + az : 0;
    if (active) {
        const int az_start = q.az_boundary ? 0 : 1;
        active = !(de < 1 || de >= q.nde - 1 || az < az_start || az >= q.naz - 1) && !C.on_edge[i];
    }
    if (!__syncthreads_or(active)) return;
    /* local coordinates about the patch's middle ray */
    const int i_ref = min(de0 + CPA_PATCH_DE / 2, q.nde - 1) * q.naz + min(az0 + CPA_PATCH_AZ / 2, q.naz - 1);
    const double rho0 = C.cpa[0][i_ref], th0 = C.cpa[1][i_ref], ph0 = C.cpa[2][i_ref];

    /* this thread's ray: feature differences next-curr and prev-curr */
    float dxc[8], dvc[8];
    {
        double fq[3][8];
        const FrontPtrs* fr[3] = {&V, &C, &X};
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const double rho = fr[m]->cpa[0][i], sn = fr[m]->cpa[3][i];
            const double r = rho - rho0, x = fr[m]->cpa[1][i] - th0, y = fr[m]->cpa[2][i] - ph0;
            const double rs = rho * sn;
            fq[m][0] = r * r;
            fq[m][1] = r;
            fq[m][2] = rho * x * x;
            fq[m][3] = rho * x;
            fq[m][4] = rho;
            fq[m][5] = rs * y * y;
            fq[m][6] = rs * y;
            fq[m][7] = rs;
        }
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            dxc[m] = (float)(fq[2][m] - fq[1][m]);
            dvc[m] = (float)(fq[0][m] - fq[1][m]);
        }
    }
    /* feature ranges over the patch's active rays: bound[0..7] / [8..15]
     * low / high of dxc, [16..23] / [24..31] of dvc */
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const unsigned l1 = __reduce_min_sync(0xffffffffu, f2key(active ? dxc[m] : INFINITY));
        const unsigned h1 = __reduce_max_sync(0xffffffffu, f2key(active ? dxc[m] : -INFINITY));
        const unsigned l2 = __reduce_min_sync(0xffffffffu, f2key(active ? dvc[m] : INFINITY));
        const unsigned h2 = __reduce_max_sync(0xffffffffu, f2key(active ? dvc[m] : -INFINITY));
        if (lane == 0) {
            red[w][m] = key2f(l1);
            red[w][8 + m] = key2f(h1);
            red[w][16 + m] = key2f(l2);
            red[w][24 + m] = key2f(h2);
        }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const bool low = (threadIdx.x & 8) == 0;
        float v = red[0][threadIdx.x];
        for (int j = 1; j < CPA_THREADS / 32; ++j) v = low ? fminf(v, red[j][threadIdx.x]) : fmaxf(v, red[j][threadIdx.x]);
        bound[threadIdx.x] = v;
    }

    uint32_t* myq = wq[w].e;
    const unsigned lt = (1u << lane) - 1u;
    const float u = 5.9604645e-8f;
    /* this block's tile of targets (grid.y splits a patch's targets) */
    {
        const int t0 = blockIdx.y * F32_TARGETS;
        if (t0 >= q.nt) return;
        const int nt_tile = min(F32_TARGETS, q.nt - t0);
        float W[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = threadIdx.x; j < nt_tile; j += blockDim.x) {
            const int t = t0 + j;
            const double R = q.tgt[0][t], T = q.tgt[1][t], P = q.tgt[2][t], S = q.tgt_sin[t];
            tile[j] = TgtS{T, P, S, q.tgt_R2[t], q.tgt_2R[t]};
            const double Rr = R - rho0, Xo = T - th0, Yo = P - ph0, RS = R * S;
            TgtW g;
            g.w[0] = 1.0f;
            g.w[1] = (float)(-2.0 * Rr);
            g.w[2] = (float)R;
            g.w[3] = (float)(-2.0 * R * Xo);
            g.w[4] = (float)(R * Xo * Xo);
            g.w[5] = (float)RS;
            g.w[6] = (float)(-2.0 * RS * Yo);
            g.w[7] = (float)(RS * Yo * Yo);
            tw[j] = g;
#pragma unroll
            for (int m = 0; m < 8; ++m) W[m] = fmaxf(W[m], fabsf(g.w[m]));
        }
        /* W >= 0: its bit patterns order as unsigned integers */
#pragma unroll
        for (int m = 0; m < 8; ++m)
            W[m] = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(W[m])));
        if (lane == 0)
            for (int m = 0; m < 8; ++m) wmax[w][m] = W[m];
        if (threadIdx.x == 0) nsurv = 0;
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            float v = 0.0f;
            for (int j = 0; j < CPA_THREADS / 32; ++j) v = fmaxf(v, wmax[j][m]);
            W[m] = v * 1.0001f;
        }
        /* the guards of this tile, per ray and for the patch bound */
        const float r0 = (float)rho0;
        const float c0 = fmaxf(1.0f, 4.0e-15f * (r0 * r0 + W[2] * W[2]));
        float gxc = 0.0f, gvc = 0.0f;
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            gxc = fmaf(W[m], fabsf(dxc[m]), gxc);
            gvc = fmaf(W[m], fabsf(dvc[m]), gvc);
        }
        gxc = fmaf(32.0f * u, gxc, c0);
        gvc = fmaf(32.0f * u, gvc, c0);
        /* targets that some ray of the patch may keep */
        const PatchGuard px = patch_guard(&bound[0], &bound[8], W, c0);
        const PatchGuard pv = patch_guard(&bound[16], &bound[24], W, c0);
        for (int j = threadIdx.x; j < nt_tile; j += blockDim.x) {
            const TgtW g = tw[j];
            if (patch_rejects(g, &bound[0], &bound[8], px)) continue;
            if (patch_rejects(g, &bound[16], &bound[24], pv)) continue;
            surv[atomicAdd(&nsurv, 1)] = (uint16_t)j;
        }
        __syncthreads();
        const int ns = nsurv;
        int qn = 0;
        /* appends this lane's pair if "want"; finishes 32 at a time */
        auto push = [&](bool want, int j) {
            const unsigned mask = __ballot_sync(0xffffffffu, want);
            if (mask) {
                if (want) myq[qn + __popc(mask & lt)] = ((uint32_t)threadIdx.x << 16) | (uint32_t)j;
                qn += __popc(mask);
                __syncwarp();
                if (qn >= 32) {
                    cpa_finish(q, s, V, C, X, tile, t0, de0, az0, myq, 32, lane);
                    __syncwarp();
                    if (lane < qn - 32) myq[lane] = myq[32 + lane];
                    __syncwarp();
                    qn -= 32;
                }
            }
        };
        int sidx = 0;
        for (; sidx + 1 < ns; sidx += 2) {
            const int j0 = surv[sidx], j1 = surv[sidx + 1];
            const TgtW g0 = tw[j0], g1 = tw[j1];
            bool w0 = active, w1 = active;
            if (SCREEN) {
                const float a0 = screen_dot(g0, dxc), a1 = screen_dot(g1, dxc);
                w0 = w0 && !(a0 < -gxc);
                w1 = w1 && !(a1 < -gxc);
                if (w0 || w1) {
                    const float b0 = screen_dot(g0, dvc), b1 = screen_dot(g1, dvc);
                    w0 = w0 && !(b0 < -gvc);
                    w1 = w1 && !(b1 < -gvc);
                }
            }
            push(w0, j0);
            push(w1, j1);
        }
        if (sidx < ns) {
            const int j = surv[sidx];
            const TgtW g = tw[j];
            bool want = active;
            if (SCREEN) {
                want = want && !(screen_dot(g, dxc) < -gxc);
                if (want) want = !(screen_dot(g, dvc) < -gvc);
            }
            push(want, j);
        }
        if (qn > 0) cpa_finish(q, s, V, C, X, tile, t0, de0, az0, myq, qn, lane);
    }
}

/* four resident blocks (128 registers): the reflection chain that runs
 * beside the search keeps issue slots */
__global__ void __launch_bounds__(CPA_THREADS, 3) k_cpa_f32(__grid_constant__ const QueueDev q, int k) {
    cpa_patch<true>(q, k);
}

__global__ void __launch_bounds__(CPA_THREADS, 3) k_cpa(__grid_constant__ const QueueDev q, int k) {
    cpa_patch<false>(q, k);
}

/* ------------------------------------------------------------------ */
/* eigenray construction (wave_queue.cc:495-977 + spreading models)    */
/* ------------------------------------------------------------------ */
namespace {

/* One warp builds one eigenray (with a second warp for the AZ walks of
 * hybrid Gaussian spreading).  Lanes share the parallel parts (the 27
 * distance2 values, the 54 direction angles, the cell widths and Gaussian
 * terms of the beam walks, the per-frequency sums); every value that feeds
 * a rounding-sensitive recurrence (cell distances, the running intensity
 * and its threshold test) is formed in the reference's sequential order,
 * so results equal the one-thread-per-eigenray evaluation. */
constexpr int EIG_FG = 8; /* frequencies per pass of a walk chunk's Gaussian terms */

struct WarpBuild {
    const QueueDev* q;
    const FrontPtrs* pV;
    const FrontPtrs* pC;
    const FrontPtrs* pX;
    const double* spread2;   /* [nf] for this target */
    int lane;
    double Ilo, Ihi;         /* running intensity of frequencies lane, lane+32 */
    double (*sg)[EIG_FG + 1]; /* this warp's [cell][frequency] Gaussian terms */

    __device__ double fdist(const FrontPtrs& f, int d1, int a1, int d2, int a2) const {
        const int i = d1 * q->naz + a1, j = d2 * q->naz + a2;
        return sqrt(wdist2(f.pos[0][i], f.pos[1][i], f.pos[2][i], f.pos[0][j],
                           f.pos[1][j], f.pos[2][j]));
    }
    __device__ double de_inc(int d) const { return q->de_inc[min(max(d, 0), q->nde - 1)]; }
    __device__ double az_inc(int a) const { return q->az_inc[min(max(a, 0), q->naz - 1)]; }

    /* spreading_hybrid_gaussian.h:148-153 for one frequency */
    __device__ double gauss(double d, double w, double A, int f) const {
        const double bw = spread2[f] + 2.0 * 2.0 * w * w;
        return exp((-0.5 * d * d) / bw) / sqrt(bw) * A;
    }
    /* running intensity += gaussian, frequencies spread over the lanes */
    __device__ void acc(double d, double w, double A, bool first) {
        const int nf = q->nf;
        if (lane < nf) {
            const double g = gauss(d, w, A, lane);
            Ilo = first ? g : Ilo + g;
        }
        if (lane + 32 < nf) {
            const double g = gauss(d, w, A, lane + 32);
            Ihi = first ? g : Ihi + g;
        }
    }
    __device__ double I0() const { return __shfl_sync(0xffffffffu, Ilo, 0); }

    /* The lowest frequency's running intensity over cells 0..ncell-1 (lane
     * k holds cell k's term g0), added in cell order, and the reference's
     * threshold test after each cell (new / old < 1.002305238).  Returns
     * the first cell that passes it, or -1.  The sums are sequential; the
     * divisions of the tests are not, so they run on all lanes at once. */
    __device__ int threshold_cell(int ncell, double g0) const {
        double i0 = I0();
        double my_new = 1.0, my_old = 1.0;
        for (int k = 0; k < ncell; ++k) {
            const double old = i0;
            i0 += __shfl_sync(0xffffffffu, g0, k);
            if (lane == k) {
                my_new = i0;
                my_old = old;
            }
        }
        const unsigned hit = __ballot_sync(0xffffffffu, lane < ncell && my_new / my_old < 1.002305238);
        return hit ? __ffs(hit) - 1 : -1;
    }

    /* acc() of cells 0..ncell-1 in cell order, for every frequency: lane k
     * computes cell k's Gaussian terms (EIG_FG frequencies per pass), then
     * the lane that owns a frequency adds them up in cell order */
    __device__ void acc_cells(int ncell, double cd, double cw, double nm) {
        const int nf = q->nf;
        for (int f0 = 0; f0 < nf; f0 += EIG_FG) {
            const int nfg = min(EIG_FG, nf - f0);
            if (lane < ncell)
                for (int j = 0; j < nfg; ++j) sg[lane][j] = gauss(cd, cw, nm, f0 + j);
            __syncwarp();
            if (lane >= f0 && lane < f0 + nfg) {
                double I = Ilo;
                for (int k = 0; k < ncell; ++k) I = I + sg[k][lane - f0];
                Ilo = I;
            }
            if (lane + 32 >= f0 && lane + 32 < f0 + nfg) {
                double I = Ihi;
                for (int k = 0; k < ncell; ++k) I = I + sg[k][lane + 32 - f0];
                Ihi = I;
            }
            __syncwarp();
        }
    }

    /* spreading_hybrid_gaussian.cc:430-495 */
    __device__ double width_de(int d, int a, const double* offset) const {
        const double u = fabs(offset[0]) / q->dt;
        const double v = fabs(offset[2]) / az_inc(a);
        const int max_az = q->naz - 1;
        const int az_wrap = (a + 1 >= max_az) ? 0 : a + 1;
        const FrontPtrs& C = *pC;
        double L1 = fdist(C, d, a, d + 1, a), L2, length1, length2;
        if (v < 1e-10) {
            length1 = L1;
        } else {
            L2 = fdist(C, d, az_wrap, d + 1, az_wrap);
            length1 = (1.0 - v) * L1 + v * L2;
        }
        if (u < 1e-10) return 0.5 * length1;
        const FrontPtrs& p2 = (offset[0] < 0.0) ? *pV : *pX;
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
    __device__ double width_az(int d, int a, const double* offset) const {
        const double u = fabs(offset[0]) / q->dt;
        const double v = fabs(offset[1]) / de_inc(d);
        const int max_az = q->naz - 1;
        const int max_de = q->nde - 1;
        const int de_upper = (d + 1 >= max_de) ? max_de - 2 : d;
        const int az_wrap = (a + 1 > max_az) ? 0 : a + 1;
        const FrontPtrs& C = *pC;
        double L1 = fdist(C, d, a, d, az_wrap), L2, length1, length2;
        if (v < 1e-10 || fabs(v - 1.0) < 1e-10) {
            length1 = L1;
        } else {
            L2 = fdist(C, de_upper + 1, a, de_upper + 1, az_wrap);
            length1 = (1.0 - v) * L1 + v * L2;
        }
        if (u < 1e-10) return 0.5 * length1;
        const FrontPtrs& p2 = (offset[0] < 0.0) ? *pV : *pX;
        L1 = fdist(p2, d, a, d, az_wrap);
        if (v < 1e-10 || fabs(v - 1.0) < 1e-10) {
            length2 = L1;
        } else {
            L2 = fdist(p2, de_upper + 1, a, de_upper + 1, az_wrap);
            length2 = (1.0 - v) * L1 + v * L2;
        }
        return 0.5 * ((1.0 - u) * length1 + u * length2);
    }

    /* Processes up to 32 prepared cells of one walk.  Lane k holds cell k's
     * width (w_k), whether the cell is a virtual ray (virt_k) and the two
     * normalisation candidates.  sign = +1 for a walk away from the lower
     * side (cell distances grow), -1 otherwise.  Returns true when the walk
     * stops inside these cells. */
    __device__ bool run_cells(int ncell, double w_k, bool virt_k, double norm_k,
                              double norm_virt_k, double sign, double& cell_dist,
                              double& cell_width) {
        double my_cd = 0.0, my_cw = 0.0, my_nm = 0.0;
        int nend = ncell;
        bool stop = false;
        for (int k = 0; k < ncell; ++k) {
            const bool v = __shfl_sync(0xffffffffu, virt_k, k);
            const double wk = __shfl_sync(0xffffffffu, w_k, k);
            const double nk = __shfl_sync(0xffffffffu, v ? norm_virt_k : norm_k, k);
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
                my_nm = nk;
            }
            if (v) {
                nend = k + 1;
                stop = true;
                break;
            }
        }
        /* threshold scan on the lowest frequency, in order */
        const double g0 = (lane < nend) ? gauss(my_cd, my_cw, my_nm, 0) : 0.0;
        int kstar = threshold_cell(nend, g0);
        if (kstar >= 0) {
            stop = true;
        } else {
            kstar = nend - 1;
        }
        /* accumulate every frequency over cells 0..kstar, in order */
        acc_cells(kstar + 1, my_cd, my_cw, my_nm);
        return stop;
    }

    /* spreading_hybrid_gaussian.cc:124-258 */
    __device__ void intensity_de(int de0, int a, const double* offset, const double* distance) {
        const QueueDev& Q = *q;
        const FrontPtrs& C = *pC;
        double wl = 0.0, wc = 0.0;
        if (lane == 0) wc = width_de(de0, a, offset);
        if (lane == 1) wl = width_de(de0 - 1, a, offset);
        wc = __shfl_sync(0xffffffffu, wc, 0);
        wl = __shfl_sync(0xffffffffu, wl, 1);
        const double L = distance[1];
        acc(L - wc, wc, Q.norm_de[de0], true);
        acc(L + wl, wl, Q.norm_de[de0 - 1], false);
        if (I0() < 1e-10) return;
        /* lower D/E cells: de0-2 down to 0 */
        double cell_width = wl, cell_dist = L + wl;
        for (int d0 = de0 - 2; d0 >= 0; d0 -= 32) {
            const int d = d0 - lane;
            const int ncell = min(32, d0 + 1);
            bool virt = false;
            double w = 0.0, nm = 0.0, nmv = 0.0;
            if (lane < ncell) {
                virt = C.on_edge[(d + 1) * Q.naz + a] && C.on_edge[d * Q.naz + a];
                if (!virt) w = width_de(d, a, offset);
                nm = Q.norm_de[d];
                nmv = Q.norm_de[d + 1];
            }
            if (run_cells(ncell, w, virt, nm, nmv, 1.0, cell_dist, cell_width)) break;
        }
        /* upper D/E cells: de0+1 up to num_de-2 */
        cell_width = wc;
        cell_dist = L - wc;
        const int size = Q.nde - 1;
        for (int d0 = de0 + 1; d0 < size; d0 += 32) {
            const int d = d0 + lane;
            const int ncell = min(32, size - d0);
            bool virt = false;
            double w = 0.0, nm = 0.0, nmv = 0.0;
            if (lane < ncell) {
                virt = C.on_edge[(d + 1) * Q.naz + a] && C.on_edge[d * Q.naz + a];
                if (!virt) w = width_de(d, a, offset);
                nm = Q.norm_de[d];
                nmv = Q.norm_de[d - 1];
            }
            if (run_cells(ncell, w, virt, nm, nmv, -1.0, cell_dist, cell_width)) break;
        }
    }

    /* spreading_hybrid_gaussian.cc:264-425.  The duplicate mask of the
     * reference is a cyclic range: the lower walk marks a contiguous run of
     * AZ indices below the centre, so membership is a range test. */
    __device__ void intensity_az(int d, int az0, const double* offset, const double* distance) {
        const QueueDev& Q = *q;
        const FrontPtrs& C = *pC;
        const int max_de = Q.nde - 2;
        const int max_az = Q.naz - 1;
        const int az_lower = Q.az_boundary ? az0 : 0;
        const int az_upper = Q.az_boundary ? az0 : max_az - 1;
        auto norm = [&](int aa) { return (d >= max_de) ? Q.norm_az[1 * Q.naz + aa] : Q.norm_az[d * Q.naz + aa]; };
        const int a1 = (az0 < 1) ? max_az - 1 : az0 - 1;
        double wc = 0.0, wl = 0.0;
        if (lane == 0) wc = width_az(d, az0, offset);
        if (lane == 1) wl = width_az(d, a1, offset);
        wc = __shfl_sync(0xffffffffu, wc, 0);
        wl = __shfl_sync(0xffffffffu, wl, 1);
        const double L = distance[2];
        acc(L - wc, wc, norm(az0), true);
        acc(L + wl, wl, norm(a1), false);
        if (I0() < 1e-10) return;
        /* lower walk: a1-1, a1-2, ... (cyclic) until az_lower */
        const int start = (a1 < 1) ? max_az - 1 : a1 - 1;
        double cell_width = wl, cell_dist = L + wl;
        int marked = -1; /* index (in walk order) of the last cell marked */
        bool done = false;
        for (int k0 = 0; !done && k0 < max_az; k0 += 32) {
            const int k = k0 + lane;
            int a = start - k;
            a = ((a % max_az) + max_az) % max_az;
            /* per-cell stop tests, in the reference's order */
            int kind = 0; /* 0 process, 1 loop end (not marked), 2 marked stop */
            if (k >= max_az || a == az_lower) {
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
            double w = 0.0;
            if (lane < ncell) w = width_az(d, a, offset);
            const double nm = (lane < ncell) ? norm(a) : 0.0;
            int kst = -1;
            const bool brk = (ncell > 0) && run_cells_az(ncell, w, nm, 1.0, cell_dist, cell_width, kst);
            if (brk) {
                marked = k0 + kst; /* the threshold stop happens on a marked cell */
                done = true;
            } else {
                if (ncell > 0) marked = k0 + ncell - 1;
                if (stopmask) {
                    done = true;
                    if (fk == 2) marked = k0 + first; /* on_edge cells are marked, not used */
                }
            }
        }
        /* upper walk: az0+1, az0+2, ... (cyclic) until az_upper */
        cell_width = wc;
        cell_dist = L - wc;
        done = false;
        for (int k0 = 0; !done && k0 < max_az; k0 += 32) {
            const int k = k0 + lane;
            const int a = (az0 + 1 + k) % max_az;
            int kind = 0;
            /* membership of the lower walk's marked cells: start-j, j <= marked */
            const int off = ((start - a) % max_az + max_az) % max_az;
            const bool dup = (a == az0) || (a == a1) || (marked >= 0 && off <= marked);
            if (k >= max_az || a == az_upper) {
                kind = 1;
            } else if (dup) {
                kind = 1;
            } else if (C.on_edge[d * Q.naz + a]) {
                kind = 1;
            }
            const unsigned stopmask = __ballot_sync(0xffffffffu, kind != 0);
            int ncell = 32;
            if (stopmask) {
                ncell = __ffs(stopmask) - 1;
                done = true;
            }
            double w = 0.0;
            if (lane < ncell) w = width_az(d, a, offset);
            const double nm = (lane < ncell) ? norm(a) : 0.0;
            int kst = -1;
            if (ncell > 0 && run_cells_az(ncell, w, nm, -1.0, cell_dist, cell_width, kst)) done = true;
        }
    }

    /* AZ walks have no virtual rays; a threshold stop marks the cell it
     * happened on (for the upper walk's duplicate test) */
    __device__ bool run_cells_az(int ncell, double w_k, double norm_k, double sign,
                                 double& cell_dist, double& cell_width, int& kstop) {
        double my_cd = 0.0, my_cw = 0.0, my_nm = 0.0;
        for (int k = 0; k < ncell; ++k) {
            const double wk = __shfl_sync(0xffffffffu, w_k, k);
            const double nk = __shfl_sync(0xffffffffu, norm_k, k);
            if (sign > 0.0) {
                cell_dist += cell_width;
                cell_width = wk;
                cell_dist += cell_width;
            } else {
                cell_dist -= cell_width;
                cell_width = wk;
                cell_dist -= cell_width;
            }
            if (lane == k) {
                my_cd = cell_dist;
                my_cw = cell_width;
                my_nm = nk;
            }
        }
        const double g0 = (lane < ncell) ? gauss(my_cd, my_cw, my_nm, 0) : 0.0;
        int kstar = threshold_cell(ncell, g0);
        const bool stop = kstar >= 0;
        if (!stop) kstar = ncell - 1;
        acc_cells(kstar + 1, my_cd, my_cw, my_nm);
        if (stop) kstop = kstar;
        return stop;
    }

    /* wvector1::area on four points (types/wvector1.cc) */
    __device__ double area4(const FrontPtrs& f, int d, int a) const {
        double aa = fdist(f, d, a, d + 1, a);
        const double b = fdist(f, d, a, d + 1, a + 1);
        double c = fdist(f, d + 1, a, d + 1, a + 1);
        const double area1 = 0.25 * sqrt((aa + b + c) * (b + c - aa) * (c + aa - b) * (aa + b - c));
        aa = fdist(f, d, a, d, a + 1);
        c = fdist(f, d, a + 1, d + 1, a + 1);
        const double area2 = 0.25 * sqrt((aa + b + c) * (b + c - aa) * (c + aa - b) * (aa + b - c));
        return area1 + area2;
    }
};

__device__ __forceinline__ void make_taylor_coeff(const double v[3][3][3], const double* delta,
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

__device__ __forceinline__ double dot3(const double* a, const double* b) {
    double t = 0.0;
    t += a[0] * b[0];
    t += a[1] * b[1];
    t += a[2] * b[2];
    return t;
}
__device__ __forceinline__ void matvec(const double m[3][3], const double* x, double* y) {
    for (int r = 0; r < 3; ++r) {
        double t = 0.0;
        t += m[r][0] * x[0];
        t += m[r][1] * x[1];
        t += m[r][2] * x[2];
        y[r] = t;
    }
}
__device__ __forceinline__ double norm2(const double* g) {
    double t = 0.0;
    t += fabs(g[0]) * fabs(g[0]);
    t += fabs(g[1]) * fabs(g[1]);
    t += fabs(g[2]) * fabs(g[2]);
    return sqrt(t);
}

/* wave_queue::compute_offsets (wave_queue.cc:708-924).  Called by a whole
 * warp: lanes 0-8 test the 3x3 neighbours' stability at once. */
__device__ void compute_offsets(const QueueDev& q, const FrontPtrs& V, const FrontPtrs& C,
                                const FrontPtrs& X, int t, int de0, int az0,
                                const double cube[3][3][3], const double* delta,
                                double* offset, double* distance) {
    const int ic = de0 * q.naz + az0;
    bool bad = false;
    {
        const int lane = threadIdx.x & 31;
        if (lane < 9) {
            const int surface = C.surface[ic], bottom = C.bottom[ic], caustic = C.caustic[ic];
            const int i = (de0 + lane / 3 - 1) * q.naz + wrap_az(q, az0, lane % 3);
            bad = V.surface[i] != surface || C.surface[i] != surface || X.surface[i] != surface ||
                  V.bottom[i] != bottom || C.bottom[i] != bottom || X.bottom[i] != bottom ||
                  V.caustic[i] != caustic || C.caustic[i] != caustic || X.caustic[i] != caustic ||
                  V.on_edge[i];
        }
    }
    bool unstable = __any_sync(0xffffffffu, bad);
    double center, g[3], h[3][3], inv[3][3];
    make_taylor_coeff(cube, delta, center, g, h);
    /* kept: hessian(2,1)*hessian(2,0) in the last cofactor (wave_queue.cc:762-763) */
    double determinant = fmax(1e-6, h[0][0] * (h[1][1] * h[2][2] - h[1][2] * h[2][1]) +
                                        h[0][1] * (h[1][2] * h[2][0] - h[1][0] * h[2][2]) +
                                        h[0][2] * (h[1][0] * h[2][1] - h[2][1] * h[2][0]));
    unstable = unstable || determinant < norm2(g);
    for (int k = 0; k < 3; ++k) {
        const double hh = fmax(1e-10, h[k][k]);
        offset[k] = -g[k] / hh;
        if (fabs(offset[k] / delta[k]) > 0.5) {
            unstable = true;
            offset[k] = (offset[k] < 0.0) ? -(0.5 * delta[k]) : 0.5 * delta[k];
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
        unstable = unstable || fabs(offset[1]) >= 0.5 * fabs(delta[1]);
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
        distance[k] = sqrt(fmax(0.0, distance[k]));
        if (offset[k] < 0.0) distance[k] *= -1.0;
    }
    if (unstable) {
        distance[1] = center - distance[0] * distance[0] - distance[2] * distance[2];
        if (distance[1] <= 0.0) {
            distance[1] = 0.0;
            offset[1] = 0.0;
        } else {
            distance[1] = sqrt(distance[1]);
            offset[1] = fabs(offset[1]);
            double cpa[3], nxt[3], prv[3], dir[3], speed;
            collision_location(q, V, C, X, ic, offset[0], cpa, dir, &speed);
            collision_location(q, V, C, X, ic + q.naz, offset[0], nxt, dir, &speed);
            collision_location(q, V, C, X, ic - q.naz, offset[0], prv, dir, &speed);
            double nxt_dir[3], tgt_dir[3];
            nxt_dir[0] = nxt[0] - cpa[0];
            nxt_dir[1] = (nxt[1] - prv[1]) * cpa[0];
            nxt_dir[2] = (nxt[2] - prv[2]) * cpa[0] * sin(cpa[1]);
            if (fabs(nxt_dir[0]) < 0.01) nxt_dir[0] = 0.0;
            tgt_dir[0] = q.tgt[0][t] - cpa[0];
            tgt_dir[1] = (q.tgt[1][t] - cpa[1]) * cpa[0];
            tgt_dir[2] = (q.tgt[2][t] - cpa[2]) * cpa[0] * sin(cpa[1]);
            if (dot3(nxt_dir, tgt_dir) < 0.0) {
                distance[1] *= -1.0;
                offset[1] *= -1.0;
            }
        }
    }
}

}  // namespace

constexpr int EIG_WARPS = 4;

/* the two warps of pair p (warps 2p, 2p+1 of the block) meet here */
__device__ __forceinline__ void pair_sync(int pair) {
    static_assert(EIG_WARPS == 4, "two warp pairs per block: named barriers 1 and 2");
    if (pair == 0)
        asm volatile("bar.sync 1, 64;" ::: "memory");
    else
        asm volatile("bar.sync 2, 64;" ::: "memory");
}

__global__ void __launch_bounds__(32 * EIG_WARPS) k_eigenray(__grid_constant__ const QueueDev q, int k) {
    __shared__ double s_cube[EIG_WARPS][27];
    __shared__ double s_ang[EIG_WARPS][2][27];
    __shared__ double s_g[EIG_WARPS][32][EIG_FG + 1];
    __shared__ double s_az[EIG_WARPS / 2][64];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    /* a warp pair per candidate: with hybrid Gaussian spreading the even
     * warp runs the D/E walks and the odd warp the AZ walks, which are
     * independent sums; the odd warp hands its sums over and moves on */
    const int pair = warp >> 1, half = warp & 1;
    const int64_t s = *q.d_base + k + 1;
    const double time = q.d_times[k + 1];
    const int list = cand_list(s);
    const uint32_t ncand = min(q.n_cand[list], q.cap_cand);
    const uint32_t* cand = q.cand + (size_t)list * 2 * q.cap_cand;
    WarpBuild B;
    B.q = &q;
    B.pV = &q.F[ring_slot(s + 1)];
    B.pC = &q.F[ring_slot(s + 2)];
    B.pX = &q.F[ring_slot(s + 3)];
    B.lane = lane;
    B.sg = s_g[warp];
    const FrontPtrs& V = *B.pV;
    const FrontPtrs& C = *B.pC;
    const FrontPtrs& X = *B.pX;
    double (*cube)[3][3] = reinterpret_cast<double (*)[3][3]>(s_cube[warp]);
    const uint32_t npairs = gridDim.x * (EIG_WARPS / 2);
    for (uint32_t c = blockIdx.x * (EIG_WARPS / 2) + pair; c < ncand; c += npairs) {
        __syncwarp();
        const uint32_t tu = cand[2 * c], iu = cand[2 * c + 1];
        /* the CPA kernels only queue interior rays and real targets */
        if (tu >= (uint32_t)q.nt || iu >= (uint32_t)q.n || iu / q.naz < 1 || iu / q.naz > (uint32_t)q.nde - 2) {
            if (lane == 0) set_err(q, ERR_BAD_CANDIDATE);
            continue;
        }
        const int t = (int)tu;
        const int i = (int)iu;
        const int de0 = i / q.naz, az0 = i % q.naz;
        /* above_bounce_threshold (wave_thresholds.h:192-199) */
        if (C.bottom[i] > q.max_bottom || C.surface[i] > q.max_surface ||
            C.caustic[i] > q.max_caustic || C.upper[i] > q.max_upper || C.lower[i] > q.max_lower)
            continue;
        const TgtS tg{q.tgt[1][t], q.tgt[2][t], q.tgt_sin[t], q.tgt_R2[t], q.tgt_2R[t]};
        /* the 27 distance2 values, one per lane */
        if (lane < 27) {
            const int m = lane / 9, nd_ = (lane / 3) % 3, na = lane % 3;
            const int j = (de0 + nd_ - 1) * q.naz + wrap_az(q, az0, na);
            const FrontPtrs& F = (m == 0) ? V : (m == 1) ? C : X;
            s_cube[warp][lane] = d2_at(F, j, tg);
        }
        __syncwarp();
        double delta[3] = {q.dt, q.de_inc[de0], q.az_inc[az0]};
        double offset[3], distance[3];
        compute_offsets(q, V, C, X, t, de0, az0, cube, delta, offset, distance);

        /* spreading: lane f holds frequency f (and f + 32) */
        double si_lo = 0.0, si_hi = 0.0;
        B.spread2 = q.tgt_spread2 + (size_t)t * q.nf;
        if (q.spreading == WQ3D_HYBRID_GAUSSIAN) {
            /* spreading_hybrid_gaussian.cc:65-119 */
            int a = az0;
            double no[3] = {offset[0], offset[1], offset[2]};
            if (offset[2] < 0.0) {
                if (az0 > 0) {
                    a = az0 - 1;
                } else if (q.az_boundary) {
                    a = q.naz - 2;
                }
                no[2] = offset[2] + B.az_inc(a);
            }
            double de_lo = 0.0, de_hi = 0.0;
            if (half == 0) {
                B.Ilo = B.Ihi = 0.0;
                B.intensity_de(de0, a, no, distance);
                de_lo = B.Ilo;
                de_hi = B.Ihi;
            } else {
                no[2] = offset[2];
                int d = de0;
                if (offset[1] < 0.0 && !C.on_edge[i - q.naz]) {
                    d = de0 - 1;
                    no[1] = offset[1] + B.de_inc(d);
                }
                B.Ilo = B.Ihi = 0.0;
                B.intensity_az(d, az0, no, distance);
                s_az[pair][lane] = B.Ilo;
                s_az[pair][32 + lane] = B.Ihi;
            }
            /* both warps pass both barriers once per candidate */
            pair_sync(pair);
            if (half == 1) {
                pair_sync(pair);
                continue;
            }
            const double az_lo = s_az[pair][lane], az_hi = s_az[pair][32 + lane];
            pair_sync(pair);
            si_lo = de_lo * az_lo;
            si_hi = de_hi * az_hi;
        } else {
            if (half == 1) continue;
            /* spreading_ray.cc:47-133; an AZ wrap below index 0 is wrapped */
            int d = de0, a = az0;
            if (offset[1] < 0.0) --d;
            if (offset[2] < 0.0) a = (a == 0) ? q.naz - 2 : a - 1;
            const double area1 = B.area4(C, d, a);
            const double area2 = (offset[0] < 0.0) ? B.area4(V, d, a) : B.area4(X, d, a);
            double u = fabs(offset[0]) / q.dt;
            const double area = (1.0 - u) * area1 + u * area2;
            const double loss = q.init_area[d * q.naz + a] * q.tgt_c[t] / (area * q.init_sound_speed);
            bool zero = false;
            u = fabs(offset[1]) / B.de_inc(d) - 1.0;
            if (u > 4.0) zero = true;
            u = fabs(offset[2]) / B.az_inc(a) - 1.0;
            if (u > 4.0) zero = true;
            si_lo = si_hi = zero ? loss * 0.0 : loss;
        }
        const bool has_lo = lane < q.nf, has_hi = lane + 32 < q.nf;
        const bool bad = (has_lo && isnan(si_lo)) || (has_hi && isnan(si_hi));
        if (__any_sync(0xffffffffu, bad)) continue;
        double tl_lo = -10.0 * log10(fmax(si_lo, 1e-30));
        double tl_hi = -10.0 * log10(fmax(si_hi, 1e-30));
        double ddt = offset[0] / q.dt;
        const FrontPtrs& A0 = (ddt >= 0.0) ? C : V;
        const FrontPtrs& A1 = (ddt >= 0.0) ? X : C;
        if (ddt < 0.0) ddt = 1.0 + ddt;
        if (has_lo)
            tl_lo = tl_lo + A0.atten[(size_t)lane * q.n + i] * (1.0 - ddt) +
                    A1.atten[(size_t)lane * q.n + i] * ddt;
        if (has_hi)
            tl_hi = tl_hi + A0.atten[(size_t)(lane + 32) * q.n + i] * (1.0 - ddt) +
                    A1.atten[(size_t)(lane + 32) * q.n + i] * ddt;
        const bool above = (has_lo && tl_lo < q.intensity_threshold) ||
                           (has_hi && tl_hi < q.intensity_threshold);
        if (!__any_sync(0xffffffffu, above)) continue;

        /* direction angles of the 27 neighbours on three fronts
         * (wvector1::direction, types/wvector1.cc) */
        if (lane < 27) {
            const int m = lane / 9, nd_ = (lane / 3) % 3, na = lane % 3;
            const int j = (de0 + nd_ - 1) * q.naz + wrap_az(q, az0, na);
            const FrontPtrs& F = (m == 0) ? V : (m == 1) ? C : X;
            const double n0 = F.nd[0][j], n1 = F.nd[1][j], n2 = F.nd[2][j];
            s_ang[warp][0][lane] = atan2(n0, sqrt(n1 * n1 + n2 * n2)) * (180.0 / M_PI);
            s_ang[warp][1][lane] = atan2(n2, -n1) * (180.0 / M_PI);
        }
        __syncwarp();
        double tang[2];
        for (int which = 0; which < 2; ++which) {
            double center, g[3], h[3][3], hv[3];
            make_taylor_coeff(reinterpret_cast<double (*)[3][3]>(s_ang[warp][which]), delta, center, g, h);
            matvec(h, offset, hv);
            tang[which] = center + dot3(g, offset) + 0.5 * dot3(offset, hv);
        }
        uint32_t slot = 0;
        if (lane == 0) slot = atomicAdd(q.n_rec, 1u);
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (slot >= q.cap_rec) {
            if (lane == 0) set_err(q, ERR_REC_OVERFLOW);
            __syncwarp();
            continue;
        }
        if (lane == 0) {
            wq3d_eigenray r;
            r.time = time + offset[0];
            r.source_de = q.de[de0] + offset[1];
            r.source_az = q.az[az0] + offset[2];
            r.target_de = tang[0];
            r.target_az = tang[1];
            r.surface = C.surface[i];
            r.bottom = C.bottom[i];
            r.caustic = C.caustic[i];
            r.upper = C.upper[i];
            r.lower = C.lower[i];
            r.t1 = t / q.nt2;
            r.t2 = t % q.nt2;
            r.de = de0;
            r.az = az0;
            r.pad = 0;
            r.step = s;
            q.rec[slot] = r;
        }
        if (q.sens && lane < 3)
            q.rec_sens[(size_t)slot * 3 + lane] = A0.dA[(size_t)lane * q.n + i] * (1.0 - ddt) +
                                                  A1.dA[(size_t)lane * q.n + i] * ddt;
        if (has_lo) {
            q.rec_inten[(size_t)slot * q.nf + lane] = tl_lo;
            q.rec_phase[(size_t)slot * q.nf + lane] = C.phase[(size_t)lane * q.n + i];
        }
        if (has_hi) {
            q.rec_inten[(size_t)slot * q.nf + lane + 32] = tl_hi;
            q.rec_phase[(size_t)slot * q.nf + lane + 32] = C.phase[(size_t)(lane + 32) * q.n + i];
        }
        __syncwarp();
    }
}

/* ------------------------------------------------------------------ */
/* single-point model evaluations (ocean parity tests)                 */
/* ------------------------------------------------------------------ */
__global__ void k_sound_speed(OceanDev oc, double R, int n, const double* rho,
                              const double* theta, const double* phi, double* c,
                              double* g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double cc, gg[3];
    sound_speed(oc.prof, R, rho[i], theta[i], phi[i], &cc, gg);
    c[i] = cc;
    if (g) {
        g[i] = gg[0];
        g[n + i] = gg[1];
        g[2 * n + i] = gg[2];
    }
}

__global__ void k_height(BoundaryDev b, int n, const double* theta, const double* phi,
                         double* h, double* nrm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double nn[3];
    h[i] = boundary_height_normal(b, theta[i], phi[i], nn);
    if (nrm) {
        nrm[i] = nn[0];
        nrm[n + i] = nn[1];
        nrm[2 * n + i] = nn[2];
    }
}

/* attenuation_thorp.cc:29-35 with the per-frequency alpha precomputed on
 * the host, or attenuation_constant.cc:14-25 */
__global__ void k_attenuation(ProfileDev pr, double R, int n, const double* rho,
                              const double* dist, int nf, const double* freq,
                              const double* alpha, double* atten) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double alt = rho[i] - R;
    for (int f = 0; f < nf; ++f) {
        atten[(size_t)i * nf + f] = (pr.atten == WQ3D_ATTEN_CONSTANT)
                                        ? pr.atten_coef * dist[i] * freq[f]
                                        : dist[i] * alpha[f] * (1.0 + 5.88264e-6 * alt);
    }
}

__global__ void k_reflect_loss(BoundaryDev b, int n, const double* grazing, int nf,
                               const double* freq, double* amp, double* ph) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const LossDev& L = b.loss;
    double a0 = 0.0, p0 = 0.0;
    if (L.kind != WQ3D_LOSS_ECKART) reflect_loss_scalar(L, grazing[i], &a0, &p0);
    const double w2 = L.p[0] * L.p[0];
    const double sg = sin(grazing[i]);
    for (int f = 0; f < nf; ++f) {
        double a = a0, p = p0;
        if (L.kind == WQ3D_LOSS_ECKART) {
            const double x = freq[f] * w2 * sg;
            a = 8.6e-9 * (x * x);
            p = M_PI;
        }
        amp[(size_t)i * nf + f] = a;
        if (ph) ph[(size_t)i * nf + f] = p;
    }
}

#endif  // !WQ3D_STEP_KERNELS_ONLY

}  // namespace wq3d

#if WQ3D_WITH_GRID && !WQ3D_STEP_KERNELS_ONLY
/* the adjoint's kernels reuse the step functions above */
#define WQ3D_ADJOINT_IMPL 1
#include "wq3d_adjoint.cuh"
#endif
