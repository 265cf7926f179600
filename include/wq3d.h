/*
 * wq3d.h -- C ABI of the B200-native WaveQ3D wavefront propagation engine.
 *
 * This is the drop-in boundary for USML's WaveQ3D propagator.  Every entry
 * point below replaces one piece of the reference C++ interface; the
 * reference location is cited beside each declaration (paths are relative
 * to the USML source tree).  The ABI uses only plain C types: no C++
 * exceptions, no torch types and no CUDA types cross it.  Every function
 * returns an int status: WQ3D_OK (0) on success, a negative WQ3D_ERR_* code
 * otherwise; wq3d_last_error_string() then describes the failure.
 *
 * Coordinates follow USML's spherical earth system (types/wposition.h):
 *   rho   = distance from the earth's centre (m),
 *   theta = colatitude (rad),  phi = longitude (rad).
 * Ray fan angles are in degrees (D/E positive up, AZ clockwise from north),
 * exactly as the reference seq_vector fans hold them.
 *
 * Device memory is owned by the library.  Host arrays passed in are copied
 * during the call; the caller keeps ownership of them.  An ocean lives on
 * the device that was current when it was created; evaluating it with
 * another device current, or building a queue for another device from it,
 * returns WQ3D_ERR_INVALID.
 *
 * The library keeps per-device state between calls (the staging array's
 * address of wq3d_ocean_sound_speed_noalloc, the bistatic eigenverb
 * workspace).  cudaDeviceReset destroys the device objects behind that
 * state: do not call into the library after a cudaDeviceReset in the same
 * process.
 */
#ifndef WQ3D_H
#define WQ3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WQ3D_ABI_VERSION 1

/* ------------------------------------------------------------------ */
/* status codes                                                        */
/* ------------------------------------------------------------------ */
enum {
    WQ3D_OK = 0,
    WQ3D_ERR_INVALID = -1,     /* bad argument (reference: std::invalid_argument) */
    WQ3D_ERR_CUDA = -2,        /* CUDA runtime failure or no device          */
    WQ3D_ERR_NOMEM = -3,       /* device or host allocation failed            */
    WQ3D_ERR_OVERFLOW = -4,    /* a result buffer was too small               */
    WQ3D_ERR_TIMEOUT = -5,     /* a bounded device wait gave up               */
    WQ3D_ERR_UNSUPPORTED = -6, /* option not built into this library          */
    WQ3D_ERR_NUMERIC = -7,     /* a kernel's own bounds/iteration check fired */
    WQ3D_ERR_ABORTED = -8      /* caller's cancellation flag was set          */
};

/* ------------------------------------------------------------------ */
/* ocean description (replaces ocean/ocean_model.h:31-124)             */
/* ------------------------------------------------------------------ */

/* sound speed profiles: ocean/profile_{linear,munk,catenary,n2,grid}.h */
enum {
    WQ3D_PROFILE_LINEAR = 0,   /* p = {c0, g0, z1, g1}      profile_linear.cc:14-40   */
    WQ3D_PROFILE_MUNK = 1,     /* p = {axis_depth, scale, axis_speed, epsilon}
                                                          profile_munk.cc:19-32     */
    WQ3D_PROFILE_CATENARY = 2, /* p = {c1, g1, z1}        profile_catenary.cc:14-29 */
    WQ3D_PROFILE_N2 = 3,       /* p = {c0, g0}            profile_n2.cc:14-24       */
    WQ3D_PROFILE_GRID = 4      /* gen_grid over (rho[,theta[,phi]])  profile_grid.h:68-130 */
};

/* attenuation models: ocean/attenuation_{thorp,constant}.cc */
enum {
    WQ3D_ATTEN_THORP = 0,      /* default of profile_model (profile_model.h:40-47) */
    WQ3D_ATTEN_CONSTANT = 1    /* coef * distance * frequency                      */
};

/* boundary height models: ocean/boundary_{flat,slope,grid}.h */
enum {
    WQ3D_BOUNDARY_FLAT = 0,    /* boundary_flat.cc:19-63  */
    WQ3D_BOUNDARY_SLOPE = 1,   /* boundary_slope.cc:13-68 */
    WQ3D_BOUNDARY_GRID = 2     /* boundary_grid.h:88-196  */
};

/* reflection loss models: ocean/reflect_loss_{constant,rayleigh,eckart}.h */
enum {
    WQ3D_LOSS_DEFAULT = -1,    /* the boundary's own default (boundary_model.h:77-90,
                                  boundary_flat.cc:19-31)                           */
    WQ3D_LOSS_CONSTANT = 0,    /* p = {amplitude_dB, phase_rad}                     */
    WQ3D_LOSS_RAYLEIGH = 1,    /* p = {density, speed, att_bottom, speed_shear, att_shear}
                                  (ratios to water, dB/wavelength)
                                  reflect_loss_rayleigh.cc:68-144                   */
    WQ3D_LOSS_ECKART = 2       /* p = {wind_speed}        reflect_loss_eckart.h:76-85 */
};

/* interpolation per grid axis (types/data_grid.h interp_enum) */
enum {
    WQ3D_INTERP_NEAREST = -1,
    WQ3D_INTERP_LINEAR = 0,
    WQ3D_INTERP_PCHIP = 1
};

/* N-dimensional rectilinear grid (types/gen_grid.h:83-520).  Data is
 * row-major with the last axis fastest (types/data_grid.h:47-61). */
/* sequence kinds of a grid axis; they differ in find_index
 * (types/seq_linear.h:89-94, seq_log.h:88-94, seq_data.cc:15-36) */
enum { WQ3D_AXIS_LINEAR = 0, WQ3D_AXIS_LOG = 1, WQ3D_AXIS_DATA = 2 };

typedef struct wq3d_grid_desc {
    int ndim;                  /* 0 = unused, else 1..3 */
    const double* axis[3];     /* axis values, monotonic, at least 2 each */
    const double* axis_inc[3]; /* seq_vector::increment(i) of each axis */
    size_t axis_size[3];
    int axis_kind[3];          /* WQ3D_AXIS_* */
    const double* data;        /* prod(axis_size) values */
    int interp[3];             /* WQ3D_INTERP_* per axis */
    int edge_limit[3];         /* nonzero: clamp outside the axis range */
} wq3d_grid_desc;

typedef struct wq3d_profile_desc {
    int kind;                  /* WQ3D_PROFILE_* */
    double p[4];
    int flat_earth;            /* profile_model::flat_earth() (profile_model.cc:14-26) */
    int attenuation;           /* WQ3D_ATTEN_* */
    double attenuation_coef;   /* WQ3D_ATTEN_CONSTANT coefficient */
    wq3d_grid_desc grid;       /* WQ3D_PROFILE_GRID sound speed (m/s) */
} wq3d_profile_desc;

typedef struct wq3d_reflect_loss_desc {
    int kind;                  /* WQ3D_LOSS_* */
    double p[5];
} wq3d_reflect_loss_desc;

typedef struct wq3d_boundary_desc {
    int kind;                  /* WQ3D_BOUNDARY_* */
    double depth;              /* flat: depth (m, 0 = ocean surface); slope: depth
                                  at the reference location */
    double location[3];        /* slope: reference location (rho, theta, phi) */
    double lat_slope;          /* slope: radians */
    double lng_slope;          /* slope: radians */
    wq3d_grid_desc grid;       /* grid: boundary rho over (theta[, phi]) */
    wq3d_reflect_loss_desc loss;
} wq3d_boundary_desc;

/* Volume scattering layers an ocean may hold (ocean_model::add_volume,
 * ocean/ocean_model.h:49-52). */
#define WQ3D_MAX_VOLUME 4

/* A flat volume scattering layer (ocean/volume_flat.h:32-90).  The
 * propagator only needs its depth; thickness and the constant scattering
 * strength are kept for the caller's reverberation model. */
typedef struct wq3d_volume_desc {
    double depth;              /* m below mean sea level (abs taken)      */
    double thickness;          /* m                                       */
    double amplitude;          /* scattering strength, dB                 */
} wq3d_volume_desc;

typedef struct wq3d_ocean_desc {
    /* value of wposition::earth_radius when the boundaries were built; the
     * reference bakes it into boundary heights at construction time
     * (boundary_flat.cc:19-21, boundary_slope.cc:13-20) */
    double earth_radius;
    wq3d_profile_desc profile;
    wq3d_boundary_desc surface;
    wq3d_boundary_desc bottom;
    int num_volume;            /* 0..WQ3D_MAX_VOLUME layers               */
    wq3d_volume_desc volume[WQ3D_MAX_VOLUME];
} wq3d_ocean_desc;

typedef struct wq3d_ocean wq3d_ocean;

/* Builds a device-resident ocean.  Replaces ocean_model::ocean_model
 * (ocean/ocean_model.h:31-60) together with the profile/boundary ctors. */
int wq3d_ocean_create(const wq3d_ocean_desc* desc, wq3d_ocean** out);
int wq3d_ocean_destroy(wq3d_ocean* ocean);

/* Evaluates the sound speed profile at n points on the GPU.  Replaces
 * profile_model::sound_speed (ocean/profile_model.h:71-72).  grad may be
 * NULL, else it receives 3*n values (rho, theta, phi blocks). */
int wq3d_ocean_sound_speed(const wq3d_ocean* ocean, double earth_radius,
                           size_t n, const double* rho, const double* theta,
                           const double* phi, double* speed, double* grad);

/* Evaluates a boundary height and normal at n points on the GPU.
 * which = 0 surface, 1 bottom.  Replaces boundary_model::height
 * (ocean/boundary_model.h:109-121).  normal may be NULL (else 3*n). */
int wq3d_ocean_height(const wq3d_ocean* ocean, int which, size_t n,
                      const double* rho, const double* theta,
                      const double* phi, double* height, double* normal);

/* Evaluates a boundary's reflection loss at n grazing angles for nf
 * frequencies on the GPU.  Replaces boundary_model::reflect_loss
 * (ocean/boundary_model.h:144-150).  amplitude and phase hold n*nf values. */
int wq3d_ocean_reflect_loss(const wq3d_ocean* ocean, int which, size_t n,
                            const double* rho, const double* theta,
                            const double* phi, const double* grazing,
                            size_t nf, const double* freq, double* amplitude,
                            double* phase);

/* Evaluates the profile's sea-water absorption (dB) over the distance
 * travelled at n points for nf frequencies on the GPU: Thorp
 * (ocean/attenuation_thorp.cc:14-36) or constant
 * (ocean/attenuation_constant.cc:14-25).  Replaces
 * attenuation_model::attenuation (ocean/attenuation_model.h:45-48).
 * attenuation holds n*nf values, point-major. */
int wq3d_ocean_attenuation(const wq3d_ocean* ocean, double earth_radius, size_t n,
                           const double* rho, const double* distance, size_t nf,
                           const double* freq, double* attenuation);

/* Largest number of points one wq3d_ocean_sound_speed_noalloc call takes. */
#define WQ3D_NOALLOC_MAX_POINTS 16384

/* Same evaluation as wq3d_ocean_sound_speed, for callers that cannot
 * allocate device memory when they need it (for example a processing loop
 * that reserves its GPU memory up front, or code under a real-time budget
 * where cudaMalloc's latency and synchronisation are not allowed).  It has
 * no counterpart in the reference.  The points are staged in one fixed
 * device array built into the library (7 doubles per point, 0.9 MB per
 * device, kept until the process exits); nothing is allocated or freed.
 * n above WQ3D_NOALLOC_MAX_POINTS returns WQ3D_ERR_INVALID.  All calls on a
 * device share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  The first call on a device looks up the
 * array's address with that device current; make it before any CUDA stream
 * capture starts. */
int wq3d_ocean_sound_speed_noalloc(const wq3d_ocean* ocean, double earth_radius,
                                   size_t n, const double* rho,
                                   const double* theta, const double* phi,
                                   double* speed, double* grad);

/* ------------------------------------------------------------------ */
/* wave queue (replaces waveq3d/wave_queue.h:122-264)                  */
/* ------------------------------------------------------------------ */

enum { WQ3D_CLASSIC_RAY = 0, WQ3D_HYBRID_GAUSSIAN = 1 }; /* wave_queue.h:90 */
/* Arithmetic form.  WQ3D_FP64: the reference's FP64 arithmetic throughout.
 * WQ3D_FP32C: the same, with the CPA search's comparisons screened in FP32
 * and finished in FP64 where the screen cannot decide (the eigenrays equal
 * the FP64 form's bit for bit).  WQ3D_FP32: additionally the sound speed,
 * its gradient and the ray derivatives of every wave_front::update
 * (wave_front.cc:125-178) in FP32, at the altitude offset rho - R, while
 * positions, directions, travel time, the distance terms and the CPA
 * Taylor fit stay FP64; its error against the FP64 form is measured, not
 * zero.  The adjoint is refused for WQ3D_FP32. */
enum { WQ3D_FP64 = 0, WQ3D_FP32C = 1, WQ3D_FP32 = 2 };

typedef struct wq3d_queue_desc {
    const double* freq;        /* frequencies (Hz), seq_vector freq       */
    size_t num_freq;
    double source[3];          /* rho, theta, phi of the source (wposition1) */
    const double* de;          /* D/E fan values (deg), seq_vector de     */
    const double* de_inc;      /* seq_vector::increment(i) for each i     */
    size_t num_de;
    const double* az;          /* AZ fan values (deg)                     */
    const double* az_inc;
    size_t num_az;
    double time_step;          /* seconds                                 */
    const double* targets;     /* 3*num_targets1*num_targets2 doubles: all rho,
                                  then all theta, then all phi (row-major
                                  t1,t2), or NULL for no eigenrays        */
    size_t num_targets1;
    size_t num_targets2;
    int spreading;             /* WQ3D_CLASSIC_RAY or WQ3D_HYBRID_GAUSSIAN */
    int precision;             /* WQ3D_FP64, WQ3D_FP32C or WQ3D_FP32       */
    double earth_radius;       /* wposition::earth_radius while propagating */
    size_t eigenray_capacity;  /* device records kept per step chunk; 0 = default */
    int device;                /* CUDA device ordinal                     */
    uint64_t run_id;           /* wave_queue::runID                       */
} wq3d_queue_desc;

typedef struct wq3d_thresholds {   /* waveq3d/wave_thresholds.h:38-199 */
    double intensity;          /* dB, stored as abs() like the reference  */
    double eigenverb;          /* dB, stored as abs()                     */
    int max_bottom;
    int max_surface;
    int max_caustic;
    int max_upper;
    int max_lower;
} wq3d_thresholds;

/* One acoustic path (eigenrays/eigenray_model.h:24-102) plus the CPA
 * bracket (step, de, az) that found it, which the reference does not
 * record.  intensity[] and phase[] (num_freq values each) travel beside it. */
typedef struct wq3d_eigenray {
    double time;
    double source_de;
    double source_az;
    double target_de;
    double target_az;
    int32_t surface;
    int32_t bottom;
    int32_t caustic;
    int32_t upper;
    int32_t lower;
    int32_t t1;
    int32_t t2;
    int32_t de;
    int32_t az;
    int32_t pad;
    int64_t step;
} wq3d_eigenray;

/* One boundary collision (waveq3d/reflection_listener.h:46-49). */
typedef struct wq3d_reflection {
    double time;
    double dt;
    double grazing;
    double speed;
    double position[3];        /* rho, theta, phi */
    double ndirection[3];
    int32_t de;
    int32_t az;
    int32_t type;              /* 0 bottom, 1 surface (eigenverb_model.h:42-47) */
    int32_t pad;
    int64_t step;
} wq3d_reflection;

/* Interfaces an eigenverb can come from (eigenverbs/eigenverb_model.h:27-32):
 * volume layer k gives 2 + 2k (upper side) and 3 + 2k (lower side). */
enum { WQ3D_VERB_BOTTOM = 0, WQ3D_VERB_SURFACE = 1, WQ3D_VERB_VOLUME_UPPER = 2,
       WQ3D_VERB_VOLUME_LOWER = 3 };

/* One eigenverb (eigenverbs/eigenverb_model.h:34-150): a Gaussian beam's
 * footprint at a boundary or volume layer collision, built by
 * wave_queue::build_eigenverb (wave_queue.cc:1063-1164).  power[]
 * (num_freq linear values) travels beside it; frequencies are the queue's. */
typedef struct wq3d_eigenverb {
    double travel_time;        /* s                                        */
    double length;             /* half-length along the beam, m            */
    double width;              /* half-width across the beam, m            */
    double position[3];        /* rho, theta, phi of the collision         */
    double direction;          /* rad, clockwise from true north            */
    double grazing;            /* rad                                      */
    double sound_speed;        /* m/s at the collision                     */
    double source_de;          /* rad                                      */
    double source_az;          /* rad                                      */
    int32_t de;                /* de_index                                 */
    int32_t az;                /* az_index                                 */
    int32_t surface;
    int32_t bottom;
    int32_t caustic;
    int32_t upper;
    int32_t lower;
    int32_t interface_num;     /* WQ3D_VERB_*                               */
    int64_t step;              /* the wave_queue::step that produced it     */
    int32_t seq;               /* order of the ray's events in that step   */
    int32_t pad;
} wq3d_eigenverb;

/* Listener callbacks, invoked on the calling thread inside wq3d_queue_step
 * in reference order: for every completed step, add_eigenray for each path
 * in (t1, t2, de, az) order (wave_queue.cc:361-373) and then one
 * check_eigenrays (wave_queue.cc:191).  Replaces eigenray_listener
 * (eigenrays/eigenray_listener.h:41-53) and reflection_listener. */
typedef struct wq3d_callbacks {
    void (*add_eigenray)(void* ctx, size_t t1, size_t t2,
                         const wq3d_eigenray* ray, const double* intensity,
                         const double* phase, size_t num_freq,
                         uint64_t run_id);
    void (*check_eigenrays)(void* ctx, double time, uint64_t run_id);
    void (*reflect)(void* ctx, const wq3d_reflection* reflection);
    /* eigenverb_listener::add_eigenverb (eigenverbs/eigenverb_listener.h:40-41);
     * for every completed step, in the order the reference's
     * detect_reflections loop makes them (de, az, then the ray's events),
     * before that step's add_eigenray calls */
    void (*add_eigenverb)(void* ctx, const wq3d_eigenverb* verb,
                          const double* power, size_t num_freq,
                          int interface_num);
} wq3d_callbacks;

/* Host copy of one wavefront (waveq3d/wave_front.h:152-258).  Every pointer
 * is optional (NULL = skip); arrays are num_de*num_az, row-major (de, az),
 * attenuation/phase are num_de*num_az*num_freq with frequency fastest. */
typedef struct wq3d_front_view {
    double* rho;
    double* theta;
    double* phi;
    double* pos_grad[3];
    double* ndir[3];
    double* ndir_grad[3];
    double* sound_speed;
    double* sound_grad[3];
    double* distance;
    double* path_length;
    double* attenuation;
    double* phase;
    int32_t* surface;
    int32_t* bottom;
    int32_t* caustic;
    int32_t* upper;
    int32_t* lower;
    uint8_t* on_edge;
} wq3d_front_view;

enum { WQ3D_FRONT_PAST = 0, WQ3D_FRONT_PREV = 1, WQ3D_FRONT_CURR = 2,
       WQ3D_FRONT_NEXT = 3 };                /* wave_queue.h:179-216 */

typedef struct wq3d_queue wq3d_queue;

/* Builds the queue and runs the RK3 start-up on the GPU.  Replaces
 * wave_queue::wave_queue (wave_queue.h:122-126, wave_queue.cc:30-98),
 * including the 0.1 m source clamp (wave_queue.cc:58-68). */
int wq3d_queue_create(const wq3d_ocean* ocean, const wq3d_queue_desc* desc,
                      wq3d_queue** out);
int wq3d_queue_destroy(wq3d_queue* q);

/* Cache of destroyed queues.  wq3d_queue_destroy keeps up to max_queues
 * queues (2 by default; the oldest is freed first) whose buffers still have
 * their creation sizes (no eigenverb listener, reflection buffer not grown,
 * no sensitivity or adjoint mode), and wq3d_queue_create re-initialises one
 * of the same device, fan, frequency, target and eigenray-capacity shape
 * instead of allocating: a create-run-destroy loop then allocates and
 * instantiates its graphs once.  Results are those of a fresh queue.
 * max_queues = 0 frees the cached queues and turns the cache off.  The
 * reference has no counterpart (each wave_queue owns its fronts). */
int wq3d_set_queue_cache(size_t max_queues);

/* Sensitivity mode (call before the first step): every eigenray also
 * carries the exact derivatives of its transmission loss (dB, the same at
 * every frequency) with respect to the bottom's Rayleigh parameters --
 * density ratio, speed ratio and attenuation in dB per wavelength
 * (reflect_loss_rayleigh.cc:68-78) -- carried along each ray as the
 * derivative of its accumulated reflection loss.  The ray geometry does not
 * depend on these parameters, so this is the derivative of the whole
 * propagation.  No reference counterpart: the reference has no
 * differentiation. */
int wq3d_queue_enable_sensitivity(wq3d_queue* q);

/* Adjoint recording (call before the first step): while the queue runs,
 * every ray's state is kept every checkpoint_interval steps (max_steps
 * bounds the run) and every eigenray record (at most max_eigenrays; 0 for
 * 65536) gets the partial derivatives of its first-frequency TL and its
 * travel time with respect to the fronts it was built from.
 * wq3d_queue_adjoint then runs the reverse sweep.  Supported oceans: a
 * profile_grid<1> linear in depth (its nodes, at most 64 and more than a
 * step's reach apart, are the parameters), flat or sloped boundaries with
 * constant, fluid Rayleigh (no shear) or Eckart loss, no volume layers;
 * hybrid Gaussian spreading; targets required.  Other oceans return
 * WQ3D_ERR_UNSUPPORTED.  No reference counterpart: the reference has no
 * differentiation. */
int wq3d_queue_enable_adjoint(wq3d_queue* q, int checkpoint_interval, size_t max_steps,
                              size_t max_eigenrays);

/* The reverse sweep at the forward pass's eigenray topology.  For weights
 * w_tl[k] and w_time[k] of the eigenrays rays[k] (records as
 * wq3d_queue_take_eigenrays returned them), grad[j] receives
 *   sum_k w_tl[k] dTL_k / dc_j + w_time[k] dT_k / dc_j
 * for the num_nodes nodes c_j of the profile grid (TL of the first
 * frequency, dB; travel time, s; c_j in m/s).  From each checkpoint, last
 * first, the states of the rays that reach a weighted eigenray are
 * recomputed, the eigenrays' partials are taken to them, and the sweep runs
 * back to the previous checkpoint; the start-up (init_wave and the RK3
 * start, wave_queue.cc:114-150) closes it.  ms (may be NULL) receives the
 * sweep's device time.  A record the forward did not see returns
 * WQ3D_ERR_INVALID; an eigenray whose beam walk outran the recorded cells,
 * or a step that reached nodes beyond its window, returns
 * WQ3D_ERR_NUMERIC.  No reference counterpart. */
int wq3d_queue_adjoint(wq3d_queue* q, const wq3d_eigenray* rays, const double* w_tl,
                       const double* w_time, size_t n, double* grad, size_t num_nodes, double* ms);

/* The reverse sweep for one ray's state instead of eigenrays: grad[j]
 * receives d x / d c_j for component `component` of ray `ray`'s state
 * after step `step` (0-17: position rho, theta, phi then normalised
 * direction of the prev, curr and next fronts as that step's eigenray
 * search reads them; 18-20: their first-frequency attenuation).  Checks
 * the sweep's propagation part against differences of the fronts
 * (wq3d_queue_get_front).  No reference counterpart. */
int wq3d_queue_adjoint_state(wq3d_queue* q, int ray, int64_t step, int component, double* grad,
                             size_t num_nodes);

/* Eigenverb counting sink: with on != 0 the queue builds eigenverbs as
 * for an eigenverb listener (wave_queue.cc:1063-1164), reads them back per
 * chunk and counts them per interface instead of calling add_eigenverb;
 * counts (2 + 2 * WQ3D_MAX_VOLUME entries, indexed by interface number)
 * accumulate until the queue is destroyed.  For callers that measure or
 * subsample the eigenverb stream without a callback per eigenverb.  No
 * reference counterpart (the reference always calls its listeners). */
int wq3d_queue_count_eigenverbs(wq3d_queue* q, int on);
int wq3d_queue_eigenverb_counts(const wq3d_queue* q, uint64_t* counts);

/* eigenray_collection::sum_eigenrays (eigenrays/eigenray_collection.cc:
 * 105-191) on the GPU: for every target of a num_targets1 x num_targets2
 * grid, the coherent (or, with coherent = 0, incoherent) phasor sum of its
 * eigenrays per frequency, and their power-weighted travel time, D/E
 * angles and AZ angles; the counts are the strongest path's.  rays[k]
 * (intensity and phase: n x nf, frequency fastest) names its target in
 * t1, t2; a target's eigenrays are summed in the order they appear, as the
 * reference's per-target lists hold them.  total (num_targets1 x
 * num_targets2 records, de, az and step set to -1), total_intensity and
 * total_phase (targets x nf) receive the sums; a target without eigenrays
 * gets 300 dB, NaN time and angles, and counts of -1, as in the
 * reference. */
int wq3d_sum_eigenrays(const wq3d_eigenray* rays, const double* intensity, const double* phase,
                       size_t n, const double* freq, size_t nf, size_t num_targets1,
                       size_t num_targets2, int coherent, wq3d_eigenray* total,
                       double* total_intensity, double* total_phase);

/* The three derivatives of each eigenray that wq3d_queue_take_eigenrays
 * would return next, in the same order (3 values per eigenray; NaN when
 * sensitivity mode is off).  Does not consume the eigenrays. */
int wq3d_queue_sensitivities(const wq3d_queue* q, double* sens, size_t capacity, size_t* count);

/* Replaces the wave_thresholds setters (wave_thresholds.h:54-182). */
int wq3d_queue_set_thresholds(wq3d_queue* q, const wq3d_thresholds* t);

/* Replaces add/remove_*_listener (eigenray_notifier.h:41-70,
 * reflection_notifier.h).  NULL callbacks = no listeners. */
int wq3d_queue_set_callbacks(wq3d_queue* q, const wq3d_callbacks* cb,
                             void* ctx);

/* Advances nsteps calls of wave_queue::step() (wave_queue.cc:155-192).
 * Callbacks fire before it returns. */
int wq3d_queue_step(wq3d_queue* q, size_t nsteps);

/* Advances while time() < time_max, the loop every reference caller uses
 * (wavegen/wavefront_generator.cc:98-112).  *steps_done may be NULL. */
int wq3d_queue_run(wq3d_queue* q, double time_max, size_t* steps_done);

/* Runs count independent queues, each until its time() reaches
 * time_max[i] (the reference loop of wq3d_queue_run), concurrently on one
 * GPU: every queue's next chunk of steps is launched before any is drained,
 * so the host delivers one queue's results while the others compute.  It
 * replaces the reference's thread pool of wavefront_generator tasks, one
 * wave_queue each (wavegen/wavefront_generator.cc:52-127,
 * threads/thread_pool.cc:21-56).  Listener callbacks arrive on the calling
 * thread, per queue in reference order.  steps_done (count values) and
 * ms_device (device time from the batch's start to the last queue's end)
 * may be NULL.  All queues must be on one device. */
int wq3d_batch_run(wq3d_queue* const* queues, size_t count, const double* time_max,
                   size_t* steps_done, double* ms_device);

/* Read-only state: wave_queue::time(), source_pos(), num_de/az. */
int wq3d_queue_time(const wq3d_queue* q, double* time);
int wq3d_queue_source(const wq3d_queue* q, double* rho_theta_phi);
int wq3d_queue_steps(const wq3d_queue* q, int64_t* steps);

/* Copies one front (wave_queue::curr()/next()/prev()/past()) to the host. */
int wq3d_queue_get_front(wq3d_queue* q, int which,
                         const wq3d_front_view* view);

/* Eigenrays found so far and not yet taken, in reference order.  With
 * rays == NULL only *count is returned.  Taken records are removed. */
int wq3d_queue_take_eigenrays(wq3d_queue* q, wq3d_eigenray* rays,
                              double* intensity, double* phase,
                              size_t capacity, size_t* count);

/* Cooperative cancellation, polled between step chunks
 * (thread_task::abort, wavegen/wavefront_generator.cc:55-58,100-108). */
int wq3d_queue_abort(wq3d_queue* q);

/* Device time (ms, CUDA events) accumulated since the last reset. */
typedef struct wq3d_timing {
    double ms_total;     /* whole wq3d_queue_step/run calls on the queue's
                            stream, host result handling between chunks
                            included                                    */
    double ms_advance;   /* k_advance (and k_volume), timing mode only  */
    double ms_reflect;   /* k_reflect on its side stream, timing mode only */
    double ms_cpa;       /* k_cpa / k_cpa_f32, timing mode only          */
    double ms_eigenray;  /* k_eigenray, timing mode only                 */
    int64_t launches;    /* kernel launches                              */
} wq3d_timing;

/* Reads (and optionally resets) the timing counters.  No reference
 * counterpart: benchmarking aid. */
int wq3d_queue_timing(wq3d_queue* q, wq3d_timing* out, int reset);

/* Turns per-kernel CUDA-event timing on (direct launches, events around
 * every kernel) or off (chunks replayed as one CUDA graph, the default).
 * No reference counterpart: benchmarking aid. */
int wq3d_queue_set_timing(wq3d_queue* q, int on);

/* Where the reflections of a step run (results are identical bit for bit):
 *   WQ3D_REFLECT_SIDE    k_reflect, a separate launch on a high-priority
 *                        stream over a compact list of the reflecting rays;
 *                        the next step's advance waits for it.  Best when
 *                        the fan fills the GPU: reflecting rays take few
 *                        blocks.
 *   WQ3D_REFLECT_INLINE  the advance of step s reflects step s+1's rays as
 *                        soon as it has written their next front, so a step
 *                        costs the longer of the advance and the longest
 *                        reflection chain instead of their sum.  Best for
 *                        small fans, whose steps are bound by that chain.
 *                        (Eigenverb listeners and volume layers always use
 *                        the side stream.)
 *   WQ3D_REFLECT_AUTO    (default) a queue run alone follows a plan per
 *                        queue shape and per 128-step bucket of the run
 *                        (which schedule wins changes as the fan spreads):
 *                        the first queue of a shape tries both schedules
 *                        on one chunk of each bucket, every later chunk and
 *                        queue of that shape takes the faster.  Queues run
 *                        by wq3d_batch_run and queues recording for the
 *                        adjoint use the side stream.
 * No reference counterpart (the reference reflects inside its step). */
enum { WQ3D_REFLECT_AUTO = 0, WQ3D_REFLECT_SIDE = 1, WQ3D_REFLECT_INLINE = 2 };
int wq3d_queue_set_reflect_schedule(wq3d_queue* q, int schedule);

/* The schedule of the queue's last chunk (WQ3D_REFLECT_SIDE or
 * WQ3D_REFLECT_INLINE), the one set, or WQ3D_REFLECT_AUTO before any run
 * under the tuned schedule. */
int wq3d_queue_reflect_schedule(const wq3d_queue* q, int* schedule);

/* ------------------------------------------------------------------ */
/* bistatic eigenverbs (biverbs/)                                      */
/* ------------------------------------------------------------------ */

/* Scattering strength models of one interface
 * (ocean/scattering_{constant,lambert,chapman}.h), chosen per interface the
 * way ocean_model::scattering does (ocean/ocean_model.h:88-112). */
enum {
    WQ3D_SCATTER_CONSTANT = 0, /* p = strength in dB (scattering_constant.h) */
    WQ3D_SCATTER_LAMBERT = 1,  /* p = bss in dB: 10^(bss/10) |sin a sin b|
                                  (scattering_lambert.h)                  */
    WQ3D_SCATTER_CHAPMAN = 2   /* p = wind speed, m/s (scattering_chapman.h) */
};
typedef struct wq3d_scattering_desc {
    int32_t kind;
    int32_t pad;
    double p;
} wq3d_scattering_desc;

/* One bistatic eigenverb (biverbs/biverb_model.h): the overlap of a
 * source eigenverb and a receiver eigenverb on one interface.  The power
 * for each frequency is returned beside it. */
typedef struct wq3d_biverb {
    double travel_time;        /* source + receiver travel time, s        */
    double duration;           /* s                                       */
    double source_de;          /* rad                                     */
    double source_az;
    double receiver_de;
    double receiver_az;
    int32_t de_index;          /* the receiver eigenverb's                */
    int32_t az_index;
    int32_t source_surface, source_bottom, source_caustic, source_upper, source_lower;
    int32_t receiver_surface, receiver_bottom, receiver_caustic, receiver_upper, receiver_lower;
    int32_t source;            /* index of the source eigenverb           */
    int32_t receiver;          /* index of the receiver eigenverb         */
} wq3d_biverb;

/* The biverbs of one interface (biverb_generator::run,
 * biverbs/biverb_generator.cc:50-72, with biverb_collection::add_biverb,
 * biverbs/biverb_collection.cc:44-172).  For every receiver eigenverb, the
 * source eigenverbs whose centres lie strictly inside its search
 * quadrilateral (eigenverb_collection::find_eigenverbs,
 * eigenverbs/eigenverb_collection.cc:60-93, corners search_scale x length
 * and width away) are overlapped with it; pairs whose largest power over
 * frequency is below power_threshold are dropped.  Results come back in
 * (receiver, source) index order, at most `capacity` of them; *count is the
 * number that exist (with out == NULL only *count is computed).  Arrays are
 * host memory: src_power is num_src x num_freq, rcv_power num_rcv x
 * num_freq, out_power capacity x num_freq.  A count above capacity
 * returns WQ3D_ERR_OVERFLOW after filling the first `capacity`.  Runs on the
 * current device; its device buffers stay allocated for the next call on
 * that device (they only grow), and calls on one device are serialised. */
int wq3d_biverbs(const wq3d_eigenverb* src, const double* src_power, size_t num_src,
                 const wq3d_eigenverb* rcv, const double* rcv_power, size_t num_rcv,
                 const double* freq, size_t num_freq, const wq3d_scattering_desc* scattering,
                 double earth_radius, double search_scale, double power_threshold,
                 wq3d_biverb* out, double* out_power, size_t capacity, size_t* count);

/* ------------------------------------------------------------------ */
/* misc                                                                */
/* ------------------------------------------------------------------ */
const char* wq3d_last_error_string(void);
int wq3d_abi_version(void);
int wq3d_device_count(int* count);

#ifdef __cplusplus
}
#endif
#endif /* WQ3D_H */
