/*
 * wq3d_engine.cuh -- device-side layout of one wave queue and the kernel
 * entry points of the FP64 propagation engine.
 *
 * HBM layout: wavefronts in a ring of RING slots (the reference's
 * past/prev/curr/next circular queue, waveq3d/wave_queue.h:350, plus one
 * slot).  Every per-ray field is its own contiguous array of N = num_de *
 * num_az values in (de, az) row-major order, so one thread per ray reads
 * and writes fully coalesced.  Per frequency fields are frequency-major
 * ([f][N]).  A ring role is selected by the step number: at the start of
 * step s the roles are past = F[s % RING], prev = F[(s+1) % RING], curr =
 * F[(s+2) % RING], next = F[(s+3) % RING], and step s writes its new front
 * into F[(s+4) % RING]: the reference's pointer rotation
 * (wave_queue.cc:162-167) without copying.  The fifth slot lets step s+1
 * write its new front while step s-1's eigenray construction, on its own
 * stream, still reads that step's prev / curr / next fronts.
 *
 * Instead of the reference's num_targets x N distance2 matrices per front
 * (wave_front.h:258), each front keeps the four terms that
 * compute_target_distance used when the front was last updated
 * (rho, theta, phi, sin(theta)); the CPA kernels recompute distance2 from
 * them.  A reflection re-initialises a ray's positions but, as in the
 * reference, not its distance2, so these terms are only written by update.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "wq3d_models.cuh"

namespace wq3d {

constexpr int MAX_FREQ = 64;     /* frequencies per queue                */
constexpr int RING = 5;          /* wavefront slots                      */
constexpr int CAND_LISTS = 3;    /* eigenray candidate lists             */
constexpr int SHADOW_SETS = 3;   /* reflection shadow slot sets          */
constexpr int MAX_AZ = 4096;     /* AZ fan size (duplicate bit mask)     */
constexpr int MAX_BOUNCE = 64;   /* reflections of one ray in one step   */

/* error bits written by kernels (never a trap) */
enum : uint32_t {
    ERR_BOUNCE_LIMIT = 1u,       /* more than MAX_BOUNCE reflections in a step */
    ERR_CAND_OVERFLOW = 2u,      /* eigenray candidate list full               */
    ERR_REC_OVERFLOW = 4u,       /* eigenray record buffer full                */
    ERR_REFL_OVERFLOW = 8u,      /* reflection record buffer full              */
    ERR_WALK_LIMIT = 16u,        /* a Gaussian-beam walk exceeded its bound    */
    ERR_VERB_OVERFLOW = 32u,     /* eigenverb record buffer full               */
    ERR_NONFINITE = 64u,         /* a ray's new position or direction is NaN/Inf */
    ERR_ADJ_OVERFLOW = 128u,     /* adjoint checkpoint or record buffer full    */
    ERR_BAD_CANDIDATE = 256u,    /* a candidate names a ray or target outside the fan (skipped) */
    ERR_SLOT_OVERFLOW = 512u,    /* more inline reflections in a step than rays (skipped) */
    ERR_BOUNDS = 1024u           /* WQ3D_CHECKED build: an index read from device data was out of range */
};

/* The WQ3D_CHECKED build (libwq3d_checked.so) tests every index a kernel
 * reads from device data -- worklist entries, shadow slot numbers,
 * queued CPA pairs -- before it uses one: a failed test sets ERR_BOUNDS
 * and takes the given way out instead of the access.  The default build
 * compiles the tests away. */
#ifndef WQ3D_CHECKED
#define WQ3D_CHECKED 0
#endif
#if WQ3D_CHECKED
#define WQ_CHECKED_OR(q, cond, action)         \
    do {                                       \
        if (!(cond)) {                         \
            atomicOr((q).err, wq3d::ERR_BOUNDS); \
            action;                            \
        }                                      \
    } while (0)
#else
#define WQ_CHECKED_OR(q, cond, action) \
    do {                               \
    } while (0)
#endif

/* k_advance's decisions for k_commit (QueueDev::commit_flag) */
enum : uint8_t { COMMIT_REFLECT = 1, COMMIT_FOLD = 2, COMMIT_UPPER = 4, COMMIT_LOWER = 8 };

/* Per-eigenray partial derivatives recorded for the adjoint (one per
 * eigenray record while adjoint recording is on).  TL is the first
 * frequency's.  The cube values are the 27 target distance2 values that
 * build_eigenray reads on the prev / curr / next fronts; cells are the
 * beam-walk cells whose widths the hybrid Gaussian sum used. */
constexpr int ADJ_MAX_CELLS = 256;
struct AdjRec {
    int64_t step;          /* eigenray step (its fronts are that step's)  */
    int32_t t;             /* target index                                 */
    int32_t i;             /* ray index de * num_az + az                   */
    int32_t ncell;
    int32_t flags;         /* ADJ_VALID, ADJ_CELL_OVERFLOW                 */
    int32_t a_de;          /* AZ column of the D/E walk                    */
    int32_t d_az;          /* D/E row of the AZ walk                       */
    int32_t role_a0;       /* fronts (0 prev, 1 curr, 2 next) holding the  */
    int32_t role_a1;       /* two attenuations interpolated in time        */
    double no_de[3];       /* offsets the D/E walk's widths use            */
    double no_az[3];       /* offsets the AZ walk's widths use             */
    double dT[27];         /* d travel time / d cube value                 */
    double dTL[27];        /* d TL / d cube value                          */
    double dTL_da0, dTL_da1;
    double dTL_ds2;        /* d TL / d (2 pi c_target / f)^2               */
    int16_t cell_d[ADJ_MAX_CELLS];
    int16_t cell_a[ADJ_MAX_CELLS];
    uint8_t cell_kind[ADJ_MAX_CELLS]; /* 0 width_de, 1 width_az */
    double cell_g[ADJ_MAX_CELLS];     /* d TL / d cell width   */
};
enum : int32_t { ADJ_VALID = 1, ADJ_CELL_OVERFLOW = 2 };

struct FrontPtrs {
    double* pos[3];
    double* pg[3];
    double* nd[3];
    double* ng[3];
    double* c;
    double* sg[3];
    double* dist;
    double* plen;
    double* atten;   /* [nf][n] */
    double* phase;   /* [nf][n] */
    double* cpa[4];  /* rho, theta, phi, sin(theta) at the last update */
    double* dA;      /* [3][n] d attenuation / d (bottom density ratio,
                        speed ratio, attenuation); sensitivity mode only */
    int32_t* surface;
    int32_t* bottom;
    int32_t* caustic;
    int32_t* upper;
    int32_t* lower;
    uint8_t* on_edge;
};

struct QueueDev {
    FrontPtrs F[RING];
    OceanDev oc;
    int nde, naz, nf, n;
    int nt, nt1, nt2;
    int az_boundary;
    int spreading;
    int precision;
    double dt;
    double R;
    /* fans and frequencies */
    const double* freq;
    const double* alpha;     /* Thorp coefficient per frequency */
    const double* de;
    const double* de_inc;
    const double* az;
    const double* az_inc;
    const double* cos_de;
    const double* sin_de;
    const double* cos_az;
    const double* sin_az;
    double source[3];        /* unclamped, as passed to init_wave */
    double c_source;
    /* targets */
    const double* tgt[3];
    const double* tgt_sin;
    const double* tgt_R2;
    const double* tgt_2R;
    const double* tgt_spread2;   /* [nt][nf] (2 pi c_target / f)^2 */
    const double* tgt_c;         /* sound speed at each target */
    const uint8_t* de_branch;
    /* spreading normalisation */
    const double* norm_de;
    const double* norm_az;
    const double* init_area;
    double init_sound_speed;
    /* thresholds */
    double intensity_threshold;
    int max_bottom, max_surface, max_caustic, max_upper, max_lower;
    /* chunk control */
    const int64_t* d_base;   /* steps completed before this chunk          */
    const double* d_times;   /* time after base + k steps, k = 0..K         */
    uint8_t* flag[2];        /* reflection decision for the "next" front    */
    uint32_t* work[2];       /* rays that reflect at the start of a step     */
    uint32_t* n_work[2];     /* surface part (front of the list)             */
    uint32_t* n_work_b[2];   /* bottom part (back of the list)               */
    uint32_t* n_done;        /* finished blocks of k_reflect              */
    /* reflections of step s, in set shadow_set(s): step s+1 reads step s's
     * slots while k_commit of step s has not yet run, and an advance that
     * reflects the following step's rays itself fills a third set while
     * it reads the two before */
    double* shadow[SHADOW_SETS];       /* reflected prev/curr/next per slot */
    int32_t* shadow_cnt[SHADOW_SETS];  /* surface, bottom, caustic per slot */
    int32_t* shadow_slot[SHADOW_SETS]; /* slot of each reflecting ray       */
    uint8_t* commit_flag[SHADOW_SETS]; /* per ray: COMMIT_* bits k_advance leaves for k_commit */
    uint32_t* n_slot;        /* [SHADOW_SETS] slots taken by inline reflections */
    /* eigenray candidates: CAND_LISTS lists by step (cand_list), so the
     * next steps' advance and CPA search fill others while this step's
     * eigenray construction, on its own stream, reads its list */
    uint32_t* cand;          /* [CAND_LISTS][cap_cand] packed: target, ray   */
    uint32_t* n_cand;        /* [CAND_LISTS] counts                          */
    uint32_t cap_cand;
    /* eigenray records of the chunk */
    wq3d_eigenray* rec;
    double* rec_inten;       /* [cap][nf] */
    double* rec_phase;
    uint32_t* n_rec;
    uint32_t cap_rec;
    double* rec_sens;        /* [cap][3] dTL / d bottom parameters        */
    int sens;                /* sensitivity mode                          */
    /* reflection records (only when a listener wants them) */
    wq3d_reflection* refl;
    uint32_t* n_refl;
    uint32_t cap_refl;
    int want_refl;
    /* eigenverb records (only when a listener wants them) */
    wq3d_eigenverb* verb;
    double* verb_power;      /* [cap][nf] */
    uint32_t* n_verb;
    uint32_t cap_verb;
    int want_verbs;
    double verb_threshold;   /* linear power (wave_thresholds.h:87-89)     */
    uint32_t* err;
    /* adjoint recording (wq3d_queue_enable_adjoint) */
    int adj;                 /* record checkpoints and eigenray partials   */
    int adj_K;               /* checkpoint interval (steps)                 */
    int adj_nckpt;           /* checkpoint slots                            */
    double* adj_ckpt;        /* [slot][18][n]: pos, ndir of prev/curr/next  */
    AdjRec* adj_rec;
    uint32_t* adj_n;         /* AdjRec entries written                      */
    uint32_t adj_cap;
    uint32_t* adj_mark;      /* eigenray records of the chunk processed     */
};

/* the ring slot of step-relative index s (s >= 0) */
__device__ __forceinline__ int ring_slot(int64_t s) { return (int)(s % RING); }

/* the shadow slot set of the reflections at the start of step s (s >= 0) */
__device__ __forceinline__ int shadow_set(int64_t s) { return (int)(s % SHADOW_SETS); }

/* The candidate list of the step whose rotated roles start at s (the "s"
 * of the CPA and eigenray kernels, one more than the advance's).  Step k's
 * eigenray construction reads its list while steps k+1 and k+2 fill the
 * others; step k+3's advance clears it again only after step k+2's
 * commit, which follows step k's eigenray construction on its stream. */
__device__ __forceinline__ int cand_list(int64_t s) { return (int)((s + 2) % CAND_LISTS); }

/* kernels (wq3d_kernels.cu).  Every kernel takes the queue descriptor by
 * value as a __grid_constant__ parameter, so its fields are read through
 * the constant cache.  The ray-stepping kernels come in two
 * builds: "gridded" evaluates every profile and boundary kind, "analytic"
 * leaves out the gridded ones (whose out-of-line interpolation calls cost
 * the stepping kernels registers) and serves oceans without grids. */
#define WQ3D_DECLARE_STEP_KERNELS                         \
    __global__ void k_startup(__grid_constant__ const QueueDev q);         \
    __global__ void k_reflect(__grid_constant__ const QueueDev q, int k);  \
    __global__ void k_advance(__grid_constant__ const QueueDev q, int k);         \
    __global__ void k_advance_inline(__grid_constant__ const QueueDev q, int k);
namespace gridded {
WQ3D_DECLARE_STEP_KERNELS
}
namespace analytic {
WQ3D_DECLARE_STEP_KERNELS
}
__global__ void k_volume(__grid_constant__ const QueueDev q, int k);
__global__ void k_commit(__grid_constant__ const QueueDev q, int k);
__global__ void k_cpa(__grid_constant__ const QueueDev q, int k);
__global__ void k_cpa_f32(__grid_constant__ const QueueDev q, int k);
/* k_eigenray blocks (4 warps each, one candidate per warp pair at a
 * time): four per SM, so a step's candidates usually all run at once */
constexpr int EIG_BLOCKS = 4 * 148;
__global__ void k_eigenray(__grid_constant__ const QueueDev q, int k);
__global__ void k_sound_speed(OceanDev oc, double R, int n, const double* rho,
                              const double* theta, const double* phi,
                              double* c, double* g);
__global__ void k_height(BoundaryDev b, int n, const double* theta,
                         const double* phi, double* h, double* nrm);
__global__ void k_attenuation(ProfileDev pr, double R, int n, const double* rho,
                              const double* dist, int nf, const double* freq,
                              const double* alpha, double* atten);
__global__ void k_reflect_loss(BoundaryDev b, int n, const double* grazing,
                               int nf, const double* freq, double* amp,
                               double* ph);
/* adjoint recording (wq3d_adjoint.cuh) */
__global__ void k_adj_checkpoint(__grid_constant__ const QueueDev q, int k);
__global__ void k_eigenray_jac(__grid_constant__ const QueueDev q, int k);
__global__ void k_adj_mark(__grid_constant__ const QueueDev q);

/* adjoint sweep (wq3d_adjoint.cuh) */
constexpr int ADJ_S = 18;         /* state doubles per ray                   */
constexpr int ADJ_L = 21;         /* adjoint doubles: state + 3 attenuations */
constexpr int ADJ_W = 6;          /* profile nodes one step's Jacobian covers */
constexpr int ADJ_NB = 8;         /* dual directions per pass                */
constexpr int ADJ_MAX_NODES = 64; /* profile nodes the gradient can have     */

/* adjoint error bits (AdjSweep::err) */
enum : uint32_t {
    ADJ_ERR_WINDOW = 1u,   /* a step reached profile nodes beyond its window */
    ADJ_ERR_CHAIN = 2u,    /* more than 8 reflections in one step            */
    ADJ_ERR_TOPOLOGY = 4u  /* the dual re-evaluation took another branch     */
};

struct AdjSweep {
    int64_t m0, m1;        /* segment of states [m0, m1)                 */
    int64_t m_end;         /* the last state of the run                  */
    int ckpt;              /* checkpoint slot of m0                      */
    int nrec;              /* AdjRec entries                              */
    const double* w_tl;    /* per AdjRec: weight of TL                    */
    const double* w_t;     /* per AdjRec: weight of travel time           */
    double* seg;           /* [K+1][18][n] states of the segment          */
    uint32_t* chain;       /* [K+1][n] reflection chain of each step       */
    double* seed;          /* [K+1][21][n]                                */
    double* lam;           /* [21][n] lambda at the segment's end          */
    int64_t* last;         /* [n] last seeded state, -1 for none            */
    double* grad;          /* [nodes] d L / d node                         */
    int nodes;
    double alpha0;         /* absorption per metre factor, frequency 0     */
    uint32_t* err;
};

__global__ void k_adj_touch(AdjSweep a, __grid_constant__ const QueueDev q);
__global__ void k_adj_recompute(AdjSweep a, __grid_constant__ const QueueDev q);
__global__ void k_adj_expand(AdjSweep a, __grid_constant__ const QueueDev q);
__global__ void k_adj_reverse(AdjSweep a, __grid_constant__ const QueueDev q);
__global__ void k_adj_startup(AdjSweep a, __grid_constant__ const QueueDev q);


constexpr int CPA_THREADS = 128;     /* rays per CPA block            */
constexpr int CPA_F32_TARGETS = 256; /* targets per FP32C CPA tile    */
constexpr int CPA_PATCH_AZ = 8;      /* FP32C CPA block: 16 D/E x 8 AZ rays */
constexpr int CPA_PATCH_DE = CPA_THREADS / CPA_PATCH_AZ;

}  // namespace wq3d
