/*
 * wq3d_api.cu -- host side of the C ABI declared in include/wq3d.h.
 *
 * Owns device memory, precomputes everything that depends only on inputs
 * (fan trigonometry, target terms, spreading normalisation, boundary
 * constants) with the same arithmetic the reference uses, runs the step
 * loop in chunks of K steps (captured once as a CUDA graph and replayed),
 * and turns the device's eigenray/reflection records into listener calls
 * in the reference's order.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "wq3d_engine.cuh"

using namespace wq3d;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define WQ_CK(x)                                                                  \
    do {                                                                          \
        cudaError_t e_ = (x);                                                     \
        if (e_ != cudaSuccess)                                                    \
            return fail(WQ3D_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

inline double to_radians(double t) { return t * (M_PI / 180.0); }
inline double to_degrees(double t) { return t * (180.0 / M_PI); }

/* reflect loss constants (reflect_loss_rayleigh.cc:17,68-78) and the
 * defaults of boundary_model.h:77-90 / boundary_flat.cc:19-31 */
void setup_boundary(BoundaryDev& b, const wq3d_boundary_desc& d, double R) {
    std::memset(&b, 0, sizeof(b));
    b.kind = d.kind;
    b.loss.kind = d.loss.kind;
    for (int k = 0; k < 5; ++k) b.loss.p[k] = d.loss.p[k];
    if (d.kind == WQ3D_BOUNDARY_SLOPE) {
        /* boundary_slope.cc:13-24 and the constant factors of :55-68 */
        b.height = R - d.depth;
        b.normal[1] = std::sin(d.lat_slope);
        b.normal[2] = -std::sin(d.lng_slope);
        b.normal[0] = std::sqrt(1.0 - b.normal[1] * b.normal[1] - b.normal[2] * b.normal[2]);
        const double alpha = -std::asin(b.normal[1]);
        const double beta = -std::asin(b.normal[2]);
        b.loc_theta = d.location[1];
        b.loc_phi = d.location[2];
        b.slope_a = std::sin(d.location[1]) * std::tan(beta);
        b.slope_b = std::tan(alpha);
        if (b.loss.kind == WQ3D_LOSS_DEFAULT) {
            b.loss.kind = WQ3D_LOSS_CONSTANT;
            b.loss.p[0] = 0.0;
            b.loss.p[1] = 0.0;
        }
    } else if (d.kind == WQ3D_BOUNDARY_GRID) {
        /* boundary_grid.h:56-59: Rayleigh sand unless a loss is given */
        if (b.loss.kind == WQ3D_LOSS_DEFAULT) {
            b.loss.kind = WQ3D_LOSS_RAYLEIGH;
            const double sand[5] = {1.9, 1.10, 0.8, 0.00, 2.5};
            for (int k = 0; k < 5; ++k) b.loss.p[k] = sand[k];
        }
    } else {
        b.kind = WQ3D_BOUNDARY_FLAT;
        b.height = R - std::abs(d.depth);
        if (std::abs(d.depth) < 1e-6) {
            b.normal[0] = -1.0;
            if (b.loss.kind == WQ3D_LOSS_DEFAULT) {
                b.loss.kind = WQ3D_LOSS_CONSTANT;
                b.loss.p[0] = 0.0;
                b.loss.p[1] = M_PI;
            }
        } else {
            b.normal[0] = 1.0;
        }
        if (b.loss.kind == WQ3D_LOSS_DEFAULT) {
            b.loss.kind = WQ3D_LOSS_CONSTANT;
            b.loss.p[0] = 0.0;
            b.loss.p[1] = 0.0;
        }
    }
    if (b.loss.kind == WQ3D_LOSS_RAYLEIGH) {
        const double ATT_CONVERT = 1.0 / (20.0 * M_LOG10E * (2.0 * M_PI));
        b.loss.rl_den = 1000.0 * b.loss.p[0];
        b.loss.rl_spd = 1500.0 * b.loss.p[1];
        b.loss.rl_att = b.loss.p[2] * ATT_CONVERT;
        b.loss.rl_shr = 1500.0 * b.loss.p[3];
        b.loss.rl_satt = b.loss.p[4] * ATT_CONVERT;
    }
}

/* attenuation_thorp.cc:14-24: the Thorp coefficient (dB/m at 1000 m
 * depth) per frequency */
void thorp_alpha(const double* freq, size_t nf, double* alpha) {
    for (size_t k = 0; k < nf; ++k) {
        double F2 = freq[k];
        F2 = 1e-6 * F2 * F2;
        alpha[k] = 1e-3 * (3.3e-3 + F2 * (0.11 / (1.0 + F2) + 44.0 / (4100.0 + F2) + 3.0e-4)) /
                   (1.0 - 5.88264e-6 * 1000.0);
    }
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

struct wq3d_ocean {
    OceanDev dev;   /* device pointers, passed to kernels        */
    OceanDev host;  /* host pointers, for host-side evaluations  */
    double build_radius;
    int device = 0;  /* the device holding dmem: where the ocean can be used */
    std::vector<std::vector<double>> store;  /* host copies of grid arrays */
    std::vector<void*> dmem;                 /* device copies             */
    ~wq3d_ocean() {
        for (void* p : dmem) cudaFree(p);
    }
};

namespace {

/* Copies a grid description into a host GridDev and a device GridDev.
 * Interpolation types follow data_grid::interp_type (data_grid.h:137-145):
 * PCHIP needs 4 points and anything but nearest needs 2. */
int make_grid(wq3d_ocean* o, const wq3d_grid_desc& d, int max_dims, GridDev* hg, GridDev* dg) {
    if (d.ndim < 1 || d.ndim > max_dims) return fail(WQ3D_ERR_INVALID, "grid dimension out of range");
    std::memset(hg, 0, sizeof(*hg));
    hg->ndim = d.ndim;
    size_t total = 1;
    for (int k = 0; k < d.ndim; ++k) {
        const size_t n = d.axis_size[k];
        if (n < 2 || !d.axis[k] || !d.axis_inc[k]) return fail(WQ3D_ERR_INVALID, "grid axes need at least 2 values");
        if (d.axis_kind[k] < WQ3D_AXIS_LINEAR || d.axis_kind[k] > WQ3D_AXIS_DATA)
            return fail(WQ3D_ERR_INVALID, "bad axis kind");
        total *= n;
        o->store.emplace_back(d.axis[k], d.axis[k] + n);
        hg->ax[k].x = o->store.back().data();
        o->store.emplace_back(d.axis_inc[k], d.axis_inc[k] + n);
        hg->ax[k].inc = o->store.back().data();
        hg->ax[k].n = (int)n;
        hg->ax[k].kind = d.axis_kind[k];
        hg->ax[k].sign = (d.axis[k][1] - d.axis[k][0] < 0) ? -1.0 : 1.0;
        int it = d.interp[k];
        if (it > WQ3D_INTERP_NEAREST && n < 2) {
            it = WQ3D_INTERP_NEAREST;
        } else if (it > WQ3D_INTERP_LINEAR && n < 4) {
            it = WQ3D_INTERP_LINEAR;
        }
        hg->interp[k] = it;
        hg->edge[k] = d.edge_limit[k] ? 1 : 0;
    }
    if (!d.data) return fail(WQ3D_ERR_INVALID, "grid data missing");
    hg->all_linear = 1;
    for (int k = 0; k < d.ndim; ++k)
        if (hg->interp[k] != WQ3D_INTERP_LINEAR) hg->all_linear = 0;
    hg->pchip0 = hg->interp[0] == WQ3D_INTERP_PCHIP;
    for (int k = 1; k < d.ndim; ++k)
        if (hg->interp[k] != WQ3D_INTERP_LINEAR) hg->pchip0 = 0;
    o->store.emplace_back(d.data, d.data + total);
    hg->data = o->store.back().data();
    *dg = *hg;
    auto up = [&](const double* src, size_t n, const double** out) -> int {
        void* p = nullptr;
        WQ_CK(cudaMalloc(&p, n * sizeof(double)));
        o->dmem.push_back(p);
        WQ_CK(cudaMemcpy(p, src, n * sizeof(double), cudaMemcpyHostToDevice));
        *out = static_cast<const double*>(p);
        return WQ3D_OK;
    };
    int rc = 0;
    for (int k = 0; k < d.ndim && !rc; ++k) {
        rc = up(hg->ax[k].x, hg->ax[k].n, &dg->ax[k].x);
        if (!rc) rc = up(hg->ax[k].inc, hg->ax[k].n, &dg->ax[k].inc);
    }
    if (!rc) rc = up(hg->data, total, &dg->data);
    return rc;
}

}  // namespace

/* The reflection-schedule plan learnt per queue shape (fan, targets,
 * frequencies, kernel build, chunk length), shared by every queue of the
 * process.  A run is cut into buckets of TUNE_BUCKET steps, since which
 * schedule wins changes as the fan spreads and meets the boundaries.  The
 * first two full chunks that reach a bucket try one schedule each and
 * their device times are kept; every later chunk in that bucket, of this
 * queue or a later one of the same shape, runs the faster. */
constexpr int TUNE_BUCKET = 128;
struct TunePlan {
    std::string key;
    std::vector<double> ms[2];
    std::vector<int> cnt[2];
    std::vector<int> pend[2]; /* chunks chosen but not yet measured */
};
std::mutex g_tune_mu;
std::vector<TunePlan> g_plans;

TunePlan& tune_plan(const std::string& key, size_t bucket) {
    TunePlan* e = nullptr;
    for (auto& t : g_plans)
        if (t.key == key) e = &t;
    if (!e) {
        g_plans.emplace_back();
        e = &g_plans.back();
        e->key = key;
    }
    for (int m = 0; m < 2; ++m)
        if (e->ms[m].size() <= bucket) {
            e->ms[m].resize(bucket + 1, 0.0);
            e->cnt[m].resize(bucket + 1, 0);
            e->pend[m].resize(bucket + 1, 0);
        }
    return *e;
}

/* the schedule of a full chunk in this bucket (1 inline, 0 side), and in
 * *trial whether the chunk is one of the bucket's two timed trials */
int tune_choose(const std::string& key, size_t bucket, bool* trial) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    TunePlan& t = tune_plan(key, bucket);
    int m;
    *trial = false;
    if (t.cnt[1][bucket] + t.pend[1][bucket] == 0) {
        m = 1;
        *trial = true;
    } else if (t.cnt[0][bucket] + t.pend[0][bucket] == 0) {
        m = 0;
        *trial = true;
    } else if (t.cnt[0][bucket] == 0 || t.cnt[1][bucket] == 0) {
        m = t.cnt[0][bucket] == 0 ? 1 : 0; /* the measured one until both are */
    } else {
        m = t.ms[1][bucket] < t.ms[0][bucket] ? 1 : 0;
    }
    if (*trial) t.pend[m][bucket] += 1;
    return m;
}

void tune_record(const std::string& key, size_t bucket, int m, bool ok, double ms) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    TunePlan& t = tune_plan(key, bucket);
    if (t.pend[m][bucket] > 0) t.pend[m][bucket] -= 1;
    if (ok) {
        t.ms[m][bucket] += ms;
        t.cnt[m][bucket] += 1;
    }
}

/* eigenrays kept for wq3d_queue_take_eigenrays (no listener), as flat
 * arrays: nf intensities and phases and 3 bottom sensitivities per ray */
struct PendingRays {
    std::vector<wq3d_eigenray> rec;
    std::vector<double> inten, phase, sens;
    size_t size() const { return rec.size(); }
    void clear() {
        rec.clear();
        inten.clear();
        phase.clear();
        sens.clear();
    }
};

struct wq3d_queue {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;
    cudaStream_t eig = nullptr; /* k_commit and the eigenray construction */
    cudaStream_t adv = nullptr; /* k_advance, checkpoints, volume eigenverbs */
    cudaEvent_t start_ev = nullptr;
    std::vector<cudaEvent_t> fork_ev, join_ev;
    std::vector<cudaEvent_t> adv_ev, com_ev, cpa_ev; /* per step of a chunk */
    cudaEvent_t eig_end = nullptr;
    QueueDev h{};
    std::vector<void*> allocs;
    void* pinned = nullptr;
    /* per result set: chunk base step, chunk times, counters read back
     * (n_rec, n_refl, err, -, work lists, n_done, -, n_verb); d_counts also
     * holds the bottom work lists (9, 10), the adjoint's mark and entry
     * count (11, 12), the three candidate counts (13-15) and the three
     * shadow sets' inline slot counts (16-18) */
    int64_t* h_base[2] = {nullptr, nullptr};
    double* h_times[2] = {nullptr, nullptr};
    uint32_t* h_counts[2] = {nullptr, nullptr};
    int64_t* d_base = nullptr;
    double* d_times = nullptr;
    uint32_t* d_counts = nullptr;
    int chunk = 16;
    /* [result set][prefetches the next chunk's first reflection][inline
     * reflections] */
    cudaGraphExec_t graph[2][2][2] = {};
    bool graph_failed[2][2][2] = {};
    int64_t graph_launches[2][2][2] = {}; /* kernels in each graph */
    /* Reflection schedule (wq3d_queue_set_reflect_schedule).  Under
     * WQ3D_REFLECT_AUTO a queue run alone follows its shape's plan
     * (tune_choose) for every full chunk but a run's first, and times the
     * plan's trial chunks.  Both schedules give the same results bit for
     * bit. */
    int refl_sched = WQ3D_REFLECT_AUTO;
    int last_inl = -1;             /* schedule of the last chunk launched */
    bool in_batch = false;         /* queues of a batch use the side stream, as do
                                    * queues recording for the adjoint */
    bool chunk_trial[2] = {false, false}; /* per result set: the chunk in flight is a timed trial */
    int chunk_inl[2] = {0, 0};            /* its schedule */
    size_t chunk_bucket[2] = {0, 0};      /* and its bucket */
    cudaEvent_t tune_ev[2][2] = {};
    /* Result set 1: a second copy of the record buffers, so that chunk c
     * writes set c & 1 while the host reads the other chunk's records
     * (made by the first run of more than one chunk; set 0 lives in h). */
    struct ResultSet {
        wq3d_eigenray* rec = nullptr;
        double* rec_inten = nullptr;
        double* rec_phase = nullptr;
        double* rec_sens = nullptr;
        wq3d_reflection* refl = nullptr;
        wq3d_eigenverb* verb = nullptr;
        double* verb_power = nullptr;
    } set1;
    bool have_set1 = false;
    cudaEvent_t done_ev[2] = {nullptr, nullptr}; /* a chunk's counters are on the host */
    cudaStream_t copy = nullptr;                 /* record read-back */
    /* delivered state (time(), steps()) and launched-through state */
    double time = 0.0;
    int64_t steps = 0;
    double ltime = 0.0;
    int64_t lsteps = 0;
    /* reflection notices and eigenverbs of a step that a chunk's tail
     * reflection made for the next chunk, delivered with that chunk */
    std::vector<wq3d_reflection> carry_refl;
    std::vector<wq3d_eigenverb> carry_verb;
    std::vector<double> carry_vpower;
    double src_clamped[3] = {0, 0, 0};
    wq3d_callbacks cb{};
    void* cb_ctx = nullptr;
    uint64_t run_id = 0;
    PendingRays pending;
    std::atomic<bool> abort_flag{false};
    bool timing = false;
    std::vector<cudaEvent_t> events;
    double ms_step = 0.0, ms_cpa = 0.0, ms_eig = 0.0, ms_total = 0.0, ms_refl = 0.0;
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    int64_t launches = 0;
    /* the stepping kernels' build: "gridded" when the ocean has a grid */
    bool gridded = false;
    void (*k_reflect_fn)(const QueueDev, int) = analytic::k_reflect;
    void (*k_advance_fn)(const QueueDev, int) = analytic::k_advance;
    void (*k_advance_inline_fn)(const QueueDev, int) = analytic::k_advance_inline;
    /* eigenverb counting sink (wq3d_queue_count_eigenverbs) */
    bool count_verbs = false;
    uint64_t verb_counts[2 + 2 * WQ3D_MAX_VOLUME] = {0};
    /* set while wq3d_queue_create re-initialises a queue taken from the
     * cache of destroyed queues: uploads then copy into the buffers the
     * queue already has */
    bool reuse = false;
    char* ring = nullptr;   /* the wavefront ring's allocation */
    size_t ring_bytes = 0;
    /* adjoint workspace (wq3d_queue_adjoint), made on first use */
    struct AdjWork {
        double* seg = nullptr;
        uint32_t* chain = nullptr;
        double* seed = nullptr;
        double* lam = nullptr;
        int64_t* last = nullptr;
        double* grad = nullptr;
        double* w = nullptr;
        uint32_t* err = nullptr;
        size_t w_cap = 0;
    } adjw;
    std::vector<wq3d_eigenray> h_rec;
    std::vector<double> h_rinten, h_rphase, h_rsens;
    std::vector<wq3d_reflection> h_refl;
    std::vector<wq3d_eigenverb> h_verb;
    std::vector<double> h_vpower;

    /* the chunk graph holds the queue descriptor by value (kernel
     * parameters), so it is rebuilt whenever the descriptor or the launch
     * sequence changes */
    void drop_graph() {
        for (int p = 0; p < 2; ++p)
            for (int t = 0; t < 2; ++t)
                for (int m = 0; m < 2; ++m) {
                    if (graph[p][t][m]) cudaGraphExecDestroy(graph[p][t][m]);
                    graph[p][t][m] = nullptr;
                    graph_failed[p][t][m] = false;
                }
    }

    /* the descriptor that writes result set p */
    QueueDev dev(int p) const {
        QueueDev d = h;
        if (p == 1) {
            d.rec = set1.rec;
            d.rec_inten = set1.rec_inten;
            d.rec_phase = set1.rec_phase;
            d.rec_sens = set1.rec_sens;
            d.refl = set1.refl;
            d.verb = set1.verb;
            d.verb_power = set1.verb_power;
        }
        return d;
    }

    /* Result set 1, the same sizes as set 0.  Returns false (and the run
     * stays on set 0, one chunk at a time) when the memory is not there. */
    bool ensure_set1() {
        if (have_set1) return true;
        const size_t nf = (size_t)h.nf;
        ResultSet s;
        std::vector<void*> got;
        auto take = [&](auto** out, size_t count) {
            void* p = nullptr;
            if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(**out)) != cudaSuccess) {
                cudaGetLastError();
                return false;
            }
            got.push_back(p);
            *out = static_cast<std::remove_reference_t<decltype(*out)>>(p);
            return true;
        };
        bool ok = take(&s.rec, h.cap_rec) && take(&s.rec_inten, (size_t)h.cap_rec * nf) &&
                  take(&s.rec_phase, (size_t)h.cap_rec * nf) && take(&s.refl, h.cap_refl) &&
                  (!h.sens || take(&s.rec_sens, (size_t)h.cap_rec * 3)) &&
                  (!h.verb || (take(&s.verb, h.cap_verb) && take(&s.verb_power, (size_t)h.cap_verb * nf)));
        if (!ok) {
            for (void* p : got) cudaFree(p);
            return false;
        }
        allocs.insert(allocs.end(), got.begin(), got.end());
        set1 = s;
        have_set1 = true;
        return true;
    }

    bool volume_pass() const { return h.want_verbs && h.oc.nvol > 0; }

    void release(void* p) {
        if (!p) return;
        auto it = std::find(allocs.begin(), allocs.end(), p);
        if (it != allocs.end()) allocs.erase(it);
        cudaFree(p);
    }

    /* A record buffer's capacity for "need" records of rec_bytes each: at
     * least 4096, at most a quarter of the free device memory. */
    int record_capacity(size_t need, size_t rec_bytes, size_t* out) {
        size_t free_b = 0, total_b = 0;
        WQ_CK(cudaMemGetInfo(&free_b, &total_b));
        const size_t limit = std::max<size_t>(4096, (free_b / 4) / rec_bytes);
        *out = std::min<size_t>({std::max<size_t>(need, 4096), limit, (size_t)UINT32_MAX / 2});
        return WQ3D_OK;
    }
    template <class T>
    int remake(T** p, size_t count) {
        release(*p);
        *p = nullptr;
        return alloc(p, count);
    }

    /* Eigenverb buffers (both result sets) hold at least "need" records.
     * They start at half a record per ray, step and interface of a chunk
     * and grow when a chunk fills more than half of them.  Runs with no
     * chunk in flight; drops the graphs, which hold the pointers. */
    int ensure_verb_capacity(size_t need) {
        if (h.verb && need <= h.cap_verb) return WQ3D_OK;
        size_t cap = 0;
        int rc = record_capacity(need, sizeof(wq3d_eigenverb) + (size_t)h.nf * sizeof(double), &cap);
        if (rc) return rc;
        if (h.verb && cap <= h.cap_verb) return WQ3D_OK;
        WQ_CK(cudaStreamSynchronize(stream));
        h.cap_verb = 0;
        rc = remake(&h.verb, cap);
        if (!rc) rc = remake(&h.verb_power, cap * (size_t)h.nf);
        if (!rc && have_set1) rc = remake(&set1.verb, cap);
        if (!rc && have_set1) rc = remake(&set1.verb_power, cap * (size_t)h.nf);
        if (rc) return rc;
        h.cap_verb = (uint32_t)cap;
        drop_graph();
        return WQ3D_OK;
    }

    /* Reflection buffers: half a record per ray and step of a chunk when a
     * reflection listener first asks, grown like the eigenverb buffers. */
    int ensure_refl_capacity(size_t need) {
        if (need <= h.cap_refl) return WQ3D_OK;
        size_t cap = 0;
        int rc = record_capacity(need, sizeof(wq3d_reflection), &cap);
        if (rc) return rc;
        if (cap <= h.cap_refl) return WQ3D_OK;
        WQ_CK(cudaStreamSynchronize(stream));
        h.cap_refl = 0;
        rc = remake(&h.refl, cap);
        if (!rc && have_set1) rc = remake(&set1.refl, cap);
        if (rc) return rc;
        h.cap_refl = (uint32_t)cap;
        drop_graph();
        return WQ3D_OK;
    }

    /* growth asked for by a chunk's counts, done when nothing is in flight */
    size_t grow_verb = 0, grow_refl = 0;
    int apply_growth() {
        int rc = WQ3D_OK;
        if (grow_verb) rc = ensure_verb_capacity(grow_verb);
        if (!rc && grow_refl) rc = ensure_refl_capacity(grow_refl);
        grow_verb = grow_refl = 0;
        return rc;
    }

    ~wq3d_queue() {
        drop_graph();
        for (auto e : done_ev)
            if (e) cudaEventDestroy(e);
        for (auto& pe : tune_ev)
            for (auto e : pe)
                if (e) cudaEventDestroy(e);
        if (copy) cudaStreamDestroy(copy);
        for (auto e : events)
            if (e) cudaEventDestroy(e);
        for (auto e : fork_ev) cudaEventDestroy(e);
        for (auto e : join_ev) cudaEventDestroy(e);
        for (auto* v : {&adv_ev, &com_ev, &cpa_ev})
            for (auto e : *v) cudaEventDestroy(e);
        if (eig_end) cudaEventDestroy(eig_end);
        if (start_ev) cudaEventDestroy(start_ev);
        if (adv) cudaStreamDestroy(adv);
        if (eig) cudaStreamDestroy(eig);
        if (side) cudaStreamDestroy(side);
        if (ev_begin) cudaEventDestroy(ev_begin);
        if (ev_end) cudaEventDestroy(ev_end);
        for (void* p : allocs) cudaFree(p);
        if (pinned) cudaFreeHost(pinned);
        if (stream) cudaStreamDestroy(stream);
    }

    template <class T>
    int alloc(T** out, size_t count) {
        void* p = nullptr;
        const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
        WQ_CK(cudaMalloc(&p, bytes));
        allocs.push_back(p);
        *out = static_cast<T*>(p);
        return WQ3D_OK;
    }
    template <class T>
    int upload(const T** out, const std::vector<T>& v) {
        T* p = nullptr;
        if (reuse && *out) {
            p = const_cast<T*>(*out); /* same size: the cache key fixes every length */
        } else {
            int rc = alloc(&p, v.size());
            if (rc) return rc;
        }
        if (!v.empty()) WQ_CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
        *out = p;
        return WQ3D_OK;
    }

    /* One chunk of K steps writing result set p.  Without per-kernel
     * timing it runs on four streams:
     *   adv   k_advance(k) after k_reflect(k); the adjoint's checkpoint and
     *         the volume eigenverbs of a step run before its advance
     *   main  k_cpa(k) after k_advance(k), beside k_advance(k+1)
     *   side  k_reflect(k+1) (high priority), right after k_advance(k),
     *         beside k_cpa(k)
     *   eig   k_commit(k) after k_advance(k), k_eigenray(k) after k_cpa(k),
     *         and the adjoint's eigenray partials
     * Step k+1 reads the rays that reflected at step k from step k's shadow
     * slots, so neither k_reflect(k+1) nor k_advance(k+1) waits for
     * k_commit(k) (except with eigenverbs: an eigenverb reads the curr
     * front's losses and counts, so k_reflect(k+1) then waits for it).
     * k_reflect(k+1) reuses step k-1's slot set and k_advance(k+1) its
     * commit flags, so k_reflect(k+1) waits for k_commit(k-1); that also
     * orders k_advance(k+1) after step k-2's eigenray construction, whose
     * prev front and candidate list it overwrites (five ring slots, three
     * candidate lists).  With "tail" the reflections of the
     * next chunk's first step run beside this chunk's last CPA search; that
     * chunk's own k_reflect(0) then finds an empty worklist and returns.
     * Without eigenverbs (which read the committed curr front) there is no
     * side stream: k_advance(k) runs step k+1's reflection chains for its
     * own rays as soon as it has written their next front, so a step costs
     * the longer of the advance and the longest reflection chain instead of
     * their sum.  Those chains fill the shadow set of step k+1, the set
     * step k-2 used, so k_advance(k) waits for k_commit(k-2).
     * With per-kernel timing the steps run one launch after another on the
     * main stream, except k_reflect(k+1) beside k_cpa(k) and k_eigenray(k).
     * (An advance split into the rays that need none of the step's
     * reflections, run beside k_reflect and k_cpa, and the rest was slower:
     * 149.5 against 131.9 ms per propagation of the sloped workload, the
     * memory-bound advance taking SM time from the CPA search.) */
    int launch_chunk(int K, int p, bool tail, bool inl_wanted) {
        const QueueDev d = dev(p);
        const int n = h.n;
        const dim3 blk(128);
        const dim3 grd((n + 127) / 128);
        const int rgrid = std::max(1, std::min(4 * 148, (n + 63) / 64));
        /* eigenray candidates grow with the fan: one block per SM for small
         * fans, up to EIG_BLOCKS */
        const int eig_blocks = std::min(EIG_BLOCKS, std::max(148, (n + 255) / 256));
        if (timing) tail = false;
        auto cpa_launch = [&](int k, cudaStream_t st) {
            const dim3 cgrid(((h.nde + CPA_PATCH_DE - 1) / CPA_PATCH_DE) * ((h.naz + CPA_PATCH_AZ - 1) / CPA_PATCH_AZ),
                             (h.nt + CPA_F32_TARGETS - 1) / CPA_F32_TARGETS);
            if (h.precision != WQ3D_FP64)
                k_cpa_f32<<<cgrid, CPA_THREADS, 0, st>>>(d, k);
            else
                k_cpa<<<cgrid, CPA_THREADS, 0, st>>>(d, k);
        };
        auto eig_launch = [&](int k, cudaStream_t st) {
            k_eigenray<<<eig_blocks, 128, 0, st>>>(d, k);
            launches += 1;
            if (h.adj) {
                k_eigenray_jac<<<4 * 148, 64, 0, st>>>(d, k);
                k_adj_mark<<<1, 1, 0, st>>>(d);
                launches += 2;
            }
        };
        if (timing) cudaEventRecord(events[7 * K], stream);
        k_reflect_fn<<<rgrid, 64, 0, stream>>>(d, 0);
        if (timing) cudaEventRecord(events[7 * K + 1], stream);
        launches += 1;
        if (timing) {
            for (int k = 0; k < K; ++k) {
                cudaEvent_t* ev = &events[7 * k];
                cudaEventRecord(ev[0], stream);
                if (h.adj) {
                    k_adj_checkpoint<<<grd, blk, 0, stream>>>(d, k);
                    launches += 1;
                }
                if (volume_pass()) {
                    k_volume<<<grd, blk, 0, stream>>>(d, k);
                    launches += 1;
                }
                k_advance_fn<<<grd, blk, 0, stream>>>(d, k);
                k_commit<<<grd, blk, 0, stream>>>(d, k);
                launches += 2;
                cudaEventRecord(ev[1], stream);
                if (k + 1 < K) {
                    cudaEventRecord(fork_ev[k], stream);
                    cudaStreamWaitEvent(side, fork_ev[k], 0);
                    cudaEventRecord(ev[5], side);
                    k_reflect_fn<<<rgrid, 64, 0, side>>>(d, k + 1);
                    cudaEventRecord(ev[6], side);
                    cudaEventRecord(join_ev[k], side);
                    launches += 1;
                }
                cudaEventRecord(ev[2], stream);
                if (h.nt > 0) {
                    cpa_launch(k, stream);
                    launches += 1;
                    cudaEventRecord(ev[3], stream);
                    eig_launch(k, stream);
                } else {
                    cudaEventRecord(ev[3], stream);
                }
                cudaEventRecord(ev[4], stream);
                if (k + 1 < K) cudaStreamWaitEvent(stream, join_ev[k], 0);
            }
            return WQ3D_OK;
        }
        cudaEventRecord(start_ev, stream);
        cudaStreamWaitEvent(adv, start_ev, 0);
        /* inline schedule: k_advance(k) reflects step k+1's rays itself
         * (into the third shadow set) once their next front is written;
         * nothing else in that reflection waits for step k's commit unless
         * it makes eigenverbs */
        const bool inl = inl_wanted && !h.want_verbs && !volume_pass();
        for (int k = 0; k < K; ++k) {
            const bool more = k + 1 < K || tail;
            /* adv: step k's checkpoint, volume eigenverbs and advance, after
             * its reflections; an inline advance also after step k-2's
             * commit (it refills that step's shadow set, and so follows step
             * k-3's eigenray construction, whose prev front and candidate
             * list it overwrites) */
            if (!inl && k >= 1) cudaStreamWaitEvent(adv, join_ev[k - 1], 0);
            if (inl && k >= 2) cudaStreamWaitEvent(adv, com_ev[k - 2], 0);
            if (h.adj) {
                k_adj_checkpoint<<<grd, blk, 0, adv>>>(d, k);
                launches += 1;
            }
            if (volume_pass()) {
                k_volume<<<grd, blk, 0, adv>>>(d, k);
                launches += 1;
            }
            (inl && more ? k_advance_inline_fn : k_advance_fn)<<<grd, blk, 0, adv>>>(d, k);
            launches += 1;
            cudaEventRecord(adv_ev[k], adv);
            /* eig: step k's commit */
            cudaStreamWaitEvent(eig, adv_ev[k], 0);
            k_commit<<<grd, blk, 0, eig>>>(d, k);
            launches += 1;
            cudaEventRecord(com_ev[k], eig);
            if (more && !inl) {
                /* side: step k+1's reflections */
                cudaStreamWaitEvent(side, adv_ev[k], 0);
                if (k >= 1) cudaStreamWaitEvent(side, com_ev[k - 1], 0);
                if (h.want_verbs) cudaStreamWaitEvent(side, com_ev[k], 0);
                k_reflect_fn<<<rgrid, 64, 0, side>>>(d, k + 1);
                cudaEventRecord(join_ev[k], side);
                launches += 1;
            }
            /* main: step k's CPA search (beside step k+1's advance);
             * eig: its eigenray construction */
            cudaStreamWaitEvent(stream, adv_ev[k], 0);
            if (h.nt > 0) {
                cpa_launch(k, stream);
                launches += 1;
                cudaEventRecord(cpa_ev[k], stream);
                cudaStreamWaitEvent(eig, cpa_ev[k], 0);
                eig_launch(k, eig);
            }
        }
        /* every stream joins the main stream */
        cudaEventRecord(eig_end, eig);
        cudaStreamWaitEvent(stream, eig_end, 0);
        if (tail && !inl) cudaStreamWaitEvent(stream, join_ev[K - 1], 0);
        cudaStreamWaitEvent(stream, adv_ev[K - 1], 0);
        return WQ3D_OK;
    }

    /* the shape a tuned reflection schedule applies to: the fan, targets,
     * frequencies, kernel build and chunk length (the arithmetic form,
     * sensitivities and adjoint recording change the CPA and eigenray work
     * beside the chain, not the chain itself, so they share a plan) */
    std::string tune_key() const {
        return std::to_string(h.nde) + "x" + std::to_string(h.naz) + " t" + std::to_string(h.nt) + " f" +
               std::to_string(h.nf) + (gridded ? " g" : " a") + " c" + std::to_string(chunk);
    }

    int build_graph(int p, bool tail, bool inl) {
        const int t = tail ? 1 : 0, m = inl ? 1 : 0;
        if (graph[p][t][m] || graph_failed[p][t][m]) return WQ3D_OK;
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            graph_failed[p][t][m] = true;
            cudaGetLastError();
            return WQ3D_OK;
        }
        const bool save = timing;
        timing = false;
        const int64_t saved_launches = launches;
        launch_chunk(chunk, p, tail, inl);
        graph_launches[p][t][m] = launches - saved_launches;
        launches = saved_launches;
        timing = save;
        if (cudaStreamEndCapture(stream, &g) != cudaSuccess ||
            cudaGraphInstantiate(&graph[p][t][m], g, 0) != cudaSuccess) {
            graph_failed[p][t][m] = true;
            graph[p][t][m] = nullptr;
            cudaGetLastError();
        }
        if (g) cudaGraphDestroy(g);
        return WQ3D_OK;
    }

    /* Listener calls for the K steps after "steps", in the reference's
     * order.  Reflection notices and eigenverbs of the step after the
     * chunk (made by its tail reflection) are kept for the next chunk. */
    void deliver(int K, size_t nrec, size_t nrefl, size_t nverb, const double* ht) {
        const int nf = h.nf;
        /* reference order: (step, t1, t2, de, az) for eigenrays
         * (wave_queue.cc:361-373), (step, de, az) for reflections */
        std::vector<size_t> order(nrec);
        for (size_t i = 0; i < nrec; ++i) order[i] = i;
        std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            const wq3d_eigenray& x = h_rec[a];
            const wq3d_eigenray& y = h_rec[b];
            if (x.step != y.step) return x.step < y.step;
            if (x.t1 != y.t1) return x.t1 < y.t1;
            if (x.t2 != y.t2) return x.t2 < y.t2;
            if (x.de != y.de) return x.de < y.de;
            return x.az < y.az;
        });
        std::vector<wq3d_reflection> refl;
        refl.swap(carry_refl);
        refl.insert(refl.end(), h_refl.begin(), h_refl.begin() + nrefl);
        std::sort(refl.begin(), refl.end(), [](const wq3d_reflection& x, const wq3d_reflection& y) {
            if (x.step != y.step) return x.step < y.step;
            if (x.de != y.de) return x.de < y.de;
            if (x.az != y.az) return x.az < y.az;
            return x.pad < y.pad;
        });
        /* eigenverbs: (step, de, az, seq) is the order of the reference's
         * detect_reflections loop (wave_queue.cc:197-216) */
        std::vector<wq3d_eigenverb> verbs;
        std::vector<double> vpower;
        verbs.swap(carry_verb);
        vpower.swap(carry_vpower);
        verbs.insert(verbs.end(), h_verb.begin(), h_verb.begin() + nverb);
        vpower.insert(vpower.end(), h_vpower.begin(), h_vpower.begin() + nverb * nf);
        std::vector<size_t> vorder(verbs.size());
        for (size_t i = 0; i < vorder.size(); ++i) vorder[i] = i;
        std::sort(vorder.begin(), vorder.end(), [&](size_t a, size_t b) {
            const wq3d_eigenverb& x = verbs[a];
            const wq3d_eigenverb& y = verbs[b];
            if (x.step != y.step) return x.step < y.step;
            if (x.de != y.de) return x.de < y.de;
            if (x.az != y.az) return x.az < y.az;
            return x.seq < y.seq;
        });
        size_t ir = 0, ie = 0, iv = 0;
        for (int k = 0; k < K; ++k) {
            const int64_t step = steps + k + 1;
            /* a reflection is announced before the eigenverb it makes, and
             * both carry the ray's event number */
            while ((ir < refl.size() && refl[ir].step == step) ||
                   (iv < vorder.size() && verbs[vorder[iv]].step == step)) {
                const bool verb_here = iv < vorder.size() && verbs[vorder[iv]].step == step;
                const bool refl_here = ir < refl.size() && refl[ir].step == step;
                bool take_refl = refl_here;
                if (refl_here && verb_here) {
                    const wq3d_eigenverb& v = verbs[vorder[iv]];
                    take_refl = !(std::make_tuple(v.de, v.az, v.seq) <
                                  std::make_tuple(refl[ir].de, refl[ir].az, refl[ir].pad));
                }
                if (take_refl) {
                    if (cb.reflect) cb.reflect(cb_ctx, &refl[ir]);
                    ++ir;
                } else {
                    const size_t j = vorder[iv];
                    if (count_verbs) {
                        const int in = verbs[j].interface_num;
                        if (in >= 0 && in < 2 + 2 * WQ3D_MAX_VOLUME) ++verb_counts[in];
                    } else if (cb.add_eigenverb) {
                        cb.add_eigenverb(cb_ctx, &verbs[j], &vpower[j * nf], (size_t)nf, verbs[j].interface_num);
                    }
                    ++iv;
                }
            }
            while (ie < order.size() && h_rec[order[ie]].step == step) {
                const size_t j = order[ie];
                if (cb.add_eigenray) {
                    cb.add_eigenray(cb_ctx, (size_t)h_rec[j].t1, (size_t)h_rec[j].t2, &h_rec[j],
                                    &h_rinten[j * nf], &h_rphase[j * nf], (size_t)nf, run_id);
                } else {
                    pending.rec.push_back(h_rec[j]);
                    pending.inten.insert(pending.inten.end(), &h_rinten[j * nf], &h_rinten[j * nf] + nf);
                    pending.phase.insert(pending.phase.end(), &h_rphase[j * nf], &h_rphase[j * nf] + nf);
                    for (int m = 0; m < 3; ++m) pending.sens.push_back(h.sens ? h_rsens[j * 3 + m] : 0.0);
                }
                ++ie;
            }
            if (cb.check_eigenrays) cb.check_eigenrays(cb_ctx, ht[k + 1], run_id);
        }
        carry_refl.assign(refl.begin() + ir, refl.end());
        for (; iv < vorder.size(); ++iv) {
            const size_t j = vorder[iv];
            carry_verb.push_back(verbs[j]);
            carry_vpower.insert(carry_vpower.end(), &vpower[j * nf], &vpower[j * nf] + nf);
        }
    }

    /* Queues chunk K's work (result set p) on the stream without waiting
     * for it; "tail" also reflects the following chunk's first step. */
    int chunk_launch(int K, int p, bool tail) {
        int64_t* hb = h_base[p];
        double* ht = h_times[p];
        hb[0] = lsteps;
        ht[0] = ltime;
        for (int k = 0; k < K; ++k) ht[k + 1] = ht[k] + h.dt;
        WQ_CK(cudaMemcpyAsync(d_base, hb, sizeof(int64_t), cudaMemcpyHostToDevice, stream));
        WQ_CK(cudaMemcpyAsync(d_times, ht, (K + 1) * sizeof(double), cudaMemcpyHostToDevice, stream));
        WQ_CK(cudaMemsetAsync(d_counts, 0, 3 * sizeof(uint32_t), stream));
        WQ_CK(cudaMemsetAsync(d_counts + 8, 0, sizeof(uint32_t), stream));
        if (h.adj) WQ_CK(cudaMemsetAsync(d_counts + 11, 0, sizeof(uint32_t), stream));
        if (timing) tail = false;
        const int t = tail ? 1 : 0;
        /* the reflection schedule of this chunk, from the plan when tuned */
        const bool can_inline = !timing && !h.want_verbs && !volume_pass();
        bool inl = false, trial = false;
        size_t bucket = 0;
        if (can_inline) {
            if (refl_sched == WQ3D_REFLECT_INLINE) {
                inl = true;
            } else if (refl_sched == WQ3D_REFLECT_AUTO && !in_batch && !h.adj && K == chunk && lsteps > 0) {
                /* not a run's first chunk, whose start-up reflections are
                 * not typical */
                bucket = (size_t)(lsteps / TUNE_BUCKET);
                inl = tune_choose(tune_key(), bucket, &trial) != 0;
            } else if (refl_sched == WQ3D_REFLECT_AUTO && !in_batch && !h.adj) {
                inl = last_inl > 0;
            }
        }
        last_inl = inl ? 1 : 0;
        const int m = inl ? 1 : 0;
        chunk_trial[p] = trial;
        chunk_inl[p] = m;
        chunk_bucket[p] = bucket;
        if (!timing && K == chunk) build_graph(p, tail, inl);
        /* a trial times the chunk's device work only: its start is marked
         * after any graph building on the host */
        if (trial) {
            for (int e = 0; e < 2; ++e)
                if (!tune_ev[p][e]) WQ_CK(cudaEventCreate(&tune_ev[p][e]));
            WQ_CK(cudaEventRecord(tune_ev[p][0], stream));
        }
        if (!timing && K == chunk && graph[p][t][m]) {
            WQ_CK(cudaGraphLaunch(graph[p][t][m], stream));
            launches += graph_launches[p][t][m];
        } else {
            launch_chunk(K, p, tail, inl);
        }
        if (trial) WQ_CK(cudaEventRecord(tune_ev[p][1], stream));
        WQ_CK(cudaGetLastError());
        WQ_CK(cudaMemcpyAsync(h_counts[p], d_counts, 9 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        WQ_CK(cudaEventRecord(done_ev[p], stream));
        lsteps += K;
        ltime = ht[K];
        return WQ3D_OK;
    }

    /* Waits for chunk K of result set p (the oldest one in flight), reads
     * its records back and delivers them. */
    int chunk_finish(int K, int p) {
        WQ_CK(cudaEventSynchronize(done_ev[p]));
        if (chunk_trial[p]) {
            chunk_trial[p] = false;
            float ms = 0.0f;
            const bool ok = cudaEventElapsedTime(&ms, tune_ev[p][0], tune_ev[p][1]) == cudaSuccess;
            tune_record(tune_key(), chunk_bucket[p], chunk_inl[p], ok, ms);
        }
        if (timing) {
            WQ_CK(cudaStreamSynchronize(side));
            float r0 = 0;
            cudaEventElapsedTime(&r0, events[7 * K], events[7 * K + 1]);
            ms_refl += r0;
            for (int k = 0; k < K; ++k) {
                float a = 0, b = 0, c = 0, r = 0;
                cudaEventElapsedTime(&a, events[7 * k], events[7 * k + 1]);
                cudaEventElapsedTime(&b, events[7 * k + 2], events[7 * k + 3]);
                cudaEventElapsedTime(&c, events[7 * k + 3], events[7 * k + 4]);
                if (k + 1 < K) cudaEventElapsedTime(&r, events[7 * k + 5], events[7 * k + 6]);
                ms_step += a;
                ms_cpa += b;
                ms_eig += c;
                ms_refl += r;
            }
        }
        const QueueDev d = dev(p);
        const uint32_t* hc = h_counts[p];
        const uint32_t nrec = std::min(hc[0], h.cap_rec);
        const uint32_t nrefl = std::min(hc[1], h.cap_refl);
        const uint32_t err = hc[2];
        const uint32_t nverb = h.want_verbs ? std::min(hc[8], h.cap_verb) : 0;
        const uint32_t verbs_made = h.want_verbs ? hc[8] : 0;
        auto get = [&](void* dst, const void* src, size_t bytes) {
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, copy);
        };
        if (nrec > 0) {
            if (h_rec.size() < nrec) {
                h_rec.resize(nrec);
                h_rinten.resize((size_t)nrec * h.nf);
                h_rphase.resize((size_t)nrec * h.nf);
            }
            WQ_CK(get(h_rec.data(), d.rec, nrec * sizeof(wq3d_eigenray)));
            WQ_CK(get(h_rinten.data(), d.rec_inten, (size_t)nrec * h.nf * sizeof(double)));
            WQ_CK(get(h_rphase.data(), d.rec_phase, (size_t)nrec * h.nf * sizeof(double)));
            if (h.sens) {
                if (h_rsens.size() < (size_t)nrec * 3) h_rsens.resize((size_t)nrec * 3);
                WQ_CK(get(h_rsens.data(), d.rec_sens, (size_t)nrec * 3 * sizeof(double)));
            }
        }
        if (nrefl > 0) {
            if (h_refl.size() < nrefl) h_refl.resize(nrefl);
            WQ_CK(get(h_refl.data(), d.refl, nrefl * sizeof(wq3d_reflection)));
        }
        if (nverb > 0) {
            if (h_verb.size() < nverb) {
                h_verb.resize(nverb);
                h_vpower.resize((size_t)nverb * h.nf);
            }
            WQ_CK(get(h_verb.data(), d.verb, nverb * sizeof(wq3d_eigenverb)));
            WQ_CK(get(h_vpower.data(), d.verb_power, (size_t)nverb * h.nf * sizeof(double)));
        }
        WQ_CK(cudaStreamSynchronize(copy));
        deliver(K, nrec, nrefl, nverb, h_times[p]);
        if (verbs_made > h.cap_verb / 2) grow_verb = std::max(grow_verb, 4 * (size_t)verbs_made);
        if (h.want_refl && hc[1] > h.cap_refl / 2) grow_refl = std::max(grow_refl, 4 * (size_t)hc[1]);
        steps += K;
        time = h_times[p][K];
        if (err & (ERR_CAND_OVERFLOW | ERR_REC_OVERFLOW | ERR_REFL_OVERFLOW | ERR_VERB_OVERFLOW))
            return fail(WQ3D_ERR_OVERFLOW, "eigenray, reflection or eigenverb buffer overflow (error bits " +
                                               std::to_string(err) + "); recreate the queue with a larger eigenray_capacity");
        if (err & ERR_ADJ_OVERFLOW)
            return fail(WQ3D_ERR_OVERFLOW, "adjoint checkpoint or eigenray record buffer full (error bits " +
                                               std::to_string(err) + "); enable the adjoint with larger limits");
        if (err & ERR_NONFINITE)
            return fail(WQ3D_ERR_NUMERIC, "a ray's position or direction became NaN or Inf (error bits " +
                                              std::to_string(err) + "); check the ocean's profile and boundaries");
        if (err & ERR_BAD_CANDIDATE)
            return fail(WQ3D_ERR_CUDA, "internal error: an eigenray candidate named a ray or target outside "
                                       "the fan (error bits " + std::to_string(err) + ")");
        if (err & ERR_BOUNDS)
            return fail(WQ3D_ERR_CUDA, "internal error: a bounds check of the checked build failed (error bits " +
                                           std::to_string(err) + ")");
        if (err & ERR_SLOT_OVERFLOW)
            return fail(WQ3D_ERR_CUDA, "internal error: more reflecting rays in a step than rays (error bits " +
                                           std::to_string(err) + ")");
        if (err)
            return fail(WQ3D_ERR_NUMERIC, "kernel iteration bound reached (error bits " + std::to_string(err) + ")");
        return WQ3D_OK;
    }

    /* nsteps steps in chunks.  Without per-kernel timing, chunk c+1 is
     * queued before chunk c is delivered (result sets alternate), so the
     * device does not wait for the host between chunks.  Each chunk but
     * the last reflects the next one's first step.  A record buffer that a
     * chunk filled past half grows once nothing is in flight.  An error or
     * an abort stops further launches; the chunks already in flight are
     * still delivered, and the first error is returned. */
    int run_steps(size_t nsteps) {
        const bool pipe = !timing && nsteps > (size_t)chunk && ensure_set1();
        const size_t depth = pipe ? 2 : 1;
        int K_in[2] = {0, 0}, p_in[2] = {0, 0};
        size_t n_in = 0;
        int next_p = 0;
        int rc = WQ3D_OK;
        size_t left = nsteps;
        for (;;) {
            if (n_in == 0 && !rc && (grow_verb || grow_refl)) rc = apply_growth();
            while (left > 0 && !rc && n_in < depth && !grow_verb && !grow_refl) {
                if (abort_flag.exchange(false)) {
                    rc = fail(WQ3D_ERR_ABORTED, "aborted by caller");
                    break;
                }
                const int K = (int)std::min<size_t>(left, (size_t)chunk);
                left -= (size_t)K;
                const int r = chunk_launch(K, next_p, left > 0);
                if (r) {
                    rc = r;
                    break;
                }
                K_in[n_in] = K;
                p_in[n_in] = next_p;
                ++n_in;
                if (pipe) next_p ^= 1;
            }
            if (n_in == 0) {
                if (left > 0 && !rc && (grow_verb || grow_refl)) continue;
                break;
            }
            const int r = chunk_finish(K_in[0], p_in[0]);
            if (r && !rc) rc = r;
            K_in[0] = K_in[1];
            p_in[0] = p_in[1];
            --n_in;
        }
        return rc;
    }

    /* steps of the reference loop "while (time() < time_max) step();" */
    size_t steps_until(double time_max) const {
        size_t n = 0;
        double t = time;
        while (t < time_max) {
            t += h.dt;
            ++n;
        }
        return n;
    }
};

extern "C" {

const char* wq3d_last_error_string(void) { return g_err.c_str(); }

/* Internal hooks for the other source files of the library. */
void wq3d_internal_set_error(const char* msg) { g_err = msg ? msg : ""; }

/* An ocean's device arrays live on the device that was current when it
 * was created; using them with another device current would hand kernels
 * pointers into a different GPU's memory. */
static int ocean_device_check(const wq3d_ocean* o, int device) {
    if (device != o->device)
        return fail(WQ3D_ERR_INVALID, "the ocean was created on device " + std::to_string(o->device) +
                                          " and cannot be used on device " + std::to_string(device));
    return WQ3D_OK;
}

static int ocean_on_current_device(const wq3d_ocean* o) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(WQ3D_ERR_CUDA, "cudaGetDevice failed");
    return ocean_device_check(o, dev);
}

int wq3d_internal_ocean_model(const wq3d_ocean* ocean, OceanDev* out) {
    if (!ocean || !out) return fail(WQ3D_ERR_INVALID, "null argument");
    const int rc = ocean_on_current_device(ocean);
    if (rc) return rc;
    *out = ocean->dev;
    return WQ3D_OK;
}
int wq3d_abi_version(void) { return WQ3D_ABI_VERSION; }

int wq3d_device_count(int* count) {
    if (!count) return fail(WQ3D_ERR_INVALID, "null count");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *count = 0;
        return fail(WQ3D_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    }
    *count = n;
    return WQ3D_OK;
}

int wq3d_ocean_create(const wq3d_ocean_desc* d, wq3d_ocean** out) {
    if (!d || !out) return fail(WQ3D_ERR_INVALID, "null argument");
    if (d->profile.kind < WQ3D_PROFILE_LINEAR || d->profile.kind > WQ3D_PROFILE_GRID)
        return fail(WQ3D_ERR_UNSUPPORTED, "profile kind not supported by this build");
    for (const wq3d_boundary_desc* b : {&d->surface, &d->bottom})
        if (b->kind < WQ3D_BOUNDARY_FLAT || b->kind > WQ3D_BOUNDARY_GRID)
            return fail(WQ3D_ERR_UNSUPPORTED, "boundary kind not supported by this build");
    int cur_dev = 0;
    if (cudaGetDevice(&cur_dev) != cudaSuccess) return fail(WQ3D_ERR_CUDA, "no CUDA device is available");
    wq3d_ocean* o = new wq3d_ocean();
    o->device = cur_dev;
    std::memset(&o->dev, 0, sizeof(o->dev));
    ProfileDev& p = o->dev.prof;
    p.kind = d->profile.kind;
    for (int k = 0; k < 4; ++k) p.p[k] = d->profile.p[k];
    p.munk_k = -p.p[3] * p.p[2] * 2.0 / p.p[1];
    p.n2_factor = 2.0 * p.p[1] / p.p[0];
    p.flat_earth = d->profile.flat_earth;
    p.atten = d->profile.attenuation;
    p.atten_coef = d->profile.attenuation_coef;
    setup_boundary(o->dev.surf, d->surface, d->earth_radius);
    setup_boundary(o->dev.bot, d->bottom, d->earth_radius);
    if (d->num_volume < 0 || d->num_volume > WQ3D_MAX_VOLUME) {
        delete o;
        return fail(WQ3D_ERR_INVALID, "num_volume must be 0.." + std::to_string(WQ3D_MAX_VOLUME));
    }
    /* volume_flat.h:32-37: the layer's rho under the construction radius */
    o->dev.nvol = d->num_volume;
    for (int k = 0; k < d->num_volume; ++k) o->dev.vol_rho[k] = d->earth_radius - std::abs(d->volume[k].depth);
    o->host = o->dev;
    int rc = WQ3D_OK;
    if (p.kind == WQ3D_PROFILE_GRID)
        rc = make_grid(o, d->profile.grid, 3, &o->host.prof.grid, &o->dev.prof.grid);
    if (!rc && d->surface.kind == WQ3D_BOUNDARY_GRID)
        rc = make_grid(o, d->surface.grid, 2, &o->host.surf.grid, &o->dev.surf.grid);
    if (!rc && d->bottom.kind == WQ3D_BOUNDARY_GRID)
        rc = make_grid(o, d->bottom.grid, 2, &o->host.bot.grid, &o->dev.bot.grid);
    if (rc) {
        const std::string msg = g_err;
        delete o;
        g_err = msg;
        return rc;
    }
    o->build_radius = d->earth_radius;
    *out = o;
    return WQ3D_OK;
}

int wq3d_ocean_destroy(wq3d_ocean* o) {
    delete o;
    return WQ3D_OK;
}

static int eval_points(size_t n, std::vector<double*>& dev_in, const std::vector<const double*>& host_in) {
    for (size_t k = 0; k < host_in.size(); ++k) {
        double* p = nullptr;
        WQ_CK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(double)));
        dev_in.push_back(p);
        if (host_in[k])
            WQ_CK(cudaMemcpy(p, host_in[k], n * sizeof(double), cudaMemcpyHostToDevice));
        else
            WQ_CK(cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(double)));
    }
    return WQ3D_OK;
}

int wq3d_ocean_sound_speed(const wq3d_ocean* o, double R, size_t n, const double* rho,
                           const double* theta, const double* phi, double* speed, double* grad) {
    if (!o || !rho || !speed) return fail(WQ3D_ERR_INVALID, "null argument");
    if (ocean_on_current_device(o)) return WQ3D_ERR_INVALID;
    std::vector<double*> d;
    int rc = eval_points(n, d, {rho, theta, phi});
    double *dc = nullptr, *dg = nullptr;
    if (!rc && cudaMalloc(&dc, std::max<size_t>(n, 1) * sizeof(double)) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && cudaMalloc(&dg, std::max<size_t>(3 * n, 1) * sizeof(double)) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && n > 0) {
        k_sound_speed<<<(unsigned)((n + 127) / 128), 128>>>(o->dev, R, (int)n, d[0], d[1], d[2], dc, dg);
        if (cudaMemcpy(speed, dc, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) rc = WQ3D_ERR_CUDA;
        if (!rc && grad && cudaMemcpy(grad, dg, 3 * n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = WQ3D_ERR_CUDA;
    }
    for (double* p : d) cudaFree(p);
    cudaFree(dc);
    cudaFree(dg);
    if (rc) return fail(rc, "wq3d_ocean_sound_speed failed");
    return WQ3D_OK;
}

int wq3d_ocean_height(const wq3d_ocean* o, int which, size_t n, const double* rho,
                      const double* theta, const double* phi, double* height, double* normal) {
    if (!o || !theta || !phi || !height) return fail(WQ3D_ERR_INVALID, "null argument");
    if (ocean_on_current_device(o)) return WQ3D_ERR_INVALID;
    (void)rho;
    std::vector<double*> d;
    int rc = eval_points(n, d, {theta, phi});
    double *dh = nullptr, *dn = nullptr;
    if (!rc && cudaMalloc(&dh, std::max<size_t>(n, 1) * sizeof(double)) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && cudaMalloc(&dn, std::max<size_t>(3 * n, 1) * sizeof(double)) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && n > 0) {
        k_height<<<(unsigned)((n + 127) / 128), 128>>>(which == 0 ? o->dev.surf : o->dev.bot, (int)n, d[0],
                                                        d[1], dh, dn);
        if (cudaMemcpy(height, dh, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) rc = WQ3D_ERR_CUDA;
        if (!rc && normal && cudaMemcpy(normal, dn, 3 * n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = WQ3D_ERR_CUDA;
    }
    for (double* p : d) cudaFree(p);
    cudaFree(dh);
    cudaFree(dn);
    if (rc) return fail(rc, "wq3d_ocean_height failed");
    return WQ3D_OK;
}

int wq3d_ocean_attenuation(const wq3d_ocean* o, double earth_radius, size_t n, const double* rho,
                           const double* distance, size_t nf, const double* freq, double* attenuation) {
    if (!o || !rho || !distance || !freq || !attenuation) return fail(WQ3D_ERR_INVALID, "null argument");
    if (ocean_on_current_device(o)) return WQ3D_ERR_INVALID;
    if (n == 0 || nf == 0) return WQ3D_OK;
    std::vector<double> alpha(nf);
    thorp_alpha(freq, nf, alpha.data());
    std::vector<double*> d;
    int rc = eval_points(n, d, {rho, distance});
    double *df = nullptr, *dal = nullptr, *da = nullptr;
    if (!rc && cudaMalloc(&df, nf * sizeof(double)) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && cudaMalloc(&dal, nf * sizeof(double)) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && cudaMalloc(&da, n * nf * sizeof(double)) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && cudaMemcpy(df, freq, nf * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && cudaMemcpy(dal, alpha.data(), nf * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = WQ3D_ERR_CUDA;
    if (!rc) {
        k_attenuation<<<(unsigned)((n + 127) / 128), 128>>>(o->dev.prof, earth_radius, (int)n, d[0], d[1],
                                                             (int)nf, df, dal, da);
        if (cudaGetLastError() != cudaSuccess) rc = WQ3D_ERR_CUDA;
    }
    if (!rc && cudaMemcpy(attenuation, da, n * nf * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = WQ3D_ERR_CUDA;
    for (double* p : d) cudaFree(p);
    cudaFree(df);
    cudaFree(dal);
    cudaFree(da);
    if (rc) return fail(rc, "wq3d_ocean_attenuation failed");
    return WQ3D_OK;
}

int wq3d_ocean_reflect_loss(const wq3d_ocean* o, int which, size_t n, const double* rho,
                            const double* theta, const double* phi, const double* grazing,
                            size_t nf, const double* freq, double* amplitude, double* phase) {
    if (!o || !grazing || !freq || !amplitude) return fail(WQ3D_ERR_INVALID, "null argument");
    if (ocean_on_current_device(o)) return WQ3D_ERR_INVALID;
    (void)rho;
    (void)theta;
    (void)phi;
    std::vector<double*> d;
    int rc = eval_points(n, d, {grazing});
    double *df = nullptr, *da = nullptr, *dp = nullptr;
    if (!rc && cudaMalloc(&df, std::max<size_t>(nf, 1) * sizeof(double)) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && cudaMalloc(&da, std::max<size_t>(n * nf, 1) * sizeof(double)) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && cudaMalloc(&dp, std::max<size_t>(n * nf, 1) * sizeof(double)) != cudaSuccess) rc = WQ3D_ERR_CUDA;
    if (!rc && n > 0) {
        cudaMemcpy(df, freq, nf * sizeof(double), cudaMemcpyHostToDevice);
        k_reflect_loss<<<(unsigned)((n + 127) / 128), 128>>>(which == 0 ? o->dev.surf : o->dev.bot, (int)n,
                                                              d[0], (int)nf, df, da, dp);
        if (cudaMemcpy(amplitude, da, n * nf * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = WQ3D_ERR_CUDA;
        if (!rc && phase && cudaMemcpy(phase, dp, n * nf * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = WQ3D_ERR_CUDA;
    }
    for (double* p : d) cudaFree(p);
    cudaFree(df);
    cudaFree(da);
    cudaFree(dp);
    if (rc) return fail(rc, "wq3d_ocean_reflect_loss failed");
    return WQ3D_OK;
}

/* Destroyed queues kept for reuse.  A propagation loop that creates a
 * queue, runs it and destroys it spends most of its host time allocating
 * and freeing device buffers, instantiating CUDA graphs and freeing them
 * again; wq3d_queue_destroy instead parks a queue whose buffers have their
 * creation sizes, and wq3d_queue_create takes one of the same shape (device,
 * fan, frequencies, targets, eigenray capacity), uploads the new inputs into
 * its buffers and runs the start-up.  The chunk graphs are kept when the
 * new queue's descriptor equals the old one.  A reused queue computes what
 * a fresh one would, bit for bit. */
namespace {
std::mutex g_cache_mu;
std::vector<wq3d_queue*>* g_cache = new std::vector<wq3d_queue*>();
size_t g_cache_max = 2;

bool cacheable(const wq3d_queue* q) {
    const QueueDev& h = q->h;
    return !h.sens && !h.adj && !h.verb && !q->set1.verb && h.cap_refl == 4096 && q->stream;
}

wq3d_queue* cache_take(int device, size_t nde, size_t naz, size_t nf, size_t nt1, size_t nt2, uint32_t cap_cand) {
    std::lock_guard<std::mutex> lock(g_cache_mu);
    for (size_t k = 0; k < g_cache->size(); ++k) {
        wq3d_queue* q = (*g_cache)[k];
        const QueueDev& h = q->h;
        if (q->device == device && (size_t)h.nde == nde && (size_t)h.naz == naz && (size_t)h.nf == nf &&
            (size_t)h.nt1 == (h.nt ? nt1 : 0) && (size_t)h.nt2 == (h.nt ? nt2 : 1) && h.cap_cand == cap_cand &&
            ((h.nt == 0) == (nt1 * nt2 == 0))) {
            g_cache->erase(g_cache->begin() + k);
            return q;
        }
    }
    return nullptr;
}
}  // namespace

int wq3d_set_queue_cache(size_t max_queues) {
    std::vector<wq3d_queue*> drop;
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        g_cache_max = max_queues;
        while (g_cache->size() > g_cache_max) {
            drop.push_back(g_cache->front());
            g_cache->erase(g_cache->begin());
        }
    }
    for (wq3d_queue* q : drop) {
        DeviceGuard guard(q->device);
        delete q;
    }
    return WQ3D_OK;
}

int wq3d_queue_create(const wq3d_ocean* ocean, const wq3d_queue_desc* d, wq3d_queue** out) {
    if (!ocean || !d || !out) return fail(WQ3D_ERR_INVALID, "null argument");
    if (d->num_de < 1 || d->num_az < 1 || !d->de || !d->az || !d->de_inc || !d->az_inc)
        return fail(WQ3D_ERR_INVALID, "ray fan must hold at least one D/E and one AZ angle");
    if (d->num_freq < 1 || !d->freq) return fail(WQ3D_ERR_INVALID, "at least one frequency is required");
    if (d->num_freq > (size_t)MAX_FREQ) return fail(WQ3D_ERR_UNSUPPORTED, "more than 64 frequencies");
    if (d->num_az > (size_t)MAX_AZ) return fail(WQ3D_ERR_UNSUPPORTED, "more than 4096 AZ angles");
    if (!(d->time_step > 0.0)) return fail(WQ3D_ERR_INVALID, "time_step must be positive");
    if (d->precision != WQ3D_FP64 && d->precision != WQ3D_FP32C && d->precision != WQ3D_FP32)
        return fail(WQ3D_ERR_INVALID, "precision must be WQ3D_FP64, WQ3D_FP32C or WQ3D_FP32");
    const size_t n = d->num_de * d->num_az;
    if (n > (size_t)0x7fffffff) return fail(WQ3D_ERR_INVALID, "ray fan too large");
    const size_t nt = (d->targets && d->num_targets1 * d->num_targets2 > 0)
                          ? d->num_targets1 * d->num_targets2 : 0;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(WQ3D_ERR_CUDA, "no CUDA device is available");
    if (d->device < 0 || d->device >= ndev) return fail(WQ3D_ERR_INVALID, "device ordinal out of range");
    if (ocean_device_check(ocean, d->device)) return WQ3D_ERR_INVALID;
    DeviceGuard guard(d->device);

    const uint32_t cap_cand = (uint32_t)(d->eigenray_capacity ? d->eigenray_capacity
                                                              : std::max<size_t>(4096, 32 * nt));
    wq3d_queue* q = cache_take(d->device, d->num_de, d->num_az, d->num_freq, d->num_targets1, d->num_targets2,
                               cap_cand);
    const bool reuse = q != nullptr;
    QueueDev old_h{};
    if (reuse) {
        /* the run state of a fresh queue; the device buffers stay */
        old_h = q->h;
        q->reuse = true;
        q->time = q->ltime = 0.0;
        q->steps = q->lsteps = 0;
        q->carry_refl.clear();
        q->carry_verb.clear();
        q->carry_vpower.clear();
        q->cb = wq3d_callbacks{};
        q->cb_ctx = nullptr;
        q->pending = PendingRays{};
        q->abort_flag = false;
        q->timing = false;
        q->ms_step = q->ms_cpa = q->ms_eig = q->ms_total = q->ms_refl = 0.0;
        q->launches = 0;
        q->grow_verb = q->grow_refl = 0;
        q->count_verbs = false;
        for (auto& c : q->verb_counts) c = 0;
        q->refl_sched = WQ3D_REFLECT_AUTO;
        q->last_inl = -1;
        q->in_batch = false;
        q->chunk_trial[0] = q->chunk_trial[1] = false;
    } else {
        q = new wq3d_queue();
    }
    q->device = d->device;
    q->run_id = d->run_id;
    QueueDev& h = q->h;
    if (!reuse) std::memset(&h, 0, sizeof(h));
    h.oc = ocean->dev;
    h.nde = (int)d->num_de;
    h.naz = (int)d->num_az;
    h.nf = (int)d->num_freq;
    h.n = (int)n;
    h.nt = (int)nt;
    h.nt1 = nt ? (int)d->num_targets1 : 0;
    h.nt2 = nt ? (int)d->num_targets2 : 1;
    h.dt = d->time_step;
    h.R = d->earth_radius;
    h.spreading = d->spreading;
    h.precision = d->precision;
    h.intensity_threshold = 300.0;
    h.max_bottom = h.max_surface = h.max_caustic = h.max_upper = h.max_lower = 999;

    auto cleanup = [&](int rc) {
        std::string msg = g_err;
        delete q;
        g_err = msg;
        return rc;
    };
    int rc = 0;
    if (!reuse && cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(WQ3D_ERR_CUDA, "cudaStreamCreate failed"));

    /* host-side inputs */
    const size_t nde = d->num_de, naz = d->num_az, nf = d->num_freq;
    std::vector<double> freq(d->freq, d->freq + nf);
    std::vector<double> de(d->de, d->de + nde), de_inc(d->de_inc, d->de_inc + nde);
    std::vector<double> az(d->az, d->az + naz), az_inc(d->az_inc, d->az_inc + naz);

    /* wave_queue.cc:47-53 */
    h.az_boundary = 0;
    if (naz > 1) {
        const double a0 = std::abs(az[0]), a1 = std::abs(az[naz - 1]);
        h.az_boundary = (std::fmod(a0 + 360.0, 360.0) == std::fmod(a1 + 360.0, 360.0)) ? 1 : 0;
    }
    /* wave_queue.cc:58-68: the clamp changes source_pos() only; init_wave
     * receives the caller's position (wave_queue.cc:83) */
    const OceanDev& hoc = ocean->host;
    for (int k = 0; k < 3; ++k) h.source[k] = q->src_clamped[k] = d->source[k];
    {
        const double offset = 0.1;
        double bottom_rho = boundary_height(hoc.bot, d->source[1], d->source[2]) + offset;
        if (q->src_clamped[0] - h.R > -offset) {
            q->src_clamped[0] = -offset + h.R;
        } else if (q->src_clamped[0] < bottom_rho) {
            q->src_clamped[0] = bottom_rho;
        }
    }
    {
        double g3[3];
        sound_speed(hoc.prof, h.R, d->source[0], d->source[1], d->source[2], &h.c_source, g3);
    }
    std::vector<double> cos_de(nde), sin_de(nde), cos_az(naz), sin_az(naz);
    for (size_t i = 0; i < nde; ++i) {
        cos_de[i] = std::cos(to_radians(de[i]));
        sin_de[i] = std::sin(to_radians(de[i]));
    }
    for (size_t i = 0; i < naz; ++i) {
        cos_az[i] = std::cos(to_radians(az[i]));
        sin_az[i] = std::sin(to_radians(az[i]));
    }
    std::vector<double> alpha(nf);
    thorp_alpha(freq.data(), nf, alpha.data());
    /* targets (wave_queue.cc:54-56, :363-369; spreading_hybrid_gaussian.cc:70-83) */
    std::vector<double> tr(nt), tt(nt), tp(nt), tsin(nt), tR2(nt), t2R(nt), tc(nt), tspread(nt * nf);
    std::vector<uint8_t> tbranch(nt);
    const double slat = 90.0 - to_degrees(q->src_clamped[1]);
    const double slng = to_degrees(q->src_clamped[2]);
    for (size_t t = 0; t < nt; ++t) {
        tr[t] = d->targets[t];
        tt[t] = d->targets[nt + t];
        tp[t] = d->targets[2 * nt + t];
        tsin[t] = std::sin(tt[t]);
        tR2[t] = tr[t] * tr[t];
        t2R[t] = 2.0 * tr[t];
        double g3[3];
        sound_speed(hoc.prof, h.R, tr[t], tt[t], tp[t], &tc[t], g3);
        for (size_t k = 0; k < nf; ++k) {
            const double s = 2.0 * M_PI * tc[t] / freq[k];
            tspread[t * nf + k] = s * s;
        }
        const double tlat = 90.0 - to_degrees(tt[t]);
        const double tlng = to_degrees(tp[t]);
        tbranch[t] = (std::abs(slat - tlat) < 1e-4 && std::abs(slng - tlng) < 1e-4) ? 1 : 0;
    }
    /* spreading normalisation (spreading_hybrid_gaussian.cc:28-59,
     * spreading_ray.cc:26-45) */
    std::vector<double> norm_de(nde, 0.0), norm_az(n, 0.0), init_area(n, 0.0);
    if (nde >= 3 && naz >= 3) {
        for (size_t dd = 0; dd < nde - 1; ++dd) {
            const double de1 = to_radians(de[dd]);
            const double de2 = to_radians(de[dd + 1]);
            norm_de[dd] = de2 - de1;
            for (size_t a = 0; a < naz - 1; ++a) {
                const double az1 = to_radians(az[a]);
                const double az2 = to_radians(az[a + 1]);
                init_area[dd * naz + a] = (std::sin(de2) - std::sin(de1)) * (az2 - az1);
                norm_az[dd * naz + a] = init_area[dd * naz + a] / norm_de[dd];
            }
            norm_az[dd * naz + naz - 1] = norm_az[dd * naz + naz - 2];
            init_area[dd * naz + naz - 1] = init_area[dd * naz + naz - 2];
        }
        norm_de[nde - 1] = norm_de[nde - 2];
        for (size_t a = 0; a < naz - 1; ++a) {
            init_area[(nde - 1) * naz + a] = init_area[(nde - 2) * naz + a];
            norm_az[(nde - 1) * naz + a] = norm_az[(nde - 2) * naz + a];
        }
        const double s = std::sqrt(2.0 * M_PI);
        for (auto& v : norm_de) v /= s;
        for (auto& v : norm_az) v /= s;
    }

    if ((rc = q->upload(&h.freq, freq)) || (rc = q->upload(&h.alpha, alpha)) ||
        (rc = q->upload(&h.de, de)) || (rc = q->upload(&h.de_inc, de_inc)) ||
        (rc = q->upload(&h.az, az)) || (rc = q->upload(&h.az_inc, az_inc)) ||
        (rc = q->upload(&h.cos_de, cos_de)) || (rc = q->upload(&h.sin_de, sin_de)) ||
        (rc = q->upload(&h.cos_az, cos_az)) || (rc = q->upload(&h.sin_az, sin_az)) ||
        (rc = q->upload(&h.tgt[0], tr)) || (rc = q->upload(&h.tgt[1], tt)) ||
        (rc = q->upload(&h.tgt[2], tp)) || (rc = q->upload(&h.tgt_sin, tsin)) ||
        (rc = q->upload(&h.tgt_R2, tR2)) || (rc = q->upload(&h.tgt_2R, t2R)) ||
        (rc = q->upload(&h.tgt_spread2, tspread)) || (rc = q->upload(&h.tgt_c, tc)) ||
        (rc = q->upload(&h.de_branch, tbranch)) || (rc = q->upload(&h.norm_de, norm_de)) ||
        (rc = q->upload(&h.norm_az, norm_az)) || (rc = q->upload(&h.init_area, init_area)))
        return cleanup(rc);

    /* wavefront ring: one allocation carved into 256-byte aligned arrays */
    {
        const size_t nd_arrays = 22 + 2 * nf;
        auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
        const size_t dbytes = al(n * sizeof(double));
        const size_t ibytes = al(n * sizeof(int32_t));
        const size_t bbytes = al(n);
        const size_t per_front = nd_arrays * dbytes + 5 * ibytes + bbytes;
        char* base = reuse ? q->ring : nullptr;
        if (!reuse && (rc = q->alloc(&base, RING * per_front + 2 * bbytes))) return cleanup(rc);
        q->ring = base;
        q->ring_bytes = RING * per_front + 2 * bbytes;
        /* only the reflection flags need zeros: the start-up writes every
         * field of the first four fronts and the counters and edge flags of
         * all five, and the first step writes the fifth before it is read
         * (zeroing the whole ring cost the 512-queue batch seconds of its
         * build) */
        if (cudaMemset(base + RING * per_front, 0, 2 * bbytes) != cudaSuccess)
            return cleanup(fail(WQ3D_ERR_CUDA, "cudaMemset failed"));
        char* p = base;
        auto dtake = [&](size_t count) {
            double* r = reinterpret_cast<double*>(p);
            p += al(count * sizeof(double));
            return r;
        };
        for (int f = 0; f < RING; ++f) {
            FrontPtrs& F = h.F[f];
            for (int k = 0; k < 3; ++k) {
                F.pos[k] = dtake(n);
                F.pg[k] = dtake(n);
                F.nd[k] = dtake(n);
                F.ng[k] = dtake(n);
                F.sg[k] = dtake(n);
            }
            F.c = dtake(n);
            F.dist = dtake(n);
            F.plen = dtake(n);
            for (int k = 0; k < 4; ++k) F.cpa[k] = dtake(n);
            F.atten = dtake(n * nf);
            F.phase = dtake(n * nf);
            int32_t** ints[5] = {&F.surface, &F.bottom, &F.caustic, &F.upper, &F.lower};
            for (auto ip : ints) {
                *ip = reinterpret_cast<int32_t*>(p);
                p += ibytes;
            }
            F.on_edge = reinterpret_cast<uint8_t*>(p);
            p += bbytes;
        }
        h.flag[0] = reinterpret_cast<uint8_t*>(p);
        p += bbytes;
        h.flag[1] = reinterpret_cast<uint8_t*>(p);
    }
    /* result buffers and chunk control */
    h.cap_cand = (uint32_t)(d->eigenray_capacity ? d->eigenray_capacity
                                                 : std::max<size_t>(4096, 32 * nt));
    h.cap_rec = (uint32_t)std::min<size_t>((size_t)h.cap_cand * q->chunk, (size_t)1 << 21);
    h.cap_refl = 4096; /* grown when a reflection listener asks */
    if (!reuse) {
        uint32_t* cand = nullptr;
        if ((rc = q->alloc(&cand, 2 * CAND_LISTS * (size_t)h.cap_cand))) return cleanup(rc);
        h.cand = cand;
        if ((rc = q->alloc(&h.rec, h.cap_rec)) || (rc = q->alloc(&h.rec_inten, (size_t)h.cap_rec * nf)) ||
            (rc = q->alloc(&h.rec_phase, (size_t)h.cap_rec * nf)) || (rc = q->alloc(&h.refl, h.cap_refl)))
            return cleanup(rc);
        if ((rc = q->alloc(&q->d_counts, 20)) || (rc = q->alloc(&q->d_base, 1)) ||
            (rc = q->alloc(&q->d_times, (size_t)q->chunk + 1)))
            return cleanup(rc);
    }
    h.n_rec = q->d_counts + 0;
    h.n_refl = q->d_counts + 1;
    h.err = q->d_counts + 2;
    h.n_cand = q->d_counts + 13; /* three lists: 13, 14, 15 */
    h.n_work[0] = q->d_counts + 4;
    h.n_work[1] = q->d_counts + 5;
    h.n_work_b[0] = q->d_counts + 9;
    h.n_work_b[1] = q->d_counts + 10;
    h.n_done = q->d_counts + 6;
    h.n_verb = q->d_counts + 8;
    h.n_slot = q->d_counts + 16; /* one per shadow set: 16, 17, 18 */
    h.want_verbs = 0;
    h.verb_threshold = 1e-30; /* wave_thresholds.h:40 */
    if (!reuse) {
        const size_t stride = 54 + 3 * nf;
        for (int p = 0; p < SHADOW_SETS; ++p)
            if ((rc = q->alloc(&h.shadow[p], n * stride)) || (rc = q->alloc(&h.shadow_cnt[p], 3 * n)) ||
                (rc = q->alloc(&h.shadow_slot[p], n)) || (rc = q->alloc(&h.commit_flag[p], n)))
                return cleanup(rc);
        if ((rc = q->alloc(&h.work[0], n)) || (rc = q->alloc(&h.work[1], n))) return cleanup(rc);
    }
    /* no ray reflected in the step before the first */
    for (int p = 0; p < SHADOW_SETS; ++p)
        if (cudaMemset(h.commit_flag[p], 0, n) != cudaSuccess)
            return cleanup(fail(WQ3D_ERR_CUDA, "cudaMemset failed"));
    h.d_base = q->d_base;
    h.d_times = q->d_times;
    h.want_refl = 0;
    {
        /* per result set: base step, counters, chunk times */
        const size_t set_bytes = 128 + (((size_t)q->chunk + 1) * sizeof(double) + 63) / 64 * 64;
        if (!reuse && cudaMallocHost(&q->pinned, 2 * set_bytes) != cudaSuccess)
            return cleanup(fail(WQ3D_ERR_NOMEM, "cudaMallocHost failed"));
        for (int s = 0; s < 2; ++s) {
            char* b = static_cast<char*>(q->pinned) + s * set_bytes;
            q->h_base[s] = reinterpret_cast<int64_t*>(b);
            q->h_counts[s] = reinterpret_cast<uint32_t*>(b + 64);
            q->h_times[s] = reinterpret_cast<double*>(b + 128);
        }
    }
    if (cudaMemset(q->d_counts, 0, 20 * sizeof(uint32_t)) != cudaSuccess)
        return cleanup(fail(WQ3D_ERR_CUDA, "cudaMemset failed"));

    /* wave_queue ctor: init_wave, update, init_wavefronts */
    q->gridded = ocean->dev.prof.kind == WQ3D_PROFILE_GRID || ocean->dev.surf.kind == WQ3D_BOUNDARY_GRID ||
                 ocean->dev.bot.kind == WQ3D_BOUNDARY_GRID;
    q->k_reflect_fn = q->gridded ? gridded::k_reflect : analytic::k_reflect;
    q->k_advance_fn = q->gridded ? gridded::k_advance : analytic::k_advance;
    q->k_advance_inline_fn = q->gridded ? gridded::k_advance_inline : analytic::k_advance_inline;
    (q->gridded ? gridded::k_startup : analytic::k_startup)<<<(unsigned)((n + 127) / 128), 128, 0, q->stream>>>(
        h);
    cudaError_t e = cudaStreamSynchronize(q->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cleanup(fail(WQ3D_ERR_CUDA, std::string("start-up kernel: ") + cudaGetErrorString(e)));
    /* spreading_ray.cc:44: sound speed of ray (0,0) on the first front */
    if (cudaMemcpy(&h.init_sound_speed, h.F[2].c, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return cleanup(fail(WQ3D_ERR_CUDA, "cudaMemcpy failed"));
    if (!reuse) {
        if (cudaEventCreate(&q->ev_begin) != cudaSuccess || cudaEventCreate(&q->ev_end) != cudaSuccess)
            return cleanup(fail(WQ3D_ERR_CUDA, "cudaEventCreate failed"));
        /* the reflections are the longest chain of a step (one thread per
         * reflecting ray): their blocks go first when SMs free up */
        int prio_low = 0, prio_high = 0;
        if (cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess) prio_high = 0;
        if (cudaStreamCreateWithPriority(&q->side, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
            cudaStreamCreateWithFlags(&q->eig, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&q->adv, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&q->copy, cudaStreamNonBlocking) != cudaSuccess)
            return cleanup(fail(WQ3D_ERR_CUDA, "cudaStreamCreate failed"));
        if (cudaEventCreateWithFlags(&q->eig_end, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&q->start_ev, cudaEventDisableTiming) != cudaSuccess)
            return cleanup(fail(WQ3D_ERR_CUDA, "cudaEventCreate failed"));
        for (auto& e : q->done_ev)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
                return cleanup(fail(WQ3D_ERR_CUDA, "cudaEventCreate failed"));
        for (auto* v : {&q->fork_ev, &q->join_ev, &q->adv_ev, &q->com_ev, &q->cpa_ev}) {
            v->resize(q->chunk);
            for (int k = 0; k < q->chunk; ++k)
                if (cudaEventCreateWithFlags(&(*v)[k], cudaEventDisableTiming) != cudaSuccess)
                    return cleanup(fail(WQ3D_ERR_CUDA, "cudaEventCreate failed"));
        }
    }
    /* the chunk graphs hold the descriptor by value */
    if (reuse && std::memcmp(&old_h, &h, sizeof(h)) != 0) q->drop_graph();
    q->reuse = false;
    /* set-up a run would otherwise do on its first chunks: the second
     * result set and the side-stream graphs of the chunks that reflect
     * the next chunk's first step (rebuilt later only if callbacks,
     * thresholds or sensitivities change the descriptor); the graphs of a
     * run's last full chunk and of the inline schedule are built when
     * first used */
    q->ensure_set1();
    for (int p = 0; p < (q->have_set1 ? 2 : 1); ++p) q->build_graph(p, true, false);
    *out = q;
    return WQ3D_OK;
}

int wq3d_queue_destroy(wq3d_queue* q) {
    if (!q) return WQ3D_OK;
    DeviceGuard guard(q->device);
    if (cacheable(q) && cudaStreamSynchronize(q->stream) == cudaSuccess &&
        cudaStreamSynchronize(q->side) == cudaSuccess && cudaStreamSynchronize(q->eig) == cudaSuccess &&
        cudaStreamSynchronize(q->adv) == cudaSuccess && cudaStreamSynchronize(q->copy) == cudaSuccess) {
        wq3d_queue* drop = nullptr;
        {
            std::lock_guard<std::mutex> lock(g_cache_mu);
            if (g_cache_max > 0) {
                q->pending = PendingRays{};
                g_cache->push_back(q);
                q = nullptr;
                if (g_cache->size() > g_cache_max) {
                    drop = g_cache->front();
                    g_cache->erase(g_cache->begin());
                }
            }
        }
        if (!q) {
            if (drop) {
                DeviceGuard g2(drop->device);
                delete drop;
            }
            return WQ3D_OK;
        }
    }
    delete q;
    return WQ3D_OK;
}

int wq3d_queue_set_thresholds(wq3d_queue* q, const wq3d_thresholds* t) {
    if (!q || !t) return fail(WQ3D_ERR_INVALID, "null argument");
    DeviceGuard guard(q->device);
    q->h.intensity_threshold = std::abs(t->intensity);
    q->h.max_bottom = t->max_bottom;
    q->h.max_surface = t->max_surface;
    q->h.max_caustic = t->max_caustic;
    q->h.max_upper = t->max_upper;
    q->h.max_lower = t->max_lower;
    q->h.verb_threshold = std::pow(10.0, -0.1 * std::abs(t->eigenverb)); /* wave_thresholds.h:87-89 */
    q->drop_graph();
    return WQ3D_OK;
}

static int apply_listener_wants(wq3d_queue* q);

int wq3d_queue_set_callbacks(wq3d_queue* q, const wq3d_callbacks* cb, void* ctx) {
    if (!q) return fail(WQ3D_ERR_INVALID, "null queue");
    DeviceGuard guard(q->device);
    if (cb)
        q->cb = *cb;
    else
        q->cb = wq3d_callbacks{};
    q->cb_ctx = ctx;
    return apply_listener_wants(q);
}

/* record buffers and descriptor flags for the notices someone will take */
static int apply_listener_wants(wq3d_queue* q) {
    const int want = q->cb.reflect ? 1 : 0;
    const int want_verbs = (q->cb.add_eigenverb || q->count_verbs) ? 1 : 0;
    if (want) {
        const int rc = q->ensure_refl_capacity((size_t)(q->chunk + 1) * q->h.n / 2);
        if (rc) return rc;
    }
    if (want_verbs && !q->h.verb) {
        /* eigenverb buffers, made the first time a listener asks */
        const int rc = q->ensure_verb_capacity((size_t)q->chunk * q->h.n * (q->h.oc.nvol + 1) / 2);
        if (rc) return rc;
    }
    if (want != q->h.want_refl || want_verbs != q->h.want_verbs) {
        q->h.want_refl = want;
        q->h.want_verbs = want_verbs;
        q->drop_graph();
    }
    return WQ3D_OK;
}

int wq3d_queue_count_eigenverbs(wq3d_queue* q, int on) {
    if (!q) return fail(WQ3D_ERR_INVALID, "null queue");
    DeviceGuard guard(q->device);
    q->count_verbs = on != 0;
    return apply_listener_wants(q);
}

int wq3d_queue_eigenverb_counts(const wq3d_queue* q, uint64_t* counts) {
    if (!q || !counts) return fail(WQ3D_ERR_INVALID, "null argument");
    for (int k = 0; k < 2 + 2 * WQ3D_MAX_VOLUME; ++k) counts[k] = q->verb_counts[k];
    return WQ3D_OK;
}

int wq3d_queue_step(wq3d_queue* q, size_t nsteps) {
    if (!q) return fail(WQ3D_ERR_INVALID, "null queue");
    DeviceGuard guard(q->device);
    if (nsteps == 0) return WQ3D_OK;
    WQ_CK(cudaEventRecord(q->ev_begin, q->stream));
    const int rc = q->run_steps(nsteps);
    WQ_CK(cudaEventRecord(q->ev_end, q->stream));
    WQ_CK(cudaEventSynchronize(q->ev_end));
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, q->ev_begin, q->ev_end) == cudaSuccess) q->ms_total += ms;
    return rc;
}

int wq3d_queue_run(wq3d_queue* q, double time_max, size_t* steps_done) {
    if (!q) return fail(WQ3D_ERR_INVALID, "null queue");
    const size_t n = q->steps_until(time_max);
    const int rc = wq3d_queue_step(q, n);
    if (steps_done) *steps_done = n;
    return rc;
}

int wq3d_batch_run(wq3d_queue* const* queues, size_t count, const double* time_max, size_t* steps_done,
                   double* ms_device) {
    if (!queues || !time_max || count == 0) return fail(WQ3D_ERR_INVALID, "null argument or empty batch");
    for (size_t i = 0; i < count; ++i) {
        if (!queues[i]) return fail(WQ3D_ERR_INVALID, "null queue in batch");
        if (queues[i]->device != queues[0]->device) return fail(WQ3D_ERR_INVALID, "batch queues on different devices");
        for (size_t j = 0; j < i; ++j)
            if (queues[j] == queues[i]) return fail(WQ3D_ERR_INVALID, "queue listed twice in batch");
    }
    DeviceGuard guard(queues[0]->device);
    /* queues sharing the GPU keep their reflecting rays in compact
     * k_reflect launches (under WQ3D_REFLECT_AUTO) */
    struct BatchMark {
        wq3d_queue* const* qs;
        size_t n;
        BatchMark(wq3d_queue* const* q, size_t c) : qs(q), n(c) {
            for (size_t i = 0; i < n; ++i) qs[i]->in_batch = n > 1;
        }
        ~BatchMark() {
            for (size_t i = 0; i < n; ++i) qs[i]->in_batch = false;
        }
    } mark(queues, count);
    std::vector<size_t> left(count), K(count, 0);
    for (size_t i = 0; i < count; ++i) {
        left[i] = queues[i]->steps_until(time_max[i]);
        if (steps_done) steps_done[i] = left[i];
    }
    /* one start event that every queue's stream waits on, so the device
     * time of the batch is the latest queue end minus this start */
    cudaEvent_t start = nullptr;
    WQ_CK(cudaEventCreate(&start));
    WQ_CK(cudaEventRecord(start, queues[0]->stream));
    for (size_t i = 1; i < count; ++i) WQ_CK(cudaStreamWaitEvent(queues[i]->stream, start, 0));
    int rc = WQ3D_OK;
    bool any = true;
    while (any && !rc) {
        any = false;
        /* launch every unfinished queue's next chunk, then drain them in
         * turn: the host delivers one queue's results while the others run */
        for (size_t i = 0; i < count && !rc; ++i) {
            K[i] = 0;
            if (left[i] == 0) continue;
            if (queues[i]->abort_flag.exchange(false)) {
                rc = fail(WQ3D_ERR_ABORTED, "aborted by caller");
                break;
            }
            K[i] = std::min<size_t>(left[i], (size_t)queues[i]->chunk);
            rc = queues[i]->chunk_launch((int)K[i], 0, left[i] > K[i]);
            if (rc) K[i] = 0;
        }
        for (size_t i = 0; i < count; ++i) {
            if (K[i] == 0) continue;
            int r = queues[i]->chunk_finish((int)K[i], 0);
            if (!r) r = queues[i]->apply_growth();
            if (r && !rc) rc = r;
            left[i] -= K[i];
            any = any || left[i] > 0;
        }
    }
    float worst = 0.0f;
    for (size_t i = 0; i < count; ++i) {
        wq3d_queue* q = queues[i];
        cudaEventRecord(q->ev_end, q->stream);
        cudaEventSynchronize(q->ev_end);
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, start, q->ev_end) == cudaSuccess) {
            q->ms_total += ms;
            worst = std::max(worst, ms);
        }
    }
    cudaEventDestroy(start);
    if (ms_device) *ms_device = worst;
    return rc;
}

int wq3d_queue_time(const wq3d_queue* q, double* t) {
    if (!q || !t) return fail(WQ3D_ERR_INVALID, "null argument");
    *t = q->time;
    return WQ3D_OK;
}

int wq3d_queue_source(const wq3d_queue* q, double* s) {
    if (!q || !s) return fail(WQ3D_ERR_INVALID, "null argument");
    for (int k = 0; k < 3; ++k) s[k] = q->src_clamped[k];
    return WQ3D_OK;
}

int wq3d_queue_steps(const wq3d_queue* q, int64_t* steps) {
    if (!q || !steps) return fail(WQ3D_ERR_INVALID, "null argument");
    *steps = q->steps;
    return WQ3D_OK;
}

int wq3d_queue_get_front(wq3d_queue* q, int which, const wq3d_front_view* v) {
    if (!q || !v || which < 0 || which > 3) return fail(WQ3D_ERR_INVALID, "bad argument");
    DeviceGuard guard(q->device);
    const FrontPtrs& F = q->h.F[(q->steps + which) % RING];
    const size_t n = q->h.n, nf = q->h.nf;
    auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
        if (!dst) return WQ3D_OK;
        WQ_CK(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
        return WQ3D_OK;
    };
    int rc = 0;
    rc |= cp(v->rho, F.pos[0], n * 8);
    rc |= cp(v->theta, F.pos[1], n * 8);
    rc |= cp(v->phi, F.pos[2], n * 8);
    for (int k = 0; k < 3; ++k) {
        rc |= cp(v->pos_grad[k], F.pg[k], n * 8);
        rc |= cp(v->ndir[k], F.nd[k], n * 8);
        rc |= cp(v->ndir_grad[k], F.ng[k], n * 8);
        rc |= cp(v->sound_grad[k], F.sg[k], n * 8);
    }
    rc |= cp(v->sound_speed, F.c, n * 8);
    rc |= cp(v->distance, F.dist, n * 8);
    rc |= cp(v->path_length, F.plen, n * 8);
    rc |= cp(v->surface, F.surface, n * 4);
    rc |= cp(v->bottom, F.bottom, n * 4);
    rc |= cp(v->caustic, F.caustic, n * 4);
    rc |= cp(v->upper, F.upper, n * 4);
    rc |= cp(v->lower, F.lower, n * 4);
    rc |= cp(v->on_edge, F.on_edge, n);
    if (v->attenuation || v->phase) {
        std::vector<double> tmp(n * nf);
        for (int w = 0; w < 2; ++w) {
            double* dst = w ? v->phase : v->attenuation;
            if (!dst) continue;
            rc |= cp(tmp.data(), w ? F.phase : F.atten, n * nf * 8);
            for (size_t f = 0; f < nf; ++f)
                for (size_t i = 0; i < n; ++i) dst[i * nf + f] = tmp[f * n + i];
        }
    }
    return rc ? WQ3D_ERR_CUDA : WQ3D_OK;
}

int wq3d_queue_take_eigenrays(wq3d_queue* q, wq3d_eigenray* rays, double* inten, double* phase,
                              size_t capacity, size_t* count) {
    if (!q || !count) return fail(WQ3D_ERR_INVALID, "null argument");
    *count = q->pending.size();
    if (!rays) return WQ3D_OK;
    if (capacity < q->pending.size()) return fail(WQ3D_ERR_OVERFLOW, "capacity smaller than the pending count");
    const size_t nf = q->h.nf;
    const size_t n = q->pending.size();
    if (n > 0) {
        std::memcpy(rays, q->pending.rec.data(), n * sizeof(wq3d_eigenray));
        if (inten) std::memcpy(inten, q->pending.inten.data(), n * nf * sizeof(double));
        if (phase) std::memcpy(phase, q->pending.phase.data(), n * nf * sizeof(double));
    }
    q->pending.clear();
    return WQ3D_OK;
}

int wq3d_queue_enable_sensitivity(wq3d_queue* q) {
    if (!q) return fail(WQ3D_ERR_INVALID, "null queue");
    if (q->h.sens) return WQ3D_OK;
    if (q->steps != 0) return fail(WQ3D_ERR_INVALID, "enable sensitivities before the first step");
    DeviceGuard guard(q->device);
    const size_t n = (size_t)q->h.n;
    double* dA = nullptr;
    int rc = q->alloc(&dA, RING * 3 * n);
    if (!rc) rc = q->alloc(&q->h.rec_sens, (size_t)q->h.cap_rec * 3);
    if (!rc && q->have_set1) rc = q->alloc(&q->set1.rec_sens, (size_t)q->h.cap_rec * 3);
    if (rc) return rc;
    WQ_CK(cudaMemset(dA, 0, RING * 3 * n * sizeof(double)));
    for (int f = 0; f < RING; ++f) q->h.F[f].dA = dA + (size_t)f * 3 * n;
    q->h.sens = 1;
    q->drop_graph();
    return WQ3D_OK;
}

int wq3d_queue_enable_adjoint(wq3d_queue* q, int checkpoint_interval, size_t max_steps,
                              size_t max_eigenrays) {
    if (!q) return fail(WQ3D_ERR_INVALID, "null queue");
    if (q->h.adj) return fail(WQ3D_ERR_INVALID, "adjoint recording is already on");
    if (q->steps != 0 || q->lsteps != 0) return fail(WQ3D_ERR_INVALID, "enable the adjoint before the first step");
    if (checkpoint_interval < 1 || max_steps < 1) return fail(WQ3D_ERR_INVALID, "checkpoint interval and steps must be positive");
    const QueueDev& h = q->h;
    if (h.precision == WQ3D_FP32)
        return fail(WQ3D_ERR_UNSUPPORTED, "the adjoint retraces FP64 steps: use WQ3D_FP64 or WQ3D_FP32C");
    const ProfileDev& pr = h.oc.prof;
    if (pr.kind != WQ3D_PROFILE_GRID || pr.grid.ndim != 1 || pr.grid.interp[0] != WQ3D_INTERP_LINEAR)
        return fail(WQ3D_ERR_UNSUPPORTED, "the adjoint needs a profile_grid<1> with linear interpolation");
    if (pr.grid.ax[0].n < 2 || pr.grid.ax[0].n > ADJ_MAX_NODES)
        return fail(WQ3D_ERR_UNSUPPORTED, "the adjoint's profile has 2 to " + std::to_string(ADJ_MAX_NODES) + " nodes");
    for (const BoundaryDev* b : {&h.oc.surf, &h.oc.bot}) {
        if (b->kind != WQ3D_BOUNDARY_FLAT && b->kind != WQ3D_BOUNDARY_SLOPE)
            return fail(WQ3D_ERR_UNSUPPORTED, "the adjoint needs flat or sloped boundaries");
        if (b->loss.kind == WQ3D_LOSS_RAYLEIGH && (b->loss.rl_shr != 0.0 || b->loss.rl_satt != 0.0))
            return fail(WQ3D_ERR_UNSUPPORTED, "the adjoint's Rayleigh loss has no shear");
    }
    if (h.oc.nvol > 0) return fail(WQ3D_ERR_UNSUPPORTED, "the adjoint does not take volume layers");
    if (h.spreading != WQ3D_HYBRID_GAUSSIAN) return fail(WQ3D_ERR_UNSUPPORTED, "the adjoint needs hybrid Gaussian spreading");
    if (h.nt < 1) return fail(WQ3D_ERR_INVALID, "the adjoint needs targets");
    DeviceGuard guard(q->device);
    const size_t n = (size_t)h.n;
    const int nckpt = (int)(max_steps / (size_t)checkpoint_interval + 1);
    const size_t cap = max_eigenrays ? max_eigenrays : 65536;
    if (cap > UINT32_MAX / 2) return fail(WQ3D_ERR_INVALID, "max_eigenrays too large");
    double* ck = nullptr;
    AdjRec* rec = nullptr;
    int rc = q->alloc(&ck, (size_t)nckpt * ADJ_S * n);
    if (!rc) rc = q->alloc(&rec, cap);
    if (rc) return rc;
    WQ_CK(cudaMemset(q->d_counts + 11, 0, 2 * sizeof(uint32_t)));
    q->h.adj = 1;
    q->h.adj_K = checkpoint_interval;
    q->h.adj_nckpt = nckpt;
    q->h.adj_ckpt = ck;
    q->h.adj_rec = rec;
    q->h.adj_cap = (uint32_t)cap;
    q->h.adj_mark = q->d_counts + 11;
    q->h.adj_n = q->d_counts + 12;
    q->drop_graph();
    return WQ3D_OK;
}

namespace {
/* one unit seed on one ray's state component (wq3d_queue_adjoint_state) */
struct AdjUnitSeed {
    int ray;
    int64_t step;
    int comp;
};
}  // namespace

static int adjoint_sweep(wq3d_queue* q, const wq3d_eigenray* rays, const double* w_tl, const double* w_time,
                         size_t n_rays, double* grad, size_t num_nodes, double* ms, const AdjUnitSeed* xs);

int wq3d_queue_adjoint(wq3d_queue* q, const wq3d_eigenray* rays, const double* w_tl, const double* w_time,
                       size_t n_rays, double* grad, size_t num_nodes, double* ms) {
    return adjoint_sweep(q, rays, w_tl, w_time, n_rays, grad, num_nodes, ms, nullptr);
}

int wq3d_queue_adjoint_state(wq3d_queue* q, int ray, int64_t step, int component, double* grad,
                             size_t num_nodes) {
    if (!q || !grad) return fail(WQ3D_ERR_INVALID, "null argument");
    if (ray < 0 || ray >= q->h.n || component < 0 || component >= ADJ_L || step < 0 || step > q->steps)
        return fail(WQ3D_ERR_INVALID, "ray, step or state component out of range");
    const AdjUnitSeed xs{ray, step, component};
    return adjoint_sweep(q, nullptr, nullptr, nullptr, 0, grad, num_nodes, nullptr, &xs);
}

static int adjoint_sweep(wq3d_queue* q, const wq3d_eigenray* rays, const double* w_tl, const double* w_time,
                         size_t n_rays, double* grad, size_t num_nodes, double* ms, const AdjUnitSeed* xs) {
    if (!q || !grad) return fail(WQ3D_ERR_INVALID, "null argument");
    if (n_rays && (!rays || !w_tl || !w_time)) return fail(WQ3D_ERR_INVALID, "null argument");
    if (!q->h.adj) return fail(WQ3D_ERR_INVALID, "adjoint recording is off (wq3d_queue_enable_adjoint)");
    const QueueDev& h = q->h;
    const int nodes = h.oc.prof.grid.ax[0].n;
    if (num_nodes != (size_t)nodes)
        return fail(WQ3D_ERR_INVALID, "the profile has " + std::to_string(nodes) + " nodes");
    for (int j = 0; j < nodes; ++j) grad[j] = 0.0;
    if (ms) *ms = 0.0;
    const int64_t m_end = q->steps;
    if (m_end < 1 || (n_rays == 0 && !xs)) return WQ3D_OK;
    DeviceGuard guard(q->device);
    WQ_CK(cudaStreamSynchronize(q->stream));
    const size_t n = (size_t)h.n;
    const int K = h.adj_K;
    /* the records' keys, flags and spread partials, strided out of AdjRec */
    uint32_t nrec = 0;
    WQ_CK(cudaMemcpy(&nrec, h.adj_n, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    nrec = std::min(nrec, h.adj_cap);
    std::vector<int64_t> kstep(nrec);
    std::vector<int32_t> kti(2 * (size_t)nrec), kflags(nrec);
    std::vector<double> kds2(nrec);
    if (nrec > 0) {
        const size_t pitch = sizeof(AdjRec);
        WQ_CK(cudaMemcpy2D(kstep.data(), sizeof(int64_t), (const char*)h.adj_rec + offsetof(AdjRec, step), pitch,
                           sizeof(int64_t), nrec, cudaMemcpyDeviceToHost));
        WQ_CK(cudaMemcpy2D(kti.data(), 2 * sizeof(int32_t), (const char*)h.adj_rec + offsetof(AdjRec, t), pitch,
                           2 * sizeof(int32_t), nrec, cudaMemcpyDeviceToHost));
        WQ_CK(cudaMemcpy2D(kflags.data(), sizeof(int32_t), (const char*)h.adj_rec + offsetof(AdjRec, flags), pitch,
                           sizeof(int32_t), nrec, cudaMemcpyDeviceToHost));
        WQ_CK(cudaMemcpy2D(kds2.data(), sizeof(double), (const char*)h.adj_rec + offsetof(AdjRec, dTL_ds2), pitch,
                           sizeof(double), nrec, cudaMemcpyDeviceToHost));
    }
    /* weights per record, matched on (step, target, ray) */
    std::vector<size_t> order(nrec);
    for (size_t r = 0; r < nrec; ++r) order[r] = r;
    auto key = [&](size_t r) { return std::make_tuple(kstep[r], kti[2 * r], kti[2 * r + 1]); };
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return key(a) < key(b); });
    std::vector<double> w(2 * (size_t)nrec, 0.0);
    std::vector<double> gs2((size_t)h.nt, 0.0);
    for (size_t k = 0; k < n_rays; ++k) {
        const wq3d_eigenray& e = rays[k];
        const auto want = std::make_tuple((int64_t)e.step, (int32_t)(e.t1 * h.nt2 + e.t2), (int32_t)(e.de * h.naz + e.az));
        auto it = std::lower_bound(order.begin(), order.end(), want,
                                   [&](size_t r, const std::tuple<int64_t, int32_t, int32_t>& v) { return key(r) < v; });
        if (it == order.end() || key(*it) != want)
            return fail(WQ3D_ERR_INVALID, "eigenray " + std::to_string(k) + " was not recorded by this queue's adjoint");
        const size_t r = *it;
        if ((w_tl[k] != 0.0 || w_time[k] != 0.0) && !(kflags[r] & ADJ_VALID))
            return fail(WQ3D_ERR_NUMERIC, "eigenray " + std::to_string(k) + ": its beam walk outran the " +
                                              std::to_string(ADJ_MAX_CELLS) + " recorded cells");
        w[r] += w_tl[k];
        w[nrec + r] += w_time[k];
        gs2[kti[2 * r]] += w_tl[k] * kds2[r];
    }
    /* workspace */
    auto& W = q->adjw;
    int rc = WQ3D_OK;
    if (!W.seg) {
        if ((rc = q->alloc(&W.seg, (size_t)(K + 1) * ADJ_S * n)) || (rc = q->alloc(&W.chain, (size_t)(K + 1) * n)) ||
            (rc = q->alloc(&W.seed, (size_t)(K + 1) * ADJ_L * n)) || (rc = q->alloc(&W.lam, (size_t)ADJ_L * n)) ||
            (rc = q->alloc(&W.last, n)) || (rc = q->alloc(&W.grad, ADJ_MAX_NODES)) || (rc = q->alloc(&W.err, 1)))
            return rc;
    }
    if (W.w_cap < 2 * (size_t)nrec) {
        q->release(W.w);
        W.w = nullptr;
        if ((rc = q->alloc(&W.w, std::max<size_t>(2 * (size_t)nrec, 2)))) return rc;
        W.w_cap = std::max<size_t>(2 * (size_t)nrec, 2);
    }
    cudaStream_t st = q->stream;
    cudaEvent_t e0 = q->ev_begin, e1 = q->ev_end;
    if (!e0) WQ_CK(cudaEventCreate(&q->ev_begin));
    if (!e1) WQ_CK(cudaEventCreate(&q->ev_end));
    e0 = q->ev_begin;
    e1 = q->ev_end;
    double alpha0 = 0.0;
    WQ_CK(cudaMemcpy(&alpha0, h.alpha, sizeof(double), cudaMemcpyDeviceToHost));
    WQ_CK(cudaEventRecord(e0, st));
    if (nrec > 0) WQ_CK(cudaMemcpyAsync(W.w, w.data(), 2 * (size_t)nrec * sizeof(double), cudaMemcpyHostToDevice, st));
    WQ_CK(cudaMemsetAsync(W.last, 0, n * sizeof(int64_t), st));
    if (xs) {
        const int64_t biased = xs->step + 1;
        WQ_CK(cudaMemcpyAsync(W.last + xs->ray, &biased, sizeof(int64_t), cudaMemcpyHostToDevice, st));
    }
    WQ_CK(cudaMemsetAsync(W.lam, 0, (size_t)ADJ_L * n * sizeof(double), st));
    WQ_CK(cudaMemsetAsync(W.grad, 0, ADJ_MAX_NODES * sizeof(double), st));
    WQ_CK(cudaMemsetAsync(W.err, 0, sizeof(uint32_t), st));
    AdjSweep a{};
    a.m_end = m_end;
    a.nrec = (int)nrec;
    a.w_tl = W.w;
    a.w_t = W.w + nrec;
    a.seg = W.seg;
    a.chain = W.chain;
    a.seed = W.seed;
    a.lam = W.lam;
    a.last = W.last;
    a.grad = W.grad;
    a.nodes = nodes;
    a.alpha0 = alpha0;
    a.err = W.err;
    /* the recompute retraces the forward without notices or sensitivities */
    QueueDev qa = q->dev(0);
    qa.want_refl = 0;
    qa.want_verbs = 0;
    qa.sens = 0;
    const unsigned rb = (unsigned)((nrec + 127) / 128);
    const unsigned gb = (unsigned)((n + 127) / 128);
    if (nrec > 0) k_adj_touch<<<rb, 128, 0, st>>>(a, qa);
    /* checkpoints exist for the states the forward advanced from */
    const int64_t c_last = std::min<int64_t>((m_end - 1) / K, (int64_t)h.adj_nckpt - 1);
    for (int64_t c = c_last; c >= 0; --c) {
        a.m0 = c * K;
        a.m1 = (c == c_last) ? m_end + 1 : (c + 1) * K;
        if (a.m1 - a.m0 > K + 1) return fail(WQ3D_ERR_OVERFLOW, "the run went past the adjoint's max_steps");
        a.ckpt = (int)c;
        WQ_CK(cudaMemsetAsync(W.seed, 0, (size_t)(a.m1 - a.m0) * ADJ_L * n * sizeof(double), st));
        if (xs && xs->step >= a.m0 && xs->step < a.m1) {
            const double one = 1.0;
            WQ_CK(cudaMemcpyAsync(W.seed + ((size_t)(xs->step - a.m0) * ADJ_L + xs->comp) * n + xs->ray, &one,
                                  sizeof(double), cudaMemcpyHostToDevice, st));
        }
        k_adj_recompute<<<gb, 128, 0, st>>>(a, qa);
        if (nrec > 0) k_adj_expand<<<rb, 128, 0, st>>>(a, qa);
        k_adj_reverse<<<gb, 128, 0, st>>>(a, qa);
    }
    k_adj_startup<<<gb, 128, 0, st>>>(a, qa);
    WQ_CK(cudaGetLastError());
    WQ_CK(cudaEventRecord(e1, st));
    std::vector<double> g(nodes);
    uint32_t err = 0;
    WQ_CK(cudaMemcpyAsync(g.data(), W.grad, nodes * sizeof(double), cudaMemcpyDeviceToHost, st));
    WQ_CK(cudaMemcpyAsync(&err, W.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    WQ_CK(cudaStreamSynchronize(st));
    if (ms) {
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        *ms = t;
    }
    if (err & ADJ_ERR_WINDOW)
        return fail(WQ3D_ERR_NUMERIC, "adjoint: a step reached profile nodes beyond its window (nodes closer "
                                      "than a step's reach)");
    if (err & ADJ_ERR_CHAIN) return fail(WQ3D_ERR_NUMERIC, "adjoint: more than 8 reflections in one step");
    if (err & ADJ_ERR_TOPOLOGY)
        return fail(WQ3D_ERR_NUMERIC, "adjoint: a reflection chain's re-evaluation took another branch");
    /* the beam spread s2 = (2 pi c_target / f)^2 of the first frequency
     * through the target's sound speed (d s2 / d c = 2 s2 / c), which is
     * linear in the two nodes around the target's depth */
    std::vector<double> ax((size_t)nodes), trho((size_t)h.nt), tc((size_t)h.nt), ts2((size_t)h.nt);
    WQ_CK(cudaMemcpy(ax.data(), h.oc.prof.grid.ax[0].x, nodes * sizeof(double), cudaMemcpyDeviceToHost));
    WQ_CK(cudaMemcpy(trho.data(), h.tgt[0], h.nt * sizeof(double), cudaMemcpyDeviceToHost));
    WQ_CK(cudaMemcpy(tc.data(), h.tgt_c, h.nt * sizeof(double), cudaMemcpyDeviceToHost));
    WQ_CK(cudaMemcpy2D(ts2.data(), sizeof(double), h.tgt_spread2, (size_t)h.nf * sizeof(double), sizeof(double),
                       (size_t)h.nt, cudaMemcpyDeviceToHost));
    const double sign = (ax[1] < ax[0]) ? -1.0 : 1.0;
    for (int t = 0; t < h.nt; ++t) {
        if (gs2[t] == 0.0 || tc[t] == 0.0) continue;
        const double gc = gs2[t] * 2.0 * ts2[t] / tc[t];
        const double r = trho[t];
        int k = 0;
        double u = 0.0;
        if (r * sign <= ax[0] * sign) {
            k = 0;
            u = 0.0;
        } else if (r * sign >= ax[nodes - 1] * sign) {
            k = nodes - 2;
            u = 1.0;
        } else {
            while (k < nodes - 2 && r * sign >= ax[k + 1] * sign) ++k;
            u = (r - ax[k]) / (ax[k + 1] - ax[k]);
        }
        const double fe = h.oc.prof.flat_earth ? r / h.R : 1.0;
        g[k] += gc * (1.0 - u) * fe;
        g[k + 1] += gc * u * fe;
    }
    for (int j = 0; j < nodes; ++j) grad[j] = g[j];
    return WQ3D_OK;
}

int wq3d_queue_sensitivities(const wq3d_queue* q, double* sens, size_t capacity, size_t* count) {
    if (!q || !count) return fail(WQ3D_ERR_INVALID, "null argument");
    *count = q->pending.size();
    if (!sens) return WQ3D_OK;
    if (capacity < q->pending.size()) return fail(WQ3D_ERR_OVERFLOW, "capacity smaller than the pending count");
    for (size_t i = 0; i < q->pending.size(); ++i)
        for (int m = 0; m < 3; ++m) sens[i * 3 + m] = q->h.sens ? q->pending.sens[i * 3 + m] : NAN;
    return WQ3D_OK;
}

int wq3d_queue_abort(wq3d_queue* q) {
    if (!q) return fail(WQ3D_ERR_INVALID, "null queue");
    q->abort_flag.store(true);
    return WQ3D_OK;
}

int wq3d_queue_timing(wq3d_queue* q, wq3d_timing* out, int reset) {
    if (!q) return fail(WQ3D_ERR_INVALID, "null queue");
    if (out) {
        out->ms_total = q->ms_total;
        out->ms_advance = q->ms_step;
        out->ms_reflect = q->ms_refl;
        out->ms_cpa = q->ms_cpa;
        out->ms_eigenray = q->ms_eig;
        out->launches = q->launches;
    }
    if (reset) {
        q->ms_step = q->ms_cpa = q->ms_eig = q->ms_total = q->ms_refl = 0.0;
        q->launches = 0;
    }
    return WQ3D_OK;
}

/* Turns per-kernel CUDA-event timing on or off (direct launches instead of
 * the chunk graph while on). */
int wq3d_queue_set_timing(wq3d_queue* q, int on) {
    if (!q) return fail(WQ3D_ERR_INVALID, "null queue");
    if (on && q->events.empty()) {
        DeviceGuard guard(q->device);
        q->events.resize(7 * (size_t)q->chunk + 2);
        for (auto& ev : q->events)
            if (cudaEventCreate(&ev) != cudaSuccess) {
                ev = nullptr;
                return fail(WQ3D_ERR_CUDA, "cudaEventCreate failed");
            }
    }
    q->timing = on != 0;
    return WQ3D_OK;
}

int wq3d_queue_set_reflect_schedule(wq3d_queue* q, int schedule) {
    if (!q) return fail(WQ3D_ERR_INVALID, "null queue");
    if (schedule < WQ3D_REFLECT_AUTO || schedule > WQ3D_REFLECT_INLINE)
        return fail(WQ3D_ERR_INVALID, "unknown reflection schedule");
    q->refl_sched = schedule;
    return WQ3D_OK;
}

int wq3d_queue_reflect_schedule(const wq3d_queue* q, int* schedule) {
    if (!q || !schedule) return fail(WQ3D_ERR_INVALID, "null argument");
    if (q->refl_sched != WQ3D_REFLECT_AUTO)
        *schedule = q->refl_sched;
    else if (q->last_inl >= 0)
        *schedule = q->last_inl ? WQ3D_REFLECT_INLINE : WQ3D_REFLECT_SIDE;
    else
        *schedule = WQ3D_REFLECT_AUTO;
    return WQ3D_OK;
}

}  // extern "C"
