/*
 * wq3d_biverbs.cu -- bistatic eigenverbs: the overlap of every source
 * eigenverb with every receiver eigenverb it lies under, on one interface.
 *
 * The reference (biverbs/biverb_generator.cc:50-72) walks the receiver
 * eigenverbs, asks an R-tree of source eigenverbs for the ones whose
 * centres lie inside a quadrilateral around each receiver footprint
 * (eigenverbs/eigenverb_collection.cc:60-93), evaluates the interface's
 * scattering strength for each such pair (ocean/ocean_model.h:88-112) and
 * adds the Gaussian overlap to a collection
 * (biverbs/biverb_collection.cc:44-172).
 *
 * Here every (receiver, source) pair is screened on the GPU.  One warp
 * owns one receiver: its search quadrilateral and bounding box are
 * computed once (k_biverb_boxes).  The sources are cut into groups of 32
 * consecutive ones with a bounding box each (k_biverb_groups), and the
 * groups into runs of 32 with a box each (k_biverb_supers); the warp tests
 * 32 run boxes at once against its receiver's box, one per lane, then the
 * group boxes of each run that may hold a hit, and visits only the groups
 * that may hold a hit, each lane taking one source.  A bounding-box test rejects most of their pairs before the four
 * edge tests, and only pairs inside the quadrilateral evaluate the
 * overlap.  No shared memory and no block barrier are involved, so warps
 * run independently.
 * Two passes keep the output order fixed without atomics: the first counts
 * each receiver's surviving pairs and keeps the sources of its first 256,
 * the host turns the counts into offsets, and the second writes every pair
 * at its receiver's offset plus its rank among the warp's hits (ballot +
 * popc), in source index order: from the kept sources when they are all
 * of them, else by scanning again.
 *
 * The inputs are read from HBM once and the group boxes stay in L1, so the
 * passes are bound by the latency of the group scan and of the FP64
 * compares, not by HBM or the FP64 pipe.
 */
#include <cuda_runtime.h>

#include <climits>
#include <mutex>
#include <cmath>
#include <string>
#include <vector>

#include "wq3d.h"

extern "C" void wq3d_internal_set_error(const char* msg);

namespace {

constexpr int BV_WARPS = 8;    /* receivers per block, one warp each   */
constexpr int BV_BOX = 12;     /* doubles per receiver box            */
constexpr int BV_HITS = 256;   /* hit sources the count pass keeps per receiver */

int bv_fail(int code, const std::string& msg) {
    wq3d_internal_set_error(msg.c_str());
    return code;
}

__device__ __forceinline__ double bv_deg(double r) { return r * (180.0 / M_PI); }
__device__ __forceinline__ double bv_rad(double d) { return d * (M_PI / 180.0); }

/* latitude() and longitude() of wposition1(location, range, bearing)
 * (types/wposition1.cc:23-37), through the same degree / radian round
 * trips as the reference's setters and getters */
__device__ void bv_destination(const double* pos, double R0, double range, double bearing,
                               double* lat, double* lng) {
    const double lat1 = bv_rad(90.0 - bv_deg(pos[1]));
    const double lng1 = bv_rad(bv_deg(pos[2]));
    const double R = R0 + (pos[0] - R0);
    range /= R;
    const double lat2 = asin(sin(lat1) * cos(range) + cos(lat1) * sin(range) * cos(bearing));
    const double lng2 =
        lng1 + atan2(sin(bearing) * sin(range) * cos(lat1), cos(range) - sin(lat1) * sin(lat2));
    const double theta = bv_rad(90.0 - bv_deg(lat2));
    const double phi = bv_rad(bv_deg(lng2));
    *lat = 90.0 - bv_deg(theta);
    *lng = bv_deg(phi);
}

struct BvArgs {
    const wq3d_eigenverb* src;
    const double* src_pow;
    const double* sx;       /* source latitudes, degrees  */
    const double* sy;       /* source longitudes, degrees */
    int ns;
    const wq3d_eigenverb* rcv;
    const double* rcv_pow;
    const double* box;      /* BV_BOX doubles per receiver */
    const double* groups;   /* per group of 32 sources: latitude min, max, longitude min, max */
    const double* supers;   /* the same per 32 groups */
    int nr;
    int nf;
    int kind;
    double coef;            /* constant / Lambert linear coefficient      */
    const double* chap;     /* Chapman: 2.6 - 42.4 log10(beta), 3.3 beta */
    double R0;
    double threshold;
    long long* counts;      /* pass 1 writes, pass 2 reads */
    int* hits;              /* BV_HITS source indices per receiver */
    const long long* offs;  /* pass 2 */
    wq3d_biverb* out;
    double* out_pow;
    long long cap;
};

/* the search quadrilateral of each receiver (find_eigenverbs corners A-D)
 * and its bounding box; the source centres in degrees */
__global__ void k_biverb_boxes(const BvArgs a, double search_scale, double* box, double* sx, double* sy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.nr) {
        const wq3d_eigenverb& v = a.rcv[i];
        const double d = v.direction;
        double* b = box + (size_t)i * BV_BOX;
        bv_destination(v.position, a.R0, search_scale * v.length, d, &b[0], &b[4]);
        bv_destination(v.position, a.R0, search_scale * v.width, d + M_PI_2, &b[1], &b[5]);
        bv_destination(v.position, a.R0, search_scale * v.length, d + M_PI, &b[2], &b[6]);
        bv_destination(v.position, a.R0, search_scale * v.width, d + M_PI + M_PI_2, &b[3], &b[7]);
        b[8] = fmin(fmin(b[0], b[1]), fmin(b[2], b[3]));
        b[9] = fmax(fmax(b[0], b[1]), fmax(b[2], b[3]));
        b[10] = fmin(fmin(b[4], b[5]), fmin(b[6], b[7]));
        b[11] = fmax(fmax(b[4], b[5]), fmax(b[6], b[7]));
    }
    if (i < a.ns) {
        sx[i] = 90.0 - bv_deg(a.src[i].position[1]);
        sy[i] = bv_deg(a.src[i].position[2]);
    }
}

/* the bounding box (latitude min, max, longitude min, max) of each group
 * of 32 consecutive source centres, one warp per group */
__global__ void __launch_bounds__(256) k_biverb_groups(const double* sx, const double* sy, int ns, double* groups) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[4] = {INFINITY, -INFINITY, INFINITY, -INFINITY};
    if (i < ns) {
        v[0] = v[1] = sx[i];
        v[2] = v[3] = sy[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        v[0] = fmin(v[0], __shfl_xor_sync(0xffffffffu, v[0], o));
        v[1] = fmax(v[1], __shfl_xor_sync(0xffffffffu, v[1], o));
        v[2] = fmin(v[2], __shfl_xor_sync(0xffffffffu, v[2], o));
        v[3] = fmax(v[3], __shfl_xor_sync(0xffffffffu, v[3], o));
    }
    const int g = i >> 5;
    if ((threadIdx.x & 31) == 0 && (g << 5) < ns)
        for (int k = 0; k < 4; ++k) groups[4 * (size_t)g + k] = v[k];
}

/* the bounding box of each run of 32 group boxes, one warp per run */
__global__ void __launch_bounds__(256) k_biverb_supers(const double* groups, int ngroups, double* supers) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[4] = {INFINITY, -INFINITY, INFINITY, -INFINITY};
    if (i < ngroups)
        for (int k = 0; k < 4; ++k) v[k] = groups[4 * (size_t)i + k];
    for (int o = 16; o > 0; o >>= 1) {
        v[0] = fmin(v[0], __shfl_xor_sync(0xffffffffu, v[0], o));
        v[1] = fmax(v[1], __shfl_xor_sync(0xffffffffu, v[1], o));
        v[2] = fmin(v[2], __shfl_xor_sync(0xffffffffu, v[2], o));
        v[3] = fmax(v[3], __shfl_xor_sync(0xffffffffu, v[3], o));
    }
    const int h = i >> 5;
    if ((threadIdx.x & 31) == 0 && (h << 5) < ngroups)
        for (int k = 0; k < 4; ++k) supers[4 * (size_t)h + k] = v[k];
}

/* a box (latitude min, max, longitude min, max) that holds no point
 * strictly inside the receiver box b[8..11] */
__device__ __forceinline__ bool bv_misses(const double* box, const double* b) {
    return box[1] <= b[8] || box[0] >= b[9] || box[3] <= b[10] || box[2] >= b[11];
}

/* strictly inside the quadrilateral: all four edge cross products have
 * one sign (the corners go round in either sense) */
__device__ __forceinline__ bool bv_inside(const double* b, double x, double y) {
    if (!(x > b[8] && x < b[9] && y > b[10] && y < b[11])) return false;
    int pos = 0, neg = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int k2 = (k + 1) & 3;
        const double c = (b[k2] - b[k]) * (y - b[4 + k]) - (b[4 + k2] - b[4 + k]) * (x - b[k]);
        pos += c > 0.0;
        neg += c < 0.0;
    }
    return pos == 4 || neg == 4;
}

/* geometry of one pair (biverb_collection.cc:58-163): the power scale of
 * the overlap (before the eigenverb powers and the scattering strength) and
 * the duration */
struct BvOverlap {
    double scale;
    double duration;
};

__device__ BvOverlap bv_overlap(const wq3d_eigenverb& s, const wq3d_eigenverb& r, double R0) {
    /* rcv.position.gc_range(src.position, &bearing) (types/wposition1.cc:57-92) */
    const double lat1 = bv_rad(90.0 - bv_deg(r.position[1]));
    const double lng1 = bv_rad(bv_deg(r.position[2]));
    const double R = R0 + (r.position[0] - R0);
    const double lat2 = bv_rad(90.0 - bv_deg(s.position[1]));
    const double lng2 = bv_rad(bv_deg(s.position[2]));
    double hav1at = sin(0.5 * (lat1 - lat2));
    hav1at *= hav1at;
    double havlng = sin(0.5 * (lng1 - lng2));
    havlng *= havlng;
    const double arc = 2.0 * asin(sqrt(hav1at + cos(lat1) * cos(lat2) * havlng));
    double bearing;
    if (fabs(arc) < 1e-6 || fabs(lat1) < 1e-10) {
        bearing = (lat1 > 0) ? M_PI : 0.0;
    } else {
        bearing = atan2(sin(lng1 - lng2) * cos(lat2), cos(lat1) * sin(lat2) - sin(lat1) * cos(lat2) * cos(lng1 - lng2));
        bearing = fmod(2.0 * M_PI - bearing, 2.0 * M_PI);
    }
    const double range = arc * R;
    if (range < 1e-6) bearing = 0;
    bearing -= r.direction;
    const double ys = range * cos(bearing);
    const double ys2 = ys * ys;
    const double xs = range * sin(bearing);
    const double xs2 = xs * xs;

    const double alpha = s.direction - r.direction;
    const double cos2alpha = cos(2.0 * alpha);
    const double sin2alpha = sin(2.0 * alpha);
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
    const double new_prod = src_diff * cos2alpha;
    const double kappa = -0.25 *
                         (xs2 * (src_sum + new_prod + 2.0 * rcv_length2) +
                          ys2 * (src_sum - new_prod + 2.0 * rcv_width2) -
                          2.0 * sqrt(xs2 * ys2) * src_diff * sin2alpha) /
                         det_sr;
    BvOverlap o;
    o.scale = exp(kappa) / sqrt(det_sr);
    det_sr = det_sr / (src_prod * rcv_prod);
    const double sigma = 0.5 *
                         ((1.0 / src_width2 + 1.0 / src_length2) +
                          (1.0 / src_width2 - 1.0 / src_length2) * cos2alpha + 2.0 / rcv_width2) /
                         det_sr;
    const double factor = cos(r.grazing) / r.sound_speed;
    o.duration = 0.5 * factor * sqrt(sigma);
    return o;
}

/* scattering strength at frequency f (ocean/scattering_*.h) */
__device__ __forceinline__ double bv_scatter(const BvArgs& a, int f, double de_incident, double de_scattered) {
    if (a.kind == WQ3D_SCATTER_LAMBERT) return fabs(a.coef * sin(de_incident) * sin(de_scattered));
    if (a.kind == WQ3D_SCATTER_CHAPMAN) {
        const double grazing = 0.5 * (de_incident + de_scattered) * 180.0 / M_PI;
        const double amp = a.chap[2 * f] + a.chap[2 * f + 1] * log10(grazing / 30.0 + 1e-6);
        return pow(10.0, amp / 10.0);
    }
    return a.coef;
}

/* power of pair frequency f: 0.25 * 0.5 * src * rcv * scatter * overlap */
__device__ __forceinline__ double bv_power(const BvArgs& a, int si, int ri, int f, double scale, double gs,
                                           double gr) {
    double p = 0.125 * a.src_pow[(size_t)si * a.nf + f];
    p = p * a.rcv_pow[(size_t)ri * a.nf + f];
    p = p * bv_scatter(a, f, gs, gr);
    return p * scale;
}

/* writes the biverb of source si and receiver ri at output slot k */
__device__ __noinline__ void bv_write(const BvArgs& a, int si, int ri, const BvOverlap& o, long long k) {
    const wq3d_eigenverb& s = a.src[si];
    const wq3d_eigenverb& r = a.rcv[ri];
    wq3d_biverb v;
    v.travel_time = s.travel_time + r.travel_time;
    v.duration = o.duration;
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
    v.source = si;
    v.receiver = ri;
    a.out[k] = v;
    for (int f = 0; f < a.nf; ++f)
        a.out_pow[(size_t)k * a.nf + f] = bv_power(a, si, ri, f, o.scale, s.grazing, r.grazing);
}

/* three blocks per SM (80 registers): the group scan is latency-bound, and
 * the extra warps hide more of it than the rare overlap code loses */
template <bool WRITE>
__global__ void __launch_bounds__(BV_WARPS * 32, 3) k_biverb_pairs(const BvArgs a) {
    const int lane = threadIdx.x & 31;
    const int ri = blockIdx.x * BV_WARPS + (threadIdx.x >> 5);
    if (ri >= a.nr) return;  /* a whole warp: no block barrier follows */
    double b[BV_BOX];
#pragma unroll
    for (int k = 0; k < BV_BOX; ++k) b[k] = a.box[(size_t)ri * BV_BOX + k];
    const long long base = WRITE ? a.offs[ri] : 0;
    if (WRITE) {
        /* the count pass stored the sources of up to BV_HITS hits, in
         * source order: write those without scanning again */
        const long long cnt = a.counts[ri];
        if (cnt <= BV_HITS) {
            for (int k = lane; k < cnt; k += 32) {
                const int si = a.hits[(size_t)ri * BV_HITS + k];
                if (base + k < a.cap) bv_write(a, si, ri, bv_overlap(a.src[si], a.rcv[ri], a.R0), base + k);
            }
            return;
        }
    }
    const unsigned below = (1u << lane) - 1u;
    const int ngroups = (a.ns + 31) >> 5;
    long long n = 0;
    /* a centre strictly inside the quadrilateral lies strictly inside the
     * receiver's bounding box: each lane tests one box of 32 groups, then,
     * inside each that may hold a hit, one group box, and the warp visits
     * the groups that may hold a hit in increasing order */
    const int nsupers = (ngroups + 31) >> 5;
    for (int h0 = 0; h0 < nsupers; h0 += 32) {
        const int hl = h0 + lane;
        const bool hneed = hl < nsupers && !bv_misses(a.supers + 4 * (size_t)hl, b);
        unsigned htodo = __ballot_sync(0xffffffffu, hneed);
        while (htodo) {
            const int g0 = (h0 + __ffs(htodo) - 1) << 5;
            htodo &= htodo - 1;
            const int gl = g0 + lane;
            const bool need = gl < ngroups && !bv_misses(a.groups + 4 * (size_t)gl, b);
            unsigned todo = __ballot_sync(0xffffffffu, need);
            while (todo) {
                const int g = g0 + __ffs(todo) - 1;
                todo &= todo - 1;
                const int si = (g << 5) + lane;
                bool hit = false;
                BvOverlap o{0.0, 0.0};
                if (si < a.ns && bv_inside(b, a.sx[si], a.sy[si])) {
                    const wq3d_eigenverb& s = a.src[si];
                    const wq3d_eigenverb& r = a.rcv[ri];
                    o = bv_overlap(s, r, a.R0);
                    double pmax = 0.0;
                    for (int f = 0; f < a.nf; ++f) pmax = fmax(pmax, fabs(bv_power(a, si, ri, f, o.scale, s.grazing, r.grazing)));
                    hit = pmax >= a.threshold;
                }
                const unsigned bal = __ballot_sync(0xffffffffu, hit);
                if (hit) {
                    const long long k = n + __popc(bal & below);
                    if (WRITE) {
                        if (base + k < a.cap) bv_write(a, si, ri, o, base + k);
                    } else if (k < BV_HITS) {
                        a.hits[(size_t)ri * BV_HITS + k] = si;
                    }
                }
                n += __popc(bal);
            }
        }
    }
    if (!WRITE && lane == 0) a.counts[ri] = n;
}

/* Device buffers and a stream kept per device from one call to the next,
 * so that a call allocates nothing once the buffers are large enough
 * (they only grow, by a quarter more than asked).  The mutex serialises
 * calls on one device.  The buffers live until the process exits. */
constexpr int BV_MAX_DEVICES = 64;
enum { BV_SRC, BV_RCV, BV_SPOW, BV_RPOW, BV_SX, BV_SY, BV_BOXES, BV_GROUPS_BUF, BV_COUNTS, BV_CHAP,
       BV_OFFS, BV_OUT, BV_OPOW, BV_HITS_BUF, BV_SUPERS_BUF, BV_NBUF };

struct BvWorkspace {
    std::mutex m;
    cudaStream_t s = nullptr;
    void* p[BV_NBUF] = {};
    size_t cap[BV_NBUF] = {};
    template <class T>
    cudaError_t get(int k, T** out, size_t n) {
        const size_t bytes = (n ? n : 1) * sizeof(T);
        if (bytes > cap[k]) {
            if (p[k]) cudaFree(p[k]);
            p[k] = nullptr;
            cap[k] = 0;
            const size_t want = bytes + bytes / 4;
            const cudaError_t e = cudaMalloc(&p[k], want);
            if (e != cudaSuccess) {
                p[k] = nullptr;
                return e;
            }
            cap[k] = want;
        }
        *out = static_cast<T*>(p[k]);
        return cudaSuccess;
    }
};

BvWorkspace g_bv[BV_MAX_DEVICES];

}  // namespace

#define BV_CK(call)                                                                  \
    do {                                                                             \
        const cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) return bv_fail(WQ3D_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

extern "C" int wq3d_biverbs(const wq3d_eigenverb* src, const double* src_power, size_t num_src,
                            const wq3d_eigenverb* rcv, const double* rcv_power, size_t num_rcv,
                            const double* freq, size_t num_freq, const wq3d_scattering_desc* scattering,
                            double earth_radius, double search_scale, double power_threshold,
                            wq3d_biverb* out, double* out_power, size_t capacity, size_t* count) {
    if (!count || !scattering) return bv_fail(WQ3D_ERR_INVALID, "null count or scattering");
    *count = 0;
    if (num_freq == 0 || !freq) return bv_fail(WQ3D_ERR_INVALID, "no frequencies");
    if ((num_src && (!src || !src_power)) || (num_rcv && (!rcv || !rcv_power)))
        return bv_fail(WQ3D_ERR_INVALID, "null eigenverbs");
    if (out && capacity && !out_power) return bv_fail(WQ3D_ERR_INVALID, "null out_power");
    if (!(earth_radius > 0.0) || !(search_scale > 0.0))
        return bv_fail(WQ3D_ERR_INVALID, "earth_radius and search_scale must be positive");
    if (scattering->kind < WQ3D_SCATTER_CONSTANT || scattering->kind > WQ3D_SCATTER_CHAPMAN)
        return bv_fail(WQ3D_ERR_INVALID, "unknown scattering model");
    if (num_src > (size_t)INT_MAX || num_rcv > (size_t)INT_MAX || num_freq > 65536)
        return bv_fail(WQ3D_ERR_INVALID, "too many eigenverbs or frequencies");
    if (num_src == 0 || num_rcv == 0) return WQ3D_OK;

    /* scattering coefficients that do not depend on the pair, evaluated
     * as the reference's constructors and vector expressions do */
    BvArgs a{};
    a.kind = scattering->kind;
    std::vector<double> chap;
    if (a.kind == WQ3D_SCATTER_CHAPMAN) {
        const double speed = scattering->p * 1.94384449;
        chap.resize(2 * num_freq);
        for (size_t f = 0; f < num_freq; ++f) {
            const double beta = 158.0 * std::pow(speed * std::pow(freq[f], 1.0 / 3.0), -0.58);
            chap[2 * f] = 2.6 - 42.4 * std::log10(beta);
            chap[2 * f + 1] = 3.3 * beta;
        }
    } else {
        a.coef = std::pow(10.0, scattering->p / 10.0);
    }

    int dev = 0;
    BV_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= BV_MAX_DEVICES) return bv_fail(WQ3D_ERR_CUDA, "device index out of range");
    BvWorkspace& ws = g_bv[dev];
    std::lock_guard<std::mutex> lock(ws.m);
    if (!ws.s) BV_CK(cudaStreamCreateWithFlags(&ws.s, cudaStreamNonBlocking));
    wq3d_eigenverb *d_src, *d_rcv;
    double *d_spow, *d_rpow, *d_sx, *d_sy, *d_box, *d_groups, *d_chap = nullptr;
    long long* d_counts;
    int* d_hits;
    BV_CK(ws.get(BV_SRC, &d_src, num_src));
    BV_CK(ws.get(BV_RCV, &d_rcv, num_rcv));
    BV_CK(ws.get(BV_SPOW, &d_spow, num_src * num_freq));
    BV_CK(ws.get(BV_RPOW, &d_rpow, num_rcv * num_freq));
    BV_CK(ws.get(BV_SX, &d_sx, num_src));
    BV_CK(ws.get(BV_SY, &d_sy, num_src));
    BV_CK(ws.get(BV_BOXES, &d_box, num_rcv * BV_BOX));
    const size_t num_groups = (num_src + 31) / 32;
    BV_CK(ws.get(BV_GROUPS_BUF, &d_groups, num_groups * 4));
    const size_t num_supers = (num_groups + 31) / 32;
    double* d_supers;
    BV_CK(ws.get(BV_SUPERS_BUF, &d_supers, num_supers * 4));
    BV_CK(ws.get(BV_COUNTS, &d_counts, num_rcv));
    BV_CK(ws.get(BV_HITS_BUF, &d_hits, num_rcv * BV_HITS));
    if (!chap.empty()) BV_CK(ws.get(BV_CHAP, &d_chap, chap.size()));
    BV_CK(cudaMemcpyAsync(d_src, src, num_src * sizeof(wq3d_eigenverb), cudaMemcpyHostToDevice, ws.s));
    BV_CK(cudaMemcpyAsync(d_rcv, rcv, num_rcv * sizeof(wq3d_eigenverb), cudaMemcpyHostToDevice, ws.s));
    BV_CK(cudaMemcpyAsync(d_spow, src_power, num_src * num_freq * sizeof(double), cudaMemcpyHostToDevice, ws.s));
    BV_CK(cudaMemcpyAsync(d_rpow, rcv_power, num_rcv * num_freq * sizeof(double), cudaMemcpyHostToDevice, ws.s));
    if (d_chap)
        BV_CK(cudaMemcpyAsync(d_chap, chap.data(), chap.size() * sizeof(double), cudaMemcpyHostToDevice, ws.s));

    a.src = d_src;
    a.src_pow = d_spow;
    a.sx = d_sx;
    a.sy = d_sy;
    a.ns = (int)num_src;
    a.rcv = d_rcv;
    a.rcv_pow = d_rpow;
    a.box = d_box;
    a.groups = d_groups;
    a.supers = d_supers;
    a.nr = (int)num_rcv;
    a.nf = (int)num_freq;
    a.chap = d_chap;
    a.R0 = earth_radius;
    a.threshold = power_threshold;
    a.counts = d_counts;
    a.hits = d_hits;

    const size_t nmax = num_src > num_rcv ? num_src : num_rcv;
    k_biverb_boxes<<<(unsigned)((nmax + 127) / 128), 128, 0, ws.s>>>(a, search_scale, d_box, d_sx, d_sy);
    BV_CK(cudaGetLastError());
    k_biverb_groups<<<(unsigned)((num_src + 255) / 256), 256, 0, ws.s>>>(d_sx, d_sy, (int)num_src, d_groups);
    BV_CK(cudaGetLastError());
    k_biverb_supers<<<(unsigned)((num_groups + 255) / 256), 256, 0, ws.s>>>(d_groups, (int)num_groups, d_supers);
    BV_CK(cudaGetLastError());
    const unsigned blocks = (unsigned)((num_rcv + BV_WARPS - 1) / BV_WARPS);
    k_biverb_pairs<false><<<blocks, BV_WARPS * 32, 0, ws.s>>>(a);
    BV_CK(cudaGetLastError());
    std::vector<long long> counts(num_rcv);
    BV_CK(cudaMemcpyAsync(counts.data(), d_counts, num_rcv * sizeof(long long), cudaMemcpyDeviceToHost, ws.s));
    BV_CK(cudaStreamSynchronize(ws.s));
    std::vector<long long> offs(num_rcv);
    long long total = 0;
    for (size_t i = 0; i < num_rcv; ++i) {
        offs[i] = total;
        total += counts[i];
    }
    *count = (size_t)total;
    if (!out || capacity == 0 || total == 0) return (out && total > (long long)capacity)
                                                       ? bv_fail(WQ3D_ERR_OVERFLOW, "biverb capacity too small")
                                                       : WQ3D_OK;

    const size_t nout = (size_t)total < capacity ? (size_t)total : capacity;
    long long* d_offs;
    wq3d_biverb* d_out;
    double* d_opow;
    BV_CK(ws.get(BV_OFFS, &d_offs, num_rcv));
    BV_CK(ws.get(BV_OUT, &d_out, nout));
    BV_CK(ws.get(BV_OPOW, &d_opow, nout * num_freq));
    BV_CK(cudaMemcpyAsync(d_offs, offs.data(), num_rcv * sizeof(long long), cudaMemcpyHostToDevice, ws.s));
    a.offs = d_offs;
    a.out = d_out;
    a.out_pow = d_opow;
    a.cap = (long long)nout;
    k_biverb_pairs<true><<<blocks, BV_WARPS * 32, 0, ws.s>>>(a);
    BV_CK(cudaGetLastError());
    BV_CK(cudaMemcpyAsync(out, d_out, nout * sizeof(wq3d_biverb), cudaMemcpyDeviceToHost, ws.s));
    BV_CK(cudaMemcpyAsync(out_power, d_opow, nout * num_freq * sizeof(double), cudaMemcpyDeviceToHost, ws.s));
    BV_CK(cudaStreamSynchronize(ws.s));
    if ((size_t)total > capacity) return bv_fail(WQ3D_ERR_OVERFLOW, "biverb capacity too small");
    return WQ3D_OK;
}
