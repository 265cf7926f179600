/*
 * wq3d_sum.cu -- eigenray_collection::sum_eigenrays on the GPU
 * (eigenrays/eigenray_collection.cc:105-191).
 *
 * One thread per target walks that target's eigenrays in the order they
 * were added, frequency by frequency, exactly as the reference's loops do:
 * the phasor of each frequency, and the power weights a^2 summed over
 * (frequency, eigenray) with the weighted travel time, D/E angles and AZ
 * unit vectors.  The strongest path (the first largest weight in that
 * order) gives the counts.  The sums are sequential, so the results differ
 * from the reference only through CUDA's versus the host's pow / sin / cos
 * / log10 / atan2 in the last place.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "wq3d_engine.cuh"

using namespace wq3d;

extern "C" void wq3d_internal_set_error(const char* msg);

namespace {

int sum_fail(int code, const std::string& msg) {
    wq3d_internal_set_error(msg.c_str());
    return code;
}

struct SumRay {
    double time, sde, saz, tde, taz;
    int32_t surface, bottom, caustic, upper, lower, pad;
};

__global__ void k_sum_eigenrays(int nt, const int32_t* first, const int32_t* order, const SumRay* rays,
                                const double* inten, const double* phase, int nf, const double* freq,
                                int coherent, SumRay* total, double* tot_inten, double* tot_phase) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int b = first[t], e = first[t + 1];
    const double TWO_PI = 2.0 * M_PI;
    double time = 0.0, sde = 0.0, sax = 0.0, say = 0.0, tde = 0.0, tax = 0.0, tay = 0.0;
    double wgt = 0.0, max_a = 0.0;
    int32_t cnt[5] = {-1, -1, -1, -1, -1};
    for (int f = 0; f < nf; ++f) {
        double re = 0.0, im = 0.0;
        for (int k = b; k < e; ++k) {
            const int j = order[k];
            const SumRay& r = rays[j];
            double a = pow(10.0, inten[(size_t)j * nf + f] / -20.0);
            if (coherent) {
                double p = TWO_PI * freq[f] * r.time + phase[(size_t)j * nf + f];
                p = fmod(p, TWO_PI);
                re += a * cos(p);
                im += a * sin(p);
            } else {
                re += a;
            }
            a *= a;
            wgt += a;
            time += a * r.time;
            sde += a * r.sde;
            sax += a * sin(r.saz * (M_PI / 180.0));
            say += a * cos(r.saz * (M_PI / 180.0));
            tde += a * r.tde;
            tax += a * sin(r.taz * (M_PI / 180.0));
            tay += a * cos(r.taz * (M_PI / 180.0));
            if (a > max_a) {
                max_a = a;
                cnt[0] = r.surface;
                cnt[1] = r.bottom;
                cnt[2] = r.caustic;
                cnt[3] = r.upper;
                cnt[4] = r.lower;
            }
        }
        tot_inten[(size_t)t * nf + f] = -20.0 * log10(fmax(1e-15, hypot(re, im)));
        tot_phase[(size_t)t * nf + f] = atan2(im, re);
    }
    SumRay o;
    o.time = time / wgt;
    o.sde = sde / wgt;
    o.saz = 90.0 - atan2(say, sax) * (180.0 / M_PI);
    o.tde = tde / wgt;
    o.taz = 90.0 - atan2(tay, tax) * (180.0 / M_PI);
    o.surface = cnt[0];
    o.bottom = cnt[1];
    o.caustic = cnt[2];
    o.upper = cnt[3];
    o.lower = cnt[4];
    o.pad = 0;
    total[t] = o;
}

}  // namespace

extern "C" int wq3d_sum_eigenrays(const wq3d_eigenray* rays, const double* intensity, const double* phase,
                                  size_t n, const double* freq, size_t nf, size_t num_targets1,
                                  size_t num_targets2, int coherent, wq3d_eigenray* total,
                                  double* total_intensity, double* total_phase) {
    const size_t nt = num_targets1 * num_targets2;
    if (nf == 0 || !freq || !total || !total_intensity || !total_phase)
        return sum_fail(WQ3D_ERR_INVALID, "null argument");
    if (n > 0 && (!rays || !intensity || !phase)) return sum_fail(WQ3D_ERR_INVALID, "null argument");
    if (nt == 0) return WQ3D_OK;
    if (n > 0x7fffffff || nt > 0x7fffffff) return sum_fail(WQ3D_ERR_INVALID, "too many eigenrays or targets");
    /* eigenrays grouped by target, each group in the order given (a stable
     * counting sort), as the reference's per-target lists hold them */
    std::vector<int32_t> first(nt + 1, 0), order(std::max<size_t>(n, 1));
    for (size_t k = 0; k < n; ++k) {
        if (rays[k].t1 < 0 || rays[k].t2 < 0 || (size_t)rays[k].t2 >= num_targets2 ||
            (size_t)rays[k].t1 >= num_targets1)
            return sum_fail(WQ3D_ERR_INVALID, "eigenray " + std::to_string(k) + " names a target outside the grid");
        ++first[(size_t)rays[k].t1 * num_targets2 + (size_t)rays[k].t2 + 1];
    }
    for (size_t t = 0; t < nt; ++t) first[t + 1] += first[t];
    {
        std::vector<int32_t> fill(first.begin(), first.end() - 1);
        for (size_t k = 0; k < n; ++k) order[fill[(size_t)rays[k].t1 * num_targets2 + rays[k].t2]++] = (int32_t)k;
    }
    std::vector<SumRay> sr(std::max<size_t>(n, 1));
    for (size_t k = 0; k < n; ++k) {
        const wq3d_eigenray& r = rays[k];
        sr[k] = SumRay{r.time, r.source_de, r.source_az, r.target_de, r.target_az,
                       r.surface, r.bottom, r.caustic, r.upper, r.lower, 0};
    }
    char* dmem = nullptr;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t b_first = al((nt + 1) * 4), b_order = al(std::max<size_t>(n, 1) * 4);
    const size_t b_rays = al(std::max<size_t>(n, 1) * sizeof(SumRay));
    const size_t b_in = al(std::max<size_t>(n, 1) * nf * 8), b_freq = al(nf * 8);
    const size_t b_tot = al(nt * sizeof(SumRay)), b_ti = al(nt * nf * 8);
    const size_t bytes = b_first + b_order + b_rays + 2 * b_in + b_freq + b_tot + 2 * b_ti;
    cudaError_t e = cudaMalloc(&dmem, bytes);
    if (e != cudaSuccess) return sum_fail(WQ3D_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    char* p = dmem;
    auto take = [&](size_t b) {
        char* r = p;
        p += b;
        return r;
    };
    int32_t* d_first = (int32_t*)take(b_first);
    int32_t* d_order = (int32_t*)take(b_order);
    SumRay* d_rays = (SumRay*)take(b_rays);
    double* d_in = (double*)take(b_in);
    double* d_ph = (double*)take(b_in);
    double* d_freq = (double*)take(b_freq);
    SumRay* d_tot = (SumRay*)take(b_tot);
    double* d_ti = (double*)take(b_ti);
    double* d_tp = (double*)take(b_ti);
    e = cudaMemcpy(d_first, first.data(), (nt + 1) * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n) e = cudaMemcpy(d_order, order.data(), n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n) e = cudaMemcpy(d_rays, sr.data(), n * sizeof(SumRay), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n) e = cudaMemcpy(d_in, intensity, n * nf * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n) e = cudaMemcpy(d_ph, phase, n * nf * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_freq, freq, nf * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_sum_eigenrays<<<(unsigned)((nt + 127) / 128), 128>>>((int)nt, d_first, d_order, d_rays, d_in, d_ph,
                                                               (int)nf, d_freq, coherent, d_tot, d_ti, d_tp);
        e = cudaGetLastError();
    }
    std::vector<SumRay> tot(nt);
    if (e == cudaSuccess) e = cudaMemcpy(tot.data(), d_tot, nt * sizeof(SumRay), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(total_intensity, d_ti, nt * nf * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(total_phase, d_tp, nt * nf * 8, cudaMemcpyDeviceToHost);
    cudaFree(dmem);
    if (e != cudaSuccess) return sum_fail(WQ3D_ERR_CUDA, std::string("sum_eigenrays: ") + cudaGetErrorString(e));
    for (size_t t = 0; t < nt; ++t) {
        wq3d_eigenray& o = total[t];
        o = wq3d_eigenray{};
        o.time = tot[t].time;
        o.source_de = tot[t].sde;
        o.source_az = tot[t].saz;
        o.target_de = tot[t].tde;
        o.target_az = tot[t].taz;
        o.surface = tot[t].surface;
        o.bottom = tot[t].bottom;
        o.caustic = tot[t].caustic;
        o.upper = tot[t].upper;
        o.lower = tot[t].lower;
        o.t1 = (int32_t)(t / num_targets2);
        o.t2 = (int32_t)(t % num_targets2);
        o.de = o.az = -1;
        o.step = -1;
    }
    return WQ3D_OK;
}
