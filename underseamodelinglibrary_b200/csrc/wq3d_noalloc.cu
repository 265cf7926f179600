/*
 * wq3d_noalloc.cu -- sound speed evaluation that allocates no memory.
 *
 * wq3d_ocean_sound_speed stages the caller's host points in device
 * buffers that it allocates and frees on every call.  Some callers cannot
 * allocate device memory at the time they need the answer: a sonar
 * processing loop that reserves all of its GPU memory up front and forbids
 * allocation afterwards, code running under a memory pool or a real-time
 * budget where cudaMalloc's latency and implicit synchronisation are not
 * acceptable, or a host application whose device heap is owned by another
 * component.  wq3d_ocean_sound_speed_noalloc serves them: it stages the
 * points in one fixed array that lives in the library's device image (it
 * is created when the library is loaded on a device and stays until the
 * process exits), so a call allocates nothing.
 *
 * Limits and rules of use:
 *  - at most WQ3D_NOALLOC_MAX_POINTS points per call; more is rejected
 *    with WQ3D_ERR_INVALID and a message, nothing is evaluated;
 *  - the array is shared by every call on a device, so calls that overlap
 *    on the GPU (from several host threads at once) race on it and must be
 *    serialised by the caller;
 *  - the first call on each device looks the array's device address up
 *    (cudaGetSymbolAddress) with that device current; make that first call
 *    before any CUDA stream capture begins on the device;
 *  - every element a call returns is written by that call, so nothing in
 *    the array has to be cleared between calls.
 */
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "wq3d_engine.cuh"

using namespace wq3d;

namespace {

/* per point: rho, theta, phi in; speed and three gradient components out */
constexpr size_t NOALLOC_STRIDE = 7;

/* The staging array.  In host code this name is only a stand-in for the
 * device object: its device address comes from cudaGetSymbolAddress. */
static __device__ __align__(256) double g_noalloc_points[WQ3D_NOALLOC_MAX_POINTS * NOALLOC_STRIDE];

}  // namespace

/* Records a message for wq3d_last_error_string (defined in wq3d_api.cu). */
extern "C" void wq3d_internal_set_error(const char* msg);

namespace {

int noalloc_fail(int code, const std::string& msg) {
    wq3d_internal_set_error(msg.c_str());
    return code;
}

constexpr int MAX_DEVICES = 64;
std::mutex g_addr_mutex;
double* g_addr[MAX_DEVICES] = {nullptr};

/* device address of the staging array on the current device (looked up
 * once per device, with that device current) */
int staging_address(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(WQ3D_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= MAX_DEVICES) return noalloc_fail(WQ3D_ERR_UNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_points);
        if (e != cudaSuccess || p == nullptr)
            return noalloc_fail(WQ3D_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_addr[dev] = static_cast<double*>(p);
    }
    *out = g_addr[dev];
    return WQ3D_OK;
}

/* the profile evaluation of k_sound_speed, reading and writing the staging
 * array passed in as "pts" (points are SoA blocks of n values) */
__global__ void k_sound_speed_noalloc(OceanDev oc, double R, int n, double* pts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double c, g[3];
    sound_speed(oc.prof, R, pts[i], pts[n + i], pts[2 * (size_t)n + i], &c, g);
    pts[3 * (size_t)n + i] = c;
    pts[4 * (size_t)n + i] = g[0];
    pts[5 * (size_t)n + i] = g[1];
    pts[6 * (size_t)n + i] = g[2];
}

}  // namespace

/* The ocean's device-side model description (defined in wq3d_api.cu). */
extern "C" int wq3d_internal_ocean_model(const wq3d_ocean* ocean, OceanDev* out);

extern "C" int wq3d_ocean_sound_speed_noalloc(const wq3d_ocean* ocean, double earth_radius, size_t n,
                                              const double* rho, const double* theta,
                                              const double* phi, double* speed, double* grad) {
    if (!ocean || !rho || !speed) return noalloc_fail(WQ3D_ERR_INVALID, "null argument");
    if (n > (size_t)WQ3D_NOALLOC_MAX_POINTS)
        return noalloc_fail(WQ3D_ERR_INVALID, "wq3d_ocean_sound_speed_noalloc: " + std::to_string(n) +
                                                  " points exceed the limit of " +
                                                  std::to_string(WQ3D_NOALLOC_MAX_POINTS));
    if (n == 0) return WQ3D_OK;
    OceanDev oc;
    const int orc = wq3d_internal_ocean_model(ocean, &oc); /* also checks the ocean's device */
    if (orc != WQ3D_OK) return orc;
    double* pts = nullptr;
    int rc = staging_address(&pts);
    if (rc) return rc;
    const size_t bytes = n * sizeof(double);
    cudaError_t e = cudaMemcpy(pts, rho, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        if (theta) e = cudaMemcpy(pts + n, theta, bytes, cudaMemcpyHostToDevice);
        else e = cudaMemset(pts + n, 0, bytes);
    }
    if (e == cudaSuccess) {
        if (phi) e = cudaMemcpy(pts + 2 * n, phi, bytes, cudaMemcpyHostToDevice);
        else e = cudaMemset(pts + 2 * n, 0, bytes);
    }
    if (e != cudaSuccess) return noalloc_fail(WQ3D_ERR_CUDA, std::string("cudaMemcpy: ") + cudaGetErrorString(e));
    k_sound_speed_noalloc<<<(unsigned)((n + 127) / 128), 128>>>(oc, earth_radius, (int)n, pts);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(speed, pts + 3 * n, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && grad) e = cudaMemcpy(grad, pts + 4 * n, 3 * bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return noalloc_fail(WQ3D_ERR_CUDA, std::string("sound speed kernel: ") + cudaGetErrorString(e));
    return WQ3D_OK;
}
