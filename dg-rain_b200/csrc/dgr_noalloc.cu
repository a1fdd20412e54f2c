/*
 * dgr_slope_limiter_noalloc: the vertex-based slope limiter on caller-owned device
 * arrays, with no device allocation at all.
 *
 * Who needs it: code that runs where it may not allocate device memory, because it is
 * handed buffers by a host framework or an external memory pool, or because it runs
 * inside a region where cudaMalloc/cudaFree are not allowed (cudaFree synchronises the
 * device, and allocation during a stream capture is an error).  Such a caller passes its
 * own inputs and outputs; the only other memory this entry point touches is the
 * file-scope scratch array below.
 *
 * Scratch: node max/min bounds, 6 values per node, in a static __device__ array sized for
 * DGR_NOALLOC_MAX_NODES nodes (6 MiB).  Every process that loads this library holds that
 * array on every GPU it uses, until the process exits.  Each call clears the part it uses
 * before reading it, so nothing from an earlier call leaks into a result; but every call
 * uses the same array, so calls whose kernels overlap on the GPU (on different streams,
 * or from different host threads) race on it and must be ordered by the caller.
 *
 * Set-up: host code cannot use the array's name as a device address (on the host it is
 * only a stand-in symbol), so the first call on each device, with that device current,
 * looks the address up with cudaGetSymbolAddress and keeps it.  Make that first call
 * outside any stream capture.
 */
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/dgrain.h"
#include "dgr_device.cuh"

namespace {

/* Node bounds as order-preserving 64-bit keys: [6][DGR_NOALLOC_MAX_NODES]
 * (max zeta, max Qx, max Qy, min zeta, min Qx, min Qy). */
static __device__ __align__(256) long long g_noalloc_bounds[6 * DGR_NOALLOC_MAX_NODES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
long long *g_scratch_ptr[kMaxDevices] = {nullptr};

/* Doubles compared as signed 64-bit integers: flipping the magnitude bits of negative
 * values makes integer order equal numeric order (NaN aside), so atomicMax/atomicMin on
 * the keys give the same max/min as the reference's sequential comparisons. */
__device__ __forceinline__ long long dkey(double x)
{
    const long long b = __double_as_longlong(x);
    return b ^ ((b >> 63) & 0x7fffffffffffffffLL);
}
__device__ __forceinline__ double dval(long long k)
{
    return __longlong_as_double(k ^ ((k >> 63) & 0x7fffffffffffffffLL));
}

/* The reference's starting values -99999 (max) and 99999 (min),
 * 2DCode/SlopeLimiter2D.c:108-113. */
__global__ void k_na_clear(long long *bounds, int nn)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    for (int v = 0; v < 3; ++v) {
        bounds[v * DGR_NOALLOC_MAX_NODES + n] = dkey(-99999.0);
        bounds[(3 + v) * DGR_NOALLOC_MAX_NODES + n] = dkey(99999.0);
    }
}

/* Element means (2DCode/SlopeLimiter2D.c:120-122) folded into the bounds of the
 * element's three nodes. */
__global__ void k_na_bounds(int ne, int nn, const int *__restrict__ el2v, const double *__restrict__ zeta,
                            const double *__restrict__ qx, const double *__restrict__ qy, long long *bounds)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= ne) return;
    const double *s[3] = {zeta, qx, qy};
    for (int v = 0; v < 3; ++v) {
        const double avg = (s[v][3 * el] + s[v][3 * el + 1] + s[v][3 * el + 2]) / 3;
        if (avg != avg) continue;
        const long long k = dkey(avg);
        for (int j = 0; j < 3; ++j) {
            const int n = el2v[3 * el + j];
            if (n < 0 || n >= nn) continue; /* out-of-range vertex: never touch memory outside */
            atomicMax(&bounds[v * DGR_NOALLOC_MAX_NODES + n], k);
            atomicMin(&bounds[(3 + v) * DGR_NOALLOC_MAX_NODES + n], k);
        }
    }
}

/* Element pass of 2DCode/SlopeLimiter2D.c:157-343 on the reference layout [3*el+k]. */
__global__ void k_na_limit(int ne, int nn, const int *__restrict__ el2v, const double *__restrict__ z,
                           double *zeta, double *qx, double *qy, const long long *__restrict__ bounds, double h0)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= ne) return;
    using dgr::rmin;
    using dgr::sgn;
    const int nd[3] = {el2v[3 * el], el2v[3 * el + 1], el2v[3 * el + 2]};
    for (int k = 0; k < 3; ++k)
        if (nd[k] < 0 || nd[k] >= nn) return; /* out-of-range vertex: leave the element as it is */
    const double zn[3] = {z[nd[0]], z[nd[1]], z[nd[2]]};
    double *s[3] = {zeta, qx, qy};
    double out[3][3];
    int modify = 0;
    for (int v = 0; v < 3; ++v) {
        const double w1 = s[v][3 * el], w2 = s[v][3 * el + 1], w3 = s[v][3 * el + 2];
        double vx[3] = {w1 - w2 + w3, w1 + w2 - w3, -w1 + w2 + w3};
        double vmax[3], vmin[3];
        for (int k = 0; k < 3; ++k) {
            vmax[k] = dval(bounds[v * DGR_NOALLOC_MAX_NODES + nd[k]]);
            vmin[k] = dval(bounds[(3 + v) * DGR_NOALLOC_MAX_NODES + nd[k]]);
        }
        const double avg = (w1 + w2 + w3) / 3;
        if (v == 0) {
            const double h1 = vx[0] + zn[0], h2 = vx[1] + zn[1], h3 = vx[2] + zn[2];
            const double m0 = vmin[0] + zn[0], m1 = vmin[1] + zn[1], m2 = vmin[2] + zn[2];
            if (h1 > h0 && h2 > h0 && h3 > h0 && m0 > h0 && m1 > h0 && m2 > h0) modify = 1;
        }
        for (int k = 0; k < 3; ++k) vx[k] = fmax(rmin(vx[k], vmax[k]), vmin[k]);
        for (int ll = 0; ll < 3; ++ll) {
            const double sumloc = (vx[0] + vx[1] + vx[2]) / 3;
            double sumdiff = (sumloc - avg) * 3;
            const int sd = sgn(sumdiff);
            const double sdd = (double)sd;
            const double diff[3] = {(vx[0] - avg) * sdd, (vx[1] - avg) * sdd, (vx[2] - avg) * sdd};
            double kdp = (double)((diff[0] > 0) + (diff[1] > 0) + (diff[2] > 0));
            for (int k = 0; k < 3; ++k) {
                const double div = fmax(1.0, kdp);
                double redfac;
                if (diff[k] > 0) {
                    redfac = sumdiff * sdd / div;
                    kdp -= 1;
                } else {
                    redfac = 0;
                }
                const double redmax = (sd > 0) ? vx[k] - vmin[k] : vmax[k] - vx[k];
                redfac = rmin(redfac, redmax);
                sumdiff -= redfac * sdd;
                vx[k] -= redfac * sdd;
            }
        }
        out[v][0] = (vx[0] + vx[1]) / 2;
        out[v][1] = (vx[1] + vx[2]) / 2;
        out[v][2] = (vx[2] + vx[0]) / 2;
        if (v == 0) {
            const double h1 = vx[0] + zn[0], h2 = vx[1] + zn[1], h3 = vx[2] + zn[2];
            if (h1 < h0 || h2 < h0 || h3 < h0) modify = 0;
        }
    }
    if (modify)
        for (int v = 0; v < 3; ++v)
            for (int k = 0; k < 3; ++k) s[v][3 * el + k] = out[v][k];
}

/* First call on a device: resolve the scratch array's device address. */
int scratch_for_current_device(long long **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return e == cudaErrorNoDevice ? DGR_ERR_NO_DEVICE : DGR_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        long long *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_noalloc_bounds);
        if (e != cudaSuccess || !p) return DGR_ERR_CUDA;
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return DGR_OK;
}

}  // namespace

extern "C" int dgr_slope_limiter_noalloc(int num_el, int num_nodes, const int *d_EltoVert, const double *d_z,
                                         double *d_zeta, double *d_Qx, double *d_Qy, double H0, void *stream)
{
    if (num_el <= 0 || num_nodes <= 0 || !d_EltoVert || !d_z || !d_zeta || !d_Qx || !d_Qy) return DGR_ERR_INVALID;
    if (num_nodes > DGR_NOALLOC_MAX_NODES) return DGR_ERR_TOO_LARGE; /* beyond the static scratch */
    long long *bounds = nullptr;
    int rc = scratch_for_current_device(&bounds);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    k_na_clear<<<(num_nodes + 255) / 256, 256, 0, s>>>(bounds, num_nodes);
    k_na_bounds<<<(num_el + 255) / 256, 256, 0, s>>>(num_el, num_nodes, d_EltoVert, d_zeta, d_Qx, d_Qy, bounds);
    k_na_limit<<<(num_el + 127) / 128, 128, 0, s>>>(num_el, num_nodes, d_EltoVert, d_z, d_zeta, d_Qx, d_Qy, bounds,
                                                    H0);
    return cudaGetLastError() == cudaSuccess ? DGR_OK : DGR_ERR_CUDA;
}
