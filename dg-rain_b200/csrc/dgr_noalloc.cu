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
 * Scratch: per node, the max/min bounds of the three variables (6 x 8 bytes) and, per
 * variable, the first element whose mean is a zero (3 x 4 bytes), in a static __device__
 * array sized for DGR_NOALLOC_MAX_NODES nodes (7.5 MiB).  Every process that loads this
 * library holds that array on every GPU it uses, until the process exits.  Each call
 * clears the part it uses before reading it, so nothing from an earlier call leaks into a
 * result; but every call uses the same array, so calls whose kernels overlap on the GPU
 * (on different streams, or from different host threads) race on it and must be ordered
 * by the caller.
 *
 * Set-up: host code cannot use the array's name as a device address (on the host it is
 * only a stand-in symbol), so the first call on each device, with that device current,
 * looks the address up with cudaGetSymbolAddress and keeps it for the life of the
 * process.  Make that first call outside any stream capture.  The kept address belongs to
 * the device's context: after a cudaDeviceReset in the same process it is stale, and this
 * entry point must not be called on that device again.
 */
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/dgrain.h"
#include "dgr_ptr.h"
#include "dgr_scheme.cuh"

namespace {

/* Per node: the bounds as order-preserving 64-bit keys, [6][DGR_NOALLOC_MAX_NODES] (max
 * zeta, max Qx, max Qy, min zeta, min Qx, min Qy), and per variable the first element (in
 * index order) whose mean is a zero, [3][DGR_NOALLOC_MAX_NODES] as (element << 1 | sign). */
struct NoallocScratch {
    long long bounds[6 * DGR_NOALLOC_MAX_NODES];
    unsigned int first_zero[3 * DGR_NOALLOC_MAX_NODES];
};
static __device__ __align__(256) NoallocScratch g_noalloc;

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
NoallocScratch *g_scratch_ptr[kMaxDevices] = {nullptr};

/* Doubles compared as signed 64-bit integers: flipping the magnitude bits of negative
 * values makes integer order equal numeric order (NaN aside).  Both zeros map to the key
 * of +0, so that they tie as they do under the reference's comparisons. */
__device__ __forceinline__ long long dkey(double x)
{
    const long long b = __double_as_longlong(x == 0.0 ? 0.0 : x);
    return b ^ ((b >> 63) & 0x7fffffffffffffffLL);
}
__device__ __forceinline__ double dval(long long k)
{
    return __longlong_as_double(k ^ ((k >> 63) & 0x7fffffffffffffffLL));
}

/* The reference's starting values -99999 (max) and 99999 (min); no zero seen yet. */
__global__ void k_na_clear(NoallocScratch *sc, int nn)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    for (int v = 0; v < 3; ++v) {
        sc->bounds[v * DGR_NOALLOC_MAX_NODES + n] = dkey(-99999.0);
        sc->bounds[(3 + v) * DGR_NOALLOC_MAX_NODES + n] = dkey(99999.0);
        sc->first_zero[v * DGR_NOALLOC_MAX_NODES + n] = 0xffffffffu;
    }
}

/* Element means folded into the bounds of the element's three nodes.  The reference
 * scans a node's elements in index order with strict comparisons, so a bound that ends at
 * zero keeps the sign of the first zero mean in that order: atomicMin over
 * (element << 1 | sign bit) records it. */
__global__ void k_na_bounds(int ne, int nn, const int *__restrict__ el2v, const double *__restrict__ zeta,
                            const double *__restrict__ qx, const double *__restrict__ qy, NoallocScratch *sc)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= ne) return;
    const double *s[3] = {zeta, qx, qy};
    for (int v = 0; v < 3; ++v) {
        const double avg = (s[v][3 * el] + s[v][3 * el + 1] + s[v][3 * el + 2]) / 3;
        if (avg != avg) continue;
        const long long k = dkey(avg);
        const unsigned zero_tag = ((unsigned)el << 1) | (unsigned)(__double_as_longlong(avg) < 0 ? 1 : 0);
        for (int j = 0; j < 3; ++j) {
            const int n = el2v[3 * el + j];
            if (n < 0 || n >= nn) continue; /* out-of-range vertex: never touch memory outside */
            atomicMax(&sc->bounds[v * DGR_NOALLOC_MAX_NODES + n], k);
            atomicMin(&sc->bounds[(3 + v) * DGR_NOALLOC_MAX_NODES + n], k);
            if (avg == 0.0) atomicMin(&sc->first_zero[v * DGR_NOALLOC_MAX_NODES + n], zero_tag);
        }
    }
}

/* Element pass of the limiter (the same limit_core as the context limiter, without PDop)
 * on the reference layout [3*el+k]. */
__global__ void k_na_limit(int ne, int nn, const int *__restrict__ el2v, const double *__restrict__ z,
                           double *zeta, double *qx, double *qy, const NoallocScratch *__restrict__ sc, double h0)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= ne) return;
    const int nd[3] = {el2v[3 * el], el2v[3 * el + 1], el2v[3 * el + 2]};
    for (int k = 0; k < 3; ++k)
        if (nd[k] < 0 || nd[k] >= nn) return; /* out-of-range vertex: leave the element as it is */
    const double zn[3] = {z[nd[0]], z[nd[1]], z[nd[2]]};
    double *s[3] = {zeta, qx, qy};
    double w[3][3];
    for (int v = 0; v < 3; ++v)
        for (int k = 0; k < 3; ++k) w[v][k] = s[v][3 * el + k];
    const auto bnd = [sc, &nd](int v, int k, int is_min) {
        const double b = dval(sc->bounds[(3 * is_min + v) * DGR_NOALLOC_MAX_NODES + nd[k]]);
        if (b != 0.0) return b;
        return (sc->first_zero[v * DGR_NOALLOC_MAX_NODES + nd[k]] & 1u) ? -0.0 : 0.0;
    };
    dgr::LimitDecisions dec;
    dgr::limit_core<true, false, double>(w, bnd, zn, h0, 0.0, dec);
    if (dec.modify)
        for (int v = 0; v < 3; ++v)
            for (int k = 0; k < 3; ++k) s[v][3 * el + k] = w[v][k];
}

/* First call on a device: resolve the scratch array's device address. */
int scratch_for_current_device(int dev, NoallocScratch **out)
{
    if (dev < 0 || dev >= kMaxDevices) return DGR_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        NoallocScratch *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc);
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
    int dev = -1;
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e == cudaErrorNoDevice ? DGR_ERR_NO_DEVICE : DGR_ERR_CUDA;
    /* every caller array must be memory a kernel on this device may use (host-side check,
     * nothing launched yet) */
    for (const void *p : {(const void *)d_EltoVert, (const void *)d_z, (const void *)d_zeta, (const void *)d_Qx,
                          (const void *)d_Qy})
        if (!dgr_device_addressable(p, dev)) return DGR_ERR_INVALID;
    NoallocScratch *sc = nullptr;
    const int rc = scratch_for_current_device(dev, &sc);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    k_na_clear<<<(num_nodes + 255) / 256, 256, 0, s>>>(sc, num_nodes);
    k_na_bounds<<<(num_el + 255) / 256, 256, 0, s>>>(num_el, num_nodes, d_EltoVert, d_zeta, d_Qx, d_Qy, sc);
    k_na_limit<<<(num_el + 127) / 128, 128, 0, s>>>(num_el, num_nodes, d_EltoVert, d_z, d_zeta, d_Qx, d_Qy, sc, H0);
    return cudaGetLastError() == cudaSuccess ? DGR_OK : DGR_ERR_CUDA;
}
