/*
 * Device-side writer of the reference's snapshot files (2DCode/time_evolution.c:284-306,
 * 363-386: one element per line, each value as "%1.15f\t\t"): the lines are formatted on
 * the GPU from the device state (dgr_format.cuh, byte-identical to printf), in chunks of
 * elements: a length pass, an exclusive scan of the line lengths, a write pass, then one
 * copy of the chunk's bytes to pinned host memory and one fwrite.  The state itself never
 * leaves the device.
 */
#include <cub/cub.cuh>

#include "dgr_format.cuh"
#include "dgr_internal.cuh"

using namespace dgr;

namespace {

constexpr int DAT_CHUNK = 1 << 18; /* elements per pass */

/* length of each element's line: nm values + 2 tabs each, then '\n'; bad = 1 if a value
 * cannot be formatted (|v| >= 2^63) */
__global__ void __launch_bounds__(128) k_dat_len(int n, int ld, int nm, const double *__restrict__ V,
                                                 int *__restrict__ len, int *bad)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el > n) return;
    if (el == n) {
        len[n] = 0; /* the scan's last entry is the chunk's byte count */
        return;
    }
    char buf[F15_MAX];
    int L = 1;
    for (int k = 0; k < nm; ++k) {
        const int l = format_f15(V[(size_t)k * ld + el], buf);
        if (l < 0) {
            *bad = 1;
            continue;
        }
        L += l + 2;
    }
    len[el] = L;
}

__global__ void __launch_bounds__(128) k_dat_write(int n, int ld, int nm, const double *__restrict__ V,
                                                   const int *__restrict__ off, char *__restrict__ out)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= n) return;
    char line[8 * (F15_MAX + 2) + 1];
    int p = 0;
    for (int k = 0; k < nm; ++k) {
        const int l = format_f15(V[(size_t)k * ld + el], line + p);
        if (l < 0) continue; /* refused by the length pass */
        p += l;
        line[p++] = '\t';
        line[p++] = '\t';
    }
    line[p++] = '\n';
    char *dst = out + off[el];
    for (int j = 0; j < p; ++j) dst[j] = line[j];
}

struct DatScratch {
    int *len = nullptr, *off = nullptr, *bad = nullptr;
    void *scan = nullptr;
    char *buf = nullptr, *host = nullptr;
    size_t scan_bytes = 0;
    ~DatScratch()
    {
        cudaFree(len);
        cudaFree(off);
        cudaFree(bad);
        cudaFree(scan);
        cudaFree(buf);
        if (host) cudaFreeHost(host);
    }
};

/* values planes V[k * ldE + el], k < nm, elements [0, n) -> path */
int write_planes(dgr_ctx *c, const char *path, const double *V, int n, DatScratch &s)
{
    cudaStream_t st = c->stream;
    const int nm = c->nm;
    CK(cudaMemsetAsync(s.bad, 0, 4, st));
    FILE *f = fopen(path, "wb");
    if (!f) return DGR_ERR_IO;
    int rc = DGR_OK;
    for (int e0 = 0; e0 < n && rc == DGR_OK; e0 += DAT_CHUNK) {
        const int cnt = std::min(DAT_CHUNK, n - e0);
        k_dat_len<<<blocks(cnt + 1, 128), 128, 0, st>>>(cnt, c->ldE, nm, V + e0, s.len, s.bad);
        size_t sb = s.scan_bytes;
        if (cub::DeviceScan::ExclusiveSum(s.scan, sb, s.len, s.off, cnt + 1, st) != cudaSuccess) {
            rc = DGR_ERR_CUDA;
            break;
        }
        k_dat_write<<<blocks(cnt, 128), 128, 0, st>>>(cnt, c->ldE, nm, V + e0, s.off, s.buf);
        c->launches += 3;
        int hdr[2];
        cudaError_t e = cudaMemcpyAsync(hdr, s.off + cnt, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hdr + 1, s.bad, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            snprintf(dgr_cuda_err_buffer(), 256, "dat writer: %s", cudaGetErrorString(e));
            rc = DGR_ERR_CUDA;
            break;
        }
        if (hdr[1]) {
            rc = DGR_ERR_INVALID;
            break;
        }
        e = cudaMemcpyAsync(s.host, s.buf, (size_t)hdr[0], cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            snprintf(dgr_cuda_err_buffer(), 256, "dat writer: %s", cudaGetErrorString(e));
            rc = DGR_ERR_CUDA;
            break;
        }
        if (fwrite(s.host, 1, (size_t)hdr[0], f) != (size_t)hdr[0]) rc = DGR_ERR_IO;
    }
    if (fclose(f) != 0 && rc == DGR_OK) rc = DGR_ERR_IO;
    if (rc != DGR_OK) remove(path);
    return rc;
}

int write_state(dgr_ctx *c, int scenario, const char *zeta_path, const char *qx_path, const char *qy_path)
{
    if (!c || scenario < 0 || scenario >= c->nscen) return DGR_ERR_INVALID;
    if (!zeta_path && !qx_path && !qy_path) return DGR_OK;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    const int el0 = c->el_off[scenario], n = c->el_off[scenario + 1] - el0;
    const int chunk = std::min(DAT_CHUNK, n);
    const size_t line_max = (size_t)c->nm * (F15_MAX + 2) + 1;
    DatScratch s;
    CK(cudaMalloc((void **)&s.len, (size_t)(chunk + 1) * 4));
    CK(cudaMalloc((void **)&s.off, (size_t)(chunk + 1) * 4));
    CK(cudaMalloc((void **)&s.bad, 4));
    CK(cub::DeviceScan::ExclusiveSum(nullptr, s.scan_bytes, s.len, s.off, chunk + 1, c->stream));
    CK(cudaMalloc(&s.scan, s.scan_bytes ? s.scan_bytes : 1));
    CK(cudaMalloc((void **)&s.buf, line_max * chunk));
    CK(cudaHostAlloc((void **)&s.host, line_max * chunk, cudaHostAllocDefault));
    const char *paths[3] = {zeta_path, qx_path, qy_path};
    for (int v = 0; v < 3; ++v) {
        if (!paths[v]) continue;
        const int r = write_planes(c, paths[v], c->U + (size_t)v * c->nm * c->ldE + el0, n, s);
        if (r) return r;
    }
    return DGR_OK;
}

}  // namespace

extern "C" int dgr_write_state_dat(dgr_ctx *c, const char *zeta_path, const char *qx_path, const char *qy_path)
{
    if (!c || c->nscen != 1) return DGR_ERR_INVALID;
    return write_state(c, 0, zeta_path, qx_path, qy_path);
}

extern "C" int dgr_ensemble_write_state_dat(dgr_ctx *c, int scenario, const char *zeta_path, const char *qx_path,
                                            const char *qy_path)
{
    return write_state(c, scenario, zeta_path, qx_path, qy_path);
}
