/*
 * Mesh connectivity built on the GPU: the arrays of dgr_build_connectivity (EdgtoVert,
 * EdgtoEls, BdryPrescribed, minEdgLength of 2DCode/extract_mesh_attributes.c:143-361),
 * bit for bit, by sorting instead of the reference's O(E*N) searches.  The reference's
 * rules (restated in dgr_host.c) become:
 *   1. node adjacency in first-seen order: incidence record i = 2 (3 el + n) + j names
 *      neighbour j of local vertex n of element el; a stable radix sort of the records by
 *      (node, neighbour) leaves each pair's first record at the head of its run, and a
 *      second sort by (node, first record) gives every node's list in first-seen order;
 *   2. edges: the entries of that order whose neighbour is above the node, numbered by an
 *      exclusive scan;
 *   3. EdgtoEls: per edge the smallest element (atomicMin), then the smallest other
 *      element (second atomicMin pass), repeated when there is none;
 *   4. BdryPrescribed: each listed boundary pair ORs its list bit into its edge, then the
 *      reference's priority (second inflow list, first inflow list, outflow list);
 *   5. minEdgLength: the minimum over edges of the same expression, from 9999999 (a min is
 *      order-independent, so a parallel reduction gives the reference's bits).
 * Edges are looked up by binary search in the sorted (lower node, upper node) keys.
 * Restriction: every element has three distinct vertices (else DGR_ERR_MESH; the host
 * builder accepts such elements), and 6 x elements < 2^31.
 */
#include <cub/cub.cuh>

#include <climits>

#include "dgr_internal.cuh"

namespace {

using u64 = unsigned long long;

constexpr int NO_ELEMENT = 0x7f7f7f7f; /* byte-filled start value of the element slots, above any element */

__global__ void k_incidences(int ne, const int *__restrict__ el2v, u64 *__restrict__ key, int *__restrict__ rec)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 6LL * ne) return;
    const int el = (int)(i / 6), r = (int)(i % 6), n = r >> 1, j = r & 1;
    const int a = el2v[3 * el + n], c = el2v[3 * el + (n + 1 + j) % 3];
    key[i] = ((u64)a << 32) | (unsigned)c;
    rec[i] = (int)i;
}

/* run heads of the sorted (node, neighbour) keys */
__global__ void k_heads(long long n, const u64 *__restrict__ key, int *__restrict__ flag)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

/* unique (node, neighbour) -> key (node, first record), value neighbour */
__global__ void k_unique(long long n, const u64 *__restrict__ key, const int *__restrict__ rec,
                         const int *__restrict__ flag, const int *__restrict__ pos, u64 *__restrict__ ukey,
                         int *__restrict__ unb)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    const int p = pos[i];
    ukey[p] = (key[i] & 0xffffffff00000000ull) | (unsigned)rec[i];
    unb[p] = (int)(key[i] & 0xffffffffull);
}

__global__ void k_upper(int n, const u64 *__restrict__ ukey, const int *__restrict__ unb, int *__restrict__ flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flag[i] = unb[i] > (int)(ukey[i] >> 32) ? 1 : 0;
}

__global__ void k_edges(int n, const u64 *__restrict__ ukey, const int *__restrict__ unb, const int *__restrict__ flag,
                        const int *__restrict__ pos, int *__restrict__ ed2v, u64 *__restrict__ ekey,
                        int *__restrict__ eid)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    const int e = pos[i], a = (int)(ukey[i] >> 32), c = unb[i];
    ed2v[2 * e] = a;
    ed2v[2 * e + 1] = c;
    ekey[e] = ((u64)a << 32) | (unsigned)c;
    eid[e] = e;
}

__device__ int find_edge(int nf, const u64 *__restrict__ skey, const int *__restrict__ sid, int a, int b)
{
    const u64 k = a < b ? (((u64)a << 32) | (unsigned)b) : (((u64)b << 32) | (unsigned)a);
    int lo = 0, hi = nf;
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (skey[mid] < k)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < nf && skey[lo] == k) ? sid[lo] : -1;
}

/* pass 0: the smallest element of every edge; pass 1: the smallest other element */
__global__ void k_edge_elements(int ne, int nf, const int *__restrict__ el2v, const u64 *__restrict__ skey,
                                const int *__restrict__ sid, int *slot0, int *slot1, int pass, int *err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * ne) return;
    const int el = i / 3, k = i % 3;
    const int e = find_edge(nf, skey, sid, el2v[3 * el + k], el2v[3 * el + (k + 1) % 3]);
    if (e < 0) {
        atomicExch(err, 1);
        return;
    }
    if (pass == 0)
        atomicMin(slot0 + e, el);
    else if (slot0[e] != el)
        atomicMin(slot1 + e, el);
}

__global__ void k_boundary_bits(int nb, const int *__restrict__ pairs, int bit, int nf, const u64 *__restrict__ skey,
                                const int *__restrict__ sid, int *mask)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    const int e = find_edge(nf, skey, sid, pairs[2 * k], pairs[2 * k + 1]);
    if (e >= 0) atomicOr(mask + e, bit);
}

/* EdgtoEls, BdryPrescribed and the edge lengths' minimum */
__global__ void k_finish(int nf, const int *__restrict__ ed2v, const int *__restrict__ slot0,
                         const int *__restrict__ slot1, const int *__restrict__ mask, const double *__restrict__ x,
                         const double *__restrict__ y, int *__restrict__ ed2el, int *__restrict__ bdry,
                         u64 *min_bits)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nf) return;
    const int s0 = slot0[e], s1 = slot1[e];
    ed2el[2 * e] = s0;
    ed2el[2 * e + 1] = s1 == NO_ELEMENT ? s0 : s1;
    const int m = mask[e];
    bdry[e] = (m & 2) ? 3 : ((m & 1) ? 1 : ((m & 4) ? 2 : 0));
    const int n0 = ed2v[2 * e], n1 = ed2v[2 * e + 1];
    const double l = sqrt((x[n1] - x[n0]) * (x[n1] - x[n0]) + (y[n1] - y[n0]) * (y[n1] - y[n0]));
    /* non-negative doubles order as their bit patterns */
    atomicMin(min_bits, (u64)__double_as_longlong(l));
}

/* device buffers of one build, freed on every return path */
struct Bufs {
    std::vector<void *> p;
    ~Bufs()
    {
        for (void *q : p) cudaFree(q);
    }
    template <class T>
    int get(T **out, size_t n)
    {
        *out = nullptr;
        CK(cudaMalloc((void **)out, (n ? n : 1) * sizeof(T)));
        p.push_back(*out);
        return DGR_OK;
    }
};

int scan_exclusive(Bufs &b, const int *in, int *out, long long n, cudaStream_t s)
{
    size_t bytes = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    void *tmp = nullptr;
    int r = b.get((char **)&tmp, bytes);
    if (r) return r;
    CK(cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, s));
    return DGR_OK;
}

int sort_pairs(Bufs &b, cub::DoubleBuffer<u64> &keys, cub::DoubleBuffer<int> &vals, long long n, int end_bit,
               cudaStream_t s)
{
    size_t bytes = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, vals, n, 0, end_bit, s));
    void *tmp = nullptr;
    int r = b.get((char **)&tmp, bytes);
    if (r) return r;
    CK(cub::DeviceRadixSort::SortPairs(tmp, bytes, keys, vals, n, 0, end_bit, s));
    return DGR_OK;
}

int count_at(const int *flag, const int *pos, long long n, cudaStream_t s, long long *total)
{
    int a = 0, b = 0;
    CK(cudaMemcpyAsync(&a, flag + n - 1, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&b, pos + n - 1, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *total = (long long)a + b;
    return DGR_OK;
}

}  // namespace

extern "C" int dgr_build_connectivity_device(int ne, int nn, const int *el2v, const double *x, const double *y,
                                             int n_in1, const int *in1, int n_in2, const int *in2, int n_out,
                                             const int *out, int *ed2v, int *ed2el, int *bdry, double *min_edge)
{
    if (ne <= 0 || nn <= 0 || !el2v || !x || !y || !ed2v || !ed2el || !bdry || !min_edge) return DGR_ERR_INVALID;
    if (n_in1 < 0 || n_in2 < 0 || n_out < 0 || (n_in1 && !in1) || (n_in2 && !in2) || (n_out && !out))
        return DGR_ERR_INVALID;
    if ((long long)ne * 6 >= INT_MAX) return DGR_ERR_TOO_LARGE; /* record numbers are int */
    /* indices are checked here, so that no kernel reads out of bounds */
    for (long long i = 0; i < 3LL * ne; i += 3) {
        const int a = el2v[i], b = el2v[i + 1], c = el2v[i + 2];
        if (a < 0 || a >= nn || b < 0 || b >= nn || c < 0 || c >= nn) return DGR_ERR_MESH;
        if (a == b || b == c || a == c) return DGR_ERR_MESH;
    }
    const int *lists[3] = {in1, in2, out};
    const int counts[3] = {n_in1, n_in2, n_out};
    for (int l = 0; l < 3; ++l)
        for (long long k = 0; k < 2LL * counts[l]; ++k)
            if (lists[l][k] < 0 || lists[l][k] >= nn) return DGR_ERR_MESH;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    cudaStream_t s = nullptr;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{s};
    Bufs b;
    const long long nr = 6LL * ne;
    const long long nf_expect = (long long)nn + ne - 1;
    /* sort keys are (node << 32 | 32-bit payload): bits [0, 32 + bits of the largest node) */
    int end_bit = 33;
    while (end_bit < 64 && (1ull << (end_bit - 32)) < (unsigned long long)nn) ++end_bit;
    int *d_el2v, *rec0, *rec1, *flag, *pos, *unb0, *unb1, *d_ed2v, *eid0, *eid1, *slot0, *slot1, *mask, *d_ed2el,
        *d_bdry, *err;
    u64 *key0, *key1, *ekey0, *ekey1, *d_min;
    double *d_x, *d_y;
    int r = 0;
    if ((r = b.get(&d_el2v, 3 * (size_t)ne)) || (r = b.get(&d_x, nn)) || (r = b.get(&d_y, nn)) ||
        (r = b.get(&key0, nr)) || (r = b.get(&key1, nr)) || (r = b.get(&rec0, nr)) || (r = b.get(&rec1, nr)) ||
        (r = b.get(&flag, nr)) || (r = b.get(&pos, nr)) || (r = b.get(&err, 1)) || (r = b.get(&d_min, 1)))
        return r;
    CK(cudaMemcpyAsync(d_el2v, el2v, 12 * (size_t)ne, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_x, x, 8 * (size_t)nn, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_y, y, 8 * (size_t)nn, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(err, 0, 4, s));
    const unsigned T = 256;
    k_incidences<<<(unsigned)((nr + T - 1) / T), T, 0, s>>>(ne, d_el2v, key0, rec0);
    /* rule 1: stable sort by (node, neighbour); run heads hold each pair's first record */
    cub::DoubleBuffer<u64> kb(key0, key1);
    cub::DoubleBuffer<int> vb(rec0, rec1);
    if ((r = sort_pairs(b, kb, vb, nr, end_bit, s))) return r;
    k_heads<<<(unsigned)((nr + T - 1) / T), T, 0, s>>>(nr, kb.Current(), flag);
    if ((r = scan_exclusive(b, flag, pos, nr, s))) return r;
    long long nu = 0;
    if ((r = count_at(flag, pos, nr, s, &nu))) return r;
    if (nu != 2 * nf_expect) return DGR_ERR_MESH; /* every edge seen from both ends */
    u64 *uk0 = kb.Alternate(), *uk1 = nullptr;
    if ((r = b.get(&uk1, nu)) || (r = b.get(&unb0, nu)) || (r = b.get(&unb1, nu))) return r;
    k_unique<<<(unsigned)((nr + T - 1) / T), T, 0, s>>>(nr, kb.Current(), vb.Current(), flag, pos, uk0, unb0);
    /* ... and by (node, first record): every node's list in first-seen order */
    cub::DoubleBuffer<u64> ub(uk0, uk1);
    cub::DoubleBuffer<int> nbb(unb0, unb1);
    if ((r = sort_pairs(b, ub, nbb, nu, end_bit, s))) return r;
    /* rule 2 */
    const int n_u = (int)nu;
    k_upper<<<blocks(n_u, T), T, 0, s>>>(n_u, ub.Current(), nbb.Current(), flag);
    if ((r = scan_exclusive(b, flag, pos, nu, s))) return r;
    long long nf_ll = 0;
    if ((r = count_at(flag, pos, nu, s, &nf_ll))) return r;
    if (nf_ll != nf_expect) return DGR_ERR_MESH; /* Euler's relation, as the reference requires */
    const int nf = (int)nf_ll;
    if ((r = b.get(&d_ed2v, 2 * (size_t)nf)) || (r = b.get(&ekey0, nf)) || (r = b.get(&ekey1, nf)) ||
        (r = b.get(&eid0, nf)) || (r = b.get(&eid1, nf)) || (r = b.get(&slot0, nf)) || (r = b.get(&slot1, nf)) ||
        (r = b.get(&mask, nf)) || (r = b.get(&d_ed2el, 2 * (size_t)nf)) || (r = b.get(&d_bdry, nf)))
        return r;
    k_edges<<<blocks(n_u, T), T, 0, s>>>(n_u, ub.Current(), nbb.Current(), flag, pos, d_ed2v, ekey0, eid0);
    cub::DoubleBuffer<u64> eb(ekey0, ekey1);
    cub::DoubleBuffer<int> ib(eid0, eid1);
    if ((r = sort_pairs(b, eb, ib, nf, end_bit, s))) return r;
    /* rule 3 */
    CK(cudaMemsetAsync(slot0, 0x7f, 4 * (size_t)nf, s)); /* NO_ELEMENT */
    CK(cudaMemsetAsync(mask, 0, 4 * (size_t)nf, s));
    CK(cudaMemsetAsync(slot1, 0x7f, 4 * (size_t)nf, s));
    k_edge_elements<<<blocks(3 * ne, T), T, 0, s>>>(ne, nf, d_el2v, eb.Current(), ib.Current(), slot0, slot1, 0, err);
    k_edge_elements<<<blocks(3 * ne, T), T, 0, s>>>(ne, nf, d_el2v, eb.Current(), ib.Current(), slot0, slot1, 1, err);
    /* rule 4 */
    for (int l = 0; l < 3; ++l) {
        if (!counts[l]) continue;
        int *d_pairs = nullptr;
        if ((r = b.get(&d_pairs, 2 * (size_t)counts[l]))) return r;
        CK(cudaMemcpyAsync(d_pairs, lists[l], 8 * (size_t)counts[l], cudaMemcpyHostToDevice, s));
        k_boundary_bits<<<blocks(counts[l], T), T, 0, s>>>(counts[l], d_pairs, 1 << l, nf, eb.Current(), ib.Current(),
                                                           mask);
    }
    /* rules 3 (finish), 4 (priority), 5 */
    const double start = 9999999;
    u64 start_bits;
    memcpy(&start_bits, &start, 8);
    CK(cudaMemcpyAsync(d_min, &start_bits, 8, cudaMemcpyHostToDevice, s));
    k_finish<<<blocks(nf, T), T, 0, s>>>(nf, d_ed2v, slot0, slot1, mask, d_x, d_y, d_ed2el, d_bdry, d_min);
    CK(cudaGetLastError());
    int h_err = 0;
    u64 h_min = 0;
    CK(cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&h_min, d_min, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ed2v, d_ed2v, 8 * (size_t)nf, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ed2el, d_ed2el, 8 * (size_t)nf, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(bdry, d_bdry, 4 * (size_t)nf, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h_err) return DGR_ERR_MESH;
    memcpy(min_edge, &h_min, 8);
    return DGR_OK;
}
