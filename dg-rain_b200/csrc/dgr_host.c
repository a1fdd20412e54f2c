/*
 * Host-side mesh ingest and I/O of the C ABI (include/dgrain.h).  Plain C99, no GPU.
 *
 *  dgr_read_fort14        <- store_mesh, 2DCode/extract_mesh_attributes.c:39-141
 *  dgr_build_connectivity <- extract_mesh_attributes, 2DCode/extract_mesh_attributes.c:143-361
 *  dgr_initial_state      <- initialize, 2DCode/initialize.c:117-126
 *  dgr_write_dat          <- the .dat writer of 2DCode/time_evolution.c:284-306,363-386
 *
 * The connectivity builder must give the reference's arrays exactly, because edge
 * numbering decides which element is "in" for every edge and therefore the sign and
 * rounding of every flux.  The reference's rules, restated:
 *   1. Node adjacency in first-seen order: elements in index order, and for local
 *      vertex n of an element the neighbours v[(n+1)%3] then v[(n+2)%3] are appended
 *      when not yet listed (:166-212).
 *   2. Edges numbered by their lower node, then by the position of the higher node in
 *      the lower node's adjacency list (:225-250).
 *   3. EdgtoEls: the first two elements, in index order, that own the edge; an edge with
 *      one element repeats it in both slots (:259-295).
 *   4. BdryPrescribed: 3 if the edge is in the second inflow list, else 1 if in the first
 *      inflow list, else 2 if in the outflow list, else 0 (:297-354).
 *   5. minEdgLength: the running min over edges in edge order, from 9999999 (:25,:302-303).
 * The reference searches with O(E*N) loops; this version uses per-node lists and an
 * open-addressing hash of node pairs, O(E) overall.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/dgrain.h"

/* ------------------------------------------------------------------ fort.14 ---- */

static int read_line(FILE *f, char *buf, int n) { return fgets(buf, n, f) != NULL; }

static int read_pairs(FILE *f, int *count, int **pairs)
{
    char line[1024];
    *count = 0;
    *pairs = NULL;
    if (!read_line(f, line, sizeof line)) return DGR_ERR_IO;
    if (sscanf(line, "%d", count) != 1 || *count < 0) return DGR_ERR_IO;
    *pairs = (int *)malloc(sizeof(int) * 2 * (size_t)(*count ? *count : 1));
    if (!*pairs) return DGR_ERR_TOO_LARGE;
    for (int k = 0; k < *count; ++k) {
        int a, b;
        if (!read_line(f, line, sizeof line) || sscanf(line, "%d %d", &a, &b) != 2) return DGR_ERR_IO;
        (*pairs)[2 * k] = a - 1;
        (*pairs)[2 * k + 1] = b - 1;
    }
    return DGR_OK;
}

void dgr_fort14_free(dgr_fort14 *m)
{
    if (!m) return;
    free(m->x_coord);
    free(m->y_coord);
    free(m->z);
    free(m->nFriction);
    free(m->EltoVert);
    free(m->inflow1);
    free(m->inflow2);
    free(m->outflow);
    free(m);
}

int dgr_read_fort14(const char *path, dgr_fort14 **out)
{
    if (!path || !out) return DGR_ERR_INVALID;
    *out = NULL;
    FILE *f = fopen(path, "r");
    if (!f) return DGR_ERR_IO;
    dgr_fort14 *m = (dgr_fort14 *)calloc(1, sizeof(dgr_fort14));
    char line[1024];
    int rc = DGR_ERR_IO;
    if (!m) {
        rc = DGR_ERR_TOO_LARGE;
        goto fail;
    }
    if (!read_line(f, line, sizeof line)) goto fail; /* title */
    if (!read_line(f, line, sizeof line) || sscanf(line, "%d %d", &m->num_el, &m->num_nodes) != 2)
        goto fail;
    if (m->num_el <= 0 || m->num_nodes <= 0) goto fail;
    size_t nn = (size_t)m->num_nodes, ne = (size_t)m->num_el;
    m->x_coord = (double *)malloc(nn * sizeof(double));
    m->y_coord = (double *)malloc(nn * sizeof(double));
    m->z = (double *)malloc(nn * sizeof(double));
    m->nFriction = (double *)malloc(nn * sizeof(double));
    m->EltoVert = (int *)malloc(3 * ne * sizeof(int));
    if (!m->x_coord || !m->y_coord || !m->z || !m->nFriction || !m->EltoVert) {
        rc = DGR_ERR_TOO_LARGE;
        goto fail;
    }
    /* node lines "id x y z n" (:62-69); strtod rounds exactly like the reference's %lf */
    for (size_t j = 0; j < nn; ++j) {
        if (!read_line(f, line, sizeof line)) goto fail;
        char *p = line, *q;
        strtol(p, &q, 10);
        if (q == p) goto fail;
        p = q;
        double v[4];
        for (int t = 0; t < 4; ++t) {
            v[t] = strtod(p, &q);
            if (q == p) goto fail;
            p = q;
        }
        m->x_coord[j] = v[0];
        m->y_coord[j] = v[1];
        m->z[j] = v[2];
        m->nFriction[j] = v[3];
    }
    /* element lines "id 3 v1 v2 v3", 1-based (:74-84) */
    for (size_t j = 0; j < ne; ++j) {
        int id, nv, a, b, c;
        if (!read_line(f, line, sizeof line) || sscanf(line, "%d %d %d %d %d", &id, &nv, &a, &b, &c) != 5)
            goto fail;
        m->EltoVert[3 * j] = a - 1;
        m->EltoVert[3 * j + 1] = b - 1;
        m->EltoVert[3 * j + 2] = c - 1;
        if (a < 1 || b < 1 || c < 1 || a > m->num_nodes || b > m->num_nodes || c > m->num_nodes) {
            rc = DGR_ERR_MESH;
            goto fail;
        }
    }
    if (!read_line(f, line, sizeof line)) goto fail; /* discarded line (:87-88) */
    if ((rc = read_pairs(f, &m->num_inflow1, &m->inflow1))) goto fail;
    if ((rc = read_pairs(f, &m->num_inflow2, &m->inflow2))) goto fail;
    if ((rc = read_pairs(f, &m->num_outflow, &m->outflow))) goto fail;
    fclose(f);
    *out = m;
    return DGR_OK;
fail:
    fclose(f);
    dgr_fort14_free(m);
    return rc == DGR_OK ? DGR_ERR_IO : rc;
}

/* ------------------------------------------------------------ connectivity ---- */

/* open-addressing hash of unordered node pairs -> small payload */
typedef struct {
    uint64_t *keys; /* (lo << 32 | hi) + 1, 0 = empty */
    int *vals;
    size_t mask;
} pair_map;

static uint64_t pair_key(int a, int b)
{
    uint32_t lo = (uint32_t)(a < b ? a : b), hi = (uint32_t)(a < b ? b : a);
    return (((uint64_t)lo << 32) | hi) + 1;
}

static size_t hash64(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return (size_t)k;
}

static int pm_init(pair_map *m, size_t n)
{
    size_t cap = 16;
    while (cap < 2 * n + 16) cap <<= 1;
    m->keys = (uint64_t *)calloc(cap, sizeof(uint64_t));
    m->vals = (int *)malloc(cap * sizeof(int));
    m->mask = cap - 1;
    return (m->keys && m->vals) ? 0 : -1;
}

static void pm_free(pair_map *m)
{
    free(m->keys);
    free(m->vals);
}

/* returns pointer to the value slot; *inserted = 1 if new */
static int *pm_slot(pair_map *m, uint64_t key, int *inserted)
{
    size_t h = hash64(key) & m->mask;
    for (;;) {
        if (m->keys[h] == key) {
            *inserted = 0;
            return &m->vals[h];
        }
        if (m->keys[h] == 0) {
            m->keys[h] = key;
            *inserted = 1;
            return &m->vals[h];
        }
        h = (h + 1) & m->mask;
    }
}

static const int *pm_find(const pair_map *m, uint64_t key)
{
    size_t h = hash64(key) & m->mask;
    for (;;) {
        if (m->keys[h] == key) return &m->vals[h];
        if (m->keys[h] == 0) return NULL;
        h = (h + 1) & m->mask;
    }
}

/* Adjacency lists in the reference's first-seen order (rule 1).  adj_ptr has num_nodes+1
 * entries; list of node n is adj[adj_ptr[n] .. adj_ptr[n]+adj_len[n]). */
static int build_adjacency(int ne, int nn, const int *el2v, int **adj_ptr_out, int **adj_len_out,
                           int **adj_out)
{
    int *ptr = (int *)calloc((size_t)nn + 1, sizeof(int));
    int *len = (int *)calloc((size_t)nn, sizeof(int));
    if (!ptr || !len) {
        free(ptr);
        free(len);
        return DGR_ERR_TOO_LARGE;
    }
    for (size_t i = 0; i < 3 * (size_t)ne; ++i) {
        int v = el2v[i];
        if (v < 0 || v >= nn) {
            free(ptr);
            free(len);
            return DGR_ERR_MESH;
        }
        ptr[v + 1] += 2; /* each incidence adds at most two neighbours */
    }
    for (int n = 0; n < nn; ++n) ptr[n + 1] += ptr[n];
    int *adj = (int *)malloc(sizeof(int) * (size_t)(ptr[nn] ? ptr[nn] : 1));
    if (!adj) {
        free(ptr);
        free(len);
        return DGR_ERR_TOO_LARGE;
    }
    for (int el = 0; el < ne; ++el) {
        for (int n = 0; n < 3; ++n) {
            int node = el2v[3 * el + n];
            int nb0 = el2v[3 * el + (n + 1) % 3], nb1 = el2v[3 * el + (n + 2) % 3];
            int *lst = adj + ptr[node];
            int f0 = 0, f1 = 0;
            for (int j = 0; j < len[node]; ++j) {
                if (lst[j] == nb0) f0 = 1;
                if (lst[j] == nb1) f1 = 1;
            }
            if (!f0) lst[len[node]++] = nb0;
            if (!f1) lst[len[node]++] = nb1;
        }
    }
    *adj_ptr_out = ptr;
    *adj_len_out = len;
    *adj_out = adj;
    return DGR_OK;
}

int dgr_count_edges(int ne, int nn, const int *el2v, int *num_edges)
{
    if (ne <= 0 || nn <= 0 || !el2v || !num_edges) return DGR_ERR_INVALID;
    int *ptr, *len, *adj;
    int rc = build_adjacency(ne, nn, el2v, &ptr, &len, &adj);
    if (rc) return rc;
    long long cnt = 0;
    for (int n = 0; n < nn; ++n)
        for (int k = 0; k < len[n]; ++k)
            if (adj[ptr[n] + k] > n) ++cnt;
    free(ptr);
    free(len);
    free(adj);
    *num_edges = (int)cnt;
    return DGR_OK;
}

int dgr_build_connectivity(int ne, int nn, const int *el2v, const double *x, const double *y,
                           int n_in1, const int *in1, int n_in2, const int *in2, int n_out,
                           const int *out, int *ed2v, int *ed2el, int *bdry, double *min_edge)
{
    if (ne <= 0 || nn <= 0 || !el2v || !x || !y || !ed2v || !ed2el || !bdry || !min_edge)
        return DGR_ERR_INVALID;
    const long long nf_expect = (long long)nn + ne - 1; /* Euler's relation (:218-219) */
    int *ptr, *len, *adj;
    int rc = build_adjacency(ne, nn, el2v, &ptr, &len, &adj);
    if (rc) return rc;

    /* rule 2: edge numbering; edge id of (n, adj[..]) stored alongside for lookup */
    pair_map em;
    if (pm_init(&em, (size_t)nf_expect)) {
        rc = DGR_ERR_TOO_LARGE;
        goto done0;
    }
    long long cnt = 0;
    for (int n = 0; n < nn; ++n) {
        for (int k = 0; k < len[n]; ++k) {
            int c = adj[ptr[n] + k];
            if (c > n) {
                if (cnt >= nf_expect) {
                    rc = DGR_ERR_MESH;
                    goto done1;
                }
                ed2v[2 * cnt] = n;
                ed2v[2 * cnt + 1] = c;
                int ins;
                *pm_slot(&em, pair_key(n, c), &ins) = (int)cnt;
                ++cnt;
            }
        }
    }
    if (cnt != nf_expect) {
        rc = DGR_ERR_MESH;
        goto done1;
    }
    const int nf = (int)cnt;

    /* rule 3: element slots in element order */
    for (int e = 0; e < nf; ++e) ed2el[2 * e] = ed2el[2 * e + 1] = -1;
    for (int el = 0; el < ne; ++el) {
        for (int k = 0; k < 3; ++k) {
            int a = el2v[3 * el + k], b = el2v[3 * el + (k + 1) % 3];
            if (a == b) continue;
            const int *pe = pm_find(&em, pair_key(a, b));
            if (!pe) {
                rc = DGR_ERR_MESH;
                goto done1;
            }
            int e = *pe;
            /* one element counts once per edge even if it matched twice */
            if (ed2el[2 * e] == el || ed2el[2 * e + 1] == el) continue;
            if (ed2el[2 * e] < 0)
                ed2el[2 * e] = el;
            else if (ed2el[2 * e + 1] < 0)
                ed2el[2 * e + 1] = el;
        }
    }
    for (int e = 0; e < nf; ++e)
        if (ed2el[2 * e + 1] < 0) ed2el[2 * e + 1] = ed2el[2 * e];

    /* rule 4: boundary types */
    {
        pair_map bm;
        if (pm_init(&bm, (size_t)(n_in1 + n_in2 + n_out))) {
            rc = DGR_ERR_TOO_LARGE;
            goto done1;
        }
        /* bit 1: inflow-1, bit 2: inflow-2, bit 4: outflow */
        const int *lists[3] = {in1, in2, out};
        const int counts[3] = {n_in1, n_in2, n_out};
        for (int l = 0; l < 3; ++l)
            for (int k = 0; k < counts[l]; ++k) {
                int ins;
                int *v = pm_slot(&bm, pair_key(lists[l][2 * k], lists[l][2 * k + 1]), &ins);
                if (ins) *v = 0;
                *v |= (1 << l);
            }
        for (int e = 0; e < nf; ++e) {
            const int *v = pm_find(&bm, pair_key(ed2v[2 * e], ed2v[2 * e + 1]));
            int m = v ? *v : 0;
            if (m & 2)
                bdry[e] = 3;
            else if (m & 1)
                bdry[e] = 1;
            else if (m & 4)
                bdry[e] = 2;
            else
                bdry[e] = 0;
        }
        pm_free(&bm);
    }

    /* rule 5 */
    double me = 9999999;
    for (int e = 0; e < nf; ++e) {
        int n0 = ed2v[2 * e], n1 = ed2v[2 * e + 1];
        double l = sqrt((x[n1] - x[n0]) * (x[n1] - x[n0]) + (y[n1] - y[n0]) * (y[n1] - y[n0]));
        me = (me < l) ? me : l;
    }
    *min_edge = me;
    rc = DGR_OK;
done1:
    pm_free(&em);
done0:
    free(ptr);
    free(len);
    free(adj);
    return rc;
}

/* ---------------------------------------------------------------- state / io ---- */

int dgr_initial_state(int ne, const int *el2v, const double *zeta_nodal, double *zeta, double *qx,
                      double *qy, int *wd)
{
    if (ne <= 0 || !el2v || !zeta || !qx || !qy) return DGR_ERR_INVALID;
    for (int el = 0; el < ne; ++el) {
        double nz[3];
        for (int k = 0; k < 3; ++k) {
            nz[k] = zeta_nodal ? zeta_nodal[el2v[3 * el + k]] : 0.1;
            qx[3 * el + k] = 0;
            qy[3 * el + k] = 0;
        }
        zeta[3 * el] = 0.5 * (nz[0] + nz[1]);
        zeta[3 * el + 1] = 0.5 * (nz[1] + nz[2]);
        zeta[3 * el + 2] = 0.5 * (nz[2] + nz[0]);
        if (wd) wd[el] = -1;
    }
    return DGR_OK;
}

int dgr_write_dat(const char *path, int ne, const double *v)
{
    if (!path || ne <= 0 || !v) return DGR_ERR_INVALID;
    FILE *f = fopen(path, "w");
    if (!f) return DGR_ERR_IO;
    for (int j = 0; j < ne; ++j) {
        for (int k = 0; k < 3; ++k) fprintf(f, "%1.15f\t\t", v[3 * j + k]);
        fprintf(f, "\n");
    }
    return fclose(f) == 0 ? DGR_OK : DGR_ERR_IO;
}

/* ---------------------------------------------------------------- restart ---- */

/* Restart file: the .dat row layout of the state (one element per line, tab-separated,
 * 2DCode/time_evolution.c:284-306) with every value printed with 17 significant digits,
 * which strtod reads back to the same double (signed zeros included), followed by the
 * element's wet/dry flag; a three-line header gives the format, the sizes and the clock.
 *
 *   DG-RAIN restart 1
 *   <num_el> <nm>
 *   time <t> dt <dt>
 *   z_0 .. z_{nm-1}  Qx_0 .. Qx_{nm-1}  Qy_0 .. Qy_{nm-1}  WD      (num_el lines)
 */
static const char RESTART_MAGIC[] = "DG-RAIN restart 1";

int dgr_write_restart(const char *path, int ne, int nm, const double *zeta, const double *qx, const double *qy,
                      const int *wd, double time, double dt)
{
    if (!path || ne <= 0 || nm <= 0 || !zeta || !qx || !qy || !wd) return DGR_ERR_INVALID;
    FILE *f = fopen(path, "w");
    if (!f) return DGR_ERR_IO;
    fprintf(f, "%s\n%d %d\ntime %.17g dt %.17g\n", RESTART_MAGIC, ne, nm, time, dt);
    const double *vars[3] = {zeta, qx, qy};
    for (int j = 0; j < ne; ++j) {
        for (int v = 0; v < 3; ++v)
            for (int k = 0; k < nm; ++k) fprintf(f, "%.17g\t\t", vars[v][(size_t)nm * j + k]);
        fprintf(f, "%d\n", wd[j]);
    }
    return fclose(f) == 0 ? DGR_OK : DGR_ERR_IO;
}

/* reads one whitespace-separated number; 0 on success */
static int next_double(char **p, double *out)
{
    char *q;
    *out = strtod(*p, &q);
    if (q == *p) return 1;
    *p = q;
    return 0;
}

int dgr_read_restart(const char *path, int ne, int nm, double *zeta, double *qx, double *qy, int *wd,
                     double *time, double *dt)
{
    if (!path || ne <= 0 || nm <= 0 || !zeta || !qx || !qy || !wd || !time || !dt) return DGR_ERR_INVALID;
    FILE *f = fopen(path, "r");
    if (!f) return DGR_ERR_IO;
    int rc = DGR_ERR_IO;
    size_t cap = 64 + 3 * (size_t)nm * 32;
    char *line = (char *)malloc(cap);
    if (!line) {
        fclose(f);
        return DGR_ERR_TOO_LARGE;
    }
    int fne = 0, fnm = 0;
    if (!fgets(line, (int)cap, f) || strncmp(line, RESTART_MAGIC, sizeof RESTART_MAGIC - 1) != 0) goto done;
    if (!fgets(line, (int)cap, f) || sscanf(line, "%d %d", &fne, &fnm) != 2) goto done;
    if (fne != ne || fnm != nm) {
        rc = DGR_ERR_MESH; /* written for another mesh or order */
        goto done;
    }
    {
        char *p = line;
        if (!fgets(line, (int)cap, f) || strncmp(p, "time", 4) != 0) goto done;
        p += 4;
        if (next_double(&p, time)) goto done;
        while (*p == ' ' || *p == '\t') ++p;
        if (strncmp(p, "dt", 2) != 0) goto done;
        p += 2;
        if (next_double(&p, dt)) goto done;
    }
    double *vars[3] = {zeta, qx, qy};
    for (int j = 0; j < ne; ++j) {
        if (!fgets(line, (int)cap, f)) goto done;
        char *p = line;
        for (int v = 0; v < 3; ++v)
            for (int k = 0; k < nm; ++k)
                if (next_double(&p, &vars[v][(size_t)nm * j + k])) goto done;
        char *q;
        const long w = strtol(p, &q, 10);
        if (q == p || w < -1 || w > 1) goto done;
        wd[j] = (int)w;
    }
    rc = DGR_OK;
done:
    free(line);
    fclose(f);
    return rc;
}

const char *dgr_status_string(int code)
{
    switch (code) {
    case DGR_OK: return "ok";
    case DGR_ERR_NAN_FLUX: return "numerical flux not a number";
    case DGR_ERR_NAN_FLUX_IN: return "interior element dry flux not a number";
    case DGR_ERR_NAN_FLUX_EX: return "exterior element dry flux not a number";
    case DGR_ERR_NEG_DEPTH: return "water height negative during wetting and drying treatment";
    case DGR_ERR_NAN_VELOCITY: return "WD-modified velocity NaN";
    case DGR_ERR_EDGE_MATCH: return "local edge number not found";
    case DGR_ERR_BAD_INDEX: return "connectivity index out of range (checked build)";
    case DGR_ERR_INVALID: return "invalid argument";
    case DGR_ERR_MESH: return "inconsistent mesh";
    case DGR_ERR_IO: return "file i/o error";
    case DGR_ERR_CUDA: return "CUDA error";
    case DGR_ERR_NO_DEVICE: return "no CUDA device";
    case DGR_ERR_TOO_LARGE: return "size beyond limit";
    case DGR_ERR_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
    }
}

int dgr_abi_version(void) { return DGR_ABI_VERSION; }
