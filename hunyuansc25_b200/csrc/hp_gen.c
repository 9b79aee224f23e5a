/*
 * hp_gen.c — seeded synthetic graph generators (host C, OpenMP).
 * Interface and conventions: include/hp_gen.h.
 */
#include "hp_gen.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

uint64_t hp_gen_mix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

int32_t hp_gen_edge_weight(uint64_t seed, int32_t u, int32_t v, int32_t wmin, int32_t wmax)
{
    if (wmax <= wmin) return wmin;
    uint32_t a = (uint32_t)(u < v ? u : v), b = (uint32_t)(u < v ? v : u);
    uint64_t h = hp_gen_mix64(hp_gen_mix64(seed ^ 0x5eedc0deULL) ^ (((uint64_t)a << 32) | b));
    return wmin + (int32_t)(h % (uint64_t)(wmax - wmin + 1));
}

void hp_gen_set_threads(int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

void hp_graph_free(hp_graph *g)
{
    if (!g) return;
    free(g->xadj); free(g->adjncy); free(g->vwgt); free(g->adjwgt);
    memset(g, 0, sizeof(*g));
}

static int alloc_graph(hp_graph *g, int32_t n, int64_t m)
{
    memset(g, 0, sizeof(*g));
    g->nvtxs = n;
    g->nedges = m;
    g->xadj = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n + 1));
    g->adjncy = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    g->adjwgt = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    g->vwgt = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    if (!g->xadj || !g->adjncy || !g->adjwgt || !g->vwgt) { hp_graph_free(g); return -3; }
    for (int64_t i = 0; i < n; i++) g->vwgt[i] = 1;
    return 0;
}

static void fill_weights(hp_graph *g, uint64_t seed, int32_t wmin, int32_t wmax)
{
    const int32_t n = g->nvtxs;
#pragma omp parallel for schedule(dynamic, 4096)
    for (int32_t v = 0; v < n; v++)
        for (int64_t j = g->xadj[v]; j < g->xadj[v + 1]; j++)
            g->adjwgt[j] = hp_gen_edge_weight(seed, v, g->adjncy[j], wmin, wmax);
}

int hp_gen_grid2d(int32_t nx, int32_t ny, uint64_t seed, int32_t wmin, int32_t wmax, hp_graph *out)
{
    if (nx <= 0 || ny <= 0 || !out) return -1;
    int64_t n = (int64_t)nx * ny;
    if (n > INT32_MAX - 1) return -7;
    int64_t m = 2 * ((int64_t)(nx - 1) * ny + (int64_t)nx * (ny - 1));
    int rc = alloc_graph(out, (int32_t)n, m);
    if (rc) return rc;
    /* degree of (x,y) = [y>0] + [x>0] + [x<nx-1] + [y<ny-1]; rows in id order */
    int64_t e = 0;
    for (int32_t y = 0; y < ny; y++)
        for (int32_t x = 0; x < nx; x++) {
            int32_t v = y * nx + x;
            out->xadj[v] = (int32_t)e;
            if (y > 0) out->adjncy[e++] = v - nx;
            if (x > 0) out->adjncy[e++] = v - 1;
            if (x < nx - 1) out->adjncy[e++] = v + 1;
            if (y < ny - 1) out->adjncy[e++] = v + nx;
        }
    out->xadj[n] = (int32_t)e;
    fill_weights(out, seed, wmin, wmax);
    return 0;
}

int hp_gen_grid3d(int32_t nx, int32_t ny, int32_t nz, uint64_t seed, int32_t wmin,
                  int32_t wmax, hp_graph *out)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || !out) return -1;
    int64_t n = (int64_t)nx * ny * nz;
    if (n > INT32_MAX - 1) return -7;
    int64_t m = 2 * ((int64_t)(nx - 1) * ny * nz + (int64_t)nx * (ny - 1) * nz +
                     (int64_t)nx * ny * (nz - 1));
    if (m > INT32_MAX) return -7;
    int rc = alloc_graph(out, (int32_t)n, m);
    if (rc) return rc;
    const int32_t pl = nx * ny;
    int64_t e = 0;
    for (int32_t z = 0; z < nz; z++)
        for (int32_t y = 0; y < ny; y++)
            for (int32_t x = 0; x < nx; x++) {
                int32_t v = (z * ny + y) * nx + x;
                out->xadj[v] = (int32_t)e;
                if (z > 0) out->adjncy[e++] = v - pl;
                if (y > 0) out->adjncy[e++] = v - nx;
                if (x > 0) out->adjncy[e++] = v - 1;
                if (x < nx - 1) out->adjncy[e++] = v + 1;
                if (y < ny - 1) out->adjncy[e++] = v + nx;
                if (z < nz - 1) out->adjncy[e++] = v + pl;
            }
    out->xadj[n] = (int32_t)m;
    fill_weights(out, seed, wmin, wmax);
    return 0;
}

static int cmp_i32(const void *a, const void *b)
{
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

static void sort_row(int32_t *r, int64_t len)
{
    if (len < 24) {
        for (int64_t i = 1; i < len; i++) {
            int32_t t = r[i];
            int64_t j = i - 1;
            while (j >= 0 && r[j] > t) { r[j + 1] = r[j]; j--; }
            r[j + 1] = t;
        }
    } else {
        qsort(r, (size_t)len, sizeof(int32_t), cmp_i32);
    }
}

/* Build a simple symmetric CSR from directed pair lists (both directions
 * present): bucket by source, sort rows, drop duplicates, compact. */
static int csr_from_pairs(int32_t n, int64_t npairs, const int32_t *src, const int32_t *dst,
                          hp_graph *out)
{
    int64_t *cnt = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    if (!cnt) return -3;
    for (int64_t i = 0; i < npairs; i++) cnt[src[i] + 1]++;
    for (int32_t v = 0; v < n; v++) cnt[v + 1] += cnt[v];
    int32_t *tmp = (int32_t *)malloc(sizeof(int32_t) * (size_t)(npairs > 0 ? npairs : 1));
    int64_t *pos = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1));
    if (!tmp || !pos) { free(cnt); free(tmp); free(pos); return -3; }
    memcpy(pos, cnt, sizeof(int64_t) * ((size_t)n + 1));
    for (int64_t i = 0; i < npairs; i++) tmp[pos[src[i]]++] = dst[i];
    free(pos);
    int64_t *ulen = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1));
    if (!ulen) { free(cnt); free(tmp); return -3; }
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t v = 0; v < n; v++) {
        int32_t *r = tmp + cnt[v];
        int64_t len = cnt[v + 1] - cnt[v];
        sort_row(r, len);
        int64_t u = 0;
        for (int64_t j = 0; j < len; j++)
            if (j == 0 || r[j] != r[j - 1]) r[u++] = r[j];
        ulen[v] = u;
    }
    int64_t m = 0;
    for (int32_t v = 0; v < n; v++) m += ulen[v];
    if (m > INT32_MAX) { free(cnt); free(tmp); free(ulen); return -7; }
    int rc = alloc_graph(out, n, m);
    if (rc) { free(cnt); free(tmp); free(ulen); return rc; }
    int64_t e = 0;
    for (int32_t v = 0; v < n; v++) {
        out->xadj[v] = (int32_t)e;
        e += ulen[v];
    }
    out->xadj[n] = (int32_t)e;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t v = 0; v < n; v++)
        memcpy(out->adjncy + out->xadj[v], tmp + cnt[v], sizeof(int32_t) * (size_t)ulen[v]);
    free(cnt); free(tmp); free(ulen);
    return 0;
}

static inline double u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

int hp_gen_rmat(int32_t scale, int32_t edgefactor, double a, double b, double c,
                uint64_t seed, int32_t wmin, int32_t wmax, int32_t nvtxs_limit,
                hp_graph *out)
{
    if (scale <= 0 || scale > 30 || edgefactor <= 0 || !out) return -1;
    int64_t nfull = (int64_t)1 << scale;
    int32_t n = nvtxs_limit > 0 ? nvtxs_limit : (int32_t)nfull;
    if (nvtxs_limit > nfull) return -1;
    int64_t ngen = (int64_t)edgefactor * (nvtxs_limit > 0 ? nvtxs_limit : nfull);
    int32_t *eu = (int32_t *)malloc(sizeof(int32_t) * (size_t)ngen);
    int32_t *ev = (int32_t *)malloc(sizeof(int32_t) * (size_t)ngen);
    if (!eu || !ev) { free(eu); free(ev); return -3; }
    const double ab = a + b, abc = a + b + c;
    const uint64_t key = hp_gen_mix64(seed ^ 0x726d6174ULL);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < ngen; e++) {
        int64_t u = 0, v = 0;
        uint64_t h = hp_gen_mix64(key ^ (uint64_t)e);
        for (int32_t l = 0; l < scale; l++) {
            h = hp_gen_mix64(h + (uint64_t)l);
            double r = u01(h);
            int qu = 0, qv = 0;
            if (r < a) { qu = 0; qv = 0; }
            else if (r < ab) { qu = 0; qv = 1; }
            else if (r < abc) { qu = 1; qv = 0; }
            else { qu = 1; qv = 1; }
            u = (u << 1) | qu;
            v = (v << 1) | qv;
        }
        if (u == v || u >= n || v >= n) { eu[e] = -1; ev[e] = -1; }
        else { eu[e] = (int32_t)u; ev[e] = (int32_t)v; }
    }
    /* keep valid pairs, both directions */
    int64_t nv = 0;
    for (int64_t e = 0; e < ngen; e++) nv += (eu[e] >= 0);
    int32_t *src = (int32_t *)malloc(sizeof(int32_t) * (size_t)(2 * nv + 1));
    int32_t *dst = (int32_t *)malloc(sizeof(int32_t) * (size_t)(2 * nv + 1));
    if (!src || !dst) { free(eu); free(ev); free(src); free(dst); return -3; }
    int64_t p = 0;
    for (int64_t e = 0; e < ngen; e++) {
        if (eu[e] < 0) continue;
        src[p] = eu[e]; dst[p] = ev[e]; p++;
        src[p] = ev[e]; dst[p] = eu[e]; p++;
    }
    free(eu); free(ev);
    int rc = csr_from_pairs(n, p, src, dst, out);
    free(src); free(dst);
    if (rc) return rc;
    fill_weights(out, seed, wmin, wmax);
    return 0;
}

int hp_gen_rgg(int32_t n, double radius, uint64_t seed, hp_graph *out)
{
    if (n <= 0 || !(radius > 0.0) || !out) return -1;
    double *px = (double *)malloc(sizeof(double) * (size_t)n);
    double *py = (double *)malloc(sizeof(double) * (size_t)n);
    if (!px || !py) { free(px); free(py); return -3; }
    const uint64_t key = hp_gen_mix64(seed ^ 0x72676721ULL);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; i++) {
        px[i] = u01(hp_gen_mix64(key ^ (2 * (uint64_t)i)));
        py[i] = u01(hp_gen_mix64(key ^ (2 * (uint64_t)i + 1)));
    }
    int64_t g = (int64_t)floor(1.0 / radius);
    if (g < 1) g = 1;
    if (g > 65536) g = 65536;
    int64_t ncell = g * g;
    int64_t *cstart = (int64_t *)calloc((size_t)ncell + 1, sizeof(int64_t));
    int32_t *cell_of = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    int32_t *bucket = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    if (!cstart || !cell_of || !bucket) {
        free(px); free(py); free(cstart); free(cell_of); free(bucket); return -3;
    }
    for (int32_t i = 0; i < n; i++) {
        int64_t cx = (int64_t)(px[i] * g), cy = (int64_t)(py[i] * g);
        if (cx >= g) cx = g - 1;
        if (cy >= g) cy = g - 1;
        cell_of[i] = (int32_t)(cy * g + cx);
        cstart[cell_of[i] + 1]++;
    }
    for (int64_t c = 0; c < ncell; c++) cstart[c + 1] += cstart[c];
    {
        int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)ncell);
        if (!fill) { free(px); free(py); free(cstart); free(cell_of); free(bucket); return -3; }
        memcpy(fill, cstart, sizeof(int64_t) * (size_t)ncell);
        for (int32_t i = 0; i < n; i++) bucket[fill[cell_of[i]]++] = i; /* ascending ids */
        free(fill);
    }
    const double r2 = radius * radius;
    int64_t *deg = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    if (!deg) { free(px); free(py); free(cstart); free(cell_of); free(bucket); return -3; }
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1) {
            int64_t m = 0;
            for (int32_t i = 0; i < n; i++) m += deg[i];
            if (m > INT32_MAX) {
                free(px); free(py); free(cstart); free(cell_of); free(bucket); free(deg); return -7;
            }
            int rc = alloc_graph(out, n, m);
            if (rc) { free(px); free(py); free(cstart); free(cell_of); free(bucket); free(deg); return rc; }
            int64_t e = 0;
            for (int32_t i = 0; i < n; i++) { out->xadj[i] = (int32_t)e; e += deg[i]; }
            out->xadj[n] = (int32_t)e;
        }
#pragma omp parallel for schedule(dynamic, 4096)
        for (int32_t i = 0; i < n; i++) {
            int64_t cx = cell_of[i] % g, cy = cell_of[i] / g;
            int64_t cnt = 0;
            int64_t base = pass ? out->xadj[i] : 0;
            for (int64_t dy = -1; dy <= 1; dy++) {
                int64_t yy = cy + dy;
                if (yy < 0 || yy >= g) continue;
                for (int64_t dx = -1; dx <= 1; dx++) {
                    int64_t xx = cx + dx;
                    if (xx < 0 || xx >= g) continue;
                    int64_t c = yy * g + xx;
                    for (int64_t q = cstart[c]; q < cstart[c + 1]; q++) {
                        int32_t j = bucket[q];
                        if (j == i) continue;
                        double ddx = px[i] - px[j], ddy = py[i] - py[j];
                        double d2 = ddx * ddx + ddy * ddy;
                        if (d2 < r2) {
                            if (pass) {
                                double d = sqrt(d2);
                                out->adjncy[base + cnt] = j;
                                out->adjwgt[base + cnt] = (int32_t)(1000.0 * (1.0 - d / radius)) + 1;
                            }
                            cnt++;
                        }
                    }
                }
            }
            if (!pass) deg[i] = cnt;
        }
    }
    /* sort each row by neighbour id, carrying weights */
#pragma omp parallel for schedule(dynamic, 4096)
    for (int32_t i = 0; i < n; i++) {
        int32_t *r = out->adjncy + out->xadj[i];
        int32_t *w = out->adjwgt + out->xadj[i];
        int64_t len = out->xadj[i + 1] - out->xadj[i];
        for (int64_t s = 1; s < len; s++) {
            int32_t t = r[s], tw = w[s];
            int64_t j = s - 1;
            while (j >= 0 && r[j] > t) { r[j + 1] = r[j]; w[j + 1] = w[j]; j--; }
            r[j + 1] = t; w[j + 1] = tw;
        }
    }
    free(px); free(py); free(cstart); free(cell_of); free(bucket); free(deg);
    return 0;
}
