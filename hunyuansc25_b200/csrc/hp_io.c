/*
 * hp_io.c — METIS .graph reader and .part writer, MatrixMarket reader (include/hp_io.h).
 */
#define _GNU_SOURCE
#include "hp_io.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

static int fail(char *err, int errlen, const char *msg, long a, long b)
{
    if (err && errlen > 0) snprintf(err, (size_t)errlen, msg, a, b);
    return -2;
}

static ssize_t next_line(char **line, size_t *cap, FILE *f)
{
    ssize_t r;
    do {
        r = getline(line, cap, f);
    } while (r != -1 && (*line)[0] == '%');
    return r;
}

int hp_read_metis(const char *path, hp_graph *out, char *err, int errlen)
{
    memset(out, 0, sizeof(*out));
    FILE *f = fopen(path, "r");
    if (!f) {
        if (err && errlen > 0) snprintf(err, (size_t)errlen, "cannot open %s", path);
        return -1;
    }
    char *line = NULL;
    size_t cap = 0;
    int rc = 0;
    long n = 0, m = 0, fmt = 0;
    if (next_line(&line, &cap, f) == -1) { rc = fail(err, errlen, "empty file%.0ld%.0ld", 0, 0); goto done; }
    if (sscanf(line, "%ld %ld %ld", &n, &m, &fmt) < 2) {
        rc = fail(err, errlen, "header must give the vertex and edge counts%.0ld%.0ld", 0, 0);
        goto done;
    }
    if (n <= 0 || m < 0 || n > INT32_MAX - 1 || 2 * m > INT32_MAX || fmt < 0 || fmt > 111) {
        rc = fail(err, errlen, "bad header: nvtxs=%ld nedges=%ld", n, m);
        goto done;
    }
    const int readvs = (int)(fmt / 100) % 10 == 1, readvw = (int)(fmt / 10) % 10 == 1, readew = (int)fmt % 10 == 1;
    const long nd = 2 * m;
    out->nvtxs = (int32_t)n;
    out->nedges = nd;
    out->xadj = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
    out->adjncy = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nd > 0 ? nd : 1));
    out->adjwgt = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nd > 0 ? nd : 1));
    out->vwgt = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    if (!out->xadj || !out->adjncy || !out->adjwgt || !out->vwgt) { rc = -3; goto done; }
    long k = 0;
    out->xadj[0] = 0;
    for (long i = 0; i < n; i++) {
        if (next_line(&line, &cap, f) == -1) {
            rc = fail(err, errlen, "premature end of file at vertex %ld%.0ld", i + 1, 0);
            goto done;
        }
        char *cur = line, *nx = NULL;
        if (readvs) {
            strtol(cur, &nx, 10);
            if (nx == cur) { rc = fail(err, errlen, "vertex %ld: missing size%.0ld", i + 1, 0); goto done; }
            cur = nx;
        }
        out->vwgt[i] = 1;
        if (readvw) {
            long w = strtol(cur, &nx, 10);
            if (nx == cur) { rc = fail(err, errlen, "vertex %ld: missing weight%.0ld", i + 1, 0); goto done; }
            if (w < 0) { rc = fail(err, errlen, "vertex %ld: negative weight %ld", i + 1, w); goto done; }
            out->vwgt[i] = (int32_t)w;
            cur = nx;
        }
        for (;;) {
            long e = strtol(cur, &nx, 10);
            if (nx == cur) break;
            cur = nx;
            if (e < 1 || e > n) { rc = fail(err, errlen, "vertex %ld: neighbour %ld out of range", i + 1, e); goto done; }
            long w = 1;
            if (readew) {
                w = strtol(cur, &nx, 10);
                if (nx == cur) { rc = fail(err, errlen, "vertex %ld: missing edge weight%.0ld", i + 1, 0); goto done; }
                if (w <= 0) { rc = fail(err, errlen, "vertex %ld: edge weight %ld must be positive", i + 1, w); goto done; }
                cur = nx;
            }
            if (k == nd) { rc = fail(err, errlen, "more edges than the %ld in the header%.0ld", m, 0); goto done; }
            out->adjncy[k] = (int32_t)(e - 1);
            out->adjwgt[k] = (int32_t)w;
            k++;
        }
        out->xadj[i + 1] = (int32_t)k;
    }
    if (k != nd) rc = fail(err, errlen, "header gives %ld edges, file has %ld", m, k / 2);
done:
    free(line);
    fclose(f);
    if (rc) hp_graph_free(out);
    return rc;
}

int hp_write_partition(const char *fname, const int32_t *part, int32_t n, int32_t nparts)
{
    char path[4096];
    snprintf(path, sizeof(path), "%s.part.%d", fname, nparts);
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    for (int32_t i = 0; i < n; i++) fprintf(f, "%d\n", part[i]);
    fclose(f);
    return 0;
}

int hp_write_metis(const char *path, const hp_graph *g)
{
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    fprintf(f, "%d %lld 011\n", g->nvtxs, (long long)(g->nedges / 2));
    for (int32_t v = 0; v < g->nvtxs; v++) {
        fprintf(f, "%d", g->vwgt ? g->vwgt[v] : 1);
        for (int32_t j = g->xadj[v]; j < g->xadj[v + 1]; j++)
            fprintf(f, " %d %d", g->adjncy[j] + 1, g->adjwgt ? g->adjwgt[j] : 1);
        fputc('\n', f);
    }
    fclose(f);
    return 0;
}

/* ---- MatrixMarket -------------------------------------------------------------- */
static int cmp_u64(const void *a, const void *b)
{
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : (x > y);
}

int hp_read_mtx(const char *path, hp_graph *out, char *err, int errlen)
{
    memset(out, 0, sizeof(*out));
    FILE *f = fopen(path, "r");
    if (!f) {
        if (err && errlen > 0) snprintf(err, (size_t)errlen, "cannot open %s", path);
        return -1;
    }
    char *line = NULL;
    size_t cap = 0;
    int rc = 0;
    uint64_t *pairs = NULL;
    if (getline(&line, &cap, f) == -1 || strncasecmp(line, "%%MatrixMarket", 14) != 0) {
        rc = fail(err, errlen, "missing %%%%MatrixMarket banner%.0ld%.0ld", 0, 0);
        goto done;
    }
    char obj[64] = {0}, fmtw[64] = {0}, field[64] = {0}, sym[64] = {0};
    if (sscanf(line + 14, "%63s %63s %63s %63s", obj, fmtw, field, sym) != 4 || strcasecmp(obj, "matrix") != 0 ||
        strcasecmp(fmtw, "coordinate") != 0) {
        rc = fail(err, errlen, "only 'matrix coordinate' files are supported%.0ld%.0ld", 0, 0);
        goto done;
    }
    if (strcasecmp(field, "pattern") && strcasecmp(field, "integer") && strcasecmp(field, "real") &&
        strcasecmp(field, "complex")) {
        rc = fail(err, errlen, "unknown field type%.0ld%.0ld", 0, 0);
        goto done;
    }
    if (strcasecmp(sym, "general") && strcasecmp(sym, "symmetric") && strcasecmp(sym, "skew-symmetric") &&
        strcasecmp(sym, "hermitian")) {
        rc = fail(err, errlen, "unknown symmetry%.0ld%.0ld", 0, 0);
        goto done;
    }
    long M = 0, N = 0, nnz = 0;
    if (next_line(&line, &cap, f) == -1 || sscanf(line, "%ld %ld %ld", &M, &N, &nnz) != 3) {
        rc = fail(err, errlen, "missing size line%.0ld%.0ld", 0, 0);
        goto done;
    }
    if (M != N || M <= 0 || M > INT32_MAX - 1 || nnz < 0 || nnz > INT32_MAX / 2) {
        rc = fail(err, errlen, "need a square matrix of supported size (rows %ld, cols %ld)", M, N);
        goto done;
    }
    /* every off-diagonal entry gives both directions */
    pairs = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(2 * nnz > 0 ? 2 * nnz : 1));
    if (!pairs) { rc = -3; goto done; }
    long np = 0;
    for (long e = 0; e < nnz; e++) {
        if (next_line(&line, &cap, f) == -1) {
            rc = fail(err, errlen, "premature end of file at entry %ld of %ld", e + 1, nnz);
            goto done;
        }
        long i = 0, j = 0;
        if (sscanf(line, "%ld %ld", &i, &j) != 2 || i < 1 || j < 1 || i > M || j > N) {
            rc = fail(err, errlen, "bad entry %ld%.0ld", e + 1, 0);
            goto done;
        }
        if (i == j) continue;
        const uint64_t a = (uint64_t)(i - 1), b = (uint64_t)(j - 1);
        pairs[np++] = a << 32 | b;
        pairs[np++] = b << 32 | a;
    }
    qsort(pairs, (size_t)np, sizeof(uint64_t), cmp_u64);
    long m = 0;
    for (long t = 0; t < np; t++)
        if (t == 0 || pairs[t] != pairs[t - 1]) pairs[m++] = pairs[t];
    out->nvtxs = (int32_t)M;
    out->nedges = m;
    out->xadj = (int32_t *)calloc((size_t)M + 1, sizeof(int32_t));
    out->adjncy = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    out->adjwgt = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    out->vwgt = (int32_t *)malloc(sizeof(int32_t) * (size_t)M);
    if (!out->xadj || !out->adjncy || !out->adjwgt || !out->vwgt) { rc = -3; goto done; }
    for (long t = 0; t < m; t++) {
        out->xadj[(pairs[t] >> 32) + 1]++;
        out->adjncy[t] = (int32_t)(pairs[t] & 0xffffffffu);
        out->adjwgt[t] = 1;
    }
    for (long i = 0; i < M; i++) {
        out->xadj[i + 1] += out->xadj[i];
        out->vwgt[i] = 1;
    }
done:
    free(pairs);
    free(line);
    fclose(f);
    if (rc != 0) hp_graph_free(out);
    return rc;
}
