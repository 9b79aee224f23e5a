/*
 * hp_io.c — METIS .graph reader and .part writer (include/hp_io.h).
 */
#define _GNU_SOURCE
#include "hp_io.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

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
