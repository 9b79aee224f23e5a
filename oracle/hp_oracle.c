/*
 * hp_oracle.c — CPU oracle of the multilevel k-way partition path.
 *
 * TEST INFRASTRUCTURE ONLY (see hp_oracle.h): the checker for the CUDA path,
 * never linked into the product.
 *
 * Each function restates one step of the reference's partition path with the
 * tie-breaks made explicit, so that the CUDA kernels and this file compute the
 * same integers:
 *   matching       hunyuangraph_CPU_match.h:285-380 (eligibility, maxvwgt cap,
 *                  cmap numbering), hunyuangraph_GPU_match.h:800-861 (mutual
 *                  proposal rounds), :1374-1716 (leaf/relative/isolate/forced
 *                  fallbacks gated at 75 % matched, :2577)
 *   contraction    hunyuangraph_CPU_contraction.h:9-100 (sum duplicates, drop
 *                  self loop) with rows sorted by coarse id
 *                  (hunyuangraph_GPU_contraction.h:886)
 *   coarsening     hunyuangraph_GPU_coarsen.h:163-253 (maxvwgt, stop rule)
 *   bisection      hunyuangraph_CPU_initialpartition.h:36-145 (BFS growth),
 *                  hunyuangraph_CPU_2wayrefine.h:77-245 (2-way FM),
 *                  hunyuangraph_GPU_initialpartition.h:3913-4386 (multi-start,
 *                  best cut, split and recurse)
 *   refinement     hunyuangraph_GPU_krefine.h:1995-2221 (LP + afterburner +
 *                  lock), 2477-2513 (gain bucket), 3136-3563 (weak rebalance),
 *                  2515-3135 (strong rebalance), 3933-4155 (moves, cut),
 *                  4434-4882 (pass loop, best partition)
 *   projection     hunyuangraph_GPU_uncoarsen.h:196-223
 *   cut            hunyuangraph_graph.h:144-155 (int64 here)
 */
#include "hp_oracle.h"

#define ORA_MAX_REFINE_PASSES (1 << 14)

#include <limits.h>
#include <stdio.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
static int g_threads = 1;

void ora_set_threads(int nthreads)
{
    g_threads = nthreads > 0 ? nthreads : 1;
#ifdef _OPENMP
    omp_set_num_threads(g_threads);
#endif
}

int ora_get_threads(void) { return g_threads; }

void ora_free(void *p) { free(p); }

static void *xmalloc(size_t bytes)
{
    void *p = malloc(bytes ? bytes : 1);
    return p;
}

/* splitmix64 finaliser (Vigna); the matching tie-break key. */
static inline uint64_t mix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static inline uint64_t level_key(uint64_t seed, int32_t level)
{
    return mix64(seed ^ (0x6d61746368ULL + (uint64_t)level * 0x100000001b3ULL));
}

static inline uint32_t edge_tie(uint64_t lkey, int32_t a, int32_t b)
{
    uint32_t lo = (uint32_t)(a < b ? a : b), hi = (uint32_t)(a < b ? b : a);
    return (uint32_t)(mix64(lkey ^ (((uint64_t)lo << 32) | hi)) >> 32);
}

/* Candidate order for matching: heavier edge first, then lower tie key, then
 * lower neighbour id. */
static inline int better(int32_t w1, uint32_t h1, int32_t u1, int32_t w2, uint32_t h2, int32_t u2)
{
    if (w1 != w2) return w1 > w2;
    if (h1 != h2) return h1 < h2;
    return u1 < u2;
}

/* ------------------------------------------------------------------------- */
int64_t ora_edgecut(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                    const int32_t *adjwgt, const int32_t *where)
{
    int64_t cut = 0;
#pragma omp parallel for reduction(+ : cut) schedule(dynamic, 2048)
    for (int32_t v = 0; v < n; v++)
        for (int32_t j = xadj[v]; j < xadj[v + 1]; j++)
            if (where[adjncy[j]] != where[v]) cut += adjwgt ? adjwgt[j] : 1;
    return cut / 2;
}

/* ------------------------------------------------------------------------- */
/* Matching.                                                                  */

static int32_t count_matched(int32_t n, const int32_t *match)
{
    int32_t c = 0;
#pragma omp parallel for reduction(+ : c)
    for (int32_t v = 0; v < n; v++) c += (match[v] != -1);
    return c;
}

/* Pair consecutive entries of list[0..len) whose weight sum fits. */
static void pair_list(const int32_t *list, int32_t len, const int32_t *vwgt, int64_t maxvwgt,
                      int32_t *match)
{
    for (int32_t i = 0; i + 1 < len; i += 2) {
        int32_t a = list[i], b = list[i + 1];
        if ((int64_t)vwgt[a] + vwgt[b] <= maxvwgt) { match[a] = b; match[b] = a; }
    }
}

int32_t ora_match(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                  const int32_t *vwgt, const int32_t *adjwgt, int32_t level,
                  uint64_t seed, int64_t maxvwgt, int32_t rounds,
                  int32_t *match, int32_t *cmap)
{
    const uint64_t lkey = level_key(seed, level);
    int32_t *pref = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    for (int32_t v = 0; v < n; v++) match[v] = -1;

    /* Handshake rounds: every unmatched vertex names its best eligible
     * neighbour; mutual names become pairs. */
    for (int32_t r = 0; r < rounds; r++) {
        int32_t made = 0;
#pragma omp parallel for schedule(dynamic, 2048)
        for (int32_t v = 0; v < n; v++) {
            pref[v] = -1;
            if (match[v] != -1) continue;
            int32_t bu = -1, bw = 0;
            uint32_t bh = 0;
            for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) {
                int32_t u = adjncy[j];
                if (u == v || match[u] != -1) continue;
                if ((int64_t)vwgt[v] + vwgt[u] > maxvwgt) continue;
                int32_t w = adjwgt[j];
                uint32_t h = edge_tie(lkey, v, u);
                if (bu < 0 || better(w, h, u, bw, bh, bu)) { bu = u; bw = w; bh = h; }
            }
            pref[v] = bu;
        }
#pragma omp parallel for reduction(+ : made)
        for (int32_t v = 0; v < n; v++) {
            int32_t u = pref[v];
            if (u >= 0 && pref[u] == v) { match[v] = u; made++; }
        }
        if (made == 0) break; /* state unchanged: later rounds would repeat */
    }

    /* Fallbacks, each gated at 75 % matched. */
    if (4 * (int64_t)count_matched(n, match) < 3 * (int64_t)n) {
        /* two-hop: unmatched vertices that share their heaviest neighbour (the
         * hub) are paired in ascending id -- the hub's row order, rows being
         * sorted (hunyuangraph_GPU_match.h:1374-1716 pairs its leaf/relative
         * classes through a shared neighbour as well) */
        int32_t *hub = pref;
#pragma omp parallel for schedule(dynamic, 2048)
        for (int32_t v = 0; v < n; v++) {
            hub[v] = -1;
            if (match[v] != -1) continue;
            int32_t bu = -1, bw = 0;
            uint32_t bh = 0;
            for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) {
                int32_t u = adjncy[j];
                if (u == v) continue;
                int32_t w = adjwgt[j];
                uint32_t h = edge_tie(lkey, v, u);
                if (bu < 0 || better(w, h, u, bw, bh, bu)) { bu = u; bw = w; bh = h; }
            }
            hub[v] = bu;
        }
        /* clients bucketed by hub in ascending id (a counting sort), then paired
         * per hub: (c0,c1), (c2,c3), ... */
        int32_t *start = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
        int32_t *ord = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
        for (int32_t c = 0; c < n; c++)
            if (match[c] == -1 && hub[c] >= 0) start[hub[c] + 1]++;
        for (int32_t h = 0; h < n; h++) start[h + 1] += start[h];
        {
            int32_t *fill = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
            for (int32_t h = 0; h < n; h++) fill[h] = start[h];
            for (int32_t c = 0; c < n; c++)
                if (match[c] == -1 && hub[c] >= 0) ord[fill[hub[c]]++] = c;
            free(fill);
        }
        for (int32_t h = 0; h < n; h++) pair_list(ord + start[h], start[h + 1] - start[h], vwgt, maxvwgt, match);
        free(start);
        free(ord);
    }
    if (4 * (int64_t)count_matched(n, match) < 3 * (int64_t)n) {
        /* isolated vertices, paired in id order */
        int32_t len = 0;
        for (int32_t v = 0; v < n; v++)
            if (match[v] == -1 && xadj[v] == xadj[v + 1]) pref[len++] = v;
        pair_list(pref, len, vwgt, maxvwgt, match);
    }
    if (4 * (int64_t)count_matched(n, match) < 3 * (int64_t)n) {
        /* forced: remaining unmatched vertices paired in id order */
        int32_t len = 0;
        for (int32_t v = 0; v < n; v++)
            if (match[v] == -1) pref[len++] = v;
        pair_list(pref, len, vwgt, maxvwgt, match);
    }

    /* cmap: coarse ids in increasing order of the smaller endpoint */
    int32_t cn = 0;
    for (int32_t v = 0; v < n; v++) {
        if (match[v] == -1) match[v] = v;
        if (v <= match[v]) cmap[v] = cn++;
    }
    for (int32_t v = 0; v < n; v++)
        if (v > match[v]) cmap[v] = cmap[match[v]];
    free(pref);
    return cn;
}

/* ------------------------------------------------------------------------- */
/* Contraction.                                                               */

/* Coarse weights accumulate in int64 (they are stored as int32 once merged;
 * ora_weight_range_ok below guarantees that every merged weight fits). */
typedef struct { int32_t k; int64_t w; } kw_t;

static int cmp_kw(const void *a, const void *b)
{
    int32_t x = ((const kw_t *)a)->k, y = ((const kw_t *)b)->k;
    return (x > y) - (x < y);
}

static void sort_kw(kw_t *r, int64_t len)
{
    if (len < 32) {
        for (int64_t i = 1; i < len; i++) {
            kw_t t = r[i];
            int64_t j = i - 1;
            while (j >= 0 && r[j].k > t.k) { r[j + 1] = r[j]; j--; }
            r[j + 1] = t;
        }
    } else {
        qsort(r, (size_t)len, sizeof(kw_t), cmp_kw);
    }
}

/* Weight range (the library's rule, checked when the input's total edge
 * weight reaches 2^31): every coarse edge weight and every connectivity of a
 * vertex is at most the vertex's weighted degree, so the int32 weights cannot
 * wrap while every vertex of every level has a weighted degree below 2^31.
 * Returns 1 when every row of the graph sums below 2^31. */
int ora_weight_range_ok(int32_t n, const int32_t *xadj, const int32_t *adjwgt)
{
    int ok = 1;
#pragma omp parallel for schedule(dynamic, 4096) reduction(&& : ok)
    for (int32_t v = 0; v < n; v++) {
        int64_t s = 0;
        for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) s += adjwgt[j];
        ok = ok && s < (int64_t)INT32_MAX;
    }
    return ok;
}

int64_t ora_contract(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                     const int32_t *vwgt, const int32_t *adjwgt,
                     const int32_t *match, const int32_t *cmap, int32_t cn,
                     int32_t **cxadj_o, int32_t **cadjncy_o, int32_t **cadjwgt_o,
                     int32_t **cvwgt_o)
{
    int32_t *leader = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)cn);
    for (int32_t v = 0; v < n; v++)
        if (v <= match[v]) leader[cmap[v]] = v;
    int64_t *toff = (int64_t *)xmalloc(sizeof(int64_t) * ((size_t)cn + 1));
    toff[0] = 0;
    for (int32_t c = 0; c < cn; c++) {
        int32_t v = leader[c], u = match[v];
        int64_t len = xadj[v + 1] - xadj[v];
        if (u != v) len += xadj[u + 1] - xadj[u];
        toff[c + 1] = toff[c] + len;
    }
    kw_t *tmp = (kw_t *)xmalloc(sizeof(kw_t) * (size_t)toff[cn]);
    int32_t *ucnt = (int32_t *)xmalloc(sizeof(int32_t) * ((size_t)cn + 1));
    int32_t *cvwgt = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)cn);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t c = 0; c < cn; c++) {
        int32_t v = leader[c], u = match[v];
        kw_t *r = tmp + toff[c];
        int64_t len = 0;
        for (int pass = 0; pass < (u != v ? 2 : 1); pass++) {
            int32_t x = pass ? u : v;
            for (int32_t j = xadj[x]; j < xadj[x + 1]; j++) {
                int32_t k = cmap[adjncy[j]];
                if (k == c) continue; /* self loop of the coarse vertex */
                r[len].k = k;
                r[len].w = adjwgt[j];
                len++;
            }
        }
        sort_kw(r, len);
        int64_t q = 0;
        for (int64_t j = 0; j < len; j++) {
            if (q > 0 && r[q - 1].k == r[j].k) r[q - 1].w += r[j].w;
            else r[q++] = r[j];
        }
        ucnt[c] = (int32_t)q;
        cvwgt[c] = vwgt[v] + (u != v ? vwgt[u] : 0);
    }
    int32_t *cxadj = (int32_t *)xmalloc(sizeof(int32_t) * ((size_t)cn + 1));
    int64_t m = 0;
    for (int32_t c = 0; c < cn; c++) { cxadj[c] = (int32_t)m; m += ucnt[c]; }
    cxadj[cn] = (int32_t)m;
    int32_t *cadj = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)m);
    int32_t *cwgt = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)m);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t c = 0; c < cn; c++) {
        const kw_t *r = tmp + toff[c];
        for (int32_t j = 0; j < ucnt[c]; j++) {
            cadj[cxadj[c] + j] = r[j].k;
            /* saturated: a merged weight beyond int32 makes its row fail the
             * weight-range check, as the row's sum is at least as large */
            cwgt[cxadj[c] + j] = r[j].w > INT32_MAX ? INT32_MAX : (int32_t)r[j].w;
        }
    }
    free(leader); free(toff); free(tmp); free(ucnt);
    *cxadj_o = cxadj; *cadjncy_o = cadj; *cadjwgt_o = cwgt; *cvwgt_o = cvwgt;
    return m;
}

/* ------------------------------------------------------------------------- */
/* Part weight targets.                                                       */

void ora_part_targets(int64_t tvwgt, int32_t nparts, const float *tpwgts, float ubfactor,
                      int64_t *opt, int64_t *maxp)
{
    double sum = 0.0;
    if (tpwgts)
        for (int32_t p = 0; p < nparts; p++) sum += (double)tpwgts[p];
    for (int32_t p = 0; p < nparts; p++) {
        double frac = tpwgts ? (double)tpwgts[p] / sum : 1.0 / (double)nparts;
        double t = (double)tvwgt * frac;
        double u = (double)ubfactor * t;
        opt[p] = (int64_t)floor(t);
        maxp[p] = (int64_t)floor(u);
        if (maxp[p] < opt[p]) maxp[p] = opt[p];
    }
}

/* Bisection imbalance ub^(1/ln k) (hunyuangraph_GPU_initialpartition.h:4433),
 * as 16.16 fixed point. */
int64_t ora_bisect_ub_fx(float ubfactor, int32_t nparts)
{
    double ub2 = nparts > 1 ? pow((double)ubfactor, 1.0 / log((double)nparts)) : (double)ubfactor;
    return (int64_t)floor(ub2 * 65536.0 + 0.5);
}

/* ------------------------------------------------------------------------- */
/* 2-way FM with a max-heap ordered by (gain desc, vertex asc).               */

typedef struct {
    int32_t *heap;   /* vertices */
    int32_t *pos;    /* pos[v] = index in heap or -1 (shared by both queues) */
    int32_t *key;    /* key[v] (shared) */
    int32_t len;
} pq_t;

static inline int pq_above(const pq_t *q, int32_t a, int32_t b)
{
    int32_t ka = q->key[a], kb = q->key[b];
    return ka > kb || (ka == kb && a < b);
}

static void pq_up(pq_t *q, int32_t i)
{
    int32_t v = q->heap[i];
    while (i > 0) {
        int32_t p = (i - 1) >> 1;
        if (!pq_above(q, v, q->heap[p])) break;
        q->heap[i] = q->heap[p];
        q->pos[q->heap[i]] = i;
        i = p;
    }
    q->heap[i] = v;
    q->pos[v] = i;
}

static void pq_down(pq_t *q, int32_t i)
{
    int32_t v = q->heap[i];
    for (;;) {
        int32_t l = 2 * i + 1, r = l + 1, b = i;
        int32_t bv = v;
        if (l < q->len && pq_above(q, q->heap[l], bv)) { b = l; bv = q->heap[l]; }
        if (r < q->len && pq_above(q, q->heap[r], bv)) { b = r; bv = q->heap[r]; }
        if (b == i) break;
        q->heap[i] = bv;
        q->pos[bv] = i;
        i = b;
    }
    q->heap[i] = v;
    q->pos[v] = i;
}

static void pq_insert(pq_t *q, int32_t v, int32_t k)
{
    q->key[v] = k;
    q->heap[q->len] = v;
    q->pos[v] = q->len;
    q->len++;
    pq_up(q, q->len - 1);
}

static void pq_delete(pq_t *q, int32_t v)
{
    int32_t i = q->pos[v];
    q->pos[v] = -1;
    q->len--;
    if (i == q->len) return;
    int32_t last = q->heap[q->len];
    q->heap[i] = last;
    q->pos[last] = i;
    pq_up(q, i);
    pq_down(q, q->pos[last]);
}

static void pq_update(pq_t *q, int32_t v, int32_t k)
{
    q->key[v] = k;
    int32_t i = q->pos[v];
    pq_up(q, i);
    pq_down(q, q->pos[v]);
}

static int32_t pq_pop(pq_t *q)
{
    if (q->len == 0) return -1;
    int32_t v = q->heap[0];
    pq_delete(q, v);
    return v;
}

static inline int64_t iabs64(int64_t x) { return x < 0 ? -x : x; }

typedef struct {
    int32_t *id, *ed, *moved, *swaps, *queue, *pos, *key, *heap0, *heap1;
    int8_t  *bnd, *vis;
} fm_ws;

/* One bisection trial: BFS growth from `start` then FM.  where[] (0/1) and
 * the trial's cut are returned.  want1 = target weight of side 1. */
static int64_t bisect_trial(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                            const int32_t *vwgt, const int32_t *adjwgt, int64_t tv,
                            int64_t want1, int64_t onemin, int64_t onemax, int32_t start,
                            int32_t fm_passes, fm_ws *ws, int32_t *where, int64_t *pw_out)
{
    int32_t *id = ws->id, *ed = ws->ed, *moved = ws->moved, *swaps = ws->swaps;
    int32_t *queue = ws->queue;
    int8_t *bnd = ws->bnd, *vis = ws->vis;
    int64_t pw[2];

    /* ---- BFS growth of side 0 (hunyuangraph_CPU_initialpartition.h:66-120) */
    for (int32_t v = 0; v < n; v++) { where[v] = 1; vis[v] = 0; }
    pw[0] = 0; pw[1] = tv;
    int32_t first = 0, last = 1, nleft = n - 1, drain = 0, next_unvis = 0;
    queue[0] = start; vis[start] = 1;
    for (;;) {
        if (first == last) {
            if (nleft == 0 || drain) break;
            while (vis[next_unvis]) next_unvis++;
            queue[0] = next_unvis; vis[next_unvis] = 1;
            first = 0; last = 1; nleft--;
        }
        int32_t i = queue[first++];
        if (pw[0] > 0 && pw[1] - vwgt[i] < onemin) { drain = 1; continue; }
        where[i] = 0;
        pw[0] += vwgt[i]; pw[1] -= vwgt[i];
        if (pw[1] <= onemax) break;
        drain = 0;
        for (int32_t j = xadj[i]; j < xadj[i + 1]; j++) {
            int32_t k = adjncy[j];
            if (!vis[k]) { queue[last++] = k; vis[k] = 1; nleft--; }
        }
    }

    /* ---- 2-way FM (hunyuangraph_CPU_2wayrefine.h:24-245) */
    int64_t cut = 0;
    for (int32_t v = 0; v < n; v++) {
        int32_t tid = 0, ted = 0;
        for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) {
            if (where[adjncy[j]] == where[v]) tid += adjwgt[j];
            else ted += adjwgt[j];
        }
        id[v] = tid; ed[v] = ted;
        bnd[v] = (ted > 0 || xadj[v] == xadj[v + 1]);
        cut += ted;
        moved[v] = -1;
        ws->pos[v] = -1;
    }
    cut /= 2;
    const int64_t tpw0 = tv - want1, tpw1 = want1;
    int64_t limit = n / 100;
    if (limit < 15) limit = 15;
    if (limit > 100) limit = 100;
    int64_t avgvwgt = (pw[0] + pw[1]) / 20;
    if (n > 0 && 2 * (pw[0] + pw[1]) / n < avgvwgt) avgvwgt = 2 * (pw[0] + pw[1]) / n;
    const int64_t origdiff = iabs64(tpw0 - pw[0]);
    pq_t q[2];
    q[0].heap = ws->heap0; q[1].heap = ws->heap1;
    q[0].pos = q[1].pos = ws->pos;
    q[0].key = q[1].key = ws->key;

    for (int32_t pass = 0; pass < fm_passes; pass++) {
        q[0].len = q[1].len = 0;
        for (int32_t v = 0; v < n; v++) ws->pos[v] = -1;
        int64_t mincutorder = -1;
        int64_t newcut = cut, mincut = cut, initcut = cut;
        int64_t mindiff = iabs64(tpw0 - pw[0]);
        for (int32_t v = 0; v < n; v++)
            if (bnd[v]) pq_insert(&q[where[v]], v, ed[v] - id[v]);
        int32_t nswaps;
        for (nswaps = 0; nswaps < n; nswaps++) {
            int from = (tpw0 - pw[0] < tpw1 - pw[1]) ? 0 : 1;
            int to = 1 - from;
            int32_t h = pq_pop(&q[from]);
            if (h < 0) break;
            newcut -= (ed[h] - id[h]);
            pw[to] += vwgt[h]; pw[from] -= vwgt[h];
            if ((newcut < mincut && iabs64(tpw0 - pw[0]) <= origdiff + avgvwgt) ||
                (newcut == mincut && iabs64(tpw0 - pw[0]) < mindiff)) {
                mincut = newcut;
                mindiff = iabs64(tpw0 - pw[0]);
                mincutorder = nswaps;
            } else if (nswaps - mincutorder > limit) {
                newcut += (ed[h] - id[h]);
                pw[from] += vwgt[h]; pw[to] -= vwgt[h];
                break;
            }
            where[h] = to;
            moved[h] = nswaps;
            swaps[nswaps] = h;
            { int32_t t = id[h]; id[h] = ed[h]; ed[h] = t; }
            if (ed[h] == 0 && xadj[h] < xadj[h + 1]) bnd[h] = 0;
            for (int32_t j = xadj[h]; j < xadj[h + 1]; j++) {
                int32_t k = adjncy[j];
                int32_t kw = (to == where[k]) ? adjwgt[j] : -adjwgt[j];
                id[k] += kw; ed[k] -= kw;
                if (bnd[k]) {
                    if (ed[k] == 0) {
                        bnd[k] = 0;
                        if (moved[k] == -1 && ws->pos[k] >= 0) pq_delete(&q[where[k]], k);
                    } else if (moved[k] == -1 && ws->pos[k] >= 0) {
                        pq_update(&q[where[k]], k, ed[k] - id[k]);
                    }
                } else if (ed[k] > 0) {
                    bnd[k] = 1;
                    if (moved[k] == -1) pq_insert(&q[where[k]], k, ed[k] - id[k]);
                }
            }
        }
        for (int32_t i = 0; i < nswaps; i++) moved[swaps[i]] = -1;
        for (nswaps--; nswaps > mincutorder; nswaps--) {
            int32_t h = swaps[nswaps];
            int to = where[h] = 1 - where[h];
            { int32_t t = id[h]; id[h] = ed[h]; ed[h] = t; }
            if (ed[h] == 0 && bnd[h] && xadj[h] < xadj[h + 1]) bnd[h] = 0;
            else if (ed[h] > 0 && !bnd[h]) bnd[h] = 1;
            pw[to] += vwgt[h]; pw[1 - to] -= vwgt[h];
            for (int32_t j = xadj[h]; j < xadj[h + 1]; j++) {
                int32_t k = adjncy[j];
                int32_t kw = (to == where[k]) ? adjwgt[j] : -adjwgt[j];
                id[k] += kw; ed[k] -= kw;
                if (bnd[k] && ed[k] == 0) bnd[k] = 0;
                if (!bnd[k] && ed[k] > 0) bnd[k] = 1;
            }
        }
        cut = mincut;
        if (mincutorder <= 0 || mincut == initcut) break;
    }
    pw_out[0] = pw[0]; pw_out[1] = pw[1];
    return cut;
}

typedef struct {
    int32_t n;
    int32_t *xadj, *adjncy, *adjwgt, *vwgt, *label;
} sub_t;

/* The two induced subgraphs of a 2-way split (hunyuangraph_splitgraph,
 * hunyuangraph_CPU_splitgraph.h:8-167): each side's vertices renumbered in id
 * order, rows in their original order with the other side's neighbours
 * dropped, vertex weights and labels carried over. */
static void split2(const sub_t *g, const int32_t *side_of, sub_t s[2])
{
    const int32_t n = g->n;
    int32_t *lid = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t cnt[2] = {0, 0};
    for (int32_t v = 0; v < n; v++) lid[v] = cnt[side_of[v]]++;
    for (int side = 0; side < 2; side++) {
        s[side].n = cnt[side];
        s[side].xadj = (int32_t *)xmalloc(sizeof(int32_t) * ((size_t)cnt[side] + 1));
        s[side].vwgt = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(cnt[side] > 0 ? cnt[side] : 1));
        s[side].label = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(cnt[side] > 0 ? cnt[side] : 1));
        int64_t m = 0;
        for (int32_t v = 0; v < n; v++) {
            if (side_of[v] != side) continue;
            for (int32_t j = g->xadj[v]; j < g->xadj[v + 1]; j++) m += (side_of[g->adjncy[j]] == side);
        }
        s[side].adjncy = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
        s[side].adjwgt = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
        int64_t e = 0;
        for (int32_t v = 0; v < n; v++) {
            if (side_of[v] != side) continue;
            int32_t lv = lid[v];
            s[side].xadj[lv] = (int32_t)e;
            s[side].vwgt[lv] = g->vwgt[v];
            s[side].label[lv] = g->label[v];
            for (int32_t j = g->xadj[v]; j < g->xadj[v + 1]; j++) {
                int32_t u = g->adjncy[j];
                if (side_of[u] != side) continue;
                s[side].adjncy[e] = lid[u];
                s[side].adjwgt[e] = g->adjwgt[j];
                e++;
            }
        }
        s[side].xadj[cnt[side]] = (int32_t)e;
    }
    free(lid);
}

static void rb(const sub_t *g, int32_t nparts, int32_t fpart, const int64_t *tw, int64_t ub2_fx,
               int32_t starts, int32_t fm_passes, int32_t *out_where)
{
    if (g->n == 0) return;
    if (nparts == 1) {
        for (int32_t v = 0; v < g->n; v++) out_where[g->label[v]] = fpart;
        return;
    }
    const int32_t n = g->n;
    const int32_t kl = nparts >> 1;
    int64_t wl = 0, wr = 0, tv = 0;
    for (int32_t p = 0; p < kl; p++) wl += tw[fpart + p];
    for (int32_t p = kl; p < nparts; p++) wr += tw[fpart + p];
    for (int32_t v = 0; v < n; v++) tv += g->vwgt[v];
    int64_t want1 = (wl + wr) > 0 ? (tv * wr) / (wl + wr) : tv / 2;
    int64_t onemax = (want1 * ub2_fx) >> 16;
    int64_t onemin = (want1 << 16) / ub2_fx;
    int32_t ntr = n <= starts ? n : starts;

    int32_t *best = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    int64_t best_viol = -1, best_cut = 0;
#pragma omp parallel
    {
        fm_ws ws;
        ws.id = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
        ws.ed = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
        ws.moved = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
        ws.swaps = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
        ws.queue = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
        ws.pos = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
        ws.key = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
        ws.heap0 = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
        ws.heap1 = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
        ws.bnd = (int8_t *)xmalloc((size_t)n);
        ws.vis = (int8_t *)xmalloc((size_t)n);
        int32_t *w = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
#pragma omp for schedule(dynamic, 1) ordered
        for (int32_t t = 0; t < ntr; t++) {
            int32_t s = (n <= starts) ? t : (int32_t)(((int64_t)t * n) / starts);
            int64_t pw[2];
            int64_t cut = bisect_trial(n, g->xadj, g->adjncy, g->vwgt, g->adjwgt, tv, want1,
                                       onemin, onemax, s, fm_passes, &ws, w, pw);
            int64_t viol = 0;
            if (pw[1] > onemax) viol += pw[1] - onemax;
            if (pw[1] < onemin) viol += onemin - pw[1];
#pragma omp ordered
            {
                if (best_viol < 0 || viol < best_viol || (viol == best_viol && cut < best_cut)) {
                    best_viol = viol; best_cut = cut;
                    memcpy(best, w, sizeof(int32_t) * (size_t)n);
                }
            }
        }
        free(ws.id); free(ws.ed); free(ws.moved); free(ws.swaps); free(ws.queue);
        free(ws.pos); free(ws.key); free(ws.heap0); free(ws.heap1); free(ws.bnd); free(ws.vis);
        free(w);
    }

    /* split into the two induced subgraphs, vertex order preserved */
    sub_t s[2];
    split2(g, best, s);
    free(best);
    rb(&s[0], kl, fpart, tw, ub2_fx, starts, fm_passes, out_where);
    rb(&s[1], nparts - kl, fpart + kl, tw, ub2_fx, starts, fm_passes, out_where);
    for (int side = 0; side < 2; side++) {
        free(s[side].xadj); free(s[side].adjncy); free(s[side].adjwgt);
        free(s[side].vwgt); free(s[side].label);
    }
}

int64_t ora_split(int32_t n, const int32_t *xadj, const int32_t *adjncy, const int32_t *vwgt,
                  const int32_t *adjwgt, const int32_t *where, int32_t side, int32_t *sn,
                  int32_t *sxadj, int32_t *sadjncy, int32_t *sadjwgt, int32_t *svwgt, int32_t *slabel)
{
    if (n < 0 || side < 0 || side > 1 || !sn) return -1;
    for (int32_t v = 0; v < n; v++)
        if (where[v] != 0 && where[v] != 1) return -1;
    int32_t *label = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int32_t v = 0; v < n; v++) label[v] = v;
    sub_t g = {n, (int32_t *)xadj, (int32_t *)adjncy, (int32_t *)adjwgt, (int32_t *)vwgt, label};
    sub_t s[2];
    split2(&g, where, s);
    const sub_t *o = &s[side];
    const int64_t m = o->xadj[o->n];
    *sn = o->n;
    memcpy(sxadj, o->xadj, sizeof(int32_t) * ((size_t)o->n + 1));
    memcpy(sadjncy, o->adjncy, sizeof(int32_t) * (size_t)m);
    memcpy(sadjwgt, o->adjwgt, sizeof(int32_t) * (size_t)m);
    memcpy(svwgt, o->vwgt, sizeof(int32_t) * (size_t)o->n);
    memcpy(slabel, o->label, sizeof(int32_t) * (size_t)o->n);
    for (int k = 0; k < 2; k++) {
        free(s[k].xadj); free(s[k].adjncy); free(s[k].adjwgt); free(s[k].vwgt); free(s[k].label);
    }
    free(label);
    return m;
}

int ora_initpart(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                 const int32_t *vwgt, const int32_t *adjwgt, int32_t nparts,
                 const int64_t *tw, int64_t ub2_fx, int32_t starts, int32_t fm_passes,
                 int32_t *where)
{
    sub_t g;
    g.n = n;
    g.xadj = (int32_t *)xadj; g.adjncy = (int32_t *)adjncy;
    g.adjwgt = (int32_t *)adjwgt; g.vwgt = (int32_t *)vwgt;
    g.label = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    for (int32_t v = 0; v < n; v++) g.label[v] = v;
    rb(&g, nparts, 0, tw, ub2_fx, starts, fm_passes, where);
    free(g.label);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Refinement.                                                                */

int32_t ora_gain_bucket(int32_t gain, int32_t vwgt)
{
    /* float semantics of gain_bucket (hunyuangraph_GPU_krefine.h:2477-2513);
     * the reference lets the upper clamp reach max_buckets (50), which indexes
     * the next part's buckets, so the clamp here is to 49. */
    float g = (float)gain / (float)(vwgt > 0 ? vwgt : 1);
    int32_t t;
    if (g > 0.0f) return 0;
    if (g == 0.0f) return 1;
    t = 25;
    g = fabsf(g);
    if (g < 1.0f) {
        while (g < 1.0f) { g *= 1.5f; t--; }
        if (t < 2) t = 2;
    } else {
        while (g > 1.0f) { g /= 1.5f; t++; }
        if (t > 49) t = 49;
    }
    return t;
}

/* Connectivity of v to every adjacent part, accumulated in conn[] (dense k)
 * with the touched parts listed in parts[]; returns the number of parts. */
static inline int32_t gather_conn(int32_t v, const int32_t *xadj, const int32_t *adjncy,
                                  const int32_t *adjwgt, const int32_t *where, int64_t *conn,
                                  int32_t *parts)
{
    int32_t np = 0;
    for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) {
        int32_t q = where[adjncy[j]];
        if (conn[q] == 0) parts[np++] = q;
        conn[q] += adjwgt[j];
    }
    return np;
}

static inline void clear_conn(int64_t *conn, const int32_t *parts, int32_t np)
{
    for (int32_t i = 0; i < np; i++) conn[parts[i]] = 0;
}

typedef struct { int32_t key; int32_t v; } kv_t;
static int cmp_kv(const void *a, const void *b)
{
    const kv_t *x = (const kv_t *)a, *y = (const kv_t *)b;
    if (x->key != y->key) return (x->key > y->key) - (x->key < y->key);
    return (x->v > y->v) - (x->v < y->v);
}

typedef struct {
    int32_t n, k;
    const int32_t *xadj, *adjncy, *vwgt, *adjwgt;
    const int64_t *opt, *maxp;
    int32_t *where, *dest, *pregain, *moves;
    int8_t *lock;
    int64_t *pw;
    int64_t **conn_t;
    int32_t **parts_t;
} rstate;

/* Label-propagation move set with afterburner (jetlp). Returns #moves;
 * *ncand_out = number of candidates before the afterburner. */
static int32_t lp_moves(rstate *s, int32_t finest, int32_t *ncand_out)
{
    const int32_t n = s->n;
    int32_t ncand = 0;
#pragma omp parallel for reduction(+ : ncand) schedule(dynamic, 2048)
    for (int32_t v = 0; v < n; v++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int64_t *conn = s->conn_t[tid];
        int32_t *parts = s->parts_t[tid];
        int32_t p = s->where[v];
        int32_t np = gather_conn(v, s->xadj, s->adjncy, s->adjwgt, s->where, conn, parts);
        int64_t pc = conn[p], bc = 0;
        int32_t b = -1;
        for (int32_t i = 0; i < np; i++) {
            int32_t q = parts[i];
            if (q == p) continue;
            if (conn[q] > bc || (conn[q] == bc && b >= 0 && q < b)) { bc = conn[q]; b = q; }
        }
        clear_conn(conn, parts, np);
        s->pregain[v] = INT32_MIN;
        s->dest[v] = p;
        if (b < 0) continue;
        int64_t thr = finest ? pc / 4 : (3 * pc) / 4;
        if ((bc >= pc || (pc - bc) < thr) && !s->lock[v]) {
            s->pregain[v] = (int32_t)(bc - pc);
            s->dest[v] = b;
            ncand++;
        }
    }
    *ncand_out = ncand;
    if (ncand == 0) return 0;
    int32_t nm = 0;
    int8_t *sel = (int8_t *)xmalloc((size_t)n);
#pragma omp parallel for schedule(dynamic, 2048)
    for (int32_t v = 0; v < n; v++) {
        sel[v] = 0;
        int32_t g = s->pregain[v];
        if (g == INT32_MIN) continue;
        int32_t p = s->where[v], b = s->dest[v];
        int64_t change = 0;
        for (int32_t j = s->xadj[v]; j < s->xadj[v + 1]; j++) {
            int32_t u = s->adjncy[j];
            int32_t gu = s->pregain[u];
            if (gu > g || (gu == g && u < v)) {
                int32_t w = s->adjwgt[j];
                int32_t du = s->dest[u], wu = s->where[u];
                if (du == p) change -= w;
                else if (du == b) change += w;
                if (wu == p) change += w;
                else if (wu == b) change -= w;
            }
        }
        if ((int64_t)g + change >= 0) sel[v] = 1;
    }
    for (int32_t v = 0; v < n; v++) {
        s->lock[v] = sel[v];
        if (sel[v]) s->moves[nm++] = v;
    }
    free(sel);
    return nm;
}

/* Weak rebalance (jetrw). */
static int32_t rw_moves(rstate *s)
{
    const int32_t n = s->n, k = s->k;
    int32_t *und = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)k);
    int32_t nu = 0;
    for (int32_t p = 0; p < k; p++) {
        int64_t md = (s->maxp[p] * 99) / 100;
        if (md < s->maxp[p] - 100) md = s->maxp[p] - 100;
        if (s->pw[p] < md) und[nu++] = p;
    }
    kv_t *cand = (kv_t *)xmalloc(sizeof(kv_t) * (size_t)n);
    int32_t *bkt = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
#pragma omp parallel for schedule(dynamic, 2048)
    for (int32_t v = 0; v < n; v++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int32_t p = s->where[v];
        s->dest[v] = p;
        bkt[v] = -1;
        if (!(s->pw[p] > s->maxp[p] && 2 * (int64_t)s->vwgt[v] < 3 * (s->pw[p] - s->opt[p])))
            continue;
        int64_t *conn = s->conn_t[tid];
        int32_t *parts = s->parts_t[tid];
        int32_t np = gather_conn(v, s->xadj, s->adjncy, s->adjwgt, s->where, conn, parts);
        int64_t pc = conn[p], bc = 0;
        int32_t b = -1;
        for (int32_t i = 0; i < np; i++) {
            int32_t q = parts[i];
            if (!(s->pw[q] < s->maxp[q])) continue;
            if (conn[q] > bc || (conn[q] == bc && b >= 0 && q < b)) { bc = conn[q]; b = q; }
        }
        clear_conn(conn, parts, np);
        int64_t g;
        if (b >= 0) { g = bc - pc; }
        else {
            if (nu == 0) continue;
            b = und[v % nu];
            g = -pc;
        }
        s->dest[v] = b;
        bkt[v] = ora_gain_bucket((int32_t)g, s->vwgt[v]);
    }
    int32_t nc = 0;
    for (int32_t v = 0; v < n; v++)
        if (bkt[v] >= 0) { cand[nc].key = s->where[v] * 64 + bkt[v]; cand[nc].v = v; nc++; }
    qsort(cand, (size_t)nc, sizeof(kv_t), cmp_kv);
    int8_t *sel = (int8_t *)calloc((size_t)n, 1);
    int64_t acc = 0;
    int32_t curp = -1;
    for (int32_t i = 0; i < nc; i++) {
        int32_t v = cand[i].v, p = s->where[v];
        if (p != curp) { curp = p; acc = 0; }
        if (acc < s->pw[p] - s->maxp[p]) sel[v] = 1;
        acc += s->vwgt[v];
    }
    int32_t nm = 0;
    for (int32_t v = 0; v < n; v++)
        if (sel[v]) s->moves[nm++] = v;
        else s->dest[v] = s->where[v];
    free(sel); free(cand); free(bkt); free(und);
    return nm;
}

/* Strong rebalance (jetrs) with the cookie cutter. */
static int32_t rs_moves(rstate *s)
{
    const int32_t n = s->n, k = s->k;
    kv_t *cand = (kv_t *)xmalloc(sizeof(kv_t) * (size_t)n);
    int32_t *bkt = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
#pragma omp parallel for schedule(dynamic, 2048)
    for (int32_t v = 0; v < n; v++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        int32_t p = s->where[v];
        s->dest[v] = p;
        bkt[v] = -1;
        if (!(s->pw[p] > s->maxp[p])) continue;
        if (!((int64_t)s->vwgt[v] < 2 * (s->pw[p] - s->opt[p]))) continue;
        int64_t *conn = s->conn_t[tid];
        int32_t *parts = s->parts_t[tid];
        int32_t np = gather_conn(v, s->xadj, s->adjncy, s->adjwgt, s->where, conn, parts);
        int64_t pc = conn[p];
        clear_conn(conn, parts, np);
        bkt[v] = ora_gain_bucket((int32_t)(-pc), s->vwgt[v]);
    }
    int32_t nc = 0;
    for (int32_t v = 0; v < n; v++)
        if (bkt[v] >= 0) { cand[nc].key = s->where[v] * 64 + bkt[v]; cand[nc].v = v; nc++; }
    qsort(cand, (size_t)nc, sizeof(kv_t), cmp_kv);
    /* evicted prefix of every overweight part */
    int32_t *ev = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(nc + 1));
    int32_t ne = 0;
    for (int32_t i = 0; i < nc;) {
        int32_t p = s->where[cand[i].v];
        int32_t j = i;
        while (j < nc && s->where[cand[j].v] == p) j++;
        int64_t need = s->pw[p] - s->maxp[p], acc = 0;
        int32_t e = i;
        while (e < j && acc < need) { acc += s->vwgt[cand[e].v]; e++; }
        for (int32_t t = i; t < e; t++) ev[ne++] = cand[t].v;
        i = j;
    }
    int64_t *sc = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)(ne + 1));
    sc[0] = 0;
    for (int32_t i = 0; i < ne; i++) sc[i + 1] = sc[i] + s->vwgt[ev[i]];
    int32_t *es = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)k);
    int32_t *ee = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)k);
    int32_t st = 0;
    for (int32_t p = 0; p < k; p++) {
        int64_t room = s->maxp[p] > s->pw[p] ? s->maxp[p] - s->pw[p] : 0;
        es[p] = st;
        int32_t lo = st, hi = ne;
        int64_t find = sc[lo] + room;
        while (lo + 1 < hi) {
            int32_t mid = (lo + hi) / 2;
            if (sc[mid] >= find) hi = mid; else lo = mid;
        }
        int64_t dh = iabs64(sc[hi] - find), dl = iabs64(sc[lo] - find);
        ee[p] = dh < dl ? hi : lo;
        st = ee[p];
    }
    int32_t nm = 0;
    for (int32_t i = 0; i < ne; i++) {
        int32_t p = k - 1;
        while (p > 0 && es[p] > i) p--;
        int32_t v = ev[i];
        if (i < ee[p] && p != s->where[v]) { s->dest[v] = p; s->moves[nm++] = v; }
    }
    free(cand); free(bkt); free(ev); free(sc); free(es); free(ee);
    return nm;
}

int64_t ora_refine(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                   const int32_t *vwgt, const int32_t *adjwgt, int32_t nparts,
                   const int64_t *opt, const int64_t *maxp, int32_t finest,
                   int32_t patience, int32_t *where, int32_t *passes_out)
{
    rstate s;
    s.n = n; s.k = nparts;
    s.xadj = xadj; s.adjncy = adjncy; s.vwgt = vwgt; s.adjwgt = adjwgt;
    s.opt = opt; s.maxp = maxp; s.where = where;
    s.dest = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    s.pregain = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    s.moves = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    s.lock = (int8_t *)calloc((size_t)(n > 0 ? n : 1), 1);
    s.pw = (int64_t *)calloc((size_t)nparts, sizeof(int64_t));
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    s.conn_t = (int64_t **)xmalloc(sizeof(int64_t *) * (size_t)nt);
    s.parts_t = (int32_t **)xmalloc(sizeof(int32_t *) * (size_t)nt);
    for (int t = 0; t < nt; t++) {
        s.conn_t[t] = (int64_t *)calloc((size_t)nparts, sizeof(int64_t));
        s.parts_t[t] = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nparts);
    }
    int32_t *best = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    for (int32_t v = 0; v < n; v++) s.pw[where[v]] += vwgt[v];
    int64_t cut = ora_edgecut(n, xadj, adjncy, adjwgt, where);
    int64_t excess = INT64_MIN;
    for (int32_t p = 0; p < nparts; p++)
        if (s.pw[p] - maxp[p] > excess) excess = s.pw[p] - maxp[p];
    memcpy(best, where, sizeof(int32_t) * (size_t)n);
    int64_t best_cut = cut, best_excess = excess;
    int32_t count = 0, bal_counter = 0, passes = 0;
    int lp_idle = 0;
    const int dbg = getenv("HP_DEBUG_PASSES") != NULL;

    while (count++ <= patience) {
        passes++;
        int32_t nm, ncand = -1;
        int mode;
        if (excess <= 0) {
            nm = lp_moves(&s, finest, &ncand);
            bal_counter = 0;
            mode = 0;
        } else if (bal_counter < 2) {
            nm = rw_moves(&s);
            bal_counter++;
            mode = 1;
        } else {
            nm = rs_moves(&s);
            bal_counter++;
            mode = 2;
        }
        for (int32_t i = 0; i < nm; i++) {
            int32_t v = s.moves[i];
            s.pw[where[v]] -= vwgt[v];
            s.pw[s.dest[v]] += vwgt[v];
        }
        for (int32_t i = 0; i < nm; i++) {
            int32_t v = s.moves[i];
            where[v] = s.dest[v];
        }
        if (nm > 0) cut = ora_edgecut(n, xadj, adjncy, adjwgt, where);
        excess = INT64_MIN;
        for (int32_t p = 0; p < nparts; p++)
            if (s.pw[p] - maxp[p] > excess) excess = s.pw[p] - maxp[p];
        if (dbg)
            fprintf(stderr, "ora pass n=%d pass=%d mode=%d moves=%d cut=%lld excess=%lld\n", n, passes,
                    mode, nm, (long long)cut, (long long)excess);

        if (best_excess > 0 && excess < best_excess) {
            best_excess = excess; best_cut = cut;
            memcpy(best, where, sizeof(int32_t) * (size_t)n);
            count = 0;
        } else if (cut < best_cut && (excess <= 0 || excess <= best_excess)) {
            if (1000 * cut < 999 * best_cut) count = 0;
            best_excess = excess; best_cut = cut;
            memcpy(best, where, sizeof(int32_t) * (size_t)n);
        }
        /* A pass that changed nothing repeats identically: stop (same result). */
        int stalled = nm == 0 && (mode == 2 || (mode == 0 && (ncand == 0 || lp_idle)));
        lp_idle = (mode == 0 && nm == 0);
        if (stalled) break;
        /* hard bound on passes per level, the same as the device-side loop's */
        if (passes >= ORA_MAX_REFINE_PASSES) break;
    }
    memcpy(where, best, sizeof(int32_t) * (size_t)n);
    for (int t = 0; t < nt; t++) { free(s.conn_t[t]); free(s.parts_t[t]); }
    free(s.conn_t); free(s.parts_t);
    free(s.dest); free(s.pregain); free(s.moves); free(s.lock); free(s.pw); free(best);
    if (passes_out) *passes_out = passes;
    return best_cut;
}

/* ------------------------------------------------------------------------- */
/* V-cycle.                                                                   */

typedef struct {
    int32_t n;
    int64_t m;
    int32_t *xadj, *adjncy, *adjwgt, *vwgt, *match, *cmap, *where_start, *where_final;
    int64_t cut_start, cut_final;
    int owns_graph;
} olevel;

struct ora_trace {
    int32_t nlevels;
    olevel *lv;
};

int ora_trace_nlevels(const ora_trace *t) { return t ? t->nlevels : 0; }

int ora_trace_level(const ora_trace *t, int level, int32_t *n, int64_t *m,
                    int64_t *cut_start, int64_t *cut_final)
{
    if (!t || level < 0 || level >= t->nlevels) return HP_ERR_INVALID_ARG;
    if (n) *n = t->lv[level].n;
    if (m) *m = t->lv[level].m;
    if (cut_start) *cut_start = t->lv[level].cut_start;
    if (cut_final) *cut_final = t->lv[level].cut_final;
    return HP_OK;
}

int ora_trace_copy(const ora_trace *t, int level, int what, int32_t *dst, int64_t count)
{
    if (!t || level < 0 || level >= t->nlevels || !dst) return HP_ERR_INVALID_ARG;
    const olevel *l = &t->lv[level];
    const int32_t *src = NULL;
    int64_t len = 0;
    switch (what) {
    case HP_TRACE_XADJ: src = l->xadj; len = (int64_t)l->n + 1; break;
    case HP_TRACE_ADJNCY: src = l->adjncy; len = l->m; break;
    case HP_TRACE_ADJWGT: src = l->adjwgt; len = l->m; break;
    case HP_TRACE_VWGT: src = l->vwgt; len = l->n; break;
    case HP_TRACE_MATCH: src = l->match; len = l->n; break;
    case HP_TRACE_CMAP: src = l->cmap; len = l->n; break;
    case HP_TRACE_WHERE_START: src = l->where_start; len = l->n; break;
    case HP_TRACE_WHERE_FINAL: src = l->where_final; len = l->n; break;
    default: return HP_ERR_INVALID_ARG;
    }
    if (!src || count < len) return HP_ERR_INVALID_ARG;
    memcpy(dst, src, sizeof(int32_t) * (size_t)len);
    return HP_OK;
}

void ora_trace_free(ora_trace *t)
{
    if (!t) return;
    for (int i = 0; i < t->nlevels; i++) {
        olevel *l = &t->lv[i];
        if (l->owns_graph) { free(l->xadj); free(l->adjncy); free(l->adjwgt); free(l->vwgt); }
        free(l->match); free(l->cmap); free(l->where_start); free(l->where_final);
    }
    free(t->lv);
    free(t);
}

/* Defaults of the tunables (same values as the library's hp_options_default). */
static void ora_options_default(hp_options *o)
{
    memset(o, 0, sizeof(*o));
    o->version = HP_OPTIONS_VERSION;
    o->coarsen_to = 0;
    o->match_rounds = 6;
    o->refine_patience = 5;
    o->init_starts = 256;
    o->fm_passes = 10;
    o->max_levels = 64;
    o->learned = 0;
    o->validate = 1;
    o->trace = 0;
    o->profile = 0;
    o->seed = 1;
}

static int32_t default_coarsen_to(int32_t nparts)
{
    /* hunyuangraph_partitiongraph.h:298-302 */
    int32_t thr = nparts * 8;
    if (thr > 1024) {
        thr = nparts * 2;
        if (thr < 1024) thr = 1024;
    }
    return thr;
}

int ora_partition(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                  const int32_t *vwgt_in, const int32_t *adjwgt_in, int32_t nparts,
                  const float *tpwgts, float ubfactor, const hp_options *opt_in,
                  int32_t *part, int64_t *edgecut, ora_trace **trace_out)
{
    hp_options opt;
    if (opt_in) opt = *opt_in; else ora_options_default(&opt);
    if (n < 0 || nparts < 1 || !xadj || (n > 0 && !adjncy) || !part) return HP_ERR_INVALID_ARG;
    if (nparts > HP_MAX_PARTS) return HP_ERR_UNSUPPORTED;
    if (!(ubfactor >= 1.0f)) return HP_ERR_INVALID_ARG;
    const int64_t m0 = xadj[n];
    int32_t *vw = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    int32_t *ew = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)m0);
    for (int32_t v = 0; v < n; v++) vw[v] = vwgt_in ? vwgt_in[v] : 1;
    for (int64_t j = 0; j < m0; j++) ew[j] = adjwgt_in ? adjwgt_in[j] : 1;
    int64_t tv = 0;
    for (int32_t v = 0; v < n; v++) tv += vw[v];
    if (tv >= INT32_MAX) { free(vw); free(ew); return HP_ERR_UNSUPPORTED; }
    int64_t tw = 0;
    for (int64_t j = 0; j < m0; j++) tw += ew[j];
    const int weight_check = tw >= (int64_t)INT32_MAX;
    if (weight_check && !ora_weight_range_ok(n, xadj, ew)) {
        free(vw); free(ew);
        return HP_ERR_UNSUPPORTED;
    }

    int cap = 16;
    olevel *lv = (olevel *)calloc((size_t)cap, sizeof(olevel));
    lv[0].n = n; lv[0].m = m0;
    lv[0].xadj = (int32_t *)xadj; lv[0].adjncy = (int32_t *)adjncy;
    lv[0].adjwgt = ew; lv[0].vwgt = vw; lv[0].owns_graph = 0;
    int32_t L = 0;
    const int32_t thr = opt.coarsen_to > 0 ? opt.coarsen_to : default_coarsen_to(nparts);
    const int64_t maxvwgt = (3 * tv) / (2 * (int64_t)thr);

    while (L < opt.max_levels && lv[L].n > thr) {
        olevel *f = &lv[L];
        f->match = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)f->n);
        f->cmap = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)f->n);
        int32_t cn = ora_match(f->n, f->xadj, f->adjncy, f->vwgt, f->adjwgt, L, opt.seed,
                               maxvwgt, opt.match_rounds, f->match, f->cmap);
        if (L + 1 >= cap) {
            cap *= 2;
            lv = (olevel *)realloc(lv, sizeof(olevel) * (size_t)cap);
            memset(lv + L + 1, 0, sizeof(olevel) * (size_t)(cap - L - 1));
            f = &lv[L];
        }
        olevel *c = &lv[L + 1];
        c->n = cn;
        c->m = ora_contract(f->n, f->xadj, f->adjncy, f->vwgt, f->adjwgt, f->match, f->cmap, cn,
                            &c->xadj, &c->adjncy, &c->adjwgt, &c->vwgt);
        c->owns_graph = 1;
        L++;
        if (weight_check && !ora_weight_range_ok(c->n, c->xadj, c->adjwgt)) {
            /* a coarse vertex's weighted degree reaches 2^31: the call fails as the library's does */
            for (int32_t l = 0; l <= L; l++) {
                olevel *g = &lv[l];
                if (g->owns_graph) { free(g->xadj); free(g->adjncy); free(g->adjwgt); free(g->vwgt); }
                free(g->match); free(g->cmap);
            }
            free(lv); free(vw); free(ew);
            return HP_ERR_UNSUPPORTED;
        }
        if (!(100 * (int64_t)c->n < 85 * (int64_t)f->n && c->m > c->n / 2)) break;
    }

    int64_t *topt = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)nparts);
    int64_t *tmax = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)nparts);
    ora_part_targets(tv, nparts, tpwgts, ubfactor, topt, tmax);
    const int64_t ub2 = ora_bisect_ub_fx(ubfactor, nparts);

    /* initial partition of the coarsest level */
    olevel *cl = &lv[L];
    cl->where_start = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)cl->n);
    ora_initpart(cl->n, cl->xadj, cl->adjncy, cl->vwgt, cl->adjwgt, nparts, topt, ub2,
                 opt.init_starts, opt.fm_passes, cl->where_start);

    /* uncoarsening */
    int32_t *where = NULL;
    for (int32_t l = L; l >= 0; l--) {
        olevel *g = &lv[l];
        if (l < L) {
            g->where_start = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)g->n);
            const int32_t *cw = lv[l + 1].where_final;
            for (int32_t v = 0; v < g->n; v++) g->where_start[v] = cw[g->cmap[v]];
        }
        g->where_final = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)g->n);
        memcpy(g->where_final, g->where_start, sizeof(int32_t) * (size_t)g->n);
        g->cut_start = ora_edgecut(g->n, g->xadj, g->adjncy, g->adjwgt, g->where_start);
        int32_t passes = 0;
        g->cut_final = ora_refine(g->n, g->xadj, g->adjncy, g->vwgt, g->adjwgt, nparts, topt,
                                  tmax, l == 0, opt.refine_patience, g->where_final, &passes);
        where = g->where_final;
    }
    memcpy(part, where, sizeof(int32_t) * (size_t)n);
    if (edgecut) *edgecut = lv[0].cut_final;
    free(topt); free(tmax);

    /* lv[0] graph arrays are borrowed except the weight copies */
    if (trace_out) {
        ora_trace *t = (ora_trace *)calloc(1, sizeof(ora_trace));
        /* give level 0 its own graph copy so the trace outlives the inputs */
        int32_t *x = (int32_t *)xmalloc(sizeof(int32_t) * ((size_t)n + 1));
        int32_t *a = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)m0);
        memcpy(x, xadj, sizeof(int32_t) * ((size_t)n + 1));
        memcpy(a, adjncy, sizeof(int32_t) * (size_t)m0);
        lv[0].xadj = x; lv[0].adjncy = a; lv[0].owns_graph = 1;
        t->nlevels = L + 1;
        t->lv = lv;
        *trace_out = t;
    } else {
        lv[0].xadj = NULL; lv[0].adjncy = NULL;
        free(ew); free(vw);
        lv[0].adjwgt = NULL; lv[0].vwgt = NULL;
        for (int32_t l = 0; l <= L; l++) {
            olevel *g = &lv[l];
            if (g->owns_graph) { free(g->xadj); free(g->adjncy); free(g->adjwgt); free(g->vwgt); }
            free(g->match); free(g->cmap); free(g->where_start); free(g->where_final);
        }
        free(lv);
    }
    return HP_OK;
}

/* ------------------------------------------------------------------------- */
/* Move-scoring MLP, FP32 (the reference for the device forward/backward).   */
/* Parameters: W1[32][8], b1[32], W2[32][32], b2[32], w3[32], b3.            */

#define OMLP_IN 8
#define OMLP_H 32
#define OMLP_W1 0
#define OMLP_B1 (OMLP_W1 + OMLP_H * OMLP_IN)
#define OMLP_W2 (OMLP_B1 + OMLP_H)
#define OMLP_B2 (OMLP_W2 + OMLP_H * OMLP_H)
#define OMLP_W3 (OMLP_B2 + OMLP_H)
#define OMLP_B3 (OMLP_W3 + OMLP_H)
#define OMLP_N (OMLP_B3 + 1)

static float omlp_fwd(const float *P, const float *x, float *z1, float *z2)
{
    float a1[OMLP_H];
    for (int j = 0; j < OMLP_H; j++) {
        float s = P[OMLP_B1 + j];
        for (int i = 0; i < OMLP_IN; i++) s += P[OMLP_W1 + j * OMLP_IN + i] * x[i];
        z1[j] = s;
        a1[j] = s > 0.f ? s : 0.f;
    }
    float y = P[OMLP_B3];
    for (int j = 0; j < OMLP_H; j++) {
        float s = P[OMLP_B2 + j];
        for (int i = 0; i < OMLP_H; i++) s += P[OMLP_W2 + j * OMLP_H + i] * a1[i];
        z2[j] = s;
        y += P[OMLP_W3 + j] * (s > 0.f ? s : 0.f);
    }
    return y;
}

void ora_mlp_forward(const float *P, const float *X, int64_t n, float *out)
{
    float z1[OMLP_H], z2[OMLP_H];
    for (int64_t r = 0; r < n; r++) out[r] = omlp_fwd(P, X + r * OMLP_IN, z1, z2);
}

/* Mean binary cross-entropy with logits and its gradient (double accumulators). */
float ora_mlp_loss_grad(const float *P, const float *X, const float *Y, int64_t n, float *grad)
{
    double g[OMLP_N];
    memset(g, 0, sizeof(g));
    double loss = 0.0;
    for (int64_t r = 0; r < n; r++) {
        const float *x = X + r * OMLP_IN;
        float z1[OMLP_H], z2[OMLP_H];
        const float y = omlp_fwd(P, x, z1, z2);
        const float t = Y[r];
        const double sp = y > 0 ? y + log1p(exp(-(double)y)) : log1p(exp((double)y));
        loss += sp - (double)t * y;
        const double dy = 1.0 / (1.0 + exp(-(double)y)) - t;
        g[OMLP_B3] += dy;
        double da1[OMLP_H];
        memset(da1, 0, sizeof(da1));
        for (int j = 0; j < OMLP_H; j++) {
            g[OMLP_W3 + j] += dy * (z2[j] > 0.f ? z2[j] : 0.f);
            const double dz2 = z2[j] > 0.f ? dy * P[OMLP_W3 + j] : 0.0;
            g[OMLP_B2 + j] += dz2;
            for (int i = 0; i < OMLP_H; i++) {
                g[OMLP_W2 + j * OMLP_H + i] += dz2 * (z1[i] > 0.f ? z1[i] : 0.f);
                da1[i] += dz2 * P[OMLP_W2 + j * OMLP_H + i];
            }
        }
        for (int i = 0; i < OMLP_H; i++) {
            const double dz1 = z1[i] > 0.f ? da1[i] : 0.0;
            g[OMLP_B1 + i] += dz1;
            for (int c = 0; c < OMLP_IN; c++) g[OMLP_W1 + i * OMLP_IN + c] += dz1 * x[c];
        }
    }
    for (int i = 0; i < OMLP_N; i++) grad[i] = (float)(g[i] / (double)n);
    return (float)(loss / (double)n);
}

/* ------------------------------------------------------------------------- */
/* Nested-dissection ordering (the library's hp_node_nd).                     */
/*
 * Follows the structure of the reference's NestedBisection / ReorderGraph
 * (mygp_0.9.9_test_initpartition/reordergraph.h:177-306): a vertex separator
 * of the graph is numbered last, the two sides are split off as induced
 * subgraphs and ordered recursively (left side first, then right), and a
 * subgraph of at most ND_LEAF vertices or without edges is ordered directly
 * (the reference calls MMD_Order from mmdorder.h, which the reference tree
 * does not contain; here an exact minimum-degree elimination).  The rules
 * that the reference leaves to randomised code are fixed:
 *   - the 2-way partition is this library's multilevel partition (k = 2,
 *     imbalance ND_UB, unit edge weights, the caller's vertex weights and
 *     options, coarsened to ND_COARSEN_TO vertices unless the caller sets
 *     coarsen_to), where the reference runs its own randomised bisection with
 *     node refinement (reordergraph.h:17-135, refine.h:1398-1856);
 *   - separator: the boundary vertices of the side with fewer of them (side
 *     0 on a tie), then thinning: a separator vertex without a neighbour in
 *     the rest of its own side joins the other side (decided for every
 *     separator vertex at once, which keeps a separator);
 *   - numbering: separator vertices in increasing local id take the highest
 *     numbers of the subgraph's range; the left side the lowest block, the
 *     right side the block before the separator;
 *   - a split that leaves the whole subgraph on one side (no separator, an
 *     empty side) orders the subgraph by increasing vertex id;
 *   - leaves: repeatedly the live vertex of least degree in the elimination
 *     graph (ties: lowest id) takes the next number and its live neighbours
 *     become a clique.
 */
#define ND_LEAF 120
#define ND_UB 1.05f
/* the separator partitions coarsen to graphs of about leaf size (when the
 * caller's coarsen_to is 0), not to the 2-way rule's 16 vertices: every level
 * below that costs a subgraph's partition its launches and buys nothing */
#define ND_COARSEN_TO 128

typedef struct {
    int32_t n;
    int32_t *xadj, *adjncy, *vwgt, *label;
} nd_sub;

static void nd_free(nd_sub *s)
{
    free(s->xadj); free(s->adjncy); free(s->vwgt); free(s->label);
    memset(s, 0, sizeof(*s));
}

/* Exact minimum-degree elimination of a leaf (n <= ND_LEAF), numbers lo.. */
static void nd_leaf(const nd_sub *g, int32_t lo, int32_t *iperm)
{
    const int32_t n = g->n;
    if (n == 0) return;
    if (n > ND_LEAF || g->xadj[n] == 0) {   /* no edges: every degree stays 0 */
        for (int32_t v = 0; v < n; v++) iperm[g->label[v]] = lo + v;
        return;
    }
    enum { W = (ND_LEAF + 63) / 64 };
    uint64_t adj[ND_LEAF][W];
    memset(adj, 0, sizeof(adj));
    for (int32_t v = 0; v < n; v++)
        for (int32_t j = g->xadj[v]; j < g->xadj[v + 1]; j++) {
            const int32_t u = g->adjncy[j];
            adj[v][u >> 6] |= 1ull << (u & 63);
        }
    uint64_t alive[W];
    memset(alive, 0, sizeof(alive));
    for (int32_t v = 0; v < n; v++) alive[v >> 6] |= 1ull << (v & 63);
    for (int32_t step = 0; step < n; step++) {
        int32_t best = -1, bdeg = 0;
        for (int32_t v = 0; v < n; v++) {
            if (!(alive[v >> 6] >> (v & 63) & 1)) continue;
            int32_t d = 0;
            for (int w = 0; w < W; w++) d += __builtin_popcountll(adj[v][w] & alive[w]);
            if (best < 0 || d < bdeg) { best = v; bdeg = d; }
        }
        iperm[g->label[best]] = lo + step;
        alive[best >> 6] &= ~(1ull << (best & 63));
        uint64_t nb[W];
        for (int w = 0; w < W; w++) nb[w] = adj[best][w] & alive[w];
        for (int32_t u = 0; u < n; u++) {
            if (!(nb[u >> 6] >> (u & 63) & 1)) continue;
            for (int w = 0; w < W; w++) adj[u][w] |= nb[w];
            adj[u][u >> 6] &= ~(1ull << (u & 63));
        }
    }
}

/* One side (0 or 1) of a 3-way side_of (2 = separator) as an induced subgraph,
 * vertex order and row order kept. */
static void nd_split(const nd_sub *g, const int32_t *side_of, int32_t side, nd_sub *out)
{
    const int32_t n = g->n;
    int32_t *lid = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t cnt = 0;
    for (int32_t v = 0; v < n; v++) lid[v] = side_of[v] == side ? cnt++ : -1;
    out->n = cnt;
    out->xadj = (int32_t *)xmalloc(sizeof(int32_t) * ((size_t)cnt + 1));
    out->vwgt = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(cnt > 0 ? cnt : 1));
    out->label = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(cnt > 0 ? cnt : 1));
    int64_t m = 0;
    for (int32_t v = 0; v < n; v++)
        if (side_of[v] == side)
            for (int32_t j = g->xadj[v]; j < g->xadj[v + 1]; j++) m += side_of[g->adjncy[j]] == side;
    out->adjncy = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    int64_t e = 0;
    for (int32_t v = 0; v < n; v++) {
        if (side_of[v] != side) continue;
        out->xadj[lid[v]] = (int32_t)e;
        out->vwgt[lid[v]] = g->vwgt[v];
        out->label[lid[v]] = g->label[v];
        for (int32_t j = g->xadj[v]; j < g->xadj[v + 1]; j++)
            if (side_of[g->adjncy[j]] == side) out->adjncy[e++] = lid[g->adjncy[j]];
    }
    out->xadj[cnt] = (int32_t)e;
    free(lid);
}

/* The separator rule: side_of[v] in {0, 1, 2 (separator)} from a 2-way where. */
void ora_nd_separator(int32_t n, const int32_t *xadj, const int32_t *adjncy, const int32_t *where,
                      int32_t *side_of)
{
    int32_t bnd[2] = {0, 0};
    uint8_t *b = (uint8_t *)xmalloc((size_t)(n > 0 ? n : 1));
    for (int32_t v = 0; v < n; v++) {
        b[v] = 0;
        for (int32_t j = xadj[v]; j < xadj[v + 1]; j++)
            if (where[adjncy[j]] != where[v]) { b[v] = 1; break; }
        bnd[where[v]] += b[v];
    }
    const int32_t a = bnd[0] <= bnd[1] ? 0 : 1;
    for (int32_t v = 0; v < n; v++) {
        side_of[v] = where[v];
        if (where[v] != a || !b[v]) continue;
        int keep = 0;   /* a neighbour in the rest of side a keeps v in the separator */
        for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) {
            const int32_t u = adjncy[j];
            if (where[u] == a && !b[u]) { keep = 1; break; }
        }
        side_of[v] = keep ? 2 : 1 - a;
    }
    free(b);
}

static int nd_rec(nd_sub *g, int32_t hi, const hp_options *opt, int32_t *iperm)
{
    const int32_t n = g->n;
    if (n == 0) return HP_OK;
    const int32_t lo = hi - n;
    if (n <= ND_LEAF || g->xadj[n] == 0) {
        nd_leaf(g, lo, iperm);
        return HP_OK;
    }
    int32_t *where = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    int64_t cut = 0;
    int rc = ora_partition(n, g->xadj, g->adjncy, g->vwgt, NULL, 2, NULL, ND_UB, opt, where, &cut, NULL);
    if (rc != HP_OK) { free(where); return rc; }
    int32_t *side_of = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    ora_nd_separator(n, g->xadj, g->adjncy, where, side_of);
    free(where);
    int32_t cnt[3] = {0, 0, 0};
    for (int32_t v = 0; v < n; v++) cnt[side_of[v]]++;
    if (cnt[0] == n || cnt[1] == n) {   /* no progress: vertex order */
        for (int32_t v = 0; v < n; v++) iperm[g->label[v]] = lo + v;
        free(side_of);
        return HP_OK;
    }
    int32_t r = 0;
    for (int32_t v = 0; v < n; v++)
        if (side_of[v] == 2) iperm[g->label[v]] = hi - cnt[2] + r++;
    nd_sub L, R;
    nd_split(g, side_of, 0, &L);
    nd_split(g, side_of, 1, &R);
    free(side_of);
    nd_free(g);   /* the parent is not needed below */
    rc = nd_rec(&L, hi - cnt[2] - cnt[1], opt, iperm);
    if (rc == HP_OK) rc = nd_rec(&R, hi - cnt[2], opt, iperm);
    nd_free(&L);
    nd_free(&R);
    return rc;
}

int ora_node_nd(int32_t n, const int32_t *xadj, const int32_t *adjncy, const int32_t *vwgt,
                const hp_options *opt_in, int32_t *perm, int32_t *iperm)
{
    if (n < 0 || !xadj || (n > 0 && !adjncy) || !iperm) return HP_ERR_INVALID_ARG;
    hp_options opt;
    if (opt_in) opt = *opt_in; else ora_options_default(&opt);
    opt.trace = 0;
    if (opt.coarsen_to <= 0) opt.coarsen_to = ND_COARSEN_TO;
    nd_sub g;
    g.n = n;
    const int64_t m = xadj[n];
    g.xadj = (int32_t *)xmalloc(sizeof(int32_t) * ((size_t)n + 1));
    g.adjncy = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    g.vwgt = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    g.label = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    memcpy(g.xadj, xadj, sizeof(int32_t) * ((size_t)n + 1));
    if (m > 0) memcpy(g.adjncy, adjncy, sizeof(int32_t) * (size_t)m);
    for (int32_t v = 0; v < n; v++) { g.vwgt[v] = vwgt ? vwgt[v] : 1; g.label[v] = v; }
    const int rc = nd_rec(&g, n, &opt, iperm);
    nd_free(&g);
    if (rc == HP_OK && perm)
        for (int32_t v = 0; v < n; v++) perm[iperm[v]] = v;
    return rc;
}

/* Entries of the Cholesky factor L (diagonal included) of the symmetric
 * matrix with this sparsity under the ordering iperm (old -> new): the
 * elimination tree (Liu's algorithm with path compression), then each row's
 * subtree walked from its below-diagonal entries up to the marked nodes. */
int64_t ora_cholesky_nnz(int32_t n, const int32_t *xadj, const int32_t *adjncy, const int32_t *iperm)
{
    if (n <= 0) return 0;
    int32_t *perm = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    for (int32_t v = 0; v < n; v++) perm[iperm[v]] = v;
    int32_t *parent = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    int32_t *anc = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    for (int32_t i = 0; i < n; i++) {
        parent[i] = -1;
        anc[i] = -1;
        const int32_t v = perm[i];
        for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) {
            int32_t k = iperm[adjncy[j]];
            while (k >= 0 && k < i) {
                const int32_t next = anc[k];
                anc[k] = i;
                if (next < 0) { parent[k] = i; break; }
                k = next;
            }
        }
    }
    int32_t *mark = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    for (int32_t i = 0; i < n; i++) mark[i] = -1;
    int64_t nnz = 0;
    for (int32_t i = 0; i < n; i++) {
        nnz++;   /* diagonal */
        mark[i] = i;
        const int32_t v = perm[i];
        for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) {
            int32_t k = iperm[adjncy[j]];
            if (k >= i) continue;
            for (; mark[k] != i; k = parent[k]) {   /* row i of L has column k */
                nnz++;
                mark[k] = i;
            }
        }
    }
    free(perm); free(parent); free(anc); free(mark);
    return nnz;
}
