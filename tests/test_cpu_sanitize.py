"""The host C code under AddressSanitizer and UndefinedBehaviorSanitizer: the
oracle's V-cycle and components, the graph generators, and the METIS and
MatrixMarket readers and writers, driven by a small C program (valid graphs of
every generator, edge cases, and malformed files).  Any out-of-bounds access,
leak, or undefined operation ends the program with a sanitizer report."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FLAGS = ["-std=c11", "-g", "-O1", "-fno-omit-frame-pointer", "-fopenmp",
         "-fsanitize=address,undefined", "-fno-sanitize-recover=all"]

DRIVER = r'''
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "hp_partition.h"
#include "hp_gen.h"
#include "hp_io.h"
#include "hp_oracle.h"

static int failures = 0;
#define CHECK(c) do { if (!(c)) { fprintf(stderr, "check failed line %d: %s\n", __LINE__, #c); failures++; } } while (0)

static hp_options opts(int trace)
{
    hp_options o;
    memset(&o, 0, sizeof o);
    o.version = HP_OPTIONS_VERSION;
    o.match_rounds = 6;
    o.refine_patience = 5;
    o.init_starts = 16;
    o.fm_passes = 4;
    o.max_levels = 64;
    o.validate = 1;
    o.trace = trace;
    o.seed = 1;
    return o;
}

/* One V-cycle; checks part ids and the returned cut, and copies every traced array. */
static void run(const hp_graph *g, int32_t k, const float *tp, int trace)
{
    int32_t *part = malloc(sizeof(int32_t) * (size_t)(g->nvtxs > 0 ? g->nvtxs : 1));
    int64_t cut = -1;
    ora_trace *t = NULL;
    hp_options o = opts(trace);
    int rc = ora_partition(g->nvtxs, g->xadj, g->adjncy, g->vwgt, g->adjwgt, k, tp, 1.03f, &o, part, &cut,
                           trace ? &t : NULL);
    CHECK(rc == 0);
    if (rc == 0) {
        for (int32_t i = 0; i < g->nvtxs; i++) CHECK(part[i] >= 0 && part[i] < k);
        CHECK(ora_edgecut(g->nvtxs, g->xadj, g->adjncy, g->adjwgt, part) == cut);
    }
    if (t) {
        const int L = ora_trace_nlevels(t);
        CHECK(L >= 1);
        for (int l = 0; l < L; l++) {
            int32_t n;
            int64_t m, c0, c1;
            CHECK(ora_trace_level(t, l, &n, &m, &c0, &c1) == 0);
            const int64_t cap = (m > n + 1 ? m : n + 1);
            int32_t *buf = malloc(sizeof(int32_t) * (size_t)(cap > 0 ? cap : 1));
            for (int what = 0; what < 8; what++) ora_trace_copy(t, l, what, buf, cap);
            CHECK(ora_trace_copy(t, l, 0, buf, n) != 0);   /* too small: refused */
            free(buf);
        }
        CHECK(ora_trace_copy(t, L, 0, part, 1) != 0);
        ora_trace_free(t);
    }
    free(part);
}

/* One matching level and its contraction through the component entry points. */
static void components(const hp_graph *g)
{
    const int32_t n = g->nvtxs;
    int32_t *match = malloc(sizeof(int32_t) * (size_t)n), *cmap = malloc(sizeof(int32_t) * (size_t)(n + 1));
    const int32_t cn = ora_match(n, g->xadj, g->adjncy, g->vwgt, g->adjwgt, 0, 1, 1 << 20, 6, match, cmap);
    CHECK(cn > 0 && cn <= n);
    int32_t *cx = NULL, *ca = NULL, *cw = NULL, *cv = NULL;
    const int64_t cm = ora_contract(n, g->xadj, g->adjncy, g->vwgt, g->adjwgt, match, cmap, cn, &cx, &ca, &cw, &cv);
    CHECK(cm >= 0 && cm <= g->nedges && cx[cn] == cm);
    ora_free(cx); ora_free(ca); ora_free(cw); ora_free(cv);
    /* both sides of a 2-way split, and a where[] outside {0, 1} refused */
    int32_t *where = malloc(sizeof(int32_t) * (size_t)n);
    for (int32_t i = 0; i < n; i++) where[i] = (int32_t)((i * 2654435761u) % 3u == 0);
    int32_t *sx = malloc(sizeof(int32_t) * (size_t)(n + 1)), *sv = malloc(sizeof(int32_t) * (size_t)n);
    int32_t *sl = malloc(sizeof(int32_t) * (size_t)n);
    int32_t *sa = malloc(sizeof(int32_t) * (size_t)g->nedges), *sw = malloc(sizeof(int32_t) * (size_t)g->nedges);
    int64_t total = 0;
    for (int side = 0; side < 2; side++) {
        int32_t sn = -1;
        const int64_t sm = ora_split(n, g->xadj, g->adjncy, g->vwgt, g->adjwgt, where, side, &sn, sx, sa, sw, sv, sl);
        CHECK(sm >= 0 && sn >= 0 && sx[sn] == sm);
        total += sn;
    }
    CHECK(total == n);
    where[0] = 5;
    int32_t sn = 0;
    CHECK(ora_split(n, g->xadj, g->adjncy, g->vwgt, g->adjwgt, where, 0, &sn, sx, sa, sw, sv, sl) == -1);
    free(where); free(sx); free(sv); free(sl); free(sa); free(sw);
    free(match); free(cmap);
}

static void write_file(const char *path, const char *text)
{
    FILE *f = fopen(path, "w");
    fputs(text, f);
    fclose(f);
}

static int read_metis_text(const char *dir, const char *text)
{
    char path[512], err[256];
    snprintf(path, sizeof path, "%s/x.graph", dir);
    write_file(path, text);
    hp_graph g;
    memset(&g, 0, sizeof g);
    const int rc = hp_read_metis(path, &g, err, sizeof err);
    if (rc == 0) hp_graph_free(&g);
    return rc;
}

static int read_mtx_text(const char *dir, const char *text)
{
    char path[512], err[256];
    snprintf(path, sizeof path, "%s/x.mtx", dir);
    write_file(path, text);
    hp_graph g;
    memset(&g, 0, sizeof g);
    const int rc = hp_read_mtx(path, &g, err, sizeof err);
    if (rc == 0) hp_graph_free(&g);
    return rc;
}

int main(int argc, char **argv)
{
    const char *dir = argc > 1 ? argv[1] : ".";
    ora_set_threads(4);
    hp_gen_set_threads(4);
    hp_graph g;

    /* generators, partitions at several k (k = 1, odd k with targets, k > n) */
    CHECK(hp_gen_grid2d(40, 30, 6, 1, 5, &g) == 0);
    run(&g, 1, NULL, 0);
    run(&g, 8, NULL, 1);
    const float tp[7] = {0.3f, 0.2f, 0.2f, 0.1f, 0.1f, 0.05f, 0.05f};
    run(&g, 7, tp, 0);
    components(&g);
    hp_graph_free(&g);
    CHECK(hp_gen_grid2d(3, 2, 1, 1, 1, &g) == 0);
    run(&g, 9, NULL, 1);
    hp_graph_free(&g);
    CHECK(hp_gen_grid3d(10, 9, 8, 2, 1, 10, &g) == 0);
    run(&g, 64, NULL, 1);
    components(&g);
    hp_graph_free(&g);
    CHECK(hp_gen_rmat(11, 8, 0.57, 0.19, 0.19, 3, 1, 100, 0, &g) == 0);
    run(&g, 32, NULL, 1);
    components(&g);
    hp_graph_free(&g);
    CHECK(hp_gen_rgg(3000, 0.036, 4, &g) == 0);
    run(&g, 16, NULL, 0);
    hp_graph_free(&g);

    /* empty graph; isolated vertices and two components */
    {
        int32_t x0[1] = {0}, p0[1];
        int64_t cut = -1;
        hp_options o = opts(0);
        CHECK(ora_partition(0, x0, NULL, NULL, NULL, 4, NULL, 1.03f, &o, p0, &cut, NULL) == 0 && cut == 0);
        int32_t xadj[8] = {0, 1, 2, 2, 2, 4, 5, 6}, adj[6] = {1, 0, 5, 6, 4, 4};
        int32_t vw[7] = {1, 1, 1, 1, 1, 1, 1}, ew[6] = {1, 1, 1, 1, 1, 1};
        hp_graph s = {7, 6, xadj, adj, vw, ew};
        run(&s, 2, NULL, 1);
        run(&s, 3, NULL, 0);
    }

    /* METIS round trip, partition file */
    {
        char path[512], err[256];
        CHECK(hp_gen_grid2d(7, 5, 2, 1, 9, &g) == 0);
        snprintf(path, sizeof path, "%s/rt.graph", dir);
        CHECK(hp_write_metis(path, &g) == 0);
        hp_graph h;
        memset(&h, 0, sizeof h);
        CHECK(hp_read_metis(path, &h, err, sizeof err) == 0);
        CHECK(h.nvtxs == g.nvtxs && h.nedges == g.nedges);
        CHECK(memcmp(h.adjncy, g.adjncy, sizeof(int32_t) * (size_t)g.nedges) == 0);
        CHECK(memcmp(h.adjwgt, g.adjwgt, sizeof(int32_t) * (size_t)g.nedges) == 0);
        int32_t *part = calloc((size_t)g.nvtxs, sizeof(int32_t));
        CHECK(hp_write_partition(path, part, g.nvtxs, 4) == 0);
        free(part);
        hp_graph_free(&h);
        hp_graph_free(&g);
        snprintf(path, sizeof path, "%s/missing.graph", dir);
        CHECK(hp_read_metis(path, &h, err, sizeof err) == -1);
    }

    /* METIS: valid forms, then malformed files (format errors, never a crash) */
    CHECK(read_metis_text(dir, "% comment\n3 2\n2\n1 3\n2\n") == 0);
    CHECK(read_metis_text(dir, "3 2 011\n5 2 7\n1 1 7 3 4\n2 2 4\n") == 0);
    CHECK(read_metis_text(dir, "3 2 100\n9 2\n9 1 3\n9 2\n") == 0);
    CHECK(read_metis_text(dir, "") == -2);
    CHECK(read_metis_text(dir, "3\n") == -2);
    CHECK(read_metis_text(dir, "-3 2\n") == -2);
    CHECK(read_metis_text(dir, "3 2\n2\n1 3\n") == -2);            /* premature end */
    CHECK(read_metis_text(dir, "3 2\n2\n1 4\n2\n") == -2);         /* neighbour out of range */
    CHECK(read_metis_text(dir, "3 2\n0\n1 3\n2\n") == -2);         /* neighbour 0 */
    CHECK(read_metis_text(dir, "3 1\n2\n1 3\n2\n") == -2);         /* more edges than the header */
    CHECK(read_metis_text(dir, "3 5\n2\n1 3\n2\n") == -2);         /* fewer edges */
    CHECK(read_metis_text(dir, "3 2 011\n-1 2 7\n1 1 7 3 4\n2 2 4\n") == -2);
    CHECK(read_metis_text(dir, "3 2 001\n2 0\n1 0 3 4\n2 4\n") == -2);
    CHECK(read_metis_text(dir, "3 2 001\n2\n1 5 3 4\n2 4\n") == -2);   /* missing edge weight */
    CHECK(read_metis_text(dir, "3 2 010\n\n1 3\n2\n") == -2);          /* missing vertex weight */
    {
        /* one very long line */
        const int n = 20000;
        size_t cap = (size_t)n * 8 + 64, len = 0;
        char *text = malloc(cap);
        len += (size_t)snprintf(text + len, cap - len, "%d %d\n", n, n - 1);
        for (int i = 2; i <= n; i++) len += (size_t)snprintf(text + len, cap - len, "%d ", i);
        text[len++] = '\n';
        for (int i = 2; i <= n; i++) len += (size_t)snprintf(text + len, cap - len, "1\n");
        text[len] = 0;
        CHECK(read_metis_text(dir, text) == 0);
        free(text);
    }

    /* MatrixMarket: valid forms, then malformed files */
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2 1\n3 2\n") == 0);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate real general\n% c\n3 3 4\n1 2 0.5\n2 1 1\n3 3 2\n1 3 -1\n") == 0);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate complex hermitian\n2 2 1\n2 1 1 1\n") == 0);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate integer skew-symmetric\n2 2 1\n2 1 3\n") == 0);
    CHECK(read_mtx_text(dir, "") == -2);
    CHECK(read_mtx_text(dir, "3 3 2\n2 1\n3 2\n") == -2);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n") == -2);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate quaternion general\n2 2 1\n1 2 1\n") == -2);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate real weird\n2 2 1\n1 2 1\n") == -2);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate real general\n") == -2);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate real general\n2 3 1\n1 2 1\n") == -2);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate real general\n3 3 3\n1 2 1\n") == -2);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate real general\n3 3 1\n4 2 1\n") == -2);
    CHECK(read_mtx_text(dir, "%%MatrixMarket matrix coordinate real general\n3 3 1\n0 2 1\n") == -2);

    if (failures) { fprintf(stderr, "%d checks failed\n", failures); return 1; }
    printf("SANITIZED OK\n");
    return 0;
}
'''


def _sanitizers_available(tmp_path):
    cc = shutil.which("gcc")
    if not cc:
        return None
    src = tmp_path / "probe.c"
    src.write_text("int main(void) { return 0; }\n")
    r = subprocess.run([cc, *FLAGS, str(src), "-o", str(tmp_path / "probe")], capture_output=True)
    return cc if r.returncode == 0 else None


def test_host_code_under_asan_and_ubsan(tmp_path):
    cc = _sanitizers_available(tmp_path)
    if cc is None:
        pytest.skip("gcc with AddressSanitizer/UndefinedBehaviorSanitizer is not available")
    src = tmp_path / "driver.c"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    csrc = os.path.join(ROOT, "hunyuansc25_b200", "csrc")
    subprocess.run([cc, *FLAGS, "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "oracle"),
                    str(src), os.path.join(ROOT, "oracle", "hp_oracle.c"), os.path.join(csrc, "hp_io.c"),
                    os.path.join(csrc, "hp_gen.c"), "-lm", "-o", str(exe)], check=True)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-4000:]
    assert "SANITIZED OK" in r.stdout
