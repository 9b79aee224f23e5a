// ref_harness.cu — TEST INFRASTRUCTURE ONLY.  C wrappers around the
// reference's own CPU routines, compiled from the reference sources where they
// lie (see build_ref.sh; nothing of the reference is copied into this
// repository).  Used by tests/ to pin the oracle's contraction, edge-cut and
// graph-split semantics against the reference implementation, and by
// bench.py's CPU-baseline leg to time the reference's CPU coarsening
// (ref_cpu_coarsen).
#include "HunyuanGRAPH.h"

extern "C" {

// hunyuangraph_cpu_create_cgraph (hunyuangraph_CPU_contraction.h:9-100) on a
// caller-supplied matching.  Rows come back in the reference's insertion order.
int ref_cpu_contract(int n, const int *xadj, const int *adjncy, const int *vwgt, const int *adjwgt,
                     const int *match, const int *cmap, int cnvtxs, int *cxadj, int *cadjncy,
                     int *cadjwgt, int *cvwgt)
{
    hunyuangraph_admin_t admin;
    memset(&admin, 0, sizeof(admin));
    admin.mcore = hunyuangraph_create_mcore(0);
    hunyuangraph_graph_t *g = hunyuangraph_set_first_level_graph(
        n, (int *)xadj, (int *)adjncy, (int *)vwgt, (int *)adjwgt);
    g->cmap = (int *)cmap;
    hunyuangraph_cpu_create_cgraph(&admin, g, cnvtxs, (int *)match);
    hunyuangraph_graph_t *c = g->coarser;
    memcpy(cxadj, c->xadj, sizeof(int) * (cnvtxs + 1));
    memcpy(cadjncy, c->adjncy, sizeof(int) * c->xadj[cnvtxs]);
    memcpy(cadjwgt, c->adjwgt, sizeof(int) * c->xadj[cnvtxs]);
    memcpy(cvwgt, c->vwgt, sizeof(int) * cnvtxs);
    return c->xadj[cnvtxs];
}

// hunyuangraph_computecut_cpu (hunyuangraph_graph.h:144-155), int cut.
int ref_cpu_edgecut(int n, const int *xadj, const int *adjncy, const int *adjwgt, const int *where)
{
    hunyuangraph_graph_t g;
    memset(&g, 0, sizeof(g));
    g.nvtxs = n;
    g.xadj = (int *)xadj;
    g.adjncy = (int *)adjncy;
    g.adjwgt = (int *)adjwgt;
    return hunyuangraph_computecut_cpu(&g, (int *)where);
}

// The reference's CPU coarsening (hunyuangraph_cpu_coarsen,
// hunyuangraph_CPU_coarsen.h:11-46: HEM matching + hash contraction per level)
// down to coarsen_to vertices; returns the number of levels and the coarsest
// vertex count.  Weighted graphs only (the unit-weight RM path of the
// reference dereferences an uninitialised pointer).
int ref_cpu_coarsen(int n, const int *xadj, const int *adjncy, const int *vwgt, const int *adjwgt,
                    int coarsen_to, int *coarsest_n)
{
    hunyuangraph_admin_t admin;
    memset(&admin, 0, sizeof(admin));
    admin.mcore = hunyuangraph_create_mcore(0);
    admin.Coarsen_threshold = coarsen_to;
    admin.no2hop = 1;
    hunyuangraph_graph_t *g = hunyuangraph_set_first_level_graph(
        n, (int *)xadj, (int *)adjncy, (int *)vwgt, (int *)adjwgt);
    hunyuangraph_graph_t *c = hunyuangraph_cpu_coarsen(&admin, g);
    int levels = 0;
    for (hunyuangraph_graph_t *t = c; t->finer; t = t->finer) levels++;
    *coarsest_n = c->nvtxs;
    return levels;
}

// hunyuangraph_splitgraph (hunyuangraph_CPU_splitgraph.h:8-167): the two
// induced subgraphs of a 2-way partition; side 0 or 1 is copied out.  The
// function copies the rows of vertices whose bndptr is -1 whole and filters
// the others, so bndptr is set here to -1 exactly for the vertices with no
// neighbour on the other side.  Labels start as the vertex ids.
int ref_cpu_split(int n, const int *xadj, const int *adjncy, const int *vwgt, const int *adjwgt,
                  const int *where, int side, int *sn, int *sxadj, int *sadjncy, int *sadjwgt, int *svwgt,
                  int *slabel)
{
    hunyuangraph_admin_t admin;
    memset(&admin, 0, sizeof(admin));
    admin.mcore = hunyuangraph_create_mcore(0);
    hunyuangraph_graph_t *g = hunyuangraph_set_first_level_graph(
        n, (int *)xadj, (int *)adjncy, (int *)vwgt, (int *)adjwgt);
    const size_t cap = (size_t)(n > 0 ? n : 1);
    int *label = (int *)malloc(sizeof(int) * cap);
    int *wh = (int *)malloc(sizeof(int) * cap);
    int *bnd = (int *)malloc(sizeof(int) * cap);
    for (int i = 0; i < n; i++) {
        label[i] = i;
        wh[i] = where[i];
        bnd[i] = -1;
        for (int j = xadj[i]; j < xadj[i + 1]; j++)
            if (where[adjncy[j]] != where[i]) bnd[i] = 0;
    }
    g->label = label;
    g->where = wh;
    g->bndptr = bnd;
    hunyuangraph_graph_t *l = nullptr, *r = nullptr;
    hunyuangraph_splitgraph(&admin, g, &l, &r);
    hunyuangraph_graph_t *o = side ? r : l;
    *sn = o->nvtxs;
    memcpy(sxadj, o->xadj, sizeof(int) * (o->nvtxs + 1));
    memcpy(sadjncy, o->adjncy, sizeof(int) * o->nedges);
    memcpy(sadjwgt, o->adjwgt, sizeof(int) * o->nedges);
    memcpy(svwgt, o->vwgt, sizeof(int) * o->nvtxs);
    memcpy(slabel, o->label, sizeof(int) * o->nvtxs);
    return o->nedges;
}

}
