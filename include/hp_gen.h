/*
 * hp_gen.h — seeded synthetic graph generators (host, C ABI).
 *
 * The reference benchmarks SuiteSparse graphs that are downloaded on demand
 * (install_matrix.sh, graph_9.csv); these generators produce seeded stand-ins
 * with the shapes of the partition workloads: 2-D / 3-D grids, R-MAT and random
 * geometric graphs.  Every generated graph is symmetric, 0-based, free of self
 * loops and duplicate edges, with rows sorted by neighbour id.  Symmetric edge
 * weights come from a keyed hash of (seed, min(u,v), max(u,v)), so any two
 * generators run with the same seed agree bit for bit.
 *
 * No counterpart in the reference's partition interface: the reference reads a
 * METIS .graph file instead (hunyuangraph_io.h:25-187).
 */
#ifndef HP_GEN_H
#define HP_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hp_graph {
    int32_t  nvtxs;
    int64_t  nedges;   /* directed adjacency entries = 2 x undirected edges */
    int32_t *xadj;     /* malloc'ed; release with hp_graph_free()           */
    int32_t *adjncy;
    int32_t *vwgt;
    int32_t *adjwgt;
} hp_graph;

/* splitmix64 finaliser (Vigna) used for every keyed hash in the generators. */
uint64_t hp_gen_mix64(uint64_t z);
/* Weight of undirected edge {u,v}: wmin + hash(seed, min, max) mod (wmax-wmin+1). */
int32_t  hp_gen_edge_weight(uint64_t seed, int32_t u, int32_t v, int32_t wmin, int32_t wmax);

/* nx*ny 5-point grid, id = y*nx + x; unit vertex weights. */
int hp_gen_grid2d(int32_t nx, int32_t ny, uint64_t seed, int32_t wmin, int32_t wmax, hp_graph *out);
/* nx*ny*nz 7-point grid, id = (z*ny + y)*nx + x. */
int hp_gen_grid3d(int32_t nx, int32_t ny, int32_t nz, uint64_t seed, int32_t wmin,
                  int32_t wmax, hp_graph *out);
/* R-MAT: edgefactor * 2^scale generated pairs with quadrant probabilities
 * a, b, c (d = 1-a-b-c), self loops dropped, duplicates merged, symmetrised.
 * nvtxs_limit > 0 keeps only pairs with both ends < nvtxs_limit and sets the
 * vertex count to nvtxs_limit (used by the batch generator); 0 = 2^scale. */
int hp_gen_rmat(int32_t scale, int32_t edgefactor, double a, double b, double c,
                uint64_t seed, int32_t wmin, int32_t wmax, int32_t nvtxs_limit,
                hp_graph *out);
/* Random geometric graph: n points uniform in [0,1)^2 from (seed, i), edge when
 * distance < radius, weight = (int)(1000 * (1 - d / radius)) + 1. */
int hp_gen_rgg(int32_t n, double radius, uint64_t seed, hp_graph *out);

void hp_graph_free(hp_graph *g);

/* Host threads the generators use (OpenMP); 0 = all. */
void hp_gen_set_threads(int nthreads);

#ifdef __cplusplus
}
#endif

#endif /* HP_GEN_H */
