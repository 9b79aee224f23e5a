/*
 * hp_io.h — METIS .graph reader and .part writer, MatrixMarket reader (host, C ABI).
 *
 * Reference interface replaced:
 *   hunyuangraph_graph_t *hunyuangraph_readgraph(char *filename)   hunyuangraph_io.h:25-187
 *   void hunyuangraph_writetofile(char *fname, int *part, int n,
 *                                 int nparts)                      hunyuangraph_io.h:190-205
 * Same file format: '%' comment lines, header "nvtxs nedges [fmt]" with
 * fmt digits (vertex size, vertex weight, edge weight), 1-based neighbour
 * ids, the header counting undirected edges.  Errors are returned as codes
 * with a message instead of exit(); vertex sizes (fmt 1xx), which the
 * reference parses as a neighbour, are skipped.
 */
#ifndef HP_IO_H
#define HP_IO_H

#include <stdint.h>
#include "hp_gen.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Reads a METIS graph into *out (arrays malloc'ed; release with hp_graph_free).
 * Returns 0, or -1 (cannot open), -2 (format error; message in err). */
int hp_read_metis(const char *path, hp_graph *out, char *err, int errlen);

/* Writes one part id per line to "<fname>.part.<nparts>" (the reference's
 * naming).  Returns 0 or -1. */
int hp_write_partition(const char *fname, const int32_t *part, int32_t n, int32_t nparts);

/* Writes a graph in METIS format (fmt 011 when weights are present). */
int hp_write_metis(const char *path, const hp_graph *g);

/* Reads a square MatrixMarket coordinate matrix (pattern, integer, real or
 * complex; general, symmetric, skew-symmetric or hermitian) as the graph of
 * its symmetrised pattern: an edge {i, j} for every stored entry off the
 * diagonal, duplicates merged, rows sorted, unit vertex and edge weights.
 * Replaces the reference's converter (matrix_to_graph/matrix_to_graph.c:
 * union of the rows of A and A^T, diagonal removed, written as METIS).
 * Returns 0, -1 (cannot open), -2 (format error; message in err), -3 (memory). */
int hp_read_mtx(const char *path, hp_graph *out, char *err, int errlen);

#ifdef __cplusplus
}
#endif

#endif
