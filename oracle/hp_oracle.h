/*
 * hp_oracle.h — CPU oracle of the multilevel k-way partition path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a sequential (optionally OpenMP) C
 * restatement of the partition path that the CUDA library implements; it is
 * the checker in tests/, __graft_entry__.smoke() and bench.py's CPU baseline,
 * and nothing in the product links or calls it.
 *
 * Pins: the contraction and edge-cut semantics are checked against the
 * reference's own CPU code (hunyuangraph_cpu_create_cgraph,
 * hunyuangraph_computecut_cpu) compiled from the reference's sources by
 * oracle/build_ref.sh, and against committed fixtures in tests/golden/.
 * The reference publishes no golden vectors for matching, bisection or
 * refinement (it ships no tests); those rules are pinned only by this
 * restatement (parity unpinned at the reference-test level).
 */
#ifndef HP_ORACLE_H
#define HP_ORACLE_H

#include <stdint.h>
#include "hp_partition.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_trace ora_trace;

void ora_set_threads(int nthreads);
int  ora_get_threads(void);

/* Full V-cycle; same contract as hp_partition(). trace may be NULL. */
int ora_partition(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                  const int32_t *vwgt, const int32_t *adjwgt, int32_t nparts,
                  const float *tpwgts, float ubfactor, const hp_options *opt,
                  int32_t *part, int64_t *edgecut, ora_trace **trace);

int  ora_trace_nlevels(const ora_trace *t);
int  ora_trace_level(const ora_trace *t, int level, int32_t *n, int64_t *m,
                     int64_t *cut_start, int64_t *cut_final);
int  ora_trace_copy(const ora_trace *t, int level, int what, int32_t *dst, int64_t count);
void ora_trace_free(ora_trace *t);

/* ---- components (each follows the same rule as the CUDA path) ------------- */
/* 1 when every vertex's weighted degree is below 2^31 (the library's
 * weight-range rule, applied to the input and to every coarse level). */
int ora_weight_range_ok(int32_t n, const int32_t *xadj, const int32_t *adjwgt);
int64_t ora_edgecut(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                    const int32_t *adjwgt, const int32_t *where);

/* One matching level: fills match[n] (self when unmatched) and cmap[n];
 * returns the coarse vertex count. */
int32_t ora_match(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                  const int32_t *vwgt, const int32_t *adjwgt, int32_t level,
                  uint64_t seed, int64_t maxvwgt, int32_t rounds,
                  int32_t *match, int32_t *cmap);

/* Contraction of a matching: coarse CSR with rows sorted by neighbour id.
 * Output arrays are malloc'ed (free with ora_free). Returns coarse m. */
int64_t ora_contract(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                     const int32_t *vwgt, const int32_t *adjwgt,
                     const int32_t *match, const int32_t *cmap, int32_t cn,
                     int32_t **cxadj, int32_t **cadjncy, int32_t **cadjwgt,
                     int32_t **cvwgt);
void ora_free(void *p);

/* Target / maximum part weights shared by initial partitioning and refinement. */
void ora_part_targets(int64_t tvwgt, int32_t nparts, const float *tpwgts, float ubfactor,
                      int64_t *opt, int64_t *maxp);
int64_t ora_bisect_ub_fx(float ubfactor, int32_t nparts);

/* One side (0 or 1) of a 2-way split into induced subgraphs, as the recursive
 * bisection splits: vertices renumbered in id order, rows in their original
 * order without the other side's neighbours, labels = original ids.  Buffers:
 * n + 1 (sxadj), m (sadjncy, sadjwgt), n (svwgt, slabel).  Returns the side's
 * adjacency count, or -1 for a where[] entry outside {0, 1}. */
int64_t ora_split(int32_t n, const int32_t *xadj, const int32_t *adjncy, const int32_t *vwgt,
                  const int32_t *adjwgt, const int32_t *where, int32_t side, int32_t *sn,
                  int32_t *sxadj, int32_t *sadjncy, int32_t *sadjwgt, int32_t *svwgt, int32_t *slabel);

/* Recursive-bisection initial partition of a (small) graph. */
int ora_initpart(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                 const int32_t *vwgt, const int32_t *adjwgt, int32_t nparts,
                 const int64_t *tw, int64_t ub2_fx, int32_t starts, int32_t fm_passes,
                 int32_t *where);

/* Refinement of one level in place; returns the final cut. */
int64_t ora_refine(int32_t n, const int32_t *xadj, const int32_t *adjncy,
                   const int32_t *vwgt, const int32_t *adjwgt, int32_t nparts,
                   const int64_t *opt, const int64_t *maxp, int32_t finest,
                   int32_t patience, int32_t *where, int32_t *passes);

/* Move-scoring MLP in FP32 (parameters as in hp_mlp_set_params). */
void  ora_mlp_forward(const float *params, const float *x, int64_t n, float *out);
float ora_mlp_loss_grad(const float *params, const float *x, const float *y, int64_t n, float *grad);

/* Weak-rebalance gain bucket (float semantics of the reference). */
int32_t ora_gain_bucket(int32_t gain, int32_t vwgt);

/* Nested-dissection ordering (the library's hp_node_nd): perm[new] = old,
 * iperm[old] = new (perm may be NULL). */
int ora_node_nd(int32_t n, const int32_t *xadj, const int32_t *adjncy, const int32_t *vwgt,
                const hp_options *opt, int32_t *perm, int32_t *iperm);
/* The nested dissection's separator rule: side_of in {0, 1, 2 = separator}. */
void ora_nd_separator(int32_t n, const int32_t *xadj, const int32_t *adjncy, const int32_t *where,
                      int32_t *side_of);
/* Entries of the Cholesky factor (diagonal included) under the ordering iperm. */
int64_t ora_cholesky_nnz(int32_t n, const int32_t *xadj, const int32_t *adjncy, const int32_t *iperm);

#ifdef __cplusplus
}
#endif

#endif
