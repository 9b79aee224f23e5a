/*
 * hp_partition.h — C ABI of the B200 multilevel k-way graph partitioner.
 *
 * Plain C types only: host or device pointers and sizes, int32 CSR, int64 cut.
 * Every entry point returns HP_OK (0) or a negative HP_ERR_* code; nothing in
 * the library calls exit().
 *
 * Reference interface replaced (HunyuanGraph, Elegancejiang/HunyuanSC25):
 *   void hunyuangraph_PartitionGraph(int *nvtxs, int *xadj, int *adjncy,
 *        int *vwgt, int *adjwgt, int *nparts, float *tpwgts, float *ubvec,
 *        int *part)                       hunyuangraph_partitiongraph.h:284-347
 *   prototype                             HunyuanGRAPH.h:57
 * hp_partition() is the reentrant, error-returning form of that call; the
 * legacy symbol hunyuangraph_PartitionGraph() below keeps the exact signature
 * and forwards to it so existing callers relink unchanged.
 *
 * Behavioural differences from the reference entry point (deliberate):
 *   - vwgt/adjwgt are honoured (the reference overwrites both with 1,
 *     hunyuangraph_partitiongraph.h:220-221); NULL means unit weights.
 *   - ubfactor is honoured (the reference hard-codes IMB 1.04,
 *     hunyuangraph_define.h:8, hunyuangraph_GPU_uncoarsen.h:428-437).
 *   - the edge cut is int64 (the reference uses int, hunyuangraph_graph.h:144).
 *   - results are deterministic for a given seed (the reference matching is an
 *     atomicCAS race, hunyuangraph_GPU_match.h:800-861).
 */
#ifndef HP_PARTITION_H
#define HP_PARTITION_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HP_OK                   0
#define HP_ERR_INVALID_ARG     -1  /* bad scalar argument (nparts, ubfactor, NULL pointer) */
#define HP_ERR_INVALID_GRAPH   -2  /* CSR failed validation (range, self loop, weight) */
#define HP_ERR_NOMEM           -3  /* device arena could not be sized or allocated */
#define HP_ERR_CUDA            -4  /* a CUDA runtime call failed */
#define HP_ERR_TIMEOUT         -5  /* a bounded device wait expired (status word set) */
#define HP_ERR_NO_DEVICE       -6  /* no CUDA device / context could not be created */
#define HP_ERR_UNSUPPORTED     -7  /* request outside the supported envelope (e.g. nparts > HP_MAX_PARTS) */
#define HP_ERR_INTERNAL        -8  /* an internal consistency check failed (tracked vs exact cut) */

#define HP_MAX_PARTS        16384  /* gain rows use a dense shared-memory part vector */

#define HP_OPTIONS_VERSION      1

/* Tunables; hp_options_default() fills the defaults listed beside each field. */
typedef struct hp_options {
    int32_t  version;          /* HP_OPTIONS_VERSION                                          */
    int32_t  coarsen_to;       /* 0: reference rule 8k, or max(1024, 2k) if 8k > 1024
                                  (hunyuangraph_partitiongraph.h:298-302)                     */
    int32_t  match_rounds;     /* handshake rounds per level (default 6)                      */
    int32_t  refine_patience;  /* refinement passes without improvement (default 5,
                                  hunyuangraph_GPU_krefine.h:4659)                            */
    int32_t  init_starts;      /* bisection trials per subproblem (default 256)              */
    int32_t  fm_passes;        /* 2-way FM passes per trial (default 10,
                                  hunyuangraph_admin.h:14)                                    */
    int32_t  max_levels;       /* coarsening level cap (default 64)                           */
    int32_t  learned;          /* 0 plain refinement, 1 MLP move proposals, 2 record move log,
                                  3 MLP move proposals judged pass by pass: the plain refiner
                                  takes over for the rest of a level as soon as a learned
                                  pass lowers the exact cut less than the plain pass would
                                  have on the same state (with 1, as soon as a learned pass
                                  does not lower it).  1 and 3 apply to inputs whose largest
                                  degree is at least 16x the mean degree (the power-law
                                  graphs the network is validated on); other inputs are
                                  refined by the plain rule                                   */
    int32_t  validate;         /* 0 none, 1 structural check on the device (default)          */
    int32_t  trace;            /* 1: keep every level for hp_trace_*() (tests)                */
    int32_t  profile;          /* 1: time kernel classes with CUDA events into hp_stats.prof_* */
    int32_t  eager;            /* 0: each level's refinement passes run as one CUDA graph
                                  (device-side WHILE/SWITCH control, default); 1: passes
                                  launched one by one with a host read per pass.  Results
                                  are identical.  With profile = 1 the graphed LP and
                                  gain-rebuild launches are not timed (eager ones are).    */
    uint64_t seed;             /* matching tie-break seed (default 1)                         */
} hp_options;

/* Kernel classes timed when hp_options.profile = 1 (hp_stats.prof_*[class]). */
#define HP_PROF_MATCH     0   /* handshake rounds (proposal + commit)          */
#define HP_PROF_CONTRACT  1   /* coarse-row aggregation + coarse CSR assembly  */
#define HP_PROF_GAIN      2   /* full gain-table build of a level              */
#define HP_PROF_LP        3   /* LP destination selection + afterburner        */
#define HP_PROF_REBUILD   4   /* gain rows of moved vertices' neighbourhoods   */
#define HP_PROF_INIT      5   /* bisection trials                              */
#define HP_PROF_MATCH_MORE 6  /* handshake rounds after the first + fallbacks  */
#define HP_PROF_REBALANCE 7   /* weak/strong rebalance proposals (eager passes) */
#define HP_PROF_APPLY     8   /* move application, exact cut change, pass control
                                 and best-partition copy (eager passes)         */
#define HP_PROF_NCLASS   12   /* array size; classes 9-11 are unused (zero)    */

/* Timing and quality of the last call on a context. */
typedef struct hp_stats {
    int64_t edgecut;           /* exact int64 cut of the returned partition                   */
    int64_t max_excess;        /* max_p (pwgts[p] - maxpwgt[p]); <= 0 means balanced          */
    int64_t tvwgt;             /* total vertex weight                                         */
    int32_t nlevels;           /* coarse levels built (level 0 = input)                       */
    int32_t coarsest_nvtxs;
    int64_t coarsest_nedges;
    int32_t refine_passes;     /* total refinement passes over all levels                     */
    int32_t kernel_launches;   /* kernels this library launched during the call              */
    float   ms_total;          /* device time of the whole call (CUDA events)                 */
    float   ms_coarsen;
    float   ms_init;
    float   ms_uncoarsen;
    float   ms_h2d;            /* host<->device copies inside hp_partition() (0 for _device) */
    float   ms_d2h;
    float   prof_ms[HP_PROF_NCLASS];       /* device time per kernel class (HP_PROF_*)        */
    int64_t prof_bytes[HP_PROF_NCLASS];    /* algorithmic HBM bytes per kernel class: fixed
                                              per-launch terms plus the data-dependent terms
                                              (rows walked, candidates, moves, dirty rows)
                                              counted on the device in profiled calls     */
    int32_t prof_launches[HP_PROF_NCLASS]; /* kernel launches per class                       */
} hp_stats;

typedef struct hp_context hp_context;

void        hp_options_default(hp_options *opt);
const char *hp_strerror(int code);

/* A context owns one device arena and the per-call state; one context per
 * thread (contexts share nothing). device = CUDA ordinal. */
int  hp_context_create(int device, hp_context **out);
void hp_context_destroy(hp_context *ctx);

/* Partition a host CSR graph into nparts parts.
 *   xadj[nvtxs+1], adjncy[xadj[nvtxs]], symmetric, 0-based, no self loops and
 *   no duplicate edges; vwgt[nvtxs] (NULL = 1), adjwgt[xadj[nvtxs]] (NULL = 1);
 *   tpwgts[nparts] target fractions (NULL = uniform); ubfactor >= 1.0.
 * Output: part[nvtxs] in [0, nparts), *edgecut (may be NULL).
 * Replaces hunyuangraph_PartitionGraph (hunyuangraph_partitiongraph.h:284). */
int hp_partition(hp_context *ctx, int32_t nvtxs, const int32_t *xadj,
                 const int32_t *adjncy, const int32_t *vwgt, const int32_t *adjwgt,
                 int32_t nparts, const float *tpwgts, float ubfactor,
                 const hp_options *opt, int32_t *part, int64_t *edgecut);

/* Same, with every array already resident on the context's device (device
 * pointers; vwgt/adjwgt may be NULL) and the work issued on `stream`
 * (cudaStream_t, NULL = legacy default).  d_part is a device pointer. */
int hp_partition_device(hp_context *ctx, int32_t nvtxs, int64_t nedges,
                        const int32_t *d_xadj, const int32_t *d_adjncy,
                        const int32_t *d_vwgt, const int32_t *d_adjwgt,
                        int32_t nparts, const float *tpwgts, float ubfactor,
                        const hp_options *opt, void *stream,
                        int32_t *d_part, int64_t *edgecut);

/* Statistics of the last hp_partition*() call on ctx. */
int hp_last_stats(const hp_context *ctx, hp_stats *out);

/* ---- kernel tuning ---------------------------------------------------------------
 * Speed-only parameters of the kernels: degree-class bounds (which kernel
 * aggregates a row), grid sizes and the accumulator layout.  Every setting in
 * range gives the same partition and cut bit for bit -- each class produces
 * the same canonical rows and proposals -- so a tuning changes time only.
 * The project's autotuner (hunyuansc25_b200/tune.py) searches them per
 * workload and stores the result in a tuning file.  No counterpart in the
 * reference, whose class bounds and block sizes are compile-time constants
 * (hunyuangraph_GPU_match.h, hunyuangraph_GPU_contraction.h). */
typedef struct hp_tuning {
    int32_t match_warp_deg;      /* matching: rows longer than this take a warp  [4, 256]      32 */
    int32_t match_cta_deg;       /* matching: rows longer than this take a CTA   [match_warp_deg, 2^24] 4096 */
    int32_t contract_thread_row; /* contraction: coarse rows up to this many
                                    entries merge in one thread's registers      [8, 32]       32 */
    int32_t contract_warp_row;   /* ... up to this by a warp radix sort           [contract_thread_row, 256] 256 */
    int32_t contract_cta_row;    /* ... up to this by a 256-thread CTA radix sort [contract_warp_row, 4096] 4096;
                                    longer rows: 1024-thread radix up to 12288, dense above */
    int32_t gain_thread_deg;     /* refinement: gain rows of up to this many entries by a
                                    thread or lane segment                        [8, 32]       32 */
    int32_t gain_hub_deg;        /* refinement: rows longer than this are hubs (CTA gain
                                    rows, grid-wide chunked moves and afterburner) [gain_thread_deg, 2^24] 4096 */
    int32_t warp_dense_k;        /* refinement: warp gain rows with shared-memory
                                    accumulators when nparts <= this              [0, 1024]     1024 */
    int32_t grid_ctas_per_sm;    /* grid-stride kernels: CTAs per SM              [1, 32]       8 */
    int32_t dense_sparse_ratio;  /* dense contraction rows: the two-level bitmap when
                                    entries * ratio < bitmap words                [1, 4096]     4 */
    int32_t small_level_n;       /* refinement: levels of at most this many vertices
                                    (and 16x as many adjacency entries, nparts <= 1024)
                                    run all their passes in one CTA; 0 = never    [0, 32768]    4096 */
    int32_t chunk_deg;           /* refinement: the afterburner and move application
                                    split rows longer than this into chunks of 512
                                    entries over the whole grid                  [gain_thread_deg, 2^24] 4096 */
    int32_t trial_cta_n;         /* initial bisection: a recursion depth whose largest
                                    subgraph has at least this many vertices runs
                                    a CTA per trial instead of a warp             [1, 2^24]     512 */
    int32_t contract_smem_cn;    /* contraction: a level with at most this many coarse
                                    vertices merges its long rows in a shared-memory
                                    dense accumulator instead of radix sorts      [0, 49152]    49152 */
    int32_t batch_workers;       /* hp_partition_batch: worker contexts (streams) that
                                    partition graphs concurrently                 [1, 64]       16 */
    int32_t small_match_n;       /* coarsening: levels of at most this many vertices (and
                                    64x as many adjacency entries) are matched by one
                                    CTA; 0 = never                               [0, 8192]     8192 */
    int32_t contract_hybrid;     /* contraction: on levels with more coarse vertices than
                                    contract_smem_cn and at most 131072, rows longer than
                                    contract_warp_row accumulate their ids below 32768 in
                                    a shared-memory dense accumulator and radix-sort the
                                    rest (1), or radix-sort every entry (0)      [0, 1]        1 */
    int32_t apply_chunk_deg;     /* refinement: move application splits rows longer than
                                    this into chunks of 512 entries over the whole grid
                                    (chunk_deg is the afterburner's)     [gain_thread_deg, 2^24] 4096 */
    int32_t pdl;                 /* launches: each kernel of a call may be launched while the
                                    previous one drains and waits for it on the device
                                    (programmatic dependent launch) (1), or after it (0)
                                                                                  [0, 1]        1 */
    int32_t graph_passes;        /* refinement: each level's pass loop as one CUDA graph with
                                    device-side control (1), or its passes launched one by one
                                    (0); hp_options.eager = 1 forces the latter.  Results are
                                    identical                                     [0, 1]        1 */
    int32_t reserved[4];         /* zero */
} hp_tuning;

void hp_tuning_default(hp_tuning *t);
/* Validates and installs a tuning on ctx (batch workers inherit it); returns
 * HP_ERR_INVALID_ARG, with a message on stderr, for a value out of range. */
int hp_context_set_tuning(hp_context *ctx, const hp_tuning *t);
int hp_context_get_tuning(const hp_context *ctx, hp_tuning *t);

/* ---- level trace (opt.trace = 1), for parity checks of every level ----------- */
#define HP_TRACE_XADJ         0   /* int32[n+1]  CSR of level l                      */
#define HP_TRACE_ADJNCY       1   /* int32[m]                                        */
#define HP_TRACE_ADJWGT       2   /* int32[m]                                        */
#define HP_TRACE_VWGT         3   /* int32[n]                                        */
#define HP_TRACE_MATCH        4   /* int32[n]  mate (self when unmatched), l < last  */
#define HP_TRACE_CMAP         5   /* int32[n]  coarse id,                  l < last  */
#define HP_TRACE_WHERE_START  6   /* int32[n]  partition entering refinement of l:
                                     initial partition (coarsest) or projection      */
#define HP_TRACE_WHERE_FINAL  7   /* int32[n]  partition after refinement of l        */

int hp_trace_nlevels(const hp_context *ctx);
int hp_trace_level(const hp_context *ctx, int level, int32_t *nvtxs, int64_t *nedges,
                   int64_t *cut_start, int64_t *cut_final);
int hp_trace_copy(const hp_context *ctx, int level, int what, int32_t *dst, int64_t count);

/* ---- batched partition of many independent graphs ------------------------------
 * Graph g has vertices [vtxdist[g], vtxdist[g+1]) and adjacency entries
 * [edgedist[g], edgedist[g+1]) of the concatenated host arrays; xadj is the
 * concatenation of the per-graph xadj arrays (each starting at 0, length n_g+1,
 * so xadj has vtxdist[G] + G entries); adjncy ids are local to their graph.
 * nparts[g], ubfactor[g] per graph; part is concatenated like vwgt. */
int hp_partition_batch(hp_context *ctx, int32_t ngraphs, const int64_t *vtxdist,
                       const int64_t *edgedist, const int32_t *xadj,
                       const int32_t *adjncy, const int32_t *vwgt,
                       const int32_t *adjwgt, const int32_t *nparts,
                       const float *ubfactor, const hp_options *opt,
                       int32_t *part, int64_t *edgecut);

/* ---- learned move proposals --------------------------------------------------------
 * No counterpart in the reference (its refinement has no learned component).
 * An MLP 8 -> 32 -> 32 -> 1 scores each label-propagation candidate from eight
 * integer-derived features (normalised gain, own/best connectivity fractions,
 * adjacent-part count, log degree, target/own part slack, finest-level flag).
 * With hp_options.learned = 1, candidates scoring below `threshold` are not
 * proposed; the exact integer afterburner and balance rules still decide
 * every move, and a level returns to the plain rule as soon as a learned pass
 * fails to lower the exact cut.  Inference runs on BF16 tensor cores with FP32
 * accumulation inside the LP kernel; training is FP32 (forward, backward,
 * Adam) on the device.  Parameters are HP_MLP_NPARAM floats:
 * W1[32][8], b1[32], W2[32][32], b2[32], w3[32], b3. */
#define HP_MLP_NPARAM 1377
int hp_mlp_set_params(hp_context *ctx, const float *params, int32_t count, float threshold);
int hp_mlp_get_params(hp_context *ctx, float *params, int32_t count);
/* Mean BCE-with-logits loss and its gradient over n samples (device arrays
 * d_x[n][8], d_y[n] in {0,1}); grad and loss are host outputs. */
int hp_mlp_loss_grad(hp_context *ctx, const float *d_x, const float *d_y, int64_t n, float *grad,
                     float *loss);
/* Mini-batch Adam on the device; d_perm (nullable) orders the samples. */
int hp_mlp_train(hp_context *ctx, const float *d_x, const float *d_y, const int32_t *d_perm, int64_t n,
                 int32_t epochs, int32_t batch, float lr, float *final_loss);
/* Logits of n samples (device arrays); tensor_cores = 1 uses the BF16 MMA path
 * of the LP kernel, 0 the FP32 path. */
int hp_mlp_infer(hp_context *ctx, const float *d_x, int64_t n, float *d_out, int32_t tensor_cores);
/* Move log of the plain refiner (hp_options.learned = 2): every LP candidate's
 * features, labelled 1 when the afterburner accepted the move and the vertex
 * ends its level in that part. */
int     hp_movelog_enable(hp_context *ctx, int64_t capacity);
int64_t hp_movelog_count(hp_context *ctx);
int     hp_movelog_copy(hp_context *ctx, float *features, float *labels, int64_t count);
int     hp_movelog_reset(hp_context *ctx);

/* ---- nested-dissection ordering -------------------------------------------------
 * Fill-reducing ordering of a symmetric sparsity pattern (host CSR as for
 * hp_partition; vwgt may be NULL; edge weights are not used).  Replaces the
 * reference's ReorderGraph / NestedBisection
 * (mygp_0.9.9_test_initpartition/reordergraph.h:177-306): a vertex separator
 * of every subgraph takes the highest numbers of the subgraph's range, the
 * two sides are ordered recursively (left side first) and subgraphs of at
 * most 120 vertices, or without edges, are ordered by an exact minimum-degree
 * elimination (the reference's MMD_Order, whose source is not in its tree).
 * Separators come from 2-way partitions by this library (imbalance 1.05, the
 * options in opt, NULL = defaults; coarsening to 128 vertices when
 * opt->coarsen_to is 0), so the ordering is deterministic.  Output:
 * iperm[old] = new and, when perm is not NULL, perm[new] = old (METIS_NodeND's
 * convention; the reference's reflect array is iperm).  hp_last_stats reports
 * the recursion depths in nlevels and the 2-way partitions in refine_passes. */
int hp_node_nd(hp_context *ctx, int32_t nvtxs, const int32_t *xadj, const int32_t *adjncy,
               const int32_t *vwgt, const hp_options *opt, int32_t *perm, int32_t *iperm);

/* ---- device primitives (device pointers, issued on `stream`) ------------------- */
/* Exclusive int32 prefix sum, single-pass decoupled look-back.  Writes n+1
 * outputs (out[n] = total); in == out is allowed.  Replaces prefixsum()
 * (hunyuangraph_GPU_prefixsum.h:141-188), which is inclusive and recursive. */
int hp_scan_exclusive_i32(hp_context *ctx, const int32_t *d_in, int32_t *d_out,
                          int64_t n, void *stream);

/* Exclusive int32 prefix sum that allocates nothing: same result as
 * hp_scan_exclusive_i32, without a context.  No counterpart in the reference
 * (its prefix sum draws scratch from its device pool).
 *
 * For callers that cannot call cudaMalloc: code whose device memory is owned
 * by a host framework's caching allocator that admits no outside allocations,
 * and latency-critical pipelines that cannot take cudaMalloc's implicit device
 * synchronisation.  The scan's look-back scratch is a fixed array in the
 * library's device image (about 128 KiB, held by every GPU that loads the
 * library until the process exits), so n is limited to
 * HP_SCAN_NOALLOC_MAX_N; larger n returns HP_ERR_UNSUPPORTED with a message
 * on stderr.  The caller still passes d_in and d_out (n + 1 entries).
 *   - Every call looks up the array's device address with the caller's device
 *     and context current (so a cudaDeviceReset or a non-primary context is
 *     handled); the lookup allocates nothing once the library's device code is
 *     loaded, which the first call in a context does: make that first call
 *     before any stream capture.
 *   - A CUDA error already pending from the caller's earlier work is not
 *     cleared: the call returns HP_ERR_CUDA without launching anything.
 *   - Runs on the calling thread's current device and `stream`, and returns
 *     after the scan completed (it reads the status word back).
 *   - All calls share the one array: calls that overlap on the GPU (other
 *     streams, other threads) race and must be serialised by the caller. */
#define HP_SCAN_NOALLOC_MAX_N ((int64_t)1 << 26)
int hp_scan_exclusive_i32_noalloc(const int32_t *d_in, int32_t *d_out, int64_t n, void *stream);

/* Exact int64 edge cut of a device-resident partition.  Replaces
 * compute_edgecut_gpu (hunyuangraph_graph.h:230-268). */
int hp_edgecut_device(hp_context *ctx, int32_t nvtxs, const int32_t *d_xadj,
                      const int32_t *d_adjncy, const int32_t *d_adjwgt,
                      const int32_t *d_where, void *stream, int64_t *cut);

/* Test of the failure path of the bounded device waits: runs the scans'
 * look-back wait against a predecessor flag that nothing sets.  The wait gives
 * up after its spin limit (2^22 polls) and the call returns what a
 * partition would: HP_ERR_TIMEOUT.  The status word is cleared afterwards, so
 * the context stays usable.  No counterpart in the reference (its one device
 * spin-wait, hunyuangraph_GPU_match.h:350-358, is unbounded). */
int hp_test_wait_expiry(hp_context *ctx);

/* Test of the arena's grow-and-retry path.  bytes > 0 frees the context's
 * arena and makes the next hp_partition / hp_partition_device call start with
 * an arena of exactly `bytes` instead of the size estimated from (n, m); an
 * attempt that runs out launches nothing more, unwinds with HP_ERR_NOMEM and
 * restarts with twice the arena, at most four attempts in all, after which
 * the call returns HP_ERR_NOMEM.  bytes == 0 clears a pending override.
 * hp_test_arena_restarts returns how many restarts the last partition call
 * made.  The reference prints and calls exit() when its device memory
 * manager runs out (hunyuangraph_GPU_memory.h:117-121). */
int hp_test_arena_first(hp_context *ctx, int64_t bytes);
int hp_test_arena_restarts(hp_context *ctx);

/* ---- legacy drop-in ------------------------------------------------------------
 * Identical signature to the reference (hunyuangraph_partitiongraph.h:284).
 * Uses a process-wide context on device 0 and hp_options_default(); ubvec[0]
 * is the imbalance factor.  On error every part[] entry is set to -1 and a
 * message goes to stderr (the reference prints and calls exit()). */
void hunyuangraph_PartitionGraph(int *nvtxs, int *xadj, int *adjncy, int *vwgt,
                                 int *adjwgt, int *nparts, float *tpwgts,
                                 float *ubvec, int *part);

#ifdef __cplusplus
}
#endif

#endif /* HP_PARTITION_H */
