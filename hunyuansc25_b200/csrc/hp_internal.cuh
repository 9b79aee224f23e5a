// hp_internal.cuh — context, device arena and the interfaces between the kernel files.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <utility>
#include <vector>

#include "hp_common.cuh"

// One coarsening level resident in the arena.
struct HpLevel {
    int32_t n = 0;
    int64_t m = 0;
    int32_t *xadj = nullptr, *adjncy = nullptr, *adjwgt = nullptr, *vwgt = nullptr;
    int32_t *match = nullptr, *cmap = nullptr;        // set when a coarser level exists
    int32_t *where = nullptr;                          // working partition
    int32_t *where_start = nullptr, *where_final = nullptr;  // trace copies
    int64_t cut_start = 0, cut_final = 0;
};

struct hp_context {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;   // stream of the current call
    cudaStream_t own_stream = nullptr;

    // Device arena: one allocation, used as a two-ended stack.  The low end
    // holds the level chain and per-call state (lalloc), the high end holds
    // temporaries released in LIFO order (ralloc).
    char *arena = nullptr;
    size_t arena_cap = 0, lo = 0, hi = 0;
    bool oom = false;
    size_t arena_first = 0;     // hp_test_arena_first: size of the next call's first attempt
    int arena_restarts = 0;     // restarts of the last partition call after running out

    // Small fixed device block: status word + scalar slots, and a pinned
    // host mirror for blocking scalar reads.
    unsigned *d_status = nullptr;
    unsigned long long *d_scal = nullptr;   // HP_NSCAL slots
    long long *h_pin = nullptr;             // HP_NSCAL slots, pinned

    cudaEvent_t ev[8] = {};
    int launches = 0;

    // Epoch look-back region of the single-pass kernels (hp_common.cuh): tile
    // words (only those kernels write them) and the tile counter / epoch block.
    unsigned long long *lb_status = nullptr;
    int64_t lb_cap = 0;
    hp::LbCtl *lb_ctl = nullptr;

    // Kernel-class profiler (opt.profile): event pairs resolved at the end of a call.
    struct ProfRec { int cls; int ev0, ev1; int64_t bytes; int launches; };
    std::vector<cudaEvent_t> prof_events;
    std::vector<ProfRec> prof_recs;
    int prof_next = 0;
    bool prof_suspended = false;   // set while launches are captured into a CUDA graph
    // Device-side byte counts of the data-dependent terms of the class byte
    // models (HP_PROF_NCLASS slots after the scalar slots), added by the
    // profile-only counting kernels and folded into stats.prof_bytes.
    unsigned long long *d_profb = nullptr;

    hp_stats stats = {};

    // move-scoring MLP (hp_mlp.cu): params, gradient, Adam moments
    float *mlp_params = nullptr, *mlp_grad = nullptr, *mlp_m = nullptr, *mlp_v = nullptr;
    float *mlp_scratch = nullptr;   // per-sample gradient rows of a training chunk
    float mlp_threshold = 0.0f;
    bool mlp_ready = false;
    // move log recorded by the plain refiner (opt.learned = 2)
    float *log_x = nullptr, *log_y = nullptr;
    int32_t *log_v = nullptr, *log_d = nullptr, *log_acc = nullptr;
    unsigned long long *log_count = nullptr;
    int64_t log_cap = 0;

    // Graph reaper: executable graphs are released by a background thread once
    // the event recorded after their last launch has completed, so that their
    // destruction never delays the stream (hp_graph_retire, hp_api.cu).
    struct Retired {
        cudaEvent_t done;
        std::vector<std::pair<cudaGraph_t, cudaGraphExec_t>> graphs;
    };
    std::thread reaper;
    std::mutex reaper_mu;
    std::condition_variable reaper_cv;
    std::deque<Retired> reaper_q;
    bool reaper_stop = false;

    hp_tuning tune = {};                 // kernel tuning (speed only), hp_context_set_tuning
    std::vector<hp_context *> workers;   // batch worker contexts (own streams and arenas)
    std::vector<HpLevel> levels;
    bool trace_valid = false;
    bool weight_check = false;           // total edge weight >= 2^31: contractions check pair bounds
    bool learned_skewed = false;         // the input's degrees are skewed enough for the learned proposals
    hp_options opt = {};
};

// Upper bounds of the kernel tuning: the capacities the kernels are compiled for.
constexpr int HP_TUNE_THREAD_ROW_MAX = 32;       // register sorting networks (rows per thread)
constexpr int HP_TUNE_WARP_ROW_MAX = 256;        // contract_warp_radix_kernel's shared buffers
constexpr int HP_TUNE_CTA_ROW_MAX = 4096;        // contract_cta_radix_kernel<256, 4096>
constexpr int HP_TUNE_WARP_DENSE_K_MAX = 1024;   // gain_bigwarp_kernel's shared accumulators
constexpr int HP_TUNE_DEG_MAX = 1 << 24;
constexpr int HP_TUNE_SMALL_LEVEL_MAX = 32768;   // refine_small_kernel's staged prefix weights
constexpr int HP_TUNE_SMALL_MATCH_MAX = 8192;    // match_small_kernel's shared-memory state
constexpr int HP_TUNE_SMEM_CN_MAX = 49152;       // shared-memory dense accumulator of the contraction
constexpr int64_t HP_LEARNED_SKEW = 16;          // learned proposals: max degree / mean degree of the input

#define HP_NSCAL 64
#define HP_ALIGN 256

// ---- arena -------------------------------------------------------------------
inline void *hp_lalloc(hp_context *c, size_t bytes)
{
    size_t b = (bytes + HP_ALIGN - 1) / HP_ALIGN * HP_ALIGN;
    if (b == 0) b = HP_ALIGN;
    if (c->lo + b > c->hi) { c->oom = true; return nullptr; }
    void *p = c->arena + c->lo;
    c->lo += b;
    return p;
}

inline void *hp_ralloc(hp_context *c, size_t bytes)
{
    size_t b = (bytes + HP_ALIGN - 1) / HP_ALIGN * HP_ALIGN;
    if (b == 0) b = HP_ALIGN;
    if (c->hi < c->lo + b) { c->oom = true; return nullptr; }
    c->hi -= b;
    return c->arena + c->hi;
}

template <class T> inline T *lalloc_t(hp_context *c, int64_t n) { return (T *)hp_lalloc(c, sizeof(T) * (size_t)(n > 0 ? n : 1)); }
template <class T> inline T *ralloc_t(hp_context *c, int64_t n) { return (T *)hp_ralloc(c, sizeof(T) * (size_t)(n > 0 ? n : 1)); }

#define HP_CHECK_OOM(c) do { if ((c)->oom) return HP_ERR_NOMEM; } while (0)

// Launch of a kernel on the context's stream.  With hp_tuning.pdl the launch is a
// programmatic dependent of the stream's previous kernel: the hardware may start
// it while that kernel drains (the launch latency overlaps its tail), and every
// kernel of the library begins with hp::pdl_wait(), so nothing it reads or writes
// is touched before the previous kernel has completed -- the order of effects is
// exactly that of a plain launch.
template <class... P, class... A>
inline cudaError_t hp_launch_kernel(const hp_context *c, void (*kernel)(P...), unsigned grid, unsigned block,
                                    size_t smem, A &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = c->tune.pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

// Count and check every kernel launch.  Once the arena has run out nothing more is
// launched (a pointer allocated after that is null): the call unwinds with
// HP_ERR_NOMEM and partition_common retries with a larger arena.
#define HP_LAUNCH(ctx, kernel, grid, block, smem, ...)                                      \
    do {                                                                                    \
        if ((ctx)->oom) return HP_ERR_NOMEM;                                                \
        if ((grid) > 0) {                                                                   \
            cudaError_t e__ = hp_launch_kernel((ctx), kernel, (unsigned)(grid), (unsigned)(block), \
                                               (size_t)(smem), __VA_ARGS__);                \
            (ctx)->launches++;                                                              \
            if (e__ == cudaSuccess) e__ = cudaGetLastError();                               \
            if (e__ != cudaSuccess) {                                                       \
                fprintf(stderr, "hp: launch %s failed: %s\n", #kernel, cudaGetErrorString(e__)); \
                return HP_ERR_CUDA;                                                         \
            }                                                                               \
        }                                                                                   \
    } while (0)

// ---- kernel-class profiler ------------------------------------------------------
// Usage: int t = hp_prof_begin(c); ...launches...; hp_prof_end(c, t, HP_PROF_X, bytes);
int hp_prof_begin(hp_context *c);
void hp_prof_end(hp_context *c, int token, int cls, int64_t bytes);
// Algorithmic bytes of an interval that are known only after it was closed.
void hp_prof_add_bytes(hp_context *c, int token, int64_t bytes);
// The device byte counter of class cls while the profiler records launches
// (opt.profile and not capturing), else nullptr: callers launch their counting
// kernels only when it is set, after the class's hp_prof_end, so that the
// counting is not part of the class's time.
unsigned long long *hp_prof_counter(hp_context *c, int cls);
void hp_prof_resolve(hp_context *c);

// Hands graphs whose last launch is enqueued on c->stream to the reaper thread
// (started on first use); they are destroyed once that work has completed.
int hp_graph_retire(hp_context *c, std::vector<std::pair<cudaGraph_t, cudaGraphExec_t>> &&graphs);

// Ensures room for `tiles` look-back words (called at the start of a call,
// before any launch that could use them).
int hp_lb_reserve(hp_context *c, int64_t tiles);

// Blocking read of nbytes from device into the pinned mirror, then dst.
int hp_read_scalars(hp_context *c, const void *d_src, size_t nbytes, void *dst);
// Status word check after a phase (spin timeouts, bad graph).
int hp_check_status(hp_context *c);

// ---- primitives (hp_scan.cu) --------------------------------------------------
// Exclusive scan, n+1 outputs (out[n] = total). in == out allowed.
int hp_scan_excl(hp_context *c, const int32_t *in, int32_t *out, int64_t n);
// out[i] = base + i for i < n (iota)
int hp_fill_i32(hp_context *c, int32_t *p, int64_t n, int32_t value);
int hp_iota_i32(hp_context *c, int32_t *p, int64_t n);
// Stable compaction of indices i < n with flag[i] != 0 into out; count -> *d_count.
int hp_compact_flags(hp_context *c, const int32_t *flags, int64_t n, int32_t *out, int32_t *d_count);
// Stable LSD radix sort of `bound` slots (count on device) by the low key_bits
// bits of keys; ping-pongs with tkeys/tvals.  *in_tmp tells which pair holds
// the result.
int hp_sort_pairs(hp_context *c, int32_t *keys, int32_t *vals, int32_t *tkeys, int32_t *tvals,
                  int64_t bound, const int32_t *d_count, int key_bits, bool *in_tmp);
// Exact edge cut (int64) into *d_cut (device, accumulated; caller zeroes).
int hp_edgecut_launch(hp_context *c, int32_t n, int64_t m, const int32_t *xadj, const int32_t *adjncy,
                      const int32_t *adjwgt, const int32_t *where, unsigned long long *d_cut);

// ---- coarsening (hp_coarsen.cu) -----------------------------------------------
// Builds levels[1..] from levels[0]; returns HP_OK and fills c->levels.
int hp_coarsen(hp_context *c, int32_t coarsen_to, int64_t maxvwgt);
// Sets HP_STATUS_WEIGHT_RANGE when a vertex of g has a weighted degree of 2^31
// or more (the input level's check when its total edge weight reaches 2^31).
int hp_check_weight_range(hp_context *c, const HpLevel &g);

// ---- initial partition (hp_initpart.cu) ------------------------------------------
int hp_initial_partition(hp_context *c, HpLevel &g, int32_t nparts, const int64_t *h_tw,
                         int64_t ub2_fx, int32_t *d_where);

// ---- refinement (hp_refine.cu) --------------------------------------------------
int hp_uncoarsen(hp_context *c, int32_t nparts, const int64_t *h_opt, const int64_t *h_maxp);
// One-time kernel attributes (dynamic shared memory above 48 KB).
// Worker contexts of a context (own streams and arenas) for independent
// partitions run concurrently (hp_partition_batch, hp_node_nd): at least
// nworkers of them, with the context's tuning.
int hp_ensure_workers(hp_context *ctx, int nworkers);

int hp_refine_init();
int hp_initpart_init();
int hp_coarsen_init();
int hp_mlp_ensure(hp_context *c);

// ---- targets shared with the host driver -----------------------------------------
void hp_part_targets(int64_t tvwgt, int32_t nparts, const float *tpwgts, float ubfactor,
                     int64_t *opt, int64_t *maxp);
int64_t hp_bisect_ub_fx(float ubfactor, int32_t nparts);
