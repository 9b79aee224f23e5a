// hp_api.cu — C ABI (include/hp_partition.h): contexts, the V-cycle driver,
// statistics, the level trace and the legacy hunyuangraph_PartitionGraph shim.
//
// Reference entry point: hunyuangraph_PartitionGraph
// (hunyuangraph_partitiongraph.h:284-347) and the V-cycle
// hunyuangraph_kway_partition (:13-149).  The reference allocates 80 % of the
// free device memory at every call (hunyuangraph_GPU_memory.h:42-76), forces
// unit weights and exits on error; here a context keeps one arena sized from
// (n, m) and grown on demand, the caller's weights are used, and every failure
// is an error code.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <thread>

#include "hp_internal.cuh"

#define HP_API extern "C" __attribute__((visibility("default")))

namespace {

// Structural validation: vertex checks per thread, adjacency checks in
// edge-parallel tiles of VE_TILE entries, so hub rows cost no more than their
// share of the array.  The owner row of every entry of a tile comes from
// hp::tile_owners (row-start markers and a shared-memory max-scan).
// Also records the largest degree (*maxdeg, for the weight-range gate).
__global__ void validate_vertices_kernel(int32_t n, int64_t m, const int32_t *__restrict__ xadj,
                                         const int32_t *__restrict__ vwgt, unsigned *status,
                                         unsigned long long *maxdeg)
{
    hp::pdl_wait();
    bool bad = false;
    int32_t dmax = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int32_t b = xadj[v], e = xadj[v + 1];
        if (b > e || b < 0 || e > m) bad = true;
        if (vwgt && vwgt[v] < 0) bad = true;
        dmax = max(dmax, e - b);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (xadj[0] != 0 || xadj[n] != m)) bad = true;
    if (bad) atomicOr(status, HP_STATUS_BAD_GRAPH);
    dmax = hp::warp_max(dmax);
    if ((threadIdx.x & 31) == 0 && dmax > 0) atomicMax(maxdeg, (unsigned long long)dmax);
}

constexpr int VE_THREADS = 256, VE_ITEMS = 16, VE_TILE = VE_THREADS * VE_ITEMS;

// Antisymmetric fingerprint of a directed weighted entry (row v, neighbour u,
// weight w): +h for v < u, -h for v > u, with h a hash of the undirected edge
// (min, max, w).  Over a symmetric multiset of entries (every (v, u, w) with
// its (u, v, w)) the terms cancel and the sum is 0 mod 2^64; a missing reverse
// entry, or a weight that differs between the two directions, leaves a
// non-zero sum except with probability about 2^-64.
__device__ __forceinline__ unsigned long long sym_term(int32_t v, int32_t u, int32_t w)
{
    const uint32_t lo = (uint32_t)min(v, u), hi = (uint32_t)max(v, u);
    const unsigned long long h =
        hp::mix64((((uint64_t)lo << 32) | hi) + (uint64_t)(uint32_t)w * 0x9E3779B97F4A7C15ull);
    return v < u ? h : 0ull - h;
}

// Runs after validate_vertices_kernel succeeded (xadj monotone, xadj[0] = 0,
// xadj[n] = m, so every entry has exactly one owner row).  Besides the range,
// self-loop and weight checks of every entry it accumulates:
//   sums[0]           the symmetry fingerprint (0 for a symmetric adjacency);
//   sums[1]           the largest edge weight (atomic max);
//   sums[2]           the total edge weight (int64);
//   sums[3]           the entries of the rows that are not strictly increasing
//                     (unsorted[v] = 1 for those rows), the only rows that
//                     can hold a duplicate neighbour.
__global__ void __launch_bounds__(VE_THREADS)
validate_edges_kernel(int32_t n, int64_t m, const int32_t *__restrict__ xadj,
                      const int32_t *__restrict__ adjncy, const int32_t *__restrict__ adjwgt, unsigned *status,
                      int32_t *__restrict__ unsorted, unsigned long long *sums)
{
    hp::pdl_wait();
    __shared__ int32_t owner[VE_TILE];
    __shared__ int32_t s_warp[VE_THREADS / 32];
    __shared__ int32_t s_v0;
    if (*status & HP_STATUS_BAD_GRAPH) return;   // uniform over the grid
    bool bad = false;
    unsigned long long fp = 0;
    long long wsum = 0, uent = 0;
    int32_t wmax = 0;
    for (int64_t tb = (int64_t)blockIdx.x * VE_TILE; tb < m; tb += (int64_t)gridDim.x * VE_TILE) {
        const int64_t te = tb + VE_TILE < m ? tb + VE_TILE : m;
        hp::tile_owners<VE_THREADS, VE_ITEMS>(xadj, n, tb, te, owner, s_warp, &s_v0);
        // checks, coalesced over the tile
        for (int64_t j = tb + threadIdx.x; j < te; j += VE_THREADS) {
            const int32_t v = owner[j - tb];
            const int32_t u = adjncy[j];
            const int32_t w = adjwgt ? adjwgt[j] : 1;
            if (u < 0 || u >= n || u == v) bad = true;
            if (w <= 0) bad = true;
            wsum += w;
            wmax = max(wmax, w);
            fp += sym_term(v, u, w);
            // the next entry of the same row (within the tile, or across its end)
            const int64_t jn = j + 1;
            const bool same = jn < te ? owner[jn - tb] == v : (jn < m && xadj[v + 1] > jn);
            if (same && adjncy[jn] <= u && atomicExch(&unsorted[v], 1) == 0) uent += xadj[v + 1] - xadj[v];
        }
        __syncthreads();   // owner[] is rebuilt for the next tile
    }
    if (bad) atomicOr(status, HP_STATUS_BAD_GRAPH);
    hp::block_add_to<VE_THREADS>((long long)fp, &sums[0]);
    hp::block_add_to<VE_THREADS>(wsum, &sums[2]);
    wmax = hp::warp_max(wmax);
    if ((threadIdx.x & 31) == 0 && wmax > 0) atomicMax(&sums[1], (unsigned long long)wmax);
    hp::block_add_to<VE_THREADS>(uent, &sums[3]);
}

// Duplicate neighbours in the rows validate_edges_kernel found unsorted: every
// (row, neighbour) key of those rows goes into an open-addressing hash table
// (linear probing, 64-bit keys, at most half full, all ones = empty); a key
// that is already present is a duplicate edge.  One warp per row.
__global__ void __launch_bounds__(256)
dup_check_kernel(int32_t n, const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                 const int32_t *__restrict__ unsorted, unsigned long long *table, uint64_t mask, unsigned *status)
{
    hp::pdl_wait();
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    bool dup = false;
    for (int64_t v = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nwarps) {
        if (!unsorted[v]) continue;
        const int32_t e = xadj[v + 1];
        for (int32_t j = xadj[v] + lane; j < e; j += 32) {
            const unsigned long long key = ((unsigned long long)(uint32_t)v << 32) | (uint32_t)adjncy[j];
            uint64_t h = hp::mix64(key) & mask;
            for (uint64_t probe = 0; probe <= mask; probe++) {
                const unsigned long long prev = atomicCAS(&table[h], ~0ull, key);
                if (prev == ~0ull) break;
                if (prev == key) { dup = true; break; }
                h = (h + 1) & mask;
            }
        }
    }
    if (dup) atomicOr(status, HP_STATUS_BAD_GRAPH);
}

__global__ void sum_kernel(int64_t n, const int32_t *__restrict__ a, unsigned long long *out)
{
    hp::pdl_wait();
    long long acc = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += a[i];
    hp::block_add_to<256>(acc, out);
}

__global__ void final_pw_kernel(int32_t n, const int32_t *__restrict__ where, const int32_t *__restrict__ vwgt,
                                unsigned long long *pw, int32_t k, unsigned *status)
{
    hp::pdl_wait();
    extern __shared__ unsigned long long fpw[];
    const bool use_s = k <= 2048;
    if (use_s) {
        for (int i = threadIdx.x; i < k; i += blockDim.x) fpw[i] = 0;
        __syncthreads();
    }
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int32_t p = where[v];
        if (p < 0 || p >= k) { atomicOr(status, HP_STATUS_OVERFLOW); continue; }
        if (use_s) atomicAdd(&fpw[p], (unsigned long long)vwgt[v]);
        else atomicAdd(&pw[p], (unsigned long long)vwgt[v]);
    }
    if (use_s) {
        __syncthreads();
        for (int i = threadIdx.x; i < k; i += blockDim.x)
            if (fpw[i]) atomicAdd(&pw[i], fpw[i]);
    }
}

__global__ void fill_ones_kernel(int64_t n, int32_t *p)
{
    hp::pdl_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = 1;
}

inline unsigned gsz(hp_context *c, int64_t n)
{
    int64_t g = (n + 255) / 256;
    int64_t cap = (int64_t)c->sm_count * 16;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, cap));
}

int ensure_arena(hp_context *c, size_t bytes)
{
    if (c->arena && c->arena_cap >= bytes) return HP_OK;
    if (c->arena) {
        cudaFree(c->arena);
        c->arena = nullptr;
        c->arena_cap = 0;
    }
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return HP_ERR_NOMEM;
    }
    c->arena = (char *)p;
    c->arena_cap = bytes;
    return HP_OK;
}

void reset_arena(hp_context *c)
{
    c->lo = 0;
    c->hi = c->arena_cap;
    c->oom = false;
    c->levels.clear();
    c->trace_valid = false;
}

// The level chain holds sum_l (8 m_l + ~20 n_l) bytes.  On power-law graphs the
// adjacency barely shrinks for the first levels (R-MAT: sum_l m_l is about
// 7-9 m_0, against 3 m_0 on a 3-D grid and 1.7 m_0 on a geometric graph), so
// the estimate covers 8 bytes x 8 m_0 plus the uncoarsening's gain rows and
// work arrays; an arena that still runs out is doubled and the call restarts.
size_t estimate_arena(int64_t n, int64_t m)
{
    return (size_t)(160 * n + 80 * m) + ((size_t)256 << 20);
}

int32_t default_coarsen_to(int32_t nparts)
{
    int32_t thr = nparts * 8;   // hunyuangraph_partitiongraph.h:298-302
    if (thr > 1024) thr = std::max(1024, nparts * 2);
    return thr;
}

// The V-cycle on the level-0 graph already placed in c->levels[0].
int vcycle(hp_context *c, int32_t nparts, const float *tpwgts, float ubfactor, int64_t *edgecut)
{
    HpLevel &g0 = c->levels[0];
    const int32_t n = g0.n;
    hp_stats &st = c->stats;
    unsigned long long *sc = c->d_scal;

    // scalar slots: [0] total vertex weight, [1] symmetry fingerprint, [2]
    // largest edge weight, [3] total edge weight, [4] entries of unsorted rows,
    // [5] largest degree
    const size_t vmark = c->hi;
    HP_CUDA(cudaMemsetAsync(sc, 0, sizeof(unsigned long long) * 6, c->stream));
    int32_t *unsorted = nullptr;
    if (c->opt.validate) {
        unsorted = ralloc_t<int32_t>(c, n);
        HP_CHECK_OOM(c);
        HP_CUDA(cudaMemsetAsync(unsorted, 0, sizeof(int32_t) * (size_t)n, c->stream));
        HP_LAUNCH(c, validate_vertices_kernel, gsz(c, n), 256, 0, n, g0.m, g0.xadj, g0.vwgt, c->d_status, &sc[5]);
        HP_LAUNCH(c, validate_edges_kernel,
                  (unsigned)std::max<int64_t>(1, std::min<int64_t>((g0.m + VE_TILE - 1) / VE_TILE,
                                                                   (int64_t)c->sm_count * 8)),
                  VE_THREADS, 0, n, g0.m, g0.xadj, g0.adjncy,
                  g0.adjwgt, c->d_status, unsorted, &sc[1]);
    } else {
        HP_LAUNCH(c, sum_kernel, gsz(c, g0.m), 256, 0, g0.m, g0.adjwgt, &sc[3]);
    }
    HP_LAUNCH(c, sum_kernel, gsz(c, n), 256, 0, (int64_t)n, g0.vwgt, &sc[0]);
    long long vs[6] = {};
    HP_TRY(hp_read_scalars(c, &sc[0], sizeof(vs), vs));
    HP_TRY(hp_check_status(c));
    if (c->opt.validate) {
        if (vs[1] != 0) {
            fprintf(stderr, "hp: invalid graph: the adjacency is not symmetric (an entry (v, u, w) without its "
                            "reverse (u, v, w))\n");
            return HP_ERR_INVALID_GRAPH;
        }
        if (vs[4] > 0) {
            // some rows are not strictly increasing: look for duplicate neighbours in them
            uint64_t cap = 1024;
            while (cap < 2 * (uint64_t)vs[4]) cap <<= 1;
            unsigned long long *table = ralloc_t<unsigned long long>(c, (int64_t)cap);
            HP_CHECK_OOM(c);
            HP_CUDA(cudaMemsetAsync(table, 0xff, sizeof(unsigned long long) * cap, c->stream));
            HP_LAUNCH(c, dup_check_kernel, gsz(c, (int64_t)n * 32), 256, 0, n, g0.xadj, g0.adjncy, unsorted, table,
                      cap - 1, c->d_status);
            if (hp_check_status(c) == HP_ERR_INVALID_GRAPH) {
                fprintf(stderr, "hp: invalid graph: a row lists the same neighbour twice\n");
                return HP_ERR_INVALID_GRAPH;
            }
        }
    }
    c->hi = vmark;
    const long long tv = vs[0];
    if (tv >= INT32_MAX) return HP_ERR_UNSUPPORTED;
    st.tvwgt = tv;
    // Coarse edge weights, gain-row connectivities and bisection gains are
    // int32.  Each is a sum of input edge weights, so when the total edge
    // weight is below 2^31 none can wrap; otherwise the input's rows and every
    // coarse row the contraction builds must have a weighted degree below 2^31
    // (each weight or connectivity of a vertex is at most that), and the call
    // fails with HP_ERR_UNSUPPORTED if one does not.
    c->weight_check = vs[3] >= (long long)INT32_MAX;
    // the input level's rows, before any kernel sums them in int32; not needed
    // when the validation's largest degree times largest weight is below 2^31
    const bool row_bound = c->opt.validate && vs[5] * vs[2] < (long long)INT32_MAX;
    if (c->weight_check && !row_bound) {
        HP_TRY(hp_check_weight_range(c, g0));
        HP_TRY(hp_check_status(c));
    }

    const int32_t thr = c->opt.coarsen_to > 0 ? c->opt.coarsen_to : default_coarsen_to(nparts);
    const int64_t maxvwgt = (3 * (int64_t)tv) / (2 * (int64_t)thr);

    HP_CUDA(cudaEventRecord(c->ev[1], c->stream));
    HP_TRY(hp_coarsen(c, thr, maxvwgt));
    HP_CUDA(cudaEventRecord(c->ev[2], c->stream));

    for (auto &l : c->levels) {
        l.where = lalloc_t<int32_t>(c, l.n);
        HP_CHECK_OOM(c);
    }
    std::vector<int64_t> opt(nparts), maxp(nparts);
    hp_part_targets(tv, nparts, tpwgts, ubfactor, opt.data(), maxp.data());
    const int64_t ub2 = hp_bisect_ub_fx(ubfactor, nparts);
    HpLevel &cg = c->levels.back();
    HP_TRY(hp_fill_i32(c, cg.where, cg.n, 0));   // every vertex gets a part below; never garbage
    HP_TRY(hp_initial_partition(c, cg, nparts, opt.data(), ub2, cg.where));
    HP_CUDA(cudaEventRecord(c->ev[3], c->stream));
    HP_TRY(hp_uncoarsen(c, nparts, opt.data(), maxp.data()));
    HP_CUDA(cudaEventRecord(c->ev[4], c->stream));

    // exact report of the final partition (also checks the tracked cut)
    const size_t mark = c->hi;
    unsigned long long *pw = ralloc_t<unsigned long long>(c, nparts);
    HP_CHECK_OOM(c);
    HP_CUDA(cudaMemsetAsync(pw, 0, sizeof(unsigned long long) * nparts, c->stream));
    HP_CUDA(cudaMemsetAsync(sc, 0, sizeof(unsigned long long) * 2, c->stream));
    HpLevel &f = c->levels[0];
    HP_TRY(hp_edgecut_launch(c, n, f.m, f.xadj, f.adjncy, f.adjwgt, f.where, &sc[0]));
    HP_LAUNCH(c, final_pw_kernel, gsz(c, n), 256, nparts <= 2048 ? sizeof(unsigned long long) * nparts : 0, n,
              f.where, f.vwgt, pw, nparts, c->d_status);
    std::vector<unsigned long long> hpw(nparts);
    HP_CUDA(cudaMemcpyAsync(hpw.data(), pw, sizeof(unsigned long long) * nparts, cudaMemcpyDeviceToHost, c->stream));
    long long cut2 = 0;
    HP_TRY(hp_read_scalars(c, &sc[0], sizeof(long long), &cut2));
    HP_TRY(hp_check_status(c));
    c->hi = mark;
    const int64_t cut = cut2 / 2;
    if (cut != f.cut_final) {
        fprintf(stderr, "hp: internal error: tracked cut %lld != recomputed cut %lld\n",
                (long long)f.cut_final, (long long)cut);
        return HP_ERR_INTERNAL;
    }
    int64_t ex = INT64_MIN;
    for (int32_t p = 0; p < nparts; p++) ex = std::max<int64_t>(ex, (int64_t)hpw[p] - maxp[p]);
    st.edgecut = cut;
    st.max_excess = ex;
    st.nlevels = (int32_t)c->levels.size();
    st.coarsest_nvtxs = cg.n;
    st.coarsest_nedges = cg.m;
    if (edgecut) *edgecut = cut;
    return HP_OK;
}

int begin_call(hp_context *c, const hp_options *opt, void *stream)
{
    if (!c) return HP_ERR_INVALID_ARG;
    if (opt) {
        if (opt->version != HP_OPTIONS_VERSION) return HP_ERR_INVALID_ARG;
        c->opt = *opt;
    } else {
        hp_options_default(&c->opt);
    }
    HP_CUDA(cudaSetDevice(c->device));
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    c->launches = 0;
    c->prof_recs.clear();
    c->prof_next = 0;
    memset(&c->stats, 0, sizeof(c->stats));
    unsigned zero = 0;
    HP_CUDA(cudaMemcpyAsync(c->d_status, &zero, sizeof(unsigned), cudaMemcpyHostToDevice, c->stream));
    if (c->opt.profile)
        HP_CUDA(cudaMemsetAsync(c->d_profb, 0, sizeof(unsigned long long) * HP_PROF_NCLASS, c->stream));
    return HP_OK;
}

void finish_stats(hp_context *c)
{
    cudaStreamSynchronize(c->stream);
    float ms = 0;
    hp_stats &st = c->stats;
    if (cudaEventElapsedTime(&ms, c->ev[0], c->ev[5]) == cudaSuccess) st.ms_total = ms;
    if (cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]) == cudaSuccess) st.ms_coarsen = ms;
    if (cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]) == cudaSuccess) st.ms_init = ms;
    if (cudaEventElapsedTime(&ms, c->ev[3], c->ev[4]) == cudaSuccess) st.ms_uncoarsen = ms;
    st.kernel_launches = c->launches;
    hp_prof_resolve(c);
    c->trace_valid = c->opt.trace != 0;
}

}  // namespace

// ---- kernel-class profiler ----------------------------------------------------------
static int prof_event(hp_context *c)
{
    if (c->prof_next >= (int)c->prof_events.size()) {
        for (int i = 0; i < 256; i++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return -1; }
            c->prof_events.push_back(e);
        }
    }
    return c->prof_next++;
}

int hp_prof_begin(hp_context *c)
{
    if (!c->opt.profile || c->prof_suspended) return -1;
    int e0 = prof_event(c);
    if (e0 < 0) return -1;
    cudaEventRecord(c->prof_events[e0], c->stream);
    c->prof_recs.push_back({-1, e0, -1, 0, c->launches});
    return (int)c->prof_recs.size() - 1;
}

void hp_prof_end(hp_context *c, int token, int cls, int64_t bytes)
{
    if (token < 0 || token >= (int)c->prof_recs.size()) return;
    int e1 = prof_event(c);
    if (e1 < 0) return;
    cudaEventRecord(c->prof_events[e1], c->stream);
    auto &r = c->prof_recs[token];
    r.cls = cls;
    r.ev1 = e1;
    r.bytes = bytes;
    r.launches = c->launches - r.launches;
}

void hp_prof_add_bytes(hp_context *c, int token, int64_t bytes)
{
    if (token < 0 || token >= (int)c->prof_recs.size()) return;
    c->prof_recs[token].bytes += bytes;
}

unsigned long long *hp_prof_counter(hp_context *c, int cls)
{
    if (!c->opt.profile || c->prof_suspended || cls < 0 || cls >= HP_PROF_NCLASS) return nullptr;
    return c->d_profb + cls;
}

void hp_prof_resolve(hp_context *c)
{
    if (c->opt.profile) {
        // the stream is idle here (finish_stats synchronised it)
        unsigned long long dev[HP_PROF_NCLASS] = {};
        if (cudaMemcpy(dev, c->d_profb, sizeof(dev), cudaMemcpyDeviceToHost) == cudaSuccess) {
            for (int i = 0; i < HP_PROF_NCLASS; i++) c->stats.prof_bytes[i] += (int64_t)dev[i];
        } else {
            cudaGetLastError();
        }
    }
    for (const auto &r : c->prof_recs) {
        if (r.cls < 0 || r.cls >= HP_PROF_NCLASS || r.ev1 < 0) continue;
        float ms = 0;
        if (cudaEventElapsedTime(&ms, c->prof_events[r.ev0], c->prof_events[r.ev1]) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        c->stats.prof_ms[r.cls] += ms;
        c->stats.prof_bytes[r.cls] += r.bytes;
        c->stats.prof_launches[r.cls] += r.launches;
    }
    c->prof_recs.clear();
    c->prof_next = 0;
}

// ---- shared helpers -------------------------------------------------------------
static void reaper_main(hp_context *c)
{
    cudaSetDevice(c->device);
    for (;;) {
        hp_context::Retired r;
        {
            std::unique_lock<std::mutex> lk(c->reaper_mu);
            c->reaper_cv.wait(lk, [c] { return c->reaper_stop || !c->reaper_q.empty(); });
            if (c->reaper_q.empty()) return;   // stop requested and nothing left
            r = std::move(c->reaper_q.front());
            c->reaper_q.pop_front();
        }
        cudaEventSynchronize(r.done);
        for (auto &it : r.graphs) {
            if (it.second) cudaGraphExecDestroy(it.second);
            if (it.first) cudaGraphDestroy(it.first);
        }
        cudaEventDestroy(r.done);
    }
}

int hp_graph_retire(hp_context *c, std::vector<std::pair<cudaGraph_t, cudaGraphExec_t>> &&graphs)
{
    if (graphs.empty()) return HP_OK;
    hp_context::Retired r;
    r.graphs = std::move(graphs);
    cudaError_t e = cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(r.done, c->stream);
    if (e != cudaSuccess) {
        // fall back to a synchronous release
        cudaGetLastError();
        cudaStreamSynchronize(c->stream);
        for (auto &it : r.graphs) {
            if (it.second) cudaGraphExecDestroy(it.second);
            if (it.first) cudaGraphDestroy(it.first);
        }
        if (r.done) cudaEventDestroy(r.done);
        return HP_OK;
    }
    {
        std::lock_guard<std::mutex> lk(c->reaper_mu);
        if (!c->reaper.joinable()) c->reaper = std::thread(reaper_main, c);
        c->reaper_q.push_back(std::move(r));
    }
    c->reaper_cv.notify_one();
    return HP_OK;
}

int hp_lb_reserve(hp_context *c, int64_t tiles)
{
    if (tiles <= c->lb_cap && c->lb_ctl) return HP_OK;
    // between calls: nothing of this context is in flight
    HP_CUDA(cudaStreamSynchronize(c->stream));
    const int64_t cap = std::max<int64_t>(tiles, std::max<int64_t>(2 * c->lb_cap, 4096));
    if (c->lb_status) cudaFree(c->lb_status);
    c->lb_status = nullptr;
    c->lb_cap = 0;
    HP_CUDA(cudaMalloc((void **)&c->lb_status, sizeof(unsigned long long) * (size_t)cap));
    HP_CUDA(cudaMemset(c->lb_status, 0, sizeof(unsigned long long) * (size_t)cap));
    if (!c->lb_ctl) HP_CUDA(cudaMalloc((void **)&c->lb_ctl, sizeof(hp::LbCtl)));
    HP_CUDA(cudaMemset(c->lb_ctl, 0, sizeof(hp::LbCtl)));
    c->lb_cap = cap;
    return HP_OK;
}

int hp_read_scalars(hp_context *c, const void *d_src, size_t nbytes, void *dst)
{
    if (nbytes > sizeof(long long) * HP_NSCAL) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaMemcpyAsync(c->h_pin, d_src, nbytes, cudaMemcpyDeviceToHost, c->stream));
    HP_CUDA(cudaStreamSynchronize(c->stream));
    memcpy(dst, c->h_pin, nbytes);
    return HP_OK;
}

int hp_check_status(hp_context *c)
{
    unsigned s = 0;
    HP_TRY(hp_read_scalars(c, c->d_status, sizeof(unsigned), &s));
    if (s & HP_STATUS_SPIN_TIMEOUT) return HP_ERR_TIMEOUT;
    if (s & HP_STATUS_BAD_GRAPH) return HP_ERR_INVALID_GRAPH;
    if (s & HP_STATUS_OVERFLOW) return HP_ERR_INTERNAL;
    if (s & HP_STATUS_WEIGHT_RANGE) {
        fprintf(stderr, "hp: the edge weights of a matched pair sum to 2^31 or more: coarse edge weights "
                        "would not fit int32\n");
        return HP_ERR_UNSUPPORTED;
    }
    return HP_OK;
}

void hp_part_targets(int64_t tvwgt, int32_t nparts, const float *tpwgts, float ubfactor,
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

int64_t hp_bisect_ub_fx(float ubfactor, int32_t nparts)
{
    double ub2 = nparts > 1 ? pow((double)ubfactor, 1.0 / log((double)nparts)) : (double)ubfactor;
    return (int64_t)floor(ub2 * 65536.0 + 0.5);
}

// ---- C ABI ------------------------------------------------------------------------
HP_API void hp_options_default(hp_options *o)
{
    if (!o) return;
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
    o->eager = 0;
    o->seed = 1;
}

HP_API void hp_tuning_default(hp_tuning *t)
{
    if (!t) return;
    memset(t, 0, sizeof(*t));
    t->match_warp_deg = 32;
    t->match_cta_deg = 4096;
    t->contract_thread_row = HP_TUNE_THREAD_ROW_MAX;
    t->contract_warp_row = HP_TUNE_WARP_ROW_MAX;
    t->contract_cta_row = HP_TUNE_CTA_ROW_MAX;
    t->gain_thread_deg = HP_TUNE_THREAD_ROW_MAX;
    t->gain_hub_deg = 4096;
    t->warp_dense_k = HP_TUNE_WARP_DENSE_K_MAX;
    t->grid_ctas_per_sm = 8;
    t->dense_sparse_ratio = 4;
    t->small_level_n = 4096;
    t->chunk_deg = 4096;
    t->trial_cta_n = 512;
    t->contract_smem_cn = HP_TUNE_SMEM_CN_MAX;
    t->batch_workers = 16;
    t->small_match_n = 8192;
    t->contract_hybrid = 1;
    t->apply_chunk_deg = 4096;
    t->pdl = 1;
    t->graph_passes = 1;
}

namespace {
// The first field out of its range, or nullptr.
const char *tuning_violation(const hp_tuning &t)
{
    auto in = [](int32_t v, int64_t lo, int64_t hi) { return v >= lo && v <= hi; };
    if (!in(t.match_warp_deg, 4, 256)) return "match_warp_deg";
    if (!in(t.match_cta_deg, t.match_warp_deg, HP_TUNE_DEG_MAX)) return "match_cta_deg";
    if (!in(t.contract_thread_row, 8, HP_TUNE_THREAD_ROW_MAX)) return "contract_thread_row";
    if (!in(t.contract_warp_row, t.contract_thread_row, HP_TUNE_WARP_ROW_MAX)) return "contract_warp_row";
    if (!in(t.contract_cta_row, t.contract_warp_row, HP_TUNE_CTA_ROW_MAX)) return "contract_cta_row";
    if (!in(t.gain_thread_deg, 8, HP_TUNE_THREAD_ROW_MAX)) return "gain_thread_deg";
    if (!in(t.gain_hub_deg, t.gain_thread_deg, HP_TUNE_DEG_MAX)) return "gain_hub_deg";
    if (!in(t.warp_dense_k, 0, HP_TUNE_WARP_DENSE_K_MAX)) return "warp_dense_k";
    if (!in(t.grid_ctas_per_sm, 1, 32)) return "grid_ctas_per_sm";
    if (!in(t.dense_sparse_ratio, 1, 4096)) return "dense_sparse_ratio";
    if (!in(t.small_level_n, 0, HP_TUNE_SMALL_LEVEL_MAX)) return "small_level_n";
    if (!in(t.chunk_deg, t.gain_thread_deg, HP_TUNE_DEG_MAX)) return "chunk_deg";
    if (!in(t.trial_cta_n, 1, HP_TUNE_DEG_MAX)) return "trial_cta_n";
    if (!in(t.contract_smem_cn, 0, HP_TUNE_SMEM_CN_MAX)) return "contract_smem_cn";
    if (!in(t.batch_workers, 1, 64)) return "batch_workers";
    if (!in(t.small_match_n, 0, HP_TUNE_SMALL_MATCH_MAX)) return "small_match_n";
    if (!in(t.contract_hybrid, 0, 1)) return "contract_hybrid";
    if (!in(t.apply_chunk_deg, t.gain_thread_deg, HP_TUNE_DEG_MAX)) return "apply_chunk_deg";
    if (!in(t.pdl, 0, 1)) return "pdl";
    if (!in(t.graph_passes, 0, 1)) return "graph_passes";
    for (int32_t r : t.reserved)
        if (r != 0) return "reserved";
    return nullptr;
}
}  // namespace

HP_API int hp_context_set_tuning(hp_context *ctx, const hp_tuning *t)
{
    if (!ctx || !t) return HP_ERR_INVALID_ARG;
    if (const char *bad = tuning_violation(*t)) {
        fprintf(stderr, "hp: tuning field %s out of range\n", bad);
        return HP_ERR_INVALID_ARG;
    }
    ctx->tune = *t;
    return HP_OK;
}

HP_API int hp_context_get_tuning(const hp_context *ctx, hp_tuning *t)
{
    if (!ctx || !t) return HP_ERR_INVALID_ARG;
    *t = ctx->tune;
    return HP_OK;
}

HP_API const char *hp_strerror(int code)
{
    switch (code) {
    case HP_OK: return "ok";
    case HP_ERR_INVALID_ARG: return "invalid argument";
    case HP_ERR_INVALID_GRAPH: return "invalid graph (CSR validation failed)";
    case HP_ERR_NOMEM: return "device memory exhausted";
    case HP_ERR_CUDA: return "CUDA runtime error";
    case HP_ERR_TIMEOUT: return "bounded device wait expired";
    case HP_ERR_NO_DEVICE: return "no CUDA device";
    case HP_ERR_UNSUPPORTED: return "unsupported request";
    case HP_ERR_INTERNAL: return "internal consistency check failed";
    default: return "unknown error";
    }
}

HP_API int hp_context_create(int device, hp_context **out)
{
    if (!out) return HP_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return HP_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return HP_ERR_INVALID_ARG;
    hp_context *c = new hp_context();
    c->device = device;
    hp_tuning_default(&c->tune);
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return HP_ERR_NO_DEVICE; }
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    bool ok = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) == cudaSuccess;
    void *blk = nullptr;
    ok = ok && cudaMalloc(&blk, 256 + sizeof(unsigned long long) * (HP_NSCAL + HP_PROF_NCLASS)) == cudaSuccess;
    if (ok) {
        c->d_status = (unsigned *)blk;
        c->d_scal = (unsigned long long *)((char *)blk + 256);
        c->d_profb = c->d_scal + HP_NSCAL;
    }
    ok = ok && cudaMallocHost((void **)&c->h_pin, sizeof(long long) * HP_NSCAL) == cudaSuccess;
    for (int i = 0; ok && i < 8; i++) ok = cudaEventCreate(&c->ev[i]) == cudaSuccess;
    ok = ok && hp_refine_init() == HP_OK;
    ok = ok && hp_initpart_init() == HP_OK;
    ok = ok && hp_coarsen_init() == HP_OK;
    if (!ok) {
        cudaGetLastError();
        hp_context_destroy(c);
        return HP_ERR_CUDA;
    }
    *out = c;
    return HP_OK;
}

HP_API void hp_context_destroy(hp_context *c)
{
    if (!c) return;
    for (hp_context *w : c->workers) hp_context_destroy(w);
    c->workers.clear();
    if (c->reaper.joinable()) {
        {
            std::lock_guard<std::mutex> lk(c->reaper_mu);
            c->reaper_stop = true;
        }
        c->reaper_cv.notify_one();
        c->reaper.join();   // releases every queued graph first
    }
    cudaSetDevice(c->device);
    if (c->own_stream) cudaStreamSynchronize(c->own_stream);
    if (c->arena) cudaFree(c->arena);
    if (c->d_status) cudaFree(c->d_status);
    if (c->lb_status) cudaFree(c->lb_status);
    if (c->lb_ctl) cudaFree(c->lb_ctl);
    if (c->h_pin) cudaFreeHost(c->h_pin);
    for (int i = 0; i < 8; i++)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    for (auto e : c->prof_events) cudaEventDestroy(e);
    if (c->mlp_params) cudaFree(c->mlp_params);
    if (c->mlp_scratch) cudaFree(c->mlp_scratch);
    if (c->log_x) cudaFree(c->log_x);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

static int check_args(int32_t nvtxs, const void *xadj, const void *adjncy, int32_t nparts,
                      float ubfactor, const void *part)
{
    if (nvtxs < 0 || !xadj || !part) return HP_ERR_INVALID_ARG;
    if (nvtxs > 0 && !adjncy) return HP_ERR_INVALID_ARG;
    if (nparts < 1) return HP_ERR_INVALID_ARG;
    if (nparts > HP_MAX_PARTS) return HP_ERR_UNSUPPORTED;
    if (!(ubfactor >= 1.0f) || !std::isfinite(ubfactor)) return HP_ERR_INVALID_ARG;
    return HP_OK;
}

// Places the level-0 graph (copying host or device inputs into the arena).
static int place_level0(hp_context *c, int32_t n, int64_t m, const int32_t *xadj, const int32_t *adjncy,
                        const int32_t *vwgt, const int32_t *adjwgt, cudaMemcpyKind kind)
{
    c->levels.emplace_back();
    HpLevel &g = c->levels[0];
    g.n = n;
    g.m = m;
    g.xadj = lalloc_t<int32_t>(c, (int64_t)n + 1);
    g.adjncy = lalloc_t<int32_t>(c, m);
    g.adjwgt = lalloc_t<int32_t>(c, m);
    g.vwgt = lalloc_t<int32_t>(c, n);
    HP_CHECK_OOM(c);
    HP_CUDA(cudaMemcpyAsync(g.xadj, xadj, sizeof(int32_t) * ((size_t)n + 1), kind, c->stream));
    if (m > 0) HP_CUDA(cudaMemcpyAsync(g.adjncy, adjncy, sizeof(int32_t) * (size_t)m, kind, c->stream));
    if (adjwgt) {
        if (m > 0) HP_CUDA(cudaMemcpyAsync(g.adjwgt, adjwgt, sizeof(int32_t) * (size_t)m, kind, c->stream));
    } else if (m > 0) {
        HP_LAUNCH(c, fill_ones_kernel, gsz(c, m), 256, 0, m, g.adjwgt);
    }
    if (vwgt) {
        if (n > 0) HP_CUDA(cudaMemcpyAsync(g.vwgt, vwgt, sizeof(int32_t) * (size_t)n, kind, c->stream));
    } else if (n > 0) {
        HP_LAUNCH(c, fill_ones_kernel, gsz(c, n), 256, 0, (int64_t)n, g.vwgt);
    }
    return HP_OK;
}

static int partition_common(hp_context *c, int32_t n, int64_t m, const int32_t *xadj,
                            const int32_t *adjncy, const int32_t *vwgt, const int32_t *adjwgt,
                            int32_t nparts, const float *tpwgts, float ubfactor, bool host,
                            int32_t *part, int64_t *edgecut)
{
    // look-back tiles of every single-pass kernel of the call: at most one per
    // 256 vertices (the smallest tile), plus the scans' slack
    HP_TRY(hp_lb_reserve(c, ((int64_t)n + 255) / 256 + 1024));
    size_t want = estimate_arena(n, m);
    if (c->arena_first) {   // hp_test_arena_first freed the arena: this attempt gets exactly that
        want = c->arena_first;
        c->arena_first = 0;
    }
    c->arena_restarts = 0;
    int rc = HP_ERR_NOMEM;
    for (int attempt = 0; attempt < 4 && rc == HP_ERR_NOMEM; attempt++) {
        if (attempt > 0) c->arena_restarts++;
        HP_TRY(ensure_arena(c, want));
        reset_arena(c);
        unsigned zero = 0;
        HP_CUDA(cudaMemcpyAsync(c->d_status, &zero, sizeof(unsigned), cudaMemcpyHostToDevice, c->stream));
        HP_CUDA(cudaEventRecord(c->ev[0], c->stream));
        rc = place_level0(c, n, m, xadj, adjncy, vwgt, adjwgt,
                          host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice);
        if (rc == HP_OK) HP_CUDA(cudaEventRecord(c->ev[6], c->stream));
        if (rc == HP_OK) {
            if (n == 0) {
                if (edgecut) *edgecut = 0;
                HP_CUDA(cudaEventRecord(c->ev[1], c->stream));
                HP_CUDA(cudaEventRecord(c->ev[2], c->stream));
                HP_CUDA(cudaEventRecord(c->ev[3], c->stream));
                HP_CUDA(cudaEventRecord(c->ev[4], c->stream));
            } else {
                rc = vcycle(c, nparts, tpwgts, ubfactor, edgecut);
            }
        }
        if (rc == HP_ERR_NOMEM) want *= 2;
    }
    if (rc != HP_OK) return rc;
    if (n > 0) {
        HpLevel &f = c->levels[0];
        HP_CUDA(cudaEventRecord(c->ev[7], c->stream));
        HP_CUDA(cudaMemcpyAsync(part, f.where, sizeof(int32_t) * (size_t)n,
                                host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, c->stream));
    }
    HP_CUDA(cudaEventRecord(c->ev[5], c->stream));
    finish_stats(c);
    float ms = 0;
    if (host && cudaEventElapsedTime(&ms, c->ev[0], c->ev[6]) == cudaSuccess) c->stats.ms_h2d = ms;
    if (host && n > 0 && cudaEventElapsedTime(&ms, c->ev[7], c->ev[5]) == cudaSuccess) c->stats.ms_d2h = ms;
    return HP_OK;
}

HP_API int hp_partition(hp_context *ctx, int32_t nvtxs, const int32_t *xadj, const int32_t *adjncy,
                        const int32_t *vwgt, const int32_t *adjwgt, int32_t nparts, const float *tpwgts,
                        float ubfactor, const hp_options *opt, int32_t *part, int64_t *edgecut)
{
    HP_TRY(check_args(nvtxs, xadj, adjncy, nparts, ubfactor, part));
    const int64_t m = xadj[nvtxs];
    if (xadj[0] != 0 || m < 0 || m > INT32_MAX) return HP_ERR_INVALID_GRAPH;
    HP_TRY(begin_call(ctx, opt, nullptr));
    return partition_common(ctx, nvtxs, m, xadj, adjncy, vwgt, adjwgt, nparts, tpwgts, ubfactor,
                            true, part, edgecut);
}

HP_API int hp_partition_device(hp_context *ctx, int32_t nvtxs, int64_t nedges, const int32_t *d_xadj,
                               const int32_t *d_adjncy, const int32_t *d_vwgt, const int32_t *d_adjwgt,
                               int32_t nparts, const float *tpwgts, float ubfactor, const hp_options *opt,
                               void *stream, int32_t *d_part, int64_t *edgecut)
{
    HP_TRY(check_args(nvtxs, d_xadj, d_adjncy, nparts, ubfactor, d_part));
    if (nedges < 0 || nedges > INT32_MAX) return HP_ERR_INVALID_GRAPH;
    HP_TRY(begin_call(ctx, opt, stream));
    return partition_common(ctx, nvtxs, nedges, d_xadj, d_adjncy, d_vwgt, d_adjwgt, nparts, tpwgts,
                            ubfactor, false, d_part, edgecut);
}

HP_API int hp_last_stats(const hp_context *ctx, hp_stats *out)
{
    if (!ctx || !out) return HP_ERR_INVALID_ARG;
    *out = ctx->stats;
    return HP_OK;
}

HP_API int hp_trace_nlevels(const hp_context *ctx)
{
    if (!ctx || !ctx->trace_valid) return 0;
    return (int)ctx->levels.size();
}

HP_API int hp_trace_level(const hp_context *ctx, int level, int32_t *nvtxs, int64_t *nedges,
                          int64_t *cut_start, int64_t *cut_final)
{
    if (!ctx || !ctx->trace_valid || level < 0 || level >= (int)ctx->levels.size()) return HP_ERR_INVALID_ARG;
    const HpLevel &l = ctx->levels[level];
    if (nvtxs) *nvtxs = l.n;
    if (nedges) *nedges = l.m;
    if (cut_start) *cut_start = l.cut_start;
    if (cut_final) *cut_final = l.cut_final;
    return HP_OK;
}

HP_API int hp_trace_copy(const hp_context *ctx, int level, int what, int32_t *dst, int64_t count)
{
    if (!ctx || !ctx->trace_valid || level < 0 || level >= (int)ctx->levels.size() || !dst)
        return HP_ERR_INVALID_ARG;
    const HpLevel &l = ctx->levels[level];
    const int32_t *src = nullptr;
    int64_t len = 0;
    switch (what) {
    case HP_TRACE_XADJ: src = l.xadj; len = (int64_t)l.n + 1; break;
    case HP_TRACE_ADJNCY: src = l.adjncy; len = l.m; break;
    case HP_TRACE_ADJWGT: src = l.adjwgt; len = l.m; break;
    case HP_TRACE_VWGT: src = l.vwgt; len = l.n; break;
    case HP_TRACE_MATCH: src = l.match; len = l.n; break;
    case HP_TRACE_CMAP: src = l.cmap; len = l.n; break;
    case HP_TRACE_WHERE_START: src = l.where_start; len = l.n; break;
    case HP_TRACE_WHERE_FINAL: src = l.where_final; len = l.n; break;
    default: return HP_ERR_INVALID_ARG;
    }
    if (!src || count < len) return HP_ERR_INVALID_ARG;
    if (len == 0) return HP_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return HP_ERR_CUDA;
    if (cudaMemcpy(dst, src, sizeof(int32_t) * (size_t)len, cudaMemcpyDeviceToHost) != cudaSuccess)
        return HP_ERR_CUDA;
    return HP_OK;
}

int hp_ensure_workers(hp_context *ctx, int nworkers)
{
    HP_CUDA(cudaSetDevice(ctx->device));
    while ((int)ctx->workers.size() < nworkers) {
        hp_context *w = nullptr;
        HP_TRY(hp_context_create(ctx->device, &w));
        ctx->workers.push_back(w);
    }
    for (hp_context *w : ctx->workers) w->tune = ctx->tune;
    return HP_OK;
}

HP_API int hp_partition_batch(hp_context *ctx, int32_t ngraphs, const int64_t *vtxdist,
                              const int64_t *edgedist, const int32_t *xadj, const int32_t *adjncy,
                              const int32_t *vwgt, const int32_t *adjwgt, const int32_t *nparts,
                              const float *ubfactor, const hp_options *opt, int32_t *part,
                              int64_t *edgecut)
{
    // Independent graphs are partitioned by a pool of worker contexts, each
    // with its own stream and arena; a worker's host-side scalar reads overlap
    // with the other workers' kernels.  Graphs are taken largest first.  Each
    // graph's result depends only on that graph, so the batch returns exactly
    // what one hp_partition() call per graph returns.
    if (!ctx || ngraphs < 0 || !vtxdist || !edgedist || !xadj || !nparts || !ubfactor || !part)
        return HP_ERR_INVALID_ARG;
    if (ngraphs == 0) return HP_OK;
    for (int32_t gi = 0; gi < ngraphs; gi++) {
        if (vtxdist[gi + 1] < vtxdist[gi] || edgedist[gi + 1] < edgedist[gi]) return HP_ERR_INVALID_ARG;
        if (vtxdist[gi + 1] - vtxdist[gi] > INT32_MAX - 1) return HP_ERR_UNSUPPORTED;
    }
    const int nworkers = (int)std::min<int64_t>(ngraphs, ctx->tune.batch_workers);
    HP_TRY(hp_ensure_workers(ctx, nworkers));
    // The workers run their levels' pass loops eagerly: sixteen host threads that
    // capture and instantiate a CUDA graph per level contend for the driver, and
    // the graphs of small graphs' levels never amortise (the small-level kernel
    // still takes the small levels).  Results are the same in both loop modes.
    hp_options wopt;
    if (opt) wopt = *opt;
    else hp_options_default(&wopt);
    wopt.eager = 1;
    std::vector<int32_t> order(ngraphs);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return edgedist[a + 1] - edgedist[a] > edgedist[b + 1] - edgedist[b];
    });
    std::atomic<int32_t> next{0};
    std::atomic<int> first_err{HP_OK};
    std::atomic<long long> launches{0};
    auto t0 = std::chrono::steady_clock::now();
    auto work = [&](hp_context *w) {
        cudaSetDevice(w->device);
        for (;;) {
            if (first_err.load() != HP_OK) return;
            int32_t i = next.fetch_add(1);
            if (i >= ngraphs) return;
            const int32_t gi = order[i];
            const int64_t v0 = vtxdist[gi], n = vtxdist[gi + 1] - v0, e0 = edgedist[gi];
            int64_t cut = 0;
            int rc = hp_partition(w, (int32_t)n, xadj + v0 + gi, adjncy + e0, vwgt ? vwgt + v0 : nullptr,
                                  adjwgt ? adjwgt + e0 : nullptr, nparts[gi], nullptr, ubfactor[gi], &wopt,
                                  part + v0, &cut);
            if (rc != HP_OK) {
                int expected = HP_OK;
                first_err.compare_exchange_strong(expected, rc);
                return;
            }
            launches += w->stats.kernel_launches;
            if (edgecut) edgecut[gi] = cut;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < nworkers; t++) pool.emplace_back(work, ctx->workers[t]);
    for (auto &t : pool) t.join();
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    ctx->stats.ms_total = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ctx->stats.kernel_launches = (int32_t)std::min<long long>(launches.load(), INT32_MAX);
    ctx->trace_valid = false;
    return first_err.load();
}

HP_API int hp_scan_exclusive_i32(hp_context *ctx, const int32_t *d_in, int32_t *d_out, int64_t n,
                                 void *stream)
{
    if (!ctx || n < 0 || (!d_in && n > 0) || !d_out) return HP_ERR_INVALID_ARG;
    if (n >= INT32_MAX) return HP_ERR_UNSUPPORTED;
    HP_CUDA(cudaSetDevice(ctx->device));
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    size_t need = (size_t)((n + 4096) / 4096 + 2) * 8 + ((size_t)1 << 20);
    if (!ctx->arena || ctx->arena_cap < need) HP_TRY(ensure_arena(ctx, std::max(need, (size_t)64 << 20)));
    reset_arena(ctx);
    HP_TRY(hp_lb_reserve(ctx, (n + 4096) / 4096 + 2));
    unsigned zero = 0;
    HP_CUDA(cudaMemcpyAsync(ctx->d_status, &zero, sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
    HP_TRY(hp_scan_excl(ctx, d_in, d_out, n));
    return hp_check_status(ctx);
}

HP_API int hp_edgecut_device(hp_context *ctx, int32_t nvtxs, const int32_t *d_xadj, const int32_t *d_adjncy,
                             const int32_t *d_adjwgt, const int32_t *d_where, void *stream, int64_t *cut)
{
    if (!ctx || nvtxs < 0 || !d_xadj || !d_where || !cut) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(ctx->device));
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    HP_CUDA(cudaMemsetAsync(ctx->d_scal, 0, sizeof(unsigned long long), ctx->stream));
    if (d_adjwgt) {
        HP_TRY(hp_edgecut_launch(ctx, nvtxs, -1, d_xadj, d_adjncy, d_adjwgt, d_where, ctx->d_scal));
    } else {
        // unit weights: count cut entries through a ones array in the arena
        int64_t m = 0;
        int32_t last = 0;
        HP_CUDA(cudaMemcpy(&last, d_xadj + nvtxs, sizeof(int32_t), cudaMemcpyDeviceToHost));
        m = last;
        size_t need = sizeof(int32_t) * (size_t)(m + 1) + 4096;
        if (!ctx->arena || ctx->arena_cap < need) HP_TRY(ensure_arena(ctx, std::max(need, (size_t)64 << 20)));
        reset_arena(ctx);
        int32_t *ones = ralloc_t<int32_t>(ctx, m);
        HP_CHECK_OOM(ctx);
        HP_LAUNCH(ctx, fill_ones_kernel, gsz(ctx, m), 256, 0, m, ones);
        HP_TRY(hp_edgecut_launch(ctx, nvtxs, -1, d_xadj, d_adjncy, ones, d_where, ctx->d_scal));
    }
    long long c2 = 0;
    HP_TRY(hp_read_scalars(ctx, ctx->d_scal, sizeof(long long), &c2));
    *cut = c2 / 2;
    return HP_OK;
}

// ---- failure path of the bounded device waits ----------------------------------------
// One warp runs the scans' look-back wait (hp::lookback_exclusive) as tile 1,
// against a tile 0 whose status word nothing ever sets.  Lane 0 polls it
// HP_SPIN_LIMIT times, then sets HP_STATUS_SPIN_TIMEOUT and counts the
// predecessor as zero, so the kernel ends by itself.
__global__ void wait_expiry_kernel(unsigned long long *tile_status, unsigned *status, int32_t *excl)
{
    hp::pdl_wait();
    const int32_t e = hp::lookback_exclusive(tile_status, 1, 5, status);
    if (threadIdx.x == 0) *excl = e;
}

HP_API int hp_test_wait_expiry(hp_context *ctx)
{
    if (!ctx) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(ctx->device));
    ctx->stream = ctx->own_stream;
    unsigned long long *tiles = ctx->d_scal;                    // tile 0 (never set), tile 1
    int32_t *excl = reinterpret_cast<int32_t *>(ctx->d_scal + 2);
    HP_CUDA(cudaMemsetAsync(tiles, 0, 3 * sizeof(unsigned long long), ctx->stream));
    const unsigned zero = 0;
    HP_CUDA(cudaMemcpyAsync(ctx->d_status, &zero, sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
    HP_LAUNCH(ctx, wait_expiry_kernel, 1, 32, 0, tiles, ctx->d_status, excl);
    const int rc = hp_check_status(ctx);
    int32_t e = -1;
    HP_TRY(hp_read_scalars(ctx, excl, sizeof(int32_t), &e));
    // the status is cleared: the context is usable for the next call
    HP_CUDA(cudaMemcpyAsync(ctx->d_status, &zero, sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    if (rc == HP_ERR_TIMEOUT && e != 0) return HP_ERR_INTERNAL;   // the expired predecessor counts as 0
    return rc;
}

HP_API int hp_test_arena_first(hp_context *ctx, int64_t bytes)
{
    if (!ctx || bytes < 0) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(ctx->device));
    if (bytes > 0 && ctx->arena) {
        HP_CUDA(cudaStreamSynchronize(ctx->own_stream));
        cudaFree(ctx->arena);   // synchronises the device: no earlier call still reads it
        ctx->arena = nullptr;
        ctx->arena_cap = 0;
        ctx->levels.clear();    // the last call's trace lived in the arena
        ctx->trace_valid = false;
    }
    ctx->arena_first = (size_t)bytes;
    return HP_OK;
}

HP_API int hp_test_arena_restarts(hp_context *ctx)
{
    if (!ctx) return HP_ERR_INVALID_ARG;
    return ctx->arena_restarts;
}

// ---- legacy drop-in ------------------------------------------------------------------
static std::mutex g_legacy_mu;
static hp_context *g_legacy = nullptr;

HP_API void hunyuangraph_PartitionGraph(int *nvtxs, int *xadj, int *adjncy, int *vwgt, int *adjwgt,
                                        int *nparts, float *tpwgts, float *ubvec, int *part)
{
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    if (!nvtxs || !nparts || !part) {
        fprintf(stderr, "hunyuangraph_PartitionGraph: NULL argument\n");
        return;
    }
    int rc = HP_OK;
    if (!g_legacy) rc = hp_context_create(0, &g_legacy);
    if (rc == HP_OK) {
        int64_t cut = 0;
        rc = hp_partition(g_legacy, *nvtxs, xadj, adjncy, vwgt, adjwgt, *nparts, tpwgts,
                          ubvec ? ubvec[0] : 1.03f, nullptr, part, &cut);
    }
    if (rc != HP_OK) {
        fprintf(stderr, "hunyuangraph_PartitionGraph: %s (%d)\n", hp_strerror(rc), rc);
        for (int i = 0; i < *nvtxs; i++) part[i] = -1;
    }
}
