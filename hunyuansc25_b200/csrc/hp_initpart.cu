// hp_initpart.cu — initial k-way partition of the coarsest graph by batched
// recursive bisection.
//
// Reference behaviour replaced (HunyuanGraph):
//   hunyuangraph_gpu_initialpartition        hunyuangraph_GPU_initialpartition.h:4405-4498
//   hunyuangraph_gpu_RecursiveBisection      :3913-4386  (one recursion call per
//     subgraph, each with its own launches and device->host reads)
//   per-warp BFS growth + 2-way FM           :2426, :3035 (curand start sampling)
//   hunyuangraph_gpu_SplitGraph_intersect    hunyuangraph_GPU_splitgraph.h:802-945
//   CPU growth / FM the trials follow        hunyuangraph_CPU_initialpartition.h:36-145,
//                                            hunyuangraph_CPU_2wayrefine.h:77-245
// Here every subgraph of one recursion depth lives in one "forest" CSR and a
// depth costs a fixed handful of launches: trials (one thread per start vertex
// of every subgraph), best-trial selection (one CTA per subgraph), and a
// scan-based split that builds the next depth's forest.  Start vertices are
// evenly spaced instead of random, FM's priority queue is ordered by
// (gain desc, vertex asc), so every trial is reproducible.
#include <algorithm>
#include <vector>

#include "hp_internal.cuh"
#include "hp_rowagg.cuh"

// Shared memory for the trial states of one CTA (<= 227 KB per CTA on B200).
#define HP_TRIAL_SMEM (200 * 1024)

namespace {

struct SubInfo {
    int32_t vbeg, n;
    int32_t tbeg, ntr;
    int64_t tv, want1, onemin, onemax;
    int64_t slab_off;
};

// One BFS-growth + FM bisection trial per warp.  Trial state lives in shared
// memory when the largest subgraph of the depth fits (else in a global slab).
//
// FM without a heap: the reference's priority queues
// (hunyuangraph_CPU_2wayrefine.h:117-225, hunyuangraph_priorityqueue.h) only
// ever hold the vertices v with bnd[v] && moved[v] == -1, keyed by ed[v]-id[v]
// (every insert/update/delete keeps that invariant), so popping side `from`
// is an argmax of (ed-id desc, v asc) over {bnd, not moved, where == from}.
// The warp computes that argmax in n/32 steps and updates the moved vertex's
// neighbours in parallel, which is exact and needs no heap maintenance on
// dense coarse graphs.
struct TrialState {
    int8_t *where, *bnd, *vis;
    int32_t *id, *ed, *moved, *swaps;   // swaps doubles as the BFS queue
};

__host__ __device__ inline int64_t state_bytes(int32_t n)
{
    return (((int64_t)3 * n + 15) & ~(int64_t)15) + (int64_t)16 * n + 16;
}

__device__ __forceinline__ TrialState carve(char *p, int32_t n)
{
    TrialState t;
    t.where = (int8_t *)p;
    t.bnd = t.where + n;
    t.vis = t.bnd + n;
    int32_t *ip = (int32_t *)(p + (((int64_t)3 * n + 15) & ~(int64_t)15));
    t.id = ip;
    t.ed = ip + n;
    t.moved = ip + 2 * n;
    t.swaps = ip + 3 * n;
    return t;
}

__global__ void __launch_bounds__(128)
trial_warp_kernel(const SubInfo *__restrict__ subs, const int32_t *__restrict__ trial_sub,
                  int32_t ntrials, const int32_t *__restrict__ fxadj, const int32_t *__restrict__ fadj,
                  const int32_t *__restrict__ fwgt, const int32_t *__restrict__ fvwgt, char *slab_base,
                  int32_t starts, int32_t fm_passes, int64_t *tr_cut, int64_t *tr_viol,
                  int use_smem, int64_t smem_per_warp)
{
    hp::pdl_wait();
    extern __shared__ __align__(16) char tsm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int32_t t = blockIdx.x * (blockDim.x >> 5) + wib;
    if (t >= ntrials) return;
    const SubInfo S = subs[trial_sub[t]];
    const int32_t lt = t - S.tbeg;
    const int32_t n = S.n;
    const int32_t *xadj = fxadj + S.vbeg;   // global edge offsets, local neighbour ids
    const int32_t *vwgt = fvwgt + S.vbeg;
    char *base = use_smem ? tsm + (int64_t)wib * smem_per_warp
                          : slab_base + S.slab_off + (int64_t)lt * state_bytes(n);
    TrialState T = carve(base, n);
    const int32_t start = (n <= starts) ? lt : (int32_t)(((int64_t)lt * n) / starts);
    const int64_t tv = S.tv, want1 = S.want1, onemin = S.onemin, onemax = S.onemax;
    int64_t pw0 = 0, pw1 = tv;

    // ---- BFS growth of side 0 (hunyuangraph_CPU_initialpartition.h:66-120)
    for (int32_t v = lane; v < n; v += 32) { T.where[v] = 1; T.vis[v] = 0; }
    __syncwarp();
    int32_t first = 0, last = 1, nleft = n - 1, next_unvis = 0;
    bool drain = false;
    if (lane == 0) { T.swaps[0] = start; T.vis[start] = 1; }
    __syncwarp();
    for (;;) {
        if (first == last) {
            if (nleft == 0 || drain) break;
            // lowest unvisited vertex
            for (;;) {
                int32_t v = next_unvis + lane;
                bool un = v < n && !T.vis[v];
                unsigned m = __ballot_sync(HP_FULL_MASK, un);
                if (m) { next_unvis += __ffs(m) - 1; break; }
                next_unvis += 32;
            }
            if (lane == 0) { T.swaps[0] = next_unvis; T.vis[next_unvis] = 1; }
            __syncwarp();
            first = 0; last = 1; nleft--;
        }
        const int32_t i = T.swaps[first++];
        const int32_t wi = vwgt[i];
        if (pw0 > 0 && pw1 - wi < onemin) { drain = true; continue; }
        if (lane == 0) T.where[i] = 0;
        pw0 += wi; pw1 -= wi;
        if (pw1 <= onemax) break;
        drain = false;
        for (int32_t base_j = xadj[i]; base_j < xadj[i + 1]; base_j += 32) {
            int32_t j = base_j + lane;
            int32_t k = -1;
            bool un = false;
            if (j < xadj[i + 1]) { k = fadj[j]; un = !T.vis[k]; }
            unsigned m = __ballot_sync(HP_FULL_MASK, un);
            if (un) { T.swaps[last + __popc(m & hp::lanemask_lt())] = k; T.vis[k] = 1; }
            last += __popc(m);
            nleft -= __popc(m);
            __syncwarp();
        }
    }
    __syncwarp();

    // ---- 2-way FM (hunyuangraph_CPU_2wayrefine.h:24-245)
    long long cut2 = 0;
    for (int32_t v = lane; v < n; v += 32) {
        int32_t tid = 0, ted = 0;
        const int8_t wv = T.where[v];
        for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) {
            if (T.where[fadj[j]] == wv) tid += fwgt[j];
            else ted += fwgt[j];
        }
        T.id[v] = tid; T.ed[v] = ted;
        T.bnd[v] = (ted > 0 || xadj[v] == xadj[v + 1]);
        cut2 += ted;
        T.moved[v] = -1;
    }
    int64_t cut = hp::warp_sum64(cut2) / 2;
    __syncwarp();
    const int64_t tpw0 = tv - want1, tpw1 = want1;
    int64_t limit = n / 100;
    if (limit < 15) limit = 15;
    if (limit > 100) limit = 100;
    int64_t avgvwgt = (pw0 + pw1) / 20;
    if (n > 0 && 2 * (pw0 + pw1) / n < avgvwgt) avgvwgt = 2 * (pw0 + pw1) / n;
    const int64_t origdiff = hp::iabs64(tpw0 - pw0);

    // neighbour update after h moved to `to`
    auto relax = [&](int32_t h, int to) {
        for (int32_t j = xadj[h] + lane; j < xadj[h + 1]; j += 32) {
            const int32_t k = fadj[j];
            const int32_t kw = (to == T.where[k]) ? fwgt[j] : -fwgt[j];
            const int32_t nid = T.id[k] + kw, ned = T.ed[k] - kw;
            T.id[k] = nid; T.ed[k] = ned;
            if (T.bnd[k]) { if (ned == 0) T.bnd[k] = 0; }
            else if (ned > 0) T.bnd[k] = 1;
        }
        __syncwarp();
    };

    for (int32_t pass = 0; pass < fm_passes; pass++) {
        int64_t mincutorder = -1;
        int64_t newcut = cut, mincut = cut, initcut = cut;
        int64_t mindiff = hp::iabs64(tpw0 - pw0);
        int32_t nswaps;
        for (nswaps = 0; nswaps < n; nswaps++) {
            const int from = (tpw0 - pw0 < tpw1 - pw1) ? 0 : 1;
            const int to = 1 - from;
            // pop: argmax (ed-id desc, v asc) over {bnd, not moved, side from}
            int32_t bh = -1, bk = 0;
            for (int32_t v = lane; v < n; v += 32) {
                if (T.bnd[v] && T.moved[v] == -1 && T.where[v] == from) {
                    int32_t key = T.ed[v] - T.id[v];
                    if (bh < 0 || key > bk) { bh = v; bk = key; }   // ascending v per lane
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                int32_t oh = __shfl_xor_sync(HP_FULL_MASK, bh, o);
                int32_t ok = __shfl_xor_sync(HP_FULL_MASK, bk, o);
                if (oh >= 0 && (bh < 0 || ok > bk || (ok == bk && oh < bh))) { bh = oh; bk = ok; }
            }
            const int32_t h = bh;
            if (h < 0) break;
            const int32_t gain = bk, wh = vwgt[h];
            newcut -= gain;
            if (to == 0) { pw0 += wh; pw1 -= wh; } else { pw1 += wh; pw0 -= wh; }
            if ((newcut < mincut && hp::iabs64(tpw0 - pw0) <= origdiff + avgvwgt) ||
                (newcut == mincut && hp::iabs64(tpw0 - pw0) < mindiff)) {
                mincut = newcut;
                mindiff = hp::iabs64(tpw0 - pw0);
                mincutorder = nswaps;
            } else if (nswaps - mincutorder > limit) {
                newcut += gain;
                if (to == 0) { pw0 -= wh; pw1 += wh; } else { pw1 -= wh; pw0 += wh; }
                break;
            }
            if (lane == 0) {
                T.where[h] = (int8_t)to;
                T.moved[h] = nswaps;
                T.swaps[nswaps] = h;
                int32_t tt = T.id[h]; T.id[h] = T.ed[h]; T.ed[h] = tt;
                if (T.ed[h] == 0 && xadj[h] < xadj[h + 1]) T.bnd[h] = 0;
            }
            __syncwarp();
            relax(h, to);
        }
        for (int32_t i = lane; i < nswaps; i += 32) T.moved[T.swaps[i]] = -1;
        __syncwarp();
        for (nswaps--; nswaps > mincutorder; nswaps--) {
            const int32_t h = T.swaps[nswaps];
            const int to = 1 - T.where[h];
            if (lane == 0) {
                T.where[h] = (int8_t)to;
                int32_t tt = T.id[h]; T.id[h] = T.ed[h]; T.ed[h] = tt;
                if (T.ed[h] == 0 && T.bnd[h] && xadj[h] < xadj[h + 1]) T.bnd[h] = 0;
                else if (T.ed[h] > 0 && !T.bnd[h]) T.bnd[h] = 1;
            }
            const int32_t wh = vwgt[h];
            if (to == 0) { pw0 += wh; pw1 -= wh; } else { pw1 += wh; pw0 -= wh; }
            __syncwarp();
            relax(h, to);
        }
        cut = mincut;
        if (mincutorder <= 0 || mincut == initcut) break;
    }
    int64_t viol = 0;
    if (pw1 > onemax) viol += pw1 - onemax;
    if (pw1 < onemin) viol += onemin - pw1;
    // the trial's sides go to the global slab for the selection kernel
    int8_t *wout = (int8_t *)(slab_base + S.slab_off + (int64_t)lt * state_bytes(n));
    if (use_smem)
        for (int32_t v = lane; v < n; v += 32) wout[v] = T.where[v];
    if (lane == 0) { tr_cut[t] = cut; tr_viol[t] = viol; }
}

// The same trial with one CTA of TC_THREADS threads per trial, for the large
// subgraphs of the first recursion depths: the FM pop is an argmax of n/256
// candidates per thread reduced across the warps, the BFS appends a row chunk's
// unvisited neighbours in row order through a block scan, and every decision
// is taken by all threads alike from shared values, so the trial's moves, cut
// and sides are those of trial_warp_kernel.
constexpr int TC_THREADS = 256;
constexpr int TC_WARPS = TC_THREADS / 32;

__device__ __forceinline__ int32_t tc_block_min(int32_t v, int32_t *s_red)
{
    v = __reduce_min_sync(HP_FULL_MASK, v);
    __syncthreads();   // earlier readers of s_red are done
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    int32_t r = INT_MAX;
#pragma unroll
    for (int w = 0; w < TC_WARPS; w++) r = min(r, s_red[w]);
    return r;
}

__global__ void __launch_bounds__(TC_THREADS)
trial_cta_kernel(const SubInfo *__restrict__ subs, const int32_t *__restrict__ trial_sub,
                 int32_t ntrials, const int32_t *__restrict__ fxadj, const int32_t *__restrict__ fadj,
                 const int32_t *__restrict__ fwgt, const int32_t *__restrict__ fvwgt, char *slab_base,
                 int32_t starts, int32_t fm_passes, int64_t *tr_cut, int64_t *tr_viol, int use_smem)
{
    hp::pdl_wait();
    extern __shared__ __align__(16) char tsm[];
    __shared__ int32_t s_red[TC_WARPS], s_key[TC_WARPS];
    __shared__ int32_t s_scan[TC_WARPS + 2];
    __shared__ long long s_cut[TC_WARPS];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int32_t t = blockIdx.x;
    if (t >= ntrials) return;   // whole CTA
    const SubInfo S = subs[trial_sub[t]];
    const int32_t lt = t - S.tbeg;
    const int32_t n = S.n;
    const int32_t *xadj = fxadj + S.vbeg;
    const int32_t *vwgt = fvwgt + S.vbeg;
    char *base = use_smem ? tsm : slab_base + S.slab_off + (int64_t)lt * state_bytes(n);
    TrialState T = carve(base, n);
    const int32_t start = (n <= starts) ? lt : (int32_t)(((int64_t)lt * n) / starts);
    const int64_t tv = S.tv, want1 = S.want1, onemin = S.onemin, onemax = S.onemax;
    int64_t pw0 = 0, pw1 = tv;

    // ---- BFS growth of side 0
    for (int32_t v = tid; v < n; v += TC_THREADS) { T.where[v] = 1; T.vis[v] = 0; }
    __syncthreads();
    int32_t first = 0, last = 1, nleft = n - 1, next_unvis = 0;
    bool drain = false;
    if (tid == 0) { T.swaps[0] = start; T.vis[start] = 1; }
    __syncthreads();
    for (;;) {
        if (first == last) {
            if (nleft == 0 || drain) break;
            for (;;) {   // lowest unvisited vertex
                const int32_t v = next_unvis + tid;
                const int32_t mv = tc_block_min(v < n && !T.vis[v] ? v : INT_MAX, s_red);
                if (mv != INT_MAX) { next_unvis = mv; break; }
                next_unvis += TC_THREADS;
            }
            __syncthreads();
            if (tid == 0) { T.swaps[0] = next_unvis; T.vis[next_unvis] = 1; }
            __syncthreads();
            first = 0; last = 1; nleft--;
        }
        const int32_t i = T.swaps[first++];
        const int32_t wi = vwgt[i];
        if (pw0 > 0 && pw1 - wi < onemin) { drain = true; continue; }
        __syncthreads();   // every thread has read swaps[first - 1]
        if (tid == 0) T.where[i] = 0;
        pw0 += wi; pw1 -= wi;
        if (pw1 <= onemax) break;
        drain = false;
        for (int32_t base_j = xadj[i]; base_j < xadj[i + 1]; base_j += TC_THREADS) {
            const int32_t j = base_j + tid;
            int32_t k = -1;
            bool un = false;
            if (j < xadj[i + 1]) { k = fadj[j]; un = !T.vis[k]; }
            int tot;
            const int ex = hp::block_excl_scan<TC_THREADS>(un ? 1 : 0, &tot, s_scan);
            if (un) { T.swaps[last + ex] = k; T.vis[k] = 1; }
            last += tot;
            nleft -= tot;
            __syncthreads();
        }
    }
    __syncthreads();

    // ---- 2-way FM
    long long cut2 = 0;
    for (int32_t v = tid; v < n; v += TC_THREADS) {
        int32_t tid_ = 0, ted = 0;
        const int8_t wv = T.where[v];
        for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) {
            if (T.where[fadj[j]] == wv) tid_ += fwgt[j];
            else ted += fwgt[j];
        }
        T.id[v] = tid_; T.ed[v] = ted;
        T.bnd[v] = (ted > 0 || xadj[v] == xadj[v + 1]);
        cut2 += ted;
        T.moved[v] = -1;
    }
    cut2 = hp::warp_sum64(cut2);
    if (lane == 0) s_cut[wid] = cut2;
    __syncthreads();
    long long call = 0;
#pragma unroll
    for (int w = 0; w < TC_WARPS; w++) call += s_cut[w];
    int64_t cut = call / 2;
    const int64_t tpw0 = tv - want1, tpw1 = want1;
    int64_t limit = n / 100;
    if (limit < 15) limit = 15;
    if (limit > 100) limit = 100;
    int64_t avgvwgt = (pw0 + pw1) / 20;
    if (n > 0 && 2 * (pw0 + pw1) / n < avgvwgt) avgvwgt = 2 * (pw0 + pw1) / n;
    const int64_t origdiff = hp::iabs64(tpw0 - pw0);

    auto relax = [&](int32_t h, int to) {
        for (int32_t j = xadj[h] + tid; j < xadj[h + 1]; j += TC_THREADS) {
            const int32_t k = fadj[j];
            const int32_t kw = (to == T.where[k]) ? fwgt[j] : -fwgt[j];
            const int32_t nid = T.id[k] + kw, ned = T.ed[k] - kw;
            T.id[k] = nid; T.ed[k] = ned;
            if (T.bnd[k]) { if (ned == 0) T.bnd[k] = 0; }
            else if (ned > 0) T.bnd[k] = 1;
        }
        __syncthreads();
    };

    for (int32_t pass = 0; pass < fm_passes; pass++) {
        int64_t mincutorder = -1;
        int64_t newcut = cut, mincut = cut, initcut = cut;
        int64_t mindiff = hp::iabs64(tpw0 - pw0);
        int32_t nswaps;
        for (nswaps = 0; nswaps < n; nswaps++) {
            const int from = (tpw0 - pw0 < tpw1 - pw1) ? 0 : 1;
            const int to = 1 - from;
            int32_t bh = -1, bk = 0;
            for (int32_t v = tid; v < n; v += TC_THREADS) {
                if (T.bnd[v] && T.moved[v] == -1 && T.where[v] == from) {
                    const int32_t key = T.ed[v] - T.id[v];
                    if (bh < 0 || key > bk) { bh = v; bk = key; }   // ascending v per thread
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const int32_t oh = __shfl_xor_sync(HP_FULL_MASK, bh, o);
                const int32_t ok = __shfl_xor_sync(HP_FULL_MASK, bk, o);
                if (oh >= 0 && (bh < 0 || ok > bk || (ok == bk && oh < bh))) { bh = oh; bk = ok; }
            }
            __syncthreads();   // earlier readers of s_red / s_key are done
            if (lane == 0) { s_red[wid] = bh; s_key[wid] = bk; }
            __syncthreads();
            bh = -1; bk = 0;
#pragma unroll
            for (int w = 0; w < TC_WARPS; w++) {
                const int32_t oh = s_red[w], ok = s_key[w];
                if (oh >= 0 && (bh < 0 || ok > bk || (ok == bk && oh < bh))) { bh = oh; bk = ok; }
            }
            const int32_t h = bh;
            if (h < 0) break;
            const int32_t gain = bk, wh = vwgt[h];
            newcut -= gain;
            if (to == 0) { pw0 += wh; pw1 -= wh; } else { pw1 += wh; pw0 -= wh; }
            if ((newcut < mincut && hp::iabs64(tpw0 - pw0) <= origdiff + avgvwgt) ||
                (newcut == mincut && hp::iabs64(tpw0 - pw0) < mindiff)) {
                mincut = newcut;
                mindiff = hp::iabs64(tpw0 - pw0);
                mincutorder = nswaps;
            } else if (nswaps - mincutorder > limit) {
                newcut += gain;
                if (to == 0) { pw0 -= wh; pw1 += wh; } else { pw1 -= wh; pw0 += wh; }
                break;
            }
            if (tid == 0) {
                T.where[h] = (int8_t)to;
                T.moved[h] = nswaps;
                T.swaps[nswaps] = h;
                int32_t tt = T.id[h]; T.id[h] = T.ed[h]; T.ed[h] = tt;
                if (T.ed[h] == 0 && xadj[h] < xadj[h + 1]) T.bnd[h] = 0;
            }
            __syncthreads();
            relax(h, to);
        }
        __syncthreads();
        for (int32_t i = tid; i < nswaps; i += TC_THREADS) T.moved[T.swaps[i]] = -1;
        __syncthreads();
        for (nswaps--; nswaps > mincutorder; nswaps--) {
            const int32_t h = T.swaps[nswaps];
            const int to = 1 - T.where[h];
            __syncthreads();   // every thread has read where[h]
            if (tid == 0) {
                T.where[h] = (int8_t)to;
                int32_t tt = T.id[h]; T.id[h] = T.ed[h]; T.ed[h] = tt;
                if (T.ed[h] == 0 && T.bnd[h] && xadj[h] < xadj[h + 1]) T.bnd[h] = 0;
                else if (T.ed[h] > 0 && !T.bnd[h]) T.bnd[h] = 1;
            }
            const int32_t wh = vwgt[h];
            if (to == 0) { pw0 += wh; pw1 -= wh; } else { pw1 += wh; pw0 -= wh; }
            __syncthreads();
            relax(h, to);
        }
        cut = mincut;
        if (mincutorder <= 0 || mincut == initcut) break;
    }
    int64_t viol = 0;
    if (pw1 > onemax) viol += pw1 - onemax;
    if (pw1 < onemin) viol += onemin - pw1;
    int8_t *wout = (int8_t *)(slab_base + S.slab_off + (int64_t)lt * state_bytes(n));
    if (use_smem)
        for (int32_t v = tid; v < n; v += TC_THREADS) wout[v] = T.where[v];
    if (tid == 0) { tr_cut[t] = cut; tr_viol[t] = viol; }
}

// Best trial of every subgraph: min (violation, cut, trial index); copies its
// sides into side[] and reports the side-0 vertex count and weight.
__global__ void __launch_bounds__(256)
select_kernel(const SubInfo *__restrict__ subs, const int64_t *__restrict__ tr_cut,
              const int64_t *__restrict__ tr_viol, const char *slab_base,
              const int32_t *__restrict__ fvwgt, int32_t *__restrict__ side,
              int64_t *__restrict__ res /* per sub: n0, tv0 */)
{
    hp::pdl_wait();
    __shared__ long long s_v[8], s_c[8];
    __shared__ int s_t[8];
    __shared__ int s_best;
    const SubInfo S = subs[blockIdx.x];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    long long bv = LLONG_MAX, bc = LLONG_MAX;
    int bt = INT_MAX;
    for (int t = threadIdx.x; t < S.ntr; t += blockDim.x) {
        long long v = tr_viol[S.tbeg + t], c = tr_cut[S.tbeg + t];
        if (v < bv || (v == bv && (c < bc || (c == bc && t < bt)))) { bv = v; bc = c; bt = t; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        long long ov = __shfl_xor_sync(HP_FULL_MASK, bv, o);
        long long oc = __shfl_xor_sync(HP_FULL_MASK, bc, o);
        int ot = __shfl_xor_sync(HP_FULL_MASK, bt, o);
        if (ov < bv || (ov == bv && (oc < bc || (oc == bc && ot < bt)))) { bv = ov; bc = oc; bt = ot; }
    }
    if (lane == 0) { s_v[wid] = bv; s_c[wid] = bc; s_t[wid] = bt; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++)
            if (s_v[w] < bv || (s_v[w] == bv && (s_c[w] < bc || (s_c[w] == bc && s_t[w] < bt)))) {
                bv = s_v[w]; bc = s_c[w]; bt = s_t[w];
            }
        s_best = bt;
    }
    __syncthreads();
    const int8_t *w = (const int8_t *)(slab_base + S.slab_off + (int64_t)s_best * state_bytes(S.n));
    long long n0 = 0, tv0 = 0;
    for (int i = threadIdx.x; i < S.n; i += blockDim.x) {
        int sd = w[i];
        side[S.vbeg + i] = sd;
        if (sd == 0) { n0++; tv0 += fvwgt[S.vbeg + i]; }
    }
    __shared__ unsigned long long s_acc[2];
    if (threadIdx.x == 0) { s_acc[0] = 0; s_acc[1] = 0; }
    __syncthreads();
    hp::block_add_to<256>(n0, &s_acc[0]);
    __syncthreads();
    hp::block_add_to<256>(tv0, &s_acc[1]);
    __syncthreads();
    if (threadIdx.x == 0) { res[2 * blockIdx.x] = (int64_t)s_acc[0]; res[2 * blockIdx.x + 1] = (int64_t)s_acc[1]; }
}

struct ChildMap {
    int32_t newbeg[2];   // first new vertex id of each side, -1 = side not carried on
    int32_t fpart[2];    // part of a final (single-part) side, -1 otherwise
};

__global__ void __launch_bounds__(256)
sub_of_kernel(const SubInfo *__restrict__ subs, int32_t *__restrict__ sub_of,
              int32_t *__restrict__ flag0)
{
    hp::pdl_wait();
    const SubInfo S = subs[blockIdx.x];
    for (int i = threadIdx.x; i < S.n; i += blockDim.x) sub_of[S.vbeg + i] = blockIdx.x;
    (void)flag0;
}

__global__ void __launch_bounds__(256)
side_flag_kernel(int32_t nf, const int32_t *__restrict__ side, int32_t *__restrict__ f0)
{
    hp::pdl_wait();
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < nf) f0[v] = side[v] == 0;
}

// New id of every forest vertex and its degree inside its side; final sides
// write the output partition directly.
__global__ void __launch_bounds__(256)
split_count_kernel(int32_t nf, const SubInfo *__restrict__ subs, const int32_t *__restrict__ sub_of,
                   const ChildMap *__restrict__ cm, const int32_t *__restrict__ side,
                   const int32_t *__restrict__ p0, const int32_t *__restrict__ fxadj,
                   const int32_t *__restrict__ fadj, const int32_t *__restrict__ label,
                   int32_t *__restrict__ newid, int32_t *__restrict__ ndeg, int32_t *__restrict__ where_out)
{
    hp::pdl_wait();
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nf) return;
    const int32_t s = sub_of[v];
    const SubInfo S = subs[s];
    const int sd = side[v];
    const ChildMap C = cm[s];
    if (C.fpart[sd] >= 0) where_out[label[v]] = C.fpart[sd];
    if (C.newbeg[sd] < 0) { newid[v] = -1; return; }
    int32_t r0 = p0[v] - p0[S.vbeg];
    int32_t rank = sd == 0 ? r0 : (v - S.vbeg) - r0;
    int32_t nid = C.newbeg[sd] + rank;
    newid[v] = nid;
    int32_t d = 0;
    for (int32_t j = fxadj[v]; j < fxadj[v + 1]; j++) d += side[S.vbeg + fadj[j]] == sd;
    ndeg[nid] = d;
}

__global__ void __launch_bounds__(256)
split_write_kernel(int32_t nf, const SubInfo *__restrict__ subs, const int32_t *__restrict__ sub_of,
                   const ChildMap *__restrict__ cm, const int32_t *__restrict__ side,
                   const int32_t *__restrict__ newid, const int32_t *__restrict__ fxadj,
                   const int32_t *__restrict__ fadj, const int32_t *__restrict__ fwgt,
                   const int32_t *__restrict__ fvwgt, const int32_t *__restrict__ label,
                   const int32_t *__restrict__ nxadj, int32_t *__restrict__ nadj,
                   int32_t *__restrict__ nwgt, int32_t *__restrict__ nvwgt, int32_t *__restrict__ nlabel)
{
    hp::pdl_wait();
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nf) return;
    const int32_t nid = newid[v];
    if (nid < 0) return;
    const int32_t s = sub_of[v];
    const SubInfo S = subs[s];
    const int sd = side[v];
    const int32_t nb = cm[s].newbeg[sd];
    nvwgt[nid] = fvwgt[v];
    nlabel[nid] = label[v];
    int32_t e = nxadj[nid];
    for (int32_t j = fxadj[v]; j < fxadj[v + 1]; j++) {
        int32_t u = S.vbeg + fadj[j];
        if (side[u] != sd) continue;
        nadj[e] = newid[u] - nb;
        nwgt[e] = fwgt[j];
        e++;
    }
}

__global__ void assign_all_kernel(int32_t n, int32_t *where, int32_t value)
{
    hp::pdl_wait();
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) where[v] = value;
}

__global__ void copy_kernel(int64_t n, const int32_t *src, int32_t *dst)
{
    hp::pdl_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

struct HostSub {
    int32_t vbeg, n;
    int32_t k, fpart;
    int64_t tv;
};

inline unsigned nblk(int64_t n, int b = 256) { return (unsigned)std::max<int64_t>(1, (n + b - 1) / b); }

}  // namespace

int hp_initpart_init()
{
    HP_CUDA(cudaFuncSetAttribute(trial_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)HP_TRIAL_SMEM));
    HP_CUDA(cudaFuncSetAttribute(trial_cta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)HP_TRIAL_SMEM));
    return HP_OK;
}

int hp_initial_partition(hp_context *c, HpLevel &g, int32_t nparts, const int64_t *h_tw,
                         int64_t ub2_fx, int32_t *d_where)
{
    const int32_t n = g.n;
    if (n == 0) return HP_OK;
    if (nparts == 1) {
        HP_LAUNCH(c, assign_all_kernel, nblk(n), 256, 0, n, d_where, 0);
        return HP_OK;
    }
    const int32_t starts = std::max(1, c->opt.init_starts);
    const int32_t fm_passes = std::max(0, c->opt.fm_passes);
    const size_t mark = c->hi;

    // forest of depth 0 = the coarsest graph itself (labels = ids)
    int32_t nf = n;
    int64_t mf = g.m;
    int32_t *fxadj = ralloc_t<int32_t>(c, nf + 1), *fadj = ralloc_t<int32_t>(c, mf);
    int32_t *fwgt = ralloc_t<int32_t>(c, mf), *fvwgt = ralloc_t<int32_t>(c, nf);
    int32_t *flabel = ralloc_t<int32_t>(c, nf);
    // ping-pong forest
    int32_t *gxadj = ralloc_t<int32_t>(c, nf + 1), *gadj = ralloc_t<int32_t>(c, mf);
    int32_t *gwgt = ralloc_t<int32_t>(c, mf), *gvwgt = ralloc_t<int32_t>(c, nf);
    int32_t *glabel = ralloc_t<int32_t>(c, nf);
    int32_t *side = ralloc_t<int32_t>(c, nf), *p0 = ralloc_t<int32_t>(c, nf + 1);
    int32_t *sub_of = ralloc_t<int32_t>(c, nf), *newid = ralloc_t<int32_t>(c, nf);
    int32_t *ndeg = ralloc_t<int32_t>(c, nf + 1);
    HP_CHECK_OOM(c);
    HP_LAUNCH(c, copy_kernel, nblk(nf + 1), 256, 0, (int64_t)nf + 1, g.xadj, fxadj);
    HP_LAUNCH(c, copy_kernel, nblk(mf), 256, 0, mf, g.adjncy, fadj);
    HP_LAUNCH(c, copy_kernel, nblk(mf), 256, 0, mf, g.adjwgt, fwgt);
    HP_LAUNCH(c, copy_kernel, nblk(nf), 256, 0, (int64_t)nf, g.vwgt, fvwgt);
    HP_TRY(hp_iota_i32(c, flabel, nf));

    // total vertex weight of the coarsest graph
    std::vector<int32_t> hv(nf);
    HP_CUDA(cudaMemcpyAsync(hv.data(), g.vwgt, sizeof(int32_t) * (size_t)nf, cudaMemcpyDeviceToHost, c->stream));
    HP_CUDA(cudaStreamSynchronize(c->stream));
    int64_t tv0 = 0;
    for (int32_t v = 0; v < nf; v++) tv0 += hv[v];

    std::vector<HostSub> subs{{0, nf, nparts, 0, tv0}};
    while (!subs.empty()) {
        const int ns = (int)subs.size();
        std::vector<SubInfo> info(ns);
        std::vector<int32_t> trial_sub;
        int64_t slab_total = 0;
        int32_t tcount = 0;
        for (int s = 0; s < ns; s++) {
            const HostSub &H = subs[s];
            SubInfo &I = info[s];
            const int32_t kl = H.k >> 1;
            int64_t wl = 0, wr = 0;
            for (int32_t p = 0; p < kl; p++) wl += h_tw[H.fpart + p];
            for (int32_t p = kl; p < H.k; p++) wr += h_tw[H.fpart + p];
            I.vbeg = H.vbeg; I.n = H.n; I.tv = H.tv;
            I.want1 = (wl + wr) > 0 ? (H.tv * wr) / (wl + wr) : H.tv / 2;
            I.onemax = (I.want1 * ub2_fx) >> 16;
            I.onemin = (I.want1 << 16) / ub2_fx;
            I.ntr = H.n <= starts ? H.n : starts;
            I.tbeg = tcount;
            I.slab_off = slab_total;
            slab_total += (int64_t)I.ntr * state_bytes(H.n);
            for (int32_t t = 0; t < I.ntr; t++) trial_sub.push_back(s);
            tcount += I.ntr;
        }
        const size_t dmark = c->hi;
        SubInfo *d_info = ralloc_t<SubInfo>(c, ns);
        int32_t *d_tsub = ralloc_t<int32_t>(c, tcount);
        int64_t *d_cut = ralloc_t<int64_t>(c, tcount), *d_viol = ralloc_t<int64_t>(c, tcount);
        char *slab = (char *)hp_ralloc(c, (size_t)slab_total);
        int64_t *d_res = ralloc_t<int64_t>(c, 2 * (int64_t)ns);
        ChildMap *d_cm = ralloc_t<ChildMap>(c, ns);
        HP_CHECK_OOM(c);
        HP_CUDA(cudaMemcpyAsync(d_info, info.data(), sizeof(SubInfo) * ns, cudaMemcpyHostToDevice, c->stream));
        HP_CUDA(cudaMemcpyAsync(d_tsub, trial_sub.data(), sizeof(int32_t) * tcount, cudaMemcpyHostToDevice, c->stream));
        // trial state in shared memory when the largest subgraph fits
        int32_t maxn = 0;
        for (const HostSub &H : subs) maxn = std::max(maxn, H.n);
        const int64_t per = (state_bytes(maxn) + 15) & ~(int64_t)15;
        const int wpb = (int)std::max<int64_t>(1, std::min<int64_t>(4, HP_TRIAL_SMEM / per));
        const int use_smem = per <= HP_TRIAL_SMEM ? 1 : 0;
        const int wpb_eff = use_smem ? wpb : 4;
        const int tok = hp_prof_begin(c);
        if (maxn >= c->tune.trial_cta_n)   // a CTA per trial (same trial, same result)
            HP_LAUNCH(c, trial_cta_kernel, (unsigned)tcount, TC_THREADS, use_smem ? (size_t)per : 0, d_info, d_tsub,
                      tcount, fxadj, fadj, fwgt, fvwgt, slab, starts, fm_passes, d_cut, d_viol, use_smem);
        else
            HP_LAUNCH(c, trial_warp_kernel, nblk(tcount, wpb_eff), 32 * wpb_eff,
                      use_smem ? (size_t)(per * wpb_eff) : 0, d_info, d_tsub, tcount, fxadj, fadj, fwgt, fvwgt,
                      slab, starts, fm_passes, d_cut, d_viol, use_smem, per);
        hp_prof_end(c, tok, HP_PROF_INIT, 0);
        HP_LAUNCH(c, select_kernel, (unsigned)ns, 256, 0, d_info, d_cut, d_viol, slab, fvwgt, side, d_res);
        std::vector<int64_t> res(2 * ns);
        HP_CUDA(cudaMemcpyAsync(res.data(), d_res, sizeof(int64_t) * 2 * ns, cudaMemcpyDeviceToHost, c->stream));
        HP_CUDA(cudaStreamSynchronize(c->stream));

        // children
        std::vector<ChildMap> cm(ns);
        std::vector<HostSub> next;
        int32_t nnew = 0;
        for (int s = 0; s < ns; s++) {
            const HostSub &H = subs[s];
            const int32_t kl = H.k >> 1;
            const int32_t cn[2] = {(int32_t)res[2 * s], H.n - (int32_t)res[2 * s]};
            const int64_t ctv[2] = {res[2 * s + 1], H.tv - res[2 * s + 1]};
            const int32_t ck[2] = {kl, H.k - kl};
            const int32_t cf[2] = {H.fpart, H.fpart + kl};
            for (int sd = 0; sd < 2; sd++) {
                cm[s].fpart[sd] = ck[sd] == 1 ? cf[sd] : -1;
                if (ck[sd] >= 2 && cn[sd] > 0) {
                    cm[s].newbeg[sd] = nnew;
                    next.push_back({nnew, cn[sd], ck[sd], cf[sd], ctv[sd]});
                    nnew += cn[sd];
                } else {
                    cm[s].newbeg[sd] = -1;
                }
            }
        }
        HP_CUDA(cudaMemcpyAsync(d_cm, cm.data(), sizeof(ChildMap) * ns, cudaMemcpyHostToDevice, c->stream));
        HP_LAUNCH(c, sub_of_kernel, (unsigned)ns, 256, 0, d_info, sub_of, (int32_t *)nullptr);
        HP_LAUNCH(c, side_flag_kernel, nblk(nf), 256, 0, nf, side, p0);
        HP_TRY(hp_scan_excl(c, p0, p0, nf));
        HP_LAUNCH(c, split_count_kernel, nblk(nf), 256, 0, nf, d_info, sub_of, d_cm, side, p0, fxadj,
                  fadj, flabel, newid, ndeg, d_where);
        if (nnew > 0) {
            HP_TRY(hp_scan_excl(c, ndeg, gxadj, nnew));
            HP_LAUNCH(c, split_write_kernel, nblk(nf), 256, 0, nf, d_info, sub_of, d_cm, side, newid,
                      fxadj, fadj, fwgt, fvwgt, flabel, gxadj, gadj, gwgt, gvwgt, glabel);
        }
        HP_CUDA(cudaStreamSynchronize(c->stream));
        c->hi = dmark;
        std::swap(fxadj, gxadj); std::swap(fadj, gadj); std::swap(fwgt, gwgt);
        std::swap(fvwgt, gvwgt); std::swap(flabel, glabel);
        nf = nnew;
        subs.swap(next);
    }
    HP_TRY(hp_check_status(c));
    c->hi = mark;
    return HP_OK;
}
