// hp_coarsen.cu — deterministic heavy-edge matching and contraction, level loop.
//
// Reference behaviour replaced (HunyuanGraph):
//   level loop, maxvwgt, stop rule     hunyuangraph_GPU_coarsen.h:163-253
//   matching driver                    hunyuangraph_GPU_match.h:1846-3214
//     mutual top-k proposals           :800-861   (here: mutual best proposal,
//                                      heaviest edge / seeded tie key / lowest id)
//     leaf, relative, isolate, forced  :1374-1716 (gated at 75 % matched, :2577)
//     cmap / cvwgt / coarse row bound  :1012-1096
//   contraction                        hunyuangraph_GPU_contraction.h:715-1247
//     (scatter -> segmented sort -> mark -> scan -> write; here each coarse
//      row gathers both fine rows, merges equal coarse neighbours and is
//      written sorted, by size class (default bounds; hp_tuning fields):
//        <= 32 entries    staged per tile of 256 rows in shared memory, one
//                         thread's bitonic network in registers, written in
//                         place by one ordered pass with a decoupled look-back
//                         that also produces the coarse xadj
//        33..256          one warp, LSD radix sort in shared memory
//        257..4096        one CTA of 256, LSD radix sort in shared memory
//        4097..12288      one CTA of 1024, LSD radix sort in shared memory
//        larger           one CTA, dense accumulator + presence bitmap
//        (a level whose coarse ids fit contract_smem_cn merges every long row
//         in a shared-memory dense accumulator instead)
//      the long classes go through a temporary buffer and are copied to their
//      final offsets)
//   small levels (at most small_match_n vertices): one CTA runs the whole
//   matching of the level in one launch (match_small_kernel)
// The reference's matching is an atomicCAS race (nondeterministic); every
// decision here is a pure function of the level's CSR and the seed, so the
// CPU oracle reproduces each level bit for bit.
#include <cstdlib>

#include "hp_internal.cuh"
#include "hp_rowagg.cuh"

namespace {

// Row classes of matching (hp_tuning): rows of at most match_warp_deg entries
// take a thread, longer rows a warp, rows above match_cta_deg a CTA.

// ---------------------------------------------------------------------------
// matching

// ELIG: handshake proposal (unmatched neighbour, weight cap).  !ELIG: hub
// choice for two-hop matching (any neighbour).
//
// Rounds after the first keep a proposal that is still valid: between rounds
// the eligible set of a vertex only shrinks (neighbours get matched; weights
// and the cap do not change), so if the previous best neighbour is still
// unmatched it is still the best, and an empty set stays empty.  Only vertices
// whose choice was matched away rescan their row (same result as a full rescan).
__device__ __forceinline__ bool keep_proposal(bool later_round, int32_t v, const int32_t *__restrict__ pref,
                                              const int32_t *__restrict__ elig)
{
    if (!later_round) return false;
    const int32_t pu = pref[v];
    return pu < 0 || elig[pu] != INT_MAX;
}

// Running best candidate with a lazily computed tie key: a strictly heavier
// edge wins without hashing, and the seeded tie key is computed only when
// weights tie (and for the final best, before reductions compare it).  The
// order is exactly hp::better's.
struct BestCand {
    int32_t u = -1, w = 0;
    uint32_t h = 0;
    bool hv = false;
    __device__ __forceinline__ void offer(uint64_t lkey, int32_t v, int32_t cu, int32_t cw)
    {
        if (u < 0 || cw > w) { u = cu; w = cw; hv = false; return; }
        if (cw < w) return;
        if (!hv) { h = hp::edge_tie(lkey, v, u); hv = true; }
        const uint32_t ch = hp::edge_tie(lkey, v, cu);
        if (ch < h || (ch == h && cu < u)) { u = cu; h = ch; }
    }
    __device__ __forceinline__ void finish(uint64_t lkey, int32_t v)
    {
        if (u >= 0 && !hv) { h = hp::edge_tie(lkey, v, u); hv = true; }
    }
};

// The best candidate of the warp in hp::better order (heavier edge, then lower
// tie key, then lower id) among the lanes holding one (bu >= 0), in every lane:
// three warp reductions (redux.sync) in place of a shuffle butterfly.  Edge
// weights are positive, so w + 1 > 0 marks a held candidate.
__device__ __forceinline__ void warp_best(int32_t &bu, int32_t &bw, uint32_t &bh)
{
    const unsigned wk = bu >= 0 ? (unsigned)bw + 1u : 0u;
    const unsigned wm = __reduce_max_sync(HP_FULL_MASK, wk);
    const bool c1 = wm != 0u && wk == wm;
    const unsigned hm = __reduce_min_sync(HP_FULL_MASK, c1 ? bh : 0xffffffffu);
    const bool c2 = c1 && bh == hm;
    const unsigned um = __reduce_min_sync(HP_FULL_MASK, c2 ? (unsigned)bu : 0xffffffffu);
    if (wm == 0u) {
        bu = -1; bw = 0; bh = 0u;
        return;
    }
    bu = (int32_t)um; bw = (int32_t)(wm - 1u); bh = hm;
}

constexpr int PREF_BATCH = 4;

template <bool ELIG>
__global__ void __launch_bounds__(256)
pref_small_kernel(int32_t n, const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                  const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ vwgt,
                  const int32_t *__restrict__ match, const int32_t *__restrict__ elig, int32_t *__restrict__ pref,
                  uint64_t lkey, int64_t maxvwgt, const unsigned long long *made_prev, int32_t warp_deg)
{
    hp::pdl_wait();
    if (made_prev && *made_prev == 0ull) return;
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int32_t b = xadj[v], e = xadj[v + 1];
    if (e - b > warp_deg) return;
    if (match[v] != -1) { pref[v] = -1; return; }
    if (ELIG && keep_proposal(made_prev != nullptr, v, pref, elig)) return;
    const int32_t wv = vwgt[v];
    BestCand best;
    // PREF_BATCH entries at a time: the row loads, then the neighbour gathers,
    // are issued together so each thread keeps several misses in flight
    for (int32_t j0 = b; j0 < e; j0 += PREF_BATCH) {
        int32_t u[PREF_BATCH], w[PREF_BATCH], eu[PREF_BATCH];
#pragma unroll
        for (int q = 0; q < PREF_BATCH; q++) {
            const bool in = j0 + q < e;
            u[q] = in ? adjncy[j0 + q] : v;
            w[q] = in ? adjwgt[j0 + q] : 0;
        }
#pragma unroll
        for (int q = 0; q < PREF_BATCH; q++) eu[q] = (ELIG && u[q] != v) ? elig[u[q]] : 0;
#pragma unroll
        for (int q = 0; q < PREF_BATCH; q++) {
            if (u[q] == v) continue;
            if (ELIG) {
                if (eu[q] == INT_MAX) continue;                     // matched
                if ((int64_t)wv + eu[q] > maxvwgt) continue;        // weight cap
            }
            best.offer(lkey, v, u[q], w[q]);
        }
    }
    pref[v] = best.u;
}

template <bool ELIG>
__global__ void __launch_bounds__(256)
pref_big_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ vwgt,
                const int32_t *__restrict__ match, const int32_t *__restrict__ elig, int32_t *__restrict__ pref,
                uint64_t lkey, int64_t maxvwgt, const unsigned long long *made_prev)
{
    hp::pdl_wait();
    if (made_prev && *made_prev == 0ull) return;
    const int lane = threadIdx.x & 31;
    const int32_t cnt = *d_count;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < cnt;
         i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int32_t v = list[i];
        if (match[v] != -1) { if (lane == 0) pref[v] = -1; continue; }
        if (ELIG && keep_proposal(made_prev != nullptr, v, pref, elig)) continue;
        const int32_t wv = vwgt[v];
        BestCand best;
        for (int32_t j = xadj[v] + lane; j < xadj[v + 1]; j += 32) {
            int32_t u = adjncy[j];
            if (u == v) continue;
            if (ELIG) {
                const int32_t eu = elig[u];
                if (eu == INT_MAX) continue;                     // matched
                if ((int64_t)wv + eu > maxvwgt) continue;        // weight cap
            }
            best.offer(lkey, v, u, adjwgt[j]);
        }
        best.finish(lkey, v);
        int32_t bu = best.u, bw = best.w;
        uint32_t bh = best.h;
        warp_best(bu, bw, bh);
        if (lane == 0) pref[v] = bu;
    }
}

// ---- handshake proposals of long rows with a top-4 candidate cache ---------------
// A full scan of a long row keeps the TOPK best eligible candidates (in
// hp::better order).  Between rounds the eligible set only shrinks, so in a
// later round the first cached candidate that is still unmatched is exactly the
// best eligible neighbour; if the cache held fewer than TOPK candidates its
// exhaustion means none is left.  Only a vertex whose full cache was matched
// away rescans its row.  Results equal a full rescan every round.  (Eight
// candidates made the R-MAT matching slower: the first round's scans nearly
// doubled and the later rounds did not get cheaper.)
constexpr int TOPK = 4;

// The TOPK best candidates of a row, kept by a whole warp: every lane holds the
// same list, best first (u = -1 in the unused slots).  Entries are offered one
// per lane; only those that can enter (weight at least the last held weight once
// the list is full) are hashed and merged, best first by warp_best, until the
// best remaining one cannot enter -- so after the first few batches of a row an
// offer costs one ballot.  The list is the TOPK best of everything offered,
// whatever the order of the offers (hp::better is a total order on distinct ids).
struct WarpTop {
    int32_t u[TOPK], w[TOPK];
    uint32_t h[TOPK];
    __device__ __forceinline__ void init()
    {
#pragma unroll
        for (int q = 0; q < TOPK; q++) { u[q] = -1; w[q] = 0; h[q] = 0u; }
    }
    __device__ __forceinline__ bool full() const { return u[TOPK - 1] >= 0; }
    // the same candidate in every lane; it is better than the last entry or the list is not full
    __device__ __forceinline__ void insert(int32_t cu, int32_t cw, uint32_t ch)
    {
#pragma unroll
        for (int q = 0; q < TOPK; q++) {
            if (cu >= 0 && (u[q] < 0 || hp::better(cw, ch, cu, w[q], h[q], u[q]))) {
                const int32_t tu = u[q], tw = w[q];
                const uint32_t th = h[q];
                u[q] = cu; w[q] = cw; h[q] = ch;
                cu = tu; cw = tw; ch = th;
            }
        }
    }
    // Merges the lanes' candidates (cu < 0: none) whose tie keys are known; all
    // lanes call.  At most TOPK insertions and one failed test.
    __device__ __forceinline__ void merge(int32_t cu, int32_t cw, uint32_t ch)
    {
        for (;;) {
            int32_t bu = cu, bw = cw;
            uint32_t bh = ch;
            warp_best(bu, bw, bh);
            if (bu < 0) return;
            if (full() && !hp::better(bw, bh, bu, w[TOPK - 1], h[TOPK - 1], u[TOPK - 1])) return;
            insert(bu, bw, bh);
            if (cu == bu) cu = -1;
        }
    }
    // Offers one entry of v's row per lane (cu < 0: none); all lanes call.
    __device__ __forceinline__ void offer(uint64_t lkey, int32_t v, int32_t cu, int32_t cw)
    {
        const bool c = cu >= 0 && (!full() || cw >= w[TOPK - 1]);
        if (!__ballot_sync(HP_FULL_MASK, c)) return;
        merge(c ? cu : -1, cw, c ? hp::edge_tie(lkey, v, cu) : 0u);
    }
    // u[q] of lane q (q < TOPK), -1 elsewhere
    __device__ __forceinline__ int32_t lane_entry() const
    {
        const int lane = threadIdx.x & 31;
        int32_t r = -1;
#pragma unroll
        for (int q = 0; q < TOPK; q++)
            if (lane == q) r = u[q];
        return r;
    }
};

// The entries [j0, e) of v's row, `step` apart per batch of 4 x 32 (the warp's
// share: j0 and step are the same in all its lanes), offered to the warp's list.
// The four row loads of a lane, then their eligibility gathers, are in flight
// together.
__device__ __forceinline__ void scan_row_top(WarpTop &t, int32_t v, int32_t j0, int32_t e, int32_t step,
                                             const int32_t *__restrict__ adjncy, const int32_t *__restrict__ adjwgt,
                                             const int32_t *__restrict__ elig, int32_t wv, uint64_t lkey,
                                             int64_t maxvwgt)
{
    const int lane = threadIdx.x & 31;
    for (int32_t j = j0; j < e; j += step) {
        int32_t u[4], w[4], eu[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int32_t jj = j + lane + 32 * q;
            const bool in = jj < e;
            u[q] = in ? adjncy[jj] : v;
            w[q] = in ? adjwgt[jj] : 0;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) eu[q] = u[q] != v ? elig[u[q]] : INT_MAX;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            // matched (or no entry), or over the weight cap: not a candidate
            const bool ok = eu[q] != INT_MAX && (int64_t)wv + eu[q] <= maxvwgt;
            t.offer(lkey, v, ok ? u[q] : -1, w[q]);
        }
    }
}

// Later rounds: the proposal from the cache, or -2 when the row must be
// rescanned.  All 32 lanes call with the same v: lane q < TOPK checks entry q,
// so the cache costs two dependent loads whatever its length.  The first entry
// (in cache order) that is empty (-1: the cache held every eligible candidate)
// or still unmatched (the best now) decides.
static_assert(TOPK <= 32, "one cache entry per lane");
__device__ __forceinline__ int32_t cached_proposal(const int32_t *__restrict__ cand, int32_t v,
                                                  const int32_t *__restrict__ elig)
{
    const int lane = threadIdx.x & 31;
    const int32_t cu = lane < TOPK ? cand[(int64_t)v * TOPK + lane] : INT_MAX;
    const bool empty = lane < TOPK && cu < 0;
    const bool live = lane < TOPK && cu >= 0 && elig[cu] != INT_MAX;
    const unsigned em = __ballot_sync(HP_FULL_MASK, empty), lm = __ballot_sync(HP_FULL_MASK, live);
    const unsigned ev = em | lm;
    if (!ev) return -2;
    const int f = __ffs(ev) - 1;
    const int32_t pick = __shfl_sync(HP_FULL_MASK, cu, f);
    return (em >> f) & 1u ? -1 : pick;
}

__global__ void __launch_bounds__(256)
pref_big_topk_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                     const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                     const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ vwgt,
                     const int32_t *__restrict__ match, const int32_t *__restrict__ elig,
                     int32_t *__restrict__ pref, int32_t *__restrict__ cand, uint64_t lkey, int64_t maxvwgt,
                     const unsigned long long *made_prev)
{
    hp::pdl_wait();
    if (made_prev && *made_prev == 0ull) return;
    const int lane = threadIdx.x & 31;
    const int32_t cnt = *d_count;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < cnt;
         i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int32_t v = list[i];
        if (match[v] != -1) { if (lane == 0) pref[v] = -1; continue; }
        if (made_prev) {
            const int32_t cp = cached_proposal(cand, v, elig);
            if (cp != -2) { if (lane == 0) pref[v] = cp; continue; }
        }
        WarpTop t;
        t.init();
        scan_row_top(t, v, xadj[v], xadj[v + 1], 4 * 32, adjncy, adjwgt, elig, vwgt[v], lkey, maxvwgt);
        const int32_t mine = t.lane_entry();
        if (lane < TOPK) cand[(int64_t)v * TOPK + lane] = mine;
        if (lane == 0) pref[v] = t.u[0];
    }
}

// CTA per row for rows above match_cta_deg: each warp keeps the list of its
// batches of the row, then warp 0 merges the warps' lists.
constexpr int HUGE_TOPK_THREADS = 512;

__global__ void __launch_bounds__(HUGE_TOPK_THREADS)
pref_huge_topk_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                      const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                      const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ vwgt,
                      const int32_t *__restrict__ match, const int32_t *__restrict__ elig,
                      int32_t *__restrict__ pref, int32_t *__restrict__ cand, uint64_t lkey, int64_t maxvwgt,
                      const unsigned long long *made_prev)
{
    hp::pdl_wait();
    if (made_prev && *made_prev == 0ull) return;
    constexpr int NW = HUGE_TOPK_THREADS / 32;
    __shared__ int32_t su[TOPK][NW], sw[TOPK][NW];
    __shared__ uint32_t sh[TOPK][NW];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t v = list[li];
        if (match[v] != -1) { if (threadIdx.x == 0) pref[v] = -1; continue; }
        if (made_prev) {
            const int32_t cp = cached_proposal(cand, v, elig);
            if (cp != -2) { if (threadIdx.x == 0) pref[v] = cp; continue; }
        }
        WarpTop t;
        t.init();
        scan_row_top(t, v, xadj[v] + 4 * 32 * wid, xadj[v + 1], 4 * 32 * NW, adjncy, adjwgt, elig, vwgt[v], lkey,
                     maxvwgt);
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < TOPK; q++) { su[q][wid] = t.u[q]; sw[q][wid] = t.w[q]; sh[q][wid] = t.h[q]; }
        }
        __syncthreads();
        if (wid == 0) {
            WarpTop m;
            m.init();
#pragma unroll
            for (int q = 0; q < TOPK; q++) {
                const bool in = lane < NW;
                m.merge(in ? su[q][lane] : -1, in ? sw[q][lane] : 0, in ? sh[q][lane] : 0u);
            }
            const int32_t mine = m.lane_entry();
            if (lane < TOPK) cand[(int64_t)v * TOPK + lane] = mine;
            if (lane == 0) pref[v] = m.u[0];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256)
commit_kernel(int32_t n, int32_t *__restrict__ match, const int32_t *__restrict__ pref,
              int32_t *__restrict__ elig, unsigned long long *made_cur, const unsigned long long *made_prev)
{
    hp::pdl_wait();
    if (made_prev && *made_prev == 0ull) return;
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    int made = 0;
    if (v < n && match[v] == -1) {
        int32_t u = pref[v];
        if (u >= 0 && pref[u] == v) {
            match[v] = u;
            elig[v] = INT_MAX;   // no longer a candidate of anyone
            made = 1;
        }
    }
    hp::block_add_to<256>(made, made_cur);
}

__global__ void __launch_bounds__(256)
big_list_kernel(int32_t n, const int32_t *__restrict__ xadj, int32_t *list, int32_t *d_count,
                int32_t *huge, int32_t *d_huge, const int32_t *__restrict__ vwgt, int32_t *__restrict__ elig,
                int32_t warp_deg, int32_t cta_deg)
{
    hp::pdl_wait();
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t d = 0;
    if (v < n) {
        elig[v] = vwgt[v];   // every vertex starts unmatched
        d = xadj[v + 1] - xadj[v];
    }
    const bool is_huge = v < n && d > cta_deg, is_big = v < n && !is_huge && d > warp_deg;
    const int32_t ph = hp::warp_append(d_huge, is_huge);
    const int32_t pb = hp::warp_append(d_count, is_big);
    if (is_huge) huge[ph] = v;
    if (is_big) list[pb] = v;
}

// CTA per vertex for rows longer than match_cta_deg (R-MAT hubs).
template <bool ELIG>
__global__ void __launch_bounds__(512)
pref_huge_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                 const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                 const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ vwgt,
                 const int32_t *__restrict__ match, const int32_t *__restrict__ elig, int32_t *__restrict__ pref,
                 uint64_t lkey, int64_t maxvwgt, const unsigned long long *made_prev)
{
    hp::pdl_wait();
    if (made_prev && *made_prev == 0ull) return;
    __shared__ int32_t su[16], sw[16];
    __shared__ uint32_t sh[16];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t v = list[li];
        if (match[v] != -1) { if (threadIdx.x == 0) pref[v] = -1; continue; }
        if (ELIG && keep_proposal(made_prev != nullptr, v, pref, elig)) continue;
        const int32_t wv = vwgt[v];
        BestCand best;
        for (int32_t j = xadj[v] + threadIdx.x; j < xadj[v + 1]; j += blockDim.x) {
            int32_t u = adjncy[j];
            if (u == v) continue;
            if (ELIG) {
                const int32_t eu = elig[u];
                if (eu == INT_MAX) continue;                     // matched
                if ((int64_t)wv + eu > maxvwgt) continue;        // weight cap
            }
            best.offer(lkey, v, u, adjwgt[j]);
        }
        best.finish(lkey, v);
        int32_t bu = best.u, bw = best.w;
        uint32_t bh = best.h;
        warp_best(bu, bw, bh);
        if (lane == 0) { su[wid] = bu; sw[wid] = bw; sh[wid] = bh; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w2 = 1; w2 < (int)(blockDim.x >> 5); w2++)
                if (su[w2] >= 0 && (bu < 0 || hp::better(sw[w2], sh[w2], su[w2], bw, bh, bu))) {
                    bu = su[w2]; bw = sw[w2]; bh = sh[w2];
                }
            pref[v] = bu;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256)
count_matched_kernel(int32_t n, const int32_t *__restrict__ match, unsigned long long *out)
{
    hp::pdl_wait();
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    hp::block_add_to<256>((v < n && match[v] != -1) ? 1 : 0, out);
}

// Two-hop pairing.  The clients of hub h (unmatched vertices whose hub is h)
// are paired in h's row order -- (c0,c1), (c2,c3), ... when the weight sum
// fits.  Rows are sorted by neighbour id, so h's row order is ascending client
// id, and the pairs follow from the clients sorted stably by hub: a client at
// an odd offset in its hub's run pairs with the one before it.  The work is
// proportional to the number of clients, not to the length of the hubs' rows.
__global__ void __launch_bounds__(256)
client_flag_kernel(int32_t n, const int32_t *__restrict__ match, const int32_t *__restrict__ hub,
                   int32_t *__restrict__ flags)
{
    hp::pdl_wait();
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) flags[v] = match[v] == -1 && hub[v] >= 0;
}

__global__ void __launch_bounds__(256)
client_keys_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                   const int32_t *__restrict__ hub, int32_t *__restrict__ keys)
{
    hp::pdl_wait();
    const int32_t cnt = *d_count;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x)
        keys[i] = hub[list[i]];
}

__global__ void __launch_bounds__(256)
pair_clients_kernel(const int32_t *__restrict__ keys, const int32_t *__restrict__ vals,
                    const int32_t *__restrict__ d_count, const int32_t *__restrict__ vwgt,
                    int32_t *__restrict__ match, int64_t maxvwgt)
{
    hp::pdl_wait();
    const int32_t cnt = *d_count;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t h = keys[i];
        int32_t lo = 0, hi = (int32_t)i;   // first index of the run of h
        while (lo < hi) {
            const int32_t mid = (lo + hi) >> 1;
            if (keys[mid] < h) lo = mid + 1; else hi = mid;
        }
        if (((int32_t)i - lo) & 1) {
            const int32_t a = vals[i - 1], b = vals[i];
            if ((int64_t)vwgt[a] + vwgt[b] <= maxvwgt) { match[a] = b; match[b] = a; }
        }
    }
}

__global__ void __launch_bounds__(256)
flag_unmatched_kernel(int32_t n, const int32_t *__restrict__ xadj,
                      const int32_t *__restrict__ match, int32_t *__restrict__ flags, int isolated_only)
{
    hp::pdl_wait();
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    int f = match[v] == -1;
    if (isolated_only) f = f && (xadj[v] == xadj[v + 1]);
    flags[v] = f;
}

__global__ void __launch_bounds__(256)
pair_list_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                 const int32_t *__restrict__ vwgt, int32_t *__restrict__ match, int64_t maxvwgt)
{
    hp::pdl_wait();
    const int32_t cnt = *d_count;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; 2 * i + 1 < cnt;
         i += (int64_t)gridDim.x * blockDim.x) {
        int32_t a = list[2 * i], b = list[2 * i + 1];
        if ((int64_t)vwgt[a] + vwgt[b] <= maxvwgt) { match[a] = b; match[b] = a; }
    }
}

__global__ void __launch_bounds__(256)
finalize_match_kernel(int32_t n, int32_t *__restrict__ match, int32_t *__restrict__ leader_flag)
{
    hp::pdl_wait();
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    int32_t u = match[v];
    if (u == -1) { u = v; match[v] = v; }
    leader_flag[v] = (v <= u);
}

// Followers copy the leader's coarse id; leaders describe the coarse row: the
// fine rows it merges (start and length of the leader's and the mate's row)
// and its vertex weight.  Rows longer than thread_row entries are appended to
// their class list (warp radix up to warp_row, CTA radix up to cta_row, then
// the long class) and their length is counted for the temporary row buffer.

struct RowInfo {
    int32_t s0, l0, s1, l1;   // leader row start/length, mate row start/length (l1 = 0 if unmatched)
};

__global__ void __launch_bounds__(256)
coarse_setup_kernel(int32_t n, const int32_t *__restrict__ match, int32_t *__restrict__ cmap,
                    const int32_t *__restrict__ xadj, const int32_t *__restrict__ vwgt,
                    int4 *__restrict__ rinfo, int32_t *__restrict__ cvwgt, int32_t *__restrict__ ltlen,
                    int32_t *__restrict__ lists, int32_t *__restrict__ counts, int32_t cn,
                    int32_t *__restrict__ maxlen, unsigned long long *__restrict__ long_total,
                    int32_t *__restrict__ small_max, int32_t thread_row, int32_t warp_row, int32_t cta_row,
                    int32_t mid_row, int32_t mid2_row, int32_t *__restrict__ sub_counts)
{
    hp::pdl_wait();
    // no early exit: the list appends and maxima are aggregated per warp
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    bool lead = false;
    int32_t c = 0, len = 0;
    if (v < n) {
        const int32_t u = match[v];
        if (v > u) {
            cmap[v] = cmap[u];
        } else {
            lead = true;
            c = cmap[v];
            const int32_t s0 = xadj[v], l0 = xadj[v + 1] - s0;
            int32_t s1 = 0, l1 = 0;
            int32_t w = vwgt[v];
            if (u != v) {
                s1 = xadj[u];
                l1 = xadj[u + 1] - s1;
                w += vwgt[u];
            }
            rinfo[c] = make_int4(s0, l0, s1, l1);
            cvwgt[c] = w;
            len = l0 + l1;
            ltlen[c] = len > thread_row ? len : 0;
        }
    }
    const bool is_long = lead && len > thread_row;
    const int cls = !is_long ? -1 : (len <= warp_row ? 0 : (len <= cta_row ? 1 : 2));   // warp radix, CTA radix, long
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const int32_t pos = hp::warp_append(&counts[q], cls == q);
        if (cls == q) lists[(int64_t)q * cn + pos] = c;
    }
    // list 1 once more, split at mid_row and mid2_row (lists 3, 4 and 5): each
    // CTA radix instance walks only the rows it sorts
    const int sub = cls != 1 ? -1 : (len <= mid_row ? 0 : (len <= mid2_row ? 1 : 2));
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const int32_t pos = hp::warp_append(&sub_counts[q], sub == q);
        if (sub == q) lists[(int64_t)(3 + q) * cn + pos] = c;
    }
    // the longest short row above 8 entries picks the assembly kernel's network
    const int32_t sm = hp::warp_max(lead && !is_long && len > 8 ? len : 0);
    const int32_t lm = hp::warp_max(cls == 2 ? len : 0);
    const long long tot = hp::warp_sum64(is_long ? len : 0);
    if ((threadIdx.x & 31) == 0) {
        if (sm > 0) atomicMax(small_max, sm);
        if (lm > 0) atomicMax(maxlen, lm);
        if (tot > 0) atomicAdd(long_total, (unsigned long long)tot);
    }
}

// Weight range (checked when the input's total edge weight is 2^31 or more):
// every coarse edge weight and every gain-row connectivity of a vertex is at
// most the vertex's weighted degree, so the int32 weights and connectivities
// cannot wrap while every vertex of every level has a weighted degree below
// 2^31.  The contraction kernels check each coarse row's sum of kept weights
// (int64) as they gather it; this kernel checks the input level's rows (a
// thread per row, rows longer than 32 entries by the whole warp).  A row at or
// above 2^31 sets HP_STATUS_WEIGHT_RANGE, and the call fails.
__global__ void __launch_bounds__(256)
row_weight_range_kernel(int32_t n, const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjwgt,
                        unsigned *status)
{
    hp::pdl_wait();
    const int lane = threadIdx.x & 31;
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t b = v < n ? xadj[v] : 0, e = v < n ? xadj[v + 1] : 0;
    const bool coop = e - b > 32;
    bool over = false;
    if (!coop) {
        long long s = 0;
        for (int32_t j = b; j < e; j++) s += adjwgt[j];
        over = s >= (long long)INT32_MAX;
    }
    unsigned cm = __ballot_sync(HP_FULL_MASK, coop);
    while (cm) {
        const int src = __ffs(cm) - 1;
        cm &= cm - 1;
        const int32_t sb = __shfl_sync(HP_FULL_MASK, b, src), se = __shfl_sync(HP_FULL_MASK, e, src);
        long long s = 0;
        for (int32_t j = sb + lane; j < se; j += 32) s += adjwgt[j];
        s = hp::warp_sum64(s);
        over |= s >= (long long)INT32_MAX;
    }
    if (over) atomicOr(status, HP_STATUS_WEIGHT_RANGE);
}

// The fine rows merged into coarse row c: entry i is the i-th entry of the
// leader's row, then of the mate's row, mapped through cmap (the coarse self key
// is dropped).
// Entries per thread whose row loads, then coarse-id gathers, are in flight
// together in the long-row kernels.  The gathers are all issued before any of
// their results is stored, so they overlap even where the compiler cannot prove
// that the stores (or atomics) leave cmap alone.
constexpr int GATHER_DEPTH = 8;

struct ContractSrc {
    const int4 *rinfo;
    const int32_t *adjncy, *adjwgt, *cmap;
    __device__ __forceinline__ void row(int32_t c, RowInfo &r, int32_t &len) const
    {
        const int4 q = rinfo[c];
        r = RowInfo{q.x, q.y, q.z, q.w};
        len = r.l0 + r.l1;
    }
};

// ---- short rows: one thread per coarse row, aggregation in registers ------------
// The row's entries come from the tile's staging buffer (packed key << 32 |
// weight, the self key already PACK_NONE); a bitonic network of NET sorts them
// and the unique keys are counted.
template <int NET, int XN>
__device__ __forceinline__ int sort_staged_row(const unsigned long long *stage, int32_t len,
                                               unsigned long long (&x)[XN])
{
#pragma unroll
    for (int i = 0; i < NET; i++) x[i] = i < len ? stage[i] : hp::PACK_NONE;
    hp::sort_regs<NET, XN>(x);
    int u = 0;
#pragma unroll
    for (int i = 0; i < NET; i++) {
        const uint32_t k = (uint32_t)(x[i] >> 32);
        const bool head = k != (uint32_t)hp::KEY_NONE && (i == 0 || (uint32_t)(x[i - 1] >> 32) != k);
        u += head;
    }
    return u;
}

// The sorted row merged (weights of equal keys summed) into out[0..u), each
// entry tagged with the tile row t.
template <int NET, int XN>
__device__ __forceinline__ void emit_staged_row(const unsigned long long (&x)[XN], unsigned long long *out,
                                                uint8_t *orow, uint8_t t)
{
    int r = -1;
    uint32_t prev = 0xffffffffu;
    int32_t acc = 0;
#pragma unroll
    for (int i = 0; i < NET; i++) {
        const uint32_t k = (uint32_t)(x[i] >> 32);
        const int32_t w = (int32_t)(uint32_t)x[i];
        if (k == (uint32_t)hp::KEY_NONE) continue;
        if (k != prev) {
            if (r >= 0) out[r] = ((unsigned long long)prev << 32) | (uint32_t)acc;
            r++;
            orow[r] = t;
            acc = w;
            prev = k;
        } else {
            acc += w;
        }
    }
    if (r >= 0) out[r] = ((unsigned long long)prev << 32) | (uint32_t)acc;
}

// Coarse CSR assembly in one ordered pass: tiles of ASM_TILE coarse rows are
// taken in order (dynamic tile counter).  The tile's short rows are staged in
// shared memory: consecutive threads load consecutive entries of the rows (the
// row reads coalesce, the cmap gathers of one row hit neighbouring ids), each
// thread then sorts its row in registers (network of 8, 16 or 32 by the
// longest short row in the warp) or takes the unique count of a long row
// aggregated before; a block scan plus a decoupled look-back across tiles gives
// every row its final offset; the merged short rows go back through shared
// memory and are written with consecutive threads on consecutive entries.
// cxadj is written directly, with no second scan and no compaction copy; long
// rows are placed afterwards by copy_long_rows_kernel.
constexpr int ASM_TILE = 256;

// Dynamic shared memory: ASM_TILE * XN staged entries and their tile rows.
template <int XN>
constexpr size_t asm_smem_bytes()
{
    return (sizeof(unsigned long long) + sizeof(uint8_t)) * (size_t)ASM_TILE * XN;
}

// XN: the longest network the level needs (8, 16 or 32; the host reads the
// longest short row) -- every short row has at most XN entries.
template <int XN>
__global__ void __launch_bounds__(ASM_TILE)
contract_assemble_kernel(int32_t cn, ContractSrc src, const int32_t *__restrict__ ucnt,
                         int32_t *__restrict__ cxadj, int32_t *__restrict__ cadjncy,
                         int32_t *__restrict__ cadjwgt, unsigned long long *tile_status, hp::LbCtl *lb,
                         unsigned *status, int32_t thread_row, int wcheck)
{
    hp::pdl_wait();
    extern __shared__ unsigned long long asm_stage[];                      // ASM_TILE * XN
    uint8_t *s_row = reinterpret_cast<uint8_t *>(asm_stage + ASM_TILE * XN);   // tile row of each entry
    __shared__ int4 s_ri[ASM_TILE];
    __shared__ int32_t s_off[ASM_TILE];     // staged offset of the row's input, then of its output
    __shared__ int32_t s_goff[ASM_TILE];    // the row's final offset
    __shared__ int32_t s_scan[ASM_TILE / 32 + 2];
    __shared__ int32_t s_excl;
    int64_t tile;
    unsigned epoch;
    hp::lb_begin(lb, &tile, &epoch);
    const int t = threadIdx.x;
    const int32_t c0 = (int32_t)(tile * ASM_TILE);
    const int32_t c = c0 + t;
    RowInfo r{0, 0, 0, 0};
    int32_t len = 0;
    if (c < cn) src.row(c, r, len);
    const bool small = c < cn && len <= thread_row;
    int tin;
    const int ioff = hp::block_excl_scan<ASM_TILE>(small ? len : 0, &tin, s_scan);
    s_ri[t] = make_int4(r.s0, r.l0, r.s1, r.l1);
    s_off[t] = ioff;
    if (small)
        for (int i = 0; i < len; i++) s_row[ioff + i] = (uint8_t)t;
    __syncthreads();
    // stage: four entries per thread in flight (row reads, then the cmap gathers)
    for (int f0 = t; f0 < tin; f0 += 4 * ASM_TILE) {
        int32_t a[4], w[4], rt[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int f = f0 + q * ASM_TILE;
            rt[q] = -1;
            a[q] = 0;
            w[q] = 0;
            if (f < tin) {
                rt[q] = s_row[f];
                const int4 ri = s_ri[rt[q]];
                const int i = f - s_off[rt[q]];
                const int32_t j = i < ri.y ? ri.x + i : ri.z + (i - ri.y);
                a[q] = src.adjncy[j];
                w[q] = src.adjwgt[j];
            }
        }
        int32_t kq[4];
#pragma unroll
        for (int q = 0; q < 4; q++) kq[q] = rt[q] >= 0 ? src.cmap[a[q]] : 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (rt[q] < 0) continue;
            const int32_t k = kq[q];
            asm_stage[f0 + q * ASM_TILE] =
                k == c0 + rt[q] ? hp::PACK_NONE : (((unsigned long long)(uint32_t)k << 32) | (uint32_t)w[q]);
        }
    }
    __syncthreads();
    if (wcheck && small) {
        // the coarse row's weighted degree (weight range, row_weight_range_kernel)
        long long ws = 0;
        for (int i = 0; i < len; i++) {
            const unsigned long long e = asm_stage[ioff + i];
            if (e != hp::PACK_NONE) ws += (uint32_t)e;
        }
        if (ws >= (long long)INT32_MAX) atomicOr(status, HP_STATUS_WEIGHT_RANGE);
    }
    const unsigned wmax = __reduce_max_sync(HP_FULL_MASK, small ? (unsigned)len : 0u);
    unsigned long long x[XN];
    int u = 0;
    if (c < cn && !small) u = ucnt[c];
    if (XN == 8 || wmax <= 8) {
        if (small) u = sort_staged_row<8, XN>(asm_stage + ioff, len, x);
    } else if (XN == 16 || wmax <= 16) {
        if (small) u = sort_staged_row<(XN < 16 ? XN : 16), XN>(asm_stage + ioff, len, x);
    } else {
        if (small) u = sort_staged_row<XN, XN>(asm_stage + ioff, len, x);
    }
    int agg, tout;
    const int local = hp::block_excl_scan<ASM_TILE>(u, &agg, s_scan);   // (the staged input is read)
    const int ooff = hp::block_excl_scan<ASM_TILE>(small ? u : 0, &tout, s_scan);
    if (t < 32) {
        const int32_t excl = hp::lookback_epoch(tile_status, tile, agg, epoch, status);
        if (t == 0) s_excl = excl;
    }
    if (small) {
        if (XN == 8 || wmax <= 8) emit_staged_row<8, XN>(x, asm_stage + ooff, s_row + ooff, (uint8_t)t);
        else if (XN == 16 || wmax <= 16)
            emit_staged_row<(XN < 16 ? XN : 16), XN>(x, asm_stage + ooff, s_row + ooff, (uint8_t)t);
        else emit_staged_row<XN, XN>(x, asm_stage + ooff, s_row + ooff, (uint8_t)t);
    }
    s_off[t] = ooff;
    __syncthreads();
    const int32_t off = s_excl + local;
    s_goff[t] = off;
    if (c < cn) {
        cxadj[c] = off;
        if (c == cn - 1) cxadj[cn] = off + u;
    }
    __syncthreads();
    for (int f = t; f < tout; f += ASM_TILE) {
        const int rt = s_row[f];
        const int32_t pos = s_goff[rt] + (f - s_off[rt]);
        const unsigned long long e = asm_stage[f];
        cadjncy[pos] = (int32_t)(e >> 32);
        cadjwgt[pos] = (int32_t)(uint32_t)e;
    }
    hp::lb_end(lb);
}

// Long rows (aggregated into the temporary buffer at toff[c]) to their final
// place cxadj[c], coalesced: a warp per row for the warp class (list 0), a CTA
// per row for the longer classes (lists 1 and 2).
template <bool CTA>
__global__ void __launch_bounds__(256)
copy_long_rows_kernel(const int32_t *__restrict__ lists, const int32_t *__restrict__ counts, int32_t cn,
                      const int32_t *__restrict__ toff, const int32_t *__restrict__ ucnt,
                      const int32_t *__restrict__ cxadj, const int32_t *__restrict__ tk,
                      const int32_t *__restrict__ tw, int32_t *__restrict__ cadjncy, int32_t *__restrict__ cadjwgt)
{
    hp::pdl_wait();
    const int lane = CTA ? threadIdx.x : (threadIdx.x & 31);
    const int width = CTA ? blockDim.x : 32;
    const int64_t total = CTA ? (int64_t)counts[1] + counts[2] : (int64_t)counts[0];
    const int64_t first = CTA ? blockIdx.x : (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t step = CTA ? gridDim.x : ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int32_t n1 = counts[1];
    auto row_at = [&](int64_t i) -> int32_t {
        return lists[CTA ? (i < n1 ? (int64_t)cn + i : 2 * (int64_t)cn + (i - n1)) : i];
    };
    // the next row's id is loaded while the current row is copied, and each
    // thread keeps four entries' loads in flight
    int32_t c_next = first < total ? row_at(first) : 0;
    for (int64_t i = first; i < total; i += step) {
        const int32_t c = c_next;
        if (i + step < total) c_next = row_at(i + step);
        const int32_t src = toff[c], dst = cxadj[c], cnt = ucnt[c];
        for (int32_t j0 = lane; j0 < cnt; j0 += 4 * width) {
            int32_t a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int32_t j = j0 + q * width;
                if (j < cnt) {
                    a[q] = tk[src + j];
                    b[q] = tw[src + j];
                }
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int32_t j = j0 + q * width;
                if (j < cnt) {
                    cadjncy[dst + j] = a[q];
                    cadjwgt[dst + j] = b[q];
                }
            }
        }
    }
}

// ---- long rows: stable LSD radix sort of packed entries in shared memory -------
// A group of G threads (one warp, or the whole CTA) sorts the entries of one
// coarse row, packed as key << 32 | weight with the self key already dropped,
// by the low `kbits` bits of the key (8-bit digits), then merges equal keys.
// Per pass: per-warp digit histograms, one exclusive scan over them in
// digit-major order (digit d of warp w before digit d of warp w+1), and a stable
// scatter in which each warp walks its contiguous chunk 32 items at a time and
// ranks equal digits with __match_any_sync.
template <int G>
__device__ __forceinline__ void group_sync()
{
    if (G == 32) __syncwarp();
    else __syncthreads();
}

// Exclusive scan across the G threads of a group (one value per thread).
template <int G>
__device__ __forceinline__ int group_excl_scan(int v, int *total, int32_t *s_scan /* G/32 + 1 */)
{
    const int lane = threadIdx.x & 31;
    const int incl = hp::warp_incl_scan(v);
    if (G == 32) {
        *total = __shfl_sync(HP_FULL_MASK, incl, 31);
        return incl - v;
    }
    const int wid = (threadIdx.x % G) >> 5;
    if (lane == 31) s_scan[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int t = lane < G / 32 ? s_scan[lane] : 0;
        int ti = hp::warp_incl_scan(t);
        if (lane < G / 32) s_scan[lane] = ti - t;
        if (lane == G / 32 - 1) s_scan[G / 32] = ti;
    }
    __syncthreads();
    const int r = s_scan[wid] + incl - v;
    *total = s_scan[G / 32];
    __syncthreads();
    return r;
}

// Two exclusive scans across a group in one pass (a: int, b: wrapping uint32).
template <int G>
__device__ __forceinline__ void group_excl_scan2(int a, uint32_t b, int *ea, uint32_t *eb, int *ta,
                                                 int32_t *s_scan /* 2 * (G/32) + 2 */)
{
    const int lane = threadIdx.x & 31;
    int ia = a;
    uint32_t ib = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int xa = __shfl_up_sync(HP_FULL_MASK, ia, o);
        const uint32_t xb = __shfl_up_sync(HP_FULL_MASK, ib, o);
        if (lane >= o) { ia += xa; ib += xb; }
    }
    if (G == 32) {
        *ta = __shfl_sync(HP_FULL_MASK, ia, 31);
        *ea = ia - a;
        *eb = ib - b;
        return;
    }
    constexpr int W = G / 32;
    const int wid = (threadIdx.x % G) >> 5;
    if (lane == 31) { s_scan[wid] = ia; s_scan[W + wid] = (int32_t)ib; }
    __syncthreads();
    if (wid == 0) {
        int t = lane < W ? s_scan[lane] : 0;
        uint32_t u = lane < W ? (uint32_t)s_scan[W + lane] : 0u;
        int ti = t;
        uint32_t ui = u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int xa = __shfl_up_sync(HP_FULL_MASK, ti, o);
            const uint32_t xb = __shfl_up_sync(HP_FULL_MASK, ui, o);
            if (lane >= o) { ti += xa; ui += xb; }
        }
        if (lane < W) { s_scan[lane] = ti - t; s_scan[W + lane] = (int32_t)(ui - u); }
        if (lane == W - 1) s_scan[2 * W] = ti;
    }
    __syncthreads();
    *ea = s_scan[wid] + ia - a;
    *eb = (uint32_t)s_scan[W + wid] + ib - b;
    *ta = s_scan[2 * W];
    __syncthreads();
}

// Sorts A[0..N) (result in A; B is scratch of the same size); hist holds
// 256 * G/32 counters.  All G threads call it.
template <int G>
__device__ void group_radix_sort(unsigned long long *A, unsigned long long *B, int N, int kbits, int32_t *hist,
                                 int32_t *s_scan)
{
    constexpr int W = G / 32;
    const int t = threadIdx.x % G, lane = t & 31, w = t >> 5;
    const int chunk = (N + W - 1) / W;
    const int beg = min(N, w * chunk), end = min(N, beg + chunk);
    for (int shift = 0; shift < kbits; shift += 8) {
        for (int i = t; i < 256 * W; i += G) hist[i] = 0;
        group_sync<G>();
        for (int i = beg + lane; i < end; i += 32) atomicAdd(&hist[((unsigned)(A[i] >> (32 + shift)) & 255u) * W + w], 1);
        group_sync<G>();
        // digit-major exclusive offsets: thread t owns counters [8t, 8t+8)
        int s = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) s += hist[8 * t + q];
        int tot;
        int run = group_excl_scan<G>(s, &tot, s_scan);
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int h = hist[8 * t + q];
            hist[8 * t + q] = run;
            run += h;
        }
        group_sync<G>();
        for (int base = beg; base < end; base += 32) {
            const int i = base + lane;
            const bool valid = i < end;
            const unsigned long long x = valid ? A[i] : 0ull;
            const unsigned d = valid ? ((unsigned)(x >> (32 + shift)) & 255u) : 256u + lane;
            const unsigned peers = __match_any_sync(HP_FULL_MASK, d);
            const int rank = __popc(peers & hp::lanemask_lt());
            int *slot = &hist[(d & 255u) * W + w];
            if (valid) B[*slot + rank] = x;
            __syncwarp();
            if (valid && rank == 0) *slot += __popc(peers);
            __syncwarp();
        }
        group_sync<G>();
        unsigned long long *tmp = A; A = B; B = tmp;
    }
    // an odd number of passes leaves the result in the scratch buffer
    if (((kbits + 7) / 8) & 1) {
        for (int i = t; i < N; i += G) B[i] = A[i];
        group_sync<G>();
    }
}

// Merges equal keys of the sorted A[0..N): unique keys in order to out_k, the
// weight sums to out_w (a wrapping 32-bit prefix of the weights; every run sum
// is itself an int32 edge weight).  Returns the unique count (all threads).
// pre is scratch for N ints.
template <int G>
__device__ int group_merge_emit(const unsigned long long *A, int N, int32_t *out_k, int32_t *out_w, uint32_t *pre,
                                int32_t *s_scan)
{
    const int t = threadIdx.x % G;
    const int per = (N + G - 1) / G;
    const int lo = min(N, t * per), hi = min(N, lo + per);
    int heads = 0;
    uint32_t wsum = 0;
    for (int i = lo; i < hi; i++) {
        heads += (i == 0 || (uint32_t)(A[i] >> 32) != (uint32_t)(A[i - 1] >> 32));
        wsum += (uint32_t)A[i];
    }
    int o0, U;
    uint32_t p0;
    group_excl_scan2<G>(heads, wsum, &o0, &p0, &U, s_scan);
    int o = o0 - 1;   // ordinal of the current run
    uint32_t p = p0;  // weights before entry i
    for (int i = lo; i < hi; i++) {
        const uint32_t k = (uint32_t)(A[i] >> 32);
        if (i == 0 || k != (uint32_t)(A[i - 1] >> 32)) {
            o++;
            out_k[o] = (int32_t)k;
            pre[o] = p;
        }
        p += (uint32_t)A[i];
    }
    group_sync<G>();
    // second walk: the last entry of every run closes it
    o = o0 - 1;
    p = p0;
    for (int i = lo; i < hi; i++) {
        const uint32_t k = (uint32_t)(A[i] >> 32);
        if (i == 0 || k != (uint32_t)(A[i - 1] >> 32)) o++;
        p += (uint32_t)A[i];
        if (i == N - 1 || (uint32_t)(A[i + 1] >> 32) != k) out_w[o] = (int32_t)(p - pre[o]);
    }
    return U;
}

// Gathers row c into A in entry order; the coarse self key stays in as
// KEY_NONE (whose low kbits bits exceed every coarse id, so it sorts last) and
// the count of real entries is returned.
template <int G>
__device__ int group_gather_row(const ContractSrc &src, int32_t c, const RowInfo &r, int32_t len,
                                unsigned long long *A, int32_t *s_scan, long long *wpart)
{
    const int t = threadIdx.x % G;
    int self = 0;
    long long ws = 0;   // this thread's share of the row's kept weights
    // D entries per thread at a time: the row loads, then the coarse-id
    // gathers, are issued together (a warp's rows of at most 256 entries take
    // two batches of four)
    constexpr int D = G == 32 ? 4 : GATHER_DEPTH;
    for (int i0 = t; i0 < len; i0 += D * G) {
        int32_t j[D], a[D], w[D];
#pragma unroll
        for (int q = 0; q < D; q++) {
            const int i = i0 + q * G;
            j[q] = i < len ? (i < r.l0 ? r.s0 + i : r.s1 + (i - r.l0)) : -1;
            a[q] = j[q] >= 0 ? src.adjncy[j[q]] : 0;
            w[q] = j[q] >= 0 ? src.adjwgt[j[q]] : 0;
        }
        int32_t kq[D];
#pragma unroll
        for (int q = 0; q < D; q++) kq[q] = j[q] >= 0 ? src.cmap[a[q]] : 0;
#pragma unroll
        for (int q = 0; q < D; q++) {
            if (j[q] < 0) continue;
            int32_t k = kq[q];
            int32_t ww = w[q];
            if (k == c) { k = hp::KEY_NONE; ww = 0; }
            self += k == hp::KEY_NONE;
            ws += ww;
            A[i0 + q * G] = ((unsigned long long)(uint32_t)k << 32) | (uint32_t)ww;
        }
    }
    *wpart = ws;
    int tot;
    group_excl_scan<G>(self, &tot, s_scan);
    group_sync<G>();
    return len - tot;
}

// Weight range of a coarse row gathered by a group (row_weight_range_kernel's
// rule): the group's int64 total of the kept weights; s64 holds G/32 slots.
template <int G>
__device__ void group_weight_range(long long wpart, long long *s64, unsigned *status)
{
    const long long w = hp::warp_sum64(wpart);
    if (G == 32) {
        if ((threadIdx.x & 31) == 0 && w >= (long long)INT32_MAX) atomicOr(status, HP_STATUS_WEIGHT_RANGE);
        return;
    }
    const int t = threadIdx.x % G;
    if ((t & 31) == 0) s64[t >> 5] = w;
    group_sync<G>();
    if (t == 0) {
        long long tot = 0;
        for (int i = 0; i < G / 32; i++) tot += s64[i];
        if (tot >= (long long)INT32_MAX) atomicOr(status, HP_STATUS_WEIGHT_RANGE);
    }
    group_sync<G>();
}

constexpr int WROW_MAX = HP_TUNE_WARP_ROW_MAX;   // warp class: up to 256 entries
constexpr int CROW_MAX = HP_TUNE_CTA_ROW_MAX;    // CTA class: up to 4096 entries
constexpr int WROW_WARPS = 8;

// Warp class: 8 warps per CTA, one row per warp at a time.
__global__ void __launch_bounds__(32 * WROW_WARPS)
contract_warp_radix_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count, ContractSrc src,
                           const int32_t *__restrict__ toff, int32_t *__restrict__ tk, int32_t *__restrict__ tw,
                           int32_t *__restrict__ ucnt, int kbits, int wcheck, unsigned *status)
{
    hp::pdl_wait();
    __shared__ unsigned long long sA[WROW_WARPS][WROW_MAX], sB[WROW_WARPS][WROW_MAX];
    __shared__ int32_t sH[WROW_WARPS][256];
    const int wid = threadIdx.x >> 5;
    const int32_t cnt = *d_count;
    for (int64_t li = (int64_t)blockIdx.x * WROW_WARPS + wid; li < cnt; li += (int64_t)gridDim.x * WROW_WARPS) {
        const int32_t c = list[li];
        RowInfo r;
        int32_t len;
        src.row(c, r, len);
        long long wpart;
        const int N = group_gather_row<32>(src, c, r, len, sA[wid], nullptr, &wpart);
        if (wcheck) group_weight_range<32>(wpart, nullptr, status);
        group_radix_sort<32>(sA[wid], sB[wid], len, kbits, sH[wid], nullptr);
        const int32_t off = toff[c];
        const int U = group_merge_emit<32>(sA[wid], N, tk + off, tw + off, (uint32_t *)sB[wid], nullptr);
        if ((threadIdx.x & 31) == 0) ucnt[c] = U;
        __syncwarp();
    }
}

// CTA class: one CTA of NT threads per row of min_len+1 .. CAP entries.  Four
// instances: <64, 1024>, <128, 2048> and <256, 4096> split list 1, and
// <1024, 12288> takes the rows of list 2 up to 12288 entries, whose longer rows
// stay with the dense kernel; 2 CAP packed entries plus NT/32 digit histograms
// fit the 227 KB of shared memory of one CTA.  Rows of up to 1024 entries take
// two warps and 18 KB, so eleven rows are in flight per SM: on rows of 257-1024
// entries that sorts 1.5x faster than a CTA of 256 threads (fewer threads per
// barrier, more rows in flight); rows of 1025-2048 entries sort 1.24x faster
// with four warps and 36 KB (six rows per SM), rows of 2049-4096 fastest with
// 256 threads.
constexpr int CROW_THREADS = 256;
constexpr int MROW_THREADS = 64;
constexpr int NROW_THREADS = 128, NROW_MAX = 2048;   // the middle CTA instance of list 1
constexpr int XROW_THREADS = 1024, XROW_MAX = 12288;
constexpr int MROW_MAX = 1024;   // the smaller CTA instance of list 1

template <int NT, int CAP>
__global__ void __launch_bounds__(NT)
contract_cta_radix_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count, ContractSrc src,
                          const int32_t *__restrict__ toff, int32_t *__restrict__ tk, int32_t *__restrict__ tw,
                          int32_t *__restrict__ ucnt, int kbits, int32_t min_len, int wcheck, unsigned *status)
{
    hp::pdl_wait();
    extern __shared__ unsigned long long dsm[];
    unsigned long long *A = dsm, *B = dsm + CAP;
    int32_t *hist = (int32_t *)(dsm + 2 * CAP);
    __shared__ int32_t s_scan[2 * (NT / 32) + 2];
    __shared__ long long s64[NT / 32];
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t c = list[li];
        RowInfo r;
        int32_t len;
        src.row(c, r, len);
        if (len > CAP || len <= min_len) continue;   // another instance's row
        long long wpart;
        const int N = group_gather_row<NT>(src, c, r, len, A, s_scan, &wpart);
        if (wcheck) group_weight_range<NT>(wpart, s64, status);
        group_radix_sort<NT>(A, B, len, kbits, hist, s_scan);
        const int32_t off = toff[c];
        const int U = group_merge_emit<NT>(A, N, tk + off, tw + off, (uint32_t *)B, s_scan);
        if (threadIdx.x == 0) ucnt[c] = U;
        __syncthreads();
    }
}

template <int NT, int CAP>
constexpr size_t cta_radix_smem() { return sizeof(unsigned long long) * 2 * CAP + sizeof(int32_t) * 256 * (NT / 32); }


// ---- long rows, hybrid: dense accumulation of the low ids, radix sort of the rest --
// On power-law graphs a long coarse row points mostly at hubs, and hubs have
// low coarse ids (coarse ids follow the leaders' fine ids, and the R-MAT hubs
// have low ids): on R-MAT levels of 90K-160K coarse vertices 78-98 % of the
// long rows' entries have an id below 48K, 57 % at 300K.  The shared-memory
// dense accumulator is several times faster per entry than a radix sort, but
// one accumulator over all coarse ids fits only up to 48K ids.  So each CTA
// keeps a dense accumulator for the ids below HY_HOT and a buffer for the rest:
//   - gather: an entry with a low id is added to acc[id] and marked in the
//     bitmap; any other entry is appended to the cold buffer (its order does
//     not matter: equal ids are merged by summing, and the sort orders the rest);
//   - the low ids come out in ascending order from the bitmap (two words per
//     thread, a block scan for the offsets), clearing acc and the bitmap;
//   - the cold entries are radix-sorted and merged after them, so the row is
//     sorted as a whole and equals what the pure radix path writes.
// A row whose cold part exceeds HY_COLD entries is cleared and appended to the
// spill list, which the radix / dense kernels then take.  The kernel runs one
// CTA per SM (its shared memory), so it pays on levels where most entries are
// low ids: levels of at most HY_MAX_CN coarse vertices (measured on R-MAT
// scale 22: 2x faster than the radix classes at 74K coarse ids, slower from
// about 200K, where half of the entries are cold).
constexpr int HY_THREADS = 1024;
constexpr int HY_HOT = 32768;                 // ids below this accumulate densely
constexpr int HY_WORDS = HY_HOT / 32;         // bitmap words
constexpr int HY_WPT = HY_WORDS / HY_THREADS; // bitmap words per thread in the extraction
constexpr int HY_COLD = 2048;                 // cold entries a row may have
constexpr int32_t HY_MAX_CN = 4 * HY_HOT;     // levels the hybrid kernel takes
static_assert(HY_WORDS % HY_THREADS == 0 && HY_WPT >= 1, "extraction: whole words per thread");

constexpr size_t hybrid_smem()
{
    return sizeof(unsigned long long) * 2 * HY_COLD + sizeof(int32_t) * HY_HOT + sizeof(unsigned) * HY_WORDS +
           sizeof(int32_t) * 256 * (HY_THREADS / 32);
}

__global__ void __launch_bounds__(HY_THREADS, 1)
contract_hybrid_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count, ContractSrc src,
                       const int32_t *__restrict__ toff, int32_t *__restrict__ tk, int32_t *__restrict__ tw,
                       int32_t *__restrict__ ucnt, int kbits, int32_t min_len, int32_t *__restrict__ spill,
                       int32_t *d_nspill, int wcheck, unsigned *status)
{
    hp::pdl_wait();
    extern __shared__ unsigned long long hy_smem[];
    unsigned long long *A = hy_smem, *B = hy_smem + HY_COLD;
    int32_t *acc = reinterpret_cast<int32_t *>(hy_smem + 2 * HY_COLD);
    unsigned *bm = reinterpret_cast<unsigned *>(acc + HY_HOT);
    int32_t *hist = reinterpret_cast<int32_t *>(bm + HY_WORDS);
    __shared__ int32_t s_scan[2 * (HY_THREADS / 32) + 2];
    __shared__ long long s64[HY_THREADS / 32];
    __shared__ int32_t s_ncold;
    const int tid = threadIdx.x;
    for (int i = tid; i < HY_HOT; i += HY_THREADS) acc[i] = 0;   // every row leaves them zero
    for (int i = tid; i < HY_WORDS; i += HY_THREADS) bm[i] = 0u;
    if (tid == 0) s_ncold = 0;
    __syncthreads();
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t c = list[li];
        RowInfo r;
        int32_t len;
        src.row(c, r, len);
        if (len <= min_len) continue;   // (uniform over the CTA)
        long long ws = 0;
        // GATHER_DEPTH entries per thread in flight: the row loads, then the cmap gathers
        for (int32_t i0 = tid; i0 < len; i0 += GATHER_DEPTH * HY_THREADS) {
            int32_t a[GATHER_DEPTH], w[GATHER_DEPTH];
            bool in[GATHER_DEPTH];
#pragma unroll
            for (int q = 0; q < GATHER_DEPTH; q++) {
                const int32_t i = i0 + q * HY_THREADS;
                in[q] = i < len;
                const int32_t j = in[q] ? (i < r.l0 ? r.s0 + i : r.s1 + (i - r.l0)) : 0;
                a[q] = in[q] ? src.adjncy[j] : 0;
                w[q] = in[q] ? src.adjwgt[j] : 0;
            }
            int32_t kq[GATHER_DEPTH];
#pragma unroll
            for (int q = 0; q < GATHER_DEPTH; q++) kq[q] = in[q] ? src.cmap[a[q]] : 0;
#pragma unroll
            for (int q = 0; q < GATHER_DEPTH; q++) {
                if (!in[q]) continue;
                const int32_t k = kq[q];
                if (k == c) continue;   // the coarse self key
                ws += w[q];
                if (k < HY_HOT) {
                    atomicAdd(&acc[k], w[q]);
                    atomicOr(&bm[k >> 5], 1u << (k & 31));
                } else {
                    const int32_t pos = atomicAdd(&s_ncold, 1);
                    if (pos < HY_COLD) A[pos] = ((unsigned long long)(uint32_t)k << 32) | (uint32_t)w[q];
                }
            }
        }
        __syncthreads();
        if (wcheck) group_weight_range<HY_THREADS>(ws, s64, status);
        const int32_t ncold = s_ncold;
        if (ncold > HY_COLD) {
            // the cold part does not fit: clear the dense part and leave the row to the spill kernels
            for (int wi = tid; wi < HY_WORDS; wi += HY_THREADS) {
                unsigned word = bm[wi];
                if (!word) continue;
                bm[wi] = 0u;
                for (; word; word &= word - 1) acc[(wi << 5) + __ffs(word) - 1] = 0;
            }
            if (tid == 0) {
                spill[atomicAdd(d_nspill, 1)] = c;
                s_ncold = 0;
            }
            __syncthreads();
            continue;
        }
        const int32_t off = toff[c];
        // the low ids in ascending order: HY_WPT consecutive bitmap words per thread
        unsigned wd[HY_WPT];
        int hc = 0;
#pragma unroll
        for (int q = 0; q < HY_WPT; q++) {
            wd[q] = bm[tid * HY_WPT + q];
            hc += __popc(wd[q]);
        }
        int uh;
        int p = hp::block_excl_scan<HY_THREADS>(hc, &uh, s_scan);
#pragma unroll
        for (int q = 0; q < HY_WPT; q++) {
            const int wi = tid * HY_WPT + q;
            unsigned word = wd[q];
            if (word) bm[wi] = 0u;
            for (; word; word &= word - 1) {
                const int32_t k = (wi << 5) + __ffs(word) - 1;
                tk[off + p] = k;
                tw[off + p] = acc[k];
                acc[k] = 0;
                p++;
            }
        }
        // the rest, sorted and merged after them
        int uc = 0;
        if (ncold > 0) {
            group_radix_sort<HY_THREADS>(A, B, ncold, kbits, hist, s_scan);
            uc = group_merge_emit<HY_THREADS>(A, ncold, tk + off + uh, tw + off + uh, (uint32_t *)B, s_scan);
        }
        if (tid == 0) {
            ucnt[c] = uh + uc;
            s_ncold = 0;
        }
        __syncthreads();
    }
}

// Rows longer than XROW_MAX entries: dense accumulator over the coarse id space
// in a per-CTA global slab (dw: cn ints, bm: cn/32 words, bm2: cn/1024 words;
// zero on entry/exit).  A row with len * ratio < cn/32 words walks the occupied
// words through the second-level bitmap; a denser row scans the bitmap.
// SMEM: the accumulators live in the CTA's shared memory (cn + cn/32 + cn/1024
// words, zeroed here), for levels whose coarse vertex count fits; every row of
// the list longer than min_len is taken.  Otherwise they are the CTA's global
// slab and only the rows above XROW_MAX are taken (min_len).
template <int NT, bool SMEM>
__global__ void __launch_bounds__(NT)
contract_dense_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                      ContractSrc src, const int32_t *__restrict__ toff, int32_t *__restrict__ tk,
                      int32_t *__restrict__ tw, int32_t *__restrict__ ucnt, int32_t cn,
                      int32_t *slab_w, unsigned *slab_bm, unsigned *slab_bm2, int32_t ratio, int32_t min_len,
                      int wcheck, unsigned *status)
{
    hp::pdl_wait();
    extern __shared__ int32_t dsm_acc[];
    __shared__ int32_t s_scan[NT / 32 + 2];
    __shared__ long long s64[NT / 32];
    const int32_t nw = (cn + 31) / 32, nw2 = (cn + 1023) / 1024;
    int32_t *dw;
    unsigned *bm, *bm2;
    if (SMEM) {
        dw = dsm_acc;
        bm = (unsigned *)(dsm_acc + cn);
        bm2 = bm + nw;
        for (int32_t i = threadIdx.x; i < cn + nw + nw2; i += NT) dsm_acc[i] = 0;
        __syncthreads();
    } else {
        dw = slab_w + (int64_t)blockIdx.x * cn;
        bm = slab_bm + (int64_t)blockIdx.x * nw;
        bm2 = slab_bm2 + (int64_t)blockIdx.x * nw2;
    }
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t c = list[li];
        RowInfo r;
        int32_t len;
        src.row(c, r, len);
        if (len <= min_len) continue;   // another kernel's row
        const bool two_level = (int64_t)len * ratio < ((int64_t)cn + 31) / 32;
        long long ws = 0;   // this thread's share of the row's kept weights (weight range)
        for (int32_t i0 = threadIdx.x; i0 < len; i0 += GATHER_DEPTH * NT) {
            int32_t a[GATHER_DEPTH], wq[GATHER_DEPTH], kq[GATHER_DEPTH];
            bool in[GATHER_DEPTH];
#pragma unroll
            for (int q = 0; q < GATHER_DEPTH; q++) {
                const int32_t i = i0 + q * NT;
                in[q] = i < len;
                const int32_t j = in[q] ? (i < r.l0 ? r.s0 + i : r.s1 + (i - r.l0)) : 0;
                a[q] = in[q] ? src.adjncy[j] : 0;
                wq[q] = in[q] ? src.adjwgt[j] : 0;
            }
#pragma unroll
            for (int q = 0; q < GATHER_DEPTH; q++) kq[q] = in[q] ? src.cmap[a[q]] : 0;
#pragma unroll
            for (int q = 0; q < GATHER_DEPTH; q++) {
                if (!in[q]) continue;
                const int32_t k = kq[q];
                if (k == c) continue;   // the coarse self key
                ws += wq[q];
                if (two_level) {
                    hp::dense_mark2(dw, bm, bm2, k, wq[q]);
                } else {
                    atomicAdd(&dw[k], wq[q]);
                    atomicOr(&bm[k >> 5], 1u << (k & 31));
                }
            }
        }
        __syncthreads();
        if (wcheck) group_weight_range<NT>(ws, s64, status);
        int32_t off = toff[c];
        int tot = two_level ? hp::dense_extract2<NT>(dw, bm, bm2, cn, tk + off, tw + off, s_scan)
                            : hp::dense_extract<NT>(dw, bm, cn, tk + off, tw + off, s_scan);
        if (threadIdx.x == 0) ucnt[c] = tot;
    }
}

// ---- small levels: the whole matching in one CTA -------------------------------------
// A level with few vertices is matched by one CTA of MS_THREADS threads: the
// handshake rounds (a proposal that is still valid is kept, as in the cached
// kernels), the two-hop pairing (clients sorted stably by hub with a block
// radix sort), the isolated and forced pairings, each gated at 75 % matched,
// the self matches of the rest and the exclusive scan of the leader flags into
// cmap -- the rules of match_level, separated by __syncthreads instead of
// kernel boundaries and host reads.  The match, eligibility and proposal
// arrays live in shared memory (at most HP_TUNE_SMALL_MATCH_MAX vertices), so a
// row scan's only global loads are the row's own entries; cmap[n], the coarse
// vertex count, is all the host reads back.
constexpr int MS_THREADS = 1024;

inline size_t ms_smem_bytes(int32_t n)
{
    return sizeof(int32_t) * ((size_t)hp::block_sort_ints(MS_THREADS) + 3 * (size_t)n);
}

// v's best candidate over its row: a thread walks rows of up to 32 entries
// (eight loads in flight), the whole warp longer ones, one at a time, reduced
// in hp::better's order -- a total order, so the split does not change the
// winner.  ELIG: unmatched neighbours within the weight cap only (s_elig:
// vertex weight, INT_MAX once matched); else any neighbour.  All lanes of the
// warp call; act marks the lanes with a row to scan.
template <bool ELIG>
__device__ int32_t ms_best(bool act, int32_t v, const int32_t *__restrict__ xadj,
                           const int32_t *__restrict__ adjncy, const int32_t *__restrict__ adjwgt,
                           const int32_t *s_elig, int32_t wv, uint64_t lkey, int64_t maxvwgt)
{
    const int lane = threadIdx.x & 31;
    const int32_t b = act ? xadj[v] : 0, e = act ? xadj[v + 1] : 0;
    const bool coop = act && e - b > 32;
    int32_t res = -1;
    if (act && !coop) {
        BestCand best;
        for (int32_t j0 = b; j0 < e; j0 += 8) {
            int32_t u[8], w[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const bool in = j0 + q < e;
                u[q] = in ? adjncy[j0 + q] : v;
                w[q] = in ? adjwgt[j0 + q] : 0;
            }
#pragma unroll
            for (int q = 0; q < 8; q++) {
                if (u[q] == v) continue;
                if (ELIG) {
                    const int32_t eu = s_elig[u[q]];
                    if (eu == INT_MAX) continue;                     // matched
                    if ((int64_t)wv + eu > maxvwgt) continue;        // weight cap
                }
                best.offer(lkey, v, u[q], w[q]);
            }
        }
        res = best.u;
    }
    unsigned cm = __ballot_sync(HP_FULL_MASK, coop);
    while (cm) {
        const int src = __ffs(cm) - 1;
        cm &= cm - 1;
        const int32_t sv = __shfl_sync(HP_FULL_MASK, v, src), sb = __shfl_sync(HP_FULL_MASK, b, src);
        const int32_t se = __shfl_sync(HP_FULL_MASK, e, src), swv = __shfl_sync(HP_FULL_MASK, wv, src);
        BestCand best;
        for (int32_t j = sb + lane; j < se; j += 32) {
            const int32_t u = adjncy[j];
            if (u == sv) continue;
            if (ELIG) {
                const int32_t eu = s_elig[u];
                if (eu == INT_MAX) continue;
                if ((int64_t)swv + eu > maxvwgt) continue;
            }
            best.offer(lkey, sv, u, adjwgt[j]);
        }
        best.finish(lkey, sv);
        int32_t bu = best.u, bw = best.w;
        uint32_t bh = best.h;
        warp_best(bu, bw, bh);
        if (lane == src) res = bu;
    }
    return res;
}

// Number of v < n with s_match[v] != -1 (every thread gets it).
__device__ __forceinline__ int32_t ms_matched(int32_t n, const int32_t *s_match, int32_t *s_scan)
{
    int c = 0;
    for (int32_t v = threadIdx.x; v < n; v += MS_THREADS) c += s_match[v] != -1;
    int tot;
    hp::block_excl_scan<MS_THREADS>(c, &tot, s_scan);
    return tot;
}

// Pairs (list[2i], list[2i+1]) of the unmatched vertices (ISOLATED_ONLY: the
// unmatched vertices without neighbours) in id order, when the weight sum fits
// (pair_list_kernel's rule).  list: n ints.
template <bool ISOLATED_ONLY>
__device__ void ms_pair_unmatched(int32_t n, const int32_t *__restrict__ xadj, const int32_t *__restrict__ vwgt,
                                  int32_t *s_match, int32_t *__restrict__ list, int64_t maxvwgt, int32_t *s_scan)
{
    int32_t cnt = 0;
    for (int32_t b0 = 0; b0 < n; b0 += MS_THREADS) {
        const int32_t v = b0 + threadIdx.x;
        int f = v < n && s_match[v] == -1;
        if (ISOLATED_ONLY && f) f = xadj[v] == xadj[v + 1];
        int tot;
        const int ex = hp::block_excl_scan<MS_THREADS>(f, &tot, s_scan);
        if (f) list[cnt + ex] = v;
        cnt += tot;
    }
    __syncthreads();
    for (int32_t i = threadIdx.x; 2 * i + 1 < cnt; i += MS_THREADS) {
        const int32_t a = list[2 * i], b = list[2 * i + 1];
        if ((int64_t)vwgt[a] + vwgt[b] <= maxvwgt) { s_match[a] = b; s_match[b] = a; }
    }
    __syncthreads();
}

// Dynamic shared memory: ms_smem_bytes(n).  K, V, K2, V2: n ints each (the
// two-hop sort and the pairing lists).
__global__ void __launch_bounds__(MS_THREADS, 1)
match_small_kernel(int32_t n, const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                   const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ vwgt, int32_t *__restrict__ match,
                   int32_t *__restrict__ cmap, int32_t *K, int32_t *V, int32_t *K2, int32_t *V2, uint64_t lkey,
                   int64_t maxvwgt, int rounds, int key_bits)
{
    hp::pdl_wait();
    extern __shared__ int32_t ms_sh[];
    int32_t *tab = ms_sh;                                        // block radix sort
    int32_t *s_match = tab + hp::block_sort_ints(MS_THREADS);
    int32_t *s_elig = s_match + n;
    int32_t *s_pref = s_elig + n;
    __shared__ int32_t s_scan[MS_THREADS / 32 + 2];
    const int tid = threadIdx.x;
    for (int32_t v = tid; v < n; v += MS_THREADS) {
        s_match[v] = -1;
        s_elig[v] = vwgt[v];
        s_pref[v] = -1;
    }
    __syncthreads();
    // handshake rounds; a round that matched nothing ends them (the next would
    // repeat it)
    for (int r = 0; r < rounds; r++) {
        for (int32_t b0 = 0; b0 < n; b0 += MS_THREADS) {
            const int32_t v = b0 + tid;
            const bool in = v < n;
            const bool unmatched = in && s_match[v] == -1;
            bool act = unmatched;
            if (act && r > 0) {   // keep a proposal that is still valid (keep_proposal)
                const int32_t pu = s_pref[v];
                act = pu >= 0 && s_elig[pu] == INT_MAX;
            }
            const int32_t u = ms_best<true>(act, v, xadj, adjncy, adjwgt, s_elig, act ? vwgt[v] : 0, lkey, maxvwgt);
            if (act) s_pref[v] = u;
            else if (in && !unmatched) s_pref[v] = -1;
        }
        __syncthreads();
        int made = 0;
        for (int32_t v = tid; v < n; v += MS_THREADS) {
            if (s_match[v] != -1) continue;
            const int32_t u = s_pref[v];
            if (u >= 0 && s_pref[u] == v) {
                s_match[v] = u;
                s_elig[v] = INT_MAX;
                made++;
            }
        }
        int tot;
        hp::block_excl_scan<MS_THREADS>(made, &tot, s_scan);   // (ends with a barrier)
        if (tot == 0) break;
    }
    int32_t nm = ms_matched(n, s_match, s_scan);
    if (4 * (int64_t)nm < 3 * (int64_t)n) {
        // two-hop: the hub of every unmatched vertex (any neighbour), the clients
        // sorted stably by hub, odd offsets in a hub's run paired with the one before
        for (int32_t b0 = 0; b0 < n; b0 += MS_THREADS) {
            const int32_t v = b0 + tid;
            const bool in = v < n;
            const bool act = in && s_match[v] == -1;
            const int32_t u = ms_best<false>(act, v, xadj, adjncy, adjwgt, nullptr, 0, lkey, maxvwgt);
            if (in) s_pref[v] = act ? u : -1;
        }
        __syncthreads();
        int32_t cnt = 0;
        for (int32_t b0 = 0; b0 < n; b0 += MS_THREADS) {
            const int32_t c = b0 + tid;
            const int f = c < n && s_match[c] == -1 && s_pref[c] >= 0;
            int tot;
            const int ex = hp::block_excl_scan<MS_THREADS>(f, &tot, s_scan);
            if (f) {
                K[cnt + ex] = s_pref[c];
                V[cnt + ex] = c;
            }
            cnt += tot;
        }
        const bool flip = hp::block_sort_pairs<MS_THREADS>(K, V, K2, V2, cnt, key_bits, tab, s_scan);
        const int32_t *Ks = flip ? K2 : K, *Vs = flip ? V2 : V;
        for (int32_t i = tid; i < cnt; i += MS_THREADS) {
            const int32_t h = Ks[i];
            int32_t lo = 0, hi = i;   // first index of the run of h
            while (lo < hi) {
                const int32_t mid = (lo + hi) >> 1;
                if (Ks[mid] < h) lo = mid + 1; else hi = mid;
            }
            if ((i - lo) & 1) {
                const int32_t a = Vs[i - 1], b = Vs[i];
                if ((int64_t)vwgt[a] + vwgt[b] <= maxvwgt) { s_match[a] = b; s_match[b] = a; }
            }
        }
        __syncthreads();
        nm = ms_matched(n, s_match, s_scan);
    }
    if (4 * (int64_t)nm < 3 * (int64_t)n) {   // isolated vertices, in id order
        ms_pair_unmatched<true>(n, xadj, vwgt, s_match, K, maxvwgt, s_scan);
        nm = ms_matched(n, s_match, s_scan);
    }
    if (4 * (int64_t)nm < 3 * (int64_t)n)     // forced: every remaining vertex, in id order
        ms_pair_unmatched<false>(n, xadj, vwgt, s_match, K, maxvwgt, s_scan);
    // self matches of the rest; cmap = exclusive scan of the leader flags
    int32_t run = 0;
    for (int32_t b0 = 0; b0 < n; b0 += MS_THREADS) {
        const int32_t v = b0 + tid;
        int lead = 0;
        if (v < n) {
            int32_t u = s_match[v];
            if (u == -1) u = v;
            match[v] = u;
            lead = v <= u;
        }
        int tot;
        const int ex = hp::block_excl_scan<MS_THREADS>(lead, &tot, s_scan);
        if (v < n) cmap[v] = run + ex;
        run += tot;
    }
    if (tid == 0) cmap[n] = run;
}

inline unsigned blocks_for(int64_t threads, int block = 256)
{
    int64_t g = (threads + block - 1) / block;
    return (unsigned)(g > 0 ? g : 1);
}

inline unsigned persistent_grid(hp_context *c)
{
    return (unsigned)(c->sm_count * c->tune.grid_ctas_per_sm);
}

// One matching level.  On return match[] is final (self when unmatched),
// cmap[0..n] holds the exclusive scan of leader flags (cmap[n] = cn) with the
// follower entries filled in by the caller's setup kernel.
int match_level(hp_context *c, HpLevel &g, int32_t level, int64_t maxvwgt, int32_t *cn_out)
{
    const int32_t n = g.n;
    const hp_options &o = c->opt;
    const uint64_t lkey = hp::level_key(o.seed, level);
    const size_t mark = c->hi;

    const hp_tuning &tn = c->tune;
    const int rounds = o.match_rounds < 1 ? 1 : (o.match_rounds > 30 ? 30 : o.match_rounds);
    // algorithmic bytes of one full handshake round: xadj, adjncy, adjwgt,
    // vwgt, match read and write (neighbour gathers not counted)
    const int64_t round_bytes = 4 * ((int64_t)n + 1) + 8 * g.m + 12 * (int64_t)n;
    // a later round (a vertex whose previous proposal is still unmatched keeps
    // it without a rescan): xadj, match, eligibility, previous proposal in,
    // proposal out; the rows rescanned are not counted (a lower bound)
    const int64_t later_round_bytes = 4 * ((int64_t)n + 1) + 16 * (int64_t)n;
    if (n <= tn.small_match_n && g.m <= 64 * (int64_t)n) {
        // a small level: the whole matching in one CTA, one read back (cn)
        int32_t *sb = ralloc_t<int32_t>(c, 4 * ((int64_t)n + 1));
        HP_CHECK_OOM(c);
        int32_t *sk = sb, *sv = sb + (n + 1), *sk2 = sb + 2 * (n + 1), *sv2 = sb + 3 * (n + 1);
        int kbits = 0;
        while ((1ll << kbits) < (int64_t)n) kbits++;
        const int tok = hp_prof_begin(c);
        HP_LAUNCH(c, match_small_kernel, 1, MS_THREADS, ms_smem_bytes(n), n, g.xadj, g.adjncy, g.adjwgt, g.vwgt,
                  g.match, g.cmap, sk, sv, sk2, sv2, lkey, maxvwgt, rounds, kbits);
        hp_prof_end(c, tok, HP_PROF_MATCH, round_bytes);
        int32_t cn = 0;
        HP_TRY(hp_read_scalars(c, g.cmap + n, sizeof(int32_t), &cn));
        *cn_out = cn;
        c->hi = mark;
        return HP_OK;
    }

    int32_t *pref = ralloc_t<int32_t>(c, n);
    int32_t *big = ralloc_t<int32_t>(c, n);
    int32_t *huge = ralloc_t<int32_t>(c, n);
    int32_t *flags = ralloc_t<int32_t>(c, n + 1);
    int32_t *list = ralloc_t<int32_t>(c, n + 1);
    // candidate state: vwgt while unmatched, INT_MAX once matched (one gather
    // per neighbour in the proposal kernels)
    int32_t *elig = ralloc_t<int32_t>(c, n);
    int32_t *cand = ralloc_t<int32_t>(c, (int64_t)n * TOPK);   // candidate caches of the long rows
    HP_CHECK_OOM(c);
    // scalar slots: [0] big count, [1] list count, [2..2+R) made per round, [40..43] matched counts
    unsigned long long *sc = c->d_scal;
    HP_CUDA(cudaMemsetAsync(sc, 0, sizeof(unsigned long long) * HP_NSCAL, c->stream));
    int32_t *d_bigcnt = (int32_t *)&sc[0];
    int32_t *d_listcnt = (int32_t *)&sc[1];
    int32_t *d_hugecnt = (int32_t *)&sc[38];

    HP_TRY(hp_fill_i32(c, g.match, n, -1));
    HP_LAUNCH(c, big_list_kernel, blocks_for(n), 256, 0, n, g.xadj, big, d_bigcnt, huge, d_hugecnt, g.vwgt, elig,
              tn.match_warp_deg, tn.match_cta_deg);

    for (int r = 0; r < rounds; r++) {
        const int tok = hp_prof_begin(c);
        const unsigned long long *prev = r == 0 ? nullptr : &sc[2 + r - 1];
        HP_LAUNCH(c, pref_small_kernel<true>, blocks_for(n), 256, 0, n, g.xadj, g.adjncy, g.adjwgt,
                  g.vwgt, g.match, elig, pref, lkey, maxvwgt, prev, tn.match_warp_deg);
        HP_LAUNCH(c, pref_big_topk_kernel, persistent_grid(c), 256, 0, big, d_bigcnt, g.xadj, g.adjncy, g.adjwgt,
                  g.vwgt, g.match, elig, pref, cand, lkey, maxvwgt, prev);
        HP_LAUNCH(c, pref_huge_topk_kernel, (unsigned)(2 * c->sm_count), HUGE_TOPK_THREADS, 0, huge, d_hugecnt, g.xadj,
                  g.adjncy, g.adjwgt, g.vwgt, g.match, elig, pref, cand, lkey, maxvwgt, prev);
        HP_LAUNCH(c, commit_kernel, blocks_for(n), 256, 0, n, g.match, pref, elig, &sc[2 + r], prev);
        hp_prof_end(c, tok, r == 0 ? HP_PROF_MATCH : HP_PROF_MATCH_MORE, r == 0 ? round_bytes : later_round_bytes);
    }

    auto matched = [&](int slot, int64_t *out) -> int {
        HP_LAUNCH(c, count_matched_kernel, blocks_for(n), 256, 0, n, g.match, &sc[slot]);
        long long v = 0;
        HP_TRY(hp_read_scalars(c, &sc[slot], sizeof(long long), &v));
        *out = v;
        return HP_OK;
    };
    int64_t nm = 0;
    HP_TRY(matched(40, &nm));
    const int ftok = hp_prof_begin(c);
    if (4 * nm < 3 * (int64_t)n) {
        // two-hop through a shared heaviest neighbour: every unmatched vertex
        // names its heaviest neighbour (any neighbour) as its hub; the clients,
        // sorted stably by hub, are paired inside each hub's run
        int32_t *hub = pref;
        HP_LAUNCH(c, pref_small_kernel<false>, blocks_for(n), 256, 0, n, g.xadj, g.adjncy, g.adjwgt,
                  g.vwgt, g.match, elig, hub, lkey, maxvwgt, (const unsigned long long *)nullptr, tn.match_warp_deg);
        HP_LAUNCH(c, pref_big_kernel<false>, persistent_grid(c), 256, 0, big, d_bigcnt, g.xadj,
                  g.adjncy, g.adjwgt, g.vwgt, g.match, elig, hub, lkey, maxvwgt,
                  (const unsigned long long *)nullptr);
        HP_LAUNCH(c, pref_huge_kernel<false>, (unsigned)(2 * c->sm_count), 512, 0, huge, d_hugecnt, g.xadj,
                  g.adjncy, g.adjwgt, g.vwgt, g.match, elig, hub, lkey, maxvwgt,
                  (const unsigned long long *)nullptr);
        HP_LAUNCH(c, client_flag_kernel, blocks_for(n), 256, 0, n, g.match, hub, flags);
        HP_TRY(hp_compact_flags(c, flags, n, list, d_listcnt));
        // sort scratch: the candidate caches are not needed any more
        int32_t *ck = cand, *ck2 = cand + n, *cv2 = cand + 2 * (int64_t)n;
        HP_LAUNCH(c, client_keys_kernel, persistent_grid(c), 256, 0, list, d_listcnt, hub, ck);
        int kbits = 0;
        while ((1ll << kbits) < (int64_t)n) kbits++;
        bool in_tmp = false;
        HP_TRY(hp_sort_pairs(c, ck, list, ck2, cv2, n, d_listcnt, kbits, &in_tmp));
        HP_LAUNCH(c, pair_clients_kernel, persistent_grid(c), 256, 0, in_tmp ? ck2 : ck, in_tmp ? cv2 : list,
                  d_listcnt, g.vwgt, g.match, maxvwgt);
        hp_prof_end(c, ftok, HP_PROF_MATCH_MORE, 0);
        HP_TRY(matched(41, &nm));
    }
    for (int pass = 0; pass < 2; pass++) {
        if (4 * nm >= 3 * (int64_t)n) break;
        // pass 0: isolated vertices; pass 1: every remaining vertex (forced)
        HP_LAUNCH(c, flag_unmatched_kernel, blocks_for(n), 256, 0, n, g.xadj, g.match, flags,
                  pass == 0 ? 1 : 0);
        HP_TRY(hp_compact_flags(c, flags, n, list, d_listcnt));
        HP_LAUNCH(c, pair_list_kernel, blocks_for(n / 2 + 1), 256, 0, list, d_listcnt, g.vwgt,
                  g.match, maxvwgt);
        HP_TRY(matched(42 + pass, &nm));
    }
    HP_LAUNCH(c, finalize_match_kernel, blocks_for(n), 256, 0, n, g.match, flags);
    HP_TRY(hp_scan_excl(c, flags, g.cmap, n));
    int32_t cn = 0;
    HP_TRY(hp_read_scalars(c, g.cmap + n, sizeof(int32_t), &cn));
    *cn_out = cn;
    c->hi = mark;
    return HP_OK;
}

int contract_level(hp_context *c, HpLevel &g, int32_t cn, HpLevel &cg)
{
    const int32_t n = g.n;
    cg.n = cn;
    cg.xadj = lalloc_t<int32_t>(c, cn + 1);
    cg.vwgt = lalloc_t<int32_t>(c, cn);
    // coarse adjacency at the low end with the fine entry count as capacity (an
    // upper bound); the unused tail of the weights is released once m_c is known
    const int64_t cap = std::max<int64_t>(g.m, 1);
    cg.adjncy = lalloc_t<int32_t>(c, cap);
    cg.adjwgt = lalloc_t<int32_t>(c, cap);
    HP_CHECK_OOM(c);
    const size_t mark = c->hi;
    int4 *rinfo = ralloc_t<int4>(c, cn);
    int32_t *toff = ralloc_t<int32_t>(c, (int64_t)cn + 1);
    int32_t *ucnt = ralloc_t<int32_t>(c, (int64_t)cn + 1);
    int32_t *lists = ralloc_t<int32_t>(c, 6 * (int64_t)cn);
    const int64_t ntiles = ((int64_t)cn + ASM_TILE - 1) / ASM_TILE;
    if (ntiles > c->lb_cap) return HP_ERR_INTERNAL;   // reserved at the start of every call
    HP_CHECK_OOM(c);
    unsigned long long *sc = c->d_scal;
    HP_CUDA(cudaMemsetAsync(sc, 0, sizeof(unsigned long long) * 7, c->stream));
    int32_t *counts = (int32_t *)sc;          // 3 long-row class counts + max length in slots 0-1
    int32_t *maxlen = counts + 3;
    unsigned long long *long_total = &sc[2];  // entries of the long rows
    int32_t *small_max = (int32_t *)&sc[3];   // longest short row above 8 entries (0: none)
    int32_t *sub_counts = (int32_t *)&sc[5];  // list 1 split at MROW_MAX and NROW_MAX entries (lists 3-5)

    int tok = hp_prof_begin(c);
    HP_LAUNCH(c, coarse_setup_kernel, blocks_for(n), 256, 0, n, g.match, g.cmap, g.xadj, g.vwgt, rinfo, cg.vwgt,
              toff, lists, counts, cn, maxlen, long_total, small_max, c->tune.contract_thread_row,
              c->tune.contract_warp_row, c->tune.contract_cta_row, MROW_MAX, NROW_MAX, sub_counts);
    hp_prof_end(c, tok, HP_PROF_CONTRACT, 0);
    struct {
        int32_t cnt[3];
        int32_t maxlen;
        unsigned long long total;
        int32_t small_max, pad;
        unsigned long long spill;
        int32_t sub[3], pad2;
    } h;
    static_assert(sizeof(h) == 7 * sizeof(unsigned long long), "the seven scalar slots");
    HP_TRY(hp_read_scalars(c, sc, sizeof(h), &h));
    const bool any_long = h.cnt[0] + h.cnt[1] + h.cnt[2] > 0;
    ContractSrc src{rinfo, g.adjncy, g.adjwgt, g.cmap};
    const int wchk = c->weight_check ? 1 : 0;   // coarse rows' weighted degrees below 2^31
    int32_t *tk = nullptr, *tw = nullptr;
    tok = hp_prof_begin(c);
    if (any_long) {
        // long rows: aggregated into a temporary buffer (offsets by a scan of
        // their lengths), unique counts in ucnt
        HP_TRY(hp_scan_excl(c, toff, toff, cn));
        tk = ralloc_t<int32_t>(c, (int64_t)h.total);
        tw = ralloc_t<int32_t>(c, (int64_t)h.total);
        HP_CHECK_OOM(c);
        // key bits: 2^kbits > cn, so every coarse id (< cn) is below the low
        // kbits bits of KEY_NONE and the dropped self key sorts last
        int kbits = 0;
        while ((1ll << kbits) <= (int64_t)cn) kbits++;
        if (h.cnt[0] > 0)
            HP_LAUNCH(c, contract_warp_radix_kernel,
                      (unsigned)std::min<int64_t>((h.cnt[0] + WROW_WARPS - 1) / WROW_WARPS, c->sm_count * 6),
                      32 * WROW_WARPS, 0, lists, &counts[0], src, toff, tk, tw, ucnt, kbits, wchk, c->d_status);
        // a level whose coarse ids fit a shared-memory dense accumulator merges
        // every long row there (one atomic per entry, ordered extraction)
        const bool smem_dense = cn <= c->tune.contract_smem_cn;
        if (smem_dense) {
            const size_t acc = sizeof(int32_t) * ((size_t)cn + (cn + 31) / 32 + (cn + 1023) / 1024);
            for (int cls = 1; cls <= 2; cls++)
                if (h.cnt[cls] > 0)
                    HP_LAUNCH(c, (contract_dense_kernel<1024, true>),
                              (unsigned)std::min<int64_t>(h.cnt[cls], c->sm_count), 1024, acc,
                              lists + cls * (int64_t)cn, &counts[cls], src, toff, tk, tw, ucnt, cn,
                              (int32_t *)nullptr, (unsigned *)nullptr, (unsigned *)nullptr,
                              c->tune.dense_sparse_ratio, 0, wchk, c->d_status);
        }
        // hybrid: the rows of lists 1 and 2 accumulate their low ids densely and
        // radix-sort the rest; rows whose rest does not fit go to the spill list,
        // which the CTA radix (up to XROW_MAX) and dense slab kernels then take
        const bool hybrid = !smem_dense && cn <= HY_MAX_CN && c->tune.contract_hybrid && h.cnt[1] + h.cnt[2] > 0;
        int32_t *spill = nullptr;
        int32_t *d_nspill = (int32_t *)&sc[4];
        if (hybrid) {
            spill = ralloc_t<int32_t>(c, (int64_t)h.cnt[1] + h.cnt[2]);
            HP_CHECK_OOM(c);
            for (int cls = 1; cls <= 2; cls++)
                if (h.cnt[cls] > 0)
                    HP_LAUNCH(c, contract_hybrid_kernel, (unsigned)std::min<int64_t>(h.cnt[cls], c->sm_count),
                              HY_THREADS, hybrid_smem(), lists + cls * (int64_t)cn, &counts[cls], src, toff, tk, tw,
                              ucnt, kbits, 0, spill, d_nspill, wchk, c->d_status);
            HP_LAUNCH(c, (contract_cta_radix_kernel<XROW_THREADS, XROW_MAX>),
                      (unsigned)std::min<int64_t>((int64_t)h.cnt[1] + h.cnt[2], c->sm_count), XROW_THREADS,
                      (cta_radix_smem<XROW_THREADS, XROW_MAX>()), spill, d_nspill, src, toff, tk, tw, ucnt, kbits, 0,
                      wchk, c->d_status);
        }
        if (!smem_dense && !hybrid && h.sub[0] > 0)
            HP_LAUNCH(c, (contract_cta_radix_kernel<MROW_THREADS, MROW_MAX>),
                      (unsigned)std::min<int64_t>(h.sub[0], c->sm_count * 12), MROW_THREADS,
                      (cta_radix_smem<MROW_THREADS, MROW_MAX>()), lists + 3 * (int64_t)cn, &sub_counts[0], src, toff,
                      tk, tw, ucnt, kbits, 0, wchk, c->d_status);
        if (!smem_dense && !hybrid && h.sub[1] > 0)
            HP_LAUNCH(c, (contract_cta_radix_kernel<NROW_THREADS, NROW_MAX>),
                      (unsigned)std::min<int64_t>(h.sub[1], c->sm_count * 6), NROW_THREADS,
                      (cta_radix_smem<NROW_THREADS, NROW_MAX>()), lists + 4 * (int64_t)cn, &sub_counts[1], src, toff,
                      tk, tw, ucnt, kbits, MROW_MAX, wchk, c->d_status);
        if (!smem_dense && !hybrid && h.sub[2] > 0)
            HP_LAUNCH(c, (contract_cta_radix_kernel<CROW_THREADS, CROW_MAX>),
                      (unsigned)std::min<int64_t>(h.sub[2], c->sm_count * 3), CROW_THREADS,
                      (cta_radix_smem<CROW_THREADS, CROW_MAX>()), lists + 5 * (int64_t)cn, &sub_counts[2], src, toff,
                      tk, tw, ucnt, kbits, NROW_MAX, wchk, c->d_status);
        if (!smem_dense && !hybrid && h.cnt[2] > 0)
            HP_LAUNCH(c, (contract_cta_radix_kernel<XROW_THREADS, XROW_MAX>),
                      (unsigned)std::min<int64_t>(h.cnt[2], c->sm_count), XROW_THREADS,
                      (cta_radix_smem<XROW_THREADS, XROW_MAX>()), lists + 2 * (int64_t)cn, &counts[2], src, toff, tk,
                      tw, ucnt, kbits, 0, wchk, c->d_status);
        if (!smem_dense && h.maxlen > XROW_MAX) {
            // slab per CTA: cn ints + cn/32 + cn/1024 words; bounded to ~512 MB
            const int64_t nw = ((int64_t)cn + 31) / 32, nw2 = ((int64_t)cn + 1023) / 1024;
            int64_t slab = (int64_t)cn * 4 + nw * 4 + nw2 * 4;
            int64_t nb = std::min<int64_t>(h.cnt[2], 2 * (int64_t)c->sm_count);
            nb = std::max<int64_t>(1, std::min<int64_t>(nb, (512ll << 20) / std::max<int64_t>(slab, 1)));
            int32_t *sw = ralloc_t<int32_t>(c, nb * (int64_t)cn);
            unsigned *sbm = ralloc_t<unsigned>(c, nb * nw);
            unsigned *sbm2 = ralloc_t<unsigned>(c, nb * nw2);
            HP_CHECK_OOM(c);
            HP_CUDA(cudaMemsetAsync(sw, 0, sizeof(int32_t) * (size_t)(nb * cn), c->stream));
            HP_CUDA(cudaMemsetAsync(sbm, 0, sizeof(unsigned) * (size_t)(nb * nw), c->stream));
            HP_CUDA(cudaMemsetAsync(sbm2, 0, sizeof(unsigned) * (size_t)(nb * nw2), c->stream));
            HP_LAUNCH(c, (contract_dense_kernel<1024, false>), (unsigned)nb, 1024, 0,
                      hybrid ? spill : lists + 2 * (int64_t)cn, hybrid ? d_nspill : &counts[2], src, toff, tk, tw,
                      ucnt, cn, sw, sbm, sbm2, c->tune.dense_sparse_ratio, XROW_MAX, wchk, c->d_status);
        }
    }
    // short rows + coarse xadj in one ordered pass, then the long rows' copies
    if (h.small_max <= 8)
        HP_LAUNCH(c, contract_assemble_kernel<8>, (unsigned)ntiles, ASM_TILE, asm_smem_bytes<8>(), cn, src, ucnt, cg.xadj,
                  cg.adjncy, cg.adjwgt, c->lb_status, c->lb_ctl, c->d_status, c->tune.contract_thread_row, wchk);
    else if (h.small_max <= 16)
        HP_LAUNCH(c, contract_assemble_kernel<16>, (unsigned)ntiles, ASM_TILE, asm_smem_bytes<16>(), cn, src, ucnt, cg.xadj,
                  cg.adjncy, cg.adjwgt, c->lb_status, c->lb_ctl, c->d_status, c->tune.contract_thread_row, wchk);
    else
        HP_LAUNCH(c, contract_assemble_kernel<32>, (unsigned)ntiles, ASM_TILE, asm_smem_bytes<32>(), cn, src, ucnt, cg.xadj,
                  cg.adjncy, cg.adjwgt, c->lb_status, c->lb_ctl, c->d_status, c->tune.contract_thread_row, wchk);
    if (h.cnt[0] > 0)
        HP_LAUNCH(c, copy_long_rows_kernel<false>, std::min<unsigned>(blocks_for((int64_t)h.cnt[0] * 32),
                                                                     c->sm_count * 16),
                  256, 0, lists, counts, cn, toff, ucnt, cg.xadj, tk, tw, cg.adjncy, cg.adjwgt);
    if (h.cnt[1] + h.cnt[2] > 0)
        HP_LAUNCH(c, copy_long_rows_kernel<true>, (unsigned)std::min<int64_t>(h.cnt[1] + h.cnt[2], c->sm_count * 8),
                  256, 0, lists, counts, cn, toff, ucnt, cg.xadj, tk, tw, cg.adjncy, cg.adjwgt);
    hp_prof_end(c, tok, HP_PROF_CONTRACT, 0);
    int32_t mc = 0;
    HP_TRY(hp_read_scalars(c, cg.xadj + cn, sizeof(int32_t), &mc));
    // algorithmic bytes of the whole contraction: fine CSR, cmap, match, vwgt in;
    // coarse xadj, adjacency, weights, vertex weights out
    hp_prof_add_bytes(c, tok, 4 * ((int64_t)n + 1) + 8 * g.m + 12 * (int64_t)n + 4 * ((int64_t)cn + 1) +
                                  8 * (int64_t)mc + 4 * (int64_t)cn);
    if (mc < 0 || mc > cap) return HP_ERR_INTERNAL;
    cg.m = mc;
    c->lo = (size_t)((char *)cg.adjwgt - c->arena) + ((size_t)std::max<int64_t>(mc, 1) * 4 + HP_ALIGN - 1) / HP_ALIGN * HP_ALIGN;
    c->hi = mark;
    return HP_OK;
}

}  // namespace

int hp_coarsen_init()
{
    HP_CUDA(cudaFuncSetAttribute(contract_assemble_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)asm_smem_bytes<32>()));
    HP_CUDA(cudaFuncSetAttribute(match_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ms_smem_bytes(HP_TUNE_SMALL_MATCH_MAX)));
    HP_CUDA(cudaFuncSetAttribute(contract_dense_kernel<1024, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(int32_t) * (HP_TUNE_SMEM_CN_MAX + (HP_TUNE_SMEM_CN_MAX + 31) / 32 +
                                                          (HP_TUNE_SMEM_CN_MAX + 1023) / 1024))));
    HP_CUDA(cudaFuncSetAttribute(contract_hybrid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)hybrid_smem()));
    HP_CUDA(cudaFuncSetAttribute(contract_cta_radix_kernel<MROW_THREADS, MROW_MAX>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_radix_smem<MROW_THREADS, MROW_MAX>()));
    HP_CUDA(cudaFuncSetAttribute(contract_cta_radix_kernel<NROW_THREADS, NROW_MAX>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_radix_smem<NROW_THREADS, NROW_MAX>()));
    HP_CUDA(cudaFuncSetAttribute(contract_cta_radix_kernel<CROW_THREADS, CROW_MAX>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_radix_smem<CROW_THREADS, CROW_MAX>()));
    HP_CUDA(cudaFuncSetAttribute(contract_cta_radix_kernel<XROW_THREADS, XROW_MAX>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_radix_smem<XROW_THREADS, XROW_MAX>()));
    return HP_OK;
}

int hp_check_weight_range(hp_context *c, const HpLevel &g)
{
    HP_LAUNCH(c, row_weight_range_kernel, blocks_for(g.n), 256, 0, g.n, g.xadj, g.adjwgt, c->d_status);
    return HP_OK;
}

int hp_coarsen(hp_context *c, int32_t coarsen_to, int64_t maxvwgt)
{
    // HP_DEBUG_LEVELS: device time of every level's matching and contraction on stderr
    const bool dbg = getenv("HP_DEBUG_LEVELS") != nullptr;
    cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
    if (dbg)
        for (auto &x : e) HP_CUDA(cudaEventCreate(&x));
    int level = 0;
    int rc = HP_OK;
    while (level < c->opt.max_levels && c->levels[level].n > coarsen_to) {
        HpLevel &g = c->levels[level];
        g.match = lalloc_t<int32_t>(c, g.n);
        g.cmap = lalloc_t<int32_t>(c, (int64_t)g.n + 1);
        if (c->oom) { rc = HP_ERR_NOMEM; break; }
        int32_t cn = 0;
        if (dbg) cudaEventRecord(e[0], c->stream);
        if ((rc = match_level(c, g, level, maxvwgt, &cn)) != HP_OK) break;
        if (dbg) cudaEventRecord(e[1], c->stream);
        c->levels.emplace_back();
        HpLevel &f = c->levels[level];
        HpLevel &cg = c->levels[level + 1];
        if ((rc = contract_level(c, f, cn, cg)) != HP_OK) break;
        if ((rc = hp_check_status(c)) != HP_OK) break;
        if (dbg) {
            cudaEventRecord(e[2], c->stream);
            cudaEventSynchronize(e[2]);
            float ms_m = 0.f, ms_c = 0.f;
            cudaEventElapsedTime(&ms_m, e[0], e[1]);
            cudaEventElapsedTime(&ms_c, e[1], e[2]);
            fprintf(stderr, "gpu coarsen level %d n=%d m=%lld match_ms=%.3f contract_ms=%.3f\n", level, f.n,
                    (long long)f.m, ms_m, ms_c);
        }
        level++;
        if (!(100 * (int64_t)cg.n < 85 * (int64_t)f.n && cg.m > cg.n / 2)) break;
    }
    if (dbg)
        for (auto &x : e) cudaEventDestroy(x);
    return rc;
}
