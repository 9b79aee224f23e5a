// hp_refine.cu — uncoarsening: projection and Jet-style k-way refinement over an
// integer gain table, with exact int64 cut tracking.
//
// Reference behaviour replaced (HunyuanGraph):
//   uncoarsening driver / projection      hunyuangraph_GPU_uncoarsen.h:196-223, 555-587
//   pass loop + best partition            hunyuangraph_GPU_krefine.h:4434-4882
//   gain table (set_gain_offset/val)      :4202-4432, rebuild of neighbours :3632-3726
//   LP: select_dest_part, filter,         :1995-2221
//       afterburner, lock
//   weak rebalance (jetrw)                :3136-3563, gain_bucket :2477-2513
//   strong rebalance (jetrs, cookie cut)  :2515-3135
//   perform_moves + cut change            :3933-4155
// Differences by design: every count/filter is a scan or a block reduction
// instead of atomic append order, bucket order inside a part is (bucket,
// vertex id) via a stable radix sort, the cut is int64, balance is judged
// against integer maximum part weights, and one status read per pass replaces
// the reference's 4-6 blocking reads.
#include <chrono>
#include <cstdlib>

#include "hp_internal.cuh"
#include "hp_mlp.cuh"
#include "hp_rowagg.cuh"

namespace {

// Row classes of refinement (hp_tuning): rows of at most `bigd` entries take a
// thread (or a lane segment), longer rows a warp, and hub rows (more than
// `huged` entries) a CTA or grid-wide chunks.  bigd <= 32, the register
// networks' width.
constexpr int32_t NEG = INT_MIN;

inline unsigned nblk(int64_t n, int b = 256) { return (unsigned)std::max<int64_t>(1, (n + b - 1) / b); }

__global__ void project_kernel(int32_t n, const int32_t *__restrict__ cmap,
                               const int32_t *__restrict__ cwhere, int32_t *__restrict__ where)
{
    hp::pdl_wait();
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) where[v] = cwhere[cmap[v]];
}

// Row capacities min(deg, k); rows longer than bigd go on the big list, rows
// longer than huged (the caller's chunk_deg) also on the long-row list (count
// d_bigcnt[3]), rows longer than hubd (gain_hub_deg) on the hub list (count
// d_bigcnt[4]); d_bigcnt[1] records the longest short row above 8 entries,
// d_bigcnt[2] the longest row above huged.
__global__ void gain_cap_kernel(int32_t n, const int32_t *__restrict__ xadj, int32_t k,
                                int32_t *__restrict__ cap, int32_t *big, int32_t *huge, int32_t *hub,
                                int32_t *d_bigcnt, int32_t bigd, int32_t huged, int32_t hubd)
{
    hp::pdl_wait();
    // no early exit: the list appends and maxima are aggregated per warp
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t d = 0;
    if (v < n) {
        d = xadj[v + 1] - xadj[v];
        cap[v] = d < k ? d : k;
    }
    const bool is_big = v < n && d > bigd, is_huge = is_big && d > huged, is_hub = is_big && d > hubd;
    const int32_t pb = hp::warp_append(d_bigcnt, is_big);
    const int32_t ph = hp::warp_append(d_bigcnt + 3, is_huge);
    const int32_t pu = hp::warp_append(d_bigcnt + 4, is_hub);
    if (is_big) big[pb] = v;
    if (is_huge) huge[ph] = v;
    if (is_hub) hub[pu] = v;
    const int32_t hm = hp::warp_max(is_huge ? d : 0);
    const int32_t sm = hp::warp_max(v < n && !is_big && d > 8 ? d : 0);
    if ((threadIdx.x & 31) == 0) {
        if (hm > 0) atomicMax(d_bigcnt + 2, hm);
        if (sm > 0) atomicMax(d_bigcnt + 1, sm);
    }
}

// Degree statistics of a level, computed for every level at the start of
// uncoarsening so that the host chooses each level's kernels without reading
// anything back per level: rows longer than bigd, the longest row of 9..bigd
// entries, the longest row overall.
struct LevelStat {
    int32_t nbig, small_max, maxdeg, pad;
};

__global__ void __launch_bounds__(256)
level_stats_kernel(int32_t n, const int32_t *__restrict__ xadj, LevelStat *st, int32_t bigd)
{
    hp::pdl_wait();
    int32_t nbig = 0, smax = 0, dmax = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = xadj[v + 1] - xadj[v];
        if (d > bigd) nbig++;
        else if (d > 8) smax = d > smax ? d : smax;
        dmax = d > dmax ? d : dmax;
    }
    nbig = hp::warp_sum(nbig);
    smax = __reduce_max_sync(HP_FULL_MASK, (unsigned)smax);
    dmax = __reduce_max_sync(HP_FULL_MASK, (unsigned)dmax);
    if ((threadIdx.x & 31) == 0) {
        if (nbig) atomicAdd(&st->nbig, nbig);
        if (smax) atomicMax(&st->small_max, smax);
        if (dmax) atomicMax(&st->maxdeg, dmax);
    }
}

// Gain row of a vertex with at most bigd neighbours, one thread per row: the
// (part, weight) pairs are sorted by a register network and merged, then
// written as the sparse row (ascending parts, part -1 padding up to the
// capacity) or, when deg >= k, as the dense row (entry q = part q).
template <int NET, int XN>
__device__ __forceinline__ void gain_row_thread(int32_t b, int32_t d, const int32_t *__restrict__ adjncy,
                                                const int32_t *__restrict__ adjwgt,
                                                const int32_t *__restrict__ where, int32_t *__restrict__ gp,
                                                int32_t *__restrict__ gc, int32_t cap, int32_t k)
{
    unsigned long long x[XN];
#pragma unroll
    for (int i = 0; i < NET; i++)
        x[i] = i < d ? (((unsigned long long)(uint32_t)where[adjncy[b + i]] << 32) | (uint32_t)adjwgt[b + i])
                     : hp::PACK_NONE;
    hp::sort_regs<NET, XN>(x);
    const bool dense = d >= k;
    int32_t r = 0, next = 0;
    uint32_t prev = 0xffffffffu;
    int32_t acc = 0;
    auto flush = [&](int32_t q, int32_t sum) {
        if (dense) {
            for (; next < q; next++) { gp[next] = next; gc[next] = 0; }
            gp[q] = q;
            gc[q] = sum;
            next = q + 1;
        } else {
            gp[r] = q;
            gc[r] = sum;
            r++;
        }
    };
#pragma unroll
    for (int i = 0; i < NET; i++) {
        const uint32_t q = (uint32_t)(x[i] >> 32);
        const int32_t w = (int32_t)(uint32_t)x[i];
        if (q == (uint32_t)hp::KEY_NONE) continue;
        if (q != prev) {
            if (prev != 0xffffffffu) flush((int32_t)prev, acc);
            prev = q;
            acc = w;
        } else {
            acc += w;
        }
    }
    if (prev != 0xffffffffu) flush((int32_t)prev, acc);
    if (dense) {
        for (; next < k; next++) { gp[next] = next; gc[next] = 0; }
    } else {
        for (; r < cap; r++) { gp[r] = -1; gc[r] = 0; }
    }
}

// list == nullptr: every vertex (rows longer than bigd are skipped: the big-row
// kernel builds them); else the listed vertices, whose dirty flags are cleared.
template <int XN>
__global__ void __launch_bounds__(256)
gain_thread_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count, int32_t n,
                   const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                   const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ where,
                   const int32_t *__restrict__ goff, int32_t *__restrict__ gpart,
                   int32_t *__restrict__ gconn, int32_t k, int32_t *__restrict__ dirty, int32_t bigd)
{
    hp::pdl_wait();
    const int32_t cnt = list ? *d_count : n;
    for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x; i0 < cnt; i0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = i0 + threadIdx.x;
        int32_t v = -1, b = 0, d = 0;
        if (i < cnt) {
            v = list ? list[i] : (int32_t)i;
            b = xadj[v];
            d = xadj[v + 1] - b;
            if (dirty) dirty[v] = 0;
        }
        const bool mine = v >= 0 && d <= bigd;
        const unsigned wmax = __reduce_max_sync(HP_FULL_MASK, mine ? (unsigned)d : 0u);
        if (!mine) continue;
        const int32_t o = goff[v], cap = goff[v + 1] - o;
        if (XN == 8 || wmax <= 8)
            gain_row_thread<8, XN>(b, d, adjncy, adjwgt, where, gpart + o, gconn + o, cap, k);
        else if (XN == 16 || wmax <= 16)
            gain_row_thread<(XN < 16 ? XN : 16), XN>(b, d, adjncy, adjwgt, where, gpart + o, gconn + o, cap, k);
        else
            gain_row_thread<XN, XN>(b, d, adjncy, adjwgt, where, gpart + o, gconn + o, cap, k);
    }
}

// Gain row of v: (part, connectivity) for every part adjacent to v, ascending
// by part, padded with part -1 up to min(deg, k).  A vertex with deg >= k has a
// dense row instead: entry q is (q, conn to part q), zeros included; dense rows
// are updated in place by atomics when a neighbour moves and never rebuilt.
// Rebuild of the listed (dirty) rows of at most S entries (S >= the level's
// longest short row): 32/S rows per warp, one segment of S lanes per row,
// sorted and merged by seg_aggregate; dirty flags are cleared.  Rows with
// deg >= k (k <= S here) are written dense.
// (warp, nwarps: this warp's index among the nwarps warps sharing the list)
template <int S>
__device__ __forceinline__ void gain_seg_rows(int64_t warp, int64_t nwarps, const int32_t *__restrict__ list,
                                              int32_t cnt, const int32_t *__restrict__ xadj,
                                              const int32_t *__restrict__ adjncy, const int32_t *__restrict__ adjwgt,
                                              const int32_t *__restrict__ where, const int32_t *__restrict__ goff,
                                              int32_t *__restrict__ gpart, int32_t *__restrict__ gconn, int32_t k,
                                              int32_t *__restrict__ dirty)
{
    constexpr int R = 32 / S;
    const int lane = threadIdx.x & 31, sl = lane & (S - 1);
    for (int64_t i0 = warp * R; i0 < cnt; i0 += nwarps * R) {
        const int64_t i = i0 + lane / S;
        int32_t v = -1, b = 0, d = 0;
        if (i < cnt) {
            v = list[i];
            b = xadj[v];
            d = xadj[v + 1] - b;
            if (sl == 0) dirty[v] = 0;
        }
        int32_t key = hp::KEY_NONE, w = 0;
        if (v >= 0 && sl < d) {
            key = where[adjncy[b + sl]];
            w = adjwgt[b + sl];
        }
        const int32_t o = v >= 0 ? goff[v] : 0, cap = v >= 0 ? goff[v + 1] - o : 0;
        const bool dense = v >= 0 && d >= k;
        if (dense && sl < k) { gpart[o + sl] = sl; gconn[o + sl] = 0; }
        __syncwarp();
        if (dense && key != hp::KEY_NONE) atomicAdd(&gconn[o + key], w);
        const int c = hp::seg_aggregate<S>(key, w, (v >= 0 && !dense) ? gpart + o : nullptr,
                                            (v >= 0 && !dense) ? gconn + o : nullptr);
        if (v >= 0 && !dense)
            for (int32_t t = c + sl; t < cap; t += S) { gpart[o + t] = -1; gconn[o + t] = 0; }
    }
}

template <int S>
__global__ void __launch_bounds__(256)
gain_seg_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ where,
                const int32_t *__restrict__ goff, int32_t *__restrict__ gpart, int32_t *__restrict__ gconn,
                int32_t k, int32_t *__restrict__ dirty)
{
    hp::pdl_wait();
    gain_seg_rows<S>((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5, ((int64_t)gridDim.x * blockDim.x) >> 5,
                     list, *d_count, xadj, adjncy, adjwgt, where, goff, gpart, gconn, k, dirty);
}

// Gain rows of bigd+1 .. huged entries when k <= warp_dense_k: one warp per
// row with its own dense accumulator and presence bitmap over the k parts in
// shared memory (k + k/32 words per warp), extracted in part order; only warp
// synchronisation.  Longer rows (and any row when k is larger) use
// gain_dense_kernel.
constexpr int GW_WARPS = 8;   // k + k/32 words per warp: 33 KB at k = HP_TUNE_WARP_DENSE_K_MAX

// The rows of one warp: dw (k words) and bm (ceil(k/32) words) are the warp's
// own accumulators, zero on entry and left zero.
__device__ __forceinline__ void gain_bigwarp_rows(int64_t warp, int64_t nwarps, int32_t *dw, unsigned *bm,
                                                  const int32_t *__restrict__ list, int32_t cnt,
                                                  const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                                                  const int32_t *__restrict__ adjwgt,
                                                  const int32_t *__restrict__ where, const int32_t *__restrict__ goff,
                                                  int32_t *__restrict__ gpart, int32_t *__restrict__ gconn, int32_t k,
                                                  int32_t *__restrict__ dirty, int32_t bigd, int32_t huged)
{
    const int lane = threadIdx.x & 31;
    const int nwords = (k + 31) >> 5;
    for (int64_t li = warp; li < cnt; li += nwarps) {
        const int32_t v = list[li];
        const int32_t b = xadj[v], e = xadj[v + 1];
        if (e - b <= bigd || e - b > huged) continue;
        if (dirty && lane == 0) dirty[v] = 0;
        // a row of at least k entries becomes a dense row (entry q = part q):
        // its presence bits are never read
        const bool dense = e - b >= k;
        for (int32_t j = b + lane; j < e; j += 128) {   // four chunks in flight
            int32_t u[4], w[4], q[4];
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const int32_t jj = j + 32 * t;
                u[t] = jj < e ? adjncy[jj] : -1;
                w[t] = jj < e ? adjwgt[jj] : 0;
            }
#pragma unroll
            for (int t = 0; t < 4; t++) q[t] = u[t] >= 0 ? where[u[t]] : -1;   // the four gathers together
#pragma unroll
            for (int t = 0; t < 4; t++) {
                if (q[t] < 0) continue;
                atomicAdd(&dw[q[t]], w[t]);
                if (!dense) atomicOr(&bm[q[t] >> 5], 1u << (q[t] & 31));
            }
        }
        __syncwarp();
        const int32_t o = goff[v], cap = goff[v + 1] - o;
        if (dense) {   // (no presence bits were set)
            for (int32_t q = lane; q < k; q += 32) {
                gpart[o + q] = q;
                gconn[o + q] = dw[q];
                dw[q] = 0;
            }
            __syncwarp();
            continue;
        }
        int32_t run = 0;
        for (int wb = 0; wb < nwords; wb += 32) {
            const int wi = wb + lane;
            unsigned word = wi < nwords ? bm[wi] : 0u;
            const int c = __popc(word);
            const int incl = hp::warp_incl_scan(c);
            int32_t pos = run + incl - c;
            run += __shfl_sync(HP_FULL_MASK, incl, 31);
            if (word) bm[wi] = 0u;
            while (word) {
                const int bit = __ffs(word) - 1;
                word &= word - 1;
                const int32_t q = (wi << 5) + bit;
                gpart[o + pos] = q;
                gconn[o + pos] = dw[q];
                dw[q] = 0;
                pos++;
            }
        }
        for (int32_t t = run + lane; t < cap; t += 32) { gpart[o + t] = -1; gconn[o + t] = 0; }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(32 * GW_WARPS)
gain_bigwarp_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                    const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                    const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ where,
                    const int32_t *__restrict__ goff, int32_t *__restrict__ gpart,
                    int32_t *__restrict__ gconn, int32_t k, int32_t *__restrict__ dirty, int32_t bigd,
                    int32_t huged)
{
    hp::pdl_wait();
    extern __shared__ int32_t gsm[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nwords = (k + 31) >> 5;
    int32_t *dw = gsm + wid * (k + nwords);
    unsigned *bm = (unsigned *)(dw + k);
    for (int i = lane; i < k; i += 32) dw[i] = 0;
    for (int i = lane; i < nwords; i += 32) bm[i] = 0u;
    __syncwarp();
    gain_bigwarp_rows((int64_t)blockIdx.x * GW_WARPS + wid, (int64_t)gridDim.x * GW_WARPS, dw, bm, list, *d_count,
                      xadj, adjncy, adjwgt, where, goff, gpart, gconn, k, dirty, bigd, huged);
}

template <int NT>
__global__ void __launch_bounds__(NT)
gain_dense_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                  const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                  const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ where,
                  const int32_t *__restrict__ goff, int32_t *__restrict__ gpart,
                  int32_t *__restrict__ gconn, int32_t k, int32_t *__restrict__ dirty, int32_t bigd,
                  int32_t huged, int32_t warp_dense_k)
{
    hp::pdl_wait();
    extern __shared__ int32_t dsm[];
    __shared__ int32_t s_scan[NT / 32 + 2];
    int32_t *dw = dsm;
    unsigned *bm = (unsigned *)(dsm + k);
    const int nwords = (k + 31) >> 5;
    for (int i = threadIdx.x; i < k; i += NT) dw[i] = 0;
    for (int i = threadIdx.x; i < nwords; i += NT) bm[i] = 0;
    __syncthreads();
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t v = list[li];
        const int32_t b = xadj[v], e = xadj[v + 1];
        if (e - b <= bigd) continue;
        if (k <= warp_dense_k && e - b <= huged) continue;   // gain_bigwarp_kernel's rows
        if (dirty && threadIdx.x == 0) dirty[v] = 0;
        // a row of at least k entries becomes a dense row (entry q = part q):
        // its presence bits are never read
        const bool dense = e - b >= k;
        for (int32_t j = b + threadIdx.x; j < e; j += 4 * NT) {   // four entries per thread in flight
            int32_t u[4], w[4], q[4];
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const int32_t jj = j + NT * t;
                u[t] = jj < e ? adjncy[jj] : -1;
                w[t] = jj < e ? adjwgt[jj] : 0;
            }
#pragma unroll
            for (int t = 0; t < 4; t++) q[t] = u[t] >= 0 ? where[u[t]] : -1;
#pragma unroll
            for (int t = 0; t < 4; t++) {
                if (q[t] < 0) continue;
                atomicAdd(&dw[q[t]], w[t]);
                if (!dense) atomicOr(&bm[q[t] >> 5], 1u << (q[t] & 31));
            }
        }
        __syncthreads();
        const int32_t o = goff[v], cap = goff[v + 1] - o;
        if (dense) {
            for (int32_t q = threadIdx.x; q < k; q += NT) {
                gpart[o + q] = q;
                gconn[o + q] = dw[q];
                dw[q] = 0;
            }
            __syncthreads();
            continue;
        }
        int c = hp::dense_extract<NT>(dw, bm, k, gpart + o, gconn + o, s_scan);
        for (int32_t t = c + threadIdx.x; t < cap; t += NT) { gpart[o + t] = -1; gconn[o + t] = 0; }
        __syncthreads();
    }
}

__device__ __forceinline__ int32_t row_conn(const int32_t *gp, const int32_t *gc, int32_t len, int32_t q,
                                            int32_t k)
{
    if (len == k) return gc[q];   // dense row
    // rows are ascending by part and padded with -1: bisect to a short window
    // (entries before lo are parts below q; entries from hi on are padding or
    // parts >= q), then walk to the first entry that is padding or >= q
    int32_t lo = 0, hi = len;
    while (hi - lo > 8) {
        const int32_t mid = (lo + hi) >> 1;
        const int32_t p = gp[mid];
        if (p >= 0 && p < q) lo = mid + 1;
        else hi = mid;
    }
    for (int32_t j = lo; j < len; j++) {
        const int32_t p = gp[j];
        if (p == q) return gc[j];
        if (p < 0 || p > q) break;
    }
    return 0;
}

__global__ void __launch_bounds__(256)
pw_kernel(int32_t n, const int32_t *__restrict__ where, const int32_t *__restrict__ vwgt,
          unsigned long long *__restrict__ pw, int32_t k)
{
    hp::pdl_wait();
    extern __shared__ unsigned long long spw[];
    const bool use_s = k <= 2048;
    if (use_s) {
        for (int i = threadIdx.x; i < k; i += blockDim.x) spw[i] = 0;
        __syncthreads();
    }
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        if (use_s) atomicAdd(&spw[where[v]], (unsigned long long)vwgt[v]);
        else atomicAdd(&pw[where[v]], (unsigned long long)vwgt[v]);
    }
    if (use_s) {
        __syncthreads();
        for (int i = threadIdx.x; i < k; i += blockDim.x)
            if (spw[i]) atomicAdd(&pw[i], spw[i]);
    }
}

// 2 x cut from the gain rows.
__global__ void __launch_bounds__(256)
rowcut_kernel(int32_t n, const int32_t *__restrict__ goff, const int32_t *__restrict__ gpart,
              const int32_t *__restrict__ gconn, const int32_t *__restrict__ where,
              unsigned long long *cut2)
{
    hp::pdl_wait();
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    long long acc = 0;
    int32_t p = 0, o = 0, len = 0;
    if (v < n) {
        p = where[v];
        o = goff[v];
        len = goff[v + 1] - o;
    }
    // rows longer than 32 entries are summed by the whole warp, one at a time
    const bool coop = len > 32;
    if (!coop)
        for (int32_t j = o; j < o + len; j++) {
            const int32_t q = gpart[j];
            if (q < 0) break;
            if (q != p) acc += gconn[j];
        }
    unsigned cm = __ballot_sync(HP_FULL_MASK, coop);
    while (cm) {
        const int src = __ffs(cm) - 1;
        cm &= cm - 1;
        const int32_t so = __shfl_sync(HP_FULL_MASK, o, src), sl = __shfl_sync(HP_FULL_MASK, len, src);
        const int32_t sp = __shfl_sync(HP_FULL_MASK, p, src);
        for (int32_t j = lane; j < sl; j += 32) {
            const int32_t q = gpart[so + j];
            if (q < 0) break;
            if (q != sp) acc += gconn[so + j];
        }
    }
    hp::block_add_to<256>(acc, cut2);
}

// Status of a pass: [0] moves, [1] c1, [2] c2 (as written by kernels),
// [3] max excess (written here).
__global__ void excess_kernel(int32_t k, const unsigned long long *__restrict__ pw,
                              const int64_t *__restrict__ maxp, long long *out)
{
    hp::pdl_wait();
    long long m = LLONG_MIN;
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        long long e = (long long)pw[p] - maxp[p];
        m = e > m ? e : m;
    }
    m = hp::warp_max64(m);
    __shared__ long long s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = s[w] > m ? s[w] : m;
        *out = m;
    }
}

// One gain row against the own part p: connectivity to p (pc), the best other
// part b (largest connectivity, the first -- lowest -- part among equals; -1
// when no other part has positive connectivity) and bc, the row's total
// connectivity wd and its count np of parts with positive connectivity.
struct RowBest {
    int64_t pc, bc, wd;
    int32_t b, np;
};

// Called by every lane of the warp, each with its own row (len 0 for none).
// Rows of at most 32 entries are walked by their lane; longer rows by the
// whole warp, one row at a time, reduced in the serial walk's order.
__device__ __forceinline__ RowBest row_best(const int32_t *__restrict__ gpart, const int32_t *__restrict__ gconn,
                                            int32_t o, int32_t len, int32_t p, int32_t k)
{
    const int lane = threadIdx.x & 31;
    RowBest r{0, 0, 0, -1, 0};
    const bool coop = len > 32;
    if (!coop)
        for (int32_t j = o; j < o + len; j++) {
            const int32_t q = gpart[j];
            if (q < 0) break;
            const int32_t cq = gconn[j];
            r.wd += cq;
            r.np += cq > 0;
            if (q == p) { r.pc = cq; continue; }
            if (cq > r.bc) { r.bc = cq; r.b = q; }   // ascending parts: first max = lowest part
        }
    unsigned cm = __ballot_sync(HP_FULL_MASK, coop);
    while (cm) {
        const int src = __ffs(cm) - 1;
        cm &= cm - 1;
        const int32_t so = __shfl_sync(HP_FULL_MASK, o, src), sl = __shfl_sync(HP_FULL_MASK, len, src);
        const int32_t sp = __shfl_sync(HP_FULL_MASK, p, src);
        int32_t lpc = 0, lbc = 0, lb = -1, lnp = 0;
        long long lwd = 0;
        const bool dense = sl == k;   // entry j is part j
        for (int32_t j = lane; j < sl; j += 32) {
            const int32_t q = dense ? j : gpart[so + j];
            if (q < 0) break;   // padding runs to the end of the row
            const int32_t cq = gconn[so + j];
            lwd += cq;
            lnp += cq > 0;
            if (q == sp) { lpc = cq; continue; }
            if (cq > lbc) { lbc = cq; lb = q; }
        }
        lpc = hp::warp_sum(lpc);
        lnp = hp::warp_sum(lnp);
        lwd = hp::warp_sum64(lwd);
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) {
            const int32_t ob = __shfl_xor_sync(HP_FULL_MASK, lb, sh);
            const int32_t oc = __shfl_xor_sync(HP_FULL_MASK, lbc, sh);
            if (ob >= 0 && (lb < 0 || oc > lbc || (oc == lbc && ob < lb))) { lb = ob; lbc = oc; }
        }
        if (lane == src) { r.pc = lpc; r.bc = lbc; r.b = lb; r.wd = lwd; r.np = lnp; }
    }
    return r;
}

// The best partition so far, copied by the first proposal kernel of the next
// pass: when the previous pass set the control block's take flag, the partition
// it left is the best so far, and that kernel, which reads where[v] of every
// vertex anyway, stores it into best_where (and block / tile 0 the part weights
// into best_pw) before any move of its own pass is applied.  A pass that ends
// the level needs no copy: where is then either the best (take set) or
// restored from best_where.
struct BestCopy {
    const int32_t *take;
    int32_t *best_where;
    const unsigned long long *pw;
    unsigned long long *best_pw;
    int32_t k;
    __device__ __forceinline__ bool on() const { return *take != 0; }
    __device__ __forceinline__ void parts() const
    {
        for (int32_t q = threadIdx.x; q < k; q += blockDim.x) best_pw[q] = pw[q];
    }
};

// Long gain rows (more than 32 entries) of a CTA, shared by all its warps: the
// rows are queued in shared memory and the warps take them in turn, so that a
// warp with many long rows does not hold the whole CTA at its next barrier
// (the look-back of rb_candidates_kernel, the block sums of the LP selection).
// A row's result does not depend on the warp that walks it.
template <int NT>
struct CoopRows {
    int32_t o[NT], len[NT], p[NT];
    long long pc[NT], bc[NT], wd[NT];
    int32_t b[NT], np[NT];
    int32_t n;
};

// Queues the calling thread's row when it is long; returns its queue slot or -1.
// All NT threads call it; it ends with a barrier.
template <int NT>
__device__ __forceinline__ int coop_queue(CoopRows<NT> &S, bool coop, int32_t o, int32_t len, int32_t p)
{
    if (threadIdx.x == 0) S.n = 0;
    __syncthreads();
    int my = -1;
    if (coop) {
        my = atomicAdd(&S.n, 1);
        S.o[my] = o;
        S.len[my] = len;
        S.p[my] = p;
    }
    __syncthreads();
    return my;
}

// row_best with the CTA's long rows shared by all its warps (CoopRows).  All NT
// threads call it.
template <int NT>
__device__ __forceinline__ RowBest row_best_cta(CoopRows<NT> &S, const int32_t *__restrict__ gpart,
                                                const int32_t *__restrict__ gconn, int32_t o, int32_t len,
                                                int32_t p, int32_t k)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    RowBest r{0, 0, 0, -1, 0};
    const bool coop = len > 32;
    if (!coop)
        for (int32_t j = o; j < o + len; j++) {
            const int32_t q = gpart[j];
            if (q < 0) break;
            const int32_t cq = gconn[j];
            r.wd += cq;
            r.np += cq > 0;
            if (q == p) { r.pc = cq; continue; }
            if (cq > r.bc) { r.bc = cq; r.b = q; }   // ascending parts: first max = lowest part
        }
    const int my = coop_queue<NT>(S, coop, o, len, p);
    const int nc = S.n;
    for (int i = wid; i < nc; i += NT / 32) {
        const int32_t so = S.o[i], sl = S.len[i], sp = S.p[i];
        int32_t lpc = 0, lbc = 0, lb = -1, lnp = 0;
        long long lwd = 0;
        const bool dense = sl == k;   // entry j is part j
        for (int32_t j = lane; j < sl; j += 32) {
            const int32_t q = dense ? j : gpart[so + j];
            if (q < 0) break;   // padding runs to the end of the row
            const int32_t cq = gconn[so + j];
            lwd += cq;
            lnp += cq > 0;
            if (q == sp) { lpc = cq; continue; }
            if (cq > lbc) { lbc = cq; lb = q; }
        }
        lpc = hp::warp_sum(lpc);
        lnp = hp::warp_sum(lnp);
        lwd = hp::warp_sum64(lwd);
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) {
            const int32_t ob = __shfl_xor_sync(HP_FULL_MASK, lb, sh);
            const int32_t oc = __shfl_xor_sync(HP_FULL_MASK, lbc, sh);
            if (ob >= 0 && (lb < 0 || oc > lbc || (oc == lbc && ob < lb))) { lb = ob; lbc = oc; }
        }
        if (lane == 0) { S.pc[i] = lpc; S.bc[i] = lbc; S.b[i] = lb; S.wd[i] = lwd; S.np[i] = lnp; }
    }
    __syncthreads();
    if (my >= 0) { r.pc = S.pc[my]; r.bc = S.bc[my]; r.b = S.b[my]; r.wd = S.wd[my]; r.np = S.np[my]; }
    return r;
}

// ---- LP ------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
lp_select_kernel(int32_t n, const int32_t *__restrict__ goff, const int32_t *__restrict__ gpart,
                 const int32_t *__restrict__ gconn, const int32_t *__restrict__ where,
                 const int8_t *__restrict__ lock, int finest, int32_t *__restrict__ dest,
                 int32_t *__restrict__ pregain, unsigned long long *d_ncand, const int32_t *gate, int32_t k,
                 BestCopy bcp)
{
    hp::pdl_wait();
    if (gate && *gate != 0) return;   // graph mode: the learned kernel runs this pass
    __shared__ CoopRows<256> S;
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    const bool copy = bcp.on();
    if (copy && blockIdx.x == 0) bcp.parts();
    int cand = 0;
    int32_t p = 0, o = 0, len = 0;
    if (v < n) {
        p = where[v];
        o = goff[v];
        len = goff[v + 1] - o;
        if (copy) bcp.best_where[v] = p;
    }
    const RowBest rb = row_best_cta<256>(S, gpart, gconn, o, len, p, k);
    const int64_t pc = rb.pc, bc = rb.bc;
    const int32_t b = rb.b;
    if (v < n) {
        int32_t g = NEG, d = p;
        if (b >= 0) {
            int64_t thr = finest ? pc / 4 : (3 * pc) / 4;
            if ((bc >= pc || (pc - bc) < thr) && !lock[v]) { g = (int32_t)(bc - pc); d = b; cand = 1; }
        }
        pregain[v] = g;
        dest[v] = d;
    }
    hp::block_add_to<256>(cand, d_ncand);
}

// Learned LP selection: the plain rule first, then the MLP scores every
// candidate (all lanes of a warp run the tensor-core inference together) and
// drops candidates scoring below the threshold.  Dropped candidates stay put;
// under the judge (learned = 3) they keep their plain gain and destination
// with prune[v] = 1, so that the afterburner leaves them out of the learned
// move set but keeps them in the plain set it judges the pass by.  Nothing the
// network says bypasses the exact afterburner.
__global__ void __launch_bounds__(256)
lp_select_learned_kernel(int32_t n, const int32_t *__restrict__ goff, const int32_t *__restrict__ gpart,
                         const int32_t *__restrict__ gconn, const int32_t *__restrict__ where,
                         const int32_t *__restrict__ xadj, const int8_t *__restrict__ lock, int finest,
                         const unsigned long long *__restrict__ pw, const int64_t *__restrict__ maxp,
                         const int64_t *__restrict__ opt, const float *__restrict__ params, float threshold,
                         int32_t *__restrict__ dest, int32_t *__restrict__ pregain, unsigned long long *d_ncand,
                         const int32_t *gate, int32_t k, int8_t *__restrict__ prune,
                         unsigned long long *d_ncandp, const int32_t *judge_flag, BestCopy bcp)
{
    hp::pdl_wait();
    if (gate && *gate != 1) return;   // graph mode: the plain kernel runs this pass
    __shared__ hp::MlpSmem sm;
    __shared__ CoopRows<256> S;
    hp::mlp_load_smem(sm, params);
    __syncthreads();
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    const bool copy = bcp.on();
    if (copy && blockIdx.x == 0) bcp.parts();
    int cand = 0, candp = 0;
    int8_t pr = 0;
    float f[HP_MLP_IN] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int32_t g = NEG, d = 0;
    int32_t p = 0, o = 0, len = 0;
    if (v < n) {
        p = where[v];
        o = goff[v];
        len = goff[v + 1] - o;
        if (copy) bcp.best_where[v] = p;
    }
    const RowBest rb = row_best_cta<256>(S, gpart, gconn, o, len, p, k);
    if (v < n) {
        const int64_t pc = rb.pc, bc = rb.bc, wd = rb.wd;
        const int32_t b = rb.b, np = rb.np;
        d = p;
        if (b >= 0) {
            int64_t thr = finest ? pc / 4 : (3 * pc) / 4;
            if ((bc >= pc || (pc - bc) < thr) && !lock[v]) {
                g = (int32_t)(bc - pc);
                d = b;
                cand = 1;
                candp = 1;
                hp::mlp_features(pc, bc, wd, np, xadj[v + 1] - xadj[v], maxp[b] - (int64_t)pw[b], opt[b],
                                 maxp[p] - (int64_t)pw[p], opt[p], finest, f);
            }
        }
    }
    // the warp's tensor-core inference only when one of its vertices is a
    // candidate (the logit is read for candidates alone; the vote is uniform)
    float logit = 0.0f;
    if (__any_sync(HP_FULL_MASK, cand)) logit = hp::mlp_warp_logit(sm, f);
    // under the judge a dropped candidate keeps its plain gain and destination
    const bool judge = *judge_flag != 0;
    if (cand && logit < threshold) {
        cand = 0;
        if (judge) pr = 1;
        else { g = NEG; d = where[v]; }
    }
    if (v < n) {
        pregain[v] = g;
        dest[v] = d;
        if (judge) prune[v] = pr;
    }
    hp::block_add_to<256>(cand, d_ncand);
    if (judge) hp::block_add_to<256>(candp, d_ncandp);
}

// Move log (record mode): features of every LP candidate, its vertex and
// destination; rec_of[v] links the vertex to its record for the afterburner.
__global__ void __launch_bounds__(256)
log_candidates_kernel(int32_t n, const int32_t *__restrict__ goff, const int32_t *__restrict__ gpart,
                      const int32_t *__restrict__ gconn, const int32_t *__restrict__ where,
                      const int32_t *__restrict__ xadj, int finest, const unsigned long long *__restrict__ pw,
                      const int64_t *__restrict__ maxp, const int64_t *__restrict__ opt,
                      const int32_t *__restrict__ dest, const int32_t *__restrict__ pregain,
                      int32_t *__restrict__ rec_of, float *__restrict__ lx, int32_t *__restrict__ lv,
                      int32_t *__restrict__ ld, int32_t *__restrict__ lacc, unsigned long long *lcount, int64_t cap)
{
    hp::pdl_wait();
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    rec_of[v] = -1;
    if (pregain[v] == NEG) return;
    const int32_t p = where[v], b = dest[v];
    int64_t pc = 0, bc = 0, wd = 0;
    int32_t np = 0;
    for (int32_t j = goff[v]; j < goff[v + 1]; j++) {
        int32_t q = gpart[j];
        if (q < 0) break;
        int32_t cq = gconn[j];
        wd += cq;
        np += cq > 0;
        if (q == p) pc = cq;
        if (q == b) bc = cq;
    }
    const unsigned long long r = atomicAdd(lcount, 1ull);
    if ((int64_t)r >= cap) return;
    float f[HP_MLP_IN];
    hp::mlp_features(pc, bc, wd, np, xadj[v + 1] - xadj[v], maxp[b] - (int64_t)pw[b], opt[b],
                     maxp[p] - (int64_t)pw[p], opt[p], finest, f);
    for (int i = 0; i < HP_MLP_IN; i++) lx[r * HP_MLP_IN + i] = f[i];
    lv[r] = v;
    ld[r] = b;
    lacc[r] = 0;
    rec_of[v] = (int32_t)r;
}

__global__ void log_accept_kernel(int32_t n, const int32_t *__restrict__ rec_of, const int8_t *__restrict__ lock,
                                  const unsigned long long *d_ncand, int32_t *__restrict__ lacc)
{
    hp::pdl_wait();
    if (*d_ncand == 0ull) return;
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n && rec_of[v] >= 0) lacc[rec_of[v]] = lock[v];
}

// Label of a record once its level is final: the afterburner accepted the
// move and the vertex ends the level in that destination.
__global__ void log_label_kernel(int64_t r0, int64_t r1, const int32_t *__restrict__ where,
                                 const int32_t *__restrict__ lv, const int32_t *__restrict__ ld,
                                 const int32_t *__restrict__ lacc, float *__restrict__ ly)
{
    hp::pdl_wait();
    int64_t r = r0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r < r1) ly[r] = (lacc[r] && where[lv[r]] == ld[r]) ? 1.f : 0.f;
}

// Where a pass's moves go: the move list and count, the old part per move, and
// the cut-change sum c1 (conn(to) - conn(from) of every move, read from the mover's
// own gain row before any move applies).  The kernels that decide the moves append
// them through move_append and add the c1 terms per block, so no separate pass
// over the moves precedes their application.
struct MoveSink {
    int32_t *moves, *oldp;
    unsigned long long *d_nmoves, *d_c1;
    const int32_t *goff, *gpart, *gconn;
    int32_t k;
};

__device__ __forceinline__ int32_t row_conn(const int32_t *gp, const int32_t *gc, int32_t len, int32_t q,
                                            int32_t k);

// Appends the move of v from p to d; returns its c1 term.
__device__ __forceinline__ long long move_append(const MoveSink &ms, int32_t v, int32_t p, int32_t d)
{
    const unsigned long long i = atomicAdd(ms.d_nmoves, 1ull);
    ms.moves[i] = v;
    ms.oldp[i] = p;
    const int32_t o = ms.goff[v], len = ms.goff[v + 1] - o;
    return (long long)row_conn(ms.gpart + o, ms.gconn + o, len, d, ms.k) -
           row_conn(ms.gpart + o, ms.gconn + o, len, p, ms.k);
}

__device__ __forceinline__ long long ab_change(int32_t v, int32_t g, int32_t p, int32_t b,
                                               int32_t u, int32_t w, const int32_t *pregain,
                                               const int32_t *dest, const int32_t *where)
{
    int32_t gu = pregain[u];
    long long ch = 0;
    if (gu > g || (gu == g && u < v)) {
        int32_t du = dest[u], wu = where[u];
        if (du == p) ch -= w;
        else if (du == b) ch += w;
        if (wu == p) ch += w;
        else if (wu == b) ch -= w;
    }
    return ch;
}

// The plain refiner as the judge of a learned LP pass.  In such a pass the
// selection keeps the plain rule's candidates and marks the ones the MLP dropped
// (prune); the afterburner scores every candidate twice in one walk of its row --
// against the higher-priority plain candidates and against the learned ones only
// -- applies the learned decision (lock, moves) and keeps the plain one in accp.
// The vertices that either decision moves are listed (list, *d_n), and
// judge_off_kernel / judge_delta_kernel add both move sets' exact cut changes
// over their rows.  flag: the control block's learned_pass, so the plain
// refiner's passes (and every pass of a plain run) skip all of it.
struct Judge {
    const int32_t *flag;
    const int8_t *prune;
    int8_t *accp;
    int32_t *list, *d_n;
    const unsigned long long *d_ncandp;   // plain candidates of the pass
};

// ab_change of one entry into the plain sum and, when judging, into the sum
// over the learned candidates (a neighbour the MLP dropped stays put there).
__device__ __forceinline__ void ab_change2(int32_t v, int32_t g, int32_t p, int32_t b, int32_t u, int32_t w,
                                           const int32_t *pregain, const int32_t *dest, const int32_t *where,
                                           const int8_t *prune, bool judge, long long &chp, long long &chl)
{
    const long long c = ab_change(v, g, p, b, u, w, pregain, dest, where);
    chp += c;
    if (judge && c != 0 && !prune[u]) chl += c;
}

// ab_row_sum into both sums (chl only when judging).
__device__ __forceinline__ void ab_row_sum2(int32_t v, int32_t g, int32_t p, int32_t b, int32_t j0, int32_t e,
                                            int32_t stride, const int32_t *__restrict__ adjncy,
                                            const int32_t *__restrict__ adjwgt, const int32_t *pregain,
                                            const int32_t *dest, const int32_t *where, const int8_t *prune,
                                            bool judge, long long &chp, long long &chl)
{
    for (int32_t j = j0; j < e; j += 4 * stride) {
        int32_t u[4], w[4], gu[4], du[4], wu[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int32_t jj = j + q * stride;
            const bool in = jj < e;
            u[q] = in ? adjncy[jj] : v;
            w[q] = in ? adjwgt[jj] : 0;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            gu[q] = pregain[u[q]];
            du[q] = dest[u[q]];
            wu[q] = where[u[q]];
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (u[q] == v) continue;   // no entry (rows have no self loops)
            if (gu[q] > g || (gu[q] == g && u[q] < v)) {
                long long c = 0;
                if (du[q] == p) c -= w[q];
                else if (du[q] == b) c += w[q];
                if (wu[q] == p) c += w[q];
                else if (wu[q] == b) c -= w[q];
                chp += c;
                if (judge && c != 0 && !prune[u[q]]) chl += c;
            }
        }
    }
}

__global__ void __launch_bounds__(256)
afterburner_small_kernel(int32_t n, const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                         const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ where,
                         const int32_t *__restrict__ dest, const int32_t *__restrict__ pregain,
                         int8_t *__restrict__ lock, const unsigned long long *d_ncand, MoveSink ms, int32_t bigd,
                         Judge J)
{
    hp::pdl_wait();
    const bool judge = *J.flag != 0;
    if (*d_ncand == 0ull && !(judge && *J.d_ncandp != 0ull)) return;
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    long long c1 = 0;
    bool listed = false;
    if (v < n) {
        const int32_t b0 = xadj[v], e0 = xadj[v + 1];
        if (e0 - b0 <= bigd) {
            const int32_t g = pregain[v];
            int8_t sel = 0, selp = 0;
            int32_t p = 0, b = 0;
            if (g != NEG) {
                p = where[v];
                b = dest[v];
                long long chp = 0, chl = 0;
                for (int32_t j = b0; j < e0; j++)
                    ab_change2(v, g, p, b, adjncy[j], adjwgt[j], pregain, dest, where, J.prune, judge, chp, chl);
                selp = ((long long)g + chp >= 0);
                sel = judge ? (int8_t)(!J.prune[v] && (long long)g + chl >= 0) : selp;
            }
            lock[v] = sel;
            if (judge) {
                J.accp[v] = selp;
                listed = sel || selp;
            }
            if (sel) c1 = move_append(ms, v, p, b);
        }
    }
    if (judge) {
        const int32_t pos = hp::warp_append(J.d_n, listed);
        if (listed) J.list[pos] = v;
    }
    hp::block_add_to<256>(c1, ms.d_c1);
}

__global__ void __launch_bounds__(256)
afterburner_big_kernel(const int32_t *__restrict__ big, const int32_t *__restrict__ d_bigcnt,
                       const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                       const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ where,
                       const int32_t *__restrict__ dest, const int32_t *__restrict__ pregain,
                       int8_t *__restrict__ lock, const unsigned long long *d_ncand, MoveSink ms,
                       int32_t chunkd, Judge J)
{
    hp::pdl_wait();
    const bool judge = *J.flag != 0;
    if (*d_ncand == 0ull && !(judge && *J.d_ncandp != 0ull)) return;
    const int lane = threadIdx.x & 31;
    const int32_t cnt = *d_bigcnt;
    long long c1 = 0;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < cnt;
         i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int32_t v = big[i];
        if (xadj[v + 1] - xadj[v] > chunkd) continue;   // chunked over the grid
        const int32_t g = pregain[v];
        int8_t sel = 0, selp = 0;
        int32_t p = 0, b = 0;
        if (g != NEG) {
            p = where[v];
            b = dest[v];
            long long chp = 0, chl = 0;
            ab_row_sum2(v, g, p, b, xadj[v] + lane, xadj[v + 1], 32, adjncy, adjwgt, pregain, dest, where, J.prune,
                        judge, chp, chl);
            chp = hp::warp_sum64(chp);
            selp = ((long long)g + chp >= 0);
            if (judge) {
                chl = hp::warp_sum64(chl);
                sel = (int8_t)(!J.prune[v] && (long long)g + chl >= 0);
            } else {
                sel = selp;
            }
        }
        if (lane == 0) {
            lock[v] = sel;
            if (judge) {
                J.accp[v] = selp;
                if (sel || selp) J.list[atomicAdd(J.d_n, 1)] = v;
            }
            if (sel) c1 += move_append(ms, v, p, b);
        }
    }
    hp::block_add_to<256>(c1, ms.d_c1);
}

// ---- long rows (longer than chunk_deg): chunk plans ------------------------------
// The afterburner and move application of rows longer than the tuning's
// chunk_deg are cut into chunks of HUB_CHUNK entries dealt over the whole grid,
// so that no warp walks a long row alone.  A plan per pass selects the rows that
// have work (afterburner: candidates; moves: moved rows) and writes each one's
// vertex, its item (list position or move index) and the exclusive prefix of
// the chunk counts, so that a chunk finds its row by a binary search.  The plan
// is one pass of persistent CTAs over tiles of PLAN_TILE items with two epoch
// look-back chains (selected rows: tile words [0, half); chunks: [half, 2 half)).
constexpr int HUB_CHUNK = 512;
constexpr int PLAN_THREADS = 256, PLAN_ITEMS = 4, PLAN_TILE = PLAN_THREADS * PLAN_ITEMS;

template <bool MOVES>
__global__ void __launch_bounds__(PLAN_THREADS)
hub_plan_kernel(const int32_t *__restrict__ items, const int32_t *__restrict__ d_nitems,
                const int32_t *__restrict__ moves, const int32_t *__restrict__ pregain,
                const int32_t *__restrict__ xadj, int32_t *__restrict__ plan_v, int32_t *__restrict__ plan_item,
                int32_t *__restrict__ plan_off, int32_t *__restrict__ d_plan, unsigned long long *tile_status,
                int64_t half, hp::LbCtl *lb, unsigned *status)
{
    hp::pdl_wait();
    __shared__ int32_t s_scan[PLAN_THREADS / 32 + 2];
    __shared__ int32_t s_excl[2];
    const unsigned epoch = hp::lb_epoch(lb);
    const int32_t ni = *d_nitems;
    for (;;) {
        const int64_t tile = hp::lb_next(lb);
        const int64_t base = tile * PLAN_TILE;
        if (base > ni) break;   // the tile holding index ni (it writes the totals) was the last
        const int64_t t0 = base + (int64_t)threadIdx.x * PLAN_ITEMS;
        int32_t v[PLAN_ITEMS], c[PLAN_ITEMS];
        int32_t ns = 0, nc = 0;
#pragma unroll
        for (int q = 0; q < PLAN_ITEMS; q++) {
            const int64_t t = t0 + q;
            v[q] = -1;
            c[q] = 0;
            if (t < ni) {
                const int32_t vv = MOVES ? moves[items[t]] : items[t];
                if (MOVES || pregain[vv] != NEG) {
                    v[q] = vv;
                    c[q] = (xadj[vv + 1] - xadj[vv] + HUB_CHUNK - 1) / HUB_CHUNK;
                }
            }
            ns += v[q] >= 0;
            nc += c[q];
        }
        int ts, tc;
        int32_t ps = hp::block_excl_scan<PLAN_THREADS>(ns, &ts, s_scan);
        int32_t pc = hp::block_excl_scan<PLAN_THREADS>(nc, &tc, s_scan);
        if (threadIdx.x < 32) {
            const int32_t ex = hp::lookback_epoch(tile_status, tile, ts, epoch, status);
            if (threadIdx.x == 0) s_excl[0] = ex;
        } else if (threadIdx.x < 64) {
            const int32_t ex = hp::lookback_epoch(tile_status + half, tile, tc, epoch, status);
            if (threadIdx.x == 32) s_excl[1] = ex;
        }
        __syncthreads();
        ps += s_excl[0];
        pc += s_excl[1];
#pragma unroll
        for (int q = 0; q < PLAN_ITEMS; q++) {
            if (v[q] >= 0) {
                plan_v[ps] = v[q];
                plan_item[ps] = MOVES ? items[t0 + q] : (int32_t)(t0 + q);
                plan_off[ps] = pc;
                ps++;
            }
            pc += c[q];
        }
        if (ni >= base && ni < base + PLAN_TILE && threadIdx.x == 0) {
            d_plan[0] = s_excl[0] + ts;
            d_plan[1] = s_excl[1] + tc;
        }
    }
    hp::lb_end(lb);
}

// chunk gc -> selected hub j (the last j with plan_off[j] <= gc)
__device__ __forceinline__ int32_t plan_find(const int32_t *__restrict__ plan_off, int32_t nsel, int64_t gc)
{
    int32_t lo = 0, hi = nsel - 1;
    while (lo < hi) {
        const int32_t mid = (lo + hi + 1) >> 1;
        if (plan_off[mid] <= gc) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Afterburner of the candidate hubs: every chunk adds its part of the change to
// the hub's accumulator (ab_acc, indexed by hub-list position, zero on entry;
// ab_acc2 the learned candidates' sum when judging);
// afterburner_huge_final_kernel then decides from the full sums.
__global__ void __launch_bounds__(HUB_CHUNK)
afterburner_huge_kernel(const int32_t *__restrict__ plan_v, const int32_t *__restrict__ plan_item,
                        const int32_t *__restrict__ plan_off, const int32_t *__restrict__ d_plan,
                        const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                        const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ where,
                        const int32_t *__restrict__ dest, const int32_t *__restrict__ pregain,
                        const unsigned long long *d_ncand, unsigned long long *__restrict__ ab_acc,
                        unsigned long long *__restrict__ ab_acc2, Judge J)
{
    hp::pdl_wait();
    const bool judge = *J.flag != 0;
    if (*d_ncand == 0ull && !(judge && *J.d_ncandp != 0ull)) return;
    const int lane = threadIdx.x & 31;
    const int32_t nsel = d_plan[0], nch = d_plan[1];
    for (int64_t gc = blockIdx.x; gc < nch; gc += gridDim.x) {
        const int32_t jp = plan_find(plan_off, nsel, gc);
        const int32_t v = plan_v[jp];
        const int32_t g = pregain[v], p = where[v], b = dest[v];
        const int32_t e0 = xadj[v + 1];
        const int32_t j = xadj[v] + (int32_t)(gc - plan_off[jp]) * HUB_CHUNK + threadIdx.x;
        long long cp = 0, cl = 0;
        if (j < e0) ab_change2(v, g, p, b, adjncy[j], adjwgt[j], pregain, dest, where, J.prune, judge, cp, cl);
        cp = hp::warp_sum64(cp);
        if (judge) cl = hp::warp_sum64(cl);
        if (lane == 0 && cp != 0) atomicAdd(&ab_acc[plan_item[jp]], (unsigned long long)cp);
        if (lane == 0 && cl != 0) atomicAdd(&ab_acc2[plan_item[jp]], (unsigned long long)cl);
    }
}

__global__ void afterburner_huge_final_kernel(const int32_t *__restrict__ huge, const int32_t *__restrict__ d_nhuge,
                                              const int32_t *__restrict__ pregain, const unsigned long long *d_ncand,
                                              unsigned long long *__restrict__ ab_acc,
                                              unsigned long long *__restrict__ ab_acc2, int8_t *__restrict__ lock,
                                              const int32_t *__restrict__ where, const int32_t *__restrict__ dest,
                                              MoveSink ms, Judge J)
{
    hp::pdl_wait();
    const bool judge = *J.flag != 0;
    if (*d_ncand == 0ull && !(judge && *J.d_ncandp != 0ull)) return;
    const int32_t nh = *d_nhuge;
    long long c1 = 0;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x) {
        const int32_t v = huge[i];
        const int32_t g = pregain[v];
        const long long totp = (long long)ab_acc[i];
        ab_acc[i] = 0ull;
        const int8_t selp = (g != NEG) && ((long long)g + totp >= 0);
        int8_t sel = selp;
        if (judge) {
            const long long totl = (long long)ab_acc2[i];
            ab_acc2[i] = 0ull;
            sel = (g != NEG) && !J.prune[v] && ((long long)g + totl >= 0);
            J.accp[v] = selp;
            if (sel || selp) J.list[atomicAdd(J.d_n, 1)] = v;
        }
        lock[v] = sel;
        if (sel) c1 += move_append(ms, v, where[v], dest[v]);
    }
    hp::block_add_to<256>(c1, ms.d_c1);
}

// ---- the judge's exact cut changes ---------------------------------------------------
// Over the listed vertices' entries (tiles of JD_TILE, owner rows from the
// prefix): twice the exact cut decrease of the plain move set (accp) into
// sums[0] and of the learned one (lock) into sums[1].  An entry (v, u, w) of a
// moved v counts w ([p_v != p_u] - [d_v != new p_u]), twice when u stays put
// and once when u moves too (then its row counts the edge again).
constexpr int JD_THREADS = 256, JD_ITEMS = 8, JD_TILE = JD_THREADS * JD_ITEMS;

// One entry (v, u, w) of a listed vertex v (part pv, destination dv; apv / alv:
// v moves in the plain / learned set) into the two sums.
__device__ __forceinline__ void judge_entry(int32_t pv, int32_t dv, bool apv, bool alv, int32_t u, int32_t w,
                                            const int32_t *where, const int32_t *dest, const int8_t *accp,
                                            const int8_t *lock, long long &sp, long long &sl)
{
    const int32_t pu = where[u];
    const bool apu = accp[u] != 0, alu = lock[u] != 0;
    const int32_t du = (apu || alu) ? dest[u] : pu;
    const long long before = pv != pu;
    if (apv) sp += (long long)w * (before - (dv != (apu ? du : pu))) * (apu ? 1 : 2);
    if (alv) sl += (long long)w * (before - (dv != (alu ? du : pu))) * (alu ? 1 : 2);
}

__global__ void __launch_bounds__(JD_THREADS)
judge_delta_kernel(const int32_t *flag, const int32_t *__restrict__ list, const int32_t *d_n,
                   const int32_t *__restrict__ off, const int32_t *__restrict__ xadj,
                   const int32_t *__restrict__ adjncy, const int32_t *__restrict__ adjwgt,
                   const int32_t *__restrict__ where, const int32_t *__restrict__ dest,
                   const int8_t *__restrict__ accp, const int8_t *__restrict__ lock, unsigned long long *sums)
{
    hp::pdl_wait();
    __shared__ int32_t owner[JD_TILE];
    __shared__ int32_t s_warp[JD_THREADS / 32];
    __shared__ int32_t s_v0;
    if (*flag == 0) return;
    const int32_t cnt = *d_n;
    if (cnt <= 0) return;
    const int64_t tot = off[cnt];
    long long sp = 0, sl = 0;
    for (int64_t tb = (int64_t)blockIdx.x * JD_TILE; tb < tot; tb += (int64_t)gridDim.x * JD_TILE) {
        const int64_t te = tb + JD_TILE < tot ? tb + JD_TILE : tot;
        hp::tile_owners<JD_THREADS, JD_ITEMS>(off, cnt, tb, te, owner, s_warp, &s_v0);
        for (int64_t t = tb + threadIdx.x; t < te; t += JD_THREADS) {
            const int32_t i = owner[t - tb];
            const int32_t v = list[i];
            const int32_t j = xadj[v] + (int32_t)(t - off[i]);
            judge_entry(where[v], dest[v], accp[v] != 0, lock[v] != 0, adjncy[j], adjwgt[j], where, dest, accp, lock,
                        sp, sl);
        }
        __syncthreads();   // owner[] is rebuilt for the next tile
    }
    hp::block_add_to<JD_THREADS>(sp, &sums[0]);
    hp::block_add_to<JD_THREADS>(sl, &sums[1]);
}

// ---- applying moves -------------------------------------------------------------
// Effect of one move on its neighbours' gain rows.  A vertex's own row does
// not depend on its own part: only neighbours' rows change.  Dense neighbour
// rows (deg >= k) take the change in place; a sparse neighbour is queued once
// (atomicExch on its dirty flag) on the small or big rebuild list.
// o and cap: the neighbour's gain-row offset and capacity (goff[u], goff[u+1] - o),
// loaded by the caller.
__device__ __forceinline__ void touch_neighbour(bool valid, int32_t u, int32_t w, int32_t o, int32_t cap, int32_t p,
                                                int32_t d, const int32_t *__restrict__ xadj,
                                                int32_t *__restrict__ gconn, int32_t *__restrict__ dirty,
                                                int32_t *__restrict__ small_l, int32_t *__restrict__ big_l,
                                                int32_t *counts, int32_t k, int32_t bigd)
{
    // all 32 lanes call (valid marks the lanes with a neighbour); list appends
    // take one counter atomic per warp and list (ballot ranks inside the warp)
    bool sm = false, bg = false;
    if (valid) {
        if (cap == k) {
            atomicAdd(&gconn[o + p], -w);
            atomicAdd(&gconn[o + d], w);
        } else if (__ldcg(&dirty[u]) == 0 && atomicExch(&dirty[u], 1) == 0) {
            // (a row already queued in this pass is skipped without an atomic;
            // flags only go from 0 to 1 inside the kernel)
            if (xadj[u + 1] - xadj[u] > bigd) bg = true;
            else sm = true;
        }
    }
    const unsigned lt = hp::lanemask_lt();
    const unsigned ms = __ballot_sync(HP_FULL_MASK, sm), mb = __ballot_sync(HP_FULL_MASK, bg);
    const int lane = threadIdx.x & 31;
    int32_t bs = 0, bb = 0;
    if (lane == 0) {
        if (ms) bs = atomicAdd(&counts[0], __popc(ms));
        if (mb) bb = atomicAdd(&counts[1], __popc(mb));
    }
    bs = __shfl_sync(HP_FULL_MASK, bs, 0);
    bb = __shfl_sync(HP_FULL_MASK, bb, 0);
    if (sm) small_l[bs + __popc(ms & lt)] = u;
    if (bg) big_l[bb + __popc(mb & lt)] = u;
}

// One warp per move (warp, nwarps: this warp among those sharing the moves).
__device__ __forceinline__ void apply_moves_rows(int64_t warp, int64_t nwarps, const int32_t *__restrict__ moves,
                                                 int64_t nm, int32_t *__restrict__ where,
                                                 const int32_t *__restrict__ dest, const int32_t *__restrict__ vwgt,
                                                 unsigned long long *__restrict__ pw, const int32_t *__restrict__ xadj,
                                                 const int32_t *__restrict__ adjncy,
                                                 const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ goff,
                                                 int32_t *__restrict__ gconn, int32_t *__restrict__ dirty,
                                                 int32_t *__restrict__ small_l, int32_t *__restrict__ big_l,
                                                 int32_t *counts, int32_t k, int32_t *__restrict__ huge_mv,
                                                 int32_t *__restrict__ d_nhuge, int32_t bigd, int32_t chunkd)
{
    const int lane = threadIdx.x & 31;
    for (int64_t i = warp; i < nm; i += nwarps) {
        const int32_t v = moves[i];
        const int32_t p = where[v], d = dest[v];
        __syncwarp();
        if (lane == 0) {
            const unsigned long long w = (unsigned long long)vwgt[v];
            atomicAdd(&pw[d], w);
            atomicAdd(&pw[p], (unsigned long long)(-(long long)w));
        }
        const int32_t b = xadj[v], e = xadj[v + 1];
        if (e - b > chunkd) {
            // neighbours of a hub are touched by apply_moves_huge_kernel, spread
            // over the whole grid (it reads the old part from oldp)
            if (lane == 0) {
                huge_mv[atomicAdd(d_nhuge, 1)] = (int32_t)i;
                where[v] = d;
            }
            continue;
        }
        // four chunks of 32 entries at a time: row loads, then the neighbours'
        // gain-row offsets, are in flight together
        for (int32_t j0 = b; j0 < e; j0 += 128) {
            int32_t u[4], w[4], o[4], cap[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int32_t j = j0 + 32 * q + lane;
                const bool valid = j < e;
                u[q] = valid ? adjncy[j] : -1;
                w[q] = valid ? adjwgt[j] : 0;
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                o[q] = u[q] >= 0 ? goff[u[q]] : 0;
                cap[q] = u[q] >= 0 ? goff[u[q] + 1] - o[q] : 0;
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
                touch_neighbour(u[q] >= 0, u[q], w[q], o[q], cap[q], p, d, xadj, gconn, dirty, small_l, big_l, counts,
                                k, bigd);
        }
        if (lane == 0) where[v] = d;   // the move itself (every lane has read where[v])
    }
}

__global__ void __launch_bounds__(256)
apply_moves_kernel(const int32_t *__restrict__ moves, const unsigned long long *d_nmoves,
                   int32_t *__restrict__ where, const int32_t *__restrict__ dest,
                   const int32_t *__restrict__ vwgt, unsigned long long *__restrict__ pw,
                   const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                   const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ goff,
                   int32_t *__restrict__ gconn, int32_t *__restrict__ dirty, int32_t *__restrict__ small_l,
                   int32_t *__restrict__ big_l, int32_t *counts, int32_t k, int32_t *__restrict__ huge_mv,
                   int32_t *__restrict__ d_nhuge, int32_t bigd, int32_t chunkd)
{
    hp::pdl_wait();
    apply_moves_rows((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5, ((int64_t)gridDim.x * blockDim.x) >> 5,
                     moves, (int64_t)*d_nmoves, where, dest, vwgt, pw, xadj, adjncy, adjwgt, goff, gconn, dirty,
                     small_l, big_l, counts, k, huge_mv, d_nhuge, bigd, chunkd);
}

// Neighbours of the moved hubs (queued by apply_moves_kernel, planned by
// hub_plan_kernel<true>): chunks of HUB_CHUNK entries over the whole grid.  A
// hub's old part comes from oldp (the hub itself is already committed).
__global__ void __launch_bounds__(HUB_CHUNK)
apply_moves_huge_kernel(const int32_t *__restrict__ plan_v, const int32_t *__restrict__ plan_item,
                        const int32_t *__restrict__ plan_off, const int32_t *__restrict__ d_plan,
                        const int32_t *__restrict__ oldp, const int32_t *__restrict__ dest,
                        const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                        const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ goff,
                        int32_t *__restrict__ gconn, int32_t *__restrict__ dirty, int32_t *__restrict__ small_l,
                        int32_t *__restrict__ big_l, int32_t *counts, int32_t k, int32_t bigd)
{
    hp::pdl_wait();
    const int32_t nsel = d_plan[0], nch = d_plan[1];
    for (int64_t gc = blockIdx.x; gc < nch; gc += gridDim.x) {
        const int32_t jp = plan_find(plan_off, nsel, gc);
        const int32_t v = plan_v[jp];
        const int32_t p = oldp[plan_item[jp]], d = dest[v];
        const int32_t e = xadj[v + 1];
        const int32_t j = xadj[v] + (int32_t)(gc - plan_off[jp]) * HUB_CHUNK + threadIdx.x;
        const bool valid = j < e;
        const int32_t u = valid ? adjncy[j] : 0;
        const int32_t o = valid ? goff[u] : 0, cap = valid ? goff[u + 1] - o : 0;
        touch_neighbour(valid, u, valid ? adjwgt[j] : 0, o, cap, p, d, xadj, gconn, dirty, small_l, big_l, counts, k,
                        bigd);
    }
}

// ---- rebalancing ------------------------------------------------------------------
// Undersized parts (pw < max(0.99 maxp, maxp - 100)) in part order; one CTA.
__device__ __forceinline__ void undersized_block(int32_t k, const unsigned long long *__restrict__ pw,
                                                 const int64_t *__restrict__ maxp, int32_t *__restrict__ und,
                                                 int32_t *d_nu, int32_t *s_scan /* 1024/32 + 2 */)
{
    int running = 0;
    for (int base = 0; base < k; base += 1024) {
        int p = base + threadIdx.x;
        int f = 0;
        if (p < k) {
            int64_t md = (maxp[p] * 99) / 100;
            if (md < maxp[p] - 100) md = maxp[p] - 100;
            f = (int64_t)pw[p] < md;
        }
        int tot;
        int pos = running + hp::block_excl_scan<1024>(f, &tot, s_scan);
        if (f) und[pos] = p;
        running += tot;
    }
    if (threadIdx.x == 0) *d_nu = running;
}

// Rebalance candidates of a pass in one ordered pass over the vertices, tiles
// of RB_TILE in launch order with an epoch look-back: the key (part * 64 + gain
// bucket) of every candidate, compacted in vertex order into K/V, the count
// into *d_cnt, and dest[v] for every vertex (the proposed part, or its own).
//   weak  (jetrw, hunyuangraph_GPU_krefine.h:3381-3563): v in an overweight part
//         with 2 vwgt < 3 (pw - opt); destination = most connected part that
//         is not overweight (first max in part order), else an undersized part
//         (und[v % nu]); gain = conn(dest) - conn(own)
//   strong (jetrs, :2774-3135): v in an overweight part with vwgt < 2 (pw - opt);
//         loss = -conn(own)
// The part bounds pstart/pend are reset to -1 here for the rank kernel.
constexpr int RB_TILE = 256;
constexpr int RB_COOP = 32;   // weak rebalance: longer gain rows are walked by a warp

template <bool STRONG>
__global__ void __launch_bounds__(RB_TILE)
rb_candidates_kernel(int32_t n, const int32_t *__restrict__ where, const int32_t *__restrict__ vwgt,
                     const unsigned long long *__restrict__ pw, const int64_t *__restrict__ maxp,
                     const int64_t *__restrict__ opt, const int32_t *__restrict__ goff,
                     const int32_t *__restrict__ gpart, const int32_t *__restrict__ gconn,
                     const int32_t *__restrict__ und, const int32_t *__restrict__ d_nu, int32_t k,
                     int32_t *__restrict__ K, int32_t *__restrict__ V, int32_t *__restrict__ dest,
                     int32_t *__restrict__ d_cnt, int32_t *__restrict__ pstart, int32_t *__restrict__ pend,
                     unsigned long long *tile_status, hp::LbCtl *lb, unsigned *status,
                     const int8_t *__restrict__ ufl, BestCopy bcp)
{
    hp::pdl_wait();
    __shared__ int32_t s_scan[RB_TILE / 32 + 2];
    __shared__ int32_t s_excl;
    __shared__ CoopRows<RB_TILE> S;
    int64_t tile;
    unsigned epoch;
    hp::lb_begin(lb, &tile, &epoch);
    for (int64_t q = tile * RB_TILE + threadIdx.x; q < k; q += (int64_t)gridDim.x * RB_TILE) {
        pstart[q] = -1;
        pend[q] = -1;
    }
    const int64_t v64 = tile * RB_TILE + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int32_t kk = -1;
    const bool in = v64 < n;
    const int32_t v = in ? (int32_t)v64 : 0;
    int32_t p = 0;
    bool cand = false;   // in an overweight part and light enough to leave it
    const bool copy = bcp.on();
    if (copy && tile == 0) bcp.parts();
    if (in) {
        p = where[v];
        if (copy) bcp.best_where[v] = p;
        const int64_t pwp = (int64_t)pw[p];
        cand = STRONG ? (pwp > maxp[p] && (int64_t)vwgt[v] < 2 * (pwp - opt[p]))
                      : (pwp > maxp[p] && 2 * (int64_t)vwgt[v] < 3 * (pwp - opt[p]));
    }
    const int32_t o = cand ? goff[v] : 0, len = cand ? goff[v + 1] - o : 0;
    int32_t d = p;
    if (!STRONG) {
        // best underweight part by connectivity (first, i.e. lowest part, among
        // equals) and the connectivity to the own part; rows of more than
        // RB_COOP entries are walked by a whole warp, any warp of the CTA
        int64_t pc = 0, bc = 0;
        int32_t b = -1;
        const bool coop = cand && len > RB_COOP;
        if (cand && !coop) {
            for (int32_t j = o; j < o + len; j++) {
                const int32_t q = gpart[j];
                if (q < 0) break;
                const int32_t cq = gconn[j];
                if (q == p) pc = cq;
                if (ufl[q] && cq > bc) { bc = cq; b = q; }
            }
        }
        // the CTA's long rows, shared by all its warps
        const int my = coop_queue<RB_TILE>(S, coop, o, len, p);
        const int nc = S.n;
        for (int i = threadIdx.x >> 5; i < nc; i += RB_TILE / 32) {
            const int32_t so = S.o[i], sl = S.len[i], sp = S.p[i];
            int32_t lpc = 0, lbc = 0, lb = -1;
            const bool dense = sl == k;   // entry j is part j
            for (int32_t j = lane; j < sl; j += 32) {
                const int32_t q = dense ? j : gpart[so + j];
                if (q < 0) break;   // padding runs to the end of the row
                const int32_t cq = gconn[so + j];
                if (q == sp) lpc = cq;
                if (ufl[q] && cq > lbc) { lbc = cq; lb = q; }
            }
            lpc = hp::warp_sum(lpc);
#pragma unroll
            for (int sh = 16; sh > 0; sh >>= 1) {
                const int32_t ob = __shfl_xor_sync(HP_FULL_MASK, lb, sh);
                const int32_t oc = __shfl_xor_sync(HP_FULL_MASK, lbc, sh);
                if (ob >= 0 && (lb < 0 || oc > lbc || (oc == lbc && ob < lb))) { lb = ob; lbc = oc; }
            }
            if (lane == 0) { S.pc[i] = lpc; S.bc[i] = lbc; S.b[i] = lb; }
        }
        __syncthreads();
        if (my >= 0) { pc = S.pc[my]; bc = S.bc[my]; b = S.b[my]; }
        if (cand) {
            int64_t g = 0;
            bool ok = true;
            if (b >= 0) g = bc - pc;
            else {
                const int32_t nu = *d_nu;
                if (nu == 0) ok = false;
                else { b = und[v % nu]; g = -pc; }
            }
            if (ok) { d = b; kk = p * 64 + hp::gain_bucket((int32_t)g, vwgt[v]); }
        }
    } else if (cand) {
        const int32_t pc = row_conn(gpart + o, gconn + o, len, p, k);
        kk = p * 64 + hp::gain_bucket(-pc, vwgt[v]);
    }
    if (in) dest[v] = d;
    int tot;
    const int local = hp::block_excl_scan<RB_TILE>(kk >= 0 ? 1 : 0, &tot, s_scan);
    if (threadIdx.x < 32) {
        const int32_t ex = hp::lookback_epoch(tile_status, tile, tot, epoch, status);
        if (threadIdx.x == 0) s_excl = ex;
    }
    __syncthreads();
    if (kk >= 0) {
        const int32_t pos = s_excl + local;
        K[pos] = kk;
        V[pos] = (int32_t)v64;
    }
    if (tile == gridDim.x - 1 && threadIdx.x == 0) *d_cnt = s_excl + tot;
    hp::lb_end(lb);
}

// Over the sorted candidates: pre[i] = weight of the candidates before i in
// the sorted order (pre[cnt] = total), and the part bounds pstart/pend (first
// index, one past the last) from the sorted keys.  Tiles of RK_TILE items in
// launch order with an epoch look-back, taken by a fixed grid of persistent
// CTAs until the tile holding index cnt, so the work follows the count on
// the device, not n.
constexpr int RK_THREADS = 256, RK_ITEMS = 4, RK_TILE = RK_THREADS * RK_ITEMS;

__global__ void __launch_bounds__(RK_THREADS)
rb_rank_kernel(const int32_t *__restrict__ K, const int32_t *__restrict__ V, const int32_t *__restrict__ d_cnt,
               const int32_t *__restrict__ vwgt, int32_t *__restrict__ pre, int32_t *__restrict__ pstart,
               int32_t *__restrict__ pend, unsigned long long *tile_status, hp::LbCtl *lb, unsigned *status)
{
    hp::pdl_wait();
    __shared__ int32_t s_scan[RK_THREADS / 32 + 2];
    __shared__ int32_t s_excl;
    const unsigned epoch = hp::lb_epoch(lb);
    const int32_t cnt = *d_cnt;
    for (;;) {
        const int64_t tile = hp::lb_next(lb);
        const int64_t base = tile * RK_TILE;
        if (base > cnt) break;   // the tile holding index cnt was the last one
        const int64_t i0 = base + (int64_t)threadIdx.x * RK_ITEMS;
        int32_t w[RK_ITEMS];
        int32_t sum = 0;
#pragma unroll
        for (int q = 0; q < RK_ITEMS; q++) {
            w[q] = i0 + q < cnt ? vwgt[V[i0 + q]] : 0;
            sum += w[q];
        }
        int tot;
        int32_t run = hp::block_excl_scan<RK_THREADS>(sum, &tot, s_scan);
        if (threadIdx.x < 32) {
            const int32_t ex = hp::lookback_epoch(tile_status, tile, tot, epoch, status);
            if (threadIdx.x == 0) s_excl = ex;
        }
        __syncthreads();
        run += s_excl;
#pragma unroll
        for (int q = 0; q < RK_ITEMS; q++) {
            const int64_t i = i0 + q;
            if (i <= cnt) pre[i] = run;
            run += w[q];
            if (i < cnt) {
                const int32_t p = K[i] >> 6;
                if (i == 0 || (K[i - 1] >> 6) != p) pstart[p] = (int32_t)i;
                if (i == cnt - 1 || (K[i + 1] >> 6) != p) pend[p] = (int32_t)i + 1;
            }
        }
    }
    hp::lb_end(lb);
}

// The judge's list: exclusive prefix of the row lengths of the listed vertices
// (off[i]; off[cnt] = all their entries), in tiles of RK_TILE with an epoch
// look-back, by persistent CTAs until the tile holding index cnt.
__global__ void __launch_bounds__(RK_THREADS)
judge_off_kernel(const int32_t *flag, const int32_t *__restrict__ list, const int32_t *d_n,
                 const int32_t *__restrict__ xadj, int32_t *__restrict__ off, unsigned long long *tile_status,
                 hp::LbCtl *lb, unsigned *status)
{
    hp::pdl_wait();
    __shared__ int32_t s_scan[RK_THREADS / 32 + 2];
    __shared__ int32_t s_excl;
    const unsigned epoch = hp::lb_epoch(lb);
    const int32_t cnt = *flag != 0 ? *d_n : -1;   // -1: not judging, no tile
    for (;;) {
        const int64_t tile = hp::lb_next(lb);
        const int64_t base = tile * RK_TILE;
        if (base > cnt) break;   // the tile holding index cnt was the last one
        const int64_t i0 = base + (int64_t)threadIdx.x * RK_ITEMS;
        int32_t d[RK_ITEMS];
        int32_t sum = 0;
#pragma unroll
        for (int q = 0; q < RK_ITEMS; q++) {
            const int64_t i = i0 + q;
            d[q] = 0;
            if (i < cnt) {
                const int32_t v = list[i];
                d[q] = xadj[v + 1] - xadj[v];
            }
            sum += d[q];
        }
        int tot;
        int32_t run = hp::block_excl_scan<RK_THREADS>(sum, &tot, s_scan);
        if (threadIdx.x < 32) {
            const int32_t ex = hp::lookback_epoch(tile_status, tile, tot, epoch, status);
            if (threadIdx.x == 0) s_excl = ex;
        }
        __syncthreads();
        run += s_excl;
#pragma unroll
        for (int q = 0; q < RK_ITEMS; q++) {
            if (i0 + q <= cnt) off[i0 + q] = run;
            run += d[q];
        }
    }
    hp::lb_end(lb);
}

__global__ void rw_select_kernel(const int32_t *__restrict__ K, const int32_t *__restrict__ V,
                                 const int32_t *__restrict__ d_cnt, const int32_t *__restrict__ pre,
                                 const int32_t *__restrict__ pstart,
                                 const unsigned long long *__restrict__ pw,
                                 const int64_t *__restrict__ maxp, const int32_t *__restrict__ dest, MoveSink ms)
{
    hp::pdl_wait();
    const int32_t cnt = *d_cnt;
    long long c1 = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt;
         i += (int64_t)gridDim.x * blockDim.x) {
        int32_t p = K[i] >> 6;
        int64_t before = (int64_t)pre[i] - pre[pstart[p]];
        if (before < (int64_t)pw[p] - maxp[p]) {
            const int32_t v = V[i];
            c1 += move_append(ms, v, p, dest[v]);
        }
    }
    hp::block_add_to<256>(c1, ms.d_c1);
}

// Evicted prefix of every overweight part: smallest e in (s, end] with
// pre[e] - pre[s] >= excess, else end.
__global__ void evict_end_kernel(int32_t k, const int32_t *__restrict__ pstart,
                                 const int32_t *__restrict__ pend, const int32_t *__restrict__ pre,
                                 const unsigned long long *__restrict__ pw,
                                 const int64_t *__restrict__ maxp, int32_t *__restrict__ ev_end)
{
    hp::pdl_wait();
    int32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= k) return;
    int32_t s = pstart[p], e = pend[p];
    if (s < 0) { ev_end[p] = -1; return; }
    const int64_t need = (int64_t)pw[p] - maxp[p];
    int32_t lo = s, hi = e;
    while (lo + 1 < hi) {
        int32_t mid = (lo + hi) / 2;
        if ((int64_t)pre[mid] - pre[s] >= need) hi = mid; else lo = mid;
    }
    ev_end[p] = hi;
}

// Strong rebalance: the evicted prefix of every overweight part (sorted index
// i < ev_end[part]) compacted in sorted order -- P[j] = i and sp[j] = weight of
// the evicted candidates before j (sp[np] = total), *d_np = np -- in one pass
// with two epoch look-back chains (count: tile words [0, half); weight: words
// [half, 2 half)); persistent CTAs as in rb_rank_kernel.
__global__ void __launch_bounds__(RK_THREADS)
rs_evict_kernel(const int32_t *__restrict__ K, const int32_t *__restrict__ V, const int32_t *__restrict__ d_cnt,
                const int32_t *__restrict__ ev_end, const int32_t *__restrict__ vwgt, int32_t *__restrict__ P,
                int32_t *__restrict__ sp, int32_t *__restrict__ d_np, unsigned long long *tile_status,
                int64_t half, hp::LbCtl *lb, unsigned *status)
{
    hp::pdl_wait();
    __shared__ int32_t s_scan[RK_THREADS / 32 + 2];
    __shared__ int32_t s_excl[2];
    const unsigned epoch = hp::lb_epoch(lb);
    const int32_t cnt = *d_cnt;
    for (;;) {
        const int64_t tile = hp::lb_next(lb);
        const int64_t base = tile * RK_TILE;
        if (base > cnt) break;   // the tile holding index cnt was the last one
        const int64_t i0 = base + (int64_t)threadIdx.x * RK_ITEMS;
        int32_t w[RK_ITEMS];
        bool f[RK_ITEMS];
        int32_t nf = 0, sw = 0;
#pragma unroll
        for (int q = 0; q < RK_ITEMS; q++) {
            const int64_t i = i0 + q;
            f[q] = i < cnt && i < ev_end[K[i] >> 6];
            w[q] = f[q] ? vwgt[V[i]] : 0;
            nf += f[q];
            sw += w[q];
        }
        int tc, tw;
        int32_t pos = hp::block_excl_scan<RK_THREADS>(nf, &tc, s_scan);
        int32_t run = hp::block_excl_scan<RK_THREADS>(sw, &tw, s_scan);
        if (threadIdx.x < 32) {
            const int32_t ex = hp::lookback_epoch(tile_status, tile, tc, epoch, status);
            if (threadIdx.x == 0) s_excl[0] = ex;
        } else if (threadIdx.x < 64) {
            const int32_t ex = hp::lookback_epoch(tile_status + half, tile, tw, epoch, status);
            if (threadIdx.x == 32) s_excl[1] = ex;
        }
        __syncthreads();
        pos += s_excl[0];
        run += s_excl[1];
#pragma unroll
        for (int q = 0; q < RK_ITEMS; q++) {
            if (f[q]) {
                P[pos] = (int32_t)(i0 + q);
                sp[pos] = run;
                pos++;
            }
            run += w[q];
        }
        if (cnt >= base && cnt < base + RK_TILE && threadIdx.x == 0) {
            *d_np = s_excl[0] + tc;
            sp[s_excl[0] + tc] = s_excl[1] + tw;
        }
    }
    hp::lb_end(lb);
}

// Sequential cookie cutter over the parts (one warp), as in the reference
// (hunyuangraph_GPU_krefine.h:3075): part p takes the evicted range starting
// at the previous end whose weight is closest to its room maxp[p] - pw[p].
// Rooms are read 32 parts at a time; a part without room keeps an empty range
// (the rule gives end = start there); otherwise the end is searched first among
// the 32 entries after the start (one coalesced read), then 32-ary over the rest.
// Once the start reaches np the remaining parts all get the empty range [np, np).
// The whole CTA first stages sp[0..np] in shared memory when it fits
// (COOKIE_SMEM_INTS entries), then warp 0 walks the parts; every search then
// waits on shared memory instead of L2.
constexpr int COOKIE_SMEM_INTS = 50 * 1024;

__device__ void cookie_cut_warp(int32_t k, const unsigned long long *__restrict__ pw,
                                const int64_t *__restrict__ maxp, const int32_t *sp, int32_t np,
                                int32_t *__restrict__ es, int32_t *__restrict__ ee);

__global__ void __launch_bounds__(1024)
cookie_cutter_kernel(int32_t k, const unsigned long long *__restrict__ pw, const int64_t *__restrict__ maxp,
                     const int32_t *__restrict__ sp_g, const int32_t *__restrict__ d_np, int32_t *__restrict__ es,
                     int32_t *__restrict__ ee)
{
    hp::pdl_wait();
    extern __shared__ int32_t sp_s[];
    const int32_t np = *d_np;
    const bool staged = np + 1 <= COOKIE_SMEM_INTS;
    if (staged)
        for (int32_t i = threadIdx.x; i <= np; i += blockDim.x) sp_s[i] = sp_g[i];
    __syncthreads();
    if (threadIdx.x >= 32) return;
    cookie_cut_warp(k, pw, maxp, staged ? sp_s : sp_g, np, es, ee);
}

// The walk itself, by one full warp.
__device__ void cookie_cut_warp(int32_t k, const unsigned long long *__restrict__ pw,
                                const int64_t *__restrict__ maxp, const int32_t *sp, int32_t np,
                                int32_t *__restrict__ es, int32_t *__restrict__ ee)
{
    const int lane = threadIdx.x & 31;
    int32_t st = 0;
    for (int32_t p0 = 0; p0 < k; p0 += 32) {
        const int32_t pl = p0 + lane;
        const int64_t my_room = pl < k && maxp[pl] > (int64_t)pw[pl] ? maxp[pl] - (int64_t)pw[pl] : 0;
        const int cnt = min(32, k - p0);
        for (int q = 0; q < cnt; q++) {
            const int64_t room = __shfl_sync(HP_FULL_MASK, my_room, q);
            const int32_t p = p0 + q;
            const int32_t lo0 = st;
            int32_t end = lo0;
            if (room > 0) {
                const int32_t hi0 = np;
                const int64_t find = (int64_t)sp[lo0] + room;
                // first idx in (lo0, hi0] with sp[idx] >= find, else hi0
                int32_t lo = lo0, hi = hi0, e = hi0;
                bool found = false;
                {
                    const int32_t pos = lo0 + 1 + lane;
                    const bool ge = pos <= hi0 && (int64_t)sp[pos] >= find;
                    const unsigned m = __ballot_sync(HP_FULL_MASK, ge);
                    if (m) { e = lo0 + 1 + (__ffs(m) - 1); found = true; }
                    else if (lo0 + 32 >= hi0) { e = hi0; found = true; }
                    else lo = lo0 + 32;   // sp[lo0+32] < find: the answer lies in (lo0+32, hi0]
                }
                if (!found) {
                    while (hi - lo > 32) {
                        int64_t span = hi - lo;
                        int32_t pos = lo + (int32_t)((span * (lane + 1)) / 32);
                        bool ge = (int64_t)sp[pos] >= find;
                        unsigned m = __ballot_sync(HP_FULL_MASK, ge);
                        if (m == 0) { lo = __shfl_sync(HP_FULL_MASK, pos, 31); break; }
                        int f = __ffs(m) - 1;
                        int32_t nhi = __shfl_sync(HP_FULL_MASK, pos, f);
                        int32_t nlo = f == 0 ? lo : __shfl_sync(HP_FULL_MASK, pos, f - 1);
                        lo = nlo; hi = nhi;
                    }
                    e = hi;
                    if (lo < hi) {
                        int32_t pos = lo + 1 + lane;
                        bool ge = pos <= hi && (int64_t)sp[pos] >= find;
                        unsigned m = __ballot_sync(HP_FULL_MASK, ge);
                        e = m ? lo + 1 + (__ffs(m) - 1) : hi;
                    }
                }
                int32_t s0 = e > lo0 ? e - 1 : lo0;
                int64_t dh = hp::iabs64((int64_t)sp[e] - find), dl = hp::iabs64((int64_t)sp[s0] - find);
                end = dh < dl ? e : s0;
            }
            if (lane == 0) { es[p] = lo0; ee[p] = end; }
            st = end;
            if (st == np) {
                // the evicted list is used up: every later part starts at np and,
                // room or not, ends there (nothing lies beyond np), so the rest is
                // written in parallel
                for (int32_t r = p + 1 + lane; r < k; r += 32) { es[r] = np; ee[r] = np; }
                return;
            }
        }
    }
}

__global__ void rs_assign_kernel(int32_t k, const int32_t *__restrict__ P, const int32_t *__restrict__ d_np,
                                 const int32_t *__restrict__ V, const int32_t *__restrict__ es,
                                 const int32_t *__restrict__ ee, const int32_t *__restrict__ where,
                                 int32_t *__restrict__ dest, MoveSink ms)
{
    hp::pdl_wait();
    const int32_t np = *d_np;
    long long c1 = 0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < np;
         j += (int64_t)gridDim.x * blockDim.x) {
        // last part with es[p] <= j
        int32_t lo = 0, hi = k - 1;
        while (lo < hi) {
            int32_t mid = (lo + hi + 1) / 2;
            if (es[mid] <= j) lo = mid; else hi = mid - 1;
        }
        const int32_t p = lo;
        const int32_t v = V[P[j]];
        const int32_t from = where[v];
        if (j < ee[p] && p != from) {
            dest[v] = p;
            c1 += move_append(ms, v, from, p);
        }
    }
    hp::block_add_to<256>(c1, ms.d_c1);
}


// ---------------------------------------------------------------------------------
struct RefineBufs {
    int32_t *goff, *gpart, *gconn, *big, *dest, *pregain, *moves, *oldp, *dirty;
    int32_t *small_l, *big_l, *best_where, *huge_mv, *huge;
    int32_t *hub;     // rows longer than gain_hub_deg (the dense gain build's rows when k <= warp_dense_k)
    int32_t *recof;   // move log: a vertex's record (record mode)
    int32_t *plan_v, *plan_item, *plan_off, *plan_cnt;   // chunk plan of the current step
    int64_t nhub_cap;   // capacity of the long-row list and the plan (rows longer than chunk_deg)
    unsigned long long *ab_acc;   // afterburner sums of the hub rows (zero between passes)
    int8_t *lock;
    int8_t *prune, *accp;                  // the judge of a learned pass (Judge)
    int32_t *jlist, *joff;                 // its listed vertices and their row prefix
    unsigned long long *ab_acc2;           // learned-candidate sums of the hub rows
    int32_t *K, *V, *K2, *V2, *pre, *P, *sp;
    int32_t *pstart, *pend, *und, *ev_end, *es, *ee;
    int8_t *ufl;   // per part: pw < maxp (a weak pass's destination rule), set by ctl_begin
    unsigned long long *pw;
    const int64_t *opt, *maxp;
    int32_t small_max;  // longest row of at most bigd entries (picks the gain kernel's network)
    bool huge_rows;     // the level has rows longer than huged
};

// scalar slots used by refinement
// Slots below S_PASS_END are reset at the start of every pass (S_NCANDP .. S_JL:
// the judge of a learned pass -- plain candidates, listed vertices, twice the
// plain and the learned exact cut decrease); S_BIGCNT (the
// level's list of rows longer than 32) lives above it and persists.
// S_BIGCNT (slots 16-18) holds the big-row count, the longest short row, the
// longest row above huged, the long-row count and the hub-row count.
enum { S_NMOVES = 0, S_C1 = 1, S_C2 = 2, S_EXCESS = 3, S_NCAND = 4, S_CUT2 = 5, S_DIRTY = 6,
       S_HUGEMV = 7, S_LISTCNT = 8, S_NU = 9, S_NP = 10, S_NCANDP = 11, S_JN = 12, S_JP = 13, S_JL = 14,
       S_PASS_END = 16, S_BIGCNT = 16, S_DONE = 20 };

// hub_list (nullable): the rows longer than gain_hub_deg among big_list, which
// the dense build walks instead of big_list when k <= warp_dense_k (its other
// rows are gain_bigwarp_kernel's)
int build_rows(hp_context *c, HpLevel &g, RefineBufs &B, int32_t k, const int32_t *small_list,
               const int32_t *d_small_cnt, const int32_t *big_list, const int32_t *d_big_cnt,
               bool any_big, int32_t *dirty, const int32_t *hub_list = nullptr,
               const int32_t *d_hub_cnt = nullptr)
{
    const hp_tuning &tn = c->tune;
    if (small_list) {
        // rebuild of dirty rows: segments of S lanes per row (latency of a warp
        // per row, 32/S rows per warp)
        const unsigned grid = (unsigned)(c->sm_count * tn.grid_ctas_per_sm);
        if (B.small_max <= 8)
            HP_LAUNCH(c, gain_seg_kernel<8>, grid, 256, 0, small_list, d_small_cnt, g.xadj, g.adjncy, g.adjwgt,
                      g.where, B.goff, B.gpart, B.gconn, k, dirty);
        else if (B.small_max <= 16)
            HP_LAUNCH(c, gain_seg_kernel<16>, grid, 256, 0, small_list, d_small_cnt, g.xadj, g.adjncy, g.adjwgt,
                      g.where, B.goff, B.gpart, B.gconn, k, dirty);
        else
            HP_LAUNCH(c, gain_seg_kernel<32>, grid, 256, 0, small_list, d_small_cnt, g.xadj, g.adjncy, g.adjwgt,
                      g.where, B.goff, B.gpart, B.gconn, k, dirty);
    } else {
        // full build of the level: one thread per row, register network
        const unsigned grid = nblk(g.n);
        if (B.small_max <= 8)
            HP_LAUNCH(c, gain_thread_kernel<8>, grid, 256, 0, nullptr, nullptr, g.n, g.xadj, g.adjncy, g.adjwgt,
                      g.where, B.goff, B.gpart, B.gconn, k, dirty, tn.gain_thread_deg);
        else if (B.small_max <= 16)
            HP_LAUNCH(c, gain_thread_kernel<16>, grid, 256, 0, nullptr, nullptr, g.n, g.xadj, g.adjncy, g.adjwgt,
                      g.where, B.goff, B.gpart, B.gconn, k, dirty, tn.gain_thread_deg);
        else
            HP_LAUNCH(c, gain_thread_kernel<32>, grid, 256, 0, nullptr, nullptr, g.n, g.xadj, g.adjncy, g.adjwgt,
                      g.where, B.goff, B.gpart, B.gconn, k, dirty, tn.gain_thread_deg);
    }
    if (any_big) {
        const size_t smem = sizeof(int32_t) * (size_t)k + sizeof(unsigned) * (size_t)((k + 31) / 32);
        if (k <= tn.warp_dense_k)
            HP_LAUNCH(c, gain_bigwarp_kernel, (unsigned)(c->sm_count * 4), 32 * GW_WARPS, GW_WARPS * smem, big_list,
                      d_big_cnt, g.xadj, g.adjncy, g.adjwgt, g.where, B.goff, B.gpart, B.gconn, k, dirty,
                      tn.gain_thread_deg, tn.gain_hub_deg);
        // hub rows: every such row in a full build; in a rebuild only sparse
        // ones (deg < k), which exist only when k > gain_hub_deg
        const bool dense_rows = dirty ? (B.huge_rows && k > tn.gain_hub_deg) : B.huge_rows;
        const bool hubs = hub_list && k <= tn.warp_dense_k;
        if (k > tn.warp_dense_k || dense_rows)
            HP_LAUNCH(c, gain_dense_kernel<256>, (unsigned)(c->sm_count * 2), 256, smem, hubs ? hub_list : big_list,
                      hubs ? d_hub_cnt : d_big_cnt, g.xadj, g.adjncy, g.adjwgt, g.where, B.goff, B.gpart, B.gconn, k,
                      dirty, tn.gain_thread_deg, tn.gain_hub_deg, tn.warp_dense_k);
    }
    return HP_OK;
}

int key_bits_for(int32_t k)
{
    int64_t maxkey = (int64_t)k * 64;
    int bits = 0;
    while ((1ll << bits) < maxkey) bits++;
    return (bits + 7) / 8 * 8;
}

// Persistent grid of the rank/evict kernels: at most the tiles a count of n
// can need, at most grid_ctas_per_sm CTAs per SM (they take tiles until the
// device count).
unsigned rank_grid(const hp_context *c, int64_t tiles)
{
    return (unsigned)std::min<int64_t>(tiles, (int64_t)c->sm_count * c->tune.grid_ctas_per_sm);
}

// Persistent grid of a chunk plan over at most cap items (the tile holding
// index cap included).
unsigned plan_grid(const hp_context *c, int64_t cap)
{
    return rank_grid(c, cap / PLAN_TILE + 1);
}

// Candidates of the pass (rb_candidates_kernel, K/V in vertex order) -> stable
// radix sort by key -> prefix weights and part bounds (rb_rank_kernel).
// Returns the arrays holding the sorted pairs.
template <bool STRONG>
int rank_candidates(hp_context *c, HpLevel &g, RefineBufs &B, int32_t k, int32_t **Ks, int32_t **Vs,
                    const BestCopy &bcp)
{
    const int32_t n = g.n;
    unsigned long long *sc = c->d_scal;
    int32_t *d_cnt = (int32_t *)&sc[S_LISTCNT];
    const int64_t ct = ((int64_t)n + RB_TILE - 1) / RB_TILE;
    const int64_t rt = ((int64_t)n + RK_TILE) / RK_TILE;   // a tile holds index cnt <= n
    if (ct > c->lb_cap || 2 * rt > c->lb_cap) return HP_ERR_INTERNAL;
    HP_LAUNCH(c, rb_candidates_kernel<STRONG>, (unsigned)ct, RB_TILE, 0, n, g.where, g.vwgt, B.pw, B.maxp, B.opt,
              B.goff, B.gpart, B.gconn, B.und, (const int32_t *)&sc[S_NU], k, B.K, B.V, B.dest, d_cnt, B.pstart,
              B.pend, c->lb_status, c->lb_ctl, c->d_status, B.ufl, bcp);
    bool in_tmp = false;
    HP_TRY(hp_sort_pairs(c, B.K, B.V, B.K2, B.V2, n, d_cnt, key_bits_for(k), &in_tmp));
    *Ks = in_tmp ? B.K2 : B.K;
    *Vs = in_tmp ? B.V2 : B.V;
    HP_LAUNCH(c, rb_rank_kernel, rank_grid(c, rt), RK_THREADS, 0, *Ks, *Vs, d_cnt, g.vwgt, B.pre, B.pstart, B.pend,
              c->lb_status, c->lb_ctl, c->d_status);
    return HP_OK;
}

MoveSink move_sink(hp_context *c, const RefineBufs &B, int32_t k)
{
    unsigned long long *sc = c->d_scal;
    return MoveSink{B.moves, B.oldp, &sc[S_NMOVES], &sc[S_C1], B.goff, B.gpart, B.gconn, k};
}

// The undersized-part list of a weak pass is built by ctl_begin_kernel.
int weak_rebalance(hp_context *c, HpLevel &g, RefineBufs &B, int32_t k, const BestCopy &bcp)
{
    unsigned long long *sc = c->d_scal;
    int32_t *Ks, *Vs;
    HP_TRY(rank_candidates<false>(c, g, B, k, &Ks, &Vs, bcp));
    HP_LAUNCH(c, rw_select_kernel, (unsigned)(c->sm_count * 8), 256, 0, Ks, Vs,
              (const int32_t *)&sc[S_LISTCNT], B.pre, B.pstart, B.pw, B.maxp, B.dest, move_sink(c, B, k));
    return HP_OK;
}

int strong_rebalance(hp_context *c, HpLevel &g, RefineBufs &B, int32_t k, const BestCopy &bcp)
{
    const int32_t n = g.n;
    unsigned long long *sc = c->d_scal;
    int32_t *Ks, *Vs;
    HP_TRY(rank_candidates<true>(c, g, B, k, &Ks, &Vs, bcp));
    const unsigned pg = (unsigned)(c->sm_count * 8);
    const int32_t *d_cnt = (const int32_t *)&sc[S_LISTCNT];
    int32_t *d_np = (int32_t *)&sc[S_NP];
    HP_LAUNCH(c, evict_end_kernel, nblk(k), 256, 0, k, B.pstart, B.pend, B.pre, B.pw, B.maxp, B.ev_end);
    const int64_t rt = ((int64_t)n + RK_TILE) / RK_TILE;
    HP_LAUNCH(c, rs_evict_kernel, rank_grid(c, rt), RK_THREADS, 0, Ks, Vs, d_cnt, B.ev_end, g.vwgt, B.P, B.sp, d_np,
              c->lb_status, c->lb_cap / 2, c->lb_ctl, c->d_status);
    HP_LAUNCH(c, cookie_cutter_kernel, 1, 1024, sizeof(int32_t) * COOKIE_SMEM_INTS, k, B.pw, B.maxp, B.sp, d_np,
              B.es, B.ee);
    HP_LAUNCH(c, rs_assign_kernel, pg, 256, 0, k, B.P, d_np, Vs, B.es, B.ee, g.where, B.dest,
              move_sink(c, B, k));
    return HP_OK;
}

// ---- pass control ------------------------------------------------------------------
// The pass loop's bookkeeping (exact cut, best partition, patience, stall rule,
// next mode) lives in device memory and is advanced by one-thread kernels.  The
// same rule therefore drives both loops: the eager loop reads the block after
// every pass, the CUDA-graph loop lets the block set its own WHILE and SWITCH
// conditions.  Passes per level are capped (a bound on the device-side loop).
constexpr int32_t HP_MAX_REFINE_PASSES = 1 << 14;

struct RefineCtl {
    long long cut, excess, best_cut, best_excess, cut_before, cut_start, last_moves;
    int32_t count, bal, passes, lp_idle;
    int32_t learned_active, learned_pass, mode, best_current;
    int32_t take, cont, patience, last_mode;
    int32_t mode_passes[4];
    int32_t gain_entries, pad;   // G of the level (for the profiler's byte counts)
    int32_t judge_mode;          // hp_options.learned = 3: the plain refiner judges every learned pass
    int32_t judge_pass;          // the current pass is a learned LP pass under that judge
};

__device__ void ctl_prepare(RefineCtl *s)
{
    s->passes++;
    s->mode = s->excess <= 0 ? 0 : (s->bal < 2 ? 1 : 2);
    s->learned_pass = (s->excess <= 0 && s->learned_active) ? 1 : 0;
    s->judge_pass = s->learned_pass && s->judge_mode;
    s->cut_before = s->cut;
    s->bal = s->mode == 0 ? 0 : s->bal + 1;
    s->mode_passes[s->mode]++;
}

__device__ int ctl_advance(RefineCtl *s, long long m, long long c1, long long c2, long long nmoves, long long ncand,
                           long long jp2);

// The level's starting cut: the coarser level's best cut when there is one (a
// projection keeps the cut exactly: every coarse edge weight is the sum of
// the fine edges between its two clusters, and edges inside a cluster are
// never cut), else the cut summed from the gain rows (rowcut_kernel).
__device__ void ctl_init_state(RefineCtl *s, long long cut, long long excess, int32_t patience, int32_t learned,
                               int32_t gain_total, int32_t judge)
{
    s->gain_entries = gain_total;
    s->cut = cut;
    s->excess = excess;
    s->cut_start = s->cut;
    s->best_cut = s->cut;
    s->best_excess = s->excess;
    s->best_current = 1;
    s->count = 0;
    s->bal = 0;
    s->passes = 0;
    s->lp_idle = 0;
    s->learned_active = learned;
    s->learned_pass = 0;
    s->judge_mode = learned && judge;
    s->judge_pass = 0;
    s->take = 0;
    s->last_moves = 0;
    s->last_mode = -1;
    s->patience = patience;
    s->mode = 0;
    for (int i = 0; i < 4; i++) s->mode_passes[i] = 0;
    s->cont = s->count <= patience;   // while (count++ <= patience)
    s->count++;
    if (s->cont) ctl_prepare(s);
}

__global__ void ctl_init_kernel(RefineCtl *s, const unsigned long long *sc, int32_t patience, int32_t learned,
                                const int32_t *gain_total, const RefineCtl *coarser, int32_t judge)
{
    hp::pdl_wait();
    ctl_init_state(s, coarser ? coarser->best_cut : (long long)sc[S_CUT2] / 2, (long long)sc[S_EXCESS], patience,
                   learned, *gain_total, judge);
}

// End of a pass: the exact cut change, the learned fallback, the stall rule, the
// best partition and the loop condition, in the order of the host loop they replace.
// End of a pass: the after-move half of the exact cut change (c2: the moved
// vertices' gain rows, rebuilt, at the old and new parts; c1 came with the moves),
// then the control step, run by the last CTA to finish (a ticket on *done,
// reset by that CTA): the max excess over the parts (max_p pw[p] - maxp[p]) and,
// by thread 0, the control block's advance and the graph loop's condition.
// One launch instead of a cut-change kernel and a one-CTA control kernel.
__global__ void __launch_bounds__(256)
pass_end_kernel(const int32_t *__restrict__ moves, const unsigned long long *d_nmoves,
                const int32_t *__restrict__ goff, const int32_t *__restrict__ gpart,
                const int32_t *__restrict__ gconn, const int32_t *__restrict__ where,
                const int32_t *__restrict__ oldp, int32_t k, RefineCtl *s, unsigned long long *sc,
                cudaGraphConditionalHandle hloop, int graph, const unsigned long long *__restrict__ pw,
                const int64_t *__restrict__ maxp, unsigned *status, unsigned *done)
{
    hp::pdl_wait();
    __shared__ bool s_last;
    __shared__ long long s_max[256 / 32];
    const int64_t nm = (int64_t)*d_nmoves;
    long long acc = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nm; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = moves[i];
        const int32_t o = goff[v], len = goff[v + 1] - o;
        acc += (long long)row_conn(gpart + o, gconn + o, len, where[v], k) -
               row_conn(gpart + o, gconn + o, len, oldp[i], k);
    }
    hp::block_add_to<256>(acc, &sc[S_C2]);   // ends with a barrier
    if (threadIdx.x == 0) {
        __threadfence();   // this CTA's sum is visible before its ticket
        s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    long long m = LLONG_MIN;
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        const long long e = (long long)pw[p] - maxp[p];
        m = e > m ? e : m;
    }
    m = hp::warp_max64(m);
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = s_max[w] > m ? s_max[w] : m;
    *done = 0u;
    volatile unsigned long long *vs = sc;
    sc[S_EXCESS] = (unsigned long long)m;
    const long long c1 = (long long)vs[S_C1], c2 = (long long)vs[S_C2];
    // the judge's sum over the learned moves is the applied pass's exact change
    if (s->judge_pass && (long long)vs[S_JL] != c1 + c2) atomicOr(status, HP_STATUS_OVERFLOW);
    const int cont = ctl_advance(s, m, c1, c2, (long long)vs[S_NMOVES], (long long)vs[S_NCAND], (long long)vs[S_JP]);
    if (graph) cudaGraphSetConditional(hloop, cont ? 1u : 0u);
}

// The control step of a pass end (one thread): new excess m, the cut-change
// sums c1 and c2, the pass's moves and LP candidates.  Returns the loop condition.
__device__ int ctl_advance(RefineCtl *s, long long m, long long c1, long long c2, long long nmoves, long long ncand,
                           long long jp2)
{
    s->excess = m;
    s->cut -= (c1 + c2) / 2;
    s->last_moves = nmoves;
    s->last_mode = s->mode;
    // The plain refiner takes over for the rest of the level as soon as a
    // learned pass does not lower the cut, and under the judge (learned = 3) as
    // soon as it lowers the cut less than the plain pass would have on the same
    // state: c1 + c2 and jp2 are twice the exact cut decrease of the learned and
    // of the plain moves.
    bool handed = false;
    if (s->learned_pass && (c1 + c2 <= 0 || (s->judge_pass && c1 + c2 < jp2))) {
        s->learned_active = 0;
        handed = true;
    }
    const int mode = s->mode;
    // A pass that changed nothing (no moves, no lock change) is repeated
    // identically by every later pass and can never improve the best
    // partition: stop now; the result is the same as running on.  Under the
    // judge a learned pass that handed over is not such a pass: the plain pass
    // after it differs.
    const bool stalled = !(handed && s->judge_mode) && nmoves == 0 &&
                         (mode == 2 || (mode == 0 && (ncand == 0 || s->lp_idle)));
    s->lp_idle = (mode == 0 && nmoves == 0) ? 1 : 0;
    int take = 0;
    if (s->best_excess > 0 && s->excess < s->best_excess) {
        take = 1;
        s->count = 0;
    } else if (s->cut < s->best_cut && (s->excess <= 0 || s->excess <= s->best_excess)) {
        if (1000 * s->cut < 999 * s->best_cut) s->count = 0;
        take = 1;
    }
    if (take) {
        s->best_cut = s->cut;
        s->best_excess = s->excess;
    }
    s->best_current = take;
    s->take = take;
    int cont = 0;
    if (!stalled) {
        cont = s->count <= s->patience;
        s->count++;
    }
    if (s->passes >= HP_MAX_REFINE_PASSES) cont = 0;
    s->cont = cont;
    if (cont) ctl_prepare(s);
    return cont;
}

// Start of a pass (one CTA of 1024 threads): clear the per-pass scalar slots,
// in the graph loop select the proposal body (0 LP, 1 weak rebalance, 2 strong
// rebalance), and for a weak pass build the undersized-part list.
__global__ void __launch_bounds__(1024)
ctl_begin_kernel(const RefineCtl *s, unsigned long long *sc, cudaGraphConditionalHandle hmode, int graph, int32_t k,
                 const unsigned long long *__restrict__ pw, const int64_t *__restrict__ maxp,
                 int32_t *__restrict__ und, int8_t *__restrict__ ufl)
{
    hp::pdl_wait();
    __shared__ int32_t s_scan[1024 / 32 + 2];
    if (threadIdx.x < S_PASS_END) sc[threadIdx.x] = 0;
    const int mode = s->mode;
    if (graph && threadIdx.x == 0) cudaGraphSetConditional(hmode, (unsigned)mode);
    __syncthreads();
    if (mode == 1) {
        undersized_block(k, pw, maxp, und, (int32_t *)&sc[S_NU], s_scan);
        for (int32_t q = threadIdx.x; q < k; q += blockDim.x) ufl[q] = (int64_t)pw[q] < maxp[q];
    }
}

__global__ void restore_best_kernel(const RefineCtl *s, int32_t n, const int32_t *__restrict__ best_where,
                                    int32_t *__restrict__ where)
{
    hp::pdl_wait();
    if (s->best_current) return;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) where[i] = best_where[i];
}

// ---- profile-only byte counts -------------------------------------------------------
// The data-dependent terms of the refinement classes' algorithmic byte models
// (rows walked, candidates, moves, dirty rows), counted on the device in
// profiled eager passes into the class counters (hp_prof_counter) after the
// class's launches, so that the counting is not timed with them.  Neighbour
// gathers are not counted (compulsory-traffic model, as for every class).

// Bytes a gain-row walk reads: a dense row (k entries, longer than 32 and so
// walked by a warp with the part ids implied) reads k connectivities; any
// other row its (part, conn) pairs up to and including the first padding slot.
__device__ __forceinline__ long long row_walk_bytes(const int32_t *__restrict__ gpart, int32_t o, int32_t len,
                                                    int32_t k)
{
    if (len > 32 && len == k) return 4ll * k;
    int32_t f = 0;
    while (f < len && gpart[o + f] >= 0) f++;
    return 8ll * (f < len ? f + 1 : f);
}

// LP: every row's walk by the selection, and each candidate's adjacency row
// (adjncy + adjwgt) and destination read by the afterburner.
__global__ void __launch_bounds__(256)
lp_bytes_kernel(int32_t n, const int32_t *__restrict__ goff, const int32_t *__restrict__ gpart,
                const int32_t *__restrict__ xadj, const int32_t *__restrict__ pregain, int32_t k,
                unsigned long long *acc)
{
    hp::pdl_wait();
    long long b = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        b += row_walk_bytes(gpart, goff[v], goff[v + 1] - goff[v], k);
        if (pregain[v] != NEG) b += 8ll * (xadj[v + 1] - xadj[v]) + 4;
    }
    hp::block_add_to<256>(b, acc);
}

// Rebuild of the dirty rows: xadj, goff and the list entry, the adjacency row,
// the rewritten gain row (8 bytes per slot) and the dirty flag's reset.
__global__ void __launch_bounds__(256)
rebuild_bytes_kernel(const int32_t *__restrict__ small_l, const int32_t *__restrict__ d_nsmall,
                     const int32_t *__restrict__ big_l, const int32_t *__restrict__ d_nbig,
                     const int32_t *__restrict__ xadj, const int32_t *__restrict__ goff, unsigned long long *acc)
{
    hp::pdl_wait();
    const int32_t ns = *d_nsmall, nb = *d_nbig;
    long long b = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)ns + nb;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = i < ns ? small_l[i] : big_l[i - ns];
        b += 24 + 8ll * (xadj[v + 1] - xadj[v]) + 8ll * (goff[v + 1] - goff[v]);
    }
    hp::block_add_to<256>(b, acc);
}

// Rebalance proposals (counted before the moves apply, with the part weights
// the proposal saw): where and dest of every vertex; vertex weight, goff and
// the gain-row walk of every vertex of an overweight part; per candidate its
// key/value write, 20 bytes per radix pass (digit histogram read, pair
// scatter) and the rank/select (or evict) reads of the sorted pairs.
__global__ void __launch_bounds__(256)
rebalance_bytes_kernel(int32_t n, const int32_t *__restrict__ where, const unsigned long long *__restrict__ pw,
                       const int64_t *__restrict__ maxp, const int32_t *__restrict__ goff,
                       const int32_t *__restrict__ gpart, int32_t k, const int32_t *__restrict__ d_cnt,
                       int32_t radix_passes, unsigned long long *acc)
{
    hp::pdl_wait();
    long long b = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = where[v];
        b += 8;
        if ((int64_t)pw[p] > maxp[p]) b += 12 + row_walk_bytes(gpart, goff[v], goff[v + 1] - goff[v], k);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) b += (long long)(*d_cnt) * (32 + 20ll * radix_passes);
    hp::block_add_to<256>(b, acc);
}

// Move application: per move its list entries (vertex, old part), destination,
// vertex weight, xadj, adjacency row and where write, then the exact cut
// change's goff read and walk of the mover's gain row; once per pass the
// control step's part weights and bounds, and the best-partition copy when
// the pass was the best so far.
__global__ void __launch_bounds__(256)
apply_bytes_kernel(const int32_t *__restrict__ moves, const unsigned long long *__restrict__ d_nmoves,
                   const int32_t *__restrict__ xadj, const int32_t *__restrict__ goff,
                   const int32_t *__restrict__ gpart, int32_t k, int32_t n, const RefineCtl *ctl,
                   unsigned long long *acc)
{
    hp::pdl_wait();
    const int64_t nm = (int64_t)*d_nmoves;
    long long b = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nm; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = moves[i];
        b += 36 + 8ll * (xadj[v + 1] - xadj[v]) + row_walk_bytes(gpart, goff[v], goff[v + 1] - goff[v], k);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) b += 16ll * k + (ctl->take ? 8ll * n + 16ll * k : 0);
    hp::block_add_to<256>(b, acc);
}

struct PassCfg {
    int32_t k;
    bool finest, any_big, recording, huge_rows;   // huge_rows: rows longer than chunk_deg exist
    bool judged;                                  // learned = 3: learned passes are judged
    bool huge_moves;                              // rows longer than apply_chunk_deg exist
    RefineCtl *ctl;
    unsigned long long *best_pw;
};

BestCopy best_copy(const RefineBufs &B, const PassCfg &P)
{
    return BestCopy{&P.ctl->take, B.best_where, B.pw, P.best_pw, P.k};
}

// Proposal phase of one pass.  Eager mode launches the LP selection kernel the
// host chose; graph mode launches both when the MLP is loaded, gated by the
// control block's learned_pass flag.
int pass_propose(hp_context *c, HpLevel &g, RefineBufs &B, const PassCfg &P, int mode, bool learned_pass,
                 bool both_lp)
{
    const int32_t n = g.n, k = P.k;
    unsigned long long *sc = c->d_scal;
    int32_t *d_bigcnt = (int32_t *)&sc[S_BIGCNT];
    const unsigned pg = (unsigned)(c->sm_count * c->tune.grid_ctas_per_sm);
    const int32_t *gate = both_lp ? &P.ctl->learned_pass : nullptr;
    if (mode == 0) {
        const int ltok = hp_prof_begin(c);
        const Judge J{&P.ctl->judge_pass, B.prune, B.accp, B.jlist, (int32_t *)&sc[S_JN], &sc[S_NCANDP]};
        const bool judging = P.judged && (both_lp || learned_pass);
        if (both_lp || learned_pass)
            HP_LAUNCH(c, lp_select_learned_kernel, nblk(n), 256, 0, n, B.goff, B.gpart, B.gconn, g.where, g.xadj,
                      B.lock, P.finest ? 1 : 0, B.pw, B.maxp, B.opt, c->mlp_params, c->mlp_threshold, B.dest,
                      B.pregain, &sc[S_NCAND], gate, k, B.prune, &sc[S_NCANDP], J.flag, best_copy(B, P));
        if (both_lp || !learned_pass)
            HP_LAUNCH(c, lp_select_kernel, nblk(n), 256, 0, n, B.goff, B.gpart, B.gconn, g.where, B.lock,
                      P.finest ? 1 : 0, B.dest, B.pregain, &sc[S_NCAND], gate, k, best_copy(B, P));
        if (P.recording)
            HP_LAUNCH(c, log_candidates_kernel, nblk(n), 256, 0, n, B.goff, B.gpart, B.gconn, g.where, g.xadj,
                      P.finest ? 1 : 0, B.pw, B.maxp, B.opt, B.dest, B.pregain, B.recof, c->log_x, c->log_v,
                      c->log_d, c->log_acc, c->log_count, c->log_cap);
        HP_LAUNCH(c, afterburner_small_kernel, nblk(n), 256, 0, n, g.xadj, g.adjncy, g.adjwgt, g.where, B.dest,
                  B.pregain, B.lock, &sc[S_NCAND], move_sink(c, B, k), c->tune.gain_thread_deg, J);
        if (P.any_big)
            HP_LAUNCH(c, afterburner_big_kernel, pg, 256, 0, B.big, d_bigcnt, g.xadj, g.adjncy, g.adjwgt, g.where,
                      B.dest, B.pregain, B.lock, &sc[S_NCAND], move_sink(c, B, k), c->tune.chunk_deg, J);
        if (P.huge_rows) {
            const int32_t *d_nhuge = d_bigcnt + 3;
            HP_LAUNCH(c, hub_plan_kernel<false>, plan_grid(c, B.nhub_cap), PLAN_THREADS, 0, B.huge, d_nhuge, B.moves,
                      B.pregain, g.xadj, B.plan_v, B.plan_item, B.plan_off, B.plan_cnt, c->lb_status, c->lb_cap / 2,
                      c->lb_ctl, c->d_status);
            HP_LAUNCH(c, afterburner_huge_kernel, (unsigned)(4 * c->sm_count), HUB_CHUNK, 0, B.plan_v, B.plan_item,
                      B.plan_off, B.plan_cnt, g.xadj, g.adjncy, g.adjwgt, g.where, B.dest, B.pregain, &sc[S_NCAND],
                      B.ab_acc, B.ab_acc2, J);
            HP_LAUNCH(c, afterburner_huge_final_kernel, (unsigned)c->sm_count, 256, 0, B.huge, d_nhuge, B.pregain,
                      &sc[S_NCAND], B.ab_acc, B.ab_acc2, B.lock, g.where, B.dest, move_sink(c, B, k), J);
        }
        if (judging) {   // the plain refiner's exact cut change on the same state (learned passes only)
            const int64_t rt = ((int64_t)n + RK_TILE) / RK_TILE;   // a tile holds index cnt <= n
            if (rt > c->lb_cap) return HP_ERR_INTERNAL;
            HP_LAUNCH(c, judge_off_kernel, rank_grid(c, rt), RK_THREADS, 0, J.flag, B.jlist, J.d_n, g.xadj, B.joff,
                      c->lb_status, c->lb_ctl, c->d_status);
            HP_LAUNCH(c, judge_delta_kernel, pg, JD_THREADS, 0, J.flag, B.jlist, J.d_n, B.joff, g.xadj, g.adjncy,
                      g.adjwgt, g.where, B.dest, B.accp, B.lock, &sc[S_JP]);
        }
        if (P.recording)
            HP_LAUNCH(c, log_accept_kernel, nblk(n), 256, 0, n, B.recof, B.lock, &sc[S_NCAND], c->log_acc);
        // fixed terms -- selection: goff, where, lock in, dest and pregain out;
        // afterburner: xadj, pregain in, lock out.  The rows walked and the
        // candidates' adjacency rows are counted on the device.
        hp_prof_end(c, ltok, HP_PROF_LP, 8 * ((int64_t)n + 1) + 18 * (int64_t)n);
        if (unsigned long long *cnt = hp_prof_counter(c, HP_PROF_LP))
            HP_LAUNCH(c, lp_bytes_kernel, std::min(nblk(n), pg), 256, 0, n, B.goff, B.gpart, g.xadj, B.pregain, k,
                      cnt);
    } else {
        const int btok = hp_prof_begin(c);
        if (mode == 1) HP_TRY(weak_rebalance(c, g, B, k, best_copy(B, P)));
        else HP_TRY(strong_rebalance(c, g, B, k, best_copy(B, P)));
        hp_prof_end(c, btok, HP_PROF_REBALANCE, 0);
        if (unsigned long long *cnt = hp_prof_counter(c, HP_PROF_REBALANCE))
            HP_LAUNCH(c, rebalance_bytes_kernel, std::min(nblk(n), pg), 256, 0, n, g.where, B.pw, B.maxp, B.goff,
                      B.gpart, k, (const int32_t *)&sc[S_LISTCNT], key_bits_for(k) / 8, cnt);
    }
    return HP_OK;
}

// Apply phase of one pass: simultaneous moves, exact cut change from the gain
// rows before and after, gain-row maintenance, balance, then the control step.
int pass_apply(hp_context *c, HpLevel &g, RefineBufs &B, const PassCfg &P, cudaGraphConditionalHandle hloop,
               int graph)
{
    const int32_t n = g.n, k = P.k;
    unsigned long long *sc = c->d_scal;
    const unsigned pg = (unsigned)(c->sm_count * c->tune.grid_ctas_per_sm);
    const unsigned mg = std::min(nblk(n), pg);   // grid-stride over the device move count
    // (the proposal kernels appended the moves with their old parts and c1)
    int atok = hp_prof_begin(c);
    HP_LAUNCH(c, apply_moves_kernel, pg, 256, 0, B.moves, &sc[S_NMOVES], g.where, B.dest, g.vwgt, B.pw, g.xadj,
              g.adjncy, g.adjwgt, B.goff, B.gconn, B.dirty, B.small_l, B.big_l, (int32_t *)&sc[S_DIRTY], k,
              B.huge_mv, (int32_t *)&sc[S_HUGEMV], c->tune.gain_thread_deg, c->tune.apply_chunk_deg);
    if (P.huge_moves) {
        HP_LAUNCH(c, hub_plan_kernel<true>, plan_grid(c, B.nhub_cap), PLAN_THREADS, 0, B.huge_mv,
                  (const int32_t *)&sc[S_HUGEMV], B.moves, B.pregain, g.xadj, B.plan_v, B.plan_item, B.plan_off,
                  B.plan_cnt, c->lb_status, c->lb_cap / 2, c->lb_ctl, c->d_status);
        HP_LAUNCH(c, apply_moves_huge_kernel, (unsigned)(4 * c->sm_count), HUB_CHUNK, 0, B.plan_v, B.plan_item,
                  B.plan_off, B.plan_cnt, B.oldp, B.dest, g.xadj, g.adjncy, g.adjwgt, B.goff, B.gconn, B.dirty,
                  B.small_l, B.big_l, (int32_t *)&sc[S_DIRTY], k, c->tune.gain_thread_deg);
    }
    hp_prof_end(c, atok, HP_PROF_APPLY, 0);
    const int rtok = hp_prof_begin(c);
    HP_TRY(build_rows(c, g, B, k, B.small_l, (const int32_t *)&sc[S_DIRTY], B.big_l,
                      ((const int32_t *)&sc[S_DIRTY]) + 1, P.any_big, B.dirty));
    hp_prof_end(c, rtok, HP_PROF_REBUILD, 0);
    if (unsigned long long *cnt = hp_prof_counter(c, HP_PROF_REBUILD))
        HP_LAUNCH(c, rebuild_bytes_kernel, pg, 256, 0, B.small_l, (const int32_t *)&sc[S_DIRTY], B.big_l,
                  ((const int32_t *)&sc[S_DIRTY]) + 1, g.xadj, B.goff, cnt);
    atok = hp_prof_begin(c);
    HP_LAUNCH(c, pass_end_kernel, mg, 256, 0, B.moves, &sc[S_NMOVES], B.goff, B.gpart, B.gconn, g.where, B.oldp, k,
              P.ctl, sc, hloop, graph, B.pw, B.maxp, c->d_status, (unsigned *)&sc[S_DONE]);
    hp_prof_end(c, atok, HP_PROF_APPLY, 0);
    if (unsigned long long *cnt = hp_prof_counter(c, HP_PROF_APPLY))
        HP_LAUNCH(c, apply_bytes_kernel, mg, 256, 0, B.moves, &sc[S_NMOVES], g.xadj, B.goff, B.gpart, k, n, P.ctl,
                  cnt);
    return HP_OK;
}

// ---- small levels: every pass of the level in one CTA --------------------------------
// A level with few vertices runs its whole pass loop inside one CTA of
// SL_THREADS threads.  The phases are those of the multi-kernel pass, in the
// same order and through the same device functions -- LP selection and
// afterburner, weak or strong rebalance (candidates, stable radix sort, ranks,
// selection or eviction and cookie cutter), simultaneous moves, gain-row
// maintenance, the exact cut change, the control step and the best partition --
// separated by __syncthreads instead of kernel boundaries.  Gain rows,
// candidates and moves equal the multi-kernel pass's, so the level's result is
// identical; what goes away is about fifteen launches per pass, which on small
// levels cost more than the work.
constexpr int SL_THREADS = 1024;
constexpr int SL_WARPS = SL_THREADS / 32;
constexpr int SL_SORT_INTS = hp::block_sort_ints(SL_THREADS);

struct SmallLevel {
    int32_t n, k, finest, bigd, small_max, key_bits, learned_mlp;
    int32_t patience, judge;    // the control block's init (the level's setup runs in the kernel)
    const RefineCtl *coarser;   // the coarser level's control block (its best cut), or nullptr
    float mlp_threshold;
    const int32_t *xadj, *adjncy, *adjwgt, *vwgt;
    int32_t *where;
    int32_t *goff;
    int32_t *gpart, *gconn;
    int32_t *dest, *pregain, *moves, *oldp, *dirty, *small_l, *big_l, *best_where;
    int32_t *K, *V, *K2, *V2, *pre, *P, *sp;
    int32_t *pstart, *pend, *und, *ev_end, *es, *ee;
    int8_t *lock;
    int8_t *prune, *accp;   // the judge of a learned pass
    unsigned long long *pw, *best_pw;
    const int64_t *opt, *maxp;
    const float *mlp_params;
    RefineCtl *ctl;
    unsigned *status;
};

// Dynamic shared memory of the small-level kernel: the largest of the phases'
// needs (sort tables; the staged prefix weights of the cookie cutter, at most
// n + 1; the warps' dense gain-row accumulators).
size_t small_level_smem(int32_t n, int32_t k)
{
    const size_t sort = sizeof(int32_t) * SL_SORT_INTS;
    const size_t cookie = sizeof(int32_t) * ((size_t)n + 1);
    const size_t rows = sizeof(int32_t) * SL_WARPS * ((size_t)k + (k + 31) / 32);
    return std::max(sort, std::max(cookie, rows));
}

// Block-wide sum / max of a long long; every thread gets the result.
__device__ __forceinline__ long long sl_sum64(long long v, long long *s_red)
{
    v = hp::warp_sum64(v);
    __syncthreads();   // the previous reduction has been read
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    long long t = 0;
#pragma unroll 8
    for (int w = 0; w < SL_WARPS; w++) t += s_red[w];
    return t;
}

__device__ __forceinline__ long long sl_max64(long long v, long long *s_red)
{
    v = hp::warp_max64(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    long long t = LLONG_MIN;
#pragma unroll 8
    for (int w = 0; w < SL_WARPS; w++) t = s_red[w] > t ? s_red[w] : t;
    return t;
}

__global__ void __launch_bounds__(SL_THREADS, 1)
refine_small_kernel(SmallLevel a)
{
    hp::pdl_wait();
    extern __shared__ __align__(16) int32_t sl_dyn[];
    __shared__ hp::MlpSmem s_mlp;
    __shared__ int32_t s_scan[SL_THREADS / 32 + 2];
    __shared__ long long s_red[SL_WARPS];
    __shared__ int32_t s_lists[2];   // dirty rows queued this pass: short, long
    __shared__ int32_t s_nu;         // undersized parts of a weak pass
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int32_t n = a.n, k = a.k;
    RefineCtl *s = a.ctl;
    if (a.learned_mlp) hp::mlp_load_smem(s_mlp, a.mlp_params);
    // ---- the level's setup, as the launches of the multi-kernel levels:
    // gain-row capacities min(deg, k) and offsets, cleared locks and dirty
    // flags, the rows' lists by length, part weights, the full gain-row build,
    // the starting cut (the coarser level's best cut, else summed from the
    // rows), the excess, the best-partition copy and the control block
    {
        int32_t run = 0, ns = 0, nb = 0;
        for (int32_t b0 = 0; b0 < n; b0 += SL_THREADS) {
            const int32_t v = b0 + tid;
            int32_t cap = 0, d = 0;
            if (v < n) {
                d = a.xadj[v + 1] - a.xadj[v];
                cap = d < k ? d : k;
                a.lock[v] = 0;
                a.dirty[v] = 0;
                a.best_where[v] = a.where[v];
            }
            int tot;
            const int ex = hp::block_excl_scan<SL_THREADS>(cap, &tot, s_scan);
            if (v < n) a.goff[v] = run + ex;
            run += tot;
            const bool sh = v < n && d <= a.bigd, lg = v < n && d > a.bigd;
            int ts, tl;
            const int es = hp::block_excl_scan<SL_THREADS>(sh ? 1 : 0, &ts, s_scan);
            const int el = hp::block_excl_scan<SL_THREADS>(lg ? 1 : 0, &tl, s_scan);
            if (sh) a.small_l[ns + es] = v;
            if (lg) a.big_l[nb + el] = v;
            ns += ts;
            nb += tl;
        }
        if (tid == 0) a.goff[n] = run;
        unsigned long long *spw = (unsigned long long *)sl_dyn;   // k <= 1024 part weights
        for (int32_t q = tid; q < k; q += SL_THREADS) spw[q] = 0ull;
        __syncthreads();
        for (int32_t v = tid; v < n; v += SL_THREADS) atomicAdd(&spw[a.where[v]], (unsigned long long)a.vwgt[v]);
        __syncthreads();
        for (int32_t q = tid; q < k; q += SL_THREADS) { a.pw[q] = spw[q]; a.best_pw[q] = spw[q]; }
        __syncthreads();   // the accumulators below reuse the shared memory
        if (ns > 0) {
            if (a.small_max <= 8)
                gain_seg_rows<8>(wid, SL_WARPS, a.small_l, ns, a.xadj, a.adjncy, a.adjwgt, a.where, a.goff, a.gpart,
                                 a.gconn, k, a.dirty);
            else if (a.small_max <= 16)
                gain_seg_rows<16>(wid, SL_WARPS, a.small_l, ns, a.xadj, a.adjncy, a.adjwgt, a.where, a.goff, a.gpart,
                                  a.gconn, k, a.dirty);
            else
                gain_seg_rows<32>(wid, SL_WARPS, a.small_l, ns, a.xadj, a.adjncy, a.adjwgt, a.where, a.goff, a.gpart,
                                  a.gconn, k, a.dirty);
        }
        if (nb > 0) {
            const int nw = (k + 31) >> 5;
            int32_t *dw = sl_dyn + (size_t)wid * (k + nw);
            unsigned *bm = (unsigned *)(dw + k);
            for (int i = lane; i < k; i += 32) dw[i] = 0;
            for (int i = lane; i < nw; i += 32) bm[i] = 0u;
            __syncwarp();
            gain_bigwarp_rows(wid, SL_WARPS, dw, bm, a.big_l, nb, a.xadj, a.adjncy, a.adjwgt, a.where, a.goff,
                              a.gpart, a.gconn, k, a.dirty, a.bigd, INT_MAX);
        }
        __syncthreads();
        long long cut = 0;
        if (!a.coarser) {   // the coarsest level: the cut from the gain rows
            long long acc = 0;
            for (int32_t v = tid; v < n; v += SL_THREADS) {
                const int32_t p = a.where[v], o = a.goff[v], len = a.goff[v + 1] - o;
                for (int32_t j = o; j < o + len; j++) {
                    const int32_t q = a.gpart[j];
                    if (q < 0) break;
                    if (q != p) acc += a.gconn[j];
                }
            }
            cut = sl_sum64(acc, s_red) / 2;
        }
        long long m = LLONG_MIN;
        for (int32_t q = tid; q < k; q += SL_THREADS) {
            const long long e = (long long)a.pw[q] - a.maxp[q];
            m = e > m ? e : m;
        }
        m = sl_max64(m, s_red);
        if (tid == 0)
            ctl_init_state(s, a.coarser ? a.coarser->best_cut : cut, m, a.patience, a.learned_mlp, a.goff[n],
                           a.judge);
    }
    __syncthreads();
    // the control step ends the loop; the pass cap bounds it as well
    for (int32_t guard = 0; guard <= HP_MAX_REFINE_PASSES; guard++) {
        if (!*(volatile const int32_t *)&s->cont) break;   // written by thread 0 before a barrier
        const int mode = *(volatile const int32_t *)&s->mode;
        if (tid < 2) s_lists[tid] = 0;
        long long ncand = 0, jp2 = 0, jl2 = 0;
        bool judged = false;
        int32_t nmoves = 0;
        if (mode == 0) {
            // ---- LP selection (plain or learned), as lp_select[_learned]_kernel
            const bool lrn = a.learned_mlp && *(volatile const int32_t *)&s->learned_pass;
            const bool jdg = lrn && *(volatile const int32_t *)&s->judge_pass;
            int32_t my_cand = 0, my_candp = 0;
            for (int32_t b0 = 0; b0 < n; b0 += SL_THREADS) {
                const int32_t v = b0 + tid;
                const bool in = v < n;
                int32_t p = 0, o = 0, len = 0;
                if (in) {
                    p = a.where[v];
                    o = a.goff[v];
                    len = a.goff[v + 1] - o;
                }
                const RowBest rb = row_best(a.gpart, a.gconn, o, len, p, k);
                int cand = 0;
                int32_t g = NEG, d = p;
                float f[HP_MLP_IN] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (in && rb.b >= 0) {
                    const int64_t thr = a.finest ? rb.pc / 4 : (3 * rb.pc) / 4;
                    if ((rb.bc >= rb.pc || (rb.pc - rb.bc) < thr) && !a.lock[v]) {
                        g = (int32_t)(rb.bc - rb.pc);
                        d = rb.b;
                        cand = 1;
                        if (lrn)
                            hp::mlp_features(rb.pc, rb.bc, rb.wd, rb.np, a.xadj[v + 1] - a.xadj[v],
                                             a.maxp[d] - (int64_t)a.pw[d], a.opt[d], a.maxp[p] - (int64_t)a.pw[p],
                                             a.opt[p], a.finest, f);
                    }
                }
                int8_t pr = 0;   // dropped by the MLP: keeps the plain gain and destination for the judge
                my_candp += cand;
                if (lrn && __any_sync(HP_FULL_MASK, cand)) {   // a warp without candidates needs no scores
                    const float logit = hp::mlp_warp_logit(s_mlp, f);
                    if (cand && logit < a.mlp_threshold) {
                        cand = 0;
                        if (jdg) pr = 1;
                        else { g = NEG; d = p; }
                    }
                }
                if (in) {
                    a.pregain[v] = g;
                    a.dest[v] = d;
                    if (jdg) a.prune[v] = pr;
                }
                my_cand += cand;
            }
            ncand = sl_sum64(my_cand, s_red);   // (barrier: every selection is visible)
            const long long ncandp = jdg ? sl_sum64(my_candp, s_red) : ncand;
            judged = jdg;
            if (ncand > 0 || (jdg && ncandp > 0)) {
                // ---- afterburner: every candidate re-scored against the
                // higher-priority neighbours; locks and moves (in vertex order)
                int32_t run = 0;
                for (int32_t b0 = 0; b0 < n; b0 += SL_THREADS) {
                    const int32_t v = b0 + tid;
                    const bool in = v < n;
                    const int32_t g = in ? a.pregain[v] : NEG;
                    const bool act = g != NEG;
                    const int32_t ro = act ? a.xadj[v] : 0, rl = act ? a.xadj[v + 1] - ro : 0;
                    const int32_t pp = act ? a.where[v] : 0, bb = act ? a.dest[v] : 0;
                    long long chp = 0, chl = 0;
                    const bool coop = rl > 32;
                    if (act && !coop)
                        for (int32_t j = ro; j < ro + rl; j++)
                            ab_change2(v, g, pp, bb, a.adjncy[j], a.adjwgt[j], a.pregain, a.dest, a.where, a.prune,
                                       jdg, chp, chl);
                    unsigned cm = __ballot_sync(HP_FULL_MASK, coop);
                    while (cm) {
                        const int src = __ffs(cm) - 1;
                        cm &= cm - 1;
                        const int32_t sv = __shfl_sync(HP_FULL_MASK, v, src), sg = __shfl_sync(HP_FULL_MASK, g, src);
                        const int32_t sp_ = __shfl_sync(HP_FULL_MASK, pp, src), sb = __shfl_sync(HP_FULL_MASK, bb, src);
                        const int32_t so = __shfl_sync(HP_FULL_MASK, ro, src), sl = __shfl_sync(HP_FULL_MASK, rl, src);
                        long long cp = 0, cl = 0;
                        ab_row_sum2(sv, sg, sp_, sb, so + lane, so + sl, 32, a.adjncy, a.adjwgt, a.pregain, a.dest,
                                    a.where, a.prune, jdg, cp, cl);
                        cp = hp::warp_sum64(cp);
                        if (jdg) cl = hp::warp_sum64(cl);
                        if (lane == src) { chp = cp; chl = cl; }
                    }
                    const int selp = act && ((long long)g + chp >= 0);
                    const int sel = jdg ? (act && !a.prune[v] && (long long)g + chl >= 0) : selp;
                    if (in) {
                        a.lock[v] = (int8_t)sel;
                        if (jdg) a.accp[v] = (int8_t)selp;
                    }
                    int tot;
                    const int ex = hp::block_excl_scan<SL_THREADS>(sel, &tot, s_scan);
                    if (sel) a.moves[run + ex] = v;
                    run += tot;
                }
                nmoves = run;
                if (jdg) {
                    // ---- the judge: exact cut decrease of the plain and the
                    // learned move sets on this state, as judge_delta_kernel
                    __syncthreads();   // every lock / accp is visible
                    long long sp = 0, sl = 0;
                    for (int32_t b0 = 0; b0 < n; b0 += SL_THREADS) {
                        const int32_t v = b0 + tid;
                        const bool in = v < n;
                        const bool mp = in && a.accp[v] != 0, ml = in && a.lock[v] != 0;
                        const bool act = mp || ml;
                        const int32_t ro = act ? a.xadj[v] : 0, rl = act ? a.xadj[v + 1] - ro : 0;
                        const int32_t pv = act ? a.where[v] : 0, dv = act ? a.dest[v] : 0;
                        const bool coop = rl > 32;
                        if (act && !coop)
                            for (int32_t j = ro; j < ro + rl; j++)
                                judge_entry(pv, dv, mp, ml, a.adjncy[j], a.adjwgt[j], a.where, a.dest, a.accp, a.lock,
                                            sp, sl);
                        unsigned cm = __ballot_sync(HP_FULL_MASK, coop);
                        while (cm) {
                            const int src = __ffs(cm) - 1;
                            cm &= cm - 1;
                            const int32_t so = __shfl_sync(HP_FULL_MASK, ro, src), sn = __shfl_sync(HP_FULL_MASK, rl, src);
                            const int32_t spv = __shfl_sync(HP_FULL_MASK, pv, src), sdv = __shfl_sync(HP_FULL_MASK, dv, src);
                            const bool smp = __shfl_sync(HP_FULL_MASK, (int)mp, src) != 0;
                            const bool sml = __shfl_sync(HP_FULL_MASK, (int)ml, src) != 0;
                            for (int32_t j = so + lane; j < so + sn; j += 32)
                                judge_entry(spv, sdv, smp, sml, a.adjncy[j], a.adjwgt[j], a.where, a.dest, a.accp,
                                            a.lock, sp, sl);
                        }
                    }
                    jp2 = sl_sum64(sp, s_red);
                    jl2 = sl_sum64(sl, s_red);
                }
            }
        } else {
            // ---- rebalance, as rb_candidates / sort / rb_rank / rw_select or
            // evict_end / rs_evict / cookie_cutter / rs_assign
            const bool strong = mode == 2;
            if (!strong) undersized_block(k, a.pw, a.maxp, a.und, &s_nu, s_scan);
            for (int32_t p = tid; p < k; p += SL_THREADS) {
                a.pstart[p] = -1;
                a.pend[p] = -1;
            }
            __syncthreads();
            const int32_t nu = s_nu;
            int32_t cnt = 0;
            for (int32_t b0 = 0; b0 < n; b0 += SL_THREADS) {
                const int32_t v = b0 + tid;
                const bool in = v < n;
                int32_t p = 0;
                bool cand = false;
                if (in) {
                    p = a.where[v];
                    const int64_t pwp = (int64_t)a.pw[p];
                    cand = strong ? (pwp > a.maxp[p] && (int64_t)a.vwgt[v] < 2 * (pwp - a.opt[p]))
                                  : (pwp > a.maxp[p] && 2 * (int64_t)a.vwgt[v] < 3 * (pwp - a.opt[p]));
                }
                const int32_t o = cand ? a.goff[v] : 0, len = cand ? a.goff[v + 1] - o : 0;
                int32_t d = p, kk = -1;
                if (!strong) {
                    int64_t pc = 0, bc = 0;
                    int32_t b = -1;
                    const bool coop = cand && len > RB_COOP;
                    if (cand && !coop)
                        for (int32_t j = o; j < o + len; j++) {
                            const int32_t q = a.gpart[j];
                            if (q < 0) break;
                            const int32_t cq = a.gconn[j];
                            if (q == p) pc = cq;
                            if ((int64_t)a.pw[q] < a.maxp[q] && cq > bc) { bc = cq; b = q; }
                        }
                    unsigned cm = __ballot_sync(HP_FULL_MASK, coop);
                    while (cm) {
                        const int src = __ffs(cm) - 1;
                        cm &= cm - 1;
                        const int32_t so = __shfl_sync(HP_FULL_MASK, o, src), sl = __shfl_sync(HP_FULL_MASK, len, src);
                        const int32_t sp_ = __shfl_sync(HP_FULL_MASK, p, src);
                        int32_t lpc = 0, lbc = 0, lb = -1;
                        for (int32_t j = lane; j < sl; j += 32) {
                            const int32_t q = a.gpart[so + j];
                            if (q < 0) break;
                            const int32_t cq = a.gconn[so + j];
                            if (q == sp_) lpc = cq;
                            if ((int64_t)a.pw[q] < a.maxp[q] && cq > lbc) { lbc = cq; lb = q; }
                        }
                        lpc = hp::warp_sum(lpc);
#pragma unroll
                        for (int sh = 16; sh > 0; sh >>= 1) {
                            const int32_t ob = __shfl_xor_sync(HP_FULL_MASK, lb, sh);
                            const int32_t oc = __shfl_xor_sync(HP_FULL_MASK, lbc, sh);
                            if (ob >= 0 && (lb < 0 || oc > lbc || (oc == lbc && ob < lb))) { lb = ob; lbc = oc; }
                        }
                        if (lane == src) { pc = lpc; bc = lbc; b = lb; }
                    }
                    if (cand) {
                        int64_t g = 0;
                        bool ok = true;
                        if (b >= 0) g = bc - pc;
                        else if (nu == 0) ok = false;
                        else { b = a.und[v % nu]; g = -pc; }
                        if (ok) { d = b; kk = p * 64 + hp::gain_bucket((int32_t)g, a.vwgt[v]); }
                    }
                } else if (cand) {
                    const int32_t pc = row_conn(a.gpart + o, a.gconn + o, len, p, k);
                    kk = p * 64 + hp::gain_bucket(-pc, a.vwgt[v]);
                }
                if (in) a.dest[v] = d;
                int tot;
                const int ex = hp::block_excl_scan<SL_THREADS>(kk >= 0 ? 1 : 0, &tot, s_scan);
                if (kk >= 0) {
                    a.K[cnt + ex] = kk;
                    a.V[cnt + ex] = v;
                }
                cnt += tot;
            }
            const bool flip = hp::block_sort_pairs<SL_THREADS>(a.K, a.V, a.K2, a.V2, cnt, a.key_bits, sl_dyn, s_scan);
            const int32_t *Ks = flip ? a.K2 : a.K, *Vs = flip ? a.V2 : a.V;
            // prefix weights in sorted order and the part bounds
            int32_t run = 0;
            for (int32_t b0 = 0; b0 < cnt; b0 += SL_THREADS) {
                const int32_t i = b0 + tid;
                const bool valid = i < cnt;
                const int32_t w = valid ? a.vwgt[Vs[i]] : 0;
                int tot;
                const int ex = hp::block_excl_scan<SL_THREADS>(w, &tot, s_scan);
                if (valid) {
                    a.pre[i] = run + ex;
                    const int32_t p = Ks[i] >> 6;
                    if (i == 0 || (Ks[i - 1] >> 6) != p) a.pstart[p] = i;
                    if (i == cnt - 1 || (Ks[i + 1] >> 6) != p) a.pend[p] = i + 1;
                }
                run += tot;
            }
            if (tid == 0) a.pre[cnt] = run;
            __syncthreads();
            if (!strong) {
                int32_t mv = 0;
                for (int32_t b0 = 0; b0 < cnt; b0 += SL_THREADS) {
                    const int32_t i = b0 + tid;
                    int sel = 0;
                    if (i < cnt) {
                        const int32_t p = Ks[i] >> 6;
                        const int64_t before = (int64_t)a.pre[i] - a.pre[a.pstart[p]];
                        sel = before < (int64_t)a.pw[p] - a.maxp[p];
                    }
                    int tot;
                    const int ex = hp::block_excl_scan<SL_THREADS>(sel, &tot, s_scan);
                    if (sel) a.moves[mv + ex] = Vs[i];
                    mv += tot;
                }
                nmoves = mv;
            } else {
                for (int32_t p = tid; p < k; p += SL_THREADS) {   // evict_end_kernel
                    const int32_t st = a.pstart[p], en = a.pend[p];
                    if (st < 0) { a.ev_end[p] = -1; continue; }
                    const int64_t need = (int64_t)a.pw[p] - a.maxp[p];
                    int32_t lo = st, hi = en;
                    while (lo + 1 < hi) {
                        const int32_t mid = (lo + hi) / 2;
                        if ((int64_t)a.pre[mid] - a.pre[st] >= need) hi = mid; else lo = mid;
                    }
                    a.ev_end[p] = hi;
                }
                __syncthreads();
                int32_t np = 0, wrun = 0;   // rs_evict_kernel
                for (int32_t b0 = 0; b0 < cnt; b0 += SL_THREADS) {
                    const int32_t i = b0 + tid;
                    const int f = i < cnt && i < a.ev_end[Ks[i] >> 6];
                    const int32_t w = f ? a.vwgt[Vs[i]] : 0;
                    int tc, tw;
                    const int ec = hp::block_excl_scan<SL_THREADS>(f, &tc, s_scan);
                    const int ew = hp::block_excl_scan<SL_THREADS>(w, &tw, s_scan);
                    if (f) {
                        a.P[np + ec] = i;
                        a.sp[np + ec] = wrun + ew;
                    }
                    np += tc;
                    wrun += tw;
                }
                // cookie cutter on the prefix weights staged in shared memory
                for (int32_t i = tid; i < np; i += SL_THREADS) sl_dyn[i] = a.sp[i];
                if (tid == 0) {
                    sl_dyn[np] = wrun;
                    a.sp[np] = wrun;
                }
                __syncthreads();
                if (wid == 0) cookie_cut_warp(k, a.pw, a.maxp, sl_dyn, np, a.es, a.ee);
                __syncthreads();
                int32_t mv = 0;   // rs_assign_kernel
                for (int32_t b0 = 0; b0 < np; b0 += SL_THREADS) {
                    const int32_t j = b0 + tid;
                    int sel = 0;
                    int32_t v = 0;
                    if (j < np) {
                        int32_t lo = 0, hi = k - 1;   // last part with es[p] <= j
                        while (lo < hi) {
                            const int32_t mid = (lo + hi + 1) / 2;
                            if (a.es[mid] <= j) lo = mid; else hi = mid - 1;
                        }
                        v = Vs[a.P[j]];
                        if (j < a.ee[lo] && lo != a.where[v]) {
                            a.dest[v] = lo;
                            sel = 1;
                        }
                    }
                    int tot;
                    const int ex = hp::block_excl_scan<SL_THREADS>(sel, &tot, s_scan);
                    if (sel) a.moves[mv + ex] = v;
                    mv += tot;
                }
                nmoves = mv;
            }
        }
        __syncthreads();
        // ---- apply: cut change before, moves, gain-row maintenance, cut change after
        long long acc = 0;
        for (int32_t i = tid; i < nmoves; i += SL_THREADS) {
            const int32_t v = a.moves[i];
            const int32_t o = a.goff[v], len = a.goff[v + 1] - o;
            const int32_t from = a.where[v], to = a.dest[v];
            a.oldp[i] = from;
            acc += (long long)row_conn(a.gpart + o, a.gconn + o, len, to, k) -
                   row_conn(a.gpart + o, a.gconn + o, len, from, k);
        }
        const long long c1 = sl_sum64(acc, s_red);
        apply_moves_rows(wid, SL_WARPS, a.moves, nmoves, a.where, a.dest, a.vwgt, a.pw, a.xadj, a.adjncy, a.adjwgt,
                         a.goff, a.gconn, a.dirty, a.small_l, a.big_l, s_lists, k, nullptr, nullptr, a.bigd, INT_MAX);
        __syncthreads();
        const int32_t ns = s_lists[0], nb = s_lists[1];
        if (ns > 0) {
            if (a.small_max <= 8)
                gain_seg_rows<8>(wid, SL_WARPS, a.small_l, ns, a.xadj, a.adjncy, a.adjwgt, a.where, a.goff, a.gpart,
                                 a.gconn, k, a.dirty);
            else if (a.small_max <= 16)
                gain_seg_rows<16>(wid, SL_WARPS, a.small_l, ns, a.xadj, a.adjncy, a.adjwgt, a.where, a.goff, a.gpart,
                                  a.gconn, k, a.dirty);
            else
                gain_seg_rows<32>(wid, SL_WARPS, a.small_l, ns, a.xadj, a.adjncy, a.adjwgt, a.where, a.goff, a.gpart,
                                  a.gconn, k, a.dirty);
        }
        if (nb > 0) {
            const int nw = (k + 31) >> 5;
            int32_t *dw = sl_dyn + (size_t)wid * (k + nw);
            unsigned *bm = (unsigned *)(dw + k);
            for (int i = lane; i < k; i += 32) dw[i] = 0;
            for (int i = lane; i < nw; i += 32) bm[i] = 0u;
            __syncwarp();
            gain_bigwarp_rows(wid, SL_WARPS, dw, bm, a.big_l, nb, a.xadj, a.adjncy, a.adjwgt, a.where, a.goff,
                              a.gpart, a.gconn, k, a.dirty, a.bigd, INT_MAX);
        }
        __syncthreads();
        acc = 0;
        for (int32_t i = tid; i < nmoves; i += SL_THREADS) {
            const int32_t v = a.moves[i];
            const int32_t o = a.goff[v], len = a.goff[v + 1] - o;
            const int32_t from = a.oldp[i], to = a.where[v];
            acc += (long long)row_conn(a.gpart + o, a.gconn + o, len, to, k) -
                   row_conn(a.gpart + o, a.gconn + o, len, from, k);
        }
        const long long c2 = sl_sum64(acc, s_red);
        long long m = LLONG_MIN;
        for (int32_t p = tid; p < k; p += SL_THREADS) {
            const long long e = (long long)a.pw[p] - a.maxp[p];
            m = e > m ? e : m;
        }
        m = sl_max64(m, s_red);
        if (tid == 0) {
            // the judge's sum over the learned moves is the applied pass's exact change
            if (judged && jl2 != c1 + c2) atomicOr(a.status, HP_STATUS_OVERFLOW);
            ctl_advance(s, m, c1, c2, nmoves, ncand, jp2);
        }
        __syncthreads();
        if (*(volatile const int32_t *)&s->take) {
            for (int32_t i = tid; i < n; i += SL_THREADS) a.best_where[i] = a.where[i];
            for (int32_t i = tid; i < k; i += SL_THREADS) a.best_pw[i] = a.pw[i];
        }
        __syncthreads();
    }
    if (!*(volatile const int32_t *)&s->best_current)
        for (int32_t i = tid; i < n; i += SL_THREADS) a.where[i] = a.best_where[i];
}

// Graph-capture helper: records the launches of body() into `graph`.  The capture
// is always ended, also when body() fails.
template <class F>
int capture_into(hp_context *c, cudaGraph_t graph, F &&body)
{
    HP_CUDA(cudaStreamBeginCaptureToGraph(c->stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    // event records cannot sit in conditional bodies: the kernel-class profiler
    // skips the captured launches (eager calls time them)
    c->prof_suspended = true;
    const int rc = body();
    c->prof_suspended = false;
    cudaGraph_t out = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &out);
    if (rc != HP_OK) {
        cudaGetLastError();
        return rc;
    }
    if (e != cudaSuccess) {
        fprintf(stderr, "hp: graph capture failed: %s\n", cudaGetErrorString(e));
        return HP_ERR_CUDA;
    }
    return HP_OK;
}

struct GraphHold {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    ~GraphHold()
    {
        if (x) cudaGraphExecDestroy(x);
        if (g) cudaGraphDestroy(g);
    }
};

// The pass graphs of one uncoarsening.  Destroying a graph that is still
// running waits for it, so they go to the context's reaper thread, which
// releases them once the stream has passed their launches (also on error paths).
struct GraphKeep {
    hp_context *c = nullptr;
    std::vector<std::pair<cudaGraph_t, cudaGraphExec_t>> items;
    ~GraphKeep() { hp_graph_retire(c, std::move(items)); }
};

// The level's pass loop as one CUDA graph:
//   WHILE (cont) { ctl_begin; SWITCH (mode) { LP | weak | strong }; apply; pass_end }
// pass_end sets the WHILE condition, ctl_begin the SWITCH value; nothing returns to
// the host between passes.  Launch accounting: kernels per body x passes per mode,
// read back from the control block.
// host milliseconds per step of run_passes_graph (HP_DEBUG_LEVELS diagnostics):
// create+handles, body capture, mode captures, instantiate, launch, destroy
double g_graph_host_ms[6];

int run_passes_graph(hp_context *c, HpLevel &g, RefineBufs &B, const PassCfg &P, bool both_lp, int *n_common,
                     int n_mode[3], GraphKeep *keep)
{
    using clk = std::chrono::steady_clock;
    auto tick = [](clk::time_point &t, int slot) {
        const auto now = clk::now();
        g_graph_host_ms[slot] += std::chrono::duration<double, std::milli>(now - t).count();
        t = now;
    };
    auto t = clk::now();
    GraphHold H;
    HP_CUDA(cudaGraphCreate(&H.g, 0));
    cudaGraphConditionalHandle hloop;
    HP_CUDA(cudaGraphConditionalHandleCreate(&hloop, H.g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hloop;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    HP_CUDA(cudaGraphAddNode(&wnode, H.g, nullptr, 0, &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    cudaGraphConditionalHandle hmode;
    HP_CUDA(cudaGraphConditionalHandleCreate(&hmode, body, 0, 0));
    cudaGraph_t mode_body[3] = {nullptr, nullptr, nullptr};
    tick(t, 0);
    const int l0 = c->launches;
    HP_TRY(capture_into(c, body, [&]() -> int {
        HP_LAUNCH(c, ctl_begin_kernel, 1, 1024, 0, P.ctl, c->d_scal, hmode, 1, P.k, B.pw, B.maxp, B.und, B.ufl);
        cudaStreamCaptureStatus cs;
        cudaGraph_t capg = nullptr;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        HP_CUDA(cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &capg, &deps, &ndeps));
        cudaGraphNodeParams sp = {};
        sp.type = cudaGraphNodeTypeConditional;
        sp.conditional.handle = hmode;
        sp.conditional.type = cudaGraphCondTypeSwitch;
        sp.conditional.size = 3;
        cudaGraphNode_t snode;
        HP_CUDA(cudaGraphAddNode(&snode, capg, deps, ndeps, &sp));
        for (int i = 0; i < 3; i++) mode_body[i] = sp.conditional.phGraph_out[i];
        HP_CUDA(cudaStreamUpdateCaptureDependencies(c->stream, &snode, 1, cudaStreamSetCaptureDependencies));
        return pass_apply(c, g, B, P, hloop, 1);
    }));
    *n_common = c->launches - l0;
    tick(t, 1);
    for (int m = 0; m < 3; m++) {
        const int l1 = c->launches;
        HP_TRY(capture_into(c, mode_body[m], [&]() -> int { return pass_propose(c, g, B, P, m, false, both_lp); }));
        n_mode[m] = c->launches - l1;
    }
    c->launches = l0;
    tick(t, 2);
    HP_CUDA(cudaGraphInstantiate(&H.x, H.g, 0));
    tick(t, 3);
    HP_CUDA(cudaGraphLaunch(H.x, c->stream));
    tick(t, 4);
    keep->items.emplace_back(H.g, H.x);   // released after the stream has finished
    H.g = nullptr;
    H.x = nullptr;
    tick(t, 5);
    return HP_OK;
}

// Enqueues the refinement of one level; nothing is read back unless the eager
// loop, the kernel-class profiler or the move log needs it.  The level's control
// block (ctl) holds its cuts and pass count when the stream reaches the end.
// CUDA-graph pass loop unless the caller asked for eager launches, the move log
// or the per-pass debug log is on, or the stream is the legacy one.
bool graph_loop(const hp_context *c)
{
    const bool recording = c->opt.learned == 2 && c->log_x != nullptr;
    return !c->opt.eager && c->tune.graph_passes && !recording && getenv("HP_DEBUG_PASSES") == nullptr &&
           c->opt.refine_patience >= 0 &&
           c->stream != nullptr && c->stream != cudaStreamLegacy;
}

// Kernels per pass body of a graphed level (for the launch count, resolved
// with the control block's pass counts once the stream has finished).
struct LevelLaunches {
    bool graph = false;
    int n_common = 0, n_mode[3] = {0, 0, 0};
    int gain_tok = -1;   // profiler interval of the level's gain build (bytes completed at the end)
};

int refine_level(hp_context *c, HpLevel &g, int32_t k, bool finest, const int64_t *d_opt,
                 const int64_t *d_maxp, const LevelStat &ls, RefineCtl *ctl, const RefineCtl *coarser,
                 LevelLaunches *ll, GraphKeep *keep)
{
    const int32_t n = g.n;
    if (n == 0) return HP_OK;
    const size_t mark = c->hi;
    RefineBufs B{};
    B.opt = d_opt;
    B.maxp = d_maxp;
    int32_t **n_arrays[] = {&B.goff, &B.big, &B.dest, &B.pregain, &B.moves, &B.oldp, &B.dirty,
                            &B.small_l, &B.big_l, &B.best_where, &B.K, &B.V, &B.K2, &B.V2, &B.pre,
                            &B.P, &B.sp, &B.huge_mv, &B.huge, &B.recof};
    for (auto pp : n_arrays) *pp = ralloc_t<int32_t>(c, (int64_t)n + 1);
    int32_t **k_arrays[] = {&B.pstart, &B.pend, &B.und, &B.ev_end, &B.es, &B.ee};
    for (auto pp : k_arrays) *pp = ralloc_t<int32_t>(c, k);
    B.lock = ralloc_t<int8_t>(c, n);
    B.prune = ralloc_t<int8_t>(c, n);
    B.accp = ralloc_t<int8_t>(c, n);
    B.jlist = ralloc_t<int32_t>(c, (int64_t)n + 1);
    B.joff = ralloc_t<int32_t>(c, (int64_t)n + 2);
    B.ufl = ralloc_t<int8_t>(c, k);
    B.pw = ralloc_t<unsigned long long>(c, k);
    unsigned long long *best_pw = ralloc_t<unsigned long long>(c, k);
    // at most m / (t + 1) rows are longer than t: the long-row lists of the
    // afterburner (t = chunk_deg) and of the moves (t = apply_chunk_deg) share
    // the chunk-plan buffers
    const int32_t huged = c->tune.gain_hub_deg, chunkd = c->tune.chunk_deg, mchunkd = c->tune.apply_chunk_deg;
    const int64_t nhub_cap =
        std::min<int64_t>((int64_t)n, g.m / ((int64_t)std::min(chunkd, mchunkd) + 1)) + 1;
    if (2 * (nhub_cap / PLAN_TILE + 1) > c->lb_cap) return HP_ERR_INTERNAL;
    B.nhub_cap = nhub_cap;
    B.ab_acc = ralloc_t<unsigned long long>(c, nhub_cap);
    B.ab_acc2 = ralloc_t<unsigned long long>(c, nhub_cap);
    // at most m / (huged + 1) rows are longer than huged
    B.hub = ralloc_t<int32_t>(c, std::min<int64_t>((int64_t)n, g.m / ((int64_t)huged + 1)) + 1);
    B.plan_v = ralloc_t<int32_t>(c, nhub_cap);
    B.plan_item = ralloc_t<int32_t>(c, nhub_cap);
    B.plan_off = ralloc_t<int32_t>(c, nhub_cap);
    B.plan_cnt = ralloc_t<int32_t>(c, 2);
    HP_CHECK_OOM(c);
    // learned LP proposals (opt.learned = 1, or 3 with the plain refiner as the
    // judge of every learned pass) until a learned pass fails to
    // improve the exact cut; then the plain rule for the rest of the level
    const bool learned = (c->opt.learned == 1 || c->opt.learned == 3) && c->mlp_ready && c->learned_skewed;
    const bool judged = learned && c->opt.learned == 3;
    const bool recording = c->opt.learned == 2 && c->log_x != nullptr;
    const int patience = c->opt.refine_patience;
    const bool dbg = getenv("HP_DEBUG_PASSES") != nullptr;
    // small levels: the whole pass loop in one CTA (same rule, same result), in
    // either loop mode unless the per-pass move log or pass log is on
    const int32_t small_n = c->tune.small_level_n;
    const bool small_level = !recording && !dbg && n <= small_n && k <= HP_TUNE_WARP_DENSE_K_MAX &&
                             g.m <= 16 * (int64_t)small_n;
    if (small_level) {
        // the level's setup (gain rows, part weights, cut, control block) runs
        // inside the kernel: no launch per setup step
        B.gpart = ralloc_t<int32_t>(c, std::max<int64_t>(g.m, 1));
        B.gconn = ralloc_t<int32_t>(c, std::max<int64_t>(g.m, 1));
        B.small_max = ls.small_max;
        HP_CHECK_OOM(c);
        SmallLevel a{};
        a.n = n;
        a.k = k;
        a.finest = finest ? 1 : 0;
        a.bigd = c->tune.gain_thread_deg;
        a.small_max = B.small_max;
        a.key_bits = key_bits_for(k);
        a.learned_mlp = learned ? 1 : 0;
        a.patience = patience;
        a.judge = judged ? 1 : 0;
        a.coarser = coarser;
        a.mlp_threshold = c->mlp_threshold;
        a.xadj = g.xadj;
        a.adjncy = g.adjncy;
        a.adjwgt = g.adjwgt;
        a.vwgt = g.vwgt;
        a.where = g.where;
        a.goff = B.goff;
        a.gpart = B.gpart;
        a.gconn = B.gconn;
        a.dest = B.dest;
        a.pregain = B.pregain;
        a.moves = B.moves;
        a.oldp = B.oldp;
        a.dirty = B.dirty;
        a.small_l = B.small_l;
        a.big_l = B.big_l;
        a.best_where = B.best_where;
        a.K = B.K;
        a.V = B.V;
        a.K2 = B.K2;
        a.V2 = B.V2;
        a.pre = B.pre;
        a.P = B.P;
        a.sp = B.sp;
        a.pstart = B.pstart;
        a.pend = B.pend;
        a.und = B.und;
        a.ev_end = B.ev_end;
        a.es = B.es;
        a.ee = B.ee;
        a.lock = B.lock;
        a.prune = B.prune;
        a.accp = B.accp;
        a.status = c->d_status;
        a.pw = B.pw;
        a.best_pw = best_pw;
        a.opt = B.opt;
        a.maxp = B.maxp;
        a.mlp_params = c->mlp_params;
        a.ctl = ctl;
        HP_LAUNCH(c, refine_small_kernel, 1, SL_THREADS, small_level_smem(n, k), a);
        c->hi = mark;
        return HP_OK;
    }
    unsigned long long *sc = c->d_scal;
    HP_CUDA(cudaMemsetAsync(sc, 0, sizeof(unsigned long long) * (S_DONE + 1), c->stream));
    int32_t *d_bigcnt = (int32_t *)&sc[S_BIGCNT];
    HP_LAUNCH(c, gain_cap_kernel, nblk(n), 256, 0, n, g.xadj, k, B.goff, B.big, B.huge, B.hub, d_bigcnt,
              c->tune.gain_thread_deg, chunkd, huged);
    if (ls.maxdeg > chunkd) {
        HP_CUDA(cudaMemsetAsync(B.ab_acc, 0, sizeof(unsigned long long) * (size_t)nhub_cap, c->stream));
        HP_CUDA(cudaMemsetAsync(B.ab_acc2, 0, sizeof(unsigned long long) * (size_t)nhub_cap, c->stream));
    }
    HP_TRY(hp_scan_excl(c, B.goff, B.goff, n));
    // the gain rows take G = sum min(deg, k) <= m entries: allocated for m, so
    // that no count is read back (the gain-build class completes its byte
    // count with G from the control block at the end of uncoarsening)
    B.small_max = ls.small_max;
    B.huge_rows = ls.maxdeg > huged;
    B.gpart = ralloc_t<int32_t>(c, std::max<int64_t>(g.m, 1));
    B.gconn = ralloc_t<int32_t>(c, std::max<int64_t>(g.m, 1));
    HP_CHECK_OOM(c);
    const bool any_big = ls.nbig > 0;
    int tok = hp_prof_begin(c);
    HP_TRY(build_rows(c, g, B, k, nullptr, nullptr, B.big, d_bigcnt, any_big, nullptr, B.hub, d_bigcnt + 4));
    // xadj, adjncy, adjwgt, where (own), goff in; gain rows (8 G) out
    hp_prof_end(c, tok, HP_PROF_GAIN, 4 * ((int64_t)n + 1) + 8 * g.m + 4 * (int64_t)n + 4 * ((int64_t)n + 1));
    ll->gain_tok = tok;
    HP_CUDA(cudaMemsetAsync(B.pw, 0, sizeof(unsigned long long) * (size_t)k, c->stream));
    HP_CUDA(cudaMemsetAsync(B.lock, 0, (size_t)n, c->stream));
    HP_CUDA(cudaMemsetAsync(B.dirty, 0, sizeof(int32_t) * (size_t)n, c->stream));
    HP_LAUNCH(c, pw_kernel, (unsigned)std::min<int64_t>(nblk(n), c->sm_count * 8), 256,
              k <= 2048 ? sizeof(unsigned long long) * k : 0, n, g.where, g.vwgt, B.pw, k);
    if (!coarser)   // the coarsest level; the others start from the coarser level's best cut
        HP_LAUNCH(c, rowcut_kernel, nblk(n), 256, 0, n, B.goff, B.gpart, B.gconn, g.where, &sc[S_CUT2]);
    HP_LAUNCH(c, excess_kernel, 1, 1024, 0, k, B.pw, B.maxp, (long long *)&sc[S_EXCESS]);
    HP_CUDA(cudaMemcpyAsync(B.best_where, g.where, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, c->stream));
    HP_CUDA(cudaMemcpyAsync(best_pw, B.pw, sizeof(unsigned long long) * k, cudaMemcpyDeviceToDevice, c->stream));

    HP_LAUNCH(c, ctl_init_kernel, 1, 1, 0, ctl, (const unsigned long long *)sc, patience, learned ? 1 : 0,
              (const int32_t *)(B.goff + n), coarser, judged ? 1 : 0);
    int64_t log_r0 = 0;
    if (recording) {
        unsigned long long lc = 0;
        HP_TRY(hp_read_scalars(c, c->log_count, sizeof(lc), &lc));
        log_r0 = (int64_t)std::min<unsigned long long>(lc, (unsigned long long)c->log_cap);
    }
    PassCfg P{k, finest, any_big, recording, ls.maxdeg > chunkd, judged, ls.maxdeg > mchunkd, ctl, best_pw};
    const bool use_graph = graph_loop(c);
    RefineCtl h{};
    if (use_graph) {
        ll->graph = true;
        HP_TRY(run_passes_graph(c, g, B, P, learned, &ll->n_common, ll->n_mode, keep));
        HP_LAUNCH(c, restore_best_kernel, std::min<unsigned>(nblk(n), (unsigned)(c->sm_count * 4)), 256, 0, ctl, n,
                  B.best_where, g.where);
    } else {
        HP_TRY(hp_read_scalars(c, ctl, sizeof(h), &h));
        while (h.cont) {
            HP_LAUNCH(c, ctl_begin_kernel, 1, 1024, 0, ctl, sc, cudaGraphConditionalHandle{}, 0, k, B.pw, B.maxp,
                      B.und, B.ufl);
            HP_TRY(pass_propose(c, g, B, P, h.mode, h.learned_pass != 0, false));
            HP_TRY(pass_apply(c, g, B, P, 0, 0));
            HP_TRY(hp_read_scalars(c, ctl, sizeof(h), &h));
            if (dbg)
                fprintf(stderr, "gpu pass n=%d pass=%d mode=%d moves=%lld cut=%lld excess=%lld\n", n,
                        h.passes - (h.cont ? 1 : 0), h.last_mode, h.last_moves, h.cut, h.excess);
        }
        HP_LAUNCH(c, restore_best_kernel, std::min<unsigned>(nblk(n), (unsigned)(c->sm_count * 4)), 256, 0, ctl, n,
                  B.best_where, g.where);
    }
    if (recording) {
        unsigned long long lc = 0;
        HP_TRY(hp_read_scalars(c, c->log_count, sizeof(lc), &lc));
        const int64_t r1 = (int64_t)std::min<unsigned long long>(lc, (unsigned long long)c->log_cap);
        if (r1 > log_r0)
            HP_LAUNCH(c, log_label_kernel, nblk(r1 - log_r0), 256, 0, log_r0, r1, g.where, c->log_v, c->log_d,
                      c->log_acc, c->log_y);
    }
    c->hi = mark;
    return HP_OK;
}

}  // namespace

int hp_refine_init()
{
    HP_CUDA(cudaFuncSetAttribute(cookie_cutter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(int32_t) * COOKIE_SMEM_INTS)));
    const int bytes = HP_MAX_PARTS * 4 + (HP_MAX_PARTS / 32) * 4;
    HP_CUDA(cudaFuncSetAttribute(gain_dense_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    HP_CUDA(cudaFuncSetAttribute(refine_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)small_level_smem(HP_TUNE_SMALL_LEVEL_MAX, HP_TUNE_WARP_DENSE_K_MAX)));
    return HP_OK;
}

int hp_uncoarsen(hp_context *c, int32_t nparts, const int64_t *h_opt, const int64_t *h_maxp)
{
    const int L = (int)c->levels.size() - 1;
    int64_t *d_opt = lalloc_t<int64_t>(c, nparts);
    int64_t *d_maxp = lalloc_t<int64_t>(c, nparts);
    LevelStat *d_ls = lalloc_t<LevelStat>(c, L + 1);
    RefineCtl *d_ctl = lalloc_t<RefineCtl>(c, L + 1);
    HP_CHECK_OOM(c);
    HP_CUDA(cudaMemcpyAsync(d_opt, h_opt, sizeof(int64_t) * nparts, cudaMemcpyHostToDevice, c->stream));
    HP_CUDA(cudaMemcpyAsync(d_maxp, h_maxp, sizeof(int64_t) * nparts, cudaMemcpyHostToDevice, c->stream));
    // every level's degree statistics in one read: afterwards the levels are
    // enqueued without waiting, so the host builds level l-1's pass graph while
    // the device runs level l
    HP_CUDA(cudaMemsetAsync(d_ls, 0, sizeof(LevelStat) * (size_t)(L + 1), c->stream));
    HP_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(RefineCtl) * (size_t)(L + 1), c->stream));
    for (int l = 0; l <= L; l++)
        if (c->levels[l].n > 0)
            HP_LAUNCH(c, level_stats_kernel, std::min<unsigned>(nblk(c->levels[l].n), (unsigned)(c->sm_count * 8)),
                      256, 0, c->levels[l].n, c->levels[l].xadj, d_ls + l, c->tune.gain_thread_deg);
    std::vector<LevelStat> ls(L + 1);
    HP_CUDA(cudaMemcpyAsync(ls.data(), d_ls, sizeof(LevelStat) * (size_t)(L + 1), cudaMemcpyDeviceToHost,
                            c->stream));
    HP_CUDA(cudaStreamSynchronize(c->stream));
    // The learned move proposals run on inputs whose degree distribution is as
    // skewed as the power-law graphs the network was trained for and validated on
    // (largest degree at least HP_LEARNED_SKEW times the mean degree; R-MAT scale
    // 22: 10^4; the 3-D grid and the RGG: 1-3); on the others the plain refiner
    // runs, as it would after a hand-over.
    {
        const HpLevel &g0 = c->levels[0];
        const int64_t mean0 = std::max<int64_t>(1, g0.m / std::max<int64_t>(1, g0.n));
        c->learned_skewed = (int64_t)ls[0].maxdeg >= HP_LEARNED_SKEW * mean0;
    }
    std::vector<LevelLaunches> ll(L + 1);
    GraphKeep keep;
    keep.c = c;
    const bool trace = c->opt.trace != 0;
    // HP_DEBUG_LEVELS: per-level size, passes, device time, host enqueue time and
    // whether the device had gone idle before the level was enqueued (stderr,
    // printed after the last level so that nothing is serialised)
    const bool dbg_levels = getenv("HP_DEBUG_LEVELS") != nullptr;
    std::vector<cudaEvent_t> lev;
    std::vector<double> host_ms(L + 1, 0.0);
    std::vector<int> idle(L + 1, 0);
    if (dbg_levels) {
        lev.resize(2 * (L + 1));
        for (auto &e : lev) HP_CUDA(cudaEventCreate(&e));
    }
    for (int l = L; l >= 0; l--) {
        HpLevel &g = c->levels[l];
        const auto t0 = std::chrono::steady_clock::now();
        if (dbg_levels) {
            idle[l] = cudaStreamQuery(c->stream) == cudaSuccess;
            HP_CUDA(cudaEventRecord(lev[2 * l], c->stream));
        }
        if (l < L)
            HP_LAUNCH(c, project_kernel, nblk(g.n), 256, 0, g.n, g.cmap, c->levels[l + 1].where, g.where);
        if (trace) {
            g.where_start = lalloc_t<int32_t>(c, g.n);
            g.where_final = lalloc_t<int32_t>(c, g.n);
            HP_CHECK_OOM(c);
            HP_CUDA(cudaMemcpyAsync(g.where_start, g.where, sizeof(int32_t) * g.n, cudaMemcpyDeviceToDevice, c->stream));
        }
        HP_TRY(refine_level(c, g, nparts, l == 0, d_opt, d_maxp, ls[l], d_ctl + l,
                            l < L && c->levels[l + 1].n > 0 ? d_ctl + l + 1 : nullptr, &ll[l], &keep));
        if (dbg_levels) {
            HP_CUDA(cudaEventRecord(lev[2 * l + 1], c->stream));
            host_ms[l] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
        if (trace)
            HP_CUDA(cudaMemcpyAsync(g.where_final, g.where, sizeof(int32_t) * g.n, cudaMemcpyDeviceToDevice, c->stream));
    }
    // results of every level: cuts and pass counts from the control blocks
    std::vector<RefineCtl> hc(L + 1);
    HP_CUDA(cudaMemcpyAsync(hc.data(), d_ctl, sizeof(RefineCtl) * (size_t)(L + 1), cudaMemcpyDeviceToHost,
                            c->stream));
    HP_CUDA(cudaStreamSynchronize(c->stream));
    if (dbg_levels) {
        for (int l = L; l >= 0; l--) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, lev[2 * l], lev[2 * l + 1]);
            fprintf(stderr, "gpu level %d n=%d m=%lld passes=%d ms=%.3f host_ms=%.3f idle_before=%d\n", l,
                    c->levels[l].n, (long long)c->levels[l].m, hc[l].passes, ms, host_ms[l], idle[l]);
        }
        for (auto e : lev) cudaEventDestroy(e);
        fprintf(stderr, "graph host ms: create %.3f body %.3f modes %.3f instantiate %.3f launch %.3f destroy %.3f\n",
                g_graph_host_ms[0], g_graph_host_ms[1], g_graph_host_ms[2], g_graph_host_ms[3], g_graph_host_ms[4],
                g_graph_host_ms[5]);
        for (double &x : g_graph_host_ms) x = 0.0;
    }
    int total_passes = 0;
    for (int l = 0; l <= L; l++) {
        HpLevel &g = c->levels[l];
        g.cut_start = g.n > 0 ? hc[l].cut_start : 0;
        g.cut_final = g.n > 0 ? hc[l].best_cut : 0;
        total_passes += hc[l].passes;
        hp_prof_add_bytes(c, ll[l].gain_tok, 8 * (int64_t)hc[l].gain_entries);
        if (ll[l].graph)   // the graph's own launch + its kernels per pass
            c->launches += 1 + hc[l].passes * ll[l].n_common + hc[l].mode_passes[0] * ll[l].n_mode[0] +
                           hc[l].mode_passes[1] * ll[l].n_mode[1] + hc[l].mode_passes[2] * ll[l].n_mode[2];
    }
    c->stats.refine_passes = total_passes;
    return hp_check_status(c);
}
