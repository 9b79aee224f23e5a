// hp_common.cuh — device helpers shared by every kernel file of the partitioner.
#pragma once

#include <cuda_runtime.h>
#include <climits>
#include <stdint.h>
#include <stdio.h>

#include "hp_partition.h"

#define HP_FULL_MASK 0xffffffffu
#define HP_INT_MAX 0x7fffffff

// Device status word bits (ctx->d_status): set by kernels, read by the host.
#define HP_STATUS_SPIN_TIMEOUT 1u   // a bounded look-back / flag wait gave up
#define HP_STATUS_BAD_GRAPH    2u   // structural validation failed
#define HP_STATUS_OVERFLOW     4u   // a capacity bound was exceeded (never expected)
#define HP_STATUS_WEIGHT_RANGE 8u   // a matched pair's weighted degrees reach 2^31 (int32 coarse weights)

// Spin limit of every device-side wait (iterations with __nanosleep back-off).
#define HP_SPIN_LIMIT (1u << 22)

namespace hp {

// First statement of every kernel of the library: when the kernel was launched
// as a programmatic dependent of the previous kernel in its stream (hp_tuning.pdl),
// it may already be resident while that kernel drains; this waits until the
// previous kernel has completed and its writes are visible.  Without such a
// launch it returns at once.
__device__ __forceinline__ void pdl_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// splitmix64 finaliser (Vigna): the matching tie-break hash.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t level_key(uint64_t seed, int32_t level)
{
    return mix64(seed ^ (0x6d61746368ULL + (uint64_t)level * 0x100000001b3ULL));
}

__host__ __device__ __forceinline__ uint32_t edge_tie(uint64_t lkey, int32_t a, int32_t b)
{
    uint32_t lo = (uint32_t)(a < b ? a : b), hi = (uint32_t)(a < b ? b : a);
    return (uint32_t)(mix64(lkey ^ (((uint64_t)lo << 32) | hi)) >> 32);
}

// Matching candidate order: heavier edge, then lower tie key, then lower id.
__host__ __device__ __forceinline__ bool better(int32_t w1, uint32_t h1, int32_t u1,
                                                int32_t w2, uint32_t h2, int32_t u2)
{
    if (w1 != w2) return w1 > w2;
    if (h1 != h2) return h1 < h2;
    return u1 < u2;
}

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ int warp_sum(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(HP_FULL_MASK, v, o);
    return v;
}

__device__ __forceinline__ long long warp_sum64(long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(HP_FULL_MASK, v, o);
    return v;
}

__device__ __forceinline__ long long warp_max64(long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        long long t = __shfl_xor_sync(HP_FULL_MASK, v, o);
        v = t > v ? t : v;
    }
    return v;
}

__device__ __forceinline__ int warp_max(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(HP_FULL_MASK, v, o));
    return v;
}

// Warp-aggregated append: every lane with pred set gets its own slot of the
// list counted by *counter, with one atomic per warp instead of one per lane
// (same-address atomics serialise in L2).  Lanes without pred get -1.  All 32
// lanes must call it.
__device__ __forceinline__ int32_t warp_append(int32_t *counter, bool pred)
{
    const unsigned m = __ballot_sync(HP_FULL_MASK, pred);
    if (m == 0u) return -1;
    const int leader = __ffs(m) - 1;
    int32_t base = 0;
    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(HP_FULL_MASK, base, leader);
    return pred ? base + __popc(m & lanemask_lt()) : -1;
}

// The row owning entry j of a CSR: the last v with xadj[v] <= j, for
// xadj[0] = 0 <= j < xadj[n].  A 32-ary search by one warp (one load per lane
// per round, about log32(n) rounds) instead of a serial binary search's
// log2(n) dependent loads.  All 32 lanes call it and get the result.
__device__ __forceinline__ int32_t warp_find_row(const int32_t *__restrict__ xadj, int32_t n, int64_t j)
{
    const int lane = threadIdx.x & 31;
    int32_t lo = 0, hi = n - 1;   // xadj[lo] <= j; the answer lies in [lo, hi]
    while (hi - lo >= 32) {
        // 32 probes covering (lo, hi]: p(0) = lo + 1, p(31) = hi
        const int64_t span = (int64_t)hi - lo;
        const int32_t p = lo + 1 + (int32_t)((span - 1) * lane / 31);
        const unsigned m = __ballot_sync(HP_FULL_MASK, xadj[p] <= j);   // a prefix of the lanes
        if (m == 0u) return lo;
        const int L = 31 - __clz(m);
        const int32_t nlo = __shfl_sync(HP_FULL_MASK, p, L);
        const int32_t nxt = __shfl_sync(HP_FULL_MASK, p, L < 31 ? L + 1 : 31);
        hi = L < 31 ? nxt - 1 : hi;
        lo = nlo;
    }
    const int32_t p = lo + 1 + lane;
    const unsigned m = __ballot_sync(HP_FULL_MASK, p <= hi && xadj[p] <= j);
    return m ? lo + 1 + (31 - __clz(m)) : lo;
}

// Owner rows of a tile of CSR entries: owner[i] = the row of entry tb + i for
// i < te - tb <= NT * ITEMS (xadj monotone, xadj[0] = 0, xadj[n] = m > tb).
// The row holding entry tb comes from warp_find_row; every later row that
// starts inside the tile marks its first entry (an empty row shares its start
// with a later row, which wins the max), and an inclusive max-scan over the
// markers gives every entry its row.  s_warp: NT/32 ints; s_v0: one int.  All
// NT threads call it; it ends with a barrier.
template <int NT, int ITEMS>
__device__ void tile_owners(const int32_t *__restrict__ xadj, int32_t n, int64_t tb, int64_t te,
                            int32_t *owner, int32_t *s_warp, int32_t *s_v0)
{
    constexpr int TILE = NT * ITEMS;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (wid == 0) {
        const int32_t v0 = warp_find_row(xadj, n, tb);
        if (lane == 0) *s_v0 = v0;
    }
    for (int i = threadIdx.x; i < TILE; i += NT) owner[i] = -1;
    __syncthreads();
    const int32_t v0 = *s_v0;
    if (threadIdx.x == 0) owner[0] = v0;
    for (int64_t v = (int64_t)v0 + 1 + threadIdx.x; v < n; v += NT) {
        const int32_t b = xadj[v];
        if (b >= te) break;
        atomicMax(&owner[b - tb], (int32_t)v);
    }
    __syncthreads();
    // inclusive max-scan: ITEMS consecutive markers per thread
    int32_t run = -1;
#pragma unroll
    for (int q = 0; q < ITEMS; q++) run = max(run, owner[threadIdx.x * ITEMS + q]);
    int32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(HP_FULL_MASK, x, o);
        if (lane >= o) x = max(x, y);
    }
    if (lane == 31) s_warp[wid] = x;
    int32_t ex = __shfl_up_sync(HP_FULL_MASK, x, 1);
    if (lane == 0) ex = -1;
    __syncthreads();
    for (int w = 0; w < wid; w++) ex = max(ex, s_warp[w]);
    __syncthreads();   // every thread has read the markers it scans
#pragma unroll
    for (int q = 0; q < ITEMS; q++) {
        const int i = threadIdx.x * ITEMS + q;
        ex = max(ex, owner[i]);
        owner[i] = ex;
    }
    __syncthreads();
}

// Inclusive warp scan.
__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(HP_FULL_MASK, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide sum into *out (atomic add of one value per block).
template <int BLOCK>
__device__ __forceinline__ void block_add_to(long long v, unsigned long long *out)
{
    __shared__ long long s_part[BLOCK / 32];
    v = warp_sum64(v);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        long long t = threadIdx.x < BLOCK / 32 ? s_part[threadIdx.x] : 0;
        t = warp_sum64(t);
        if (threadIdx.x == 0 && t != 0) atomicAdd(out, (unsigned long long)t);
    }
    // s_part is one array for every call site of this BLOCK size: a following
    // call may write it only after the first warp has read it
    __syncthreads();
}

// Decoupled look-back (single-pass scan across CTAs).  tile_status[t] holds
// flag << 32 | value: flag 1 = the tile's own aggregate, flag 2 = its inclusive
// prefix.  Called by all 32 lanes of one warp of tile `tile` with the tile's
// aggregate; publishes it, walks back over predecessors 32 at a time until an
// inclusive prefix is found, publishes its own inclusive prefix and returns the
// exclusive prefix (same value in every lane).  Tiles must be taken in launch
// order (a dynamic tile counter), so every predecessor is running or done.  Each
// wait is bounded by HP_SPIN_LIMIT; on expiry HP_STATUS_SPIN_TIMEOUT is set in
// *status and the predecessor counts as zero, so the kernel always finishes.
constexpr unsigned long long LB_FLAG_AGG = 1ull << 32;
constexpr unsigned long long LB_FLAG_PRE = 2ull << 32;

__device__ __forceinline__ int32_t lookback_exclusive(unsigned long long *tile_status, int64_t tile, int32_t agg,
                                                      unsigned *status)
{
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) atomicExch(&tile_status[0], LB_FLAG_PRE | (unsigned)agg);
        return 0;
    }
    if (lane == 0) atomicExch(&tile_status[tile], LB_FLAG_AGG | (unsigned)agg);
    int32_t excl = 0;
    int64_t pred = tile - 1;
    for (;;) {
        const int64_t idx = pred - lane;
        unsigned long long st = LB_FLAG_PRE;  // virtual prefix 0 before tile 0
        if (idx >= 0) {
            unsigned it = 0;
            for (;;) {
                st = *(volatile unsigned long long *)&tile_status[idx];
                if (st >> 32) break;
                if (++it > HP_SPIN_LIMIT) {
                    atomicOr(status, HP_STATUS_SPIN_TIMEOUT);
                    st = LB_FLAG_PRE;
                    break;
                }
                __nanosleep(32);
            }
        }
        const unsigned pre_mask = __ballot_sync(HP_FULL_MASK, (st >> 32) == 2);
        const int32_t val = (int32_t)(unsigned)(st & 0xffffffffull);
        if (pre_mask) {
            const int first = __ffs(pre_mask) - 1;
            excl += warp_sum(lane <= first ? val : 0);
            break;
        }
        excl += warp_sum(val);
        pred -= 32;
    }
    if (lane == 0) atomicExch(&tile_status[tile], LB_FLAG_PRE | (unsigned)(excl + agg));
    return excl;
}

// ---- epoch look-back (no zeroing between uses) ------------------------------------
// Single-pass kernels of a context share one tile-status region that only they
// write.  A tile word is epoch (bits 34-63) | flag (bits 32-33: 1 aggregate,
// 2 inclusive prefix) | value (bits 0-31); a word of another epoch counts as
// not yet published, so the region never needs clearing.  LbCtl holds the
// dynamic tile counter, the count of finished CTAs and the current epoch: the
// last CTA of a launch resets the first two and advances the epoch, so the next
// launch (stream order) starts clean -- also when both are replayed from a
// CUDA graph.
struct LbCtl {
    unsigned tile_counter, done, epoch, pad;
};

__device__ __forceinline__ unsigned long long lb_word(unsigned epoch, unsigned flag, int32_t v)
{
    return ((unsigned long long)(epoch & 0x3fffffffu) << 34) | ((unsigned long long)flag << 32) | (uint32_t)v;
}

// All threads of the CTA: its tile (in launch order) and the launch's epoch.
__device__ __forceinline__ void lb_begin(LbCtl *ctl, int64_t *tile, unsigned *epoch)
{
    __shared__ unsigned s_t, s_e;
    if (threadIdx.x == 0) {
        s_t = atomicAdd(&ctl->tile_counter, 1u);
        s_e = *(volatile unsigned *)&ctl->epoch;
    }
    __syncthreads();
    *tile = s_t;
    *epoch = s_e;
}

// Persistent form: a CTA reads the launch's epoch once (lb_epoch), then takes
// tiles in launch order with lb_next until it passes its last tile; a CTA only
// waits on tiles taken before its own, by running CTAs.
__device__ __forceinline__ unsigned lb_epoch(LbCtl *ctl)
{
    __shared__ unsigned s_e;
    if (threadIdx.x == 0) s_e = *(volatile unsigned *)&ctl->epoch;
    __syncthreads();
    return s_e;
}

__device__ __forceinline__ int64_t lb_next(LbCtl *ctl)
{
    __shared__ unsigned s_t;
    __syncthreads();   // every thread is done with the previous tile's shared data
    if (threadIdx.x == 0) s_t = atomicAdd(&ctl->tile_counter, 1u);
    __syncthreads();
    return s_t;
}

// All threads of the CTA, after its last write: the last CTA to finish resets
// the counters and advances the epoch.
__device__ __forceinline__ void lb_end(LbCtl *ctl)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned d = atomicAdd(&ctl->done, 1u);
        if (d == gridDim.x - 1) {
            ctl->tile_counter = 0u;
            ctl->done = 0u;
            ctl->epoch = ctl->epoch + 1u;
            __threadfence();
        }
    }
}

// lookback_exclusive over epoch-tagged words (same contract: one full warp,
// bounded waits, returns the exclusive prefix of `tile`).
__device__ __forceinline__ int32_t lookback_epoch(unsigned long long *tile_status, int64_t tile, int32_t agg,
                                                  unsigned epoch, unsigned *status)
{
    const int lane = threadIdx.x & 31;
    const unsigned long long tag = (unsigned long long)(epoch & 0x3fffffffu);
    if (tile == 0) {
        if (lane == 0) atomicExch(&tile_status[0], lb_word(epoch, 2u, agg));
        return 0;
    }
    if (lane == 0) atomicExch(&tile_status[tile], lb_word(epoch, 1u, agg));
    int32_t excl = 0;
    int64_t pred = tile - 1;
    for (;;) {
        const int64_t idx = pred - lane;
        unsigned flag = 2u;   // virtual inclusive prefix 0 before tile 0
        int32_t val = 0;
        if (idx >= 0) {
            unsigned it = 0;
            for (;;) {
                const unsigned long long st = *(volatile unsigned long long *)&tile_status[idx];
                flag = (st >> 34) == tag ? (unsigned)(st >> 32) & 3u : 0u;
                if (flag) {
                    val = (int32_t)(unsigned)(st & 0xffffffffull);
                    break;
                }
                if (++it > HP_SPIN_LIMIT) {
                    atomicOr(status, HP_STATUS_SPIN_TIMEOUT);
                    flag = 2u;
                    val = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        const unsigned pre_mask = __ballot_sync(HP_FULL_MASK, flag == 2u);
        if (pre_mask) {
            const int first = __ffs(pre_mask) - 1;
            excl += warp_sum(lane <= first ? val : 0);
            break;
        }
        excl += warp_sum(val);
        pred -= 32;
    }
    if (lane == 0) atomicExch(&tile_status[tile], lb_word(epoch, 2u, excl + agg));
    return excl;
}

__host__ __device__ __forceinline__ int64_t iabs64(int64_t x) { return x < 0 ? -x : x; }

// Weak-rebalance gain bucket with the float semantics of the reference's
// gain_bucket (hunyuangraph_GPU_krefine.h:2477-2513); explicit _rn intrinsics
// keep the device arithmetic identical to a host IEEE evaluation.  Upper clamp
// 49 (the reference can reach 50, which aliases the next part's buckets).
__device__ __forceinline__ int32_t gain_bucket(int32_t gain, int32_t vwgt)
{
    float g = __fdiv_rn((float)gain, (float)(vwgt > 0 ? vwgt : 1));
    if (g > 0.0f) return 0;
    if (g == 0.0f) return 1;
    int32_t t = 25;
    g = fabsf(g);
    if (g < 1.0f) {
        while (g < 1.0f) { g = __fmul_rn(g, 1.5f); t--; }
        if (t < 2) t = 2;
    } else {
        while (g > 1.0f) { g = __fdiv_rn(g, 1.5f); t++; }
        if (t > 49) t = 49;
    }
    return t;
}

inline unsigned div_up(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace hp

// ---- host error handling ------------------------------------------------------
#define HP_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "hp: CUDA error %s at %s:%d\n", cudaGetErrorString(e_),    \
                    __FILE__, __LINE__);                                               \
            return HP_ERR_CUDA;                                                        \
        }                                                                              \
    } while (0)

#define HP_TRY(call)                  \
    do {                              \
        int rc_ = (call);             \
        if (rc_ != HP_OK) return rc_; \
    } while (0)
