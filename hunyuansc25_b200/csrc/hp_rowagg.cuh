// hp_rowagg.cuh — "aggregate a row": gather (key, weight) entries, merge equal
// keys by summing weights, drop an excluded key, and write the unique keys in
// ascending order.  Used by contraction (key = coarse neighbour id, the self
// key dropped) and by the gain table (key = neighbour's part).
//
// Size classes (chosen per row by its entry count):
//   S   <= 32     one warp, register bitonic sort over the 32 lanes (shuffles)
//   B   <= CAP    one CTA, shared-memory bitonic sort (CAP = 512 or 4096)
//   D   larger    one CTA, dense accumulator + presence bitmap over the key
//                 space, scanned in key order (global scratch per CTA for
//                 contraction, shared memory for part keys)
// Every class produces the same canonical row, so the class boundaries are a
// performance choice only.
#pragma once

#include "hp_common.cuh"

namespace hp {

constexpr int32_t KEY_NONE = 0x7fffffff;

// Warp-wide aggregation of up to 32 entries already held one per lane.
// Writes unique keys/sums to out_k/out_w (if non-null) and returns the count
// (same value in all lanes).
__device__ __forceinline__ int warp_aggregate32(int32_t key, int32_t w, int32_t *out_k,
                                                int32_t *out_w)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            int32_t pk = __shfl_xor_sync(HP_FULL_MASK, key, j);
            int32_t pw = __shfl_xor_sync(HP_FULL_MASK, w, j);
            bool up = (lane & k) == 0;
            bool lower = (lane & j) == 0;
            bool take = lower ? (up ? pk < key : pk > key) : (up ? pk > key : pk < key);
            if (take) { key = pk; w = pw; }
        }
    }
    // suffix sums inside runs of equal keys
    int32_t s = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int32_t t = __shfl_down_sync(HP_FULL_MASK, s, o);
        int32_t kk = __shfl_down_sync(HP_FULL_MASK, key, o);
        if (lane + o < 32 && kk == key) s += t;
    }
    int32_t prev = __shfl_up_sync(HP_FULL_MASK, key, 1);
    bool head = key != KEY_NONE && (lane == 0 || prev != key);
    unsigned hm = __ballot_sync(HP_FULL_MASK, head);
    if (head && out_k) {
        int r = __popc(hm & lanemask_lt());
        out_k[r] = key;
        out_w[r] = s;
    }
    return __popc(hm);
}

// ---- one row per thread, in registers ---------------------------------------
// Entries are packed as key << 32 | weight (padding and dropped keys are
// KEY_NONE) and sorted ascending by a bitonic network over the first NET of XN
// registers (compile-time indices only, so the array stays in registers);
// equal keys are then merged by summing the low halves.
template <int NET, int XN>
__device__ __forceinline__ void sort_regs(unsigned long long (&x)[XN])
{
#pragma unroll
    for (int size = 2; size <= NET; size <<= 1)
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1)
#pragma unroll
            for (int i = 0; i < NET; i++) {
                const int j = i ^ stride;
                if (j > i) {
                    const unsigned long long a = x[i], b = x[j];
                    const unsigned long long lo = a < b ? a : b, hi = a < b ? b : a;
                    if ((i & size) == 0) { x[i] = lo; x[j] = hi; }
                    else { x[i] = hi; x[j] = lo; }
                }
            }
}

constexpr unsigned long long PACK_NONE = (unsigned long long)(uint32_t)KEY_NONE << 32;

// Segmented version: the warp holds 32/S independent rows of up to S entries
// (lanes [S*r, S*r+S) hold row r); each segment is sorted by its own bitonic
// network (log2 S stages), equal keys are merged, and every segment writes its
// unique keys to its own out_k/out_w.  Returns the segment's unique count.
template <int S>
__device__ __forceinline__ int seg_aggregate(int32_t key, int32_t w, int32_t *out_k, int32_t *out_w)
{
    const int lane = threadIdx.x & 31;
    const int sl = lane & (S - 1);
#pragma unroll
    for (int k = 2; k <= S; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int32_t pk = __shfl_xor_sync(HP_FULL_MASK, key, j);
            const int32_t pw = __shfl_xor_sync(HP_FULL_MASK, w, j);
            const bool up = (sl & k) == 0;
            const bool lower = (sl & j) == 0;
            const bool take = lower ? (up ? pk < key : pk > key) : (up ? pk > key : pk < key);
            if (take) { key = pk; w = pw; }
        }
    }
    int32_t s = w;
#pragma unroll
    for (int o = 1; o < S; o <<= 1) {
        const int32_t t = __shfl_down_sync(HP_FULL_MASK, s, o, S);
        const int32_t kk = __shfl_down_sync(HP_FULL_MASK, key, o, S);
        if (sl + o < S && kk == key) s += t;
    }
    const int32_t prev = __shfl_up_sync(HP_FULL_MASK, key, 1, S);
    const bool head = key != KEY_NONE && (sl == 0 || prev != key);
    const unsigned seg = S == 32 ? 0xffffffffu : (((1u << S) - 1u) << (lane & ~(S - 1)));
    const unsigned hm = __ballot_sync(HP_FULL_MASK, head) & seg;
    if (head && out_k) {
        const int r = __popc(hm & lanemask_lt());
        out_k[r] = key;
        out_w[r] = s;
    }
    return __popc(hm);
}

// Same aggregation written as a dense vector over keys [0, nkeys):
// out_k[q] = q, out_w[q] = sum of the weights with key q (0 if none).
__device__ __forceinline__ void warp_aggregate32_dense(int32_t key, int32_t w, int32_t nkeys,
                                                       int32_t *out_k, int32_t *out_w)
{
    const int lane = threadIdx.x & 31;
    for (int32_t q = lane; q < nkeys; q += 32) { out_k[q] = q; out_w[q] = 0; }
    __syncwarp();
    // duplicates of a key are summed with one atomic per entry (order-free)
    if (key != KEY_NONE) atomicAdd(&out_w[key], w);
    __syncwarp();
}

// CTA-wide shared-memory aggregation of len <= CAP entries staged in sk/sw
// (entries beyond len must already be KEY_NONE up to the pow2 size P).
template <int NT, int CAP>
__device__ __forceinline__ int block_aggregate_smem(int32_t *sk, int32_t *sw, int P,
                                                    int32_t *out_k, int32_t *out_w,
                                                    int32_t *s_scan /* NT/32 + 2 */)
{
    const int tid = threadIdx.x;
    // bitonic sort of P elements
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < P; i += NT) {
                int ixj = i ^ j;
                if (ixj > i) {
                    int32_t a = sk[i], b = sk[ixj];
                    bool up = (i & k) == 0;
                    if (up ? (a > b) : (a < b)) {
                        sk[i] = b; sk[ixj] = a;
                        int32_t t = sw[i]; sw[i] = sw[ixj]; sw[ixj] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
    // heads and their positions: thread t owns elements [t*per, (t+1)*per)
    const int per = (P + NT - 1) / NT;
    const int lo = tid * per, hiE = min(lo + per, P);
    int cnt = 0;
    for (int i = lo; i < hiE; i++)
        cnt += (sk[i] != KEY_NONE && (i == 0 || sk[i - 1] != sk[i]));
    const int lane = tid & 31, wid = tid >> 5;
    int incl = warp_incl_scan(cnt);
    if (lane == 31) s_scan[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int t = lane < NT / 32 ? s_scan[lane] : 0;
        int ti = warp_incl_scan(t);
        if (lane < NT / 32) s_scan[lane] = ti - t;
        if (lane == NT / 32 - 1) s_scan[NT / 32] = ti;
    }
    __syncthreads();
    int pos = s_scan[wid] + incl - cnt;
    const int total = s_scan[NT / 32];
    for (int i = lo; i < hiE; i++) {
        int32_t key = sk[i];
        if (key == KEY_NONE || (i > 0 && sk[i - 1] == key)) continue;
        int32_t sum = 0;
        for (int j = i; j < P && sk[j] == key; j++) sum += sw[j];
        out_k[pos] = key;
        out_w[pos] = sum;
        pos++;
    }
    __syncthreads();
    return total;
}

// CTA-wide exclusive scan of one int per thread; returns exclusive value and
// writes the block total to *total.
template <int NT>
__device__ __forceinline__ int block_excl_scan(int v, int *total, int32_t *s_scan)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = warp_incl_scan(v);
    if (lane == 31) s_scan[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int t = lane < NT / 32 ? s_scan[lane] : 0;
        int ti = warp_incl_scan(t);
        if (lane < NT / 32) s_scan[lane] = ti - t;
        if (lane == NT / 32 - 1) s_scan[NT / 32] = ti;
    }
    __syncthreads();
    int r = s_scan[wid] + incl - v;
    *total = s_scan[NT / 32];
    __syncthreads();
    return r;
}

// Dense aggregation over key space [0, nkeys): dw[nkeys] (zero on entry and on
// exit), bm[(nkeys+31)/32] presence bits (zero on entry and exit).  Entries
// must have been accumulated into dw/bm by the caller (atomics) before the
// barrier that precedes this call.  Writes keys in ascending order.
template <int NT>
__device__ __forceinline__ int dense_extract(int32_t *dw, unsigned *bm, int32_t nkeys,
                                             int32_t *out_k, int32_t *out_w, int32_t *s_scan)
{
    const int nwords = (nkeys + 31) >> 5;
    int running = 0;
    for (int wb = 0; wb < nwords; wb += NT) {
        int wi = wb + threadIdx.x;
        unsigned word = wi < nwords ? bm[wi] : 0u;
        int tot;
        int p = running + block_excl_scan<NT>(__popc(word), &tot, s_scan);
        if (word) {
            bm[wi] = 0u;
            while (word) {
                int b = __ffs(word) - 1;
                word &= word - 1;
                int32_t k = (wi << 5) + b;
                out_k[p] = k;
                out_w[p] = dw[k];
                dw[k] = 0;
                p++;
            }
        }
        running += tot;
    }
    __syncthreads();
    return running;
}

// Two-level variant for large key spaces: bm2[(nwords+31)/32] has one bit per
// non-zero word of bm (set by the accumulating thread that turned the word
// non-zero), so the extraction walks nkeys/1024 words plus the occupied bm
// words instead of all nkeys/32.  dw, bm and bm2 are zero again on exit.
__device__ __forceinline__ void dense_mark2(int32_t *dw, unsigned *bm, unsigned *bm2, int32_t k, int32_t w)
{
    atomicAdd(&dw[k], w);
    const unsigned bit = 1u << (k & 31);
    if (atomicOr(&bm[k >> 5], bit) == 0u) atomicOr(&bm2[k >> 10], 1u << ((k >> 5) & 31));
}

template <int NT>
__device__ __forceinline__ int dense_extract2(int32_t *dw, unsigned *bm, unsigned *bm2, int32_t nkeys,
                                              int32_t *out_k, int32_t *out_w, int32_t *s_scan)
{
    const int nwords = (nkeys + 31) >> 5;
    const int nw2 = (nwords + 31) >> 5;
    int running = 0;
    for (int wb = 0; wb < nw2; wb += NT) {
        const int i2 = wb + threadIdx.x;
        const unsigned top = i2 < nw2 ? bm2[i2] : 0u;
        int cnt = 0;
        for (unsigned t = top; t; t &= t - 1) cnt += __popc(bm[(i2 << 5) + __ffs(t) - 1]);
        int tot;
        int p = running + block_excl_scan<NT>(cnt, &tot, s_scan);
        if (top) {
            bm2[i2] = 0u;
            for (unsigned t = top; t; t &= t - 1) {
                const int wi = (i2 << 5) + __ffs(t) - 1;
                unsigned word = bm[wi];
                bm[wi] = 0u;
                while (word) {
                    const int b = __ffs(word) - 1;
                    word &= word - 1;
                    const int32_t k = (wi << 5) + b;
                    out_k[p] = k;
                    out_w[p] = dw[k];
                    dw[k] = 0;
                    p++;
                }
            }
        }
        running += tot;
    }
    __syncthreads();
    return running;
}


// Stable LSD radix sort of cnt (key, value) pairs by the low key_bits bits of
// the keys (non-negative), by one CTA of NT threads.  Ping-pongs between (K, V)
// and (K2, V2); returns true when the result is in (K2, V2).  Per 8-bit digit: a
// histogram, the digit bases, then chunks of NT items in order, each item placed
// at its digit's base + the same digit's count in earlier warps of the chunk +
// its rank inside its warp (__match_any_sync).  tab: block_sort_ints(NT) ints of
// shared memory; s_scan: NT/32 + 2 ints.
constexpr int block_sort_ints(int nt) { return 256 + (nt / 32) * 256; }

template <int NT>
__device__ bool block_sort_pairs(int32_t *K, int32_t *V, int32_t *K2, int32_t *V2, int32_t cnt, int key_bits,
                                 int32_t *tab, int32_t *s_scan)
{
    constexpr int W = NT / 32;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    int32_t *base = tab, *wc = tab + 256;
    bool flip = false;
    for (int shift = 0; shift < key_bits; shift += 8) {
        const int32_t *ks = flip ? K2 : K, *vs = flip ? V2 : V;
        int32_t *kd = flip ? K : K2, *vd = flip ? V : V2;
        for (int q = tid; q < 256; q += NT) base[q] = 0;
        __syncthreads();
        for (int32_t i = tid; i < cnt; i += NT) atomicAdd(&base[((unsigned)ks[i] >> shift) & 255u], 1);
        __syncthreads();
        const int h = tid < 256 ? base[tid] : 0;
        int tot;
        const int ex = block_excl_scan<NT>(h, &tot, s_scan);   // ends with a barrier
        if (tid < 256) base[tid] = ex;
        for (int32_t c0 = 0; c0 < cnt; c0 += NT) {
            const int32_t i = c0 + tid;
            const bool valid = i < cnt;
            const int32_t key = valid ? ks[i] : 0;
            const unsigned d = valid ? (((unsigned)key >> shift) & 255u) : 256u + lane;
            const unsigned peers = __match_any_sync(HP_FULL_MASK, d);
            const int rank = __popc(peers & lanemask_lt());
            for (int q = tid; q < W * 256; q += NT) wc[q] = 0;
            __syncthreads();
            if (valid && rank == 0) wc[wid * 256 + d] = __popc(peers);
            __syncthreads();
            if (valid) {
                int32_t off = base[d] + rank;
                for (int w = 0; w < wid; w++) off += wc[w * 256 + d];
                kd[off] = key;
                vd[off] = vs[i];
            }
            __syncthreads();
            if (tid < 256) {   // the digit bases move past this chunk
                int32_t c = 0;
                for (int w = 0; w < W; w++) c += wc[w * 256 + tid];
                base[tid] += c;
            }
            __syncthreads();
        }
        flip = !flip;
    }
    __syncthreads();
    return flip;
}

}  // namespace hp
