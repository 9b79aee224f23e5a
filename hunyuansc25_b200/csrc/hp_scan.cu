// hp_scan.cu — single-pass decoupled look-back scan and small device primitives.
//
// Replaces the reference's recursive reduce-then-propagate prefix sum
// (hunyuangraph_GPU_prefixsum.h:53-188), which launches three kernels per
// recursion level and ends each level with cudaDeviceSynchronize().  Here one
// launch scans the whole array: each CTA takes a dynamic tile index, publishes
// its aggregate, and the first warp looks back over predecessor tiles (32 at a
// time) until it meets an inclusive prefix.  Every wait is bounded
// (HP_SPIN_LIMIT); on expiry the CTA sets HP_STATUS_SPIN_TIMEOUT and continues,
// so a stalled predecessor can never hang the device.
#include <cstring>

#include "hp_internal.cuh"

namespace {

constexpr int SCAN_BLOCK = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;  // 4096

__device__ __forceinline__ int pad(int i) { return i + (i >> 5); }

// Exclusive scan of in[0..n) into out[0..n] (out[n] = total); element n is a
// virtual zero.  EPOCH: the context's epoch look-back region (no clearing);
// else tile_status[ntiles] and ctl->tile_counter must be zero on entry.
template <bool EPOCH>
__global__ void __launch_bounds__(SCAN_BLOCK)
scan_excl_kernel(const int32_t *__restrict__ in, int32_t *__restrict__ out, int64_t n,
                 unsigned long long *tile_status, hp::LbCtl *ctl, unsigned *status)
{
    hp::pdl_wait();
    __shared__ int32_t s[SCAN_TILE + SCAN_TILE / 32];
    __shared__ int32_t s_warp[SCAN_BLOCK / 32];
    __shared__ int32_t s_excl;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

    int64_t tile;
    unsigned epoch;
    hp::lb_begin(ctl, &tile, &epoch);
    const int64_t base = tile * SCAN_TILE;

#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        int i = k * SCAN_BLOCK + tid;
        int64_t g = base + i;
        s[pad(i)] = (g < n) ? in[g] : 0;
    }
    __syncthreads();
    int32_t v[SCAN_ITEMS];
    int32_t local = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        v[k] = s[pad(tid * SCAN_ITEMS + k)];
        local += v[k];
    }
    int32_t incl = hp::warp_incl_scan(local);
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int32_t t = lane < SCAN_BLOCK / 32 ? s_warp[lane] : 0;
        int32_t ti = hp::warp_incl_scan(t);
        if (lane < SCAN_BLOCK / 32) s_warp[lane] = ti - t;  // exclusive warp offsets
        int32_t agg = __shfl_sync(HP_FULL_MASK, ti, SCAN_BLOCK / 32 - 1);
        const int32_t excl = EPOCH ? hp::lookback_epoch(tile_status, tile, agg, epoch, status)
                                   : hp::lookback_exclusive(tile_status, tile, agg, status);
        if (lane == 0) s_excl = excl;
    }
    __syncthreads();
    int32_t run = s_excl + s_warp[wid] + incl - local;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        s[pad(tid * SCAN_ITEMS + k)] = run;
        run += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        int i = k * SCAN_BLOCK + tid;
        int64_t g = base + i;
        if (g <= n) out[g] = s[pad(i)];
    }
    if (EPOCH) hp::lb_end(ctl);
}

__global__ void fill_kernel(int32_t *p, int64_t n, int32_t value)
{
    hp::pdl_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = value;
}

__global__ void iota_kernel(int32_t *p, int64_t n)
{
    hp::pdl_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = (int32_t)i;
}

__global__ void scatter_flags_kernel(const int32_t *flags, const int32_t *pos, int64_t n,
                                     int32_t *out, int32_t *d_count)
{
    hp::pdl_wait();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        if (flags[i]) out[pos[i]] = (int32_t)i;
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_count = pos[n];
}

// Exact cut, edge-parallel over the adjacency in tiles of CUT_THREADS x
// CUT_ITEMS entries (coalesced reads of adjncy and adjwgt; hub rows cost their
// share of the array): each entry's row comes from hp::tile_owners.  int64
// block partial sums of 2 x cut.
constexpr int CUT_THREADS = 256, CUT_ITEMS = 16, CUT_TILE = CUT_THREADS * CUT_ITEMS;
__global__ void __launch_bounds__(CUT_THREADS)
edgecut_kernel(int32_t n, int64_t m, const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
               const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ where, unsigned long long *cut2)
{
    hp::pdl_wait();
    __shared__ int32_t owner[CUT_TILE];
    __shared__ int32_t s_warp[CUT_THREADS / 32];
    __shared__ int32_t s_v0;
    long long acc = 0;
    for (int64_t tb = (int64_t)blockIdx.x * CUT_TILE; tb < m; tb += (int64_t)gridDim.x * CUT_TILE) {
        const int64_t te = tb + CUT_TILE < m ? tb + CUT_TILE : m;
        hp::tile_owners<CUT_THREADS, CUT_ITEMS>(xadj, n, tb, te, owner, s_warp, &s_v0);
        for (int64_t j = tb + threadIdx.x; j < te; j += CUT_THREADS)
            if (where[adjncy[j]] != where[owner[j - tb]]) acc += adjwgt ? adjwgt[j] : 1;
        __syncthreads();   // owner[] is rebuilt for the next tile
    }
    hp::block_add_to<CUT_THREADS>(acc, cut2);
}

inline unsigned grid_for(hp_context *c, int64_t n, int block)
{
    int64_t g = (n + block - 1) / block;
    int64_t cap = (int64_t)c->sm_count * 16;
    if (g > cap) g = cap;
    return (unsigned)(g > 0 ? g : 1);
}

}  // namespace

int hp_scan_excl(hp_context *c, const int32_t *in, int32_t *out, int64_t n)
{
    if (n < 0) return HP_ERR_INVALID_ARG;
    const int64_t ntiles = (n + 1 + SCAN_TILE - 1) / SCAN_TILE;
    if (ntiles > c->lb_cap) return HP_ERR_INTERNAL;   // reserved at the start of every call
    HP_LAUNCH(c, scan_excl_kernel<true>, (unsigned)ntiles, SCAN_BLOCK, 0, in, out, n, c->lb_status, c->lb_ctl,
              c->d_status);
    return HP_OK;
}

// ---- scan without any allocation ---------------------------------------------------
// Fixed scratch in the library's device image: the look-back tile status words
// for up to HP_SCAN_NOALLOC_MAX_N elements, then the tile-counter block (two
// 8-byte slots) and a status word (one slot).  Every GPU that loads the library
// holds this array (about 128 KiB) until the process exits.
#define HP_NOALLOC_TILES ((HP_SCAN_NOALLOC_MAX_N + 1 + SCAN_TILE - 1) / SCAN_TILE)
static __device__ __align__(256) unsigned long long g_scan_noalloc_scratch[HP_NOALLOC_TILES + 3];

extern "C" __attribute__((visibility("default")))
int hp_scan_exclusive_i32_noalloc(const int32_t *d_in, int32_t *d_out, int64_t n, void *stream)
{
    if (n < 0 || (!d_in && n > 0) || !d_out) return HP_ERR_INVALID_ARG;
    if (n > HP_SCAN_NOALLOC_MAX_N) {
        fprintf(stderr, "hp_scan_exclusive_i32_noalloc: n = %lld exceeds the fixed scratch limit of %lld "
                        "elements; use hp_scan_exclusive_i32 with a context\n",
                (long long)n, (long long)HP_SCAN_NOALLOC_MAX_N);
        return HP_ERR_UNSUPPORTED;
    }
    // An error left pending by the caller's earlier work would otherwise be
    // reported as this call's launch failure after the scan was enqueued:
    // refuse up front and leave the error for its owner to read.
    cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        fprintf(stderr, "hp_scan_exclusive_i32_noalloc: a CUDA error from earlier work is pending (%s); "
                        "nothing was launched\n", cudaGetErrorString(pending));
        return HP_ERR_CUDA;
    }
    // The host-side name of a __device__ array is not a device address: look
    // the address up with the caller's device and context current.  This is
    // done on every call, not cached per device number, so that a
    // cudaDeviceReset or a different (non-primary) context on the same device
    // cannot leave a stale address behind.  Once the library's device code is
    // loaded in the context the lookup allocates nothing; the first call in a
    // context loads it, which is why that first call belongs before any
    // stream capture.
    unsigned long long *scratch = nullptr;
    {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scan_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "hp_scan_exclusive_i32_noalloc: cudaGetSymbolAddress failed: %s\n",
                    cudaGetErrorString(e));
            return HP_ERR_CUDA;
        }
        scratch = (unsigned long long *)p;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t ntiles = (n + 1 + SCAN_TILE - 1) / SCAN_TILE;
    unsigned long long *counter_slot = scratch + HP_NOALLOC_TILES;     // hp::LbCtl (two slots)
    unsigned long long *status_slot = scratch + HP_NOALLOC_TILES + 2;
    // the array keeps the last call's contents: clear the tile words this call
    // uses, the counter and the status word
    HP_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned long long) * (size_t)ntiles, s));
    HP_CUDA(cudaMemsetAsync(counter_slot, 0, sizeof(unsigned long long) * 3, s));
    scan_excl_kernel<false><<<(unsigned)ntiles, SCAN_BLOCK, 0, s>>>(d_in, d_out, n, scratch,
                                                                    (hp::LbCtl *)counter_slot,
                                                                    (unsigned *)status_slot);
    HP_CUDA(cudaGetLastError());
    unsigned st = 0;
    HP_CUDA(cudaMemcpyAsync(&st, status_slot, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    HP_CUDA(cudaStreamSynchronize(s));
    return (st & HP_STATUS_SPIN_TIMEOUT) ? HP_ERR_TIMEOUT : HP_OK;
}

int hp_fill_i32(hp_context *c, int32_t *p, int64_t n, int32_t value)
{
    if (n <= 0) return HP_OK;
    HP_LAUNCH(c, fill_kernel, grid_for(c, n, 256), 256, 0, p, n, value);
    return HP_OK;
}

int hp_iota_i32(hp_context *c, int32_t *p, int64_t n)
{
    if (n <= 0) return HP_OK;
    HP_LAUNCH(c, iota_kernel, grid_for(c, n, 256), 256, 0, p, n);
    return HP_OK;
}

int hp_compact_flags(hp_context *c, const int32_t *flags, int64_t n, int32_t *out, int32_t *d_count)
{
    size_t mark = c->hi;
    int32_t *pos = ralloc_t<int32_t>(c, n + 1);
    HP_CHECK_OOM(c);
    HP_TRY(hp_scan_excl(c, flags, pos, n));
    HP_LAUNCH(c, scatter_flags_kernel, grid_for(c, n, 256), 256, 0, flags, pos, n, out, d_count);
    c->hi = mark;
    return HP_OK;
}

int hp_edgecut_launch(hp_context *c, int32_t n, int64_t m, const int32_t *xadj, const int32_t *adjncy,
                      const int32_t *adjwgt, const int32_t *where, unsigned long long *d_cut2)
{
    if (n <= 0) return HP_OK;
    if (m < 0) {   // not known to the caller: read xadj[n]
        int32_t mm = 0;
        HP_CUDA(cudaMemcpyAsync(c->h_pin, xadj + n, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
        HP_CUDA(cudaStreamSynchronize(c->stream));
        memcpy(&mm, c->h_pin, sizeof(int32_t));
        m = mm;
    }
    if (m <= 0) return HP_OK;
    const int64_t tiles = (m + CUT_TILE - 1) / CUT_TILE;
    HP_LAUNCH(c, edgecut_kernel, (unsigned)std::min<int64_t>(tiles, (int64_t)c->sm_count * 8), CUT_THREADS, 0, n, m,
              xadj, adjncy, adjwgt, where, d_cut2);
    return HP_OK;
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort of (key, value) int32 pairs, 8-bit digits, on a fixed
// grid (at most 4 blocks per SM) whatever the count on the device: block b
// owns a contiguous chunk.  Pass: per-block digit histograms stored
// digit-major, one exclusive scan over them, then a stable scatter in which
// every block walks its chunk in order and ranks its items per digit (warp
// __match_any_sync + per-warp digit counters in shared memory).
namespace {

constexpr int RS_BLOCK = 256;
constexpr int RS_ITEMS = 4;
constexpr int RS_TILE = RS_BLOCK * RS_ITEMS;

// Items of each block: the count split over the fixed grid in whole rounds of
// RS_BLOCK, block b taking [b chunk, (b+1) chunk) -- the blocks' chunks are in
// order, so a block-major digit scan keeps the sort stable.
__device__ __forceinline__ int64_t chunk_of(int32_t cnt, int32_t nblocks)
{
    int64_t ch = ((int64_t)cnt + nblocks - 1) / nblocks;
    return (ch + RS_BLOCK - 1) / RS_BLOCK * RS_BLOCK;
}

__global__ void __launch_bounds__(RS_BLOCK)
radix_hist_kernel(const int32_t *__restrict__ keys, const int32_t *__restrict__ d_count,
                  int shift, int32_t nblocks, int32_t *__restrict__ hist)
{
    hp::pdl_wait();
    __shared__ int32_t h[256];
    const int32_t cnt = *d_count;
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t chunk = chunk_of(cnt, nblocks);
    const int64_t beg = (int64_t)blockIdx.x * chunk, end = min((int64_t)cnt, beg + chunk);
    for (int64_t i = beg + threadIdx.x; i < end; i += RS_BLOCK)
        atomicAdd(&h[((unsigned)keys[i] >> shift) & 255u], 1);
    __syncthreads();
    hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_BLOCK)
radix_scatter_kernel(const int32_t *__restrict__ kin, const int32_t *__restrict__ vin,
                     const int32_t *__restrict__ d_count, int shift, int32_t nblocks,
                     const int32_t *__restrict__ hscan, int32_t *__restrict__ kout,
                     int32_t *__restrict__ vout)
{
    hp::pdl_wait();
    __shared__ int32_t run[256];                       // running per-digit offset of this block
    __shared__ int32_t wc[RS_BLOCK / 32][256];         // per-warp digit counts / offsets
    const int32_t cnt = *d_count;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    run[threadIdx.x] = hscan[(int64_t)threadIdx.x * nblocks + blockIdx.x];
    const int64_t chunk = chunk_of(cnt, nblocks);
    const int64_t beg = (int64_t)blockIdx.x * chunk, end = min((int64_t)cnt, beg + chunk);
    for (int64_t r0 = beg; r0 < end; r0 += RS_BLOCK) {   // the chunk in order, RS_BLOCK items a round
        for (int w = 0; w < RS_BLOCK / 32; w++) wc[w][threadIdx.x] = 0;
        __syncthreads();
        int64_t i = r0 + threadIdx.x;
        bool valid = i < end;
        int32_t k = valid ? kin[i] : 0, v = valid ? vin[i] : 0;
        unsigned d = valid ? (((unsigned)k >> shift) & 255u) : 256u + lane;  // invalid: unique
        unsigned peers = __match_any_sync(HP_FULL_MASK, d);
        int rank = __popc(peers & hp::lanemask_lt());
        if (valid && rank == 0) wc[wid][d] = __popc(peers);
        __syncthreads();
        {   // thread t owns digit t: turn warp counts into offsets
            int32_t acc = run[threadIdx.x];
            for (int w = 0; w < RS_BLOCK / 32; w++) {
                int32_t t = wc[w][threadIdx.x];
                wc[w][threadIdx.x] = acc;
                acc += t;
            }
            run[threadIdx.x] = acc;
        }
        __syncthreads();
        if (valid) {
            int32_t p = wc[wid][d] + rank;
            kout[p] = k;
            vout[p] = v;
        }
        __syncthreads();
    }
}

}  // namespace

int hp_sort_pairs(hp_context *c, int32_t *keys, int32_t *vals, int32_t *tkeys, int32_t *tvals,
                  int64_t bound, const int32_t *d_count, int key_bits, bool *in_tmp)
{
    *in_tmp = false;
    if (bound <= 0) return HP_OK;
    // a fixed grid whatever the count on the device: each block sorts its chunk
    const int32_t nblocks = (int32_t)std::min<int64_t>((bound + RS_TILE - 1) / RS_TILE, 4 * (int64_t)c->sm_count);
    const size_t mark = c->hi;
    int32_t *hist = ralloc_t<int32_t>(c, (int64_t)nblocks * 256 + 1);
    HP_CHECK_OOM(c);
    int32_t *ka = keys, *va = vals, *kb = tkeys, *vb = tvals;
    for (int shift = 0; shift < key_bits; shift += 8) {
        HP_LAUNCH(c, radix_hist_kernel, (unsigned)nblocks, RS_BLOCK, 0, ka, d_count, shift, nblocks, hist);
        HP_TRY(hp_scan_excl(c, hist, hist, (int64_t)nblocks * 256));
        HP_LAUNCH(c, radix_scatter_kernel, (unsigned)nblocks, RS_BLOCK, 0, ka, va, d_count, shift, nblocks,
                  hist, kb, vb);
        std::swap(ka, kb);
        std::swap(va, vb);
        *in_tmp = !*in_tmp;
    }
    c->hi = mark;
    return HP_OK;
}
