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
//     (scatter -> segmented sort -> mark -> scan -> write; here one pass per
//      coarse vertex that gathers both fine rows, merges equal coarse
//      neighbours and writes them sorted, by size class; hp_rowagg.cuh)
// The reference's matching is an atomicCAS race (nondeterministic); every
// decision here is a pure function of the level's CSR and the seed, so the
// CPU oracle reproduces each level bit for bit.
#include "hp_internal.cuh"
#include "hp_rowagg.cuh"

namespace {

constexpr int BIG_DEG = 32;      // rows longer than this use a warp per vertex
constexpr int HUGE_DEG = 4096;   // rows longer than this use a CTA per vertex

// ---------------------------------------------------------------------------
// matching

// ELIG: handshake proposal (unmatched neighbour, weight cap).  !ELIG: hub
// choice for two-hop matching (any neighbour).
template <bool ELIG>
__global__ void __launch_bounds__(256)
pref_small_kernel(int32_t n, const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                  const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ vwgt,
                  const int32_t *__restrict__ match, int32_t *__restrict__ pref, uint64_t lkey,
                  int64_t maxvwgt, const unsigned long long *made_prev)
{
    if (made_prev && *made_prev == 0ull) return;
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int32_t b = xadj[v], e = xadj[v + 1];
    if (e - b > BIG_DEG) return;
    if (match[v] != -1) { pref[v] = -1; return; }
    const int32_t wv = vwgt[v];
    int32_t bu = -1, bw = 0;
    uint32_t bh = 0;
    for (int32_t j = b; j < e; j++) {
        int32_t u = adjncy[j];
        if (u == v) continue;
        if (ELIG) {
            if (match[u] != -1) continue;
            if ((int64_t)wv + vwgt[u] > maxvwgt) continue;
        }
        int32_t w = adjwgt[j];
        uint32_t h = hp::edge_tie(lkey, v, u);
        if (bu < 0 || hp::better(w, h, u, bw, bh, bu)) { bu = u; bw = w; bh = h; }
    }
    pref[v] = bu;
}

template <bool ELIG>
__global__ void __launch_bounds__(256)
pref_big_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ vwgt,
                const int32_t *__restrict__ match, int32_t *__restrict__ pref, uint64_t lkey,
                int64_t maxvwgt, const unsigned long long *made_prev)
{
    if (made_prev && *made_prev == 0ull) return;
    const int lane = threadIdx.x & 31;
    const int32_t cnt = *d_count;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < cnt;
         i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int32_t v = list[i];
        if (match[v] != -1) { if (lane == 0) pref[v] = -1; continue; }
        const int32_t wv = vwgt[v];
        int32_t bu = -1, bw = 0;
        uint32_t bh = 0;
        for (int32_t j = xadj[v] + lane; j < xadj[v + 1]; j += 32) {
            int32_t u = adjncy[j];
            if (u == v) continue;
            if (ELIG) {
                if (match[u] != -1) continue;
                if ((int64_t)wv + vwgt[u] > maxvwgt) continue;
            }
            int32_t w = adjwgt[j];
            uint32_t h = hp::edge_tie(lkey, v, u);
            if (bu < 0 || hp::better(w, h, u, bw, bh, bu)) { bu = u; bw = w; bh = h; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            int32_t ou = __shfl_xor_sync(HP_FULL_MASK, bu, o);
            int32_t ow = __shfl_xor_sync(HP_FULL_MASK, bw, o);
            uint32_t oh = __shfl_xor_sync(HP_FULL_MASK, bh, o);
            if (ou >= 0 && (bu < 0 || hp::better(ow, oh, ou, bw, bh, bu))) { bu = ou; bw = ow; bh = oh; }
        }
        if (lane == 0) pref[v] = bu;
    }
}

__global__ void __launch_bounds__(256)
commit_kernel(int32_t n, int32_t *__restrict__ match, const int32_t *__restrict__ pref,
              unsigned long long *made_cur, const unsigned long long *made_prev)
{
    if (made_prev && *made_prev == 0ull) return;
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    int made = 0;
    if (v < n && match[v] == -1) {
        int32_t u = pref[v];
        if (u >= 0 && pref[u] == v) { match[v] = u; made = 1; }
    }
    hp::block_add_to<256>(made, made_cur);
}

__global__ void __launch_bounds__(256)
big_list_kernel(int32_t n, const int32_t *__restrict__ xadj, int32_t *list, int32_t *d_count,
                int32_t *huge, int32_t *d_huge)
{
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int32_t d = xadj[v + 1] - xadj[v];
    if (d > HUGE_DEG) huge[atomicAdd(d_huge, 1)] = v;
    else if (d > BIG_DEG) list[atomicAdd(d_count, 1)] = v;
}

// CTA per vertex for rows longer than HUGE_DEG (R-MAT hubs).
template <bool ELIG>
__global__ void __launch_bounds__(512)
pref_huge_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                 const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                 const int32_t *__restrict__ adjwgt, const int32_t *__restrict__ vwgt,
                 const int32_t *__restrict__ match, int32_t *__restrict__ pref, uint64_t lkey,
                 int64_t maxvwgt, const unsigned long long *made_prev)
{
    if (made_prev && *made_prev == 0ull) return;
    __shared__ int32_t su[16], sw[16];
    __shared__ uint32_t sh[16];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t v = list[li];
        if (match[v] != -1) { if (threadIdx.x == 0) pref[v] = -1; continue; }
        const int32_t wv = vwgt[v];
        int32_t bu = -1, bw = 0;
        uint32_t bh = 0;
        for (int32_t j = xadj[v] + threadIdx.x; j < xadj[v + 1]; j += blockDim.x) {
            int32_t u = adjncy[j];
            if (u == v) continue;
            if (ELIG) {
                if (match[u] != -1) continue;
                if ((int64_t)wv + vwgt[u] > maxvwgt) continue;
            }
            int32_t w = adjwgt[j];
            uint32_t h = hp::edge_tie(lkey, v, u);
            if (bu < 0 || hp::better(w, h, u, bw, bh, bu)) { bu = u; bw = w; bh = h; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            int32_t ou = __shfl_xor_sync(HP_FULL_MASK, bu, o);
            int32_t ow = __shfl_xor_sync(HP_FULL_MASK, bw, o);
            uint32_t oh = __shfl_xor_sync(HP_FULL_MASK, bh, o);
            if (ou >= 0 && (bu < 0 || hp::better(ow, oh, ou, bw, bh, bu))) { bu = ou; bw = ow; bh = oh; }
        }
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

// Hub pairing for rows longer than HUGE_DEG: clients ranked by a CTA scan.
__global__ void __launch_bounds__(512)
pair_hub_huge_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                     const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                     const int32_t *__restrict__ vwgt, const int32_t *__restrict__ hub,
                     int32_t *__restrict__ match, int64_t maxvwgt)
{
    __shared__ int32_t s_scan[512 / 32 + 2];
    __shared__ int32_t s_cl[512];
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t h = list[li];
        int32_t t = 0, carry = -1;
        for (int32_t base = xadj[h]; base < xadj[h + 1]; base += 512) {
            const int32_t j = base + threadIdx.x;
            int32_t c = -1;
            int isc = 0;
            if (j < xadj[h + 1]) { c = adjncy[j]; isc = hub[c] == h; }
            int tot;
            const int ex = hp::block_excl_scan<512>(isc, &tot, s_scan);
            if (isc) s_cl[ex] = c;
            __syncthreads();
            if (isc && ((t + ex) & 1)) {
                const int32_t first = ex > 0 ? s_cl[ex - 1] : carry;
                if ((int64_t)vwgt[first] + vwgt[c] <= maxvwgt) { match[first] = c; match[c] = first; }
            }
            if (tot > 0 && ((t + tot - 1) & 1) == 0) carry = s_cl[tot - 1];
            t += tot;
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(256)
count_matched_kernel(int32_t n, const int32_t *__restrict__ match, unsigned long long *out)
{
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    hp::block_add_to<256>((v < n && match[v] != -1) ? 1 : 0, out);
}

// Pair the clients of hub h (unmatched vertices whose hub is h) in h's row
// order: (c0,c1), (c2,c3), ... when the weight sum fits.
__global__ void __launch_bounds__(256)
pair_hub_small_kernel(int32_t n, const int32_t *__restrict__ xadj,
                      const int32_t *__restrict__ adjncy, const int32_t *__restrict__ vwgt,
                      const int32_t *__restrict__ hub, int32_t *__restrict__ match, int64_t maxvwgt)
{
    int32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n) return;
    const int32_t b = xadj[h], e = xadj[h + 1];
    if (e - b > BIG_DEG) return;
    int32_t first = -1, t = 0;
    for (int32_t j = b; j < e; j++) {
        int32_t c = adjncy[j];
        if (hub[c] != h) continue;
        if ((t & 1) == 0) first = c;
        else if ((int64_t)vwgt[first] + vwgt[c] <= maxvwgt) { match[first] = c; match[c] = first; }
        t++;
    }
}

__global__ void __launch_bounds__(256)
pair_hub_big_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                    const int32_t *__restrict__ xadj, const int32_t *__restrict__ adjncy,
                    const int32_t *__restrict__ vwgt, const int32_t *__restrict__ hub,
                    int32_t *__restrict__ match, int64_t maxvwgt)
{
    const int lane = threadIdx.x & 31;
    const int32_t cnt = *d_count;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < cnt;
         i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int32_t h = list[i];
        int32_t t = 0;          // clients seen so far
        int32_t carry = -1;     // unpaired client from the previous chunk (t odd)
        for (int32_t base = xadj[h]; base < xadj[h + 1]; base += 32) {
            int32_t j = base + lane;
            int32_t c = -1;
            bool isc = false;
            if (j < xadj[h + 1]) { c = adjncy[j]; isc = hub[c] == h; }
            unsigned m = __ballot_sync(HP_FULL_MASK, isc);
            // partner of an odd-ranked client is the previous client: either
            // the nearest lower lane in this chunk or the carried one
            unsigned below_all = m & hp::lanemask_lt();
            int src = below_all ? 31 - __clz(below_all) : lane;
            int32_t prevc = __shfl_sync(HP_FULL_MASK, c, src);
            if (isc) {
                int32_t r = t + __popc(below_all);
                if (r & 1) {
                    int32_t first = below_all ? prevc : carry;
                    if ((int64_t)vwgt[first] + vwgt[c] <= maxvwgt) { match[first] = c; match[c] = first; }
                }
            }
            int tot = __popc(m);
            if (tot) {
                int lastlane = 31 - __clz(m);
                int32_t lastc = __shfl_sync(HP_FULL_MASK, c, lastlane);
                if (((t + tot - 1) & 1) == 0) carry = lastc;  // last client has even rank
            }
            t += tot;
        }
    }
}

__global__ void __launch_bounds__(256)
flag_unmatched_kernel(int32_t n, const int32_t *__restrict__ xadj,
                      const int32_t *__restrict__ match, int32_t *__restrict__ flags, int isolated_only)
{
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
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    int32_t u = match[v];
    if (u == -1) { u = v; match[v] = v; }
    leader_flag[v] = (v <= u);
}

// Followers copy the leader's coarse id; leaders fill the coarse vertex.
__global__ void __launch_bounds__(256)
coarse_setup_kernel(int32_t n, const int32_t *__restrict__ match, int32_t *__restrict__ cmap,
                    const int32_t *__restrict__ xadj, const int32_t *__restrict__ vwgt,
                    int32_t *__restrict__ leader_of, int32_t *__restrict__ cvwgt,
                    int32_t *__restrict__ tlen, int32_t *__restrict__ lists,
                    int32_t *__restrict__ counts, int32_t cn, int32_t *__restrict__ maxlen)
{
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    int32_t u = match[v];
    if (v > u) { cmap[v] = cmap[u]; return; }
    int32_t c = cmap[v];
    leader_of[c] = v;
    int32_t len = xadj[v + 1] - xadj[v];
    int32_t w = vwgt[v];
    if (u != v) { len += xadj[u + 1] - xadj[u]; w += vwgt[u]; }
    cvwgt[c] = w;
    tlen[c] = len;
    if (len > 32) {
        int cls = len <= 512 ? 0 : (len <= 4096 ? 1 : 2);
        int32_t pos = atomicAdd(&counts[cls], 1);
        lists[(int64_t)cls * cn + pos] = c;
        if (cls == 2) atomicMax(maxlen, len);
    }
}

// Entry i of coarse vertex c: the i-th entry of the leader's row, then of the
// mate's row, mapped through cmap; the coarse self key is dropped.
struct ContractSrc {
    const int32_t *xadj, *adjncy, *adjwgt, *cmap, *match, *leader_of;
    __device__ __forceinline__ void row(int32_t c, int32_t &v, int32_t &u, int32_t &lv,
                                        int32_t &len) const
    {
        v = leader_of[c];
        u = match[v];
        lv = xadj[v + 1] - xadj[v];
        len = lv + (u != v ? xadj[u + 1] - xadj[u] : 0);
    }
    __device__ __forceinline__ void get(int32_t c, int32_t v, int32_t u, int32_t lv, int32_t i,
                                        int32_t &k, int32_t &w) const
    {
        int32_t j = i < lv ? xadj[v] + i : xadj[u] + (i - lv);
        k = cmap[adjncy[j]];
        w = adjwgt[j];
        if (k == c) { k = hp::KEY_NONE; w = 0; }
    }
};

__global__ void __launch_bounds__(256)
contract_warp_kernel(int32_t cn, ContractSrc src, const int32_t *__restrict__ toff,
                     int32_t *__restrict__ tk, int32_t *__restrict__ tw, int32_t *__restrict__ ucnt)
{
    const int lane = threadIdx.x & 31;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < cn;
         c += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        int32_t v, u, lv, len;
        src.row((int32_t)c, v, u, lv, len);
        if (len > 32) continue;
        int32_t k = hp::KEY_NONE, w = 0;
        if (lane < len) src.get((int32_t)c, v, u, lv, lane, k, w);
        int32_t off = toff[c];
        int cnt = hp::warp_aggregate32(k, w, tk + off, tw + off);
        if (lane == 0) ucnt[c] = cnt;
    }
}

// Rows of 33..HCAP/2 entries: one CTA merges equal coarse ids in a
// shared-memory hash table (linear probing, atomicCAS keys, atomicAdd
// weights), compacts the unique keys, and bitonic-sorts only those.
template <int NT, int HCAP>
__global__ void __launch_bounds__(NT)
contract_hash_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                     ContractSrc src, const int32_t *__restrict__ toff, int32_t *__restrict__ tk,
                     int32_t *__restrict__ tw, int32_t *__restrict__ ucnt)
{
    extern __shared__ int32_t hsm[];
    int32_t *hk = hsm, *hw = hsm + HCAP;                  // hash table
    int32_t *sk = hsm + 2 * HCAP, *sw = sk + HCAP / 2;    // unique entries to sort
    __shared__ int32_t s_scan[NT / 32 + 2];
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t c = list[li];
        int32_t v, u, lv, len;
        src.row(c, v, u, lv, len);
        // table sized to the row: H = pow2 >= 2 len (load factor <= 1/2)
        int H = 64;
        while (H < 2 * len) H <<= 1;
        for (int i = threadIdx.x; i < H; i += NT) { hk[i] = hp::KEY_NONE; hw[i] = 0; }
        __syncthreads();
        for (int32_t i = threadIdx.x; i < len; i += NT) {
            int32_t k, w;
            src.get(c, v, u, lv, i, k, w);
            if (k == hp::KEY_NONE) continue;
            uint32_t h = ((uint32_t)k * 2654435761u) & (H - 1);
            for (;;) {
                int32_t prev = atomicCAS(&hk[h], hp::KEY_NONE, k);
                if (prev == hp::KEY_NONE || prev == k) { atomicAdd(&hw[h], w); break; }
                h = (h + 1) & (H - 1);
            }
        }
        __syncthreads();
        // compact occupied slots; thread t owns slots [t*per, (t+1)*per)
        const int per = (H + NT - 1) / NT;
        const int lo = threadIdx.x * per, hi = min(lo + per, H);
        int cntl = 0;
        for (int i = lo; i < hi; i++) cntl += hk[i] != hp::KEY_NONE;
        int U;
        int pos = hp::block_excl_scan<NT>(cntl, &U, s_scan);
        for (int i = lo; i < hi; i++)
            if (hk[i] != hp::KEY_NONE) { sk[pos] = hk[i]; sw[pos] = hw[i]; pos++; }
        int P = 32;
        while (P < U) P <<= 1;
        for (int i = U + threadIdx.x; i < P; i += NT) { sk[i] = hp::KEY_NONE; sw[i] = 0; }
        __syncthreads();
        int32_t off = toff[c];
        int tot = hp::block_aggregate_smem<NT, HCAP / 2>(sk, sw, P, tk + off, tw + off, s_scan);
        if (threadIdx.x == 0) ucnt[c] = tot;
    }
}

constexpr size_t hash_smem(int hcap) { return sizeof(int32_t) * (size_t)(3 * hcap); }

// Rows longer than 4096 entries: dense accumulator over the coarse id space in
// a per-CTA global slab (dw: cn ints, bm: cn/32 words; zero on entry/exit).
template <int NT>
__global__ void __launch_bounds__(NT)
contract_dense_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                      ContractSrc src, const int32_t *__restrict__ toff, int32_t *__restrict__ tk,
                      int32_t *__restrict__ tw, int32_t *__restrict__ ucnt, int32_t cn,
                      int32_t *slab_w, unsigned *slab_bm)
{
    __shared__ int32_t s_scan[NT / 32 + 2];
    int32_t *dw = slab_w + (int64_t)blockIdx.x * cn;
    unsigned *bm = slab_bm + (int64_t)blockIdx.x * ((cn + 31) / 32);
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t c = list[li];
        int32_t v, u, lv, len;
        src.row(c, v, u, lv, len);
        for (int32_t i = threadIdx.x; i < len; i += NT) {
            int32_t k, w;
            src.get(c, v, u, lv, i, k, w);
            if (k == hp::KEY_NONE) continue;
            atomicAdd(&dw[k], w);
            atomicOr(&bm[k >> 5], 1u << (k & 31));
        }
        __syncthreads();
        int32_t off = toff[c];
        int tot = hp::dense_extract<NT>(dw, bm, cn, tk + off, tw + off, s_scan);
        if (threadIdx.x == 0) ucnt[c] = tot;
    }
}

// Compacts the unique coarse rows (at upper-bound offsets toff[c]) to their
// final places cxadj[c]: edge-parallel over the coarse adjacency in tiles of
// 256 x 32 entries; the owner of an entry is found by binary search over cxadj
// and a forward walk, so long rows cost their length, not one warp's time.
__global__ void __launch_bounds__(256)
copy_rows_kernel(int32_t cn, const int32_t *__restrict__ toff, const int32_t *__restrict__ cxadj,
                 const int32_t *__restrict__ tk, const int32_t *__restrict__ tw,
                 int32_t *__restrict__ cadjncy, int32_t *__restrict__ cadjwgt)
{
    const int64_t mc = cxadj[cn];
    const int64_t tile = 256 * 32;
    for (int64_t tb = blockIdx.x * tile; tb < mc; tb += (int64_t)gridDim.x * tile) {
        int64_t j = tb + threadIdx.x;
        if (j >= mc) continue;
        int32_t lo = 0, hi = cn - 1;
        while (lo < hi) {
            int32_t mid = (int32_t)(((int64_t)lo + hi + 1) / 2);
            if (cxadj[mid] <= j) lo = mid; else hi = mid - 1;
        }
        int32_t c = lo;
        for (int k = 0; k < 32 && j < mc; k++, j += 256) {
            while (cxadj[c + 1] <= j) c++;
            const int64_t src = toff[c] + (j - cxadj[c]);
            cadjncy[j] = tk[src];
            cadjwgt[j] = tw[src];
        }
    }
}

inline unsigned blocks_for(int64_t threads, int block = 256)
{
    int64_t g = (threads + block - 1) / block;
    return (unsigned)(g > 0 ? g : 1);
}

inline unsigned persistent_grid(hp_context *c, int per_sm = 8)
{
    return (unsigned)(c->sm_count * per_sm);
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

    int32_t *pref = ralloc_t<int32_t>(c, n);
    int32_t *big = ralloc_t<int32_t>(c, n);
    int32_t *huge = ralloc_t<int32_t>(c, n);
    int32_t *flags = ralloc_t<int32_t>(c, n + 1);
    int32_t *list = ralloc_t<int32_t>(c, n + 1);
    HP_CHECK_OOM(c);
    // scalar slots: [0] big count, [1] list count, [2..2+R) made per round, [40..43] matched counts
    unsigned long long *sc = c->d_scal;
    HP_CUDA(cudaMemsetAsync(sc, 0, sizeof(unsigned long long) * HP_NSCAL, c->stream));
    int32_t *d_bigcnt = (int32_t *)&sc[0];
    int32_t *d_listcnt = (int32_t *)&sc[1];
    int32_t *d_hugecnt = (int32_t *)&sc[38];

    HP_TRY(hp_fill_i32(c, g.match, n, -1));
    HP_LAUNCH(c, big_list_kernel, blocks_for(n), 256, 0, n, g.xadj, big, d_bigcnt, huge, d_hugecnt);

    const int rounds = o.match_rounds < 1 ? 1 : (o.match_rounds > 30 ? 30 : o.match_rounds);
    // algorithmic bytes of one full handshake round: xadj, adjncy, adjwgt,
    // vwgt, match read and write (neighbour gathers not counted)
    const int64_t round_bytes = 4 * ((int64_t)n + 1) + 8 * g.m + 12 * (int64_t)n;
    for (int r = 0; r < rounds; r++) {
        const int tok = hp_prof_begin(c);
        const unsigned long long *prev = r == 0 ? nullptr : &sc[2 + r - 1];
        HP_LAUNCH(c, pref_small_kernel<true>, blocks_for(n), 256, 0, n, g.xadj, g.adjncy, g.adjwgt,
                  g.vwgt, g.match, pref, lkey, maxvwgt, prev);
        HP_LAUNCH(c, pref_big_kernel<true>, persistent_grid(c), 256, 0, big, d_bigcnt, g.xadj,
                  g.adjncy, g.adjwgt, g.vwgt, g.match, pref, lkey, maxvwgt, prev);
        HP_LAUNCH(c, pref_huge_kernel<true>, (unsigned)(2 * c->sm_count), 512, 0, huge, d_hugecnt, g.xadj,
                  g.adjncy, g.adjwgt, g.vwgt, g.match, pref, lkey, maxvwgt, prev);
        HP_LAUNCH(c, commit_kernel, blocks_for(n), 256, 0, n, g.match, pref, &sc[2 + r], prev);
        hp_prof_end(c, tok, r == 0 ? HP_PROF_MATCH : 6, r == 0 ? round_bytes : 0);
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
    if (4 * nm < 3 * (int64_t)n) {
        // two-hop through a shared heaviest neighbour
        int32_t *hub = pref;
        HP_LAUNCH(c, pref_small_kernel<false>, blocks_for(n), 256, 0, n, g.xadj, g.adjncy, g.adjwgt,
                  g.vwgt, g.match, hub, lkey, maxvwgt, (const unsigned long long *)nullptr);
        HP_LAUNCH(c, pref_big_kernel<false>, persistent_grid(c), 256, 0, big, d_bigcnt, g.xadj,
                  g.adjncy, g.adjwgt, g.vwgt, g.match, hub, lkey, maxvwgt,
                  (const unsigned long long *)nullptr);
        HP_LAUNCH(c, pref_huge_kernel<false>, (unsigned)(2 * c->sm_count), 512, 0, huge, d_hugecnt, g.xadj,
                  g.adjncy, g.adjwgt, g.vwgt, g.match, hub, lkey, maxvwgt,
                  (const unsigned long long *)nullptr);
        HP_LAUNCH(c, pair_hub_small_kernel, blocks_for(n), 256, 0, n, g.xadj, g.adjncy, g.vwgt, hub,
                  g.match, maxvwgt);
        HP_LAUNCH(c, pair_hub_big_kernel, persistent_grid(c), 256, 0, big, d_bigcnt, g.xadj, g.adjncy,
                  g.vwgt, hub, g.match, maxvwgt);
        HP_LAUNCH(c, pair_hub_huge_kernel, (unsigned)(2 * c->sm_count), 512, 0, huge, d_hugecnt, g.xadj,
                  g.adjncy, g.vwgt, hub, g.match, maxvwgt);
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
    HP_CHECK_OOM(c);
    const size_t mark = c->hi;
    int32_t *leader_of = ralloc_t<int32_t>(c, cn);
    int32_t *toff = ralloc_t<int32_t>(c, cn + 1);
    int32_t *ucnt = ralloc_t<int32_t>(c, cn + 1);
    int32_t *lists = ralloc_t<int32_t>(c, 3 * (int64_t)cn);
    HP_CHECK_OOM(c);
    unsigned long long *sc = c->d_scal;
    HP_CUDA(cudaMemsetAsync(sc, 0, sizeof(unsigned long long) * 4, c->stream));
    int32_t *counts = (int32_t *)sc;          // 3 class counts (+ maxlen) packed in 2 slots
    int32_t *maxlen = counts + 3;

    int tok = hp_prof_begin(c);
    HP_LAUNCH(c, coarse_setup_kernel, blocks_for(n), 256, 0, n, g.match, g.cmap, g.xadj, g.vwgt,
              leader_of, cg.vwgt, toff, lists, counts, cn, maxlen);
    HP_TRY(hp_scan_excl(c, toff, toff, cn));
    hp_prof_end(c, tok, HP_PROF_CONTRACT, 0);
    struct { int32_t cnt[3]; int32_t maxlen; } h;
    HP_TRY(hp_read_scalars(c, counts, sizeof(h), &h));
    int32_t tm = 0;
    HP_TRY(hp_read_scalars(c, toff + cn, sizeof(int32_t), &tm));

    int32_t *tk = ralloc_t<int32_t>(c, tm);
    int32_t *tw = ralloc_t<int32_t>(c, tm);
    HP_CHECK_OOM(c);
    ContractSrc src{g.xadj, g.adjncy, g.adjwgt, g.cmap, g.match, leader_of};
    tok = hp_prof_begin(c);
    HP_LAUNCH(c, contract_warp_kernel, blocks_for((int64_t)cn * 32), 256, 0, cn, src, toff, tk, tw,
              ucnt);
    if (h.cnt[0] > 0)
        HP_LAUNCH(c, (contract_hash_kernel<128, 1024>), (unsigned)std::min<int64_t>(h.cnt[0], c->sm_count * 16),
                  128, hash_smem(1024), lists, &counts[0], src, toff, tk, tw, ucnt);
    if (h.cnt[1] > 0)
        HP_LAUNCH(c, (contract_hash_kernel<512, 8192>), (unsigned)std::min<int64_t>(h.cnt[1], c->sm_count * 2),
                  512, hash_smem(8192), lists + cn, &counts[1], src, toff, tk, tw, ucnt);
    if (h.cnt[2] > 0) {
        // slab per CTA: cn ints + cn/32 words; bounded to ~512 MB
        int64_t slab = (int64_t)cn * 4 + ((int64_t)cn + 31) / 32 * 4;
        int64_t nb = std::min<int64_t>(h.cnt[2], 2 * (int64_t)c->sm_count);
        nb = std::max<int64_t>(1, std::min<int64_t>(nb, (512ll << 20) / std::max<int64_t>(slab, 1)));
        int32_t *sw = ralloc_t<int32_t>(c, nb * (int64_t)cn);
        unsigned *sbm = ralloc_t<unsigned>(c, nb * (((int64_t)cn + 31) / 32));
        HP_CHECK_OOM(c);
        HP_CUDA(cudaMemsetAsync(sw, 0, sizeof(int32_t) * (size_t)(nb * cn), c->stream));
        HP_CUDA(cudaMemsetAsync(sbm, 0, sizeof(unsigned) * (size_t)(nb * ((cn + 31) / 32)), c->stream));
        HP_LAUNCH(c, contract_dense_kernel<1024>, (unsigned)nb, 1024, 0, lists + 2 * (int64_t)cn,
                  &counts[2], src, toff, tk, tw, ucnt, cn, sw, sbm);
    }
    HP_TRY(hp_scan_excl(c, ucnt, cg.xadj, cn));
    hp_prof_end(c, tok, HP_PROF_CONTRACT, 0);
    int32_t mc = 0;
    HP_TRY(hp_read_scalars(c, cg.xadj + cn, sizeof(int32_t), &mc));
    cg.m = mc;
    // the coarse adjacency goes to the low end; temporaries stay on the high end
    cg.adjncy = lalloc_t<int32_t>(c, mc);
    cg.adjwgt = lalloc_t<int32_t>(c, mc);
    HP_CHECK_OOM(c);
    tok = hp_prof_begin(c);
    HP_LAUNCH(c, copy_rows_kernel, std::min<unsigned>(blocks_for(((int64_t)mc + 31) / 32), c->sm_count * 16), 256,
              0, cn, toff, cg.xadj, tk, tw, cg.adjncy, cg.adjwgt);
    // algorithmic bytes of the whole contraction: fine CSR, cmap, match,
    // vwgt in; coarse xadj, adjacency, weights, vertex weights out
    hp_prof_end(c, tok, HP_PROF_CONTRACT,
                4 * ((int64_t)n + 1) + 8 * g.m + 12 * (int64_t)n + 4 * ((int64_t)cn + 1) + 8 * (int64_t)mc +
                    4 * (int64_t)cn);
    c->hi = mark;
    return HP_OK;
}

}  // namespace

int hp_coarsen_init()
{
    HP_CUDA(cudaFuncSetAttribute(contract_hash_kernel<512, 8192>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)hash_smem(8192)));
    return HP_OK;
}

int hp_coarsen(hp_context *c, int32_t coarsen_to, int64_t maxvwgt)
{
    int level = 0;
    while (level < c->opt.max_levels && c->levels[level].n > coarsen_to) {
        HpLevel &g = c->levels[level];
        g.match = lalloc_t<int32_t>(c, g.n);
        g.cmap = lalloc_t<int32_t>(c, (int64_t)g.n + 1);
        HP_CHECK_OOM(c);
        int32_t cn = 0;
        HP_TRY(match_level(c, g, level, maxvwgt, &cn));
        c->levels.emplace_back();
        HpLevel &f = c->levels[level];
        HpLevel &cg = c->levels[level + 1];
        HP_TRY(contract_level(c, f, cn, cg));
        HP_TRY(hp_check_status(c));
        level++;
        if (!(100 * (int64_t)cg.n < 85 * (int64_t)f.n && cg.m > cg.n / 2)) break;
    }
    return HP_OK;
}
