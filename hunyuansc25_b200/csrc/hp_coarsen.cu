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

constexpr int BIG_DEG = 32;   // rows longer than this use a warp per vertex

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
big_list_kernel(int32_t n, const int32_t *__restrict__ xadj, int32_t *list, int32_t *d_count)
{
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n && xadj[v + 1] - xadj[v] > BIG_DEG) list[atomicAdd(d_count, 1)] = v;
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

template <int NT, int CAP>
__global__ void __launch_bounds__(NT)
contract_block_kernel(const int32_t *__restrict__ list, const int32_t *__restrict__ d_count,
                      ContractSrc src, const int32_t *__restrict__ toff, int32_t *__restrict__ tk,
                      int32_t *__restrict__ tw, int32_t *__restrict__ ucnt)
{
    __shared__ int32_t sk[CAP], sw[CAP];
    __shared__ int32_t s_scan[NT / 32 + 2];
    const int32_t cnt = *d_count;
    for (int32_t li = blockIdx.x; li < cnt; li += gridDim.x) {
        const int32_t c = list[li];
        int32_t v, u, lv, len;
        src.row(c, v, u, lv, len);
        int P = 32;
        while (P < len) P <<= 1;
        for (int i = threadIdx.x; i < P; i += NT) {
            int32_t k = hp::KEY_NONE, w = 0;
            if (i < len) src.get(c, v, u, lv, i, k, w);
            sk[i] = k;
            sw[i] = w;
        }
        __syncthreads();
        int32_t off = toff[c];
        int tot = hp::block_aggregate_smem<NT, CAP>(sk, sw, P, tk + off, tw + off, s_scan);
        if (threadIdx.x == 0) ucnt[c] = tot;
    }
}

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

__global__ void __launch_bounds__(256)
copy_rows_kernel(int32_t cn, const int32_t *__restrict__ toff, const int32_t *__restrict__ cxadj,
                 const int32_t *__restrict__ tk, const int32_t *__restrict__ tw,
                 int32_t *__restrict__ cadjncy, int32_t *__restrict__ cadjwgt)
{
    const int lane = threadIdx.x & 31;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < cn;
         c += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int32_t s = toff[c], d = cxadj[c], len = cxadj[c + 1] - d;
        for (int32_t i = lane; i < len; i += 32) {
            cadjncy[d + i] = tk[s + i];
            cadjwgt[d + i] = tw[s + i];
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
    int32_t *flags = ralloc_t<int32_t>(c, n + 1);
    int32_t *list = ralloc_t<int32_t>(c, n + 1);
    HP_CHECK_OOM(c);
    // scalar slots: [0] big count, [1] list count, [2..2+R) made per round, [40..43] matched counts
    unsigned long long *sc = c->d_scal;
    HP_CUDA(cudaMemsetAsync(sc, 0, sizeof(unsigned long long) * HP_NSCAL, c->stream));
    int32_t *d_bigcnt = (int32_t *)&sc[0];
    int32_t *d_listcnt = (int32_t *)&sc[1];

    HP_TRY(hp_fill_i32(c, g.match, n, -1));
    HP_LAUNCH(c, big_list_kernel, blocks_for(n), 256, 0, n, g.xadj, big, d_bigcnt);

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
        HP_LAUNCH(c, pair_hub_small_kernel, blocks_for(n), 256, 0, n, g.xadj, g.adjncy, g.vwgt, hub,
                  g.match, maxvwgt);
        HP_LAUNCH(c, pair_hub_big_kernel, persistent_grid(c), 256, 0, big, d_bigcnt, g.xadj, g.adjncy,
                  g.vwgt, hub, g.match, maxvwgt);
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
        HP_LAUNCH(c, (contract_block_kernel<128, 512>), (unsigned)std::min<int64_t>(h.cnt[0], c->sm_count * 16),
                  128, 0, lists, &counts[0], src, toff, tk, tw, ucnt);
    if (h.cnt[1] > 0)
        HP_LAUNCH(c, (contract_block_kernel<512, 4096>), (unsigned)std::min<int64_t>(h.cnt[1], c->sm_count * 4),
                  512, 0, lists + cn, &counts[1], src, toff, tk, tw, ucnt);
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
    HP_LAUNCH(c, copy_rows_kernel, blocks_for((int64_t)cn * 32), 256, 0, cn, toff, cg.xadj, tk, tw,
              cg.adjncy, cg.adjwgt);
    // algorithmic bytes of the whole contraction: fine CSR, cmap, match,
    // vwgt in; coarse xadj, adjacency, weights, vertex weights out
    hp_prof_end(c, tok, HP_PROF_CONTRACT,
                4 * ((int64_t)n + 1) + 8 * g.m + 12 * (int64_t)n + 4 * ((int64_t)cn + 1) + 8 * (int64_t)mc +
                    4 * (int64_t)cn);
    c->hi = mark;
    return HP_OK;
}

}  // namespace

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
