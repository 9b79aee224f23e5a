// hp_nd.cu — nested-dissection fill-reducing ordering (hp_node_nd).
//
// Reference: ReorderGraph / NestedBisection
// (mygp_0.9.9_test_initpartition/reordergraph.h:177-306): a vertex separator
// of the graph takes the highest numbers, the two sides are split off as
// induced subgraphs and ordered recursively (left side first), and a subgraph
// of at most ND_LEAF vertices, or without edges, is ordered directly (the
// reference calls MMD_Order from mmdorder.h, which is not in its tree; here an
// exact minimum-degree elimination).  The reference finds separators with its
// own randomised bisection and node refinement; here a separator comes from
// this library's deterministic 2-way partition and one rule (the boundary of
// the side with fewer boundary vertices, thinned), so the ordering is a pure
// function of the graph and options, equal to the oracle's (ora_node_nd).
//
// B200 layout: the recursion runs depth by depth ("tiers").  All subgraphs of
// a tier live concatenated in one device buffer in hp_partition_batch's
// layout (per subgraph: local xadj of n+1 entries, local adjncy, vertex
// weights, and the original vertex id of every vertex).  Per tier:
//   1. the worker contexts partition the tier's inner subgraphs (k = 2)
//      concurrently on their own streams, straight from the tier buffer;
//   2. segmented kernels over the whole tier mark the separators, count each
//      side (global look-back scans, one read-back of the child sizes), number
//      the separators, and write the children into the other tier buffer;
//   3. one CTA per leaf runs the minimum-degree elimination in shared memory.
// Launches are per tier, not per subgraph, except for the partitions.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "hp_internal.cuh"

namespace {

constexpr int32_t ND_LEAF = 120;      // subgraphs of at most this many vertices are leaves
constexpr float ND_UB = 1.05f;        // imbalance of the separator partitions
// The separator partitions coarsen to graphs of about leaf size when the caller's
// coarsen_to is 0, not to the 2-way rule's 16 vertices: the levels below that
// cost every subgraph's partition its launches (the deep tiers are bound by the
// launch rate of the worker threads) and buy nothing.
constexpr int32_t ND_COARSEN_TO = 128;
constexpr int ND_LEAF_THREADS = 128;  // one thread per leaf vertex
constexpr int ND_W = 2;               // 64-bit words of a leaf adjacency row (128 >= ND_LEAF)
static_assert(ND_LEAF <= 64 * ND_W && ND_LEAF <= ND_LEAF_THREADS, "leaf rows fit the bitsets and the CTA");

// Subgraph modes of a tier.
enum : int32_t { ND_SPLIT = 0, ND_LEAFMODE = 1, ND_VERTEX_ORDER = 2 };

// One tier in the batch layout.  xadj holds n_g + 1 local offsets per subgraph
// at vtx[g] + g; adjncy the local neighbour ids at edg[g].
struct Tier {
    int32_t *xadj, *adjncy, *vwgt, *label, *vsub;
};

__device__ __forceinline__ const int32_t *row_xadj(const Tier &t, const int64_t *vtx, int32_t g)
{
    return t.xadj + vtx[g] + g;
}

// Boundary flags (a neighbour on the other side) and their count per
// (subgraph, side), for the split subgraphs; warp-aggregated counts.
__global__ void __launch_bounds__(256)
nd_boundary_kernel(int64_t N, Tier t, const int64_t *__restrict__ vtx, const int64_t *__restrict__ edg,
                   const int32_t *__restrict__ mode, const int32_t *__restrict__ where, int8_t *__restrict__ bnd,
                   int32_t *__restrict__ bcnt)
{
    hp::pdl_wait();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int key = -1;
    if (i < N) {
        const int32_t g = t.vsub[i];
        bool b = false;
        if (mode[g] == ND_SPLIT) {
            const int32_t v = (int32_t)(i - vtx[g]);
            const int32_t *x = row_xadj(t, vtx, g);
            const int32_t *a = t.adjncy + edg[g];
            const int32_t *w = where + vtx[g];
            const int32_t s = w[v];
            for (int32_t j = x[v]; j < x[v + 1]; j++)
                if (w[a[j]] != s) { b = true; break; }
            if (b) key = 2 * g + s;
        }
        bnd[i] = b;
    }
    const unsigned peers = __match_any_sync(HP_FULL_MASK, key);
    if (key >= 0 && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&bcnt[key], __popc(peers));
}

// Separator rule: side a = the side with fewer boundary vertices (0 on a tie);
// a boundary vertex of side a stays in the separator (2) when it has a
// neighbour in the rest of side a, else it joins the other side.
__global__ void __launch_bounds__(256)
nd_separator_kernel(int64_t N, Tier t, const int64_t *__restrict__ vtx, const int64_t *__restrict__ edg,
                    const int32_t *__restrict__ mode, const int32_t *__restrict__ where,
                    const int8_t *__restrict__ bnd, const int32_t *__restrict__ bcnt, int32_t *__restrict__ side)
{
    hp::pdl_wait();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int32_t g = t.vsub[i];
    if (mode[g] != ND_SPLIT) { side[i] = 3; return; }
    const int32_t v = (int32_t)(i - vtx[g]);
    const int32_t s = where[i];
    const int32_t a = bcnt[2 * g] <= bcnt[2 * g + 1] ? 0 : 1;
    if (s != a || !bnd[i]) { side[i] = s; return; }
    const int32_t *x = row_xadj(t, vtx, g);
    const int32_t *adj = t.adjncy + edg[g];
    const int32_t *w = where + vtx[g];
    const int8_t *bb = bnd + vtx[g];
    bool keep = false;
    for (int32_t j = x[v]; j < x[v + 1]; j++) {
        const int32_t u = adj[j];
        if (w[u] == a && !bb[u]) { keep = true; break; }
    }
    side[i] = keep ? 2 : 1 - a;
}

// Scan inputs: flags of the left side, right side and separator, and the
// children's row lengths (neighbours on the same side).
__global__ void __launch_bounds__(256)
nd_count_kernel(int64_t N, Tier t, const int64_t *__restrict__ vtx, const int64_t *__restrict__ edg,
                const int32_t *__restrict__ side, int32_t *__restrict__ fl, int32_t *__restrict__ fr,
                int32_t *__restrict__ fs, int32_t *__restrict__ cl, int32_t *__restrict__ cr)
{
    hp::pdl_wait();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int32_t s = side[i];
    int32_t c = 0;
    if (s <= 1) {
        const int32_t g = t.vsub[i];
        const int32_t v = (int32_t)(i - vtx[g]);
        const int32_t *x = row_xadj(t, vtx, g);
        const int32_t *a = t.adjncy + edg[g];
        const int32_t *sd = side + vtx[g];
        for (int32_t j = x[v]; j < x[v + 1]; j++) c += sd[a[j]] == s;
    }
    fl[i] = s == 0;
    fr[i] = s == 1;
    fs[i] = s == 2;
    cl[i] = s == 0 ? c : 0;
    cr[i] = s == 1 ? c : 0;
}

// Per subgraph: left, right and separator sizes and the children's entry
// counts, from the exclusive scans at the subgraph's bounds.
__global__ void nd_sizes_kernel(int32_t G, const int64_t *__restrict__ vtx, const int32_t *__restrict__ sl,
                                const int32_t *__restrict__ sr, const int32_t *__restrict__ ss,
                                const int32_t *__restrict__ scl, const int32_t *__restrict__ scr,
                                int32_t *__restrict__ sizes)
{
    hp::pdl_wait();
    const int32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const int64_t a = vtx[g], b = vtx[g + 1];
    sizes[5 * g + 0] = sl[b] - sl[a];
    sizes[5 * g + 1] = sr[b] - sr[a];
    sizes[5 * g + 2] = ss[b] - ss[a];
    sizes[5 * g + 3] = scl[b] - scl[a];
    sizes[5 * g + 4] = scr[b] - scr[a];
}

// Numbers of the separators (increasing local id, the top of the subgraph's
// range) and of the subgraphs ordered by vertex id (no progress, or no edges
// beyond the leaf size).
__global__ void __launch_bounds__(256)
nd_number_kernel(int64_t N, Tier t, const int64_t *__restrict__ vtx, const int32_t *__restrict__ mode,
                 const int32_t *__restrict__ hi, const int32_t *__restrict__ side, const int32_t *__restrict__ ss,
                 const int32_t *__restrict__ sizes, int32_t *__restrict__ iperm)
{
    hp::pdl_wait();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int32_t g = t.vsub[i];
    const int32_t md = mode[g];
    const int64_t n = vtx[g + 1] - vtx[g];
    if (md == ND_VERTEX_ORDER) {
        iperm[t.label[i]] = hi[g] - (int32_t)n + (int32_t)(i - vtx[g]);
    } else if (md == ND_SPLIT && side[i] == 2) {
        const int32_t ns = sizes[5 * g + 2];
        iperm[t.label[i]] = hi[g] - ns + (ss[i] - ss[vtx[g]]);
    }
}

// Children of the split subgraphs into the next tier: a vertex of side s of
// subgraph g goes to child child[2g + s] with its rank on that side as local
// id; its row keeps the neighbours on the same side, in row order, renumbered.
__global__ void __launch_bounds__(256)
nd_split_kernel(int64_t N, Tier t, const int64_t *__restrict__ vtx, const int64_t *__restrict__ edg,
                const int32_t *__restrict__ side, const int32_t *__restrict__ sl, const int32_t *__restrict__ sr,
                const int32_t *__restrict__ scl, const int32_t *__restrict__ scr, const int32_t *__restrict__ child,
                Tier nt, const int64_t *__restrict__ nvtx, const int64_t *__restrict__ nedg)
{
    hp::pdl_wait();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int32_t s = side[i];
    if (s > 1) return;
    const int32_t g = t.vsub[i];
    const int32_t c = child[2 * g + s];
    if (c < 0) return;   // a split that made no progress: ordered by vertex id
    const int32_t *sc = s == 0 ? sl : sr;
    const int32_t *ec = s == 0 ? scl : scr;
    const int64_t base = vtx[g];
    const int32_t lid = sc[i] - sc[base];
    const int32_t eoff = ec[i] - ec[base];
    const int64_t o = nvtx[c] + lid;
    nt.label[o] = t.label[i];
    nt.vwgt[o] = t.vwgt[i];
    nt.vsub[o] = c;
    nt.xadj[nvtx[c] + c + lid] = eoff;
    const int32_t v = (int32_t)(i - base);
    const int32_t *x = row_xadj(t, vtx, g);
    const int32_t *a = t.adjncy + edg[g];
    const int32_t *sd = side + base;
    int32_t *out = nt.adjncy + nedg[c] + eoff;
    int32_t k = 0;
    for (int32_t j = x[v]; j < x[v + 1]; j++) {
        const int32_t u = a[j];
        if (sd[u] == s) out[k++] = sc[base + u] - sc[base];
    }
}

// The closing xadj entry (the entry count) of every child.
__global__ void nd_close_kernel(int32_t G, Tier nt, const int64_t *__restrict__ nvtx,
                                const int64_t *__restrict__ nedg)
{
    hp::pdl_wait();
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= G) return;
    nt.xadj[nvtx[c + 1] + c] = (int32_t)(nedg[c + 1] - nedg[c]);
}

// Exact minimum-degree elimination of a leaf (at most ND_LEAF vertices), one
// CTA per leaf: adjacency bitsets in shared memory; each step the live vertex
// of least degree (ties: lowest id) takes the next number and its live
// neighbours become a clique.
__global__ void __launch_bounds__(ND_LEAF_THREADS)
nd_leaf_kernel(const int32_t *__restrict__ leaves, Tier t, const int64_t *__restrict__ vtx,
               const int64_t *__restrict__ edg, const int32_t *__restrict__ hi, int32_t *__restrict__ iperm)
{
    hp::pdl_wait();
    __shared__ unsigned long long adj[ND_LEAF][ND_W];
    __shared__ unsigned long long alive[ND_W];
    __shared__ unsigned long long s_key[ND_LEAF_THREADS / 32];
    __shared__ int32_t s_best;
    const int32_t g = leaves[blockIdx.x];
    const int32_t n = (int32_t)(vtx[g + 1] - vtx[g]);
    const int32_t lo = hi[g] - n;
    const int32_t *x = row_xadj(t, vtx, g);
    const int32_t *a = t.adjncy + edg[g];
    const int32_t *label = t.label + vtx[g];
    const int v = threadIdx.x;
    if (v < n) {
        unsigned long long r[ND_W] = {};
        for (int32_t j = x[v]; j < x[v + 1]; j++) r[a[j] >> 6] |= 1ull << (a[j] & 63);
        for (int w = 0; w < ND_W; w++) adj[v][w] = r[w];
    }
    if (v < ND_W) {
        const int lo_bit = 64 * v;
        const int cnt = n - lo_bit;
        alive[v] = cnt <= 0 ? 0ull : (cnt >= 64 ? ~0ull : ((1ull << cnt) - 1ull));
    }
    __syncthreads();
    for (int32_t step = 0; step < n; step++) {
        // key = degree << 32 | id; the minimum over the live vertices
        unsigned long long key = ~0ull;
        if (v < n && (alive[v >> 6] >> (v & 63) & 1ull)) {
            int d = 0;
#pragma unroll
            for (int w = 0; w < ND_W; w++) d += __popcll(adj[v][w] & alive[w]);
            key = ((unsigned long long)d << 32) | (unsigned)v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long k2 = __shfl_xor_sync(HP_FULL_MASK, key, o);
            key = k2 < key ? k2 : key;
        }
        if ((v & 31) == 0) s_key[v >> 5] = key;
        __syncthreads();
        if (v == 0) {
            unsigned long long k = s_key[0];
            for (int w = 1; w < ND_LEAF_THREADS / 32; w++) k = s_key[w] < k ? s_key[w] : k;
            const int32_t b = (int32_t)(k & 0xffffffffu);
            s_best = b;
            iperm[label[b]] = lo + step;
            alive[b >> 6] &= ~(1ull << (b & 63));
        }
        __syncthreads();
        const int32_t b = s_best;
        unsigned long long nb[ND_W];
#pragma unroll
        for (int w = 0; w < ND_W; w++) nb[w] = adj[b][w] & alive[w];
        __syncthreads();   // every thread has read row b before any row changes
        if (v < n && (nb[v >> 6] >> (v & 63) & 1ull)) {
#pragma unroll
            for (int w = 0; w < ND_W; w++) adj[v][w] |= nb[w];
            adj[v][v >> 6] &= ~(1ull << (v & 63));
        }
        __syncthreads();
    }
}

inline unsigned nd_blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + 255) / 256); }

// Device buffers of one tier (capacities from the input: a tier never holds
// more vertices, entries or subgraphs than the input has vertices/entries).
struct TierBuf {
    Tier t{};
    int64_t *d_vtx = nullptr, *d_edg = nullptr;
    int32_t *d_mode = nullptr, *d_hi = nullptr;
};

}  // namespace

#define HP_API extern "C" __attribute__((visibility("default")))

HP_API int hp_node_nd(hp_context *ctx, int32_t nvtxs, const int32_t *xadj, const int32_t *adjncy,
                      const int32_t *vwgt, const hp_options *opt, int32_t *perm, int32_t *iperm)
{
    if (!ctx || nvtxs < 0 || !xadj || (nvtxs > 0 && !adjncy) || !iperm) return HP_ERR_INVALID_ARG;
    if (opt && opt->version != HP_OPTIONS_VERSION) return HP_ERR_INVALID_ARG;
    const int64_t n = nvtxs, m = xadj[nvtxs];
    if (xadj[0] != 0 || m < 0 || m > INT32_MAX) return HP_ERR_INVALID_GRAPH;
    if (n == 0) return HP_OK;
    HP_CUDA(cudaSetDevice(ctx->device));
    hp_context *c = ctx;
    c->stream = c->own_stream;
    c->launches = 0;
    memset(&c->stats, 0, sizeof(c->stats));
    hp_options popt;
    if (opt) popt = *opt;
    else hp_options_default(&popt);
    popt.trace = 0;
    popt.profile = 0;
    if (popt.coarsen_to <= 0) popt.coarsen_to = ND_COARSEN_TO;

    // two tier buffers, plus the per-vertex work arrays of the current tier
    const int64_t cap_x = 2 * n + 1;
    std::vector<void *> allocs;
    auto dalloc = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes > 0 ? bytes : 1) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        allocs.push_back(p);
        return p;
    };
    auto release = [&]() {
        for (void *p : allocs) cudaFree(p);
        allocs.clear();
    };
    TierBuf tb[2];
    bool ok = true;
    for (auto &b : tb) {
        b.t.xadj = (int32_t *)dalloc(sizeof(int32_t) * (size_t)cap_x);
        b.t.adjncy = (int32_t *)dalloc(sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1));
        b.t.vwgt = (int32_t *)dalloc(sizeof(int32_t) * (size_t)n);
        b.t.label = (int32_t *)dalloc(sizeof(int32_t) * (size_t)n);
        b.t.vsub = (int32_t *)dalloc(sizeof(int32_t) * (size_t)n);
        b.d_vtx = (int64_t *)dalloc(sizeof(int64_t) * (size_t)(n + 1));
        b.d_edg = (int64_t *)dalloc(sizeof(int64_t) * (size_t)(n + 1));
        b.d_mode = (int32_t *)dalloc(sizeof(int32_t) * (size_t)n);
        b.d_hi = (int32_t *)dalloc(sizeof(int32_t) * (size_t)n);
        ok = ok && b.t.xadj && b.t.adjncy && b.t.vwgt && b.t.label && b.t.vsub && b.d_vtx && b.d_edg && b.d_mode &&
             b.d_hi;
    }
    int32_t *where = (int32_t *)dalloc(sizeof(int32_t) * (size_t)n);
    int32_t *side = (int32_t *)dalloc(sizeof(int32_t) * (size_t)n);
    int8_t *bnd = (int8_t *)dalloc((size_t)n);
    int32_t *scans = (int32_t *)dalloc(sizeof(int32_t) * 5 * (size_t)(n + 1));
    int32_t *bcnt = (int32_t *)dalloc(sizeof(int32_t) * 2 * (size_t)n);
    int32_t *sizes = (int32_t *)dalloc(sizeof(int32_t) * 5 * (size_t)n);
    int32_t *child = (int32_t *)dalloc(sizeof(int32_t) * 2 * (size_t)n);
    int32_t *leaves = (int32_t *)dalloc(sizeof(int32_t) * (size_t)n);
    int32_t *d_iperm = (int32_t *)dalloc(sizeof(int32_t) * (size_t)n);
    ok = ok && where && side && bnd && scans && bcnt && sizes && child && leaves && d_iperm;
    if (!ok) {
        release();
        return HP_ERR_NOMEM;
    }
    int32_t *sl = scans, *sr = scans + (n + 1), *ss = scans + 2 * (n + 1), *scl = scans + 3 * (n + 1),
            *scr = scans + 4 * (n + 1);
    int rc = HP_OK;
    int root_kernels = 0;
    auto fail = [&](int code) {
        cudaStreamSynchronize(c->stream);
        release();
        return code;
    };

    // tier 0: the input graph (vertex weights, or 1)
    std::vector<int64_t> hvtx{0, n}, hedg{0, m};
    std::vector<int32_t> hhi{(int32_t)n};
    {
        std::vector<int32_t> lab(n), vs(n, 0), vw(n);
        std::iota(lab.begin(), lab.end(), 0);
        for (int64_t v = 0; v < n; v++) vw[v] = vwgt ? vwgt[v] : 1;
        Tier &t = tb[0].t;
        if (cudaMemcpyAsync(t.xadj, xadj, sizeof(int32_t) * (size_t)(n + 1), cudaMemcpyHostToDevice, c->stream) ||
            (m > 0 && cudaMemcpyAsync(t.adjncy, adjncy, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice,
                                      c->stream)) ||
            cudaMemcpyAsync(t.vwgt, vw.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, c->stream) ||
            cudaMemcpyAsync(t.label, lab.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, c->stream) ||
            cudaMemcpyAsync(t.vsub, vs.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, c->stream) ||
            cudaStreamSynchronize(c->stream)) {
            cudaGetLastError();
            return fail(HP_ERR_CUDA);
        }
    }
    // The root's 2-way partition runs on this context with the caller's
    // validation setting, so an invalid input fails here as it would in
    // hp_partition; its result is the root's separator partition when the
    // root is an inner subgraph (validation does not change a partition).
    {
        int64_t cut = 0;
        rc = hp_partition_device(c, (int32_t)n, m, tb[0].t.xadj, tb[0].t.adjncy, tb[0].t.vwgt, nullptr, 2, nullptr,
                                 ND_UB, &popt, c->own_stream, where, &cut);
        if (rc != HP_OK) return fail(rc);
        c->stream = c->own_stream;
        root_kernels = c->stats.kernel_launches;
        c->launches = 0;
    }
    HP_TRY(hp_lb_reserve(c, (n + 1 + 4095) / 4096 + 1024));
    const int nworkers = c->tune.batch_workers;
    if ((rc = hp_ensure_workers(c, nworkers)) != HP_OK) return fail(rc);
    hp_options wopt = popt;
    wopt.validate = 0;
    wopt.eager = 1;   // the partitions of small subgraphs never amortise a pass graph

    int cur = 0;
    int64_t tiers = 0, partitions = 0, worker_launches = 0;
    const int root_launches = root_kernels;
    while (hvtx.size() > 1) {
        const int32_t G = (int32_t)(hvtx.size() - 1);
        const int64_t N = hvtx[G];
        TierBuf &B = tb[cur], &NB = tb[cur ^ 1];
        tiers++;
        // modes: split (inner), leaf (minimum degree) or vertex order (no edges, large)
        std::vector<int32_t> hmode(G);
        std::vector<int32_t> inner;
        std::vector<int32_t> hleaves;
        for (int32_t g = 0; g < G; g++) {
            const int64_t ng = hvtx[g + 1] - hvtx[g], mg = hedg[g + 1] - hedg[g];
            if (ng > ND_LEAF && mg > 0) { hmode[g] = ND_SPLIT; inner.push_back(g); }
            else if (mg > 0) { hmode[g] = ND_LEAFMODE; hleaves.push_back(g); }
            else hmode[g] = ND_VERTEX_ORDER;
        }
        if (cudaMemcpyAsync(B.d_vtx, hvtx.data(), sizeof(int64_t) * (G + 1), cudaMemcpyHostToDevice, c->stream) ||
            cudaMemcpyAsync(B.d_edg, hedg.data(), sizeof(int64_t) * (G + 1), cudaMemcpyHostToDevice, c->stream) ||
            cudaMemcpyAsync(B.d_mode, hmode.data(), sizeof(int32_t) * G, cudaMemcpyHostToDevice, c->stream) ||
            cudaMemcpyAsync(B.d_hi, hhi.data(), sizeof(int32_t) * G, cudaMemcpyHostToDevice, c->stream) ||
            (!hleaves.empty() && cudaMemcpyAsync(leaves, hleaves.data(), sizeof(int32_t) * hleaves.size(),
                                                 cudaMemcpyHostToDevice, c->stream)) ||
            cudaStreamSynchronize(c->stream)) {
            cudaGetLastError();
            return fail(HP_ERR_CUDA);
        }
        // 1. the inner subgraphs' 2-way partitions, concurrently on the workers
        // (the root's ran above)
        if (!inner.empty() && tiers > 1) {
            std::atomic<size_t> next{0};
            std::atomic<int> err{HP_OK};
            std::atomic<long long> wl{0};
            const int nw = (int)std::min<size_t>(inner.size(), (size_t)nworkers);
            auto work = [&](hp_context *w) {
                cudaSetDevice(w->device);
                for (;;) {
                    if (err.load() != HP_OK) return;
                    const size_t q = next.fetch_add(1);
                    if (q >= inner.size()) return;
                    const int32_t g = inner[q];
                    const int64_t v0 = hvtx[g], ng = hvtx[g + 1] - v0, e0 = hedg[g], mg = hedg[g + 1] - e0;
                    int64_t cut = 0;
                    const int r = hp_partition_device(w, (int32_t)ng, mg, B.t.xadj + v0 + g, B.t.adjncy + e0,
                                                      B.t.vwgt + v0, nullptr, 2, nullptr, ND_UB, &wopt, nullptr,
                                                      where + v0, &cut);
                    if (r != HP_OK) {
                        int expected = HP_OK;
                        err.compare_exchange_strong(expected, r);
                        return;
                    }
                    wl += w->stats.kernel_launches;
                }
            };
            std::vector<std::thread> pool;
            for (int t = 0; t < nw; t++) pool.emplace_back(work, c->workers[t]);
            for (auto &t : pool) t.join();
            if (err.load() != HP_OK) return fail(err.load());
            worker_launches += wl.load();
        }
        partitions += (int64_t)inner.size();
        // 2. separators, side counts and numbering over the whole tier
        if (cudaMemsetAsync(bcnt, 0, sizeof(int32_t) * 2 * (size_t)G, c->stream)) return fail(HP_ERR_CUDA);
        auto launch_ok = [&]() {
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) fprintf(stderr, "hp_node_nd: launch failed: %s\n", cudaGetErrorString(e));
            return e == cudaSuccess;
        };
        nd_boundary_kernel<<<nd_blocks(N), 256, 0, c->stream>>>(N, B.t, B.d_vtx, B.d_edg, B.d_mode, where, bnd,
                                                                  bcnt);
        nd_separator_kernel<<<nd_blocks(N), 256, 0, c->stream>>>(N, B.t, B.d_vtx, B.d_edg, B.d_mode, where, bnd,
                                                                   bcnt, side);
        nd_count_kernel<<<nd_blocks(N), 256, 0, c->stream>>>(N, B.t, B.d_vtx, B.d_edg, side, sl, sr, ss, scl, scr);
        c->launches += 3;
        if (!launch_ok()) return fail(HP_ERR_CUDA);
        for (int32_t *a : {sl, sr, ss, scl, scr})
            if ((rc = hp_scan_excl(c, a, a, N)) != HP_OK) return fail(rc);
        nd_sizes_kernel<<<nd_blocks(G), 256, 0, c->stream>>>(G, B.d_vtx, sl, sr, ss, scl, scr, sizes);
        c->launches++;
        if (!launch_ok()) return fail(HP_ERR_CUDA);
        std::vector<int32_t> hs(5 * (size_t)G);
        if (cudaMemcpyAsync(hs.data(), sizes, sizeof(int32_t) * hs.size(), cudaMemcpyDeviceToHost, c->stream) ||
            cudaStreamSynchronize(c->stream)) {
            cudaGetLastError();
            return fail(HP_ERR_CUDA);
        }
        // the next tier: the left and right children of every split subgraph
        // (in subgraph order, left first); a split without progress orders
        // its subgraph by vertex id instead
        std::vector<int64_t> nvtx{0}, nedg{0};
        std::vector<int32_t> nhi, hchild(2 * (size_t)G, -1);
        bool mode_changed = false;
        for (int32_t g : inner) {
            const int64_t ng = hvtx[g + 1] - hvtx[g];
            const int32_t nl = hs[5 * g], nr = hs[5 * g + 1], ns = hs[5 * g + 2];
            if (nl == ng || nr == ng) {
                hmode[g] = ND_VERTEX_ORDER;
                mode_changed = true;
                continue;
            }
            const int32_t top = hhi[g];
            const int32_t part_hi[2] = {top - ns - nr, top - ns};
            const int32_t part_n[2] = {nl, nr};
            const int32_t part_m[2] = {hs[5 * g + 3], hs[5 * g + 4]};
            for (int s = 0; s < 2; s++) {
                if (part_n[s] == 0) continue;
                hchild[2 * (size_t)g + s] = (int32_t)nhi.size();
                nhi.push_back(part_hi[s]);
                nvtx.push_back(nvtx.back() + part_n[s]);
                nedg.push_back(nedg.back() + part_m[s]);
            }
        }
        if (mode_changed &&
            cudaMemcpyAsync(B.d_mode, hmode.data(), sizeof(int32_t) * G, cudaMemcpyHostToDevice, c->stream))
            return fail(HP_ERR_CUDA);
        nd_number_kernel<<<nd_blocks(N), 256, 0, c->stream>>>(N, B.t, B.d_vtx, B.d_mode, B.d_hi, side, ss, sizes,
                                                                d_iperm);
        c->launches++;
        // 3. the leaves
        if (!hleaves.empty()) {
            nd_leaf_kernel<<<(unsigned)hleaves.size(), ND_LEAF_THREADS, 0, c->stream>>>(leaves, B.t, B.d_vtx,
                                                                                          B.d_edg, B.d_hi, d_iperm);
            c->launches++;
        }
        if (!launch_ok()) return fail(HP_ERR_CUDA);
        const int32_t G2 = (int32_t)nhi.size();
        if (G2 > 0) {
            if (cudaMemcpyAsync(child, hchild.data(), sizeof(int32_t) * hchild.size(), cudaMemcpyHostToDevice,
                                c->stream) ||
                cudaMemcpyAsync(NB.d_vtx, nvtx.data(), sizeof(int64_t) * (G2 + 1), cudaMemcpyHostToDevice, c->stream) ||
                cudaMemcpyAsync(NB.d_edg, nedg.data(), sizeof(int64_t) * (G2 + 1), cudaMemcpyHostToDevice, c->stream))
                return fail(HP_ERR_CUDA);
            // (the vertices of a split without progress have no child: child = -1)
            nd_split_kernel<<<nd_blocks(N), 256, 0, c->stream>>>(N, B.t, B.d_vtx, B.d_edg, side, sl, sr, scl, scr,
                                                                   child, NB.t, NB.d_vtx, NB.d_edg);
            nd_close_kernel<<<nd_blocks(G2), 256, 0, c->stream>>>(G2, NB.t, NB.d_vtx, NB.d_edg);
            c->launches += 2;
            if (!launch_ok()) return fail(HP_ERR_CUDA);
        }
        if (cudaStreamSynchronize(c->stream)) return fail(HP_ERR_CUDA);
        hvtx.swap(nvtx);
        hedg.swap(nedg);
        hhi.swap(nhi);
        cur ^= 1;
    }
    if (cudaMemcpyAsync(iperm, d_iperm, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, c->stream) ||
        cudaStreamSynchronize(c->stream))
        return fail(HP_ERR_CUDA);
    release();
    if (perm)
        for (int64_t v = 0; v < n; v++) perm[iperm[v]] = (int32_t)v;
    c->stats.nlevels = (int32_t)tiers;              // recursion depths
    c->stats.refine_passes = (int32_t)std::min<int64_t>(partitions, INT32_MAX);   // subgraph partitions
    c->stats.kernel_launches =
        (int32_t)std::min<long long>((long long)c->launches + root_launches + worker_launches, INT32_MAX);
    return hp_check_status(c);
}
