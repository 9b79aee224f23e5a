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

namespace {

struct SubInfo {
    int32_t vbeg, n;
    int32_t tbeg, ntr;
    int64_t tv, want1, onemin, onemax;
    int64_t slab_off;
};

__host__ __device__ inline int64_t slab_bytes(int32_t n)
{
    return (((int64_t)3 * n + 15) & ~(int64_t)15) + (int64_t)36 * n + 16;
}

// ---- device max-heap ordered by (key desc, vertex asc) ----------------------
struct DHeap {
    int32_t *heap, *pos, *key;
    int32_t len;
    __device__ __forceinline__ bool above(int32_t a, int32_t b) const
    {
        int32_t ka = key[a], kb = key[b];
        return ka > kb || (ka == kb && a < b);
    }
    __device__ void up(int32_t i)
    {
        int32_t v = heap[i];
        while (i > 0) {
            int32_t p = (i - 1) >> 1;
            if (!above(v, heap[p])) break;
            heap[i] = heap[p];
            pos[heap[i]] = i;
            i = p;
        }
        heap[i] = v;
        pos[v] = i;
    }
    __device__ void down(int32_t i)
    {
        int32_t v = heap[i];
        for (;;) {
            int32_t l = 2 * i + 1, r = l + 1, b = i, bv = v;
            if (l < len && above(heap[l], bv)) { b = l; bv = heap[l]; }
            if (r < len && above(heap[r], bv)) { b = r; bv = heap[r]; }
            if (b == i) break;
            heap[i] = bv;
            pos[bv] = i;
            i = b;
        }
        heap[i] = v;
        pos[v] = i;
    }
    __device__ void insert(int32_t v, int32_t k)
    {
        key[v] = k;
        heap[len] = v;
        pos[v] = len;
        len++;
        up(len - 1);
    }
    __device__ void remove(int32_t v)
    {
        int32_t i = pos[v];
        pos[v] = -1;
        len--;
        if (i == len) return;
        int32_t last = heap[len];
        heap[i] = last;
        pos[last] = i;
        up(i);
        down(pos[last]);
    }
    __device__ void update(int32_t v, int32_t k)
    {
        key[v] = k;
        up(pos[v]);
        down(pos[v]);
    }
    __device__ int32_t pop()
    {
        if (len == 0) return -1;
        int32_t v = heap[0];
        remove(v);
        return v;
    }
};

// One BFS-growth + FM bisection trial per thread.
__global__ void __launch_bounds__(128)
trial_kernel(const SubInfo *__restrict__ subs, const int32_t *__restrict__ trial_sub,
             int32_t ntrials, const int32_t *__restrict__ fxadj, const int32_t *__restrict__ fadj,
             const int32_t *__restrict__ fwgt, const int32_t *__restrict__ fvwgt, char *slab_base,
             int32_t starts, int32_t fm_passes, int64_t *tr_cut, int64_t *tr_viol)
{
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntrials) return;
    const SubInfo S = subs[trial_sub[t]];
    const int32_t lt = t - S.tbeg;
    const int32_t n = S.n;
    const int32_t *xadj = fxadj + S.vbeg;   // global edge offsets, local neighbour ids
    const int32_t *vwgt = fvwgt + S.vbeg;
    char *slab = slab_base + S.slab_off + (int64_t)lt * slab_bytes(n);
    int8_t *where = (int8_t *)slab;
    int8_t *bnd = where + n;
    int8_t *vis = bnd + n;
    int32_t *ip = (int32_t *)(slab + (((int64_t)3 * n + 15) & ~(int64_t)15));
    int32_t *id = ip, *ed = ip + n, *moved = ip + 2 * n, *swaps = ip + 3 * n, *pos = ip + 4 * n;
    int32_t *key = ip + 5 * n, *heap0 = ip + 6 * n, *heap1 = ip + 7 * n, *queue = ip + 8 * n;
    const int32_t start = (n <= starts) ? lt : (int32_t)(((int64_t)lt * n) / starts);
    const int64_t tv = S.tv, want1 = S.want1, onemin = S.onemin, onemax = S.onemax;
    int64_t pw0 = 0, pw1 = tv;

    // BFS growth of side 0 (hunyuangraph_CPU_initialpartition.h:66-120)
    for (int32_t v = 0; v < n; v++) { where[v] = 1; vis[v] = 0; }
    int32_t first = 0, last = 1, nleft = n - 1, next_unvis = 0;
    bool drain = false;
    queue[0] = start;
    vis[start] = 1;
    for (;;) {
        if (first == last) {
            if (nleft == 0 || drain) break;
            while (vis[next_unvis]) next_unvis++;
            queue[0] = next_unvis;
            vis[next_unvis] = 1;
            first = 0; last = 1; nleft--;
        }
        int32_t i = queue[first++];
        if (pw0 > 0 && pw1 - vwgt[i] < onemin) { drain = true; continue; }
        where[i] = 0;
        pw0 += vwgt[i]; pw1 -= vwgt[i];
        if (pw1 <= onemax) break;
        drain = false;
        for (int32_t j = xadj[i]; j < xadj[i + 1]; j++) {
            int32_t k = fadj[j];
            if (!vis[k]) { queue[last++] = k; vis[k] = 1; nleft--; }
        }
    }

    // 2-way FM (hunyuangraph_CPU_2wayrefine.h:77-245)
    int64_t cut = 0;
    for (int32_t v = 0; v < n; v++) {
        int32_t tid = 0, ted = 0;
        const int8_t wv = where[v];
        for (int32_t j = xadj[v]; j < xadj[v + 1]; j++) {
            if (where[fadj[j]] == wv) tid += fwgt[j];
            else ted += fwgt[j];
        }
        id[v] = tid; ed[v] = ted;
        bnd[v] = (ted > 0 || xadj[v] == xadj[v + 1]);
        cut += ted;
        moved[v] = -1;
        pos[v] = -1;
    }
    cut /= 2;
    const int64_t tpw0 = tv - want1, tpw1 = want1;
    int64_t limit = n / 100;
    if (limit < 15) limit = 15;
    if (limit > 100) limit = 100;
    int64_t avgvwgt = (pw0 + pw1) / 20;
    if (n > 0 && 2 * (pw0 + pw1) / n < avgvwgt) avgvwgt = 2 * (pw0 + pw1) / n;
    const int64_t origdiff = hp::iabs64(tpw0 - pw0);
    DHeap q[2];
    q[0].heap = heap0; q[1].heap = heap1;
    q[0].pos = q[1].pos = pos;
    q[0].key = q[1].key = key;
    for (int32_t pass = 0; pass < fm_passes; pass++) {
        q[0].len = q[1].len = 0;
        for (int32_t v = 0; v < n; v++) pos[v] = -1;
        int64_t mincutorder = -1;
        int64_t newcut = cut, mincut = cut, initcut = cut;
        int64_t mindiff = hp::iabs64(tpw0 - pw0);
        for (int32_t v = 0; v < n; v++)
            if (bnd[v]) q[where[v]].insert(v, ed[v] - id[v]);
        int32_t nswaps;
        for (nswaps = 0; nswaps < n; nswaps++) {
            int from = (tpw0 - pw0 < tpw1 - pw1) ? 0 : 1;
            int to = 1 - from;
            int32_t h = q[from].pop();
            if (h < 0) break;
            newcut -= (ed[h] - id[h]);
            if (to == 0) { pw0 += vwgt[h]; pw1 -= vwgt[h]; } else { pw1 += vwgt[h]; pw0 -= vwgt[h]; }
            if ((newcut < mincut && hp::iabs64(tpw0 - pw0) <= origdiff + avgvwgt) ||
                (newcut == mincut && hp::iabs64(tpw0 - pw0) < mindiff)) {
                mincut = newcut;
                mindiff = hp::iabs64(tpw0 - pw0);
                mincutorder = nswaps;
            } else if (nswaps - mincutorder > limit) {
                newcut += (ed[h] - id[h]);
                if (to == 0) { pw0 -= vwgt[h]; pw1 += vwgt[h]; } else { pw1 -= vwgt[h]; pw0 += vwgt[h]; }
                break;
            }
            where[h] = (int8_t)to;
            moved[h] = nswaps;
            swaps[nswaps] = h;
            { int32_t tt = id[h]; id[h] = ed[h]; ed[h] = tt; }
            if (ed[h] == 0 && xadj[h] < xadj[h + 1]) bnd[h] = 0;
            for (int32_t j = xadj[h]; j < xadj[h + 1]; j++) {
                int32_t k = fadj[j];
                int32_t kw = (to == where[k]) ? fwgt[j] : -fwgt[j];
                id[k] += kw; ed[k] -= kw;
                if (bnd[k]) {
                    if (ed[k] == 0) {
                        bnd[k] = 0;
                        if (moved[k] == -1 && pos[k] >= 0) q[where[k]].remove(k);
                    } else if (moved[k] == -1 && pos[k] >= 0) {
                        q[where[k]].update(k, ed[k] - id[k]);
                    }
                } else if (ed[k] > 0) {
                    bnd[k] = 1;
                    if (moved[k] == -1) q[where[k]].insert(k, ed[k] - id[k]);
                }
            }
        }
        for (int32_t i = 0; i < nswaps; i++) moved[swaps[i]] = -1;
        for (nswaps--; nswaps > mincutorder; nswaps--) {
            int32_t h = swaps[nswaps];
            int to = 1 - where[h];
            where[h] = (int8_t)to;
            { int32_t tt = id[h]; id[h] = ed[h]; ed[h] = tt; }
            if (ed[h] == 0 && bnd[h] && xadj[h] < xadj[h + 1]) bnd[h] = 0;
            else if (ed[h] > 0 && !bnd[h]) bnd[h] = 1;
            if (to == 0) { pw0 += vwgt[h]; pw1 -= vwgt[h]; } else { pw1 += vwgt[h]; pw0 -= vwgt[h]; }
            for (int32_t j = xadj[h]; j < xadj[h + 1]; j++) {
                int32_t k = fadj[j];
                int32_t kw = (to == where[k]) ? fwgt[j] : -fwgt[j];
                id[k] += kw; ed[k] -= kw;
                if (bnd[k] && ed[k] == 0) bnd[k] = 0;
                if (!bnd[k] && ed[k] > 0) bnd[k] = 1;
            }
        }
        cut = mincut;
        if (mincutorder <= 0 || mincut == initcut) break;
    }
    int64_t viol = 0;
    if (pw1 > onemax) viol += pw1 - onemax;
    if (pw1 < onemin) viol += onemin - pw1;
    tr_cut[t] = cut;
    tr_viol[t] = viol;
}

// Best trial of every subgraph: min (violation, cut, trial index); copies its
// sides into side[] and reports the side-0 vertex count and weight.
__global__ void __launch_bounds__(256)
select_kernel(const SubInfo *__restrict__ subs, const int64_t *__restrict__ tr_cut,
              const int64_t *__restrict__ tr_viol, const char *slab_base,
              const int32_t *__restrict__ fvwgt, int32_t *__restrict__ side,
              int64_t *__restrict__ res /* per sub: n0, tv0 */)
{
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
    const int8_t *w = (const int8_t *)(slab_base + S.slab_off + (int64_t)s_best * slab_bytes(S.n));
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
    const SubInfo S = subs[blockIdx.x];
    for (int i = threadIdx.x; i < S.n; i += blockDim.x) sub_of[S.vbeg + i] = blockIdx.x;
    (void)flag0;
}

__global__ void __launch_bounds__(256)
side_flag_kernel(int32_t nf, const int32_t *__restrict__ side, int32_t *__restrict__ f0)
{
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
    int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) where[v] = value;
}

__global__ void copy_kernel(int64_t n, const int32_t *src, int32_t *dst)
{
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
            slab_total += (int64_t)I.ntr * slab_bytes(H.n);
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
        const int tok = hp_prof_begin(c);
        HP_LAUNCH(c, trial_kernel, nblk(tcount, 128), 128, 0, d_info, d_tsub, tcount, fxadj, fadj, fwgt,
                  fvwgt, slab, starts, fm_passes, d_cut, d_viol);
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
