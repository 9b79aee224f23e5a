// hp_mlp.cu — training and stand-alone inference of the move-scoring MLP, and
// the move log the plain refiner records for training.
//
// No counterpart in the reference (its refinement has no learned component).
// Training is plain FP32 on CUDA cores (mini-batch Adam; the network has 1,377
// parameters; gradients summed in a fixed order, so training is reproducible), inference inside refinement is BF16 tensor-core MMA with FP32
// accumulation (hp_mlp.cuh).  The network only proposes: an LP candidate it
// scores below the threshold is dropped before the exact integer afterburner,
// and every accepted move is still checked and applied in integers.
#include "hp_internal.cuh"
#include "hp_mlp.cuh"

namespace {

constexpr int MLP_BLOCK = 128;

// FP32 forward of one sample; h1/h2 pre-activation kept for the backward.
__device__ __forceinline__ float mlp_fwd(const float *__restrict__ P, const float x[HP_MLP_IN],
                                         float z1[HP_MLP_H], float z2[HP_MLP_H])
{
    float a1[HP_MLP_H];
    for (int j = 0; j < HP_MLP_H; j++) {
        float s = P[HP_MLP_OFF_B1 + j];
        for (int i = 0; i < HP_MLP_IN; i++) s += P[HP_MLP_OFF_W1 + j * HP_MLP_IN + i] * x[i];
        z1[j] = s;
        a1[j] = fmaxf(s, 0.f);
    }
    float y = P[HP_MLP_OFF_B3];
    for (int j = 0; j < HP_MLP_H; j++) {
        float s = P[HP_MLP_OFF_B2 + j];
        for (int i = 0; i < HP_MLP_H; i++) s += P[HP_MLP_OFF_W2 + j * HP_MLP_H + i] * a1[i];
        z2[j] = s;
        y += P[HP_MLP_OFF_W3 + j] * fmaxf(s, 0.f);
    }
    return y;
}

// Gradient of the mean binary cross-entropy (with logits), deterministic: no
// float atomics, so the same samples and parameters give the same gradient bit
// for bit on every run.  Two kernels per chunk of at most MLP_CHUNK samples:
//   mlp_sample_grad_kernel  one thread per sample writes that sample's scaled
//                           gradient (HP_MLP_NPARAM values) and loss term
//                           parameter-major into G[(p) * nb + s] (coalesced:
//                           consecutive threads, consecutive samples);
//   mlp_reduce_kernel       one block per parameter (and one for the loss) sums
//                           its row in a fixed order -- strided per thread, then
//                           a fixed shuffle tree -- and adds it to g[p].
// Chunks are reduced one after another, so the order of every sum is fixed.
constexpr int64_t MLP_CHUNK = 8192;
constexpr int MLP_RED = 256;
constexpr int MLP_ROWS = HP_MLP_NPARAM + 1;   // the parameters, then the loss

__global__ void __launch_bounds__(MLP_BLOCK)
mlp_sample_grad_kernel(const float *__restrict__ P, const float *__restrict__ X, const float *__restrict__ Y,
                       const int32_t *__restrict__ idx, int64_t b0, int64_t nb, float scale,
                       float *__restrict__ G)
{
    hp::pdl_wait();
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= nb) return;
    const int64_t r = idx ? idx[b0 + s] : b0 + s;
    float x[HP_MLP_IN], z1[HP_MLP_H], z2[HP_MLP_H];
    for (int i = 0; i < HP_MLP_IN; i++) x[i] = X[r * HP_MLP_IN + i];
    const float y = mlp_fwd(P, x, z1, z2);
    const float t = Y[r];
    // loss = softplus(y) - t*y ; dL/dy = sigmoid(y) - t
    const float sp = y > 0 ? y + log1pf(__expf(-y)) : log1pf(__expf(y));
    G[(int64_t)HP_MLP_NPARAM * nb + s] = (sp - t * y) * scale;
    const float dy = (1.f / (1.f + __expf(-y)) - t) * scale;
    G[(int64_t)HP_MLP_OFF_B3 * nb + s] = dy;
    float da1[HP_MLP_H];
    for (int i = 0; i < HP_MLP_H; i++) da1[i] = 0.f;
    for (int j = 0; j < HP_MLP_H; j++) {
        G[(int64_t)(HP_MLP_OFF_W3 + j) * nb + s] = dy * fmaxf(z2[j], 0.f);
        const float dz2 = z2[j] > 0.f ? dy * P[HP_MLP_OFF_W3 + j] : 0.f;
        G[(int64_t)(HP_MLP_OFF_B2 + j) * nb + s] = dz2;
        for (int i = 0; i < HP_MLP_H; i++) {
            G[(int64_t)(HP_MLP_OFF_W2 + j * HP_MLP_H + i) * nb + s] = dz2 * fmaxf(z1[i], 0.f);
            da1[i] += dz2 * P[HP_MLP_OFF_W2 + j * HP_MLP_H + i];
        }
    }
    for (int i = 0; i < HP_MLP_H; i++) {
        const float dz1 = z1[i] > 0.f ? da1[i] : 0.f;
        G[(int64_t)(HP_MLP_OFF_B1 + i) * nb + s] = dz1;
        for (int c = 0; c < HP_MLP_IN; c++) G[(int64_t)(HP_MLP_OFF_W1 + i * HP_MLP_IN + c) * nb + s] = dz1 * x[c];
    }
}

// Row p of G (nb samples) summed in a fixed order and added to out[p] (p <
// HP_MLP_NPARAM) or to *loss (p = HP_MLP_NPARAM, when loss is set).
__global__ void __launch_bounds__(MLP_RED)
mlp_reduce_kernel(const float *__restrict__ G, int64_t nb, float *__restrict__ out, float *__restrict__ loss)
{
    hp::pdl_wait();
    __shared__ float sw[MLP_RED / 32];
    const int p = blockIdx.x;
    const float *row = G + (int64_t)p * nb;
    float acc = 0.f;
    for (int64_t s = threadIdx.x; s < nb; s += MLP_RED) acc += row[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(HP_FULL_MASK, acc, o);
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < MLP_RED / 32; w++) t += sw[w];
        if (p < HP_MLP_NPARAM) out[p] += t;
        else if (loss) *loss += t;
    }
}

// Gradient (and loss) of samples [b0, b0 + nb) of the index list, scaled by
// `scale`, added to g (and *loss) in a fixed order; G: MLP_ROWS * MLP_CHUNK floats.
int mlp_grad_det(cudaStream_t st, const float *P, const float *X, const float *Y, const int32_t *idx, int64_t b0,
                 int64_t nb, float scale, float *G, float *g, float *loss)
{
    for (int64_t c0 = 0; c0 < nb; c0 += MLP_CHUNK) {
        const int64_t cn = std::min<int64_t>(MLP_CHUNK, nb - c0);
        mlp_sample_grad_kernel<<<(unsigned)((cn + MLP_BLOCK - 1) / MLP_BLOCK), MLP_BLOCK, 0, st>>>(
            P, X, Y, idx, b0 + c0, cn, scale, G);
        mlp_reduce_kernel<<<loss ? MLP_ROWS : HP_MLP_NPARAM, MLP_RED, 0, st>>>(G, cn, g, loss);
        HP_CUDA(cudaGetLastError());
    }
    return HP_OK;
}

__global__ void adam_kernel(float *__restrict__ P, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    hp::pdl_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= HP_MLP_NPARAM) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Stand-alone inference: tensor-core BF16 path (one warp per 32 samples) or
// the FP32 reference path.
__global__ void __launch_bounds__(128)
mlp_infer_kernel(const float *__restrict__ P, const float *__restrict__ X, int64_t n, float *__restrict__ out,
                 int tensor)
{
    hp::pdl_wait();
    __shared__ hp::MlpSmem sm;
    hp::mlp_load_smem(sm, P);
    __syncthreads();
    const int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) & ~31ll;
    for (int64_t w0 = base; w0 < n; w0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = w0 + (threadIdx.x & 31);
        float x[HP_MLP_IN];
        for (int i = 0; i < HP_MLP_IN; i++) x[i] = r < n ? X[r * HP_MLP_IN + i] : 0.f;
        float y;
        if (tensor) {
            y = hp::mlp_warp_logit(sm, x);
        } else {
            float z1[HP_MLP_H], z2[HP_MLP_H];
            y = mlp_fwd(P, x, z1, z2);
        }
        if (r < n) out[r] = y;
    }
}

}  // namespace

// ---- context-side state ------------------------------------------------------------
int hp_mlp_ensure(hp_context *c)
{
    if (c->mlp_params) return HP_OK;
    void *p = nullptr;
    HP_CUDA(cudaMalloc(&p, sizeof(float) * 4 * HP_MLP_NPARAM));
    c->mlp_params = (float *)p;
    c->mlp_grad = c->mlp_params + HP_MLP_NPARAM;
    c->mlp_m = c->mlp_grad + HP_MLP_NPARAM;
    c->mlp_v = c->mlp_m + HP_MLP_NPARAM;
    HP_CUDA(cudaMemset(p, 0, sizeof(float) * 4 * HP_MLP_NPARAM));
    return HP_OK;
}

// Per-sample gradient rows of one chunk (MLP_ROWS x MLP_CHUNK floats, 45 MB),
// allocated on the first training or gradient call of a context.
int hp_mlp_ensure_scratch(hp_context *c)
{
    if (c->mlp_scratch) return HP_OK;
    void *p = nullptr;
    if (cudaMalloc(&p, sizeof(float) * (size_t)MLP_ROWS * MLP_CHUNK) != cudaSuccess) {
        cudaGetLastError();
        return HP_ERR_NOMEM;
    }
    c->mlp_scratch = (float *)p;
    return HP_OK;
}

#define HP_API extern "C" __attribute__((visibility("default")))

HP_API int hp_mlp_set_params(hp_context *c, const float *params, int32_t count, float threshold)
{
    if (!c || !params || count != HP_MLP_NPARAM) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(c->device));
    HP_TRY(hp_mlp_ensure(c));
    HP_CUDA(cudaMemcpy(c->mlp_params, params, sizeof(float) * HP_MLP_NPARAM, cudaMemcpyHostToDevice));
    HP_CUDA(cudaMemset(c->mlp_m, 0, sizeof(float) * 2 * HP_MLP_NPARAM));
    c->mlp_threshold = threshold;
    c->mlp_ready = true;
    return HP_OK;
}

HP_API int hp_mlp_get_params(hp_context *c, float *params, int32_t count)
{
    if (!c || !params || count != HP_MLP_NPARAM || !c->mlp_params) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(c->device));
    HP_CUDA(cudaMemcpy(params, c->mlp_params, sizeof(float) * HP_MLP_NPARAM, cudaMemcpyDeviceToHost));
    return HP_OK;
}

HP_API int hp_mlp_loss_grad(hp_context *c, const float *d_x, const float *d_y, int64_t n, float *grad,
                            float *loss)
{
    if (!c || !d_x || !d_y || n <= 0 || !grad || !c->mlp_params) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->own_stream;
    HP_TRY(hp_mlp_ensure_scratch(c));
    HP_CUDA(cudaMemsetAsync(c->mlp_grad, 0, sizeof(float) * HP_MLP_NPARAM, s));
    HP_CUDA(cudaMemsetAsync(c->d_scal, 0, sizeof(float), s));
    HP_TRY(mlp_grad_det(s, c->mlp_params, d_x, d_y, nullptr, 0, n, 1.0f / (float)n, c->mlp_scratch, c->mlp_grad,
                        (float *)c->d_scal));
    HP_CUDA(cudaMemcpyAsync(grad, c->mlp_grad, sizeof(float) * HP_MLP_NPARAM, cudaMemcpyDeviceToHost, s));
    float l = 0;
    HP_CUDA(cudaMemcpyAsync(&l, c->d_scal, sizeof(float), cudaMemcpyDeviceToHost, s));
    HP_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = l;
    return HP_OK;
}

HP_API int hp_mlp_train(hp_context *c, const float *d_x, const float *d_y, const int32_t *d_perm, int64_t n,
                        int32_t epochs, int32_t batch, float lr, float *final_loss)
{
    if (!c || !d_x || !d_y || n <= 0 || epochs <= 0 || batch <= 0 || !c->mlp_params) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->own_stream;
    HP_TRY(hp_mlp_ensure_scratch(c));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float p1 = 1.f, p2 = 1.f;
    for (int e = 0; e < epochs; e++) {
        const bool last_epoch = e == epochs - 1;
        if (last_epoch) HP_CUDA(cudaMemsetAsync(c->d_scal, 0, sizeof(float), s));
        for (int64_t b0 = 0; b0 < n; b0 += batch) {
            const int64_t nb = std::min<int64_t>(batch, n - b0);
            HP_CUDA(cudaMemsetAsync(c->mlp_grad, 0, sizeof(float) * HP_MLP_NPARAM, s));
            HP_TRY(mlp_grad_det(s, c->mlp_params, d_x, d_y, d_perm, b0, nb, 1.0f / (float)nb, c->mlp_scratch,
                                c->mlp_grad, last_epoch ? (float *)c->d_scal : (float *)nullptr));
            p1 *= b1;
            p2 *= b2;
            adam_kernel<<<(HP_MLP_NPARAM + 255) / 256, 256, 0, s>>>(c->mlp_params, c->mlp_grad, c->mlp_m, c->mlp_v,
                                                                     lr, b1, b2, eps, 1.f - p1, 1.f - p2);
            HP_CUDA(cudaGetLastError());
        }
    }
    float l = 0;
    HP_CUDA(cudaMemcpyAsync(&l, c->d_scal, sizeof(float), cudaMemcpyDeviceToHost, s));
    HP_CUDA(cudaStreamSynchronize(s));
    if (final_loss) *final_loss = l * (float)batch / (float)n;   // mean over the batches of the last epoch
    c->mlp_ready = true;
    return HP_OK;
}

HP_API int hp_mlp_infer(hp_context *c, const float *d_x, int64_t n, float *d_out, int32_t tensor_cores)
{
    if (!c || !d_x || !d_out || n < 0 || !c->mlp_params) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(c->device));
    if (n == 0) return HP_OK;
    const unsigned grid = (unsigned)std::min<int64_t>((n + 127) / 128, c->sm_count * 8);
    mlp_infer_kernel<<<grid, 128, 0, c->own_stream>>>(c->mlp_params, d_x, n, d_out, tensor_cores);
    HP_CUDA(cudaGetLastError());
    HP_CUDA(cudaStreamSynchronize(c->own_stream));
    return HP_OK;
}

// ---- move log ------------------------------------------------------------------------
HP_API int hp_movelog_enable(hp_context *c, int64_t capacity)
{
    if (!c || capacity < 0) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(c->device));
    if (c->log_x) { cudaFree(c->log_x); c->log_x = nullptr; }
    c->log_cap = capacity;
    if (capacity == 0) return HP_OK;
    void *p = nullptr;
    // features, label, and per record: vertex, destination, accepted flag
    const size_t bytes = (size_t)capacity * (sizeof(float) * (HP_MLP_IN + 1) + sizeof(int32_t) * 3) + 256;
    if (cudaMalloc(&p, bytes) != cudaSuccess) { cudaGetLastError(); c->log_cap = 0; return HP_ERR_NOMEM; }
    c->log_x = (float *)p;
    c->log_y = c->log_x + (size_t)capacity * HP_MLP_IN;
    c->log_v = (int32_t *)(c->log_y + capacity);
    c->log_d = c->log_v + capacity;
    c->log_acc = c->log_d + capacity;
    c->log_count = (unsigned long long *)(c->log_acc + capacity);
    HP_CUDA(cudaMemset(c->log_count, 0, sizeof(unsigned long long)));
    return HP_OK;
}

HP_API int64_t hp_movelog_count(hp_context *c)
{
    if (!c || !c->log_x) return 0;
    unsigned long long n = 0;
    if (cudaMemcpy(&n, c->log_count, sizeof(n), cudaMemcpyDeviceToHost) != cudaSuccess) return HP_ERR_CUDA;
    return (int64_t)std::min<unsigned long long>(n, (unsigned long long)c->log_cap);
}

HP_API int hp_movelog_copy(hp_context *c, float *features, float *labels, int64_t count)
{
    if (!c || !c->log_x || count < 0) return HP_ERR_INVALID_ARG;
    int64_t have = hp_movelog_count(c);
    if (count > have) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(c->device));
    if (features)
        HP_CUDA(cudaMemcpy(features, c->log_x, sizeof(float) * HP_MLP_IN * (size_t)count, cudaMemcpyDeviceToHost));
    if (labels) HP_CUDA(cudaMemcpy(labels, c->log_y, sizeof(float) * (size_t)count, cudaMemcpyDeviceToHost));
    return HP_OK;
}

HP_API int hp_movelog_reset(hp_context *c)
{
    if (!c || !c->log_x) return HP_ERR_INVALID_ARG;
    HP_CUDA(cudaSetDevice(c->device));
    HP_CUDA(cudaMemset(c->log_count, 0, sizeof(unsigned long long)));
    return HP_OK;
}
