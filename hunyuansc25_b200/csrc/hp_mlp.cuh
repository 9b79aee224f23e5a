// hp_mlp.cuh — the move-scoring MLP (8 -> 32 -> 32 -> 1) shared by the LP
// kernel (fused BF16 tensor-core inference) and the training kernels.
#pragma once

#include <cuda_bf16.h>

#include "hp_common.cuh"
#include "hp_partition.h"

#define HP_MLP_IN 8
#define HP_MLP_H 32
// packed FP32 parameters: W1[32][8], b1[32], W2[32][32], b2[32], w3[32], b3
#define HP_MLP_OFF_W1 0
#define HP_MLP_OFF_B1 (HP_MLP_OFF_W1 + HP_MLP_H * HP_MLP_IN)
#define HP_MLP_OFF_W2 (HP_MLP_OFF_B1 + HP_MLP_H)
#define HP_MLP_OFF_B2 (HP_MLP_OFF_W2 + HP_MLP_H * HP_MLP_H)
#define HP_MLP_OFF_W3 (HP_MLP_OFF_B2 + HP_MLP_H)
#define HP_MLP_OFF_B3 (HP_MLP_OFF_W3 + HP_MLP_H)
// the public count (HP_MLP_NPARAM, include/hp_partition.h) is this layout's size
static_assert(HP_MLP_OFF_B3 + 1 == HP_MLP_NPARAM, "parameter layout and HP_MLP_NPARAM disagree");

namespace hp {

// Features of an LP candidate, from integers only (the same expression on
// every path so logged and scored features agree):
//   0 gain / wdeg            1 conn(own) / wdeg        2 conn(best) / wdeg
//   3 min(parts-1, 8) / 8    4 log2(1+deg) / 16
//   5 clamp((maxp-pw)/opt) of the target part       6 same of the own part
//   7 1 on the finest level, else 0
__device__ __forceinline__ void mlp_features(int64_t pc, int64_t bc, int64_t wdeg, int32_t nparts_adj,
                                             int32_t deg, int64_t slack_b, int64_t opt_b, int64_t slack_p,
                                             int64_t opt_p, int finest, float f[HP_MLP_IN])
{
    const float iw = wdeg > 0 ? 1.0f / (float)wdeg : 0.0f;
    f[0] = (float)(bc - pc) * iw;
    f[1] = (float)pc * iw;
    f[2] = (float)bc * iw;
    f[3] = (float)min(max(nparts_adj - 1, 0), 8) * 0.125f;
    f[4] = __log2f(1.0f + (float)deg) * 0.0625f;
    f[5] = fminf(1.0f, fmaxf(-1.0f, opt_b > 0 ? (float)slack_b / (float)opt_b : 0.0f));
    f[6] = fminf(1.0f, fmaxf(-1.0f, opt_p > 0 ? (float)slack_p / (float)opt_p : 0.0f));
    f[7] = finest ? 1.0f : 0.0f;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

// D = A(16x16 bf16) * B(16x8 bf16) + C, FP32 accumulate (legacy warp-level
// tensor-core MMA; the MLP is ~2.6 kFLOP per vertex, so the op is HBM-bound
// and a warp-synchronous MMA keeps it inside the LP kernel).
__device__ __forceinline__ void mma_bf16_16816(float d[4], const uint32_t a[4], const uint32_t b[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Shared-memory copy of the weights in the fragment-friendly forms the warp
// inference uses (BF16 for the two tensor-core layers, FP32 for biases/w3).
struct MlpSmem {
    __nv_bfloat16 w1[HP_MLP_H][HP_MLP_IN];
    __nv_bfloat16 w2[HP_MLP_H][HP_MLP_H];
    float b1[HP_MLP_H], b2[HP_MLP_H], w3[HP_MLP_H];
    float b3;
};

__device__ __forceinline__ void mlp_load_smem(MlpSmem &s, const float *__restrict__ p)
{
    for (int i = threadIdx.x; i < HP_MLP_H * HP_MLP_IN; i += blockDim.x)
        s.w1[i / HP_MLP_IN][i % HP_MLP_IN] = __float2bfloat16_rn(p[HP_MLP_OFF_W1 + i]);
    for (int i = threadIdx.x; i < HP_MLP_H * HP_MLP_H; i += blockDim.x)
        s.w2[i / HP_MLP_H][i % HP_MLP_H] = __float2bfloat16_rn(p[HP_MLP_OFF_W2 + i]);
    for (int i = threadIdx.x; i < HP_MLP_H; i += blockDim.x) {
        s.b1[i] = p[HP_MLP_OFF_B1 + i];
        s.b2[i] = p[HP_MLP_OFF_B2 + i];
        s.w3[i] = p[HP_MLP_OFF_W3 + i];
    }
    if (threadIdx.x == 0) s.b3 = p[HP_MLP_OFF_B3];
}

// Warp-wide inference: lane L holds the features of vertex L of the warp;
// returns vertex L's logit in lane L.  All 32 lanes must participate.
// Fragment layout of mma.m16n8k16 (g = lane/4, t = lane%4):
//   A: a0,a1 = (row g, col 2t..2t+1), a2,a3 = (row g+8, ...), a4..a7 = cols +8
//   B: b0,b1 = (k 2t..2t+1, n g), b2,b3 = (k 2t+8.., n g)
//   C: c0,c1 = (row g, col 2t..2t+1), c2,c3 = (row g+8, ...)
__device__ __forceinline__ float mlp_warp_logit(const MlpSmem &s, const float f[HP_MLP_IN])
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float out = 0.0f;
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
        // A fragment of layer 1 (K = 8 features, padded to 16 with zeros)
        const int r0 = mt * 16 + g, r1 = r0 + 8;
        float x0[HP_MLP_IN], x1[HP_MLP_IN];
#pragma unroll
        for (int c = 0; c < HP_MLP_IN; c++) {
            x0[c] = __shfl_sync(HP_FULL_MASK, f[c], r0);
            x1[c] = __shfl_sync(HP_FULL_MASK, f[c], r1);
        }
        uint32_t a1[4];
        a1[0] = pack_bf16(x0[2 * t], x0[2 * t + 1]);
        a1[1] = pack_bf16(x1[2 * t], x1[2 * t + 1]);
        a1[2] = 0u;
        a1[3] = 0u;
        // layer 1: 4 n-tiles of 8 hidden units
        float h1[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            const int n = nt * 8 + g;
            uint32_t b[2];
            b[0] = pack_bf16(__bfloat162float(s.w1[n][2 * t]), __bfloat162float(s.w1[n][2 * t + 1]));
            b[1] = 0u;
            float d[4] = {0.f, 0.f, 0.f, 0.f};
            mma_bf16_16816(d, a1, b);
            const int col = nt * 8 + 2 * t;
            h1[nt][0] = fmaxf(0.f, d[0] + s.b1[col]);
            h1[nt][1] = fmaxf(0.f, d[1] + s.b1[col + 1]);
            h1[nt][2] = fmaxf(0.f, d[2] + s.b1[col]);
            h1[nt][3] = fmaxf(0.f, d[3] + s.b1[col + 1]);
        }
        // layer 2: K = 32 (two k-tiles), A fragments straight from h1's C layout
        float h2[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < 2; kt++) {
                uint32_t a[4];
                a[0] = pack_bf16(h1[2 * kt][0], h1[2 * kt][1]);
                a[1] = pack_bf16(h1[2 * kt][2], h1[2 * kt][3]);
                a[2] = pack_bf16(h1[2 * kt + 1][0], h1[2 * kt + 1][1]);
                a[3] = pack_bf16(h1[2 * kt + 1][2], h1[2 * kt + 1][3]);
                const int n = nt * 8 + g, k0 = kt * 16 + 2 * t;
                uint32_t b[2];
                b[0] = pack_bf16(__bfloat162float(s.w2[n][k0]), __bfloat162float(s.w2[n][k0 + 1]));
                b[1] = pack_bf16(__bfloat162float(s.w2[n][k0 + 8]), __bfloat162float(s.w2[n][k0 + 9]));
                mma_bf16_16816(d, a, b);
            }
            const int col = nt * 8 + 2 * t;
            h2[nt][0] = fmaxf(0.f, d[0] + s.b2[col]);
            h2[nt][1] = fmaxf(0.f, d[1] + s.b2[col + 1]);
            h2[nt][2] = fmaxf(0.f, d[2] + s.b2[col]);
            h2[nt][3] = fmaxf(0.f, d[3] + s.b2[col + 1]);
        }
        // layer 3 (FP32): rows g and g+8, reduced over the 4 lanes of a group
        float y0 = 0.f, y1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            const int col = nt * 8 + 2 * t;
            y0 += h2[nt][0] * s.w3[col] + h2[nt][1] * s.w3[col + 1];
            y1 += h2[nt][2] * s.w3[col] + h2[nt][3] * s.w3[col + 1];
        }
        y0 += __shfl_xor_sync(HP_FULL_MASK, y0, 1);
        y0 += __shfl_xor_sync(HP_FULL_MASK, y0, 2);
        y1 += __shfl_xor_sync(HP_FULL_MASK, y1, 1);
        y1 += __shfl_xor_sync(HP_FULL_MASK, y1, 2);
        // vertex r = mt*16 + j: row j < 8 lives in lane 4j (y0), row j >= 8 in lane 4(j-8) (y1)
        const int j = lane - mt * 16;
        const float v0 = __shfl_sync(HP_FULL_MASK, y0, (j & 7) * 4);
        const float v1 = __shfl_sync(HP_FULL_MASK, y1, (j & 7) * 4);
        if (j >= 0 && j < 16) out = (j < 8 ? v0 : v1) + s.b3;
    }
    return out;
}

}  // namespace hp
