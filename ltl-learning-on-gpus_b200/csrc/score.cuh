// The learned block order's scorer on the device, one warp per feature vector.  Shared by
// the planner (the level kernel's planning warp) and nothing else on the device; the training
// kernels (mlp.cu) compute the same function one record per thread.
#pragma once

#include <cuda_bf16.h>

#include "ops.cuh"

namespace ltlg {

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16(x)); }

// The scorer on one feature vector, one warp: lane l computes hidden units l and l + 32 of
// each layer.  Operands are rounded to BF16, products and sums are FP32, and every unit sums
// its inputs in index order (the same order as forward_record in mlp.cu).
__device__ __noinline__ float mlp_score_warp(const MlpDev &M, const float *x, int lane) {
    float h1[2], h2[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int j = lane + 32 * u;
        float acc = 0.0f;
        for (int i = 0; i < ORDER_NF; ++i) acc += __bfloat162float(M.w1[j * ORDER_NF + i]) * bf16r(x[i]);
        h1[u] = fmaxf(acc + M.b1[j], 0.0f);
    }
    float acc2[2] = {0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < ORDER_H; ++k) {
        const float hk = bf16r(__shfl_sync(FULL, h1[k >> 5], k & 31));
#pragma unroll
        for (int u = 0; u < 2; ++u) acc2[u] += __bfloat162float(M.w2[(lane + 32 * u) * ORDER_H + k]) * hk;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) h2[u] = fmaxf(acc2[u] + M.b2[lane + 32 * u], 0.0f);
    float z = 0.0f;
#pragma unroll
    for (int k = 0; k < ORDER_H; ++k) {
        const float hk = bf16r(__shfl_sync(FULL, h2[k >> 5], k & 31));
        z += __bfloat162float(M.w3[k]) * hk;
    }
    return z + M.b3;
}

}  // namespace ltlg
