// Training and inference kernels of the learned block order's scorer: a multilayer perceptron
// 32 -> 64 -> 64 -> 1 with ReLU, BF16 operands (inputs, weights, activations and the
// backward products' gradient operands rounded to BF16) and FP32 products and sums.  The
// gradient is that of the mean weighted binary cross-entropy with logits.  Every unit sums
// its inputs in index order, as the planner's scorer does (mlp_score_warp in score.cuh).
//
// The reference has no learned component; these kernels back the block ordering only.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "ltl_kernels.cuh"
#include "ltlgpu.h"

namespace ltlg {
namespace {

constexpr int NF = ORDER_NF, H = ORDER_H;
constexpr int REC = 64;       // records per CTA of the gradient kernel
constexpr int THREADS = 128;  // threads per CTA of the gradient kernel

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16(x)); }
__device__ __forceinline__ float wf(__nv_bfloat16 w) { return __bfloat162float(w); }

// Shared-memory layout of the gradient kernel: BF16 copies of the rounded inputs and
// activations, the (BF16-rounded) gradients of the hidden layers in FP32.
struct GradSmem {
    __nv_bfloat16 x[REC][NF];
    __nv_bfloat16 h1[REC][H];
    __nv_bfloat16 h2[REC][H];
    float dh1[REC][H];
    float dh2[REC][H];
    float dz[REC];
    float dzb[REC];
};

// Forward pass of one record (x already rounded to BF16): the logit; h1, h2 receive the
// BF16-rounded activations.
__device__ float forward_record(const MlpDev &M, const float *x, float *h1, float *h2) {
    for (int j = 0; j < H; ++j) {
        float acc = 0.0f;
        for (int i = 0; i < NF; ++i) acc += wf(M.w1[j * NF + i]) * x[i];
        h1[j] = bf(fmaxf(acc + M.b1[j], 0.0f));
    }
    for (int j = 0; j < H; ++j) {
        float acc = 0.0f;
        for (int k = 0; k < H; ++k) acc += wf(M.w2[j * H + k]) * h1[k];
        h2[j] = bf(fmaxf(acc + M.b2[j], 0.0f));
    }
    float z = 0.0f;
    for (int k = 0; k < H; ++k) z += wf(M.w3[k]) * h2[k];
    return z + M.b3;
}

__global__ void forward_kernel(const MlpDev *__restrict__ M, const float *__restrict__ X, int count,
                               float *__restrict__ logits) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= count) return;
    float x[NF], h1[H], h2[H];
    for (int i = 0; i < NF; ++i) x[i] = bf(X[(size_t)r * NF + i]);
    logits[r] = forward_record(*M, x, h1, h2);
}

// Gradient of inv_norm * sum_r w_r * BCE(z_r, y_r) over the records idx[first .. first + n)
// (or first .. first + n when idx is null), added into grad; the loss sum into *loss.
// Phase 1: one thread per record (forward, loss, backward to the hidden layers).  Phase 2:
// the CTA's threads split the parameters, each summing its gradient over the CTA's records.
__global__ void __launch_bounds__(THREADS) grad_kernel(const MlpDev *__restrict__ M, const float *__restrict__ X,
                                                       const float *__restrict__ Y, const int *__restrict__ idx,
                                                       long long first, int n, float pos_weight, float inv_norm,
                                                       float *__restrict__ grad, float *__restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem &S = *reinterpret_cast<GradSmem *>(smem_raw);
    const int t = threadIdx.x;
    const int base = blockIdx.x * REC;
    float my_loss = 0.0f;
    if (t < REC) {
        const int q = base + t;
        if (q < n) {
            const long long r = idx ? (long long)idx[first + q] : first + q;
            float x[NF], h1[H], h2[H];
            for (int i = 0; i < NF; ++i) {
                x[i] = bf(X[r * NF + i]);
                S.x[t][i] = __float2bfloat16(x[i]);
            }
            const float z = forward_record(*M, x, h1, h2);
            for (int j = 0; j < H; ++j) {
                S.h1[t][j] = __float2bfloat16(h1[j]);
                S.h2[t][j] = __float2bfloat16(h2[j]);
            }
            const float y = Y[r];
            const float w = y > 0.5f ? pos_weight : 1.0f;
            const float p = 1.0f / (1.0f + expf(-z));
            my_loss = w * (fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z))));
            const float dz = w * (p - y) * inv_norm;
            S.dz[t] = dz;
            S.dzb[t] = bf(dz);
            for (int k = 0; k < H; ++k) S.dh2[t][k] = h2[k] > 0.0f ? bf(dz * wf(M->w3[k])) : 0.0f;
            for (int j = 0; j < H; ++j) {
                float acc = 0.0f;
                for (int k = 0; k < H; ++k) acc += wf(M->w2[k * H + j]) * S.dh2[t][k];
                S.dh1[t][j] = h1[j] > 0.0f ? bf(acc) : 0.0f;
            }
        } else {
            for (int i = 0; i < NF; ++i) S.x[t][i] = __float2bfloat16(0.0f);
            for (int j = 0; j < H; ++j) {
                S.h1[t][j] = __float2bfloat16(0.0f);
                S.h2[t][j] = __float2bfloat16(0.0f);
                S.dh1[t][j] = 0.0f;
                S.dh2[t][j] = 0.0f;
            }
            S.dz[t] = 0.0f;
            S.dzb[t] = 0.0f;
        }
    }
    __syncthreads();
    for (int p = t; p < MLP_PARAMS; p += THREADS) {
        float g = 0.0f;
        if (p < MLP_B1) {
            const int j = p / NF, i = p % NF;
            for (int r = 0; r < REC; ++r) g += S.dh1[r][j] * __bfloat162float(S.x[r][i]);
        } else if (p < MLP_W2) {
            const int j = p - MLP_B1;
            for (int r = 0; r < REC; ++r) g += S.dh1[r][j];
        } else if (p < MLP_B2) {
            const int k = (p - MLP_W2) / H, j = (p - MLP_W2) % H;
            for (int r = 0; r < REC; ++r) g += S.dh2[r][k] * __bfloat162float(S.h1[r][j]);
        } else if (p < MLP_W3) {
            const int k = p - MLP_B2;
            for (int r = 0; r < REC; ++r) g += S.dh2[r][k];
        } else if (p < MLP_B3) {
            const int k = p - MLP_W3;
            for (int r = 0; r < REC; ++r) g += S.dzb[r] * __bfloat162float(S.h2[r][k]);
        } else {
            for (int r = 0; r < REC; ++r) g += S.dz[r];
        }
        if (g != 0.0f) atomicAdd(grad + p, g);
    }
    for (int o = 16; o > 0; o >>= 1) my_loss += __shfl_xor_sync(0xFFFFFFFFu, my_loss, o);
    if ((t & 31) == 0 && my_loss != 0.0f) atomicAdd(loss, my_loss);
}

// AdamW step on the FP32 master parameters (weight decay on weights only); the BF16 copy is
// refreshed afterwards by the pack kernel.
__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, float lr, float b1, float b2, float eps, float wd, float c1,
                            float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_PARAMS) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const bool weight = i < MLP_B1 || (i >= MLP_W2 && i < MLP_B2) || (i >= MLP_W3 && i < MLP_B3);
    float pi = p[i];
    if (weight) pi -= lr * wd * pi;
    p[i] = pi - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Device buffers of one scorer call, freed on scope exit.
struct Bufs {
    std::vector<void *> ptrs;
    ~Bufs() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T>
    T *alloc(size_t n, cudaError_t &err) {
        void *p = nullptr;
        if (err == cudaSuccess) err = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
        if (err == cudaSuccess) ptrs.push_back(p);
        return (T *)p;
    }
};

cudaError_t grad_smem_attr() {
    return cudaFuncSetAttribute(grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GradSmem));
}

int status_of(cudaError_t e) {
    return e == cudaSuccess ? 0 : e == cudaErrorMemoryAllocation ? LTLG_NO_MEMORY : LTLG_CUDA_ERROR;
}

bool has_device() {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}

// The scorer's device form from the packed FP32 parameters: weights rounded to BF16.
__global__ void scorer_pack_kernel(const float *__restrict__ p, MlpDev *__restrict__ m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ORDER_H * ORDER_NF) m->w1[i] = __float2bfloat16(p[MLP_W1 + i]);
    if (i < ORDER_H * ORDER_H) m->w2[i] = __float2bfloat16(p[MLP_W2 + i]);
    if (i < ORDER_H) {
        m->w3[i] = __float2bfloat16(p[MLP_W3 + i]);
        m->b1[i] = p[MLP_B1 + i];
        m->b2[i] = p[MLP_B2 + i];
    }
    if (i == 0) m->b3 = p[MLP_B3];
}

}  // namespace

cudaError_t launch_scorer_pack(const float *params, MlpDev *out, cudaStream_t s) {
    scorer_pack_kernel<<<(MLP_PARAMS + 255) / 256, 256, 0, s>>>(params, out);
    return cudaGetLastError();
}

}  // namespace ltlg

using namespace ltlg;

extern "C" LTLG_API int ltlg_scorer_forward(const float *params, const float *features, int32_t count, float *logits) {
    if (!params || count < 0 || (count > 0 && (!features || !logits))) return LTLG_BAD_ARGS;
    if (!has_device()) return LTLG_NO_DEVICE;
    if (count == 0) return 0;
    cudaError_t err = cudaSuccess;
    Bufs b;
    float *dp = b.alloc<float>(MLP_PARAMS, err);
    MlpDev *dm = b.alloc<MlpDev>(1, err);
    float *dx = b.alloc<float>((size_t)count * NF, err);
    float *dz = b.alloc<float>(count, err);
    if (err == cudaSuccess) err = cudaMemcpy(dp, params, MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dx, features, (size_t)count * NF * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = launch_scorer_pack(dp, dm, 0);
    if (err == cudaSuccess) {
        forward_kernel<<<(count + 127) / 128, 128>>>(dm, dx, count, dz);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(logits, dz, (size_t)count * sizeof(float), cudaMemcpyDeviceToHost);
    return status_of(err);
}

extern "C" LTLG_API int ltlg_scorer_grad(const float *params, const float *features, const float *labels, int32_t count,
                                         float pos_weight, float *grad, float *loss) {
    if (!params || !grad || count <= 0 || !features || !labels) return LTLG_BAD_ARGS;
    if (!has_device()) return LTLG_NO_DEVICE;
    cudaError_t err = grad_smem_attr();
    Bufs b;
    float *dp = b.alloc<float>(MLP_PARAMS, err);
    MlpDev *dm = b.alloc<MlpDev>(1, err);
    float *dx = b.alloc<float>((size_t)count * NF, err);
    float *dy = b.alloc<float>(count, err);
    float *dg = b.alloc<float>(MLP_PARAMS + 1, err);
    if (err == cudaSuccess) err = cudaMemcpy(dp, params, MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dx, features, (size_t)count * NF * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dy, labels, (size_t)count * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemset(dg, 0, (MLP_PARAMS + 1) * sizeof(float));
    if (err == cudaSuccess) err = launch_scorer_pack(dp, dm, 0);
    if (err == cudaSuccess) {
        grad_kernel<<<(count + REC - 1) / REC, THREADS, sizeof(GradSmem)>>>(dm, dx, dy, nullptr, 0, count, pos_weight,
                                                                              1.0f / (float)count, dg, dg + MLP_PARAMS);
        err = cudaGetLastError();
    }
    std::vector<float> h(MLP_PARAMS + 1);
    if (err == cudaSuccess) err = cudaMemcpy(h.data(), dg, h.size() * sizeof(float), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return status_of(err);
    memcpy(grad, h.data(), MLP_PARAMS * sizeof(float));
    if (loss) *loss = h[MLP_PARAMS] / (float)count;
    return 0;
}

extern "C" LTLG_API int ltlg_scorer_train(float *params, const float *features, const float *labels, int32_t count,
                                          const ltlg_train_config *cfg, float *epoch_loss) {
    if (!params || !cfg || count <= 0 || !features || !labels || cfg->epochs < 0 || cfg->batch <= 0)
        return LTLG_BAD_ARGS;
    if (!has_device()) return LTLG_NO_DEVICE;
    cudaError_t err = grad_smem_attr();
    Bufs b;
    float *dp = b.alloc<float>(MLP_PARAMS, err);
    float *dm1 = b.alloc<float>(MLP_PARAMS, err);
    float *dv = b.alloc<float>(MLP_PARAMS, err);
    float *dg = b.alloc<float>(MLP_PARAMS + 1, err);
    MlpDev *dm = b.alloc<MlpDev>(1, err);
    float *dx = b.alloc<float>((size_t)count * NF, err);
    float *dy = b.alloc<float>(count, err);
    int *didx = b.alloc<int>(count, err);
    if (err == cudaSuccess) err = cudaMemcpy(dp, params, MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemset(dm1, 0, MLP_PARAMS * sizeof(float));
    if (err == cudaSuccess) err = cudaMemset(dv, 0, MLP_PARAMS * sizeof(float));
    if (err == cudaSuccess) err = cudaMemcpy(dx, features, (size_t)count * NF * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dy, labels, (size_t)count * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = launch_scorer_pack(dp, dm, 0);
    std::vector<int> perm(count);
    for (int i = 0; i < count; ++i) perm[i] = i;
    uint64_t s = cfg->seed;
    auto next = [&]() {  // splitmix64
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    long long step = 0;
    for (int ep = 0; ep < cfg->epochs && err == cudaSuccess; ++ep) {
        for (int i = count - 1; i > 0; --i) std::swap(perm[i], perm[(int)(next() % (uint64_t)(i + 1))]);
        err = cudaMemcpy(didx, perm.data(), (size_t)count * sizeof(int), cudaMemcpyHostToDevice);
        if (err == cudaSuccess) err = cudaMemset(dg + MLP_PARAMS, 0, sizeof(float));
        for (long long first = 0; first < count && err == cudaSuccess; first += cfg->batch) {
            const int nb = (int)std::min<long long>(cfg->batch, count - first);
            ++step;
            err = cudaMemsetAsync(dg, 0, MLP_PARAMS * sizeof(float));
            if (err != cudaSuccess) break;
            grad_kernel<<<(nb + REC - 1) / REC, THREADS, sizeof(GradSmem)>>>(dm, dx, dy, didx, first, nb, cfg->pos_weight,
                                                                             1.0f / (float)nb, dg, dg + MLP_PARAMS);
            const float c1 = 1.0f - std::pow(cfg->beta1, (float)step), c2 = 1.0f - std::pow(cfg->beta2, (float)step);
            adam_kernel<<<(MLP_PARAMS + 255) / 256, 256>>>(dp, dg, dm1, dv, cfg->lr, cfg->beta1, cfg->beta2, cfg->eps,
                                                           cfg->weight_decay, c1, c2);
            err = cudaGetLastError();
            if (err == cudaSuccess) err = launch_scorer_pack(dp, dm, 0);
        }
        float lsum = 0.0f;
        if (err == cudaSuccess) err = cudaMemcpy(&lsum, dg + MLP_PARAMS, sizeof(float), cudaMemcpyDeviceToHost);
        if (epoch_loss) epoch_loss[ep] = lsum / (float)count;
    }
    if (err == cudaSuccess) err = cudaMemcpy(params, dp, MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost);
    return status_of(err);
}
