// Learned block ordering: the block features and the scorer's parameter layout, shared by
// the device planner, the host-side record writer and the training kernels.
//
// A level's blocks are the reference's (operator, left cost, right cost) blocks
// (ltli6463.cu:1209-1440).  The scorer is a multilayer perceptron 32 -> 64 -> 64 -> 1 with
// ReLU, BF16 operands and FP32 accumulation; a block's score is its logit of "this block
// holds an accepting candidate".  Ordering by score changes only which blocks are drained
// first: every block of the level still runs unless a find stops the level, and every lower
// level was exhausted before, so a find is still of minimal cost.
#pragma once

#include <cstdint>

#include <cuda_bf16.h>

namespace ltlg {

constexpr int ORDER_NF = 32;  // features per block
constexpr int ORDER_H = 64;   // hidden units of each of the two hidden layers

// Parameter offsets in the packed FP32 vector (row-major weights, out x in).
constexpr int MLP_W1 = 0;                            // [H][NF]
constexpr int MLP_B1 = MLP_W1 + ORDER_H * ORDER_NF;  // [H]
constexpr int MLP_W2 = MLP_B1 + ORDER_H;             // [H][H]
constexpr int MLP_B2 = MLP_W2 + ORDER_H * ORDER_H;   // [H]
constexpr int MLP_W3 = MLP_B2 + ORDER_H;             // [H]
constexpr int MLP_B3 = MLP_W3 + ORDER_H;             // [1]
constexpr int MLP_PARAMS = MLP_B3 + 1;

// The scorer on the device: BF16 weights, FP32 biases.
struct MlpDev {
    __nv_bfloat16 w1[ORDER_H * ORDER_NF];
    __nv_bfloat16 w2[ORDER_H * ORDER_H];
    __nv_bfloat16 w3[ORDER_H];
    float b1[ORDER_H];
    float b2[ORDER_H];
    float b3;
};

// What the features of one block are made of.  Costs are level costs; rows are cache rows.
struct BlockInfo {
    int op;          // 0 ~, 1 &, 2 |, 3 X, 4 F, 5 G, 6 U
    int cost;        // the level
    int c1;          // cost of a letter
    int lcost;       // cost of the (left) operand
    int rcost;       // cost of the right operand (0 for unary blocks)
    int position;    // index of the block in the reference's order within the level
    int nblocks;     // blocks of the level
    long long lrows, rrows;   // operand rows (rrows = 1 for unary blocks)
    long long candidates;     // of the block (U: two per pair)
    long long level_cands;    // of the level
    long long u_left, u_right;      // unique rows of the operand levels
    long long c_left, c_right;      // candidates of the operand levels (0 for the letter level)
    long long u_prev, c_prev;       // unique rows and candidates of level cost - 1
    int npos, nneg, nalpha;
};

// log2(x) for x >= 1 as exponent plus the linear mantissa fraction; 0 for x <= 0.  Plain
// integer and IEEE float steps only, so host and device give the same bits.
__host__ __device__ inline float lg2lin(long long x) {
    if (x <= 0) return 0.0f;
#ifdef __CUDA_ARCH__
    const int k = 63 - __clzll(x);
#else
    const int k = 63 - __builtin_clzll((unsigned long long)x);
#endif
    const long long p = 1ll << k;
    const float frac = (float)(x - p) / (float)p;
    return (float)k + frac;
}

__host__ __device__ inline float ratio(long long a, long long b) { return b > 0 ? (float)a / (float)b : 0.0f; }

// The 32 features of a block.  Every value is a plain IEEE operation on integers (no fused
// multiply-adds), so the planner on the device and the record writer on the host agree.
__host__ __device__ inline void block_features(const BlockInfo &b, float *f) {
    for (int i = 0; i < ORDER_NF; ++i) f[i] = 0.0f;
    if (b.op >= 0 && b.op < 7) f[b.op] = 1.0f;
    const bool bin = b.op == 1 || b.op == 2 || b.op == 6;
    const float c = (float)b.cost;
    f[7] = c / 16.0f;
    f[8] = (float)b.lcost / c;
    f[9] = (float)b.rcost / c;
    f[10] = lg2lin(b.lrows) / 24.0f;
    f[11] = lg2lin(b.rrows) / 24.0f;
    f[12] = lg2lin(b.candidates) / 32.0f;
    f[13] = ratio(b.candidates, b.level_cands);
    f[14] = ratio(b.position, b.nblocks);
    f[15] = (float)b.nblocks / 64.0f;
    f[16] = lg2lin(b.u_left) / 24.0f;
    f[17] = lg2lin(b.u_right) / 24.0f;
    f[18] = ratio(b.u_left, b.c_left);
    f[19] = ratio(b.u_right, b.c_right);
    f[20] = ratio(b.u_prev, b.c_prev);
    f[21] = lg2lin(b.level_cands) / 32.0f;
    f[22] = ratio(b.npos, (long long)b.npos + b.nneg);
    f[23] = lg2lin((long long)b.npos + b.nneg) / 16.0f;
    f[24] = (float)b.nalpha / 8.0f;
    const int d = b.lcost > b.rcost ? b.lcost - b.rcost : b.rcost - b.lcost;
    f[25] = bin ? (float)d / c : 0.0f;
    f[26] = bin && b.lcost == b.rcost ? 1.0f : 0.0f;
    f[27] = b.lcost == b.c1 ? 1.0f : 0.0f;
    f[28] = bin && b.rcost == b.c1 ? 1.0f : 0.0f;
    f[29] = bin ? 1.0f : 0.0f;
    f[30] = lg2lin(b.u_prev) / 24.0f;
    f[31] = 1.0f;
}

}  // namespace ltlg
