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
// Row statistics of a level: stored rows that hold at position 0 on every positive trace, and
// stored rows that hold at position 0 on no negative trace.
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
    long long lstat[2];       // row statistics of the (left) operand level
    long long rstat[2];       // of the right operand level (0 for unary blocks)
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
    f[15] = lg2lin(b.level_cands) / 32.0f;
    for (int k = 0; k < 2; ++k) {
        f[16 + k] = lg2lin(b.lstat[k] + 1) / 24.0f;
        f[18 + k] = ratio(b.lstat[k], b.lrows);
        f[20 + k] = lg2lin(b.rstat[k] + 1) / 24.0f;
        f[22 + k] = bin ? ratio(b.rstat[k], b.rrows) : 0.0f;
    }
    f[24] = ratio(b.npos, (long long)b.npos + b.nneg);
    f[25] = lg2lin((long long)b.npos + b.nneg) / 16.0f;
    f[26] = (float)b.nalpha / 8.0f;
    f[27] = bin ? 1.0f : 0.0f;
    f[28] = bin && b.lcost == b.rcost ? 1.0f : 0.0f;
    f[29] = b.lcost == b.c1 ? 1.0f : 0.0f;
    f[30] = bin && b.rcost == b.c1 ? 1.0f : 0.0f;
    f[31] = 1.0f;
}

}  // namespace ltlg
