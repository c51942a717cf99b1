// The level planner and the learned block order's scorer on the device.  Kept apart from
// the level kernel's translation unit so the level kernel's hot code stays compact in the
// instruction cache.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "ltl_kernels.cuh"

namespace ltlg {
namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;

// Operator of slot j of a fused unary block: 0 ~, 1 X, 2 F, 3 G.
__device__ __forceinline__ int unary_slot_op(int j) { return j == 0 ? OP_NEG : j == 1 ? OP_X : j == 2 ? OP_F : OP_G; }

// ---------------------------------------------------------------- learned order
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16(x)); }

// The scorer on one feature vector, one warp: lane l computes hidden units l and l + 32 of
// each layer.  Operands are rounded to BF16, products and sums are FP32, and every unit sums
// its inputs in index order (the same order as forward_record in mlp.cu).
__device__ float mlp_score_warp(const MlpDev &M, const float *x, int lane) {
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

// The planner: thread 0 turns the level starts into the next level's plan, in the
// reference's order (ltli6463.cu:1209-1440; NegType rule :1212): ~, & splits, | splits,
// X, F, G, U splits; a split i pairs cost i with cost c - i - c_op, i = c1 .. (c - c_op)/2.
// Then the item table: plain order (unary blocks, & blocks, | blocks, U blocks), or under
// PLAN_LEARNED every block scored by one warp and the table sorted by score (ties keep the
// reference's order).  One CTA of 256 threads.
__global__ void __launch_bounds__(256) plan_kernel(const LevelArgs *__restrict__ pA) {
    const LevelArgs &A = *pA;
    DevLevel *L = A.lev;
    DevCtl *C = A.ctl;
    __shared__ int s_go, s_nent, s_pos[MAX_RANGES], s_order[MAX_RANGES];
    __shared__ ItemRange s_ent[MAX_RANGES];
    __shared__ long long s_cnt[MAX_RANGES];
    __shared__ float s_score[MAX_RANGES];
    __shared__ float s_q[4 * MAX_RANGES];
    __shared__ float s_x[8][ORDER_NF];
    // The plan is built in shared memory and copied out once: thread 0 never reads back
    // what it wrote to global memory (each read-back is an L2 round trip).
    __shared__ BlockDesc s_blk[MAX_RANGES];  // the level's blocks, operator by operator
    __shared__ BlockDesc s_ub[4];
    __shared__ int s_first[8], s_c, s_nblk, s_nu;
    __shared__ long long s_ls[MAX_COSTS + 2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        s_go = 0;
        s_nent = 0;
        s_nblk = 0;
        s_nu = 0;
        L->seq = L->seq + 1;
        s_c = L->halt == 2 ? -1 : L->cost + 1;  // an over-long plan stops the rest of the graph
    }
    __syncthreads();
    const int cc = s_c;
    if (cc < 0) return;
    for (int k = threadIdx.x; k < cc && k < MAX_COSTS + 1; k += blockDim.x) s_ls[k] = A.ls[k];
    __syncthreads();
    if (threadIdx.x == 0) do {
        const int c = cc;
        L->cost = c;
        const long long rows = min((long long)C->row_count, A.cap_rows);
        if (c < MAX_COSTS + 1) {
            A.ls[c] = rows;  // level c - 1 ended here
            s_ls[c] = rows;
        }
        u32 bad = ST_WAIT | ST_TABLE | ST_TMA;
        const int on_the_fly = L->on_the_fly, flags = L->plan_flags;
        if (!on_the_fly) bad |= ST_OVERFLOW;
        const bool halt = c > A.max_cost || c >= MAX_COSTS || (A.stop_at_found && C->found != 0ull) ||
                          (C->status & bad) != 0u;
        for (int k = 0; k < 8; ++k) C->queue[k] = 0;
        L->halt = halt ? 1 : 0;
        if (halt) {
            for (int k = 0; k < 8; ++k) {
                L->nblocks[k] = 0;
                L->total_items[k] = 0;
                L->item_hi[k] = 0;
            }
            L->item_hi_all = 0;
            L->nublocks = 0;
            L->nranges = 0;
            L->learned_order = 0;
            L->items_end = 0;
            L->level_cands = 0;
            break;
        }
        const int c1 = A.cf[0];
        auto lo = [&](int k) { return (k >= 0 && k < c) ? s_ls[k] : 0ll; };
        auto hi = [&](int k) { return (k >= 0 && k < c) ? s_ls[k + 1] : 0ll; };
        u64 cands = 0;
        bool overfull = false;
        int nb = 0, cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        auto add = [&](int op, int lc, long long l0, long long l1, long long r0, long long r1, long long n) {
            if (cnt[op] >= MAX_SPLITS || nb >= MAX_RANGES) {
                overfull = true;
                return;
            }
            if (cnt[op] == 0) s_first[op] = nb;
            BlockDesc &b = s_blk[nb];
            b.op = op;
            b.lcost = lc;
            b.opmask = op == OP_NEG ? 1 : op == OP_X ? 2 : op == OP_F ? 4 : op == OP_G ? 8 : 0;
            b.pad = nb++;  // position in the reference's order
            b.l0 = l0;
            b.l1 = l1;
            b.r0 = r0;
            b.r1 = r1;
            b.candidates = n;
            ++cnt[op];
            cands += (u64)n;
        };
        auto unary = [&](int op, int k) {
            const long long a = lo(k), b = hi(k);
            if (b > a) add(op, k, 0, 0, a, b, b - a);
        };
        auto binary = [&](int op, int cop) {
            for (int i = c1; 2 * i <= c - cop; ++i) {
                const int j = c - i - cop;
                const long long a = lo(i), b = hi(i), x = lo(j), y = hi(j);
                if (b > a && y > x) add(op, i, a, b, x, y, (op == OP_U ? 2 : 1) * (b - a) * (y - x));
            }
        };
        const int *cf = A.cf;
        if ((A.neg_type == 1 && c - cf[1] >= c1) || (A.neg_type == 2 && c - cf[1] == c1)) unary(OP_NEG, c - cf[1]);
        binary(OP_AND, cf[2]);
        binary(OP_OR, cf[3]);
        if (c - cf[4] >= c1) unary(OP_X, c - cf[4]);
        if (c - cf[5] >= c1) unary(OP_F, c - cf[5]);
        if (c - cf[6] >= c1) unary(OP_G, c - cf[6]);
        binary(OP_U, cf[7]);
        if (overfull) {  // more splits than a plan holds: hand the level back to the host
            for (int k = 0; k < 8; ++k) L->nblocks[k] = 0;
            L->halt = 2;
            break;
        }
        // Work-item size: a small level is cut into one right row (or one group of source
        // rows) per warp so every SM takes part; a large level keeps the configured sizes.
        const bool small = (long long)cands < A.small_level;
        const int sr = A.small_rows > 1 ? A.small_rows : 1;
        const int rc = max(1, small ? A.nwarps * sr : A.right_chunk_big);
        const int ur = max(1, small ? A.nwarps * UNARY_ROWS * sr : A.unary_rows_big);
        L->right_chunk = rc;
        L->unary_rows = ur;
        L->check_only = on_the_fly;
        L->level_cands = cands;
        if (c < MAX_COSTS + 1) A.level_cands[c] = cands;
        const bool fuse = !(flags & PLAN_UNFUSED);
        // Unary blocks: one per operator, or (fused) one per distinct source range with every
        // operator on it.
        int nu = 0;
        for (int j = 0; j < 4; ++j) {
            const int op = unary_slot_op(j);
            if (cnt[op] == 0) continue;
            const BlockDesc &b = s_blk[s_first[op]];
            int u = 0;
            while (fuse && u < nu && !(s_ub[u].r0 == b.r0 && s_ub[u].r1 == b.r1)) ++u;
            if (!fuse || u == nu) {
                u = nu++;
                s_ub[u] = b;
                s_ub[u].opmask = 0;
                s_ub[u].candidates = 0;
            }
            s_ub[u].opmask |= 1 << j;
            s_ub[u].candidates += b.candidates;
        }
        int ne = 0;
        for (int u = 0; u < nu; ++u) {
            BlockDesc &f = s_ub[u];
            f.items = (f.r1 - f.r0 + ur - 1) / ur;
            f.tiles_r = 1;
            s_ent[ne] = ItemRange{f.items, 0, 1, u};
            s_pos[ne++] = f.pad;
        }
        for (int op = 0; op < 7; ++op) {
            long long items = 0;
            const bool bin = op == OP_AND || op == OP_OR || op == OP_U;
            const int tile = op == OP_U ? A.left_tile / 2 : A.left_tile;
            for (int k = 0; k < cnt[op]; ++k) {
                BlockDesc &b = s_blk[s_first[op] + k];
                b.item0 = items;
                if (bin) {
                    b.tiles_r = (b.r1 - b.r0 + rc - 1) / rc;
                    b.items = ((b.l1 - b.l0 + tile - 1) / tile) * b.tiles_r;
                    s_ent[ne] = ItemRange{b.items, 0, op == OP_U ? 3 : 2, op * MAX_SPLITS + k};
                    s_pos[ne++] = b.pad;
                } else {
                    b.tiles_r = 1;
                    b.items = (b.r1 - b.r0 + ur - 1) / ur;
                }
                items += b.items;
            }
            L->nblocks[op] = cnt[op];
            L->total_items[op] = items;
            L->item_hi[op] = items;
        }
        L->nblocks[7] = 0;
        L->nublocks = nu;
        s_nblk = nb;
        s_nu = nu;
        s_nent = ne;  // item0 holds each entry's item count until the table is laid out
        long long items = 0;
        for (int e = 0; e < ne; ++e) items += s_ent[e].item0;
        // order only matters when the level's items do not all start in the first wave
        s_go = (flags & PLAN_LEARNED) && A.model && items > A.grid ? 2 : 1;
    } while (0);
    __syncthreads();
    if (s_go == 0) return;
    {  // the plan's blocks and unary blocks into global memory, all threads
        const int nb = s_nblk, nu = s_nu;
        constexpr int W = sizeof(BlockDesc) / 8;
        for (int i = threadIdx.x; i < (nb + nu) * W; i += blockDim.x) {
            const int e = i / W, w = i % W;
            const BlockDesc &src = e < nb ? s_blk[e] : s_ub[e - nb];
            BlockDesc &dst = e < nb ? L->blocks[src.op][src.pad - s_first[src.op]] : L->ublocks[e - nb];
            reinterpret_cast<u64 *>(&dst)[w] = reinterpret_cast<const u64 *>(&src)[w];
        }
    }
    const int ne = s_nent;
    if (s_go == 2) {
        // Score every block (one warp per block).  A fused unary entry holds several
        // operators' blocks: its chance is that any of them accepts, 1 - prod(1 - p).  The
        // key is that chance over the square root of the entry's candidates, so likely blocks
        // go first and, of two equally likely ones, the smaller.
        const MlpDev &M = *reinterpret_cast<const MlpDev *>(A.model);
        const int c = L->cost;
        const int nbl = s_nblk;
        const int jobs = ne * 4;  // (entry, unary slot); binary entries use slot 0 only
        for (int j = threadIdx.x; j < jobs; j += blockDim.x) s_q[j] = 1.0f;
        __syncthreads();
        for (int j = warp; j < jobs; j += blockDim.x >> 5) {
            const int e = j >> 2, slot = j & 3;
            const ItemRange &R = s_ent[e];
            int op;
            const BlockDesc *b;
            if (R.cls == 1) {
                if (!((s_ub[R.idx].opmask >> slot) & 1)) continue;
                op = unary_slot_op(slot);
                b = &s_blk[s_first[op]];
            } else {
                if (slot) continue;
                op = R.idx / MAX_SPLITS;
                b = &s_blk[s_first[op] + R.idx % MAX_SPLITS];
            }
            if (lane == 0) {
                const BlockInfo bi = block_info(*b, op, c, A.cf, nbl, (long long)L->level_cands, A.lstats, A.npos,
                                                A.n, A.nalpha);
                block_features(bi, s_x[warp]);
            }
            __syncwarp();
            const float z = mlp_score_warp(M, s_x[warp], lane);
            if (lane == 0) s_q[j] = 1.0f / (1.0f + expf(z));  // 1 - sigmoid(z)
            __syncwarp();
        }
        __syncthreads();
        for (int t = threadIdx.x; t < ne; t += blockDim.x)
            s_score[t] = s_q[4 * t] * s_q[4 * t + 1] * s_q[4 * t + 2] * s_q[4 * t + 3];
        __syncthreads();
        for (int t = threadIdx.x; t < ne; t += blockDim.x) {
            const int idx = s_ent[t].idx;
            const long long cands = s_ent[t].cls == 1 ? s_ub[idx].candidates
                                                       : s_blk[s_first[idx / MAX_SPLITS] + idx % MAX_SPLITS].candidates;
            s_score[t] = (1.0f - s_score[t]) / sqrtf((float)(cands > 0 ? cands : 1));
        }
        __syncthreads();
        // rank sort: highest score first, ties in the reference's order
        for (int t = threadIdx.x; t < ne; t += blockDim.x) {
            const float st = s_score[t];
            int r = 0;
            for (int j = 0; j < ne; ++j) {
                const float sj = s_score[j];
                r += (sj > st || (sj == st && s_pos[j] < s_pos[t])) ? 1 : 0;
            }
            s_order[r] = t;
        }
    } else {
        for (int t = threadIdx.x; t < ne; t += blockDim.x) s_order[t] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // entries were made in the plain order: their plain starts are the prefix sums
        long long plain = 0;
        for (int e = 0; e < ne; ++e) {
            const long long cnt = s_ent[e].item0;  // the entry's item count
            s_ent[e].item0 = plain;
            s_cnt[e] = cnt;
            plain += cnt;
        }
        long long item0 = 0;
        for (int r = 0; r < ne; ++r) {
            const int e = s_order[r];
            const ItemRange R = s_ent[e];
            L->ranges[r] = ItemRange{item0, R.item0, R.cls, R.idx};
            L->scores[r] = s_go == 2 ? s_score[e] : 0.0f;
            item0 += s_cnt[e];
        }
        L->nranges = ne;
        L->learned_order = s_go == 2 ? 1 : 0;
        L->items_end = item0;
        L->item_hi_all = item0;
    }
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

cudaError_t launch_plan(const LevelArgs *d, cudaStream_t s) {
    plan_kernel<<<1, 256, 0, s>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_scorer_pack(const float *params, MlpDev *out, cudaStream_t s) {
    scorer_pack_kernel<<<(MLP_PARAMS + 255) / 256, 256, 0, s>>>(params, out);
    return cudaGetLastError();
}

}  // namespace ltlg
