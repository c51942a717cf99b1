// Shared host/device definitions of the CS enumeration kernels.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "order.cuh"

namespace ltlg {

using u64 = unsigned long long;
using u32 = unsigned int;

// Operator codes: the reference's region index i % 7 (code/ltli6463.cu:892-926).
enum : int { OP_NEG = 0, OP_AND = 1, OP_OR = 2, OP_X = 3, OP_F = 4, OP_G = 5, OP_U = 6, OP_ATOM = 7 };

// Uniqueness keys (ltlg_key_mode).
enum : int { KEY_EXACT = 0, KEY_REF = 1, KEY_HASH64 = 2 };

// Device status bits.
enum : u32 {
    ST_OVERFLOW = 1u,   // a new CS found no free cache row (the reference's onTheFly switch)
    ST_WAIT = 2u,       // a wait for a slot publication gave up
    ST_TABLE = 4u,      // hash set full
    ST_TMA = 8u,        // a bulk copy did not complete in time
};

// Parents of a row: op << 60 | left << 30 | right (rows < 2^30).
__host__ __device__ inline u64 pack_parent(int op, u64 l, u64 r) { return ((u64)op << 60) | (l << 30) | r; }
__host__ __device__ inline int parent_op(u64 p) { return (int)((p >> 60) & 7); }
__host__ __device__ inline u64 parent_left(u64 p) { return (p >> 30) & 0x3FFFFFFFull; }
__host__ __device__ inline u64 parent_right(u64 p) { return p & 0x3FFFFFFFull; }

struct DevCtl {
    u64 row_count;   // rows handed out, letters included (may pass cap_rows on overflow)
    u64 found;       // 0, or (1 << 63) | parents of an accepting candidate
    u64 evaluated;   // candidates evaluated
    u32 status;      // ST_* bits
    u32 found_cost;  // level at which `found` was set
    u32 overflow_cost;  // level at which the cache first overflowed
    u32 ctas_done;   // CTAs of the running level-kernel launch that have finished (the last resets it)
    u64 queue[8];    // next work item of each operator's kernel
};

// One (operator, split) block of a level.  Unary: source rows [r0, r1).
// Binary: left rows [l0, l1) x right rows [r0, r1).
struct BlockDesc {
    int op;
    int lcost;           // cost of the left operand (unary: of the operand)
    int opmask;          // fused unary blocks: bit 0 ~, 1 X, 2 F, 3 G over the same source rows
    int pad;             // position of the block in the reference's order within its level
    long long l0, l1, r0, r1;
    long long item0;     // first work item of this block within its operator
    long long items;     // work items of this block
    long long tiles_r;   // binary: right chunks per left tile
    long long candidates;  // as the reference counts them (U: two per pair)
};

constexpr int MAX_SPLITS = 64;   // blocks per operator and level in a device-planned level
constexpr int MAX_RANGES = 4 + 3 * MAX_SPLITS;  // entries of a level's item table
constexpr int UNARY_ROWS = 1;    // source rows per warp in a unary item (each with every operator of its mask)
constexpr int MAX_COSTS = 512;   // level starts kept on the device
constexpr int LSTATS = 2;        // row-statistics counters per cost (see count_row_stats)

// One entry of a level's item table: a block and where its items start.
struct ItemRange {
    long long item0;     // first item of the entry in the order the queue runs
    long long plain0;    // the same item's number in the plain order
    int cls;             // 1 unary (ublocks[idx]), 2 & or | (blocks[idx / MAX_SPLITS][idx % MAX_SPLITS]), 3 U
    int idx;
};

enum : int {
    PLAN_UNFUSED = 1,    // one unary block per operator (per-block runs, learned order, labels)
    PLAN_LEARNED = 2,    // order the item table by the scorer (LevelArgs::model), highest first
};

// The plan of the level being enumerated, in device memory.  The planner kernel writes it
// from the level starts; the host writes it directly in the per-block schedule.
struct DevLevel {
    int cost;            // the level being enumerated (the planner advances it)
    int halt;            // 1: every operator kernel of this level exits at once
    int check_only;      // on-the-fly: acceptance only, no dedupe, no storing
    int on_the_fly;      // set by the host: plan check-only levels and ignore the overflow bit
    int seq;             // planner runs since the learn started (the level's host ring slot is (seq - 1) % RING)
    int pad0;
    long long item_hi_all;  // all work items of the level
    long long items_end;    // the level kernel takes items from ctl->queue[0] below it
    int right_chunk;
    int unary_rows;
    int nblocks[8];
    long long total_items[8];
    long long item_hi[8];  // an operator kernel takes items from its queue until item_hi
    u64 level_cands;     // candidates of the level, counted as the reference counts them
    int plan_flags;      // set by the host: PLAN_* bits
    int nublocks;        // unary blocks the level kernel works from (fused over operators
                         // unless PLAN_UNFUSED)
    BlockDesc ublocks[4];
    BlockDesc blocks[7][MAX_SPLITS];
    // The level's blocks in the order the queue runs: entry e covers queue items
    // [ranges[e].item0, ranges[e + 1].item0) (the last one up to items_end).
    int nranges;
    int learned_order;   // 1: the table is sorted by score and the queue runs through it
    ItemRange ranges[MAX_RANGES];
    float scores[MAX_RANGES];  // learned order: each entry's sort key (chance of a find / sqrt(candidates))
};

static_assert(sizeof(DevCtl) % 8 == 0 && offsetof(DevLevel, blocks) % 8 == 0, "level summaries copy 8-byte words");

struct LevelArgs {
    // constant during a learn
    int n;               // traces = words per CS
    int pitch;           // words per cache row (n rounded up to a multiple of 4)
    int npos;
    int nalpha;
    int key_mode;
    int rlx_type;        // KEY_REF: 0 exact pack, 1, 2, 3
    u32 gen;             // hash-set generation (1..255)
    int stop_at_found;
    int left_tile;
    int neg_type;
    int max_cost;
    int nwarps;
    int cf[8];           // costs of p ~ & | X F G U
    int right_chunk_big, unary_rows_big;
    int small_rows;      // small levels: right rows (unary: source-row pairs) per warp and item
    int hash_kind;       // fingerprint kind of the operator kernels (0 multiply-add, 1 fmix64)
    long long wait_spins;   // polls (~128 ns apart) before a wait for a slot publication gives up
    long long small_level;  // levels with fewer candidates use one row per warp per item
    long long cap_rows;
    u64 *cache;
    u64 *parents;
    u64 *keys;           // 2 words per row for KEY_REF / KEY_HASH64, else null
    u64 *slots;
    u64 slot_mask;
    const u64 *wmeta;    // per word: length mask | (positive << 63); 0 for padding
    const u32 *kmeta;    // KEY_REF: per word start | count << 16 | step << 24
    DevCtl *ctl;
    DevLevel *lev;
    long long *ls;       // level starts: rows of cost c are [ls[c], ls[c + 1])
    u64 *level_cands;    // per cost
    const void *model;   // PLAN_LEARNED: the scorer (MlpDev)
    u64 *lstats;         // per cost, LSTATS counts of stored rows by their position-0 behaviour (or null)
    void *ring;          // device view of the host's ring of level summaries (or null)
    int ring_slots;
    long long grid;      // CTAs of a level-kernel launch (a level of fewer items runs in one wave)
    // per level (filled into the shared copy from the plan)
    int cost;
    int check_only;
    int right_chunk;
    int unary_rows;
};

// The feature inputs of block b (operator op) of level c: the same code on the device
// (planner) and on the host (training records).  ls[k] is the first row of cost k; lstats
// (or null) holds LSTATS row-statistics counters per cost.
__host__ __device__ inline BlockInfo block_info(const BlockDesc &b, int op, int c, const int *cf, int nblocks,
                                                long long level_cands, const u64 *lstats, int npos, int n,
                                                int nalpha) {
    const bool un = op == OP_NEG || op == OP_X || op == OP_F || op == OP_G;
    BlockInfo bi{};
    bi.op = op;
    bi.cost = c;
    bi.c1 = cf[0];
    bi.lcost = b.lcost;
    bi.rcost = un ? 0 : c - b.lcost - cf[op + 1];
    bi.position = b.pad;
    bi.nblocks = nblocks;
    bi.lrows = un ? b.r1 - b.r0 : b.l1 - b.l0;
    bi.rrows = un ? 1 : b.r1 - b.r0;
    bi.candidates = b.candidates;
    bi.level_cands = level_cands;
    for (int k = 0; k < 2; ++k) {
        bi.lstat[k] = (lstats && bi.lcost <= MAX_COSTS) ? (long long)lstats[(u64)bi.lcost * LSTATS + k] : 0ll;
        bi.rstat[k] = (lstats && !un && bi.rcost <= MAX_COSTS) ? (long long)lstats[(u64)bi.rcost * LSTATS + k] : 0ll;
    }
    bi.npos = npos;
    bi.nneg = n - npos;
    bi.nalpha = nalpha;
    return bi;
}

// Launch wrappers (ltl_kernels.cu).  A level is one kernel (launch_level) that drains
// ctl->queue[0]; the planner (launch_plan) writes its plan first.  The kernels read their
// arguments from `d`, a copy of `a` in device memory, so a captured graph stays valid while
// `*d` changes; `a` (host) selects the template instance and the shared-memory size.
int level_kernel_smem_bytes(int left_tile, int pitch);
int level_kernel_max_ctas_per_sm(int left_tile, int hash_kind, int block, int pitch);
cudaError_t launch_level(const LevelArgs &a, const LevelArgs *d, int grid, int block, cudaStream_t s);
cudaError_t launch_plan(const LevelArgs *d, cudaStream_t s);
cudaError_t launch_insert_letters(const LevelArgs &a, const LevelArgs *d, int nalpha, cudaStream_t s);
cudaError_t launch_walk(const u64 *parents, int nalpha, u64 found, u64 *out, int cap, cudaStream_t s);
cudaError_t launch_scorer_pack(const float *params, MlpDev *out, cudaStream_t s);
// prog: (op, arg) pairs in postfix, op OP_ATOM with arg = letter index; stack: depth x n words.
cudaError_t launch_eval_formula(const int *prog, int len, const u64 *atoms, const u64 *lenmask, int n, u64 *stack,
                                u64 *out, cudaStream_t s);
cudaError_t launch_apply_op(int op, const u64 *a, const u64 *b, const u64 *wmeta, int n, int pitch, int count,
                            u64 *out, u64 *out2, u64 *fp, cudaStream_t s);

}  // namespace ltlg
