// Shared host/device definitions of the CS enumeration kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

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
    u32 pad;
    u64 queue[8];    // next work item of each operator's kernel
};

// One (operator, split) block of a level.  Unary: source rows [r0, r1).
// Binary: left rows [l0, l1) x right rows [r0, r1).
struct BlockDesc {
    int op;
    int pad;
    long long l0, l1, r0, r1;
    long long item0;     // first work item of this block
    long long items;     // work items of this block
    long long tiles_r;   // binary: right chunks per left tile
};

struct LevelArgs {
    const BlockDesc *blocks;  // this operator's blocks
    u64 *queue;               // this operator's work-item counter
    int nblocks;
    int n;               // traces = words per CS
    int pitch;           // words per cache row (n rounded up to a multiple of 4)
    int npos;
    long long total_items;
    long long cap_rows;
    u64 *cache;
    u64 *parents;
    u64 *keys;           // 2 words per row for KEY_REF / KEY_HASH64, else null
    u64 *slots;
    u64 slot_mask;
    const u64 *wmeta;    // per word: length mask | (positive << 63); 0 for padding
    const u32 *kmeta;    // KEY_REF: per word start | count << 16 | step << 24
    DevCtl *ctl;
    int key_mode;
    int rlx_type;        // KEY_REF: 0 exact pack, 1, 2, 3
    u32 gen;             // hash-set generation (1..255)
    int stop_at_found;
    int check_only;      // on-the-fly: acceptance only, no dedupe, no storing
    int right_chunk;
    int unary_rows;
    int left_tile;
};

// Launch wrappers (ltl_kernels.cu).  One kernel per operator drains the work items of
// that operator's blocks; binary kernels stage left tiles of left_tile rows (U: half).
int op_kernel_smem_bytes(int op, int left_tile, int pitch);
cudaError_t launch_op(int op, const LevelArgs &a, int grid, int block, cudaStream_t s);
int op_kernel_max_ctas_per_sm(int op, int left_tile, int hash_kind, int block, int pitch);
cudaError_t launch_insert_letters(const LevelArgs &a, int nalpha, cudaStream_t s);
cudaError_t launch_walk(const u64 *parents, int nalpha, u64 found, u64 *out, int cap, cudaStream_t s);
cudaError_t launch_apply_op(int op, const u64 *a, const u64 *b, const u64 *wmeta, int n, int pitch, int count,
                            u64 *out, u64 *out2, u64 *fp, cudaStream_t s);

}  // namespace ltlg
