// Shared host/device definitions of the CS enumeration kernels.
//
// A learn is a sequence of cost levels.  Each level has a plan: its (operator, split) blocks,
// cut into work items and listed in the order a device queue hands them out.  The level
// kernel drains the queue; the warp that finishes the level's last item closes the level
// (level starts, the find) and plans the next one on the device, so levels follow each other
// inside one persistent launch.  One launch serves many independent instances the same way:
// each instance has its own arguments, counters and plan, and the kernel's CTAs take items
// from whichever instance has some.
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
    ST_TMA = 8u,        // a bulk copy or a pipeline wait did not complete in time
    ST_STALL = 16u,     // no level progress for too long while waiting for the next plan
};
constexpr u32 ST_FATAL = ST_WAIT | ST_TABLE | ST_TMA | ST_STALL;

// Parents of a row: op << 60 | left << 30 | right (rows < 2^30).
__host__ __device__ inline u64 pack_parent(int op, u64 l, u64 r) { return ((u64)op << 60) | (l << 30) | r; }
__host__ __device__ inline int parent_op(u64 p) { return (int)((p >> 60) & 7); }
__host__ __device__ inline u64 parent_left(u64 p) { return (p >> 30) & 0x3FFFFFFFull; }
__host__ __device__ inline u64 parent_right(u64 p) { return p & 0x3FFFFFFFull; }

// Operator of slot j of a fused unary entry: 0 ~, 1 X, 2 F, 3 G.
__host__ __device__ inline int unary_slot_op(int j) { return j == 0 ? OP_NEG : j == 1 ? OP_X : j == 2 ? OP_F : OP_G; }

constexpr int POS_NONE = 0x7FFFFFFF;
constexpr int LSTATS = 2;              // row-statistics counters per cost (see count_row_stats)
constexpr u64 NO_FIND = ~0ull;         // InstCtl::found_key before any find
constexpr int SEQ_SHIFT = 40;          // InstCtl::claimed = plan sequence << 40 | next item
constexpr u64 ITEM_MASK = (1ull << SEQ_SHIFT) - 1;

enum : int { ENT_UNARY = 1, ENT_ANDOR = 2, ENT_U = 3 };

// One entry of a level's plan, in queue order: one of the reference's (operator, split)
// blocks, or (fused) every unary operator that reads the same source rows, so one load of a
// source row serves all of them.
struct Entry {
    int kind;            // ENT_UNARY, ENT_ANDOR, ENT_U
    int op;              // binary: OP_AND / OP_OR / OP_U; unary: 0
    int opmask;          // unary: bit j = slot operator j (0 ~, 1 X, 2 F, 3 G)
    int pos;             // position in the reference's block order (unary: the smallest of its operators)
    int upos[4];         // unary: position of slot operator j's block, POS_NONE when absent
    int lcost, rcost;    // operand costs (unary: lcost is the operand's, rcost 0)
    long long l0, l1, r0, r1;  // binary: left rows [l0, l1) x right rows [r0, r1); unary: source rows [r0, r1)
    long long item0;     // first queue item of the entry
    long long items;     // queue items of the entry
    long long tiles_r;   // binary: right chunks per left tile
    long long cand;      // candidates as the reference counts them (U: two per pair)
    float score;         // learned order: the entry's sort key
    int pad;
};

// The header of a level's plan.
struct Plan {
    int cost;            // the level
    int halt;            // 1: the search is over; nothing to run
    int check_only;      // on-the-fly level: acceptance only, nothing stored
    int nentries;        // entries, in queue order
    int nblocks;         // blocks in the reference's order (positions 0 .. nblocks - 1)
    int right_chunk;     // right rows per binary item
    int unary_rows;      // source rows per unary item
    int learned;         // 1: entries sorted by the scorer
    long long items;     // queue items of the level
    u64 cand;            // candidates of the level, counted as the reference counts them
};

// The mutable state of one instance's learn (device memory).  The words that many SMs touch
// during a level sit in separate 128-byte lines, so the L2 serves them in parallel: the claim
// line (producers: claim counter, limit, find key, status), the completion line (items done,
// candidates evaluated) and the row line (row reservations).
struct alignas(128) InstCtl {
    u64 claimed;         // plan sequence << SEQ_SHIFT | next queue item
    u64 limit;           // plan sequence << SEQ_SHIFT | end of the items handed out (the plan's items, or a window's end)
    u64 found_key;       // smallest (cost << 32 | block position) of an accepting candidate; NO_FIND
    u32 status;          // ST_* bits
    u32 seq;             // plans published (the current plan is sequence seq)
    alignas(128) u64 done;  // items of the current plan (or window) finished; the level (window) ends at limit's item
    u64 evaluated;       // candidates evaluated
    alignas(128) u64 row_count;  // rows handed out, letters included (may pass cap_rows on overflow)
    alignas(128) u64 found;      // (1 << 63) | parents of the find, once the level of the find has ended
    u32 found_cost;      // level of `found`
    u32 overflow_cost;   // level at which the cache first overflowed (0: none)
    u32 ne_count;        // non-empty levels so far (InstArgs::ne)
    u32 last_cost;       // the last level that ran to its end
    u32 flags;           // CTL_* bits
    u32 pad;
    u64 t_start;         // globaltimer when the first plan was published (ns)
    Plan plan;           // the current level
};
enum : u32 {
    CTL_DONE = 1u,       // the search ended (plan.halt): results are final
    CTL_CANCELLED = 2u,  // it ended because the host's cancel flag was set (time limit)
};

enum : int {
    PLAN_UNFUSED = 1,    // one unary entry per operator (per-block runs, labels)
    PLAN_LEARNED = 2,    // the planner reorders each plan by the scorer (InstArgs::model)
};

// The constant arguments of one instance's learn (device memory).
// Per-level pipeline stamps (InstArgs::level_ns), LEVEL_TRACE words per cost.
constexpr int LEVEL_TRACE = 4;
enum { LT_END = 0, LT_PUBLISHED = 1, LT_CLAIMED = 2, LT_STARTED = 3 };

struct InstArgs {
    int n;               // traces = words per CS
    int pitch;           // words per cache row (n rounded up to a multiple of 4)
    int npos;
    int nalpha;
    int key_mode;
    int rlx_type;        // KEY_REF: 0 exact pack, 1, 2, 3
    int stop_at_found;
    int find_first;      // 1: any find stops the level; 0: the first block of the reference's order that holds one
    int neg_type;
    int max_cost;
    int on_the_fly;      // plan check-only levels, ignore the overflow bit
    int plan_flags;      // PLAN_* bits
    int cf[8];           // costs of p ~ & | X F G U
    int right_chunk_big, unary_rows_big;
    int small_rows;      // small levels: right rows (unary: source rows) per item
    int tile;            // left rows staged per binary item (U: tile / 2 left rows)
    u32 gen;             // hash-set generation (1..255)
    int pad_;
    long long small_level;  // levels with fewer candidates size their items from the level (item_target)
    long long wait_spins;   // polls (~128 ns apart) before a wait for a slot publication gives up
    long long cap_rows;
    long long cap_entries;  // capacity of entries / found_par (entries holds twice that: the second half is scratch)
    long long learn_min_items;  // PLAN_LEARNED: plans of at most this many items keep the plain order
    long long item_target;  // small levels are cut into about this many items
    u64 slot_mask;
    u64 *cache;
    u64 *parents;
    u64 *keys;           // 2 words per row for KEY_REF / KEY_HASH64, else null
    u64 *prio;           // KEY_REF: per row, the priority of the candidate it holds << 1 | lock (else null)
    u64 *slots;
    const u64 *wmeta;    // per word: length mask | (positive << 63); 0 for padding
    const u32 *kmeta;    // KEY_REF: per word start | count << 16 | step << 24
    long long *ls;       // level starts, max_cost + 2 entries: rows of cost c are [ls[c], ls[c + 1])
    int *ne;             // costs of the non-empty levels, increasing (InstCtl::ne_count of them)
    u64 *level_cands;    // per cost
    u64 *level_ns;       // per cost, LEVEL_TRACE globaltimer stamps (or null): the level ended,
                         // its plan was published, its first item was claimed, its first row began
    u64 *lstats;         // per cost, LSTATS counts of stored rows by their position-0 behaviour (or null)
    Entry *entries;      // the current plan's entries
    u64 *found_par;      // per block position of the current level: (1 << 63) | parents of an accepting candidate
    InstCtl *ctl;
    const void *model;   // PLAN_LEARNED: the scorer (MlpDev)
    const volatile u32 *cancel;  // host-mapped flag (or null): when set, the next level boundary ends the search
};

// ---- Batches: many independent instances drained by one launch.  The launch holds K
// instance slots; each slot has its own buffers (InstArgs points into them).  When the search of
// a slot's instance ends, the warp that closed its last level writes the instance's result and
// sets the slot up with the next pending instance, so one launch learns the whole batch.
constexpr int WALK_MAX = 256;  // entries of a result's formula tree (the reference's 200-node limit, the root)

struct BatchIn {               // one instance of a batch: its traces in the batch's arrays
    int npos, nneg, nalpha, pad;
    long long steps0;          // first step of its traces in BatchDev::steps
    long long offs0;           // first of its n + 1 offsets in BatchDev::offs (relative to steps0)
    char alpha[32];            // sorted letters, NUL terminated
};

struct BatchOut {              // one instance's result
    int status;                // ltlg_status; LTLG_NO_MEMORY: its slot's cache overflowed (learn it alone)
    int cost;
    u64 all_ltls;
    u64 evaluated;
    long long rows;
    u64 found;                 // (1 << 63) | parents of the find (0: none or a letter)
    int letter;                // index of the separating letter, or -1
    int walk_count;            // entries of walk: (row, parents), breadth first, entry 0 the root
    int walk_overflow;         // 1: the tree has more entries than the reference prints
    u32 device_flags;
    u64 ns;                    // device time from the slot's set-up to the result (globaltimer)
    u64 walk[2 * WALK_MAX];
};

struct BatchDev {
    const BatchIn *in;
    const u32 *steps;
    const int *offs;
    BatchOut *out;
    InstArgs *args;            // per slot (the slot's buffers and the learn's options; set-up fills the rest)
    int *cur;                  // per slot: the instance it holds
    u64 *t0;                   // per slot: globaltimer at its set-up
    long long cache_words;     // per slot: language-cache words
    long long max_rows;        // per slot: rows of parents (and keys)
    int count;                 // instances
    int nslots;
    int max_pitch;
    int pad;
    unsigned long long next;   // next instance to take
    int live;                  // slots holding an instance whose search runs
    int pad2;
};

// A launch of the level kernel over one or more instances.
struct Launch {
    const InstArgs *args;    // per instance
    BatchDev *batch;         // or null: a batch drains its pending instances through the slots
    int ninst;
    int persist;             // 1: after a level, plan and run the next one in the same launch
    int tile;                // left rows staged per binary item (U: tile / 2 left rows, two candidates each)
    int stages;              // item slots in flight per CTA
    long long tile_bytes;    // shared-memory bytes of one slot's tile
};

// The feature inputs of a block (operator op) of level c: the same code on the device
// (scorer) and on the host (training records).  lstats (or null) holds LSTATS row-statistics
// counters per cost, up to max_cost.
__host__ __device__ inline BlockInfo block_info(int op, int c, int lcost, long long lrows, long long rrows,
                                                long long cand, int position, const int *cf, int nblocks,
                                                long long level_cands, const u64 *lstats, int max_cost, int npos,
                                                int n, int nalpha) {
    const bool un = op == OP_NEG || op == OP_X || op == OP_F || op == OP_G;
    BlockInfo bi{};
    bi.op = op;
    bi.cost = c;
    bi.c1 = cf[0];
    bi.lcost = lcost;
    bi.rcost = un ? 0 : c - lcost - cf[op + 1];
    bi.position = position;
    bi.nblocks = nblocks;
    bi.lrows = lrows;
    bi.rrows = un ? 1 : rrows;
    bi.candidates = cand;
    bi.level_cands = level_cands;
    for (int k = 0; k < 2; ++k) {
        bi.lstat[k] = (lstats && bi.lcost >= 0 && bi.lcost <= max_cost) ? (long long)lstats[(u64)bi.lcost * LSTATS + k] : 0ll;
        bi.rstat[k] =
            (lstats && !un && bi.rcost >= 0 && bi.rcost <= max_cost) ? (long long)lstats[(u64)bi.rcost * LSTATS + k] : 0ll;
    }
    bi.npos = npos;
    bi.nneg = n - npos;
    bi.nalpha = nalpha;
    return bi;
}

// Threads per CTA of the level kernel (one producer warp and the consumer warps).
constexpr int LEVEL_THREADS = 1024;
constexpr int LEVEL_CONSUMERS = LEVEL_THREADS / 32 - 1;
// Shared memory of one CTA of the level kernel for `stages` slots of tile_bytes each.
size_t level_kernel_smem(int stages, long long tile_bytes);

// Launch wrappers (learn.cu).  The kernels read their arguments from device memory, so a
// launch (or a captured graph) stays valid while the arguments change between learns.
cudaError_t launch_levels(const Launch &host_copy, const Launch *dev, int grid, int hash_kind, cudaStream_t s);
cudaError_t launch_first_plan(const InstArgs *d, int ninst, int open, cudaStream_t s);
// A batch's first instances: each slot takes pending instances until one needs levels.
cudaError_t launch_batch_start(BatchDev *d, int nslots, int hash_kind, cudaStream_t s);
cudaError_t launch_insert_letters(const InstArgs *d, int nalpha, int hash_kind, cudaStream_t s);
cudaError_t launch_walk(const u64 *parents, int nalpha, u64 found, u64 *out, int cap, cudaStream_t s);
// Plans level `cost` of the instance from its level starts (the levels below must be complete) and
// publishes the plan closed: the host opens it (host-driven levels, block labels).
cudaError_t launch_plan_level(const InstArgs *d, int cost, cudaStream_t s);
cudaError_t launch_scorer_pack(const float *params, MlpDev *out, cudaStream_t s);
int level_kernel_ctas_per_sm(int hash_kind, size_t smem);
// prog: (op, arg) pairs in postfix, op OP_ATOM with arg = letter index; stack: depth x n words.
cudaError_t launch_eval_formula(const int *prog, int len, const u64 *atoms, const u64 *lenmask, int n, u64 *stack,
                                u64 *out, cudaStream_t s);
cudaError_t launch_apply_op(int op, const u64 *a, const u64 *b, const u64 *wmeta, int n, int pitch, int count,
                            u64 *out, u64 *out2, u64 *fp, cudaStream_t s);

}  // namespace ltlg
