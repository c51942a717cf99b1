/*
 * ltlgpu — C ABI of the B200 characteristic-set (CS) enumerator.
 *
 * This is the drop-in boundary for the reference's enumeration entry
 *     std::string LTLI(const unsigned short *costFun, unsigned short maxCost,
 *                      unsigned RlxUnqChkTyp, unsigned NegType, std::set<char> alphabet,
 *                      int &LTLcost, std::uint64_t &allLTLs,
 *                      vector<vector<string>> pos, vector<vector<string>> neg)
 * (MojtabaValizadeh/ltl-learning-on-gpus, code/ltli6463.cu:1043-1052), restated with plain
 * pointers and sizes.  The ltli6463-compatible executable (csrc/cli_ltli6463.cpp) and the
 * Python bindings call only what is declared here.
 *
 * Conventions
 *   - Traces: positives first, then negatives.  Each time step is a uint32 mask with
 *     bit (letter - 'a') set when that letter holds; offsets[t] .. offsets[t + 1] are the
 *     steps of trace t.  This is the reference's token strings (ltli6463.cu:1526-1565)
 *     packed into bits.
 *   - The alphabet is the sorted letter string (the reference's std::set<char> order); the
 *     letter at index j is CS row j.
 *   - Operator codes are the reference's region index i % 7 (ltli6463.cu:892-926):
 *     0 ~, 1 &, 2 |, 3 X, 4 F, 5 G, 6 U; 7 marks a letter row.
 *   - Status codes replace the reference's sentinel strings ("not_found",
 *     "see_the_error", "Size of the output is too big"); the formula string keeps the
 *     sentinel text so string-level callers see what the reference printed.
 *   - The caller owns every input buffer.  The library allocates the result's arrays and
 *     frees them in ltlg_result_free.  An engine is not thread-safe: one host thread per
 *     engine (each engine owns its own CUDA stream and device buffers).
 */
#ifndef LTLGPU_H
#define LTLGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LTLG_API __attribute__((visibility("default")))
#define LTLG_ABI_VERSION 2

typedef struct ltlg_traces {
    int32_t num_pos;
    int32_t num_neg;
    const char *alphabet;      /* sorted letters, NUL terminated */
    const uint32_t *steps;     /* per time step, bit (letter - 'a') */
    const int32_t *offsets;    /* num_pos + num_neg + 1 entries, offsets[0] == 0 */
} ltlg_traces;

enum ltlg_key_mode {
    LTLG_KEY_EXACT = 0,        /* uniqueness on the full CS (verified word by word) */
    LTLG_KEY_REF = 1,          /* the reference's relaxed keys, type = rlx_unq_chk_type (ltli6463.cu:57-141) */
    LTLG_KEY_HASH64 = 2        /* relaxed: a 64-bit fingerprint of the full CS, not verified */
};

enum ltlg_schedule {
    LTLG_SCHEDULE_FUSED = 0,   /* one persistent launch per level drains every block of the level */
    LTLG_SCHEDULE_PER_BLOCK = 1 /* one launch per (operator, split) block, in order; per-block stats */
};

enum ltlg_order {
    LTLG_ORDER_PLAIN = 0,      /* the reference's operator / split order (ltli6463.cu:1209-1440) */
    LTLG_ORDER_LEARNED = 1     /* blocks of a level sorted by the loaded scorer, highest first */
};

enum ltlg_status {
    LTLG_FOUND = 0,
    LTLG_NOT_FOUND = 1,
    LTLG_INPUT_LIMITS = 2,     /* more than 63 steps in a trace (or > 64 traces with limit_traces) */
    LTLG_TIMEOUT = 3,
    LTLG_NO_MEMORY = 4,
    LTLG_BAD_ARGS = 5,
    LTLG_CUDA_ERROR = 6,
    LTLG_DEVICE_WAIT = 7,      /* a bounded device-side wait gave up; results are not trusted */
    LTLG_TABLE_FULL = 8,
    LTLG_NO_DEVICE = 9,
    LTLG_FORMULA_TOO_LONG = 10 /* the formula does not fit the caller's buffer (ltlg_learn_noalloc) */
};

/* Bytes that always hold a returned formula and its NUL.  The reference prints "Size of the
 * output is too big" once the found formula has more than 199 operator nodes below its root
 * (its 600-int index buffer, ltli6463.cu:959-985); 200 binary nodes and 201 letters make 1,201
 * characters. */
#define LTLG_FORMULA_MAX_BYTES 1280

typedef struct ltlg_engine_config {
    int32_t device;            /* CUDA device ordinal */
    int32_t slots_log2;        /* hash-set slots = 2^slots_log2 (8-byte slots) */
    int64_t cache_bytes;       /* language-cache budget in bytes (rows = budget / (8 * pitch)) */
    int64_t max_rows;          /* upper bound on cache rows (<= 2^30); 0 = budget only */
    int32_t max_traces;        /* largest n the engine accepts */
    int32_t block_threads;     /* kept for the layout; the level kernel runs one CTA of 1024 threads
                                  per SM (a producer warp and 31 consumer warps) */
    int32_t left_tile;         /* left rows staged in shared memory per binary work item: 2, 4 or 8 */
    int32_t right_chunk;       /* right rows per binary work item of a large level */
    int32_t unary_rows;        /* source rows per unary work item of a large level */
    int32_t small_rows;        /* levels below the small-level size: right rows (unary: source rows)
                                  per work item; 0 = 1 */
    int32_t wait_spins;        /* bound of a device wait for another warp's hash-slot publication, in
                                  polls about 128 ns apart; a wait that runs out ends the learn with
                                  LTLG_DEVICE_WAIT.  0 = 2^22 (about half a second) */
    int32_t pad_;
    int64_t small_level;       /* levels with fewer candidates are cut into work items of about
                                  rows / (2 x CTAs x item slots) rows each (at least small_rows, at
                                  most right_chunk / unary_rows); larger levels use right_chunk /
                                  unary_rows.  0 = every level is sized that way */
} ltlg_engine_config;

typedef struct ltlg_options {
    int32_t cost_fun[8];       /* p ~ & | X F G U, each in 1..SHRT_MAX */
    int32_t max_cost;          /* levels up to max_cost (1..SHRT_MAX, as the reference's maxCost) are
                                  enumerated; level arrays and plans are sized for it per learn */
    int32_t rlx_unq_chk_type;  /* the reference's argument 11 (1, 2, 3), used with LTLG_KEY_REF */
    int32_t neg_type;          /* 1: negate every formula, 2: negate letters only (ltli6463.cu:1212) */
    int32_t key_mode;          /* ltlg_key_mode */
    int32_t schedule;          /* ltlg_schedule */
    int32_t order;             /* ltlg_order */
    int32_t stop_at_found;     /* 1: stop at the first accepting candidate; 0: enumerate to max_cost */
    int32_t limit_traces;      /* 1: apply the reference's 64-trace limit too (ltli6463.cu:1078) */
    int32_t record_levels;     /* 1: time each level with CUDA events */
    int32_t pad_;
    double time_limit_s;       /* > 0: stop between levels once exceeded */
} ltlg_options;

typedef struct ltlg_level_stat {
    int32_t cost;
    int32_t blocks;
    uint64_t candidates;       /* candidates the device evaluated at this cost */
    uint64_t uniques;          /* rows stored at this cost */
    double ms;                 /* device time of the level (record_levels) */
    /* record_levels, fused schedule: microseconds from the end of the level below to this
       level's plan being published, its first item claimed, its first row begun (0: none) */
    double plan_us;
    double claim_us;
    double start_us;
} ltlg_level_stat;

typedef struct ltlg_block_stat {
    int32_t cost;
    int32_t op;                /* operator code */
    int32_t left_cost;         /* split: cost of the left operand (unary: operand cost) */
    int32_t right_cost;
    int64_t stored_before;     /* rows stored when the block started (the reference's StoredLTLs) */
    uint64_t all_before;       /* candidates counted before the block (the reference's AllLTLs) */
    int64_t to_check;          /* candidates in the block (the reference's ToBeChecked) */
} ltlg_block_stat;

typedef struct ltlg_result {
    int32_t status;            /* ltlg_status */
    int32_t cost;              /* LTLcost as the reference reports it */
    uint64_t all_ltls;         /* candidates counted as the reference counts them */
    uint64_t evaluated;        /* candidates the device actually evaluated */
    int64_t rows;              /* rows in the language cache (letters included) */
    char *formula;             /* the reference's string format, or its sentinel text */
    double seconds;            /* host wall time of the call */
    double device_ms;          /* device time of the level loop */
    int32_t num_levels;
    int32_t num_blocks;
    ltlg_level_stat *levels;
    ltlg_block_stat *blocks;   /* filled with LTLG_SCHEDULE_PER_BLOCK */
    int32_t found_op;          /* root operator of the returned formula (7 for a letter) */
    uint32_t device_flags;     /* raw device status bits (overflow, waits, table) */
    int32_t on_the_fly;        /* 1 once the cache overflowed (the reference's onTheFly) */
    int32_t launches;          /* kernels this call launched */
} ltlg_result;

typedef struct ltlg_engine ltlg_engine;

/* Defaults: device 0, 2^27 slots, 16 GiB cache, n <= 8192, 1024 threads, left tile 4,
   right chunk 16, unary rows 32, small rows 1, default wait bound and small-level size. */
LTLG_API void ltlg_default_engine_config(ltlg_engine_config *cfg);
/* The reference's defaults: unit costs, maxCost 500, type 3, NegType 2, exact keys, fused, plain. */
LTLG_API void ltlg_default_options(ltlg_options *opt);

/* A handle owning one device's buffers and stream (the reference allocates and frees its
 * device memory inside every LTLI call, ltli6463.cu:1152-1190, :1487-1493).  Without a CUDA
 * device: LTLG_NO_DEVICE and no handle.  Destroy accepts NULL. */
LTLG_API int ltlg_engine_create(const ltlg_engine_config *cfg, ltlg_engine **out);
LTLG_API void ltlg_engine_destroy(ltlg_engine *eng);

/* Learn one formula.  Replaces LTLI (ltli6463.cu:1043); the engine's buffers are reused. */
LTLG_API int ltlg_engine_learn(ltlg_engine *eng, const ltlg_traces *traces, const ltlg_options *opt,
                               ltlg_result *res);

/* The engine's CUDA stream (a cudaStream_t), for callers that time or order work around
 * learns with their own events. */
LTLG_API void *ltlg_engine_stream(ltlg_engine *eng);

/* One-shot form, the reference's LTLI (ltli6463.cu:1043-1052) call for call: creates an
 * engine sized for the input, learns, destroys it.  Malformed traces (LTLG_BAD_ARGS) and
 * the input limits (LTLG_INPUT_LIMITS, ltli6463.cu:1078-1083) are reported before any
 * device call. */
LTLG_API int ltlg_learn(const ltlg_traces *traces, const ltlg_options *opt, ltlg_result *res);

/* Frees the strings and arrays of a result (the reference returns std::string; its sentinel
 * strings "not_found", "see_the_error", "Size of the output is too big" are statuses and
 * formula text here, ltli6463.cu:1461, :1082, :984).  Accepts NULL. */
LTLG_API void ltlg_result_free(ltlg_result *res);

/* Batched learning: independent instances learned by one persistent launch of the level kernel.
 * The batch holds `workers` instance slots, each with the buffers one engine of `cfg` would have
 * (cache_bytes of language cache, 2^slots_log2 hash slots); the instances are uploaded at once and
 * a device queue hands them to the slots: when an instance's search ends, the slot writes its
 * result and takes the next pending instance, so the small levels of many instances run side by
 * side and no host round trip happens between levels or instances.  results[i] belongs to
 * traces[i]; free each with ltlg_result_free.  Instances with the reference's relaxed keys, the
 * learned order, the per-block schedule or a time limit, and any instance whose slot's cache
 * overflows, are learned one at a time on one engine of `cfg` instead.  The reference has one
 * instance per process (code/dc.py:33-43 runs the binary once per sub-problem); this replaces
 * that loop. */
typedef struct ltlg_batch ltlg_batch;
LTLG_API int ltlg_batch_create(const ltlg_engine_config *cfg, int32_t workers, ltlg_batch **out);
LTLG_API void ltlg_batch_destroy(ltlg_batch *b);
LTLG_API int ltlg_batch_learn(ltlg_batch *b, const ltlg_traces *traces, int32_t count, const ltlg_options *opt,
                              ltlg_result *results);
/* The batch's stream (a cudaStream_t) for worker 0, NULL otherwise (for event timing around batch
 * calls). */
LTLG_API void *ltlg_batch_stream(ltlg_batch *b, int32_t worker);

/* Learn without allocating: no counterpart in the reference.  For callers that cannot
 * allocate device memory (GPU memory owned by another allocator, or no cudaMalloc allowed
 * after start-up): every device buffer lives in one static 64 MiB array that the library
 * holds on each GPU until exit, and host work uses stack arrays.  At most 64 traces of at
 * most 63 steps (more: LTLG_INPUT_LIMITS); exact or 64-bit-fingerprint keys; max_cost below
 * 512; a level that overflows the scratch returns LTLG_NO_MEMORY.  The formula is written to
 * the caller's buffer (formula_cap bytes, at least 16; LTLG_FORMULA_MAX_BYTES always
 * suffices), the cost and candidate count to *cost and *all_ltls.  A formula (or the
 * reference's "Size of the output is too big") that does not fit returns
 * LTLG_FORMULA_TOO_LONG with an empty string and *cost and *all_ltls set.  All calls share
 * the array: calls whose GPU work overlaps race, so callers serialise them.  The first call
 * on a device looks up the array's address there; make it before any stream capture. */
LTLG_API int ltlg_learn_noalloc(const ltlg_traces *traces, const ltlg_options *opt, char *formula,
                                int32_t formula_cap, int32_t *cost, uint64_t *all_ltls);

/* After a learn: copy cache rows [first, first + count) (n words each, pitch dropped) and
 * their packed parents (op << 60 | left << 30 | right) to host memory.  Either pointer may
 * be NULL.  Returns 0 or an ltlg_status. */
LTLG_API int ltlg_engine_read_rows(ltlg_engine *eng, int64_t first, int64_t count, uint64_t *rows,
                                   uint64_t *parents);
/* Row ranges of each cost after a learn: starts[c] for c in 0..max_cost + 1. */
LTLG_API int ltlg_engine_level_starts(ltlg_engine *eng, int64_t *starts, int32_t count);

/* Fault injection for tests (no counterpart in the reference).  Marks the hash-set slot of the
 * CS `cs` (n words, exact keys) as "publication pending" for the engine's next learn: the first
 * candidate of that learn with this CS waits for a publication that never comes, gives up after
 * wait_spins polls and the learn returns LTLG_DEVICE_WAIT.  The mark belongs to one hash-set
 * generation, so the learn after that one starts clean.  Returns 0 or an ltlg_status. */
LTLG_API int ltlg_engine_hold_slot(ltlg_engine *eng, const uint64_t *cs, int32_t n);

/* Device building blocks, for kernel-level parity tests (device buffers are allocated
 * and freed inside; host arrays in and out). */
LTLG_API int ltlg_device_apply_op(int32_t op, const uint64_t *a, const uint64_t *b, const uint64_t *lenmask,
                                  int32_t n, int32_t count, uint64_t *out, uint64_t *out2, uint64_t *fp);

/* Scarlet file reader with the reference's rules (ltli6463.cu:1500-1573).  Allocates the
 * arrays inside *out; release with ltlg_traces_free. Returns 0 or LTLG_BAD_ARGS. */
LTLG_API int ltlg_read_scarlet(const char *path, ltlg_traces *out);
LTLG_API void ltlg_traces_free(ltlg_traces *t);

/* ---- Learned block order (no counterpart in the reference: its enumerator always runs a
 * level's blocks in the fixed operator / split order).  A scorer, a multilayer perceptron
 * 32 -> 64 -> 64 -> 1 (ReLU; BF16 operands, FP32 accumulation), rates each (operator, left
 * cost, right cost) block of a level; with ltlg_options.order = LTLG_ORDER_LEARNED the level's
 * blocks are drained highest score first.  Only the order changes: the level still runs to its
 * end unless a find stops it, so the cost found is the plain enumerator's. */
#define LTLG_SCORER_FEATURES 32
#define LTLG_SCORER_PARAMS 6337  /* W1[64][32], b1[64], W2[64][64], b2[64], W3[64], b3 (FP32) */

typedef struct ltlg_block_record {
    int32_t cost;              /* the level */
    int32_t op;                /* operator code */
    int32_t lcost, rcost;      /* operand costs (rcost 0 for unary blocks) */
    int32_t position;          /* index in the reference's order within the level */
    int32_t won;               /* 1: the block holds a candidate that accepts */
    int64_t candidates;
    float features[LTLG_SCORER_FEATURES];
} ltlg_block_record;

/* What a block's features are computed from (host side; the device planner uses the same
 * function).  Costs are level costs, rows are cache rows.  lstat / rstat: stored rows of the
 * (left / right) operand level that hold at position 0 on every positive trace, and that
 * hold at position 0 on no negative trace. */
typedef struct ltlg_block_info {
    int32_t op, cost, c1, lcost, rcost, position, nblocks, pad_;
    int64_t lrows, rrows, candidates, level_cands;
    int64_t lstat[2], rstat[2];
    int32_t npos, nneg, nalpha, pad2_;
} ltlg_block_info;

LTLG_API void ltlg_block_features(const ltlg_block_info *info, float *features);

/* Load a scorer (LTLG_SCORER_PARAMS floats) into the engine / every engine of a batch. */
LTLG_API int ltlg_engine_set_scorer(ltlg_engine *eng, const float *params, int32_t count);
LTLG_API int ltlg_batch_set_scorer(ltlg_batch *b, const float *params, int32_t count);

/* Training records of one instance: learn it in plain order (stop at the first find), then run
 * every block of the level of the find again, alone, in check-only mode (acceptance tested on
 * every candidate, nothing stored) and record whether it holds an accepting candidate.  Writes
 * up to cap records and their count; res is the learn's result (free with ltlg_result_free). */
LTLG_API int ltlg_engine_label_blocks(ltlg_engine *eng, const ltlg_traces *traces, const ltlg_options *opt,
                                      ltlg_block_record *records, int32_t cap, int32_t *count, ltlg_result *res);

/* The scorer's kernels on host arrays (features: count x 32 floats, row-major).
 * forward: logits.  grad: gradient of the mean weighted binary cross-entropy (weight pos_weight
 * on label-1 records) and the loss.  train: Adam on the GPU, params updated in place; epoch_loss
 * (optional) receives the mean loss of each epoch. */
typedef struct ltlg_train_config {
    int32_t epochs;
    int32_t batch;
    float lr;
    float pos_weight;
    float beta1, beta2, eps;
    float weight_decay;
    uint64_t seed;             /* shuffling */
} ltlg_train_config;

LTLG_API int ltlg_scorer_forward(const float *params, const float *features, int32_t count, float *logits);
LTLG_API int ltlg_scorer_grad(const float *params, const float *features, const float *labels, int32_t count,
                              float pos_weight, float *grad, float *loss);
LTLG_API int ltlg_scorer_train(float *params, const float *features, const float *labels, int32_t count,
                               const ltlg_train_config *cfg, float *epoch_loss);

/* Evaluate a formula string on every trace, on the device (the reference checks formulas on
 * the host in code/dc.py:136-187).  The string uses the enumerator's output format, parsed as
 * dc.py's bitVec does: "~(f)", "X(f)", "F(f)", "G(f)", "(f)&(g)", "(f)|(g)", "(f)U(g)", single
 * letters of the alphabet.  cs (optional): the formula's CS per trace (bit k: holds at
 * position k); holds (optional): 1 where it holds at position 0.  LTLG_BAD_ARGS on a malformed
 * formula or an unknown letter, LTLG_INPUT_LIMITS on a trace longer than 63 steps. */
LTLG_API int ltlg_evaluate(const ltlg_traces *traces, const char *formula, uint64_t *cs, uint8_t *holds);

LTLG_API const char *ltlg_status_string(int status);
LTLG_API int ltlg_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
