/*
 * CPU oracle for the characteristic-set (CS) enumeration of
 * MojtabaValizadeh/ltl-learning-on-gpus (code/ltli6463.cu).
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this
 * library; only tests/, the smoke check and the CPU-baseline leg of the
 * benchmark use it, as the checker.
 *
 * Parity status: pinned against outputs of the reference binary itself (built
 * from the reference sources by oracle/Makefile into oracle/_ref/ and run on a
 * B200) on the seeded fixtures under tests/golden/.
 */
#ifndef LTL_ORACLE_H
#define LTL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Traces, positives first.  Step masks carry bit (letter - 'a'). */
typedef struct lo_traces {
    int32_t num_pos;
    int32_t num_neg;
    const char *alphabet;     /* sorted letters, NUL terminated (the reference's std::set<char>) */
    const uint32_t *steps;
    const int32_t *offsets;   /* num_pos + num_neg + 1 entries */
} lo_traces;

/* Uniqueness keys. */
enum {
    LO_KEY_EXACT = 0,   /* full CS compared word by word */
    LO_KEY_REF1 = 1,    /* reference keying, RlxUnqChkTyp 1 (exact 126-bit pack when lenSum <= 126) */
    LO_KEY_REF2 = 2,    /* reference keying, RlxUnqChkTyp 2 */
    LO_KEY_REF3 = 3,    /* reference keying, RlxUnqChkTyp 3 */
    LO_KEY_HASH64 = 4   /* 64-bit fingerprint of the full CS, no verification */
};

enum { LO_FOUND = 0, LO_NOT_FOUND = 1, LO_INPUT_LIMITS = 2, LO_TIMEOUT = 3, LO_NO_MEMORY = 4,
       LO_BAD_ARGS = 5, LO_CHUNK_TOO_SMALL = 6 };

/* Operator codes: the reference's region index i % 7 (code/ltli6463.cu:892-926). */
enum { LO_OP_NEG = 0, LO_OP_AND = 1, LO_OP_OR = 2, LO_OP_X = 3, LO_OP_F = 4, LO_OP_G = 5,
       LO_OP_U = 6, LO_OP_ATOM = 7 };

typedef struct lo_options {
    int32_t cost_fun[8];      /* p ~ & | X F G U */
    int32_t max_cost;
    int32_t key_mode;         /* LO_KEY_* */
    int32_t neg_type;         /* 1: negate every formula, 2: negate letters only */
    int32_t stop_at_found;    /* 1: stop after the chunk holding the first accepting candidate */
    int32_t threads;          /* 1: sequential (deterministic); 0: all OpenMP threads; k: k threads */
    int32_t limit_traces;     /* 1: apply the reference's 64-trace / 63-step limits */
    int32_t pad_;
    int64_t cache_rows;       /* language-cache capacity; overflow switches to on-the-fly checking */
    int64_t temp_rows;        /* chunk capacity (the reference's temp buffer); <= 0: unbounded */
    double time_limit_s;      /* > 0: give up (LO_TIMEOUT) once exceeded, checked between chunks */
} lo_options;

typedef struct lo_progress {
    int32_t cost;
    int32_t op;               /* 'A' for the letters, else one of ~ & | X F G U */
    uint64_t all_ltls;
    int64_t stored;
    int64_t to_check;
} lo_progress;

typedef struct lo_result {
    int32_t status;           /* LO_* */
    int32_t cost;             /* LTLcost as the reference reports it */
    uint64_t all_ltls;        /* candidates, counted as the reference counts them */
    char *formula;            /* reference string format; "not_found" when none */
    int32_t n;                /* traces = words per CS */
    int32_t alphabet_size;
    int64_t num_rows;         /* stored rows (letters included) */
    uint64_t *rows;           /* num_rows * n words */
    int8_t *row_op;
    int32_t *row_left;
    int32_t *row_right;
    int32_t num_costs;        /* entries in level_start - 1 */
    int32_t pad_;
    int64_t *level_start;     /* rows of cost c are [level_start[c], level_start[c + 1]) */
    uint64_t *level_candidates;
    int32_t num_progress;
    int32_t found_op;         /* operator of the returned formula's root */
    lo_progress *progress;
    double seconds;
    uint64_t evaluated;       /* candidates actually evaluated (letters included) */
    int32_t on_the_fly;       /* 1 once the cache overflowed */
    int32_t threads_used;
    void *internal_;
} lo_result;

void lo_default_options(lo_options *o);
int lo_learn(const lo_traces *t, const lo_options *o, lo_result *r);
void lo_result_free(lo_result *r);

/* Independent evaluator (positional LTLf semantics, string parsed as code/dc.py:136-183 does).
 * Writes 1/0 per trace for "holds at position 0".  Returns 0, or -1 on a malformed formula. */
int lo_eval(const char *formula, const lo_traces *t, uint8_t *holds);
/* Cost of a formula string under cost_fun; -1 on a malformed formula. */
int64_t lo_formula_cost(const char *formula, const int32_t *cost_fun);

/* Building blocks exposed for kernel-level parity tests. */
uint64_t lo_fp64(const uint64_t *cs, int32_t n);
void lo_ref_key(const uint64_t *cs, int32_t n, const uint8_t *len, int32_t len_sum, int32_t type,
                uint64_t *h, uint64_t *l);
void lo_apply_op(int32_t op, const uint64_t *a, const uint64_t *b, const uint64_t *mask, int32_t n,
                 uint64_t *out, uint64_t *out2);

#ifdef __cplusplus
}
#endif
#endif
