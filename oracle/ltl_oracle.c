/*
 * CPU oracle: a restatement of the characteristic-set (CS) enumeration of
 * MojtabaValizadeh/ltl-learning-on-gpus, code/ltli6463.cu.
 *
 * TEST INFRASTRUCTURE ONLY: the product never links or calls this file.  Only
 * tests/, the smoke check and the CPU-baseline leg of the benchmark use it, as
 * the checker.  Built by oracle/Makefile into oracle/_build/libltloracle.so.
 *
 * What is restated, and from where:
 *   - operator semantics on one uint64 per trace ......... ltli6463.cu:203-204, 295, 385, 468,
 *                                                          551-556, 638-645, 739-771
 *   - relaxed keys (types 1, 2, 3; exact pack) ........... ltli6463.cu:57-141
 *   - two-level intern == "the (hCS, lCS) pair is new" ... ltli6463.cu:164-171, 224-231
 *   - letters, early letter hit, limits .................. ltli6463.cu:1058-1136, 1078-1083
 *   - level / operator / split order, NegType ............ ltli6463.cu:1199-1445, 1212
 *   - chunking by the temp capacity, tid order ........... ltli6463.cu:1221-1238, 1254-1272, 1418-1436,
 *                                                          287-288, 727-728
 *   - compaction into the cache, on-the-fly overflow ..... ltli6463.cu:994-1035, 1202-1206, 1442-1443
 *   - acceptance test (bit 0 of each word) ............... ltli6463.cu:240-243
 *   - formula string and the 200-node limit .............. ltli6463.cu:877-991
 * The evaluator (lo_eval) is independent of all of that: it parses the string
 * the way code/dc.py:136-183 does and evaluates LTLf position by position.
 *
 * With threads == 1 candidates are handled strictly in the reference's tid
 * order, so every duplicate is resolved in favour of the earliest candidate
 * and rows are appended in the order the reference's stable compaction keeps.
 * With more threads the per-level sets of unique CSs are the same; which
 * representative formula wins a tie is a race, as in the reference.
 */
#define _GNU_SOURCE
#include "ltl_oracle.h"

#include <sched.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ------------------------------------------------------------ operators */

static inline uint64_t smear(uint64_t w)
{
    w |= w >> 1;
    w |= w >> 2;
    w |= w >> 4;
    w |= w >> 8;
    w |= w >> 16;
    w |= w >> 32;
    return w;
}

/* x U y with the doubling recurrence of ltli6463.cu:739-752. */
static inline uint64_t until_bits(uint64_t x, uint64_t y)
{
    y |= x & (y >> 1);
    x &= x >> 1;
    y |= x & (y >> 2);
    x &= x >> 2;
    y |= x & (y >> 4);
    x &= x >> 4;
    y |= x & (y >> 8);
    x &= x >> 8;
    y |= x & (y >> 16);
    x &= x >> 16;
    y |= x & (y >> 32);
    return y;
}

void lo_apply_op(int32_t op, const uint64_t *a, const uint64_t *b, const uint64_t *mask, int32_t n,
                 uint64_t *out, uint64_t *out2)
{
    for (int32_t i = 0; i < n; ++i) {
        switch (op) {
        case LO_OP_NEG: out[i] = ~a[i] & mask[i]; break;
        case LO_OP_AND: out[i] = a[i] & b[i]; break;
        case LO_OP_OR: out[i] = a[i] | b[i]; break;
        case LO_OP_X: out[i] = a[i] >> 1; break;
        case LO_OP_F: out[i] = smear(a[i]); break;
        case LO_OP_G: out[i] = a[i] & ~smear(~a[i] & mask[i]); break;
        case LO_OP_U:
            out[i] = until_bits(a[i], b[i]);
            if (out2) out2[i] = until_bits(b[i], a[i]);
            break;
        default: out[i] = a[i]; break;
        }
    }
}

/* ------------------------------------------------------------ keys */

/* MurmurHash3's 64-bit finaliser (Appleby, public domain). */
static inline uint64_t fmix64(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

/* Fingerprint of a whole CS: each word is keyed by its position (a Weyl
 * sequence), finalised, and the results summed; the sum is finalised again.
 * The GPU kernels compute the same function. */
uint64_t lo_fp64(const uint64_t *cs, int32_t n)
{
    uint64_t s = 0;
    for (int32_t i = 0; i < n; ++i)
        s += fmix64(cs[i] ^ ((uint64_t)(i + 1) * 0x9E3779B97F4A7C15ULL));
    return fmix64(s);
}

void lo_ref_key(const uint64_t *cs, int32_t n, const uint8_t *len, int32_t len_sum, int32_t type,
                uint64_t *h, uint64_t *l)
{
    uint64_t hc = 0, lc = 0;
    if (len_sum > 126) {
        if (type == 1) {
            const int stride = len_sum / 126;
            int j = 0;
            for (int i = 0; i < n; ++i) {
                for (int k = 0; k < len[i]; k += stride, ++j) {
                    if (j < 63) {
                        if (cs[i] & ((uint64_t)1 << k)) lc |= (uint64_t)1 << j;
                    } else if (j < 126) {
                        if (cs[i] & ((uint64_t)1 << k)) hc |= (uint64_t)1 << (j - 63);
                    } else
                        break;
                }
            }
        } else if (type == 2) {
            int j = 0;
            for (int i = 0; i < n; ++i) {
                uint64_t bit = 1;
                const int maxbits = (126 * len[i] + len_sum) / len_sum;
                for (int k = 0; k < maxbits; ++k, ++j, bit <<= 1) {
                    if (j < 63) {
                        if (cs[i] & bit) lc |= (uint64_t)1 << j;
                    } else if (j < 126) {
                        if (cs[i] & bit) hc |= (uint64_t)1 << (j - 63);
                    } else
                        break;
                }
            }
        } else if (type == 3) {
            for (int i = 0; i < n; ++i) {
                uint64_t x = cs[i];
                x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
                x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
                x = x ^ (x >> 31);
                if (i < n / 2)
                    hc ^= x;
                else
                    lc ^= x;
            }
        }
    } else {
        int j = 0;
        for (int i = 0; i < n; ++i) {
            uint64_t bit = 1;
            for (int k = 0; k < len[i]; ++k, ++j, bit <<= 1) {
                if (j < 63) {
                    if (cs[i] & bit) lc |= (uint64_t)1 << j;
                } else if (j < 126) {
                    if (cs[i] & bit) hc |= (uint64_t)1 << (j - 63);
                } else
                    break;
            }
        }
    }
    *h = hc;
    *l = lc;
}

/* ------------------------------------------------------------ state */

#define ROW_PENDING 0xFFFFFFFFu
#define ROW_OVERFLOW 0xFFFFFFFEu

typedef struct {
    int64_t ord;
    int32_t op, l, r;
} found_t;

typedef struct {
    int n, npos, nalpha, len_sum, key_mode;
    uint64_t *mask;
    uint8_t *len;
    uint64_t *rows;
    int64_t cap;
    int64_t reserved; /* rows handed out, may exceed cap during an overflow */
    int8_t *op;
    int32_t *left, *right;
    uint64_t *keys;
    uint64_t *slots;
    uint64_t smask;
    size_t rows_bytes, slots_bytes;
    int error;
    volatile int abort_flag;
    double deadline;
    uint64_t evaluated;
} st_t;

static void *big_alloc(size_t bytes)
{
    if (bytes == 0) bytes = 4096;
    void *p = mmap(NULL, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    return p == MAP_FAILED ? NULL : p;
}

static inline int accept_cs(const st_t *S, const uint64_t *cs)
{
    for (int i = 0; i < S->npos; ++i)
        if (!(cs[i] & 1)) return 0;
    for (int i = S->npos; i < S->n; ++i)
        if (cs[i] & 1) return 0;
    return 1;
}

static inline void make_key(const st_t *S, const uint64_t *cs, uint64_t *kh, uint64_t *kl, uint64_t *fp)
{
    if (S->key_mode == LO_KEY_EXACT) {
        *kh = *kl = 0;
        *fp = lo_fp64(cs, S->n);
    } else if (S->key_mode == LO_KEY_HASH64) {
        *kh = lo_fp64(cs, S->n);
        *kl = 0;
        *fp = *kh;
    } else {
        lo_ref_key(cs, S->n, S->len, S->len_sum, S->key_mode, kh, kl);
        *fp = fmix64(*kh ^ fmix64(*kl + 0x5ad0dedULL));
    }
}

static inline int same_key(const st_t *S, int64_t row, const uint64_t *cs, uint64_t kh, uint64_t kl)
{
    if (S->key_mode == LO_KEY_EXACT)
        return memcmp(S->rows + (size_t)row * S->n, cs, sizeof(uint64_t) * (size_t)S->n) == 0;
    return S->keys[2 * row] == kh && S->keys[2 * row + 1] == kl;
}

/* Insert a key.  Returns 1 when new (stored, or counted new while the cache
 * overflows), 0 for a duplicate, -1 when the table is full or a publication
 * never arrived.  preset >= 0 registers an already-written row (the letters). */
static int insert(st_t *S, const uint64_t *cs, uint64_t kh, uint64_t kl, uint64_t fp, int op, int32_t l,
                  int32_t r, int64_t preset)
{
    uint32_t tag = (uint32_t)(fp >> 32);
    uint64_t idx = fp & S->smask;
    for (uint64_t probe = 0; probe <= S->smask; ++probe, idx = (idx + 1) & S->smask) {
        uint64_t v = __atomic_load_n(&S->slots[idx], __ATOMIC_ACQUIRE);
        while (v == 0) {
            uint64_t want = ((uint64_t)tag << 32) | ROW_PENDING;
            if (__atomic_compare_exchange_n(&S->slots[idx], &v, want, 0, __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE)) {
                int64_t row = preset >= 0 ? preset : __atomic_fetch_add(&S->reserved, 1, __ATOMIC_RELAXED);
                uint32_t field;
                if (row >= S->cap) {
                    field = ROW_OVERFLOW;
                } else {
                    if (preset < 0) {
                        memcpy(S->rows + (size_t)row * S->n, cs, sizeof(uint64_t) * (size_t)S->n);
                        S->op[row] = (int8_t)op;
                        S->left[row] = l;
                        S->right[row] = r;
                    }
                    if (S->keys) {
                        S->keys[2 * row] = kh;
                        S->keys[2 * row + 1] = kl;
                    }
                    field = (uint32_t)(row + 1);
                }
                __atomic_store_n(&S->slots[idx], ((uint64_t)tag << 32) | field, __ATOMIC_RELEASE);
                return 1;
            }
        }
        if ((uint32_t)(v >> 32) != tag) continue;
        uint32_t field = (uint32_t)v;
        for (long spins = 0; field == ROW_PENDING; ++spins) {
            if (spins > (1L << 30)) return -1;
            sched_yield();
            v = __atomic_load_n(&S->slots[idx], __ATOMIC_ACQUIRE);
            field = (uint32_t)v;
        }
        if (field == ROW_OVERFLOW) return 0;
        if (same_key(S, (int64_t)field - 1, cs, kh, kl)) return 0;
    }
    return -1;
}

/* One candidate.  Returns nothing; records the lowest accepting ordinal. */
static inline void candidate(st_t *S, const uint64_t *cs, int op, int32_t l, int32_t r, int64_t ord, int on_the_fly,
                             found_t *best)
{
    const int acc = accept_cs(S, cs);
    if (on_the_fly) {
        if (acc && ord < best->ord) {
            best->ord = ord;
            best->op = op;
            best->l = l;
            best->r = r;
        }
        return;
    }
    uint64_t kh, kl, fp;
    make_key(S, cs, &kh, &kl, &fp);
    int res = insert(S, cs, kh, kl, fp, op, l, r, -1);
    if (res < 0) {
        S->error = 1;
        return;
    }
    if (res == 1 && acc && ord < best->ord) {
        best->ord = ord;
        best->op = op;
        best->l = l;
        best->r = r;
    }
}

static int nthreads_of(int requested)
{
#ifdef _OPENMP
    if (requested <= 0) return omp_get_max_threads();
    return requested;
#else
    (void)requested;
    return 1;
#endif
}

/* One chunk of a unary operator over source rows [x, y] or a binary operator over
 * left rows [i1, i2] x right rows [x, y].  tid order matches the reference kernels. */
static void run_chunk(st_t *S, int op, int binary, int64_t i1, int64_t i2, int64_t x, int64_t y, int on_the_fly,
                      int threads, found_t *out)
{
    const int64_t R = y - x + 1;
    const int64_t L = binary ? (i2 - i1 + 1) : 1;
    const int64_t N = binary ? L * R : R;
    const int n = S->n;
    found_t best = {INT64_MAX, 0, 0, 0};
#pragma omp parallel num_threads(threads)
    {
        uint64_t *cs = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(2 * n + 2));
        uint64_t *cs2 = cs + n + 1;
        found_t mine = {INT64_MAX, 0, 0, 0};
        uint64_t done = 0;
#pragma omp for schedule(dynamic, 64)
        for (int64_t tid = 0; tid < N; ++tid) {
            if (S->abort_flag) continue;
            if (binary) {
                const int64_t ldx = i1 + tid / R, rdx = x + tid % R;
                const uint64_t *a = S->rows + (size_t)ldx * n, *b = S->rows + (size_t)rdx * n;
                lo_apply_op(op, a, b, S->mask, n, cs, cs2);
                candidate(S, cs, op, (int32_t)ldx, (int32_t)rdx, op == LO_OP_U ? 2 * tid : tid, on_the_fly, &mine);
                if (op == LO_OP_U)
                    candidate(S, cs2, op, (int32_t)rdx, (int32_t)ldx, 2 * tid + 1, on_the_fly, &mine);
            } else {
                const int64_t src = x + tid;
                lo_apply_op(op, S->rows + (size_t)src * n, NULL, S->mask, n, cs, NULL);
                candidate(S, cs, op, (int32_t)src, 0, tid, on_the_fly, &mine);
            }
            done += (op == LO_OP_U) ? 2 : 1;
            if (S->deadline > 0 && (done & 1023) == 0 && now_s() > S->deadline) S->abort_flag = 1;
        }
#pragma omp critical
        {
            if (mine.ord < best.ord) best = mine;
            S->evaluated += done;
        }
        free(cs);
    }
    *out = best;
}

/* ------------------------------------------------------------ strings */

typedef struct {
    char *s;
    size_t len, cap;
} sbuf;

static void sb_put(sbuf *b, const char *t)
{
    size_t k = strlen(t);
    if (b->len + k + 1 > b->cap) {
        b->cap = (b->len + k + 1) * 2;
        b->s = (char *)realloc(b->s, b->cap);
    }
    memcpy(b->s + b->len, t, k + 1);
    b->len += k;
}

static void to_string(const st_t *S, const char *alpha, int op, int32_t l, int32_t r, sbuf *b);

static void row_string(const st_t *S, const char *alpha, int64_t row, sbuf *b)
{
    if (row < S->nalpha) {
        char c[2] = {alpha[row], 0};
        sb_put(b, c);
        return;
    }
    to_string(S, alpha, S->op[row], S->left[row], S->right[row], b);
}

static void to_string(const st_t *S, const char *alpha, int op, int32_t l, int32_t r, sbuf *b)
{
    static const char *pre[] = {"~(", "(", "(", "X(", "F(", "G(", "("};
    static const char *mid[] = {"", ")&(", ")|(", "", "", "", ")U("};
    sb_put(b, pre[op]);
    row_string(S, alpha, l, b);
    if (op == LO_OP_AND || op == LO_OP_OR || op == LO_OP_U) {
        sb_put(b, mid[op]);
        row_string(S, alpha, r, b);
    }
    sb_put(b, ")");
}

/* Non-letter nodes below the root in the tree expansion, stopping at limit. */
static int64_t count_nodes(const st_t *S, int64_t row, int64_t limit)
{
    if (row < S->nalpha || limit <= 0) return 0;
    int64_t c = 1;
    c += count_nodes(S, S->left[row], limit - c);
    int op = S->op[row];
    if (op == LO_OP_AND || op == LO_OP_OR || op == LO_OP_U) c += count_nodes(S, S->right[row], limit - c);
    return c;
}

/* ------------------------------------------------------------ driver */

typedef struct {
    lo_progress *v;
    int n, cap;
} plog;

static void plog_add(plog *p, int cost, int op, uint64_t all, int64_t stored, int64_t tbc)
{
    if (p->n == p->cap) {
        p->cap = p->cap ? 2 * p->cap : 64;
        p->v = (lo_progress *)realloc(p->v, sizeof(lo_progress) * (size_t)p->cap);
    }
    lo_progress e = {cost, op, all, stored, tbc};
    p->v[p->n++] = e;
}

void lo_default_options(lo_options *o)
{
    memset(o, 0, sizeof(*o));
    for (int i = 0; i < 8; ++i) o->cost_fun[i] = 1;
    o->max_cost = 500;
    o->key_mode = LO_KEY_EXACT;
    o->neg_type = 1;
    o->stop_at_found = 1;
    o->threads = 1;
    o->limit_traces = 0;
    o->cache_rows = 1 << 20;
    o->temp_rows = 0;
}

static const char OPCH[7] = {'~', '&', '|', 'X', 'F', 'G', 'U'};

int lo_learn(const lo_traces *t, const lo_options *o, lo_result *res)
{
    memset(res, 0, sizeof(*res));
    const double t0 = now_s();
    const int npos = t->num_pos, nneg = t->num_neg, n = npos + nneg;
    const int nalpha = (int)strlen(t->alphabet);
    const int c1 = o->cost_fun[0], c2 = o->cost_fun[1], c3 = o->cost_fun[2], c4 = o->cost_fun[3];
    const int c5 = o->cost_fun[4], c6 = o->cost_fun[5], c7 = o->cost_fun[6], c8 = o->cost_fun[7];
    const int max_cost = o->max_cost;
    res->n = n;
    res->alphabet_size = nalpha;
    res->cost = c1;
    for (int i = 0; i < 8; ++i)
        if (o->cost_fun[i] <= 0) {
            res->status = LO_BAD_ARGS;
            return res->status;
        }

    st_t *S = (st_t *)calloc(1, sizeof(st_t));
    res->internal_ = S;
    S->n = n;
    S->npos = npos;
    S->nalpha = nalpha;
    S->key_mode = o->key_mode;
    S->mask = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    S->len = (uint8_t *)calloc((size_t)n + 1, 1);
    int max_len = 0;
    for (int i = 0; i < n; ++i) {
        int ln = t->offsets[i + 1] - t->offsets[i];
        if (ln > max_len) max_len = ln;
        S->len_sum += ln;
        S->len[i] = (uint8_t)(ln > 255 ? 255 : ln);
        S->mask[i] = ln >= 64 ? ~0ULL : (((uint64_t)1 << ln) - 1);
    }
    if ((o->limit_traces && n > 64) || max_len > 63) {
        res->status = LO_INPUT_LIMITS;
        res->formula = strdup("see_the_error");
        return res->status;
    }

    const int64_t cap = o->cache_rows > nalpha ? o->cache_rows : nalpha + 1;
    S->cap = cap;
    S->rows_bytes = sizeof(uint64_t) * (size_t)cap * (size_t)(n > 0 ? n : 1);
    S->rows = (uint64_t *)big_alloc(S->rows_bytes);
    S->op = (int8_t *)calloc((size_t)cap, 1);
    S->left = (int32_t *)calloc((size_t)cap, sizeof(int32_t));
    S->right = (int32_t *)calloc((size_t)cap, sizeof(int32_t));
    if (o->key_mode != LO_KEY_EXACT) S->keys = (uint64_t *)calloc((size_t)cap * 2, sizeof(uint64_t));
    uint64_t slots = 1024;
    while (slots < (uint64_t)cap * 2) slots <<= 1;
    S->slots_bytes = slots * sizeof(uint64_t);
    S->slots = (uint64_t *)big_alloc(S->slots_bytes);
    S->smask = slots - 1;
    if (!S->rows || !S->slots || !S->op || !S->left || !S->right) {
        res->status = LO_NO_MEMORY;
        return res->status;
    }
    S->deadline = o->time_limit_s > 0 ? t0 + o->time_limit_s : 0;
    const int threads = nthreads_of(o->threads);
    res->threads_used = threads;

    plog P = {0};
    uint64_t all = 0;
    int64_t last = 0;
    const int ncost = (max_cost > c1 ? max_cost : c1) + 2;
    int64_t *sp = (int64_t *)calloc((size_t)ncost * 7 + 7, sizeof(int64_t));
    uint64_t *lc = (uint64_t *)calloc((size_t)ncost + 1, sizeof(uint64_t));
    int found = 0, first_found_cost = -1;
    found_t fnd = {INT64_MAX, 0, 0, 0};
    int found_letter = -1;
    int cost = c1;
    int top = c1; /* highest c whose start row sp[c * 7] is known */

    /* letters (ltli6463.cu:1096-1136) */
    plog_add(&P, c1, 'A', all, 0, nalpha);
    uint64_t *cs = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    for (int j = 0; j < nalpha; ++j) {
        const uint32_t bit = 1u << (t->alphabet[j] - 'a');
        for (int i = 0; i < n; ++i) {
            uint64_t w = 0;
            for (int k = t->offsets[i]; k < t->offsets[i + 1]; ++k)
                if (t->steps[k] & bit) w |= (uint64_t)1 << (k - t->offsets[i]);
            cs[i] = w;
        }
        memcpy(S->rows + (size_t)j * n, cs, sizeof(uint64_t) * (size_t)n);
        S->op[j] = LO_OP_ATOM;
        S->left[j] = S->right[j] = 0;
        all++;
        last++;
        if (accept_cs(S, cs) && !found) {
            found = 1;
            found_letter = j;
            first_found_cost = c1;
            if (o->stop_at_found) break;
        }
    }
    S->reserved = last;
    lc[c1 < ncost ? c1 : 0] = (uint64_t)last;
    int status = LO_NOT_FOUND;
    if (found && o->stop_at_found) {
        status = LO_FOUND;
        goto done;
    }
    for (int j = 0; j < nalpha; ++j) {
        uint64_t kh, kl, fp;
        make_key(S, S->rows + (size_t)j * n, &kh, &kl, &fp);
        if (insert(S, S->rows + (size_t)j * n, kh, kl, fp, LO_OP_ATOM, 0, 0, j) < 0) S->error = 1;
    }
    sp[c1 * 7 + 6] = last;
    sp[(c1 + 1) * 7] = last;
    top = c1 + 1;

    {
        int on_the_fly = 0, last_round = 0, shortage = -1;
        const int64_t T = o->temp_rows > 0 ? o->temp_rows : INT64_MAX / 4;
#define STORE_AFTER_CHUNK()                                                                                 \
    do {                                                                                                    \
        if (!on_the_fly) {                                                                                  \
            int64_t r_ = S->reserved;                                                                       \
            if (r_ > S->cap) {                                                                              \
                on_the_fly = 1;                                                                             \
                res->on_the_fly = 1;                                                                        \
                r_ = S->cap;                                                                                \
                S->reserved = r_;                                                                           \
            }                                                                                               \
            last = r_;                                                                                      \
        }                                                                                                   \
    } while (0)
#define CHECK_CHUNK(NUM)                                                                                    \
    do {                                                                                                    \
        all += (uint64_t)(NUM);                                                                             \
        lc[cost] += (uint64_t)(NUM);                                                                        \
        if (S->error) {                                                                                     \
            status = LO_NO_MEMORY;                                                                          \
            goto done;                                                                                      \
        }                                                                                                   \
        if (S->abort_flag) {                                                                                \
            status = LO_TIMEOUT;                                                                            \
            goto done;                                                                                      \
        }                                                                                                   \
        if (f_.ord != INT64_MAX && !found) {                                                                \
            found = 1;                                                                                      \
            fnd = f_;                                                                                       \
            first_found_cost = cost;                                                                        \
            if (o->stop_at_found) {                                                                         \
                status = LO_FOUND;                                                                          \
                goto done;                                                                                  \
            }                                                                                               \
        }                                                                                                   \
        STORE_AFTER_CHUNK();                                                                                \
        if (S->deadline > 0 && now_s() > S->deadline) {                                                     \
            status = LO_TIMEOUT;                                                                            \
            goto done;                                                                                      \
        }                                                                                                   \
    } while (0)

        for (cost = c1 + 1; cost <= max_cost; ++cost) {
            if (on_the_fly) {
                const int dif = cost - shortage;
                if (dif == c2 || dif == c1 + c3 || dif == c1 + c4 || dif == c5 || dif == c6 || dif == c7 ||
                    dif == c1 + c8)
                    last_round = 1;
            }
            for (int opk = 0; opk < 7; ++opk) {
                const int copk = o->cost_fun[opk + 1];
                const int binary = (opk == LO_OP_AND || opk == LO_OP_OR || opk == LO_OP_U);
                if (!binary) {
                    int run = cost - copk >= c1;
                    if (opk == LO_OP_NEG)
                        run = (o->neg_type == 1 && cost - c2 >= c1) || (o->neg_type == 2 && cost - c2 == c1);
                    if (run) {
                        const int64_t i1 = sp[(cost - copk) * 7], i2 = sp[(cost - copk + 1) * 7] - 1;
                        if (i2 - i1 + 1 > 0) {
                            int64_t x = i1, y;
                            do {
                                y = x + ((T - 1) < (i2 - x) ? (T - 1) : (i2 - x));
                                const int64_t N = y - x + 1;
                                plog_add(&P, cost, OPCH[opk], all, last, N);
                                found_t f_;
                                run_chunk(S, opk, 0, 0, 0, x, y, on_the_fly, threads, &f_);
                                CHECK_CHUNK(N);
                                x = y + 1;
                            } while (y < i2);
                        }
                    }
                } else {
                    for (int i = c1; 2 * i <= cost - copk; ++i) {
                        const int64_t i1 = sp[i * 7], i2 = sp[(i + 1) * 7] - 1;
                        const int64_t i3 = sp[(cost - i - copk) * 7], i4 = sp[(cost - i - copk + 1) * 7] - 1;
                        const int64_t L = i2 - i1 + 1;
                        if (L * (i4 - i3 + 1) > 0) {
                            int64_t x = i3, y;
                            do {
                                const int64_t step = (opk == LO_OP_U ? T / (2 * L) : T / L) - 1;
                                if (step < 0) {
                                    status = LO_CHUNK_TOO_SMALL;
                                    goto done;
                                }
                                y = x + (step < (i4 - x) ? step : (i4 - x));
                                const int64_t N = (y - x + 1) * L;
                                const int64_t shown = opk == LO_OP_U ? 2 * N : N;
                                plog_add(&P, cost, OPCH[opk], all, last, shown);
                                found_t f_;
                                run_chunk(S, opk, 1, i1, i2, x, y, on_the_fly, threads, &f_);
                                CHECK_CHUNK(shown);
                                x = y + 1;
                            } while (y < i4);
                        }
                    }
                }
                if (opk < 6)
                    sp[cost * 7 + opk + 1] = last;
                else
                    sp[(cost + 1) * 7] = last;
            }
            top = cost + 1;
            if (last_round) break;
            if (on_the_fly && shortage == -1) shortage = cost;
        }
        if (cost == max_cost + 1) cost--;
        status = found ? LO_FOUND : LO_NOT_FOUND;
    }

done:
    if (found && status == LO_NOT_FOUND) status = LO_FOUND;
    res->status = status;
    res->cost = found ? first_found_cost : cost;
    res->all_ltls = all;
    if (found) {
        sbuf b = {0};
        if (found_letter >= 0) {
            char c[2] = {t->alphabet[found_letter], 0};
            sb_put(&b, c);
            res->found_op = LO_OP_ATOM;
        } else {
            int64_t nodes = count_nodes(S, fnd.l, 200);
            if (fnd.op == LO_OP_AND || fnd.op == LO_OP_OR || fnd.op == LO_OP_U)
                nodes += count_nodes(S, fnd.r, 200 - nodes);
            if (nodes >= 200)
                sb_put(&b, "Size of the output is too big");
            else
                to_string(S, t->alphabet, fnd.op, fnd.l, fnd.r, &b);
            res->found_op = fnd.op;
        }
        res->formula = b.s;
    } else {
        res->formula = strdup(status == LO_TIMEOUT ? "timeout" : "not_found");
    }
    res->num_rows = S->reserved < S->cap ? S->reserved : S->cap;
    res->rows = S->rows;
    res->row_op = S->op;
    res->row_left = S->left;
    res->row_right = S->right;
    res->num_costs = ncost;
    res->level_start = (int64_t *)calloc((size_t)ncost + 1, sizeof(int64_t));
    for (int c = 0; c <= ncost; ++c)
        res->level_start[c] = c <= top ? sp[c * 7] : res->num_rows;
    res->level_candidates = lc;
    res->num_progress = P.n;
    res->progress = P.v;
    res->seconds = now_s() - t0;
    res->evaluated = S->evaluated + (uint64_t)nalpha;
    free(sp);
    free(cs);
    return res->status;
}

void lo_result_free(lo_result *r)
{
    st_t *S = (st_t *)r->internal_;
    if (S) {
        if (S->rows) munmap(S->rows, S->rows_bytes);
        if (S->slots) munmap(S->slots, S->slots_bytes);
        free(S->op);
        free(S->left);
        free(S->right);
        free(S->keys);
        free(S->mask);
        free(S->len);
        free(S);
    }
    free(r->formula);
    free(r->level_start);
    free(r->level_candidates);
    free(r->progress);
    memset(r, 0, sizeof(*r));
}

/* ------------------------------------------------------------ evaluator */

typedef struct {
    char op;
    int a, b;
    int letter;
} enode;

typedef struct {
    enode *v;
    int n, cap;
    int err;
} etree;

static int eadd(etree *T, enode e)
{
    if (T->n == T->cap) {
        T->cap = T->cap ? 2 * T->cap : 64;
        T->v = (enode *)realloc(T->v, sizeof(enode) * (size_t)T->cap);
    }
    T->v[T->n] = e;
    return T->n++;
}

/* Parse f[lo, hi) the way code/dc.py:136-176 slices it. */
static int eparse(const char *f, int lo, int hi, etree *T, int depth)
{
    if (T->err || lo >= hi || depth > 100000) {
        T->err = 1;
        return -1;
    }
    int i = lo;
    if (f[lo] == '(') {
        int p = 1;
        i = lo + 1;
        while (p != 0) {
            if (i >= hi) {
                T->err = 1;
                return -1;
            }
            if (f[i] == '(')
                p++;
            else if (f[i] == ')')
                p--;
            i++;
        }
        if (i >= hi) {
            T->err = 1;
            return -1;
        }
    }
    const char c = f[i];
    enode e = {c, -1, -1, -1};
    if (c == '~' || c == 'X' || c == 'F' || c == 'G') {
        e.a = eparse(f, lo + 2, hi - 1, T, depth + 1);
    } else if (c == '&' || c == '|' || c == 'U') {
        e.a = eparse(f, lo + 1, i - 1, T, depth + 1);
        e.b = eparse(f, i + 2, hi - 1, T, depth + 1);
    } else if (c >= 'a' && c <= 'z') {
        e.op = 'p';
        e.letter = c - 'a';
    } else {
        T->err = 1;
        return -1;
    }
    return eadd(T, e);
}

/* sat[node * (len + 1) + k] for positions k < len (index len is the boundary). */
static void eeval(const etree *T, int node, const uint32_t *steps, int len, uint8_t *sat)
{
    const enode *e = &T->v[node];
    uint8_t *o = sat + (size_t)node * (len + 1);
    const uint8_t *a = e->a >= 0 ? sat + (size_t)e->a * (len + 1) : NULL;
    const uint8_t *b = e->b >= 0 ? sat + (size_t)e->b * (len + 1) : NULL;
    switch (e->op) {
    case 'p':
        for (int k = 0; k < len; ++k) o[k] = (steps[k] >> e->letter) & 1;
        break;
    case '~':
        for (int k = 0; k < len; ++k) o[k] = !a[k];
        break;
    case '&':
        for (int k = 0; k < len; ++k) o[k] = a[k] && b[k];
        break;
    case '|':
        for (int k = 0; k < len; ++k) o[k] = a[k] || b[k];
        break;
    case 'X':
        for (int k = 0; k < len; ++k) o[k] = (k + 1 < len) ? a[k + 1] : 0;
        break;
    case 'F': {
        uint8_t acc = 0;
        for (int k = len - 1; k >= 0; --k) o[k] = acc = (uint8_t)(a[k] || acc);
        break;
    }
    case 'G': {
        uint8_t acc = 1;
        for (int k = len - 1; k >= 0; --k) o[k] = acc = (uint8_t)(a[k] && acc);
        break;
    }
    case 'U': {
        uint8_t acc = 0;
        for (int k = len - 1; k >= 0; --k) o[k] = acc = (uint8_t)(b[k] || (a[k] && acc));
        break;
    }
    }
}

int lo_eval(const char *formula, const lo_traces *t, uint8_t *holds)
{
    etree T = {0};
    const int len = (int)strlen(formula);
    const int root = eparse(formula, 0, len, &T, 0);
    if (T.err || root < 0) {
        free(T.v);
        return -1;
    }
    const int n = t->num_pos + t->num_neg;
    for (int i = 0; i < n; ++i) {
        const int ln = t->offsets[i + 1] - t->offsets[i];
        uint8_t *sat = (uint8_t *)calloc((size_t)T.n * (ln + 1), 1);
        /* children precede parents in T (post-order) */
        for (int v = 0; v < T.n; ++v) eeval(&T, v, t->steps + t->offsets[i], ln, sat);
        holds[i] = ln > 0 ? sat[(size_t)root * (ln + 1)] : 0;
        free(sat);
    }
    free(T.v);
    return 0;
}

int64_t lo_formula_cost(const char *formula, const int32_t *cf)
{
    etree T = {0};
    const int len = (int)strlen(formula);
    const int root = eparse(formula, 0, len, &T, 0);
    if (T.err || root < 0) {
        free(T.v);
        return -1;
    }
    int64_t c = 0;
    for (int v = 0; v < T.n; ++v) {
        switch (T.v[v].op) {
        case 'p': c += cf[0]; break;
        case '~': c += cf[1]; break;
        case '&': c += cf[2]; break;
        case '|': c += cf[3]; break;
        case 'X': c += cf[4]; break;
        case 'F': c += cf[5]; break;
        case 'G': c += cf[6]; break;
        case 'U': c += cf[7]; break;
        }
    }
    free(T.v);
    return c;
}
