// A learn that allocates nothing, for callers that cannot allocate device memory: code
// running inside a host application whose GPU memory is owned by another allocator (a
// framework's caching allocator, a pool handed out by a runtime), or under a policy that
// forbids cudaMalloc after start-up.  Every device buffer of the enumeration lives in one
// file-scope static array (NOALLOC_SCRATCH_BYTES, loaded with the library and held by every
// GPU that loads it until the process exits); host-side work uses fixed-size stack arrays.
//
// Limits: at most NOALLOC_MAX_TRACES traces of at most 63 steps; the language cache is what
// is left of the scratch after the fixed parts; a level that would overflow it ends the call
// with LTLG_NO_MEMORY (the reference's on-the-fly regime is not run here).
//
// The scratch is shared by every call: each call clears what must start at zero (hash set,
// control record, level starts) and overwrites the rest.  Calls whose GPU work overlaps (two
// host threads, or two devices' calls if the pointer bookkeeping were shared) race on it;
// the caller serialises them.  The first call on a device looks up the scratch address on
// that device (cudaGetSymbolAddress, with that device current); make that first call before
// any stream capture.
#include <climits>
#include <cstdio>
#include <cstring>

#include "ltl_kernels.cuh"
#include "ltlgpu.h"
#include "traces.hpp"

using namespace ltlg;

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 64ull << 20;  // 64 MiB
constexpr int NOALLOC_MAX_TRACES = 64;
constexpr int NOALLOC_SLOTS_LOG2 = 18;                 // 2^18 eight-byte slots = 2 MiB
constexpr int NOALLOC_MAX_DEVICES = 64;
constexpr int WALK_CAP = 1024;
constexpr int MAX_COSTS = 512;                         // max_cost stays below this (fixed level arrays)
constexpr int NOALLOC_MIN_FORMULA = 16;                // holds "see_the_error", "not_found" and a letter

__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

void *g_scratch_on[NOALLOC_MAX_DEVICES] = {};

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// Rows of cost k are [ls[k], ls[k + 1]); the candidates the reference counts in level c up to
// and including the block at position fpos of its block order (ltli6463.cu:1209-1440), which
// lists only blocks whose operand levels are non-empty.
unsigned long long count_to_found(int c, const int *cf, int neg_type, const long long *ls, int fpos) {
    const int c1 = cf[0];
    unsigned long long all = 0;
    int pos = 0;
    auto size = [&](int k) { return (k >= c1 && k < c) ? ls[k + 1] - ls[k] : 0ll; };
    auto take = [&](long long n) {
        if (n <= 0 || pos > fpos) return;
        all += (unsigned long long)n;
        ++pos;
    };
    auto binary = [&](int cop, int mult) {
        for (int i = c1; 2 * i <= c - cop; ++i)
            if (size(i) > 0 && size(c - i - cop) > 0) take(mult * size(i) * size(c - i - cop));
    };
    if ((neg_type == 1 && c - cf[1] >= c1) || (neg_type == 2 && c - cf[1] == c1)) take(size(c - cf[1]));
    binary(cf[2], 1);
    binary(cf[3], 1);
    if (c - cf[4] >= c1) take(size(c - cf[4]));
    if (c - cf[5] >= c1) take(size(c - cf[5]));
    if (c - cf[6] >= c1) take(size(c - cf[6]));
    binary(cf[7], 2);
    return all;
}

struct Writer {
    char *buf;
    int cap, len;
    bool over;
    void put(const char *s) {
        for (; *s; ++s) {
            if (len + 1 >= cap) {
                over = true;
                return;
            }
            buf[len++] = *s;
        }
        buf[len] = 0;
    }
};

// Formula of a node from the walk entries (row, parents), in the reference's format.
void write_node(const u64 *ent, int count, u64 parent, const char *alpha, int nalpha, Writer &w, int depth) {
    if (depth > 4096) {
        w.over = true;
        return;
    }
    const int op = parent_op(parent);
    auto child = [&](u64 r) {
        if (r < (u64)nalpha) {
            const char s[2] = {alpha[r], 0};
            w.put(s);
            return;
        }
        for (int q = 1; q < count; ++q)
            if (ent[2 * q] == r) {
                write_node(ent, count, ent[2 * q + 1], alpha, nalpha, w, depth + 1);
                return;
            }
        w.over = true;
    };
    switch (op) {
    case OP_NEG: w.put("~("); child(parent_left(parent)); w.put(")"); break;
    case OP_X: w.put("X("); child(parent_left(parent)); w.put(")"); break;
    case OP_F: w.put("F("); child(parent_left(parent)); w.put(")"); break;
    case OP_G: w.put("G("); child(parent_left(parent)); w.put(")"); break;
    default:
        w.put("(");
        child(parent_left(parent));
        w.put(op == OP_AND ? ")&(" : op == OP_OR ? ")|(" : ")U(");
        child(parent_right(parent));
        w.put(")");
        break;
    }
}

}  // namespace

extern "C" LTLG_API int ltlg_learn_noalloc(const ltlg_traces *t, const ltlg_options *opt, char *formula,
                                           int32_t formula_cap, int32_t *cost_out, uint64_t *all_ltls_out) {
    if (!t || !opt || !formula || formula_cap < NOALLOC_MIN_FORMULA || !ltlg::traces_well_formed(t))
        return LTLG_BAD_ARGS;
    formula[0] = 0;
    const int *cf = opt->cost_fun;
    for (int i = 0; i < 8; ++i)
        if (cf[i] <= 0 || cf[i] > SHRT_MAX) return LTLG_BAD_ARGS;
    const int npos = t->num_pos, nneg = t->num_neg, n = npos + nneg;
    const int nalpha = t->alphabet ? (int)strlen(t->alphabet) : 0;
    if (npos < 0 || nneg < 0 || nalpha > 26 || opt->key_mode < 0 || opt->key_mode > 2 || opt->max_cost < 1 ||
        opt->max_cost >= MAX_COSTS)
        return LTLG_BAD_ARGS;
    if (opt->key_mode == LTLG_KEY_REF) return LTLG_BAD_ARGS;  // relaxed reference keys: use ltlg_learn
    int max_len = 0;
    for (int i = 0; i < n; ++i) max_len = t->offsets[i + 1] - t->offsets[i] > max_len ? t->offsets[i + 1] - t->offsets[i] : max_len;
    if (n > NOALLOC_MAX_TRACES || max_len > 63) {
        snprintf(formula, formula_cap, "see_the_error");
        return LTLG_INPUT_LIMITS;
    }
    const int c1 = cf[0];
    if (cost_out) *cost_out = c1;
    if (all_ltls_out) *all_ltls_out = 0;

    // Letters on the host (stack arrays): rows 0 .. nalpha-1; an early letter hit ends here.
    const int pitch = n <= 4 ? 4 : (n + 3) & ~3;
    u64 letters[26 * NOALLOC_MAX_TRACES];
    memset(letters, 0, sizeof(letters));
    unsigned long long all = 0;
    int letter_hit = -1;
    for (int j = 0; j < nalpha; ++j) {
        const uint32_t bit = 1u << (t->alphabet[j] - 'a');
        bool acc = true;
        for (int i = 0; i < n; ++i) {
            u64 w = 0;
            for (int k = t->offsets[i]; k < t->offsets[i + 1]; ++k)
                if (t->steps[k] & bit) w |= 1ull << (k - t->offsets[i]);
            letters[j * pitch + i] = w;
            if (i < npos ? !(w & 1) : (w & 1)) acc = false;
        }
        ++all;
        if (acc && letter_hit < 0) {
            letter_hit = j;
            if (opt->stop_at_found) {
                snprintf(formula, formula_cap, "%c", t->alphabet[j]);
                if (all_ltls_out) *all_ltls_out = all;
                return LTLG_FOUND;
            }
        }
    }
    if (n == 0 || nalpha == 0) {
        // nothing to enumerate: every level is empty (with no traces every letter separates
        // them vacuously, and the first one is the answer at cost c1)
        if (all_ltls_out) *all_ltls_out = all;
        if (letter_hit >= 0) {
            snprintf(formula, formula_cap, "%c", t->alphabet[letter_hit]);
            return LTLG_FOUND;
        }
        snprintf(formula, formula_cap, "not_found");
        if (cost_out) *cost_out = opt->max_cost > c1 ? opt->max_cost : c1;
        return LTLG_NOT_FOUND;
    }

    // The scratch address on this device (looked up once per device, with it current).
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return LTLG_NO_DEVICE;
    if (!g_scratch_on[dev]) {
        void *p = nullptr;
        err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess || !p) return LTLG_CUDA_ERROR;
        g_scratch_on[dev] = p;
    }
    unsigned char *base = (unsigned char *)g_scratch_on[dev];

    // Carve the scratch: fixed parts first, the language cache takes the rest.
    const int max_cost = opt->max_cost;
    const long long cap_entries = 4 + 3 * ((long long)max_cost / 2 + 2);
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        unsigned char *p = base + off;
        off += up256(bytes);
        return p;
    };
    InstCtl *ctl = (InstCtl *)carve(sizeof(InstCtl));
    InstArgs *dargs = (InstArgs *)carve(sizeof(InstArgs));
    Launch *dlaunch = (Launch *)carve(sizeof(Launch));
    long long *ls = (long long *)carve((MAX_COSTS + 3) * sizeof(long long));
    int *ne = (int *)carve((MAX_COSTS + 3) * sizeof(int));
    u64 *lcands = (u64 *)carve((MAX_COSTS + 3) * sizeof(u64));
    Entry *entries = (Entry *)carve((size_t)(2 * cap_entries) * sizeof(Entry));
    u64 *fpar = (u64 *)carve((size_t)cap_entries * 8);
    u64 *wmeta = (u64 *)carve((size_t)pitch * 8);
    u32 *kmeta = (u32 *)carve((size_t)pitch * 4);
    u64 *walk = (u64 *)carve((2 + 2 * WALK_CAP) * 8);
    const u64 nslots = 1ull << NOALLOC_SLOTS_LOG2;
    u64 *slots = (u64 *)carve(nslots * 8);
    const bool keyed = opt->key_mode != LTLG_KEY_EXACT;
    const size_t per_row = (size_t)pitch * 8 + 8 + (keyed ? 16 : 0);
    if (off >= NOALLOC_SCRATCH_BYTES) return LTLG_NO_MEMORY;
    long long cap = (long long)((NOALLOC_SCRATCH_BYTES - off - 3 * 256) / per_row);
    if (cap > (long long)(nslots / 2)) cap = (long long)(nslots / 2);
    if (cap < nalpha + 1) return LTLG_NO_MEMORY;
    u64 *parents = (u64 *)carve((size_t)cap * 8);
    u64 *keys = keyed ? (u64 *)carve((size_t)cap * 16) : nullptr;
    u64 *cache = (u64 *)carve((size_t)cap * pitch * 8);
    if (off > NOALLOC_SCRATCH_BYTES) return LTLG_NO_MEMORY;

    // Level-kernel geometry: 8-row tiles of rows of at most 64 words, eight slots.
    const int tile = 8, stages = 8;
    const long long tile_bytes = (long long)tile * pitch * 8;
    const int hk = opt->key_mode == LTLG_KEY_HASH64 ? 1 : 0;
    int num_sms = 0;
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    const int per_sm = level_kernel_ctas_per_sm(hk, level_kernel_smem(stages, tile_bytes));
    const int grid = (num_sms > 0 ? num_sms : 1) * (per_sm > 0 ? per_sm : 1);

    // Inputs and zeroed state (default stream, synchronous copies from stack arrays).
    u64 wm[NOALLOC_MAX_TRACES];
    memset(wm, 0, sizeof(wm));
    for (int i = 0; i < n; ++i) {
        const int ln = t->offsets[i + 1] - t->offsets[i];
        wm[i] = (ln >= 63 ? 0x7FFFFFFFFFFFFFFFull : ((1ull << ln) - 1)) | (i < npos ? (1ull << 63) : 0ull);
    }
    InstCtl hc;
    memset(&hc, 0, sizeof(hc));
    hc.row_count = (u64)nalpha;
    hc.found_key = NO_FIND;
    hc.plan.cost = c1;
    if ((err = cudaMemcpy(cache, letters, (size_t)nalpha * pitch * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (err = cudaMemcpy(wmeta, wm, (size_t)pitch * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (err = cudaMemset(kmeta, 0, (size_t)pitch * 4)) != cudaSuccess ||
        (err = cudaMemset(slots, 0, nslots * 8)) != cudaSuccess ||
        (err = cudaMemset(ls, 0, (MAX_COSTS + 3) * sizeof(long long))) != cudaSuccess ||
        (err = cudaMemset(lcands, 0, (MAX_COSTS + 3) * sizeof(u64))) != cudaSuccess ||
        (err = cudaMemcpy(ctl, &hc, sizeof(hc), cudaMemcpyHostToDevice)) != cudaSuccess)
        return LTLG_CUDA_ERROR;

    InstArgs A;
    memset(&A, 0, sizeof(A));
    A.n = n;
    A.pitch = pitch;
    A.npos = npos;
    A.nalpha = nalpha;
    A.key_mode = opt->key_mode == LTLG_KEY_EXACT ? KEY_EXACT : KEY_HASH64;
    A.stop_at_found = opt->stop_at_found ? 1 : 0;
    A.neg_type = opt->neg_type;
    A.max_cost = max_cost;
    for (int i = 0; i < 8; ++i) A.cf[i] = cf[i];
    A.right_chunk_big = 64;
    A.unary_rows_big = 64;
    A.small_rows = 1;
    A.tile = tile;
    A.gen = 1;  // the slots were just cleared
    A.small_level = LLONG_MAX / 2;
    A.wait_spins = 1ll << 22;
    A.item_target = (long long)grid * stages * 2;
    A.cap_rows = cap;
    A.cap_entries = cap_entries;
    A.slot_mask = nslots - 1;
    A.cache = cache;
    A.parents = parents;
    A.keys = keys;
    A.slots = slots;
    A.wmeta = wmeta;
    A.kmeta = kmeta;
    A.ls = ls;
    A.ne = ne;
    A.level_cands = lcands;
    A.entries = entries;
    A.found_par = fpar;
    A.ctl = ctl;
    Launch L;
    memset(&L, 0, sizeof(L));
    L.args = dargs;
    L.ninst = 1;
    L.persist = 1;
    L.tile = tile;
    L.stages = stages;
    L.tile_bytes = tile_bytes;
    if ((err = cudaMemcpy(dargs, &A, sizeof(A), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (err = cudaMemcpy(dlaunch, &L, sizeof(L), cudaMemcpyHostToDevice)) != cudaSuccess)
        return LTLG_CUDA_ERROR;
    if ((err = launch_insert_letters(dargs, nalpha, hk, 0)) != cudaSuccess) return LTLG_CUDA_ERROR;
    // Every level in one launch: the level kernel plans each next level on the device.
    if ((err = launch_first_plan(dargs, 1, 1, 0)) != cudaSuccess) return LTLG_CUDA_ERROR;
    if ((err = launch_levels(L, dlaunch, grid, hk, 0)) != cudaSuccess) return LTLG_CUDA_ERROR;
    if ((err = cudaMemcpy(&hc, ctl, sizeof(hc), cudaMemcpyDeviceToHost)) != cudaSuccess) return LTLG_CUDA_ERROR;
    if (hc.status & (ST_WAIT | ST_TMA | ST_STALL)) return LTLG_DEVICE_WAIT;
    // a level that overflowed the scratch rows is the cause of anything after it
    if ((hc.status & ST_OVERFLOW) && !(hc.found && opt->stop_at_found)) return LTLG_NO_MEMORY;
    if (hc.status & ST_TABLE) return LTLG_TABLE_FULL;
    const int last_cost = (int)hc.last_cost > c1 ? (int)hc.last_cost : c1;

    long long hls[MAX_COSTS + 3];
    unsigned long long hlc[MAX_COSTS + 3];
    if ((err = cudaMemcpy(hls, ls, sizeof(hls), cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (err = cudaMemcpy(hlc, lcands, sizeof(hlc), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return LTLG_CUDA_ERROR;
    const long long rows = (long long)hc.row_count < cap ? (long long)hc.row_count : cap;
    const bool stop_found = hc.found && opt->stop_at_found;
    const int top = stop_found ? (int)hc.found_cost : last_cost;
    for (int k = 0; k <= c1; ++k) hls[k] = 0;
    hls[c1 + 1] = nalpha;
    for (int k = top + 2; k < MAX_COSTS + 3; ++k) hls[k] = rows;
    for (int c = c1 + 1; c < top; ++c) all += hlc[c];
    if (!stop_found) {
        // every level up to the last one ran to its end
        if (top >= c1 + 1) all += hlc[top];
        if (all_ltls_out) *all_ltls_out = all;
        if (!hc.found && letter_hit < 0) {
            snprintf(formula, formula_cap, "not_found");
            if (cost_out) *cost_out = last_cost;
            return LTLG_NOT_FOUND;
        }
        if (cost_out) *cost_out = (int)hc.found_cost;
    } else {
        // the reference's count: the level's blocks in order up to the one the device recorded
        all += count_to_found(top, cf, opt->neg_type, hls, (int)(u32)(hc.found_key & 0xFFFFFFFFull));
        if (cost_out) *cost_out = top;
        if (all_ltls_out) *all_ltls_out = all;
    }
    if (letter_hit >= 0) {  // a letter separates; the levels above were only enumerated
        snprintf(formula, formula_cap, "%c", t->alphabet[letter_hit]);
        if (cost_out) *cost_out = c1;
        return LTLG_FOUND;
    }
    const u64 p = hc.found & ~(1ull << 63);

    if ((err = launch_walk(parents, nalpha, hc.found, walk, WALK_CAP, 0)) != cudaSuccess) return LTLG_CUDA_ERROR;
    static_assert(WALK_CAP <= 1024, "walk entries live on the stack");
    u64 ent[2 + 2 * WALK_CAP];
    if ((err = cudaMemcpy(ent, walk, sizeof(ent), cudaMemcpyDeviceToHost)) != cudaSuccess) return LTLG_CUDA_ERROR;
    const u64 count = ent[0], overflow = ent[1];
    if (overflow || count - 1 >= 200) {  // the reference's sentinel for more than 199 nodes
        static const char big[] = "Size of the output is too big";
        if ((int)sizeof(big) > formula_cap) return LTLG_FORMULA_TOO_LONG;
        memcpy(formula, big, sizeof(big));
        return LTLG_FOUND;
    }
    Writer w{formula, formula_cap, 0, false};
    formula[0] = 0;
    write_node(ent + 2, (int)count, p, t->alphabet, nalpha, w, 0);
    if (w.over) {  // the search succeeded; only the caller's buffer is too small
        formula[0] = 0;
        return LTLG_FORMULA_TOO_LONG;
    }
    return LTLG_FOUND;
}
