// Host side of the enumerator: the C ABI of include/ltlgpu.h.
//
// ltlg_engine_learn restates LTLI (code/ltli6463.cu:1043-1497) for the GPU path:
//   letters and the early letter hit ........ :1058-1136
//   level / operator / split order ........... :1199-1445 (NegType rule :1212), planned on the device
//   the find and the candidate count ......... :1232-1234 (first block in order that holds one)
//   on-the-fly overflow regime ............... :1021-1027, :1202-1206, :1442-1443
//   found -> formula string, 200-node limit .. :877-991
// The reference's per-chunk host round trips are gone: a learn is one persistent launch of the
// level kernel, which plans every next level on the device.  The per-block schedule (the
// reference's progress lines) and the on-the-fly regime run level by level from the host.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "ltl_kernels.cuh"
#include "ltlgpu.h"
#include "scarlet.hpp"
#include "traces.hpp"

using namespace ltlg;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

cudaError_t ensure(DevBuf &b, size_t bytes) {
    if (b.bytes >= bytes && b.p) return cudaSuccess;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e == cudaSuccess) b.bytes = bytes;
    return e;
}

cudaError_t ensure_host(DevBuf &b, size_t bytes) {
    if (b.bytes >= bytes && b.p) return cudaSuccess;
    if (b.p) cudaFreeHost(b.p);
    b.p = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMallocHost(&b.p, bytes);
    if (e == cudaSuccess) b.bytes = bytes;
    return e;
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

u64 host_fmix64(u64 x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

// The level kernel's exact-key fingerprint of a CS (n words, zero padding up to pitch): word i
// adds (lo(w) + lo(k)) * (hi(w) + hi(k)) with k = (i + 1) * 0x9E3779B97F4A7C15 (32-bit sums,
// 64-bit product), and the sum goes through fmix64.  The device adds the same terms in
// another order; the sum is the same modulo 2^64.
u64 host_fingerprint_exact(const uint64_t *w, int n, int pitch) {
    u64 sum = 0;
    for (int i = 0; i < pitch; ++i) {
        const u64 v = i < n ? w[i] : 0ull, k = (u64)(i + 1) * 0x9E3779B97F4A7C15ull;
        sum += (u64)((u32)v + (u32)k) * (u64)((u32)(v >> 32) + (u32)(k >> 32));
    }
    return host_fmix64(sum);
}

// Entries per level plan: 4 unary blocks and, per binary operator, a split per cost up to
// max_cost / 2.
long long entries_for(int max_cost) { return 4 + 3 * ((long long)max_cost / 2 + 2); }

}  // namespace

struct ltlg_engine {
    ltlg_engine_config cfg{};
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    // device buffers of the instance
    DevBuf cache, parents, keys, prio, slots, wmeta, kmeta, ls, ne, lcands, lns, lstats, entries, fpar;
    DevBuf ctl, args, launch, walk, snaps, scorer, scorer_params;
    // pinned host copies
    DevBuf h_ctl, h_args, h_launch, h_walk, h_stage, h_ls, h_lcands, h_lns, h_ne, h_snaps, h_win, h_entries, h_fpar,
        h_lstats;
    volatile u32 *cancel = nullptr;  // mapped host flag read by the planner
    void *cancel_dev = nullptr;
    bool has_scorer = false;
    u64 nslots = 0;
    u32 gen = 0;
    // last learn
    int n = 0, pitch = 0, nalpha = 0, max_cost = 0;
    long long cap_rows = 0;
    int tile = 0, stages = 0, grid = 0, hk = 0;
    long long tile_bytes = 0;
    std::vector<long long> level_start;
    std::string last_error;
};

namespace {

int fail_cuda(ltlg_engine *e, cudaError_t err, ltlg_result *res) {
    e->last_error = cudaGetErrorString(err);
    if (res) {
        res->status = LTLG_CUDA_ERROR;
        free(res->formula);
        res->formula = strdup(e->last_error.c_str());
    }
    return LTLG_CUDA_ERROR;
}

int fail_status(ltlg_result *res, int status) {
    res->status = status;
    free(res->formula);
    res->formula = strdup(ltlg_status_string(status));
    return status;
}

struct Block {
    int op, lcost, rcost;
    long long l0, l1, r0, r1;
    long long candidates;  // as the reference counts them (U: 2 per pair)
};

// Blocks of cost c in the reference's order (ltli6463.cu:1209-1440); positions are indices.
std::vector<Block> level_blocks(int c, const int *cf, int neg_type, const std::vector<long long> &ls) {
    const int c1 = cf[0];
    auto lo = [&](int k) { return (k >= c1 && k < c && k + 1 < (int)ls.size()) ? ls[k] : 0ll; };
    auto hi = [&](int k) { return (k >= c1 && k < c && k + 1 < (int)ls.size()) ? ls[k + 1] : 0ll; };
    std::vector<Block> out;
    auto unary = [&](int op, int k) {
        const long long a = lo(k), b = hi(k);
        if (b > a) out.push_back({op, k, 0, 0, 0, a, b, b - a});
    };
    auto binary = [&](int op, int cop) {
        for (int i = c1; 2 * i <= c - cop; ++i) {
            const int j = c - i - cop;
            const long long a = lo(i), b = hi(i), x = lo(j), y = hi(j);
            if (b > a && y > x) out.push_back({op, i, j, a, b, x, y, (op == OP_U ? 2 : 1) * (b - a) * (y - x)});
        }
    };
    if ((neg_type == 1 && c - cf[1] >= c1) || (neg_type == 2 && c - cf[1] == c1)) unary(OP_NEG, c - cf[1]);
    binary(OP_AND, cf[2]);
    binary(OP_OR, cf[3]);
    if (c - cf[4] >= c1) unary(OP_X, c - cf[4]);
    if (c - cf[5] >= c1) unary(OP_F, c - cf[5]);
    if (c - cf[6] >= c1) unary(OP_G, c - cf[6]);
    binary(OP_U, cf[7]);
    return out;
}

void build_string(const std::map<u64, u64> &par, u64 row, u64 p, bool is_root, const std::string &alpha, int nalpha,
                  std::string &out, int depth) {
    if (!is_root && row < (u64)nalpha) {
        out += alpha[row];
        return;
    }
    if (depth > 100000) return;
    const int op = parent_op(p);
    auto child = [&](u64 r) {
        if (r < (u64)nalpha) {
            out += alpha[r];
            return;
        }
        auto it = par.find(r);
        build_string(par, r, it == par.end() ? 0 : it->second, false, alpha, nalpha, out, depth + 1);
    };
    switch (op) {
    case OP_NEG: out += "~("; child(parent_left(p)); out += ")"; break;
    case OP_X: out += "X("; child(parent_left(p)); out += ")"; break;
    case OP_F: out += "F("; child(parent_left(p)); out += ")"; break;
    case OP_G: out += "G("; child(parent_left(p)); out += ")"; break;
    case OP_AND:
    case OP_OR:
    case OP_U:
        out += "(";
        child(parent_left(p));
        out += op == OP_AND ? ")&(" : op == OP_OR ? ")|(" : ")U(";
        child(parent_right(p));
        out += ")";
        break;
    default: out += alpha.empty() ? '?' : alpha[0]; break;
    }
}

// Level-kernel geometry for rows of `pitch` words: the left tile (shrunk from `want` until at
// least three item slots fit the shared memory) and the slots.  Returns false when not even one
// slot of a 2-row tile fits.
bool geometry(int want, int pitch, int &tile, int &stages, long long &tile_bytes) {
    constexpr long long BUDGET = 200 * 1024;  // dynamic shared memory for the slots' tiles
    tile = want;
    while (tile > 2 && BUDGET / ((long long)tile * pitch * 8) < 3) tile /= 2;
    tile_bytes = (long long)tile * pitch * 8;
    stages = (int)std::min<long long>(8, BUDGET / tile_bytes);
    return stages >= 1;
}

// What the level loop of one learn ends with.
struct LoopOut {
    int status = LTLG_NOT_FOUND;
    bool found = false, on_the_fly = false;
    int last_cost = 0;
    double device_ms = 0;
    int launches = 0;
    std::vector<ltlg_block_stat> bstats;
};

}  // namespace

extern "C" {

LTLG_API int ltlg_abi_version(void) { return LTLG_ABI_VERSION; }

LTLG_API const char *ltlg_status_string(int s) {
    switch (s) {
    case LTLG_FOUND: return "found";
    case LTLG_NOT_FOUND: return "not_found";
    case LTLG_INPUT_LIMITS: return "see_the_error";
    case LTLG_TIMEOUT: return "timeout";
    case LTLG_NO_MEMORY: return "no_memory";
    case LTLG_BAD_ARGS: return "bad_arguments";
    case LTLG_CUDA_ERROR: return "cuda_error";
    case LTLG_DEVICE_WAIT: return "device_wait_gave_up";
    case LTLG_TABLE_FULL: return "hash_set_full";
    case LTLG_NO_DEVICE: return "no_cuda_device";
    case LTLG_FORMULA_TOO_LONG: return "formula_too_long";
    default: return "unknown";
    }
}

LTLG_API void ltlg_default_engine_config(ltlg_engine_config *c) {
    memset(c, 0, sizeof(*c));
    c->device = 0;
    c->slots_log2 = 27;
    c->cache_bytes = 16ll << 30;
    c->max_rows = 64ll << 20;
    c->max_traces = 8192;
    c->block_threads = LEVEL_THREADS;
    c->left_tile = 4;
    c->right_chunk = 16;
    c->unary_rows = 32;
    c->small_rows = 1;
    c->wait_spins = 0;
    c->small_level = 0;
}

LTLG_API void ltlg_default_options(ltlg_options *o) {
    memset(o, 0, sizeof(*o));
    for (int i = 0; i < 8; ++i) o->cost_fun[i] = 1;
    o->max_cost = 500;
    o->rlx_unq_chk_type = 3;
    o->neg_type = 2;
    o->key_mode = LTLG_KEY_EXACT;
    o->schedule = LTLG_SCHEDULE_FUSED;
    o->order = LTLG_ORDER_PLAIN;
    o->stop_at_found = 1;
}

LTLG_API int ltlg_engine_create(const ltlg_engine_config *cfg_in, ltlg_engine **out) {
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LTLG_NO_DEVICE;
    ltlg_engine_config cfg;
    if (cfg_in)
        cfg = *cfg_in;
    else
        ltlg_default_engine_config(&cfg);
    if (cfg.device < 0 || cfg.device >= ndev) return LTLG_BAD_ARGS;
    if (cfg.slots_log2 < 10 || cfg.slots_log2 > 34) return LTLG_BAD_ARGS;
    if (cfg.left_tile != 2 && cfg.left_tile != 4 && cfg.left_tile != 8) return LTLG_BAD_ARGS;
    if (cfg.right_chunk < 1 || cfg.unary_rows < 1 || cfg.max_traces < 1 || cfg.wait_spins < 0 ||
        cfg.small_level < 0)
        return LTLG_BAD_ARGS;
    if (cfg.max_rows <= 0 || cfg.max_rows > (1ll << 30) - 1) cfg.max_rows = (1ll << 30) - 1;
    auto *e = new ltlg_engine();
    e->cfg = cfg;
    cudaError_t err = cudaSetDevice(cfg.device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, cfg.device);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreate(&e->ev_a);
    if (err == cudaSuccess) err = cudaEventCreate(&e->ev_b);
    e->nslots = 1ull << cfg.slots_log2;
    if (err == cudaSuccess) err = ensure(e->slots, e->nslots * 8);
    if (err == cudaSuccess) err = cudaMemsetAsync(e->slots.p, 0, e->nslots * 8, e->stream);
    if (err == cudaSuccess) err = ensure(e->cache, (size_t)cfg.cache_bytes);
    if (err == cudaSuccess) err = ensure(e->ctl, sizeof(InstCtl));
    if (err == cudaSuccess) err = ensure_host(e->h_ctl, sizeof(InstCtl));
    if (err == cudaSuccess) err = ensure(e->args, sizeof(InstArgs));
    if (err == cudaSuccess) err = ensure_host(e->h_args, sizeof(InstArgs));
    if (err == cudaSuccess) err = ensure(e->launch, sizeof(Launch));
    if (err == cudaSuccess) err = ensure_host(e->h_launch, sizeof(Launch));
    if (err == cudaSuccess) err = ensure(e->walk, (2 + 2 * 1024) * 8);
    if (err == cudaSuccess) err = ensure_host(e->h_walk, (2 + 2 * 1024) * 8);
    if (err == cudaSuccess) {
        void *p = nullptr;
        err = cudaHostAlloc(&p, 64, cudaHostAllocMapped);
        if (err == cudaSuccess) {
            memset(p, 0, 64);
            e->cancel = (volatile u32 *)p;
            err = cudaHostGetDevicePointer(&e->cancel_dev, p, 0);
        }
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) {
        ltlg_engine_destroy(e);
        return err == cudaErrorMemoryAllocation ? LTLG_NO_MEMORY : LTLG_CUDA_ERROR;
    }
    *out = e;
    return 0;
}

LTLG_API void ltlg_engine_destroy(ltlg_engine *e) {
    if (!e) return;
    cudaSetDevice(e->cfg.device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (DevBuf *b : {&e->cache, &e->parents, &e->keys, &e->prio, &e->slots, &e->wmeta, &e->kmeta, &e->ls, &e->ne, &e->lcands,
                      &e->lns, &e->lstats, &e->entries, &e->fpar, &e->ctl, &e->args, &e->launch, &e->walk, &e->snaps,
                      &e->scorer, &e->scorer_params})
        if (b->p) cudaFree(b->p);
    for (DevBuf *b : {&e->h_ctl, &e->h_args, &e->h_launch, &e->h_walk, &e->h_stage, &e->h_ls, &e->h_lcands, &e->h_lns,
                      &e->h_ne, &e->h_snaps, &e->h_win, &e->h_entries, &e->h_fpar, &e->h_lstats})
        if (b->p) cudaFreeHost(b->p);
    if (e->cancel) cudaFreeHost((void *)e->cancel);
    for (cudaEvent_t ev : {e->ev_a, e->ev_b})
        if (ev) cudaEventDestroy(ev);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

LTLG_API void ltlg_result_free(ltlg_result *r) {
    if (!r) return;
    free(r->formula);
    free(r->levels);
    free(r->blocks);
    memset(r, 0, sizeof(*r));
}

}  // extern "C"

namespace {

// Runs the level kernel once over the engine's instance and waits for it, with the learn's
// time limit (the planner ends the search at the next level boundary once the cancel flag is set).
cudaError_t run_levels(ltlg_engine *e, bool persist, int grid, double t0, double time_limit_s, LoopOut &o) {
    Launch *hl = (Launch *)e->h_launch.p;
    memset(hl, 0, sizeof(Launch));  // no batch: one instance
    hl->args = (const InstArgs *)e->args.p;
    hl->batch = nullptr;
    hl->ninst = 1;
    hl->persist = persist ? 1 : 0;
    hl->tile = e->tile;
    hl->stages = e->stages;
    hl->tile_bytes = e->tile_bytes;
    cudaStream_t st = e->stream;
    cudaError_t err = cudaMemcpyAsync(e->launch.p, hl, sizeof(Launch), cudaMemcpyHostToDevice, st);
    if (err != cudaSuccess) return err;
    cudaEventRecord(e->ev_a, st);
    err = launch_levels(*hl, (const Launch *)e->launch.p, grid, e->hk, st);
    if (err != cudaSuccess) return err;
    cudaEventRecord(e->ev_b, st);
    ++o.launches;
    if (time_limit_s > 0) {
        while ((err = cudaEventQuery(e->ev_b)) == cudaErrorNotReady) {
            if (now_s() - t0 > time_limit_s) *e->cancel = 1u;
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
        if (err != cudaSuccess) return err;
    } else if ((err = cudaEventSynchronize(e->ev_b)) != cudaSuccess) {
        return err;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev_a, e->ev_b);
    o.device_ms += ms;
    return cudaSuccess;
}

cudaError_t read_ctl(ltlg_engine *e, InstCtl *hc) {
    cudaError_t err = cudaMemcpyAsync(hc, e->ctl.p, sizeof(InstCtl), cudaMemcpyDeviceToHost, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    return err;
}

// Opens items [lo, hi) of the current plan (sequence seq) for claiming.
cudaError_t open_window(ltlg_engine *e, u32 seq, long long lo, long long hi, int slot) {
    u64 *w = (u64 *)e->h_win.p + 2 * slot;
    w[0] = ((u64)seq << SEQ_SHIFT) | (u64)lo;
    w[1] = ((u64)seq << SEQ_SHIFT) | (u64)hi;
    InstCtl *dc = (InstCtl *)e->ctl.p;
    cudaError_t err = cudaMemcpyAsync(&dc->limit, &w[1], 8, cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess) err = cudaMemcpyAsync(&dc->claimed, &w[0], 8, cudaMemcpyHostToDevice, e->stream);
    return err;
}

int fatal_status(u32 f) { return (f & ST_TABLE) ? LTLG_TABLE_FULL : LTLG_DEVICE_WAIT; }

}  // namespace

extern "C" {

LTLG_API int ltlg_engine_learn(ltlg_engine *e, const ltlg_traces *t, const ltlg_options *opt, ltlg_result *res) {
    memset(res, 0, sizeof(*res));
    const double t0 = now_s();
    if (!e || !t || !opt) return fail_status(res, LTLG_BAD_ARGS);
    const int *cf = opt->cost_fun;
    for (int i = 0; i < 8; ++i)
        if (cf[i] <= 0 || cf[i] > SHRT_MAX) return fail_status(res, LTLG_BAD_ARGS);
    const int c1 = cf[0];
    const int npos = t->num_pos, nneg = t->num_neg, n = npos + nneg;
    const std::string alpha = t->alphabet ? t->alphabet : "";
    const int nalpha = (int)alpha.size();
    const bool ref_keys = opt->key_mode == LTLG_KEY_REF;
    if (!traces_well_formed(t) || (ref_keys && (opt->rlx_unq_chk_type < 1 || opt->rlx_unq_chk_type > 3)) ||
        opt->key_mode < 0 || opt->key_mode > 2 || n > e->cfg.max_traces || nalpha > 26 || opt->max_cost < 1 ||
        opt->max_cost > SHRT_MAX || (opt->order != LTLG_ORDER_PLAIN && opt->order != LTLG_ORDER_LEARNED) ||
        (opt->order == LTLG_ORDER_LEARNED && !e->has_scorer))
        return fail_status(res, LTLG_BAD_ARGS);
    int max_len = 0, len_sum = 0;
    for (int i = 0; i < n; ++i) {
        const int ln = t->offsets[i + 1] - t->offsets[i];
        max_len = std::max(max_len, ln);
        len_sum += ln;
    }
    res->cost = c1;
    if ((opt->limit_traces && n > 64) || max_len > 63) {
        res->status = LTLG_INPUT_LIMITS;
        res->formula = strdup("see_the_error");
        return res->status;
    }
    cudaError_t err = cudaSetDevice(e->cfg.device);
    if (err != cudaSuccess) return fail_cuda(e, err, res);

    // Letters (ltli6463.cu:1100-1136): CS rows 0 .. nalpha-1; the first letter that
    // separates the traces ends the search at cost c1.
    const int pitch = std::max(4, (n + 3) & ~3);
    std::vector<u64> letters((size_t)nalpha * pitch, 0ull);
    int letter_hit = -1;
    uint64_t all = 0;
    for (int j = 0; j < nalpha; ++j) {
        const uint32_t bit = 1u << (alpha[j] - 'a');
        bool acc = true;
        for (int i = 0; i < n; ++i) {
            u64 w = 0;
            for (int k = t->offsets[i]; k < t->offsets[i + 1]; ++k)
                if (t->steps[k] & bit) w |= 1ull << (k - t->offsets[i]);
            letters[(size_t)j * pitch + i] = w;
            if (i < npos ? !(w & 1) : (w & 1)) acc = false;
        }
        all++;
        if (acc && letter_hit < 0) {
            letter_hit = j;
            if (opt->stop_at_found) break;
        }
    }
    const int max_cost = opt->max_cost;
    e->n = n;
    e->pitch = pitch;
    e->nalpha = nalpha;
    e->max_cost = max_cost;
    const long long cap_rows =
        std::min<long long>(e->cfg.max_rows, e->cfg.cache_bytes / ((long long)pitch * 8ll));
    e->cap_rows = cap_rows;
    e->level_start.assign((size_t)std::max(max_cost, c1) + 3, 0);
    for (size_t k = (size_t)c1 + 1; k < e->level_start.size(); ++k) e->level_start[k] = nalpha;
    if (letter_hit >= 0 && opt->stop_at_found) {
        res->status = LTLG_FOUND;
        res->cost = c1;
        res->all_ltls = all;
        res->evaluated = all;
        res->rows = letter_hit + 1;
        res->formula = strdup(std::string(1, alpha[letter_hit]).c_str());
        res->found_op = OP_ATOM;
        res->seconds = now_s() - t0;
        return res->status;
    }
    if (n == 0 || nalpha == 0) {
        // nothing to enumerate: every level is empty
        res->status = letter_hit >= 0 ? LTLG_FOUND : LTLG_NOT_FOUND;
        res->cost = letter_hit >= 0 ? c1 : std::max(c1, max_cost);
        res->all_ltls = all;
        res->evaluated = all;
        res->formula = strdup(letter_hit >= 0 ? std::string(1, alpha[letter_hit]).c_str() : "not_found");
        res->seconds = now_s() - t0;
        return res->status;
    }
    if (cap_rows < nalpha + 1) return fail_status(res, LTLG_NO_MEMORY);
    int tile = 0, stages = 0;
    long long tile_bytes = 0;
    if (!geometry(e->cfg.left_tile, pitch, tile, stages, tile_bytes)) return fail_status(res, LTLG_BAD_ARGS);
    const int hk = opt->key_mode == LTLG_KEY_HASH64 ? 1 : 0;
    const size_t smem = level_kernel_smem(stages, tile_bytes);
    const int per_sm = level_kernel_ctas_per_sm(hk, smem);
    if (per_sm < 1) return fail_status(res, LTLG_BAD_ARGS);
    e->tile = tile;
    e->stages = stages;
    e->tile_bytes = tile_bytes;
    e->hk = hk;
    e->grid = e->num_sms * per_sm;

    // Per-word metadata: length mask | positive flag; relaxed-key bit placement.
    std::vector<u64> wmeta(pitch, 0ull);
    std::vector<u32> kmeta(pitch, 0u);
    for (int i = 0; i < n; ++i) {
        const int ln = t->offsets[i + 1] - t->offsets[i];
        wmeta[i] = (ln >= 63 ? 0x7FFFFFFFFFFFFFFFull : ((1ull << ln) - 1)) | (i < npos ? (1ull << 63) : 0ull);
    }
    int rlx_type = 0;
    if (ref_keys) {
        rlx_type = len_sum > 126 ? opt->rlx_unq_chk_type : 0;
        long long start = 0;
        const int stride = len_sum > 126 ? len_sum / 126 : 1;
        for (int i = 0; i < n; ++i) {
            const int ln = t->offsets[i + 1] - t->offsets[i];
            int count = ln, step = 1;
            if (rlx_type == 1) {
                step = stride;
                count = (ln + stride - 1) / stride;
            } else if (rlx_type == 2) {
                count = (126 * ln + len_sum) / len_sum;
            }
            kmeta[i] = (u32)std::min<long long>(start, 126) | ((u32)count << 16) | ((u32)std::min(step, 255) << 24);
            start += count;
        }
    }

    // Buffers (sized for this learn's max_cost: no cap on costs or splits)
    const long long ncost = (long long)max_cost + 3;
    const long long cap_entries = entries_for(max_cost);
    const bool want_stats = opt->order == LTLG_ORDER_LEARNED || opt->record_levels >= 2;
    if ((err = ensure(e->parents, (size_t)cap_rows * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if (opt->key_mode != LTLG_KEY_EXACT && (err = ensure(e->keys, (size_t)cap_rows * 16)) != cudaSuccess)
        return fail_cuda(e, err, res);
    if (ref_keys && (err = ensure(e->prio, (size_t)cap_rows * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure(e->wmeta, (size_t)pitch * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure(e->kmeta, (size_t)pitch * 4)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure(e->ls, (size_t)ncost * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure(e->ne, (size_t)ncost * 4)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure(e->lcands, (size_t)ncost * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure(e->lns, (size_t)ncost * LEVEL_TRACE * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure(e->lstats, (size_t)ncost * LSTATS * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure(e->entries, (size_t)(2 * cap_entries) * sizeof(Entry))) != cudaSuccess)
        return fail_cuda(e, err, res);
    if ((err = ensure(e->fpar, (size_t)cap_entries * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure(e->snaps, (size_t)cap_entries * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure_host(e->h_stage, std::max<size_t>((size_t)nalpha * pitch * 8, (size_t)pitch * 12))) !=
            cudaSuccess ||
        (err = ensure_host(e->h_ls, (size_t)ncost * 8)) != cudaSuccess ||
        (err = ensure_host(e->h_lcands, (size_t)ncost * 8)) != cudaSuccess ||
        (err = ensure_host(e->h_lns, (size_t)ncost * LEVEL_TRACE * 8)) != cudaSuccess ||
        (err = ensure_host(e->h_snaps, (size_t)cap_entries * 8)) != cudaSuccess ||
        (err = ensure_host(e->h_win, (size_t)(2 * cap_entries + 2) * 8)) != cudaSuccess ||
        (err = ensure_host(e->h_entries, (size_t)cap_entries * sizeof(Entry))) != cudaSuccess)
        return fail_cuda(e, err, res);
    cudaStream_t st = e->stream;
    memcpy(e->h_stage.p, letters.data(), letters.size() * 8);
    if ((err = cudaMemcpyAsync(e->cache.p, e->h_stage.p, letters.size() * 8, cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
        return fail_cuda(e, err, res);
    if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, res);
    memcpy(e->h_stage.p, wmeta.data(), (size_t)pitch * 8);
    memcpy((char *)e->h_stage.p + (size_t)pitch * 8, kmeta.data(), (size_t)pitch * 4);
    cudaMemcpyAsync(e->wmeta.p, e->h_stage.p, (size_t)pitch * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(e->kmeta.p, (char *)e->h_stage.p + (size_t)pitch * 8, (size_t)pitch * 4, cudaMemcpyHostToDevice,
                    st);
    // Hash-set generation: slots of older generations count as empty.
    if (++e->gen > 255) {
        cudaMemsetAsync(e->slots.p, 0, e->nslots * 8, st);
        e->gen = 1;
    }
    cudaMemsetAsync(e->ls.p, 0, (size_t)ncost * 8, st);
    cudaMemsetAsync(e->lcands.p, 0, (size_t)ncost * 8, st);
    cudaMemsetAsync(e->lns.p, 0, (size_t)ncost * LEVEL_TRACE * 8, st);
    if (want_stats) cudaMemsetAsync(e->lstats.p, 0, (size_t)ncost * LSTATS * 8, st);
    InstCtl *hc = (InstCtl *)e->h_ctl.p;
    memset(hc, 0, sizeof(InstCtl));
    hc->row_count = (u64)nalpha;
    hc->found_key = NO_FIND;
    hc->plan.cost = c1;
    cudaMemcpyAsync(e->ctl.p, hc, sizeof(InstCtl), cudaMemcpyHostToDevice, st);
    *e->cancel = 0u;

    const bool per_block = opt->schedule == LTLG_SCHEDULE_PER_BLOCK;
    const bool learned = opt->order == LTLG_ORDER_LEARNED;
    InstArgs *ha = (InstArgs *)e->h_args.p;
    memset(ha, 0, sizeof(InstArgs));
    InstArgs &A = *ha;
    A.n = n;
    A.pitch = pitch;
    A.npos = npos;
    A.nalpha = nalpha;
    A.key_mode = opt->key_mode == LTLG_KEY_EXACT ? KEY_EXACT : opt->key_mode == LTLG_KEY_REF ? KEY_REF : KEY_HASH64;
    A.rlx_type = rlx_type;
    A.stop_at_found = opt->stop_at_found ? 1 : 0;
    A.find_first = learned ? 1 : 0;
    A.neg_type = opt->neg_type;
    A.max_cost = max_cost;
    A.on_the_fly = 0;
    A.plan_flags = (per_block ? PLAN_UNFUSED : 0) | (learned ? PLAN_LEARNED : 0);
    for (int i = 0; i < 8; ++i) A.cf[i] = cf[i];
    A.right_chunk_big = e->cfg.right_chunk;
    A.unary_rows_big = e->cfg.unary_rows;
    A.small_rows = std::max(1, e->cfg.small_rows);
    A.tile = tile;
    A.gen = e->gen;
    // by default every level sizes its items from its own size (up to the big sizes)
    A.small_level = e->cfg.small_level > 0 ? e->cfg.small_level : LLONG_MAX / 2;
    A.wait_spins = e->cfg.wait_spins > 0 ? e->cfg.wait_spins : (1ll << 22);
    A.cap_rows = cap_rows;
    A.cap_entries = cap_entries;
    A.learn_min_items = (long long)e->grid * stages;
    A.item_target = (long long)e->grid * stages * 2;
    A.slot_mask = e->nslots - 1;
    A.cache = (u64 *)e->cache.p;
    A.parents = (u64 *)e->parents.p;
    A.keys = opt->key_mode != LTLG_KEY_EXACT ? (u64 *)e->keys.p : nullptr;
    A.prio = ref_keys ? (u64 *)e->prio.p : nullptr;
    A.slots = (u64 *)e->slots.p;
    A.wmeta = (const u64 *)e->wmeta.p;
    A.kmeta = (const u32 *)e->kmeta.p;
    A.ls = (long long *)e->ls.p;
    A.ne = (int *)e->ne.p;
    A.level_cands = (u64 *)e->lcands.p;
    A.level_ns = (u64 *)e->lns.p;
    A.lstats = want_stats ? (u64 *)e->lstats.p : nullptr;
    A.entries = (Entry *)e->entries.p;
    A.found_par = (u64 *)e->fpar.p;
    A.ctl = (InstCtl *)e->ctl.p;
    A.model = learned ? e->scorer.p : nullptr;
    // the planner reads the (mapped host) cancel flag at each level end only under a time limit
    A.cancel = opt->time_limit_s > 0 ? (const volatile u32 *)e->cancel_dev : nullptr;
    const InstArgs *dA = (const InstArgs *)e->args.p;
    cudaMemcpyAsync(e->args.p, ha, sizeof(InstArgs), cudaMemcpyHostToDevice, st);
    if ((err = launch_insert_letters(dA, nalpha, hk, st)) != cudaSuccess) return fail_cuda(e, err, res);
    const bool persist = !per_block;
    if ((err = launch_first_plan(dA, 1, persist ? 1 : 0, st)) != cudaSuccess) return fail_cuda(e, err, res);

    LoopOut o;
    o.launches = 2;
    o.last_cost = c1;
    int shortage = -1;
    bool last_round = false;
    uint64_t all_before = all;
    InstCtl *dctl = (InstCtl *)e->ctl.p;
    const double tl = opt->time_limit_s;
    if (persist) {
        // ---- every level in one launch, planned on the device
        if ((err = run_levels(e, true, e->grid, t0, tl, o)) != cudaSuccess) return fail_cuda(e, err, res);
        if ((err = read_ctl(e, hc)) != cudaSuccess) return fail_cuda(e, err, res);
        o.last_cost = std::max<int>(c1, (int)hc->last_cost);
        if (hc->status & ST_FATAL) {
            o.status = fatal_status(hc->status);
        } else if (hc->found) {
            o.found = true;
        } else if (hc->flags & CTL_CANCELLED) {
            o.status = LTLG_TIMEOUT;
        } else if (hc->status & ST_OVERFLOW) {
            // the level that overflowed ran to its end; continue after it on the host, check-only
            o.on_the_fly = true;
            shortage = (int)hc->overflow_cost;
        }
    } else {
        if ((err = read_ctl(e, hc)) != cudaSuccess) return fail_cuda(e, err, res);
    }

    // ---- host-driven levels: the per-block schedule (per-block statistics, the reference's
    // progress lines) and the on-the-fly overflow regime (ltli6463.cu:1202-1206, 1442-1443).
    // The plan of each level is made on the device (closed); the host opens it in windows.
    const bool host_levels = (per_block || o.on_the_fly) && o.status == LTLG_NOT_FOUND && !o.found;
    auto switch_on_the_fly = [&](int next_cost) -> cudaError_t {
        A.on_the_fly = 1;
        cudaError_t x = cudaMemcpyAsync(e->args.p, ha, sizeof(InstArgs), cudaMemcpyHostToDevice, st);
        if (x != cudaSuccess) return x;
        static const u32 zero = 0;
        x = cudaMemcpyAsync(&dctl->flags, &zero, 4, cudaMemcpyHostToDevice, st);
        if (x == cudaSuccess) x = launch_plan_level(dA, next_cost, st);
        ++o.launches;
        if (x == cudaSuccess) x = read_ctl(e, hc);
        return x;
    };
    if (host_levels && o.on_the_fly)
        if ((err = switch_on_the_fly((int)hc->last_cost + 1)) != cudaSuccess) return fail_cuda(e, err, res);
    if (host_levels) {
        const size_t W = sizeof(Entry);
        for (;;) {
            if (hc->plan.halt || (hc->flags & CTL_DONE)) break;
            const int cost = hc->plan.cost;
            if (cost > max_cost) break;
            if (o.on_the_fly && shortage >= 0) {
                const int dif = cost - shortage;
                if (dif == cf[1] || dif == c1 + cf[2] || dif == c1 + cf[3] || dif == cf[4] || dif == cf[5] ||
                    dif == cf[6] || dif == c1 + cf[7])
                    last_round = true;
            }
            const u32 seq = hc->seq;
            const int ne = hc->plan.nentries;
            std::vector<int> order;
            Entry *hent = (Entry *)e->h_entries.p;
            if (per_block) {
                // one window per block, in the reference's order (unfused plans: an entry is a block)
                cudaMemcpyAsync(hent, e->entries.p, (size_t)ne * W, cudaMemcpyDeviceToHost, st);
                if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, res);
                for (int q = 0; q < ne; ++q) order.push_back(q);
                std::sort(order.begin(), order.end(), [&](int a, int b) { return hent[a].pos < hent[b].pos; });
                for (size_t q = 0; q < order.size(); ++q) {
                    const Entry &E = hent[order[q]];
                    cudaMemcpyAsync((u64 *)e->snaps.p + q, &dctl->row_count, 8, cudaMemcpyDeviceToDevice, st);
                    if ((err = open_window(e, seq, E.item0, E.item0 + E.items, (int)q)) != cudaSuccess)
                        return fail_cuda(e, err, res);
                    const int grid = (int)std::max<long long>(1, std::min<long long>(E.items, e->grid));
                    if ((err = run_levels(e, false, grid, t0, 0.0, o)) != cudaSuccess) return fail_cuda(e, err, res);
                }
                cudaMemcpyAsync(e->h_snaps.p, e->snaps.p, order.size() * 8, cudaMemcpyDeviceToHost, st);
            } else {
                if ((err = open_window(e, seq, 0, hc->plan.items, 0)) != cudaSuccess) return fail_cuda(e, err, res);
                const int grid = (int)std::max<long long>(1, std::min<long long>(hc->plan.items, e->grid));
                if ((err = run_levels(e, false, grid, t0, 0.0, o)) != cudaSuccess) return fail_cuda(e, err, res);
            }
            if ((err = read_ctl(e, hc)) != cudaSuccess) return fail_cuda(e, err, res);
            if (per_block) {
                const u64 *sn = (const u64 *)e->h_snaps.p;
                uint64_t before = all_before;
                for (size_t q = 0; q < order.size(); ++q) {
                    const Entry &E = hent[order[q]];
                    ltlg_block_stat sb{};
                    sb.cost = cost;
                    sb.op = E.kind == ENT_UNARY ? unary_slot_op(__builtin_ctz((unsigned)E.opmask)) : E.op;
                    sb.left_cost = E.lcost;
                    sb.right_cost = E.kind == ENT_UNARY ? 0 : E.rcost;
                    sb.stored_before = std::min<long long>((long long)sn[q], cap_rows);
                    sb.all_before = before;
                    sb.to_check = (long long)E.cand;
                    before += (uint64_t)E.cand;
                    o.bstats.push_back(sb);
                }
                all_before = before;
            }
            o.last_cost = cost;
            if (hc->status & ST_FATAL) {
                o.status = fatal_status(hc->status);
                break;
            }
            if (hc->found) {
                o.found = true;
                if (opt->stop_at_found) break;
            }
            if (!o.on_the_fly && (hc->status & ST_OVERFLOW)) {
                // switch to the on-the-fly regime: the next levels are check-only
                o.on_the_fly = true;
                if ((err = switch_on_the_fly(cost + 1)) != cudaSuccess) return fail_cuda(e, err, res);
            }
            if (last_round) break;
            if (o.on_the_fly && shortage == -1) shortage = cost;
            if (tl > 0 && now_s() - t0 > tl) {
                o.status = LTLG_TIMEOUT;
                break;
            }
        }
    }

    // ---- level ranges, statistics, the reference's candidate count
    cudaMemcpyAsync(e->h_ls.p, e->ls.p, (size_t)ncost * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(e->h_lcands.p, e->lcands.p, (size_t)ncost * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(e->h_lns.p, e->lns.p, (size_t)ncost * LEVEL_TRACE * 8, cudaMemcpyDeviceToHost, st);
    if ((err = read_ctl(e, hc)) != cudaSuccess) return fail_cuda(e, err, res);
    const long long rows_final = std::min<long long>((long long)hc->row_count, cap_rows);
    const long long *hls = (const long long *)e->h_ls.p;
    const u64 *hlc = (const u64 *)e->h_lcands.p;
    const u64 *hns = (const u64 *)e->h_lns.p;
    const bool found = o.found || hc->found != 0;
    const int found_cost = found ? (int)hc->found_cost : -1;
    const u64 found_word = hc->found;
    const bool stop_found = found && opt->stop_at_found;
    const int top = stop_found ? found_cost : std::max(o.last_cost, c1);
    std::vector<long long> &ls = e->level_start;
    ls.assign((size_t)std::max(max_cost, c1) + 3, rows_final);
    for (int k = 0; k <= c1 && k < (int)ls.size(); ++k) ls[k] = 0;
    if (c1 + 1 < (int)ls.size()) ls[c1 + 1] = nalpha;
    for (int k = c1 + 2; k <= top + 1 && k < (int)ls.size(); ++k) ls[k] = hls[k];
    std::vector<ltlg_level_stat> lstats;
    u64 prev_ns = hc->t_start;
    for (int c = c1 + 1; c <= top && c + 1 < (int)ls.size(); ++c) {
        ltlg_level_stat L{};
        L.cost = c;
        L.candidates = hlc[c];
        L.uniques = (uint64_t)(ls[c + 1] - ls[c]);
        const u64 *tr = hns + (size_t)c * LEVEL_TRACE;
        const u64 end = tr[LT_END];
        if (end && prev_ns) {
            L.ms = (double)(end - prev_ns) * 1e-6;
            auto since = [&](u64 t) { return t >= prev_ns ? (double)(t - prev_ns) * 1e-3 : 0.0; };
            if (tr[LT_PUBLISHED]) L.plan_us = since(tr[LT_PUBLISHED]);
            if (tr[LT_CLAIMED]) L.claim_us = since(tr[LT_CLAIMED]);
            if (tr[LT_STARTED]) L.start_us = since(tr[LT_STARTED]);
        }
        if (end) prev_ns = end;
        lstats.push_back(L);
    }
    // all_ltls: whole levels before the level of the find, then that level's blocks in the
    // reference's order up to and including the block the device recorded (the first block in
    // that order that holds an accepting candidate, or with the learned order the one found).
    for (const auto &L : lstats)
        if (!(stop_found && L.cost == found_cost)) all += L.candidates;
    if (stop_found && found_word) {
        const u32 fpos = (u32)(hc->found_key & 0xFFFFFFFFull);
        std::vector<Block> blocks = level_blocks(found_cost, cf, opt->neg_type, ls);
        for (size_t q = 0; q < blocks.size() && q <= fpos; ++q) all += (uint64_t)blocks[q].candidates;
        if (per_block) {
            // drop the blocks after the one holding the find
            size_t keep = 0;
            int seen = 0;
            for (size_t i = 0; i < o.bstats.size(); ++i) {
                keep = i + 1;
                if (o.bstats[i].cost == found_cost && seen++ == (int)fpos) break;
            }
            o.bstats.resize(keep);
        }
    }
    int status = o.status;
    if (found && (status == LTLG_NOT_FOUND || status == LTLG_FOUND)) status = LTLG_FOUND;
    if (status == LTLG_NOT_FOUND && (hc->flags & CTL_CANCELLED)) status = LTLG_TIMEOUT;
    res->status = status;
    res->cost = found ? found_cost : o.last_cost;
    res->all_ltls = all;
    res->on_the_fly = o.on_the_fly ? 1 : 0;
    res->device_flags = hc->status;
    res->device_ms = o.device_ms;
    res->evaluated = (uint64_t)nalpha + hc->evaluated;
    res->rows = rows_final;

    std::string formula;
    if (letter_hit >= 0) {
        formula = std::string(1, alpha[letter_hit]);
        res->found_op = OP_ATOM;
        res->cost = c1;
        res->status = LTLG_FOUND;
    } else if (found && found_word) {
        const int wcap = 1024;
        if ((err = launch_walk((const u64 *)e->parents.p, nalpha, found_word, (u64 *)e->walk.p, wcap, st)) !=
            cudaSuccess)
            return fail_cuda(e, err, res);
        ++o.launches;
        cudaMemcpyAsync(e->h_walk.p, e->walk.p, (2 + 2 * wcap) * 8, cudaMemcpyDeviceToHost, st);
        if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, res);
        const u64 *w = (const u64 *)e->h_walk.p;
        const u64 count = w[0], overflow = w[1];
        res->found_op = parent_op(found_word & ~(1ull << 63));
        if (overflow || count - 1 >= 200) {
            formula = "Size of the output is too big";
        } else {
            std::map<u64, u64> par;
            for (u64 q = 1; q < count; ++q) par[w[2 + 2 * q]] = w[2 + 2 * q + 1];
            build_string(par, ~0ull, found_word & ~(1ull << 63), true, alpha, nalpha, formula, 0);
        }
    } else {
        formula = status == LTLG_TIMEOUT ? "timeout" : ltlg_status_string(status);
    }
    res->formula = strdup(formula.c_str());
    res->num_levels = (int)lstats.size();
    if (!lstats.empty()) {
        res->levels = (ltlg_level_stat *)malloc(sizeof(ltlg_level_stat) * lstats.size());
        memcpy(res->levels, lstats.data(), sizeof(ltlg_level_stat) * lstats.size());
    }
    res->num_blocks = (int)o.bstats.size();
    if (!o.bstats.empty()) {
        res->blocks = (ltlg_block_stat *)malloc(sizeof(ltlg_block_stat) * o.bstats.size());
        memcpy(res->blocks, o.bstats.data(), sizeof(ltlg_block_stat) * o.bstats.size());
    }
    res->launches = o.launches;
    res->seconds = now_s() - t0;
    return res->status;
}

LTLG_API void *ltlg_engine_stream(ltlg_engine *e) { return e ? (void *)e->stream : nullptr; }

LTLG_API void ltlg_block_features(const ltlg_block_info *in, float *f) {
    BlockInfo b{};
    b.op = in->op;
    b.cost = in->cost;
    b.c1 = in->c1;
    b.lcost = in->lcost;
    b.rcost = in->rcost;
    b.position = in->position;
    b.nblocks = in->nblocks;
    b.lrows = in->lrows;
    b.rrows = in->rrows;
    b.candidates = in->candidates;
    b.level_cands = in->level_cands;
    for (int k = 0; k < 2; ++k) {
        b.lstat[k] = in->lstat[k];
        b.rstat[k] = in->rstat[k];
    }
    b.npos = in->npos;
    b.nneg = in->nneg;
    b.nalpha = in->nalpha;
    block_features(b, f);
}

LTLG_API int ltlg_engine_set_scorer(ltlg_engine *e, const float *params, int32_t count) {
    if (!e || !params || count != MLP_PARAMS) return LTLG_BAD_ARGS;
    cudaSetDevice(e->cfg.device);
    cudaError_t err = ensure(e->scorer_params, MLP_PARAMS * sizeof(float));
    if (err == cudaSuccess) err = ensure(e->scorer, sizeof(MlpDev));
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(e->scorer_params.p, params, MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess) err = launch_scorer_pack((const float *)e->scorer_params.p, (MlpDev *)e->scorer.p, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) return fail_cuda(e, err, nullptr);
    e->has_scorer = true;
    return 0;
}

LTLG_API int ltlg_engine_label_blocks(ltlg_engine *e, const ltlg_traces *t, const ltlg_options *opt_in,
                                      ltlg_block_record *rec, int32_t cap, int32_t *count, ltlg_result *res) {
    if (!e || !t || !opt_in || !count || !res || cap < 0 || (cap > 0 && !rec)) return LTLG_BAD_ARGS;
    *count = 0;
    ltlg_options opt = *opt_in;
    opt.stop_at_found = 1;
    opt.order = LTLG_ORDER_PLAIN;
    opt.schedule = LTLG_SCHEDULE_FUSED;
    opt.record_levels = 2;  // row statistics for the features
    const int rc = ltlg_engine_learn(e, t, &opt, res);
    if (rc != LTLG_FOUND || res->found_op == OP_ATOM || res->on_the_fly) return rc;
    const int c = res->cost;
    const int *cf = opt.cost_fun;
    cudaStream_t st = e->stream;
    InstArgs &A = *(InstArgs *)e->h_args.p;
    const InstArgs *dA = (const InstArgs *)e->args.p;
    const std::vector<long long> &ls = e->level_start;
    if ((int)ls.size() < c + 2) return rc;
    // Back to the start of level c: the rows of the lower levels stay, the list of non-empty
    // levels is cut at c, and level c is planned again with one entry per block, check-only
    // (every candidate's acceptance is tested, nothing stored).
    const long long ncost = (long long)e->max_cost + 3;
    cudaError_t err = ensure_host(e->h_ne, (size_t)ncost * 4);
    if (err == cudaSuccess) err = ensure_host(e->h_lstats, (size_t)ncost * LSTATS * 8);
    if (err == cudaSuccess) err = cudaMemcpyAsync(e->h_ne.p, e->ne.p, (size_t)ncost * 4, cudaMemcpyDeviceToHost, st);
    InstCtl *hc = (InstCtl *)e->h_ctl.p;
    if (err == cudaSuccess) err = read_ctl(e, hc);
    if (err != cudaSuccess) return fail_cuda(e, err, nullptr);
    u32 nec = 0;
    for (u32 q = 0; q < hc->ne_count; ++q)
        if (((const int *)e->h_ne.p)[q] < c) nec = q + 1;
    const u32 seq = hc->seq;
    memset(hc, 0, sizeof(InstCtl));
    hc->row_count = (u64)ls[c];
    hc->found_key = NO_FIND;
    hc->ne_count = nec;
    hc->seq = seq;
    hc->plan.cost = c - 1;
    A.on_the_fly = 1;
    A.plan_flags = PLAN_UNFUSED;
    A.stop_at_found = 0;
    A.find_first = 0;
    A.max_cost = c;  // the window that finishes level c plans nothing after it
    cudaMemcpyAsync(e->ctl.p, hc, sizeof(InstCtl), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(e->args.p, &A, sizeof(InstArgs), cudaMemcpyHostToDevice, st);
    err = launch_plan_level(dA, c, st);
    if (err == cudaSuccess) err = read_ctl(e, hc);
    if (err != cudaSuccess) return fail_cuda(e, err, nullptr);
    if (hc->plan.halt || hc->plan.nentries <= 0) return rc;
    const int ne = hc->plan.nentries, nbl = hc->plan.nblocks;
    if ((err = ensure_host(e->h_fpar, (size_t)std::max(nbl, 1) * 8)) != cudaSuccess) return fail_cuda(e, err, nullptr);
    Entry *hent = (Entry *)e->h_entries.p;
    cudaMemcpyAsync(hent, e->entries.p, (size_t)ne * sizeof(Entry), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(e->h_lstats.p, e->lstats.p, (size_t)ncost * LSTATS * 8, cudaMemcpyDeviceToHost, st);
    if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, nullptr);
    // One window per block: the block's accepting candidates record themselves at its position.
    LoopOut o;
    InstCtl *dctl = (InstCtl *)e->ctl.p;
    static const u64 nofind = NO_FIND;
    for (int q = 0; q < ne; ++q) {
        const Entry &E = hent[q];
        cudaMemcpyAsync(&dctl->found_key, &nofind, 8, cudaMemcpyHostToDevice, st);
        if ((err = open_window(e, hc->seq, E.item0, E.item0 + E.items, q)) != cudaSuccess)
            return fail_cuda(e, err, nullptr);
        const int grid = (int)std::max<long long>(1, std::min<long long>(E.items, e->grid));
        if ((err = run_levels(e, false, grid, now_s(), 0.0, o)) != cudaSuccess) return fail_cuda(e, err, nullptr);
    }
    cudaMemcpyAsync(e->h_fpar.p, e->fpar.p, (size_t)nbl * 8, cudaMemcpyDeviceToHost, st);
    if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, nullptr);
    const u64 *won = (const u64 *)e->h_fpar.p;
    const u64 *lst = (const u64 *)e->h_lstats.p;
    std::vector<int> order(ne);
    for (int q = 0; q < ne; ++q) order[q] = q;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return hent[a].pos < hent[b].pos; });
    int out = 0;
    for (int q : order) {
        if (out >= cap) break;
        const Entry &E = hent[q];
        const bool un = E.kind == ENT_UNARY;
        const int op = un ? unary_slot_op(__builtin_ctz((unsigned)E.opmask)) : E.op;
        const BlockInfo bi = block_info(op, c, E.lcost, un ? E.r1 - E.r0 : E.l1 - E.l0, un ? 1 : E.r1 - E.r0,
                                        (long long)E.cand, E.pos, cf, nbl, (long long)hc->plan.cand, lst, e->max_cost,
                                        A.npos, A.n, A.nalpha);
        ltlg_block_record &r = rec[out++];
        r.cost = c;
        r.op = op;
        r.lcost = bi.lcost;
        r.rcost = bi.rcost;
        r.position = E.pos;
        r.won = (E.pos >= 0 && E.pos < nbl && won[E.pos] != 0) ? 1 : 0;
        r.candidates = (long long)E.cand;
        block_features(bi, r.features);
    }
    *count = out;
    return rc;
}

LTLG_API int ltlg_learn(const ltlg_traces *t, const ltlg_options *opt, ltlg_result *res) {
    ltlg_engine_config cfg;
    ltlg_default_engine_config(&cfg);
    const int n = t ? t->num_pos + t->num_neg : 0;
    // The input limits are checked before the device is touched, as the reference checks
    // them before its first device call (ltli6463.cu:1078-1083).
    if (t && opt && res && !traces_well_formed(t)) {
        memset(res, 0, sizeof(*res));
        return fail_status(res, LTLG_BAD_ARGS);
    }
    if (t && opt && res && t->offsets && t->num_pos >= 0 && t->num_neg >= 0) {
        int max_len = 0;
        for (int i = 0; i < n; ++i) max_len = std::max(max_len, t->offsets[i + 1] - t->offsets[i]);
        if ((opt->limit_traces && n > 64) || max_len > 63) {
            memset(res, 0, sizeof(*res));
            res->status = LTLG_INPUT_LIMITS;
            res->cost = opt->cost_fun[0];
            res->formula = strdup(ltlg_status_string(LTLG_INPUT_LIMITS));
            return res->status;
        }
    }
    const long long pitch = std::max(4, (n + 3) & ~3);
    // The reference sizes its cache from the pitch limit (ltli6463.cu:1152-1156): about
    // 3 GiB of rows.  Keep that budget, bounded by free memory.
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && free_b > 0)
        cfg.cache_bytes = std::min<long long>(4ll << 30, (long long)(free_b / 4));
    cfg.max_rows = std::min<long long>((1ll << 30) - 1, cfg.cache_bytes / (pitch * 8));
    cfg.slots_log2 = 20;
    while ((1ll << cfg.slots_log2) < 2 * cfg.max_rows && cfg.slots_log2 < 28) cfg.slots_log2++;
    cfg.max_traces = std::max(n, 1);
    ltlg_engine *e = nullptr;
    int rc = ltlg_engine_create(&cfg, &e);
    if (rc != 0) {
        memset(res, 0, sizeof(*res));
        return fail_status(res, rc);
    }
    rc = ltlg_engine_learn(e, t, opt, res);
    ltlg_engine_destroy(e);
    return rc;
}

// ---- Batches: the instance slots of one persistent launch (see BatchDev).  Instances that the
// device batch does not take (the reference's relaxed keys, the learned order, the per-block
// schedule, a time limit) and instances whose slot's cache overflowed are learned one by one on
// a fallback engine with the same configuration.
struct ltlg_batch {
    ltlg_engine_config cfg{};
    int slots = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    DevBuf cache, parents, keys, hslots, wmeta, kmeta, ls, ne, lcands, entries, fpar, ctl, args;
    DevBuf bin, steps, offs, bout, cur, t0, bdev, launch;
    DevBuf h_bin, h_steps, h_offs, h_bout, h_args, h_bdev, h_launch;
    std::vector<u32> gen;          // each slot's hash-set generation after the last call
    ltlg_engine *fallback = nullptr;
    std::vector<float> scorer;     // set_scorer's parameters, for the fallback engine
};

namespace {

int batch_fallback(ltlg_batch *b, const ltlg_traces *t, const ltlg_options *opt, ltlg_result *res) {
    if (!b->fallback) {
        const int rc = ltlg_engine_create(&b->cfg, &b->fallback);
        if (rc != 0) {
            memset(res, 0, sizeof(*res));
            return fail_status(res, rc);
        }
        if (!b->scorer.empty()) ltlg_engine_set_scorer(b->fallback, b->scorer.data(), (int32_t)b->scorer.size());
    }
    return ltlg_engine_learn(b->fallback, t, opt, res);
}

}  // namespace

LTLG_API int ltlg_batch_create(const ltlg_engine_config *cfg_in, int32_t workers, ltlg_batch **out) {
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LTLG_NO_DEVICE;
    if (workers < 1 || workers > 4096) return LTLG_BAD_ARGS;
    ltlg_engine_config cfg;
    if (cfg_in)
        cfg = *cfg_in;
    else
        ltlg_default_engine_config(&cfg);
    if (cfg.device < 0 || cfg.device >= ndev || cfg.slots_log2 < 10 || cfg.slots_log2 > 34 ||
        (cfg.left_tile != 2 && cfg.left_tile != 4 && cfg.left_tile != 8) || cfg.right_chunk < 1 ||
        cfg.unary_rows < 1 || cfg.max_traces < 1 || cfg.wait_spins < 0 || cfg.small_level < 0 || cfg.cache_bytes < 64)
        return LTLG_BAD_ARGS;
    if (cfg.max_rows <= 0 || cfg.max_rows > (1ll << 30) - 1) cfg.max_rows = (1ll << 30) - 1;
    auto *b = new ltlg_batch();
    b->cfg = cfg;
    b->slots = workers;
    b->gen.assign(workers, 0u);
    cudaError_t err = cudaSetDevice(cfg.device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, cfg.device);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    const size_t nslots = (size_t)1 << cfg.slots_log2;
    const size_t cache_words = (size_t)cfg.cache_bytes / 8;
    if (err == cudaSuccess) err = ensure(b->cache, (size_t)workers * cache_words * 8);
    if (err == cudaSuccess) err = ensure(b->hslots, (size_t)workers * nslots * 8);
    if (err == cudaSuccess) err = cudaMemsetAsync(b->hslots.p, 0, (size_t)workers * nslots * 8, b->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(b->stream);
    if (err != cudaSuccess) {
        ltlg_batch_destroy(b);
        return err == cudaErrorMemoryAllocation ? LTLG_NO_MEMORY : LTLG_CUDA_ERROR;
    }
    *out = b;
    return 0;
}

LTLG_API void ltlg_batch_destroy(ltlg_batch *b) {
    if (!b) return;
    cudaSetDevice(b->cfg.device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (DevBuf *x : {&b->cache, &b->parents, &b->keys, &b->hslots, &b->wmeta, &b->kmeta, &b->ls, &b->ne, &b->lcands,
                      &b->entries, &b->fpar, &b->ctl, &b->args, &b->bin, &b->steps, &b->offs, &b->bout, &b->cur,
                      &b->t0, &b->bdev, &b->launch})
        if (x->p) cudaFree(x->p);
    for (DevBuf *x : {&b->h_bin, &b->h_steps, &b->h_offs, &b->h_bout, &b->h_args, &b->h_bdev, &b->h_launch})
        if (x->p) cudaFreeHost(x->p);
    if (b->stream) cudaStreamDestroy(b->stream);
    ltlg_engine_destroy(b->fallback);
    delete b;
}

LTLG_API void *ltlg_batch_stream(ltlg_batch *b, int32_t worker) {
    if (!b || worker != 0) return nullptr;
    return (void *)b->stream;
}

LTLG_API int ltlg_batch_learn(ltlg_batch *b, const ltlg_traces *traces, int32_t count, const ltlg_options *opt,
                              ltlg_result *results) {
    if (!b || count < 0 || (count && (!traces || !results || !opt))) return LTLG_BAD_ARGS;
    const double t0 = now_s();
    for (int i = 0; i < count; ++i) memset(&results[i], 0, sizeof(ltlg_result));
    const int *cf = opt ? opt->cost_fun : nullptr;
    bool opts_ok = opt != nullptr && opt->max_cost >= 1 && opt->max_cost <= SHRT_MAX && opt->key_mode >= 0 &&
                   opt->key_mode <= 2 && (opt->order == LTLG_ORDER_PLAIN || opt->order == LTLG_ORDER_LEARNED);
    for (int i = 0; opts_ok && i < 8; ++i)
        if (cf[i] <= 0 || cf[i] > SHRT_MAX) opts_ok = false;
    if (count && !opts_ok) {
        for (int i = 0; i < count; ++i) fail_status(&results[i], LTLG_BAD_ARGS);
        return LTLG_BAD_ARGS;
    }
    const bool device_batch = count > 0 && opt->key_mode != LTLG_KEY_REF && opt->order == LTLG_ORDER_PLAIN &&
                              opt->schedule == LTLG_SCHEDULE_FUSED && opt->time_limit_s <= 0;
    // which instances the device takes; the others are answered on the host or by the fallback
    std::vector<int> dev_idx;
    int min_pitch = INT_MAX, max_pitch = 4;
    for (int i = 0; i < count; ++i) {
        const ltlg_traces *t = &traces[i];
        ltlg_result *r = &results[i];
        const int n = t->num_pos + t->num_neg;
        const int nalpha = t->alphabet ? (int)strlen(t->alphabet) : 0;
        if (!traces_well_formed(t) || n > b->cfg.max_traces || nalpha > 26) {
            fail_status(r, LTLG_BAD_ARGS);
            continue;
        }
        int max_len = 0;
        for (int q = 0; q < n; ++q) max_len = std::max(max_len, t->offsets[q + 1] - t->offsets[q]);
        if ((opt->limit_traces && n > 64) || max_len > 63) {
            r->status = LTLG_INPUT_LIMITS;
            r->cost = cf[0];
            r->formula = strdup("see_the_error");
            continue;
        }
        if (!device_batch) {
            batch_fallback(b, t, opt, r);
            continue;
        }
        const int pitch = std::max(4, (n + 3) & ~3);
        min_pitch = std::min(min_pitch, pitch);
        max_pitch = std::max(max_pitch, pitch);
        dev_idx.push_back(i);
    }
    const int nd = (int)dev_idx.size();
    cudaError_t err = cudaSuccess;
    if (nd > 0) {
        err = cudaSetDevice(b->cfg.device);
        const int K = std::min(b->slots, nd);
        const int max_cost = opt->max_cost;
        const long long ncost = (long long)max_cost + 3;
        const long long cap_entries = entries_for(max_cost);
        const long long cache_words = b->cfg.cache_bytes / 8;
        const long long max_rows = std::min<long long>(b->cfg.max_rows, cache_words / min_pitch);
        const bool keyed = opt->key_mode != LTLG_KEY_EXACT;
        const int hk = opt->key_mode == LTLG_KEY_HASH64 ? 1 : 0;
        int tile = 0, stages = 0;
        long long tile_bytes = 0;
        if (!geometry(b->cfg.left_tile, max_pitch, tile, stages, tile_bytes)) err = cudaErrorInvalidValue;
        const int per_sm =
            err == cudaSuccess ? level_kernel_ctas_per_sm(hk, level_kernel_smem(stages, tile_bytes)) : 0;
        if (per_sm < 1 && err == cudaSuccess) err = cudaErrorInvalidConfiguration;
        const int grid = b->num_sms * std::max(per_sm, 1);
        // inputs: instance records, steps and offsets of every instance in one array each
        long long total_steps = 0, total_offs = 0;
        for (int i : dev_idx) {
            const ltlg_traces *t = &traces[i];
            const int n = t->num_pos + t->num_neg;
            total_steps += n ? t->offsets[n] - t->offsets[0] : 0;
            total_offs += n + 1;
        }
        const size_t bout_bytes = (size_t)nd * sizeof(BatchOut);
        auto dev = [&](DevBuf &x, size_t bytes) {
            if (err == cudaSuccess) err = ensure(x, std::max<size_t>(bytes, 16));
        };
        auto host = [&](DevBuf &x, size_t bytes) {
            if (err == cudaSuccess) err = ensure_host(x, std::max<size_t>(bytes, 16));
        };
        dev(b->parents, (size_t)K * max_rows * 8);
        if (keyed) dev(b->keys, (size_t)K * max_rows * 16);
        dev(b->wmeta, (size_t)K * max_pitch * 8);
        dev(b->kmeta, (size_t)K * max_pitch * 4);
        dev(b->ls, (size_t)K * ncost * 8);
        dev(b->lcands, (size_t)K * ncost * 8);
        dev(b->ne, (size_t)K * ncost * 4);
        dev(b->entries, (size_t)K * 2 * cap_entries * sizeof(Entry));
        dev(b->fpar, (size_t)K * cap_entries * 8);
        dev(b->ctl, (size_t)K * sizeof(InstCtl));
        dev(b->args, (size_t)K * sizeof(InstArgs));
        dev(b->cur, (size_t)K * 4);
        dev(b->t0, (size_t)K * 8);
        dev(b->bin, (size_t)nd * sizeof(BatchIn));
        dev(b->steps, (size_t)total_steps * 4);
        dev(b->offs, (size_t)total_offs * 4);
        dev(b->bout, bout_bytes);
        dev(b->bdev, sizeof(BatchDev));
        dev(b->launch, sizeof(Launch));
        host(b->h_bin, (size_t)nd * sizeof(BatchIn));
        host(b->h_steps, (size_t)total_steps * 4);
        host(b->h_offs, (size_t)total_offs * 4);
        host(b->h_bout, bout_bytes);
        host(b->h_args, (size_t)K * sizeof(InstArgs));
        host(b->h_bdev, sizeof(BatchDev));
        host(b->h_launch, sizeof(Launch));
        if (err == cudaSuccess) {
            BatchIn *bi = (BatchIn *)b->h_bin.p;
            u32 *hs = (u32 *)b->h_steps.p;
            int *ho = (int *)b->h_offs.p;
            long long sp = 0, op = 0;
            for (int q = 0; q < nd; ++q) {
                const ltlg_traces *t = &traces[dev_idx[q]];
                const int n = t->num_pos + t->num_neg;
                BatchIn &x = bi[q];
                memset(&x, 0, sizeof(x));
                x.npos = t->num_pos;
                x.nneg = t->num_neg;
                x.nalpha = t->alphabet ? (int)strlen(t->alphabet) : 0;
                if (x.nalpha) memcpy(x.alpha, t->alphabet, (size_t)x.nalpha);
                x.steps0 = sp;
                x.offs0 = op;
                const int base = n ? t->offsets[0] : 0;
                for (int k = 0; k <= n; ++k) ho[op + k] = n ? t->offsets[k] - base : 0;
                const long long ns = n ? t->offsets[n] - base : 0;
                if (ns) memcpy(hs + sp, t->steps + base, (size_t)ns * 4);
                sp += ns;
                op += n + 1;
            }
            // slot arguments: the slot's buffers and the learn's options (set-up fills the rest)
            InstArgs *ha = (InstArgs *)b->h_args.p;
            const u64 nslots = 1ull << b->cfg.slots_log2;
            for (int s2 = 0; s2 < K; ++s2) {
                InstArgs &A = ha[s2];
                memset(&A, 0, sizeof(A));
                A.key_mode = keyed ? KEY_HASH64 : KEY_EXACT;
                A.stop_at_found = opt->stop_at_found ? 1 : 0;
                A.neg_type = opt->neg_type;
                A.max_cost = max_cost;
                for (int q = 0; q < 8; ++q) A.cf[q] = cf[q];
                A.right_chunk_big = b->cfg.right_chunk;
                A.unary_rows_big = b->cfg.unary_rows;
                A.small_rows = std::max(1, b->cfg.small_rows);
                A.tile = tile;
                A.gen = b->gen[s2];
                A.small_level = b->cfg.small_level > 0 ? b->cfg.small_level : LLONG_MAX / 2;
                A.wait_spins = b->cfg.wait_spins > 0 ? b->cfg.wait_spins : (1ll << 22);
                A.cap_entries = cap_entries;
                A.learn_min_items = (long long)grid * stages;
                A.item_target = (long long)grid * stages * 2;
                A.slot_mask = nslots - 1;
                A.cache = (u64 *)b->cache.p + (size_t)s2 * cache_words;
                A.parents = (u64 *)b->parents.p + (size_t)s2 * max_rows;
                A.keys = keyed ? (u64 *)b->keys.p + (size_t)s2 * max_rows * 2 : nullptr;
                A.slots = (u64 *)b->hslots.p + (size_t)s2 * nslots;
                A.wmeta = (const u64 *)b->wmeta.p + (size_t)s2 * max_pitch;
                A.kmeta = (const u32 *)b->kmeta.p + (size_t)s2 * max_pitch;
                A.ls = (long long *)b->ls.p + (size_t)s2 * ncost;
                A.ne = (int *)b->ne.p + (size_t)s2 * ncost;
                A.level_cands = (u64 *)b->lcands.p + (size_t)s2 * ncost;
                A.entries = (Entry *)b->entries.p + (size_t)s2 * 2 * cap_entries;
                A.found_par = (u64 *)b->fpar.p + (size_t)s2 * cap_entries;
                A.ctl = (InstCtl *)b->ctl.p + s2;
            }
            BatchDev &D = *(BatchDev *)b->h_bdev.p;
            memset(&D, 0, sizeof(D));
            D.in = (const BatchIn *)b->bin.p;
            D.steps = (const u32 *)b->steps.p;
            D.offs = (const int *)b->offs.p;
            D.out = (BatchOut *)b->bout.p;
            D.args = (InstArgs *)b->args.p;
            D.cur = (int *)b->cur.p;
            D.t0 = (u64 *)b->t0.p;
            D.cache_words = cache_words;
            D.max_rows = max_rows;
            D.count = nd;
            D.nslots = K;
            D.max_pitch = max_pitch;
            Launch &L = *(Launch *)b->h_launch.p;
            memset(&L, 0, sizeof(L));
            L.args = (const InstArgs *)b->args.p;
            L.batch = (BatchDev *)b->bdev.p;
            L.ninst = K;
            L.persist = 1;
            L.tile = tile;
            L.stages = stages;
            L.tile_bytes = tile_bytes;
            cudaStream_t st = b->stream;
            err = cudaMemcpyAsync(b->bin.p, b->h_bin.p, (size_t)nd * sizeof(BatchIn), cudaMemcpyHostToDevice, st);
            if (err == cudaSuccess && total_steps)
                err = cudaMemcpyAsync(b->steps.p, b->h_steps.p, (size_t)total_steps * 4, cudaMemcpyHostToDevice, st);
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(b->offs.p, b->h_offs.p, (size_t)total_offs * 4, cudaMemcpyHostToDevice, st);
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(b->args.p, ha, (size_t)K * sizeof(InstArgs), cudaMemcpyHostToDevice, st);
            if (err == cudaSuccess) err = cudaMemsetAsync(b->ctl.p, 0, (size_t)K * sizeof(InstCtl), st);
            if (err == cudaSuccess) err = cudaMemcpyAsync(b->bdev.p, &D, sizeof(BatchDev), cudaMemcpyHostToDevice, st);
            if (err == cudaSuccess) err = cudaMemcpyAsync(b->launch.p, &L, sizeof(Launch), cudaMemcpyHostToDevice, st);
            if (err == cudaSuccess) err = launch_batch_start((BatchDev *)b->bdev.p, K, hk, st);
            if (err == cudaSuccess) err = launch_levels(L, (const Launch *)b->launch.p, grid, hk, st);
            if (err == cudaSuccess) err = cudaMemcpyAsync(b->h_bout.p, b->bout.p, bout_bytes, cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(ha, b->args.p, (size_t)K * sizeof(InstArgs), cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess) err = cudaStreamSynchronize(st);
            if (err == cudaSuccess)
                for (int s2 = 0; s2 < K; ++s2) b->gen[s2] = ha[s2].gen;
        }
        // results
        const BatchOut *bo = (const BatchOut *)b->h_bout.p;
        const double wall = now_s() - t0;
        for (int q = 0; q < nd; ++q) {
            const int i = dev_idx[q];
            ltlg_result *r = &results[i];
            if (err != cudaSuccess) {
                r->status = LTLG_CUDA_ERROR;
                r->formula = strdup(cudaGetErrorString(err));
                continue;
            }
            const BatchOut &o = bo[q];
            if (o.status == LTLG_NO_MEMORY) {  // its slot's cache overflowed: learn it alone
                batch_fallback(b, &traces[i], opt, r);
                continue;
            }
            const std::string alpha = traces[i].alphabet ? traces[i].alphabet : "";
            r->status = o.status;
            r->cost = o.cost;
            r->all_ltls = o.all_ltls;
            r->evaluated = o.evaluated;
            r->rows = o.rows;
            r->device_flags = o.device_flags;
            r->device_ms = (double)o.ns * 1e-6;
            r->seconds = wall;
            r->launches = 2;
            std::string formula;
            if (o.letter >= 0 && o.letter < (int)alpha.size()) {
                formula = std::string(1, alpha[o.letter]);
                r->found_op = OP_ATOM;
            } else if (o.status == LTLG_FOUND && o.found) {
                r->found_op = parent_op(o.found & ~(1ull << 63));
                if (o.walk_overflow || o.walk_count - 1 >= 200) {
                    formula = "Size of the output is too big";
                } else {
                    std::map<u64, u64> par;
                    for (int k = 1; k < o.walk_count; ++k) par[o.walk[2 * k]] = o.walk[2 * k + 1];
                    build_string(par, ~0ull, o.found & ~(1ull << 63), true, alpha, (int)alpha.size(), formula, 0);
                }
            } else {
                formula = ltlg_status_string(o.status);
            }
            r->formula = strdup(formula.c_str());
        }
    }
    int rc = err != cudaSuccess ? LTLG_CUDA_ERROR : 0;
    for (int i = 0; i < count && !rc; ++i)
        if (results[i].status != LTLG_FOUND && results[i].status != LTLG_NOT_FOUND) rc = results[i].status;
    return rc;
}

LTLG_API int ltlg_batch_set_scorer(ltlg_batch *b, const float *params, int32_t count) {
    if (!b || !params || count != MLP_PARAMS) return LTLG_BAD_ARGS;
    b->scorer.assign(params, params + count);
    if (b->fallback) return ltlg_engine_set_scorer(b->fallback, params, count);
    return 0;
}

LTLG_API int ltlg_engine_read_rows(ltlg_engine *e, int64_t first, int64_t count, uint64_t *rows, uint64_t *parents) {
    if (!e || first < 0 || count < 0 || first + count > e->cap_rows) return LTLG_BAD_ARGS;
    if (count == 0) return 0;
    cudaSetDevice(e->cfg.device);
    cudaError_t err = cudaSuccess;
    if (rows) {
        std::vector<u64> tmp((size_t)count * e->pitch);
        err = cudaMemcpy(tmp.data(), (u64 *)e->cache.p + (size_t)first * e->pitch, tmp.size() * 8,
                         cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) return fail_cuda(e, err, nullptr);
        for (int64_t r = 0; r < count; ++r)
            memcpy(rows + (size_t)r * e->n, tmp.data() + (size_t)r * e->pitch, (size_t)e->n * 8);
    }
    if (parents) {
        err = cudaMemcpy(parents, (u64 *)e->parents.p + first, (size_t)count * 8, cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) return fail_cuda(e, err, nullptr);
    }
    return 0;
}

LTLG_API int ltlg_engine_level_starts(ltlg_engine *e, int64_t *starts, int32_t count) {
    if (!e || !starts || count < 0) return LTLG_BAD_ARGS;
    for (int32_t i = 0; i < count; ++i)
        starts[i] = i < (int32_t)e->level_start.size() ? e->level_start[i] : (e->level_start.empty() ? 0 : e->level_start.back());
    return 0;
}

LTLG_API int ltlg_engine_hold_slot(ltlg_engine *e, const uint64_t *cs, int32_t n) {
    if (!e || !cs || n <= 0 || n > e->cfg.max_traces) return LTLG_BAD_ARGS;
    cudaError_t err = cudaSetDevice(e->cfg.device);
    if (err != cudaSuccess) return fail_cuda(e, err, nullptr);
    const int pitch = std::max(4, (n + 3) & ~3);
    const u64 fp = host_fingerprint_exact(cs, n, pitch);
    if (e->gen >= 255) {  // the next learn would clear the set; clear it here instead
        err = cudaMemsetAsync(e->slots.p, 0, e->nslots * 8, e->stream);
        if (err != cudaSuccess) return fail_cuda(e, err, nullptr);
        e->gen = 0;
    }
    // tag | the next learn's generation | "publication pending"
    static thread_local u64 v;
    v = ((fp >> 40) << 40) | ((u64)(e->gen + 1) << 32) | 0xFFFFFFFFull;
    u64 *slot = (u64 *)e->slots.p + (fp & (e->nslots - 1));
    err = cudaMemcpyAsync(slot, &v, sizeof(v), cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    return err == cudaSuccess ? 0 : fail_cuda(e, err, nullptr);
}

LTLG_API int ltlg_device_apply_op(int32_t op, const uint64_t *a, const uint64_t *b, const uint64_t *lenmask,
                                  int32_t n, int32_t count, uint64_t *out, uint64_t *out2, uint64_t *fp) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LTLG_NO_DEVICE;
    if (op < 0 || op > 6 || n <= 0 || count <= 0) return LTLG_BAD_ARGS;
    const int pitch = (n + 3) & ~3;
    std::vector<u64> ha((size_t)count * pitch, 0), hb((size_t)count * pitch, 0), hm(pitch, 0);
    for (int r = 0; r < count; ++r)
        for (int i = 0; i < n; ++i) {
            ha[(size_t)r * pitch + i] = a[(size_t)r * n + i];
            if (b) hb[(size_t)r * pitch + i] = b[(size_t)r * n + i];
        }
    for (int i = 0; i < n; ++i) hm[i] = lenmask[i] & 0x7FFFFFFFFFFFFFFFull;
    u64 *da = nullptr, *db = nullptr, *dm = nullptr, *dout = nullptr, *dout2 = nullptr, *dfp = nullptr;
    const size_t rb = (size_t)count * pitch * 8;
    cudaError_t err = cudaMalloc(&da, rb);
    if (err == cudaSuccess) err = cudaMalloc(&db, rb);
    if (err == cudaSuccess) err = cudaMalloc(&dm, (size_t)pitch * 8);
    if (err == cudaSuccess) err = cudaMalloc(&dout, rb);
    if (err == cudaSuccess) err = cudaMalloc(&dout2, rb);
    if (err == cudaSuccess) err = cudaMalloc(&dfp, (size_t)count * 16);
    if (err == cudaSuccess) err = cudaMemcpy(da, ha.data(), rb, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(db, hb.data(), rb, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dm, hm.data(), (size_t)pitch * 8, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = launch_apply_op(op, da, b ? db : nullptr, dm, n, pitch, count, dout, dout2, dfp, 0);
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    if (err == cudaSuccess) {
        std::vector<u64> ho((size_t)count * pitch), ho2((size_t)count * pitch), hf((size_t)count * 2);
        cudaMemcpy(ho.data(), dout, rb, cudaMemcpyDeviceToHost);
        cudaMemcpy(ho2.data(), dout2, rb, cudaMemcpyDeviceToHost);
        cudaMemcpy(hf.data(), dfp, (size_t)count * 16, cudaMemcpyDeviceToHost);
        for (int r = 0; r < count; ++r)
            for (int i = 0; i < n; ++i) {
                out[(size_t)r * n + i] = ho[(size_t)r * pitch + i];
                if (out2) out2[(size_t)r * n + i] = ho2[(size_t)r * pitch + i];
            }
        for (int r = 0; r < count; ++r) {
            fp[r] = hf[r];
            if (out2) fp[count + r] = hf[count + r];
        }
    }
    for (u64 *p : {da, db, dm, dout, dout2, dfp})
        if (p) cudaFree(p);
    return err == cudaSuccess ? 0 : LTLG_CUDA_ERROR;
}

LTLG_API int ltlg_read_scarlet(const char *path, ltlg_traces *out) {
    memset(out, 0, sizeof(*out));
    ScarletMasks f;
    if (!path || !read_scarlet_masks(path, f)) return LTLG_BAD_ARGS;
    const std::vector<uint32_t> &steps = f.steps;
    const std::vector<int32_t> &offsets = f.offsets;
    uint32_t *s = (uint32_t *)malloc(std::max<size_t>(steps.size(), 1) * 4);
    int32_t *o = (int32_t *)malloc(offsets.size() * 4);
    char *a = strdup(f.sorted_alphabet.c_str());
    if (!s || !o || !a) {
        free(s);
        free(o);
        free(a);
        return LTLG_NO_MEMORY;
    }
    if (!steps.empty()) memcpy(s, steps.data(), steps.size() * 4);
    memcpy(o, offsets.data(), offsets.size() * 4);
    out->num_pos = f.num_pos;
    out->num_neg = f.num_neg;
    out->alphabet = a;
    out->steps = s;
    out->offsets = o;
    return 0;
}

LTLG_API void ltlg_traces_free(ltlg_traces *t) {
    if (!t) return;
    free((void *)t->alphabet);
    free((void *)t->steps);
    free((void *)t->offsets);
    memset(t, 0, sizeof(*t));
}

}  // extern "C"
