// Host side of the enumerator: the C ABI of include/ltlgpu.h.
//
// ltlg_engine_learn restates LTLI (code/ltli6463.cu:1043-1497) for the GPU path:
//   letters and the early letter hit ........ :1058-1136
//   level / operator / split order ........... :1199-1445 (NegType rule :1212)
//   on-the-fly overflow regime ............... :1021-1027, :1202-1206, :1442-1443
//   found -> formula string, 200-node limit .. :877-991
// The per-chunk host round trips of the reference are gone: a level is one launch
// (or one launch per block in the per-block schedule), and the host reads a small
// control record once per level.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <thread>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
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

const char OPCH[7] = {'~', '&', '|', 'X', 'F', 'G', 'U'};

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

}  // namespace

struct ltlg_engine {
    ltlg_engine_config cfg{};
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    static constexpr int RING = 4;     // levels in flight: the host runs up to RING - 1 ahead
    cudaEvent_t ev_start[RING] = {}, ev_done[RING] = {};
    cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    DevBuf cache, parents, keys, slots, wmeta, kmeta, ctl, walk, snaps, lev, ls, lcands, args;
    // One graph per ring slot: planner, level kernel, and the copy of the level's control
    // block and plan header into that slot.  The kernels read their
    // arguments from `args`, so the graphs stay valid from one learn to the next; they are
    // captured again only when the kernel instances or grids change (graph_key).
    cudaGraphExec_t level_graph[RING] = {};
    void *ring_dev = nullptr;       // device view of h_ring
    DevBuf scorer, scorer_params;   // the learned block order's scorer (MlpDev, packed FP32)
    DevBuf lstats, h_lstats;        // row statistics per cost (LSTATS counters)
    bool has_scorer = false;
    long long graph_key[8] = {};
    DevBuf h_ctl, h_walk, h_stage, h_snaps, h_args, h_lev, h_ls, h_lcands, h_win, h_ring;

    u64 nslots = 0;
    u32 gen = 0;
    // last learn
    int n = 0, pitch = 0, nalpha = 0;
    long long cap_rows = 0;
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

struct Block {
    int op, lcost, rcost;
    long long l0, l1, r0, r1;
    long long candidates;  // as the reference counts them (U: 2 per pair)
};

// Blocks of cost c in the reference's order (ltli6463.cu:1209-1440).
std::vector<Block> level_blocks(int c, const int *cf, int neg_type, const std::vector<long long> &ls) {
    const int c1 = cf[0];
    auto lo = [&](int k) { return (k >= 0 && k + 1 < (int)ls.size()) ? ls[k] : 0ll; };
    auto hi = [&](int k) { return (k >= 0 && k + 1 < (int)ls.size()) ? ls[k + 1] : 0ll; };
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

// The window of block (op, k) in a host copy of a plan: items [lo, hi) of the level's item
// table (unary blocks must be unfused, one per operator).
void block_window(const DevLevel *hl, int op, int k, long long &lo, long long &hi) {
    const bool un = op == OP_NEG || op == OP_X || op == OP_F || op == OP_G;
    for (int r = 0; r < hl->nranges; ++r) {
        const ItemRange &R = hl->ranges[r];
        if (un ? (R.cls == 1 && hl->ublocks[R.idx].op == op) : (R.cls != 1 && R.idx == op * MAX_SPLITS + k)) {
            lo = R.item0;
            hi = r + 1 < hl->nranges ? hl->ranges[r + 1].item0 : hl->items_end;
            return;
        }
    }
    lo = hi = 0;
}

int cost_of_row(const std::vector<long long> &ls, long long row) {
    // ls[k] .. ls[k + 1] are the rows of cost k
    for (int k = (int)ls.size() - 2; k >= 0; --k)
        if (row >= ls[k] && row < ls[k + 1]) return k;
    return -1;
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
    c->block_threads = 256;
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
    if (cfg.block_threads < 32 || cfg.block_threads > 256 || cfg.block_threads % 32) return LTLG_BAD_ARGS;
    if (cfg.right_chunk < 1 || cfg.unary_rows < 1 || cfg.max_traces < 1 || cfg.wait_spins < 0 ||
        cfg.small_level < 0)
        return LTLG_BAD_ARGS;
    if (cfg.max_rows <= 0 || cfg.max_rows > (1ll << 30) - 1) cfg.max_rows = (1ll << 30) - 1;
    auto *e = new ltlg_engine();
    e->cfg = cfg;
    cudaError_t err = cudaSetDevice(cfg.device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, cfg.device);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    for (int k = 0; k < ltlg_engine::RING && err == cudaSuccess; ++k) {
        err = cudaEventCreate(&e->ev_start[k]);
        if (err == cudaSuccess) err = cudaEventCreate(&e->ev_done[k]);
    }
    if (err == cudaSuccess) err = cudaEventCreate(&e->ev_a);
    if (err == cudaSuccess) err = cudaEventCreate(&e->ev_b);
    if (err == cudaSuccess) err = cudaEventCreate(&e->ev_t0);
    if (err == cudaSuccess) err = cudaEventCreate(&e->ev_t1);
    e->nslots = 1ull << cfg.slots_log2;
    if (err == cudaSuccess) err = ensure(e->slots, e->nslots * 8);
    if (err == cudaSuccess) err = cudaMemsetAsync(e->slots.p, 0, e->nslots * 8, e->stream);
    if (err == cudaSuccess) err = ensure(e->cache, (size_t)cfg.cache_bytes);
    if (err == cudaSuccess) err = ensure(e->ctl, sizeof(DevCtl));
    if (err == cudaSuccess) err = ensure_host(e->h_ctl, sizeof(DevCtl));
    if (err == cudaSuccess) err = ensure(e->walk, (2 + 2 * 1024) * 8);
    if (err == cudaSuccess) err = ensure_host(e->h_walk, (2 + 2 * 1024) * 8);
    const size_t max_blocks = 7 * MAX_SPLITS;
    if (err == cudaSuccess) err = ensure(e->snaps, max_blocks * sizeof(DevCtl));
    if (err == cudaSuccess) err = ensure_host(e->h_snaps, max_blocks * sizeof(DevCtl));
    if (err == cudaSuccess) err = ensure_host(e->h_win, max_blocks * 8 * sizeof(long long));
    if (err == cudaSuccess) err = ensure_host(e->h_args, sizeof(LevelArgs));
    if (err == cudaSuccess) err = ensure(e->args, sizeof(LevelArgs));
    if (err == cudaSuccess) err = ensure(e->lstats, (MAX_COSTS + 2) * LSTATS * sizeof(u64));
    if (err == cudaSuccess) err = ensure_host(e->h_lstats, (MAX_COSTS + 2) * LSTATS * sizeof(u64));
    if (err == cudaSuccess) {  // the ring of level summaries: mapped, the level kernel writes it
        err = cudaHostAlloc(&e->h_ring.p, ltlg_engine::RING * (sizeof(DevCtl) + sizeof(DevLevel)), cudaHostAllocMapped);
        if (err == cudaSuccess) {
            e->h_ring.bytes = ltlg_engine::RING * (sizeof(DevCtl) + sizeof(DevLevel));
            memset(e->h_ring.p, 0, e->h_ring.bytes);
            err = cudaHostGetDevicePointer(&e->ring_dev, e->h_ring.p, 0);
        }
    }
    if (err == cudaSuccess) err = ensure(e->lev, sizeof(DevLevel));
    if (err == cudaSuccess) err = ensure_host(e->h_lev, sizeof(DevLevel));
    if (err == cudaSuccess) err = ensure(e->ls, (MAX_COSTS + 2) * sizeof(long long));
    if (err == cudaSuccess) err = ensure_host(e->h_ls, (MAX_COSTS + 2) * sizeof(long long));
    if (err == cudaSuccess) err = ensure(e->lcands, (MAX_COSTS + 2) * sizeof(u64));
    if (err == cudaSuccess) err = ensure_host(e->h_lcands, (MAX_COSTS + 2) * sizeof(u64));
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
    for (cudaGraphExec_t g : e->level_graph)
        if (g) cudaGraphExecDestroy(g);
    for (DevBuf *b : {&e->cache, &e->parents, &e->keys, &e->slots, &e->wmeta, &e->kmeta, &e->ctl, &e->walk, &e->snaps,
                      &e->lev, &e->ls, &e->lcands, &e->args, &e->scorer, &e->scorer_params, &e->lstats})
        if (b->p) cudaFree(b->p);
    for (DevBuf *b : {&e->h_ctl, &e->h_walk, &e->h_stage, &e->h_snaps, &e->h_args, &e->h_lev, &e->h_ls, &e->h_lcands,
                      &e->h_win, &e->h_ring, &e->h_lstats})
        if (b->p) cudaFreeHost(b->p);
    for (cudaEvent_t ev : {e->ev_a, e->ev_b, e->ev_t0, e->ev_t1})
        if (ev) cudaEventDestroy(ev);
    for (int k = 0; k < ltlg_engine::RING; ++k)
        for (cudaEvent_t ev : {e->ev_start[k], e->ev_done[k]})
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

LTLG_API int ltlg_engine_learn(ltlg_engine *e, const ltlg_traces *t, const ltlg_options *opt, ltlg_result *res) {
    memset(res, 0, sizeof(*res));
    const double t0 = now_s();
    if (!e || !t || !opt) {
        res->status = LTLG_BAD_ARGS;
        res->formula = strdup("bad_arguments");
        return res->status;
    }
    const int *cf = opt->cost_fun;
    for (int i = 0; i < 8; ++i)
        if (cf[i] <= 0 || cf[i] > SHRT_MAX) {
            res->status = LTLG_BAD_ARGS;
            res->formula = strdup("bad_arguments");
            return res->status;
        }
    const int c1 = cf[0];
    const int npos = t->num_pos, nneg = t->num_neg, n = npos + nneg;
    const std::string alpha = t->alphabet ? t->alphabet : "";
    const int nalpha = (int)alpha.size();
    const bool ref_keys = opt->key_mode == LTLG_KEY_REF;
    if (!traces_well_formed(t) || (ref_keys && (opt->rlx_unq_chk_type < 1 || opt->rlx_unq_chk_type > 3)) ||
        opt->key_mode < 0 || opt->key_mode > 2 || n > e->cfg.max_traces || nalpha > 26 ||
        (opt->order != LTLG_ORDER_PLAIN && opt->order != LTLG_ORDER_LEARNED) ||
        (opt->order == LTLG_ORDER_LEARNED && !e->has_scorer)) {
        res->status = LTLG_BAD_ARGS;
        res->formula = strdup("bad_arguments");
        return res->status;
    }
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
    e->n = n;
    e->pitch = pitch;
    e->nalpha = nalpha;
    const long long cap_rows =
        std::min<long long>(e->cfg.max_rows, e->cfg.cache_bytes / ((long long)pitch * 8ll));
    e->cap_rows = cap_rows;
    const int max_cost = opt->max_cost;
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
        res->formula = strdup(letter_hit >= 0 ? std::string(1, alpha[letter_hit]).c_str() : "not_found");
        res->seconds = now_s() - t0;
        return res->status;
    }
    if (cap_rows < nalpha + 1) {
        res->status = LTLG_NO_MEMORY;
        res->formula = strdup("no_memory");
        return res->status;
    }

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

    // Buffers
    if ((err = ensure(e->parents, (size_t)cap_rows * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if (opt->key_mode != LTLG_KEY_EXACT && (err = ensure(e->keys, (size_t)cap_rows * 16)) != cudaSuccess)
        return fail_cuda(e, err, res);
    if ((err = ensure(e->wmeta, (size_t)pitch * 8)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure(e->kmeta, (size_t)pitch * 4)) != cudaSuccess) return fail_cuda(e, err, res);
    if ((err = ensure_host(e->h_stage, std::max<size_t>((size_t)nalpha * pitch * 8, (size_t)pitch * 12))) !=
        cudaSuccess)
        return fail_cuda(e, err, res);
    cudaStream_t st = e->stream;
    // staging: letters, then wmeta, then kmeta (synchronised before reuse)
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
    DevCtl *hc = (DevCtl *)e->h_ctl.p;
    memset(hc, 0, sizeof(DevCtl));
    hc->row_count = (u64)nalpha;
    cudaMemcpyAsync(e->ctl.p, hc, sizeof(DevCtl), cudaMemcpyHostToDevice, st);

    int tl = e->cfg.left_tile;
    // shrink the left tile until three CTAs fit an SM's shared memory (long CS rows)
    while (tl > 2 && 3 * (size_t)level_kernel_smem_bytes(tl, pitch) > 200 * 1024) tl /= 2;
    if ((size_t)level_kernel_smem_bytes(tl, pitch) > 220 * 1024) {
        res->status = LTLG_BAD_ARGS;
        res->formula = strdup("bad_arguments");
        return res->status;
    }
    const int hk = opt->key_mode == LTLG_KEY_HASH64 ? 1 : 0;
    const int block_threads = e->cfg.block_threads;
    // resident CTAs of the level kernel on all SMs
    const long long max_grid =
        (long long)e->num_sms * std::max(1, level_kernel_max_ctas_per_sm(tl, hk, block_threads, pitch));

    // Arguments and plan in device memory.
    DevLevel *dlev = (DevLevel *)e->lev.p;
    LevelArgs *ha = (LevelArgs *)e->h_args.p;
    memset(ha, 0, sizeof(LevelArgs));
    LevelArgs &A = *ha;
    A.n = n;
    A.pitch = pitch;
    A.npos = npos;
    A.nalpha = nalpha;
    A.key_mode = opt->key_mode == LTLG_KEY_EXACT ? KEY_EXACT : opt->key_mode == LTLG_KEY_REF ? KEY_REF : KEY_HASH64;
    A.rlx_type = rlx_type;
    A.gen = e->gen;
    A.stop_at_found = opt->stop_at_found ? 1 : 0;
    A.left_tile = tl;
    A.neg_type = opt->neg_type;
    A.max_cost = max_cost;
    A.nwarps = block_threads / 32;
    for (int i = 0; i < 8; ++i) A.cf[i] = cf[i];
    A.right_chunk_big = e->cfg.right_chunk;
    A.unary_rows_big = e->cfg.unary_rows;
    A.small_level = e->cfg.small_level > 0 ? e->cfg.small_level : max_grid * 2048ll;
    A.small_rows = std::max(1, e->cfg.small_rows);
    A.wait_spins = e->cfg.wait_spins > 0 ? e->cfg.wait_spins : (1ll << 22);
    A.hash_kind = hk;
    A.cap_rows = cap_rows;
    A.cache = (u64 *)e->cache.p;
    A.parents = (u64 *)e->parents.p;
    A.keys = opt->key_mode != LTLG_KEY_EXACT ? (u64 *)e->keys.p : nullptr;
    A.slots = (u64 *)e->slots.p;
    A.slot_mask = e->nslots - 1;
    A.wmeta = (const u64 *)e->wmeta.p;
    A.kmeta = (const u32 *)e->kmeta.p;
    A.ctl = (DevCtl *)e->ctl.p;
    A.lev = dlev;
    A.ls = (long long *)e->ls.p;
    A.level_cands = (u64 *)e->lcands.p;
    A.model = opt->order == LTLG_ORDER_LEARNED ? e->scorer.p : nullptr;
    A.grid = max_grid;
    A.lstats = (u64 *)e->lstats.p;
    A.ring = e->ring_dev;
    A.ring_slots = ltlg_engine::RING;
    cudaMemsetAsync(e->lstats.p, 0, (MAX_COSTS + 2) * LSTATS * sizeof(u64), st);
    cudaMemsetAsync(e->ls.p, 0, (MAX_COSTS + 2) * sizeof(long long), st);
    cudaMemsetAsync(e->lcands.p, 0, (MAX_COSTS + 2) * sizeof(u64), st);
    DevLevel *hl = (DevLevel *)e->h_lev.p;
    memset(hl, 0, offsetof(DevLevel, blocks));
    hl->cost = c1;  // the planner advances to c1 + 1 first
    hl->plan_flags = (opt->schedule == LTLG_SCHEDULE_PER_BLOCK ? PLAN_UNFUSED : 0) |
                     (opt->order == LTLG_ORDER_LEARNED ? PLAN_LEARNED : 0);
    cudaMemcpyAsync(dlev, hl, offsetof(DevLevel, blocks), cudaMemcpyHostToDevice, st);
    const LevelArgs *dA = (const LevelArgs *)e->args.p;
    cudaMemcpyAsync(e->args.p, ha, sizeof(LevelArgs), cudaMemcpyHostToDevice, st);
    if ((err = launch_insert_letters(A, dA, nalpha, st)) != cudaSuccess) return fail_cuda(e, err, res);
    int launches = 1;

    int status = LTLG_NOT_FOUND;
    bool found = letter_hit >= 0, on_the_fly = false, last_round = false;
    int shortage = -1, found_cost = found ? c1 : -1, last_cost = c1;
    u64 found_word = 0;
    u32 dflags = 0;
    double device_ms = 0;
    std::vector<ltlg_block_stat> bstats;
    const bool per_block = opt->schedule == LTLG_SCHEDULE_PER_BLOCK;
    const u32 fatal = ST_WAIT | ST_TMA | ST_TABLE;
    auto fatal_status = [&](u32 f) { return (f & ST_TABLE) ? LTLG_TABLE_FULL : LTLG_DEVICE_WAIT; };

    // ---- device-planned levels: per level one graph launch (the planner builds the plan from
    // the level starts in device memory, then the level kernel runs it and its last CTA writes
    // the level summary into the mapped host ring), enqueued up to RING - 1 levels ahead of
    // the level the host is reading, so the GPU never waits for the host between levels.
    bool host_mode = per_block;
    std::vector<float> level_ms;
    if (!host_mode) {
        constexpr int R = ltlg_engine::RING;
        DevCtl *rctl = (DevCtl *)e->h_ring.p;
        DevLevel *rlev = (DevLevel *)((char *)e->h_ring.p + R * sizeof(DevCtl));
        int enq = 0, done = 0;
        // One graph for every level: planner and level kernel; the level kernel's last CTA
        // writes the level's summary into ring slot (seq - 1) % R of the mapped host ring.
        const long long key[8] = {tl, hk, pitch, block_threads, max_grid, 3, 0, 0};
        if (memcmp(key, e->graph_key, sizeof(key)) != 0) {
            memset(e->graph_key, 0, sizeof(e->graph_key));
            if (e->level_graph[0]) cudaGraphExecDestroy(e->level_graph[0]);
            e->level_graph[0] = nullptr;
            cudaGraph_t g = nullptr;
            err = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
            if (err == cudaSuccess) {
                cudaError_t x = launch_plan(dA, st);
                if (x == cudaSuccess) x = launch_level(A, dA, (int)max_grid, block_threads, st);
                err = cudaStreamEndCapture(st, &g);
                if (err == cudaSuccess) err = x;
                if (err == cudaSuccess) err = cudaGraphInstantiate(&e->level_graph[0], g, 0);
                if (g) cudaGraphDestroy(g);
            }
            if (err != cudaSuccess) return fail_cuda(e, err, res);
            memcpy(e->graph_key, key, sizeof(key));
        }
        auto enqueue = [&]() -> cudaError_t {
            const int k = enq % R;
            cudaEventRecord(e->ev_start[k], st);
            const cudaError_t x = cudaGraphLaunch(e->level_graph[0], st);
            cudaEventRecord(e->ev_done[k], st);
            launches += 2;
            ++enq;
            return x;
        };
        cudaEventRecord(e->ev_a, st);
        while (enq < R - 1 && c1 + enq < max_cost)
            if ((err = enqueue()) != cudaSuccess) return fail_cuda(e, err, res);
        while (done < enq) {
            const int k = done % R;
            if ((err = cudaEventSynchronize(e->ev_done[k])) != cudaSuccess) return fail_cuda(e, err, res);
            ++done;
            const DevCtl &sc = rctl[k];
            const DevLevel &sl = rlev[k];
            float ms = 0;
            cudaEventElapsedTime(&ms, e->ev_start[k], e->ev_done[k]);
            if (!sl.halt) level_ms.push_back(ms);
            dflags |= sc.status;
            bool stop = sl.halt != 0;
            if (sc.status & fatal) {
                status = fatal_status(sc.status);
                stop = true;
            } else if (sc.found && !found) {
                found = true;
                found_word = sc.found;
                found_cost = (int)sc.found_cost;
                if (opt->stop_at_found) {
                    status = LTLG_FOUND;
                    stop = true;
                }
            }
            if (!stop && (sc.status & ST_OVERFLOW)) stop = true;
            if (!sl.halt) last_cost = sl.cost;
            if (sl.halt == 2) stop = true;
            if (!stop && sl.cost >= max_cost) stop = true;
            if (!stop && opt->time_limit_s > 0 && now_s() - t0 > opt->time_limit_s) {
                status = LTLG_TIMEOUT;
                stop = true;
            }
            if (stop) break;
            if (c1 + enq < max_cost)
                if ((err = enqueue()) != cudaSuccess) return fail_cuda(e, err, res);
        }
        cudaEventRecord(e->ev_b, st);
        cudaMemcpyAsync(hc, e->ctl.p, sizeof(DevCtl), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(hl, dlev, offsetof(DevLevel, blocks), cudaMemcpyDeviceToHost, st);
        if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, res);
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev_a, e->ev_b);
        device_ms += ms;
        dflags |= hc->status;
        if (status == LTLG_NOT_FOUND && !(hc->status & fatal) && ((hc->status & ST_OVERFLOW) || hl->halt == 2))
            host_mode = true;
        if (host_mode) {
            if (hl->halt == 2) {
                status = LTLG_BAD_ARGS;  // a level with more splits than a device plan holds
                host_mode = false;
            } else {
                // the level that overflowed ran to its end; continue after it on the host
                on_the_fly = true;
                shortage = (int)hc->overflow_cost;
                hl->cost = shortage;
                hl->halt = 0;
                hl->on_the_fly = 1;
                cudaMemcpyAsync(dlev, hl, offsetof(DevLevel, blocks), cudaMemcpyHostToDevice, st);
            }
        }
    }

    // ---- host-driven levels: the per-block schedule (per-block statistics, the reference's
    // progress lines) and the on-the-fly overflow regime (ltli6463.cu:1202-1206, 1442-1443).
    if (host_mode && status == LTLG_NOT_FOUND && !(found && opt->stop_at_found)) {
        uint64_t all_before = all;
        for (;;) {
            const int cost = hl->cost + 1;
            if (cost > max_cost) {
                last_cost = max_cost;
                break;
            }
            if (on_the_fly && shortage >= 0) {
                const int dif = cost - shortage;
                if (dif == cf[1] || dif == c1 + cf[2] || dif == c1 + cf[3] || dif == cf[4] || dif == cf[5] ||
                    dif == cf[6] || dif == c1 + cf[7])
                    last_round = true;
            }
            if ((err = launch_plan(dA, st)) != cudaSuccess) return fail_cuda(e, err, res);
            ++launches;
            cudaMemcpyAsync(hl, dlev, sizeof(DevLevel), cudaMemcpyDeviceToHost, st);
            cudaMemcpyAsync(hc, e->ctl.p, sizeof(DevCtl), cudaMemcpyDeviceToHost, st);
            if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, res);
            if (hl->halt) {
                if (hl->halt == 2) status = LTLG_BAD_ARGS;  // more splits than a plan holds
                last_cost = std::min(cost, max_cost);
                break;
            }
            cudaEventRecord(e->ev_a, st);
            DevCtl *dctl = (DevCtl *)e->ctl.p;
            if (per_block) {
                // one launch per block in the reference's order, each after a snapshot; the
                // block's items are its window of the level's item table (unfused unary blocks)
                size_t nb_level = 0;
                for (int op = 0; op < 7; ++op) {
                    for (int k = 0; k < hl->nblocks[op]; ++k) {
                        cudaMemcpyAsync((DevCtl *)e->snaps.p + nb_level, e->ctl.p, sizeof(DevCtl),
                                        cudaMemcpyDeviceToDevice, st);
                        long long *win = (long long *)e->h_win.p + 8 * nb_level;
                        long long lo = 0, hi = 0;
                        block_window(hl, op, k, lo, hi);
                        win[0] = lo;  // queue[0]
                        win[1] = hi;  // items_end
                        cudaMemcpyAsync(&dctl->queue[0], &win[0], sizeof(u64), cudaMemcpyHostToDevice, st);
                        cudaMemcpyAsync(&dlev->items_end, &win[1], sizeof(long long), cudaMemcpyHostToDevice, st);
                        const int grid = (int)std::max<long long>(1, std::min<long long>(hi - lo, max_grid));
                        if ((err = launch_level(A, dA, grid, block_threads, st)) != cudaSuccess)
                            return fail_cuda(e, err, res);
                        ++launches;
                        ++nb_level;
                    }
                }
            } else {
                if (hl->items_end > 0) {
                    const int grid = (int)std::min<long long>(hl->items_end, max_grid);
                    if ((err = launch_level(A, dA, grid, block_threads, st)) != cudaSuccess)
                        return fail_cuda(e, err, res);
                    ++launches;
                }
            }
            cudaEventRecord(e->ev_b, st);
            const u64 prev_rows = hc->row_count;
            cudaMemcpyAsync(hc, e->ctl.p, sizeof(DevCtl), cudaMemcpyDeviceToHost, st);
            size_t nsnap = 0;
            for (int op = 0; op < 7; ++op) nsnap += (size_t)hl->nblocks[op];
            if (per_block && nsnap)
                cudaMemcpyAsync(e->h_snaps.p, e->snaps.p, nsnap * sizeof(DevCtl), cudaMemcpyDeviceToHost, st);
            if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, res);
            (void)prev_rows;
            float ms = 0;
            cudaEventElapsedTime(&ms, e->ev_a, e->ev_b);
            device_ms += ms;
            dflags |= hc->status;
            if (per_block) {
                const DevCtl *sn = (const DevCtl *)e->h_snaps.p;
                size_t q = 0;
                uint64_t before = all_before;
                for (int op = 0; op < 7; ++op)
                    for (int k = 0; k < hl->nblocks[op]; ++k, ++q) {
                        const BlockDesc &B = hl->blocks[op][k];
                        ltlg_block_stat sb{};
                        sb.cost = cost;
                        sb.op = op;
                        sb.left_cost = B.lcost;
                        sb.right_cost = (op == OP_AND || op == OP_OR || op == OP_U) ? cost - B.lcost - cf[op + 1] : 0;
                        sb.stored_before = std::min<long long>((long long)sn[q].row_count, cap_rows);
                        sb.all_before = before;
                        sb.to_check = B.candidates;
                        before += (uint64_t)B.candidates;
                        bstats.push_back(sb);
                    }
                all_before = before;
            }
            if (hc->status & fatal) {
                status = fatal_status(hc->status);
                last_cost = cost;
                break;
            }
            if (hc->found && !found) {
                found = true;
                found_word = hc->found;
                found_cost = (int)hc->found_cost;
                if (opt->stop_at_found) {
                    status = LTLG_FOUND;
                    break;
                }
            }
            if (!on_the_fly && (hc->status & ST_OVERFLOW)) {
                on_the_fly = true;
                hl->on_the_fly = 1;
                cudaMemcpyAsync(&dlev->on_the_fly, &hl->on_the_fly, sizeof(int), cudaMemcpyHostToDevice, st);
            }
            last_cost = cost;
            if (last_round) break;
            if (on_the_fly && shortage == -1) shortage = cost;
            if (opt->time_limit_s > 0 && now_s() - t0 > opt->time_limit_s) {
                status = LTLG_TIMEOUT;
                break;
            }
        }
    }

    // ---- level ranges, statistics, reference-style candidate count
    cudaMemcpyAsync(e->h_ls.p, e->ls.p, (MAX_COSTS + 2) * sizeof(long long), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(e->h_lcands.p, e->lcands.p, (MAX_COSTS + 2) * sizeof(u64), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hc, e->ctl.p, sizeof(DevCtl), cudaMemcpyDeviceToHost, st);
    if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, res);
    const long long rows_final = std::min<long long>((long long)hc->row_count, cap_rows);
    const long long *hls = (const long long *)e->h_ls.p;
    const u64 *hlc = (const u64 *)e->h_lcands.p;
    const int top = found && opt->stop_at_found ? found_cost : std::max(last_cost, c1);
    std::vector<long long> &ls = e->level_start;
    ls.assign((size_t)std::max(max_cost, c1) + 3, rows_final);
    for (int k = 0; k <= c1 && k < (int)ls.size(); ++k) ls[k] = 0;
    if (c1 + 1 < (int)ls.size()) ls[c1 + 1] = nalpha;
    for (int k = c1 + 1; k <= std::min(top, MAX_COSTS) && k < (int)ls.size(); ++k) ls[k] = hls[k] > 0 ? hls[k] : ls[k];
    for (int k = std::min(top, MAX_COSTS) + 1; k < (int)ls.size(); ++k) ls[k] = rows_final;
    std::vector<ltlg_level_stat> lstats;
    for (int c = c1 + 1; c <= top && c + 1 < (int)ls.size(); ++c) {
        ltlg_level_stat L{};
        L.cost = c;
        L.candidates = c <= MAX_COSTS ? hlc[c] : 0;
        L.uniques = (uint64_t)(ls[c + 1] - ls[c]);
        const size_t i = (size_t)(c - c1 - 1);
        L.ms = i < level_ms.size() ? level_ms[i] : 0.0;
        lstats.push_back(L);
    }
    // all_ltls: whole levels before the found one, then the found level's blocks in the
    // reference's order up to and including the block holding the find.
    for (const auto &L : lstats)
        if (!(found && opt->stop_at_found && L.cost == found_cost)) all += L.candidates;
    if (found && opt->stop_at_found && found_word) {
        const u64 p = found_word & ~(1ull << 63);
        const int fop = parent_op(p);
        int lc = cost_of_row(ls, (long long)parent_left(p));
        if (fop == OP_U) lc = std::min(lc, cost_of_row(ls, (long long)parent_right(p)));
        std::vector<Block> blocks = level_blocks(found_cost, cf, opt->neg_type, ls);
        for (const Block &B : blocks) {
            all += (uint64_t)B.candidates;
            if (B.op == fop && B.lcost == lc) break;
        }
        if (per_block) {
            // drop the blocks after the one holding the find
            size_t keep = 0;
            for (size_t i = 0; i < bstats.size(); ++i) {
                keep = i + 1;
                if (bstats[i].cost == found_cost && bstats[i].op == fop && bstats[i].left_cost == lc) break;
            }
            bstats.resize(keep);
        }
    }
    if (found && (status == LTLG_NOT_FOUND || status == LTLG_FOUND)) status = LTLG_FOUND;
    res->status = status;
    res->cost = found ? found_cost : last_cost;
    res->all_ltls = all;
    res->on_the_fly = on_the_fly ? 1 : 0;
    res->device_flags = dflags;
    res->device_ms = device_ms;
    res->evaluated = (uint64_t)nalpha + hc->evaluated;
    res->rows = rows_final;

    std::string formula;
    if (letter_hit >= 0) {
        formula = std::string(1, alpha[letter_hit]);
        res->found_op = OP_ATOM;
    } else if (found && found_word) {
        const int wcap = 1024;
        if ((err = launch_walk((const u64 *)e->parents.p, nalpha, found_word, (u64 *)e->walk.p, wcap, st)) !=
            cudaSuccess)
            return fail_cuda(e, err, res);
        ++launches;
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
    res->num_blocks = (int)bstats.size();
    if (!bstats.empty()) {
        res->blocks = (ltlg_block_stat *)malloc(sizeof(ltlg_block_stat) * bstats.size());
        memcpy(res->blocks, bstats.data(), sizeof(ltlg_block_stat) * bstats.size());
    }
    res->launches = launches;
    res->seconds = now_s() - t0;
    (void)OPCH;
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
    const int rc = ltlg_engine_learn(e, t, &opt, res);
    if (rc != LTLG_FOUND || res->found_op == OP_ATOM || res->on_the_fly) return rc;
    const int c = res->cost;
    const int *cf = opt.cost_fun;
    cudaStream_t st = e->stream;
    const LevelArgs &A = *(const LevelArgs *)e->h_args.p;
    const LevelArgs *dA = (const LevelArgs *)e->args.p;
    const std::vector<long long> &ls = e->level_start;
    if ((int)ls.size() < c + 2) return rc;
    // Back to the start of level c: the rows of the lower levels (the level starts below c
    // are still on the device), a clean control block, and a check-only plan of level c with
    // one block per operator.
    DevCtl *hc = (DevCtl *)e->h_ctl.p;
    memset(hc, 0, sizeof(DevCtl));
    hc->row_count = (u64)ls[c];
    DevLevel *hl = (DevLevel *)e->h_lev.p;
    memset(hl, 0, offsetof(DevLevel, blocks));
    hl->cost = c - 1;
    hl->on_the_fly = 1;
    hl->plan_flags = PLAN_UNFUSED;
    DevLevel *dlev = (DevLevel *)e->lev.p;
    DevCtl *dctl = (DevCtl *)e->ctl.p;
    cudaMemcpyAsync(dctl, hc, sizeof(DevCtl), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dlev, hl, offsetof(DevLevel, blocks), cudaMemcpyHostToDevice, st);
    cudaError_t err = launch_plan(dA, st);
    if (err == cudaSuccess) err = cudaMemcpyAsync(hl, dlev, sizeof(DevLevel), cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(e->h_lstats.p, e->lstats.p, (MAX_COSTS + 2) * LSTATS * sizeof(u64), cudaMemcpyDeviceToHost,
                              st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err != cudaSuccess) return fail_cuda(e, err, nullptr);
    if (hl->halt) return rc;
    const long long max_grid = (long long)e->num_sms *
                               std::max(1, level_kernel_max_ctas_per_sm(A.left_tile, A.hash_kind, e->cfg.block_threads, A.pitch));
    // One launch per block: clear the find, open the block's window, run, read the find.
    long long *win = (long long *)e->h_win.p;
    int nb = 0;
    for (int op = 0; op < 7; ++op)
        for (int k = 0; k < hl->nblocks[op]; ++k, ++nb) {
            long long lo = 0, hi = 0;
            block_window(hl, op, k, lo, hi);
            long long *w = win + 8 * nb;
            w[0] = lo;
            w[1] = hi;
            w[2] = 0;
            cudaMemsetAsync(&dctl->found, 0, sizeof(u64), st);
            cudaMemcpyAsync(&dctl->queue[0], &w[0], sizeof(u64), cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(&dlev->items_end, &w[1], sizeof(long long), cudaMemcpyHostToDevice, st);
            const int grid = (int)std::max<long long>(1, std::min<long long>(hi - lo, max_grid));
            if ((err = launch_level(A, dA, grid, e->cfg.block_threads, st)) != cudaSuccess) return fail_cuda(e, err, nullptr);
            cudaMemcpyAsync(&w[2], &dctl->found, sizeof(u64), cudaMemcpyDeviceToHost, st);
        }
    if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, nullptr);
    const u64 *lst = (const u64 *)e->h_lstats.p;
    int nbl = 0;
    for (int q = 0; q < 7; ++q) nbl += hl->nblocks[q];
    nb = 0;
    int out = 0;
    for (int op = 0; op < 7; ++op)
        for (int k = 0; k < hl->nblocks[op]; ++k, ++nb) {
            if (out >= cap) continue;
            const BlockDesc &b = hl->blocks[op][k];
            const BlockInfo bi = block_info(b, op, c, cf, nbl, (long long)hl->level_cands, lst, A.npos, A.n, A.nalpha);
            ltlg_block_record &r = rec[out++];
            r.cost = c;
            r.op = op;
            r.lcost = bi.lcost;
            r.rcost = bi.rcost;
            r.position = b.pad;
            r.won = win[8 * nb + 2] != 0 ? 1 : 0;
            r.candidates = b.candidates;
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
        res->status = LTLG_BAD_ARGS;
        res->formula = strdup(ltlg_status_string(LTLG_BAD_ARGS));
        return res->status;
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
        res->status = rc;
        res->formula = strdup(ltlg_status_string(rc));
        return rc;
    }
    rc = ltlg_engine_learn(e, t, opt, res);
    ltlg_engine_destroy(e);
    return rc;
}

struct ltlg_batch {
    std::vector<ltlg_engine *> engines;
};

LTLG_API int ltlg_batch_create(const ltlg_engine_config *cfg, int32_t workers, ltlg_batch **out) {
    *out = nullptr;
    if (workers < 1 || workers > 64) return LTLG_BAD_ARGS;
    auto *b = new ltlg_batch();
    for (int w = 0; w < workers; ++w) {
        ltlg_engine *e = nullptr;
        const int rc = ltlg_engine_create(cfg, &e);
        if (rc != 0) {
            ltlg_batch_destroy(b);
            return rc;
        }
        b->engines.push_back(e);
    }
    *out = b;
    return 0;
}

LTLG_API void ltlg_batch_destroy(ltlg_batch *b) {
    if (!b) return;
    for (ltlg_engine *e : b->engines) ltlg_engine_destroy(e);
    delete b;
}

LTLG_API void *ltlg_batch_stream(ltlg_batch *b, int32_t worker) {
    if (!b || worker < 0 || worker >= (int)b->engines.size()) return nullptr;
    return (void *)b->engines[worker]->stream;
}

LTLG_API int ltlg_batch_learn(ltlg_batch *b, const ltlg_traces *traces, int32_t count, const ltlg_options *opt,
                              ltlg_result *results) {
    if (!b || count < 0 || (count && (!traces || !results || !opt))) return LTLG_BAD_ARGS;
    std::atomic<int> next{0};
    auto work = [&](ltlg_engine *e) {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= count) return;
            ltlg_engine_learn(e, &traces[i], opt, &results[i]);
        }
    };
    const int workers = std::min<int>((int)b->engines.size(), std::max(count, 1));
    std::vector<std::thread> th;
    for (int w = 1; w < workers; ++w) th.emplace_back(work, b->engines[w]);
    work(b->engines[0]);
    for (auto &t : th) t.join();
    int rc = 0;
    for (int i = 0; i < count; ++i)
        if (results[i].status != LTLG_FOUND && results[i].status != LTLG_NOT_FOUND && !rc) rc = results[i].status;
    return rc;
}

LTLG_API int ltlg_batch_set_scorer(ltlg_batch *b, const float *params, int32_t count) {
    if (!b) return LTLG_BAD_ARGS;
    for (ltlg_engine *e : b->engines) {
        const int rc = ltlg_engine_set_scorer(e, params, count);
        if (rc != 0) return rc;
    }
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
    const u64 v = ((fp >> 40) << 40) | ((u64)(e->gen + 1) << 32) | 0xFFFFFFFFull;
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
