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
#include <chrono>
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

}  // namespace

struct ltlg_engine {
    ltlg_engine_config cfg{};
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t op_stream[7] = {};   // one per operator kernel, forked from and joined to stream
    cudaEvent_t ev_fork = nullptr, ev_join[7] = {};
    cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    DevBuf cache, parents, keys, slots, wmeta, kmeta, ctl, blocks, walk, snaps;
    DevBuf h_ctl, h_blocks, h_walk, h_stage, h_snaps;
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
    c->left_tile = 8;
    c->right_chunk = 64;
    c->unary_rows = 64;
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
    if (cfg.left_tile != 4 && cfg.left_tile != 8) return LTLG_BAD_ARGS;
    if (cfg.block_threads < 32 || cfg.block_threads > 256 || cfg.block_threads % 32) return LTLG_BAD_ARGS;
    if (cfg.right_chunk < 1 || cfg.unary_rows < 1 || cfg.max_traces < 1) return LTLG_BAD_ARGS;
    if (cfg.max_rows <= 0 || cfg.max_rows > (1ll << 30) - 1) cfg.max_rows = (1ll << 30) - 1;
    auto *e = new ltlg_engine();
    e->cfg = cfg;
    cudaError_t err = cudaSetDevice(cfg.device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, cfg.device);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    for (int k = 0; k < 7 && err == cudaSuccess; ++k) {
        err = cudaStreamCreateWithFlags(&e->op_stream[k], cudaStreamNonBlocking);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->ev_join[k], cudaEventDisableTiming);
    }
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming);
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
    for (DevBuf *b : {&e->cache, &e->parents, &e->keys, &e->slots, &e->wmeta, &e->kmeta, &e->ctl, &e->blocks,
                      &e->walk, &e->snaps})
        if (b->p) cudaFree(b->p);
    for (DevBuf *b : {&e->h_ctl, &e->h_blocks, &e->h_walk, &e->h_stage, &e->h_snaps})
        if (b->p) cudaFreeHost(b->p);
    for (cudaEvent_t ev : {e->ev_a, e->ev_b, e->ev_t0, e->ev_t1, e->ev_fork})
        if (ev) cudaEventDestroy(ev);
    for (int k = 0; k < 7; ++k) {
        if (e->ev_join[k]) cudaEventDestroy(e->ev_join[k]);
        if (e->op_stream[k]) cudaStreamDestroy(e->op_stream[k]);
    }
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
    if (npos < 0 || nneg < 0 || (ref_keys && (opt->rlx_unq_chk_type < 1 || opt->rlx_unq_chk_type > 3)) ||
        opt->key_mode < 0 || opt->key_mode > 2 || n > e->cfg.max_traces || nalpha > 26) {
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

    LevelArgs A{};
    A.n = n;
    A.pitch = pitch;
    A.npos = npos;
    A.cap_rows = cap_rows;
    A.cache = (u64 *)e->cache.p;
    A.parents = (u64 *)e->parents.p;
    A.keys = opt->key_mode != LTLG_KEY_EXACT ? (u64 *)e->keys.p : nullptr;
    A.slots = (u64 *)e->slots.p;
    A.slot_mask = e->nslots - 1;
    A.wmeta = (const u64 *)e->wmeta.p;
    A.kmeta = (const u32 *)e->kmeta.p;
    A.ctl = (DevCtl *)e->ctl.p;
    A.key_mode = opt->key_mode == LTLG_KEY_EXACT ? KEY_EXACT : opt->key_mode == LTLG_KEY_REF ? KEY_REF : KEY_HASH64;
    A.rlx_type = rlx_type;
    A.gen = e->gen;
    A.stop_at_found = opt->stop_at_found ? 1 : 0;
    A.right_chunk = e->cfg.right_chunk;
    A.unary_rows = e->cfg.unary_rows;
    int tl = e->cfg.left_tile;
    while (tl > 4 && (size_t)op_kernel_smem_bytes(OP_AND, tl, pitch) > 200 * 1024) tl /= 2;
    if ((size_t)op_kernel_smem_bytes(OP_AND, tl, pitch) > 220 * 1024) {
        res->status = LTLG_BAD_ARGS;
        res->formula = strdup("bad_arguments");
        return res->status;
    }
    A.left_tile = tl;
    if ((err = launch_insert_letters(A, nalpha, st)) != cudaSuccess) return fail_cuda(e, err, res);
    int launches = 1;

    const int block_threads = e->cfg.block_threads;
    long long max_grid_op[7];
    long long max_grid = 0;
    for (int k = 0; k < 7; ++k) {
        const int per_sm = std::max(1, op_kernel_max_ctas_per_sm(k, tl, A.key_mode == KEY_HASH64 ? 1 : 0,
                                                                 block_threads, pitch));
        max_grid_op[k] = (long long)e->num_sms * per_sm;
        max_grid = std::max(max_grid, max_grid_op[k]);
    }

    std::vector<ltlg_level_stat> lstats;
    std::vector<ltlg_block_stat> bstats;
    std::vector<long long> &ls = e->level_start;
    int status = LTLG_NOT_FOUND;
    bool found = false, on_the_fly = false, last_round = false;
    int shortage = -1, cost = c1, found_cost = -1;
    u64 found_word = 0;
    u32 dflags = 0;
    double device_ms = 0;
    const bool per_block = opt->schedule == LTLG_SCHEDULE_PER_BLOCK;
    if (letter_hit >= 0) {
        found = true;
        found_cost = c1;
    }
    for (cost = c1 + 1; cost <= max_cost; ++cost) {
        if (on_the_fly) {
            const int dif = cost - shortage;
            if (dif == cf[1] || dif == c1 + cf[2] || dif == c1 + cf[3] || dif == cf[4] || dif == cf[5] ||
                dif == cf[6] || dif == c1 + cf[7])
                last_round = true;
        }
        std::vector<Block> blocks = level_blocks(cost, cf, opt->neg_type, ls);
        // work items
        const size_t nb = blocks.size();
        if ((err = ensure(e->blocks, std::max<size_t>(nb, 1) * sizeof(BlockDesc))) != cudaSuccess ||
            (err = ensure_host(e->h_blocks, std::max<size_t>(nb, 1) * sizeof(BlockDesc))) != cudaSuccess ||
            (err = ensure(e->snaps, (std::max<size_t>(nb, 1) + 1) * sizeof(DevCtl))) != cudaSuccess ||
            (err = ensure_host(e->h_snaps, (std::max<size_t>(nb, 1) + 1) * sizeof(DevCtl))) != cudaSuccess)
            return fail_cuda(e, err, res);
        BlockDesc *hb = (BlockDesc *)e->h_blocks.p;
        long long items = 0;
        uint64_t level_cands = 0;
        for (const Block &B : blocks) level_cands += (uint64_t)B.candidates;
        // Work-item size: a small level is cut into one right row (or one group of source
        // rows) per warp so every SM takes part; a large level keeps the configured sizes.
        {
            const int nwarps = block_threads / 32;
            if ((long long)level_cands < max_grid * 2048ll) {
                A.right_chunk = nwarps;
                A.unary_rows = nwarps * 4;
            } else {
                A.right_chunk = e->cfg.right_chunk;
                A.unary_rows = e->cfg.unary_rows;
            }
        }
        for (size_t b = 0; b < nb; ++b) {
            const Block &B = blocks[b];
            BlockDesc d{};
            d.op = B.op;
            d.l0 = B.l0;
            d.l1 = B.l1;
            d.r0 = B.r0;
            d.r1 = B.r1;
            d.item0 = items;
            if (B.op == OP_AND || B.op == OP_OR || B.op == OP_U) {
                const int tile = B.op == OP_U ? tl / 2 : tl;  // U: two candidates per pair
                d.tiles_r = (B.r1 - B.r0 + A.right_chunk - 1) / A.right_chunk;
                d.items = ((B.l1 - B.l0 + tile - 1) / tile) * d.tiles_r;
            } else {
                d.tiles_r = 1;
                d.items = (B.r1 - B.r0 + A.unary_rows - 1) / A.unary_rows;
            }
            items += d.items;
            hb[b] = d;
        }
        const long long stored_before = ls[cost];
        // Items are numbered per operator (each operator's kernel drains its own queue);
        // the per-block schedule numbers every block from 0.
        {
            long long op_items[7] = {0, 0, 0, 0, 0, 0, 0};
            for (size_t b = 0; b < nb; ++b) {
                const int op = hb[b].op;
                hb[b].item0 = per_block ? 0 : op_items[op];
                op_items[op] += hb[b].items;
            }
        }
        if (nb) cudaMemcpyAsync(e->blocks.p, hb, nb * sizeof(BlockDesc), cudaMemcpyHostToDevice, st);
        A.check_only = on_the_fly ? 1 : 0;
        DevCtl *dctl = (DevCtl *)e->ctl.p;
        if (!per_block && items > 0) cudaMemsetAsync(dctl->queue, 0, sizeof(dctl->queue), st);
        cudaEventRecord(e->ev_a, st);
        if (!per_block) {
            if (items > 0) {
                // fork: every operator with work runs concurrently on its own stream
                cudaEventRecord(e->ev_fork, st);
                size_t b = 0;
                while (b < nb) {
                    const int op = hb[b].op;
                    size_t b2 = b;
                    long long op_total = 0;
                    while (b2 < nb && hb[b2].op == op) op_total += hb[b2++].items;
                    A.blocks = (const BlockDesc *)e->blocks.p + b;
                    A.nblocks = (int)(b2 - b);
                    A.total_items = op_total;
                    A.queue = dctl->queue + op;
                    cudaStreamWaitEvent(e->op_stream[op], e->ev_fork, 0);
                    const int grid = (int)std::min<long long>(op_total, max_grid_op[op]);
                    if ((err = launch_op(op, A, grid, block_threads, e->op_stream[op])) != cudaSuccess)
                        return fail_cuda(e, err, res);
                    ++launches;
                    cudaEventRecord(e->ev_join[op], e->op_stream[op]);
                    cudaStreamWaitEvent(st, e->ev_join[op], 0);
                    b = b2;
                }
            }
        } else {
            for (size_t b = 0; b < nb; ++b) {
                const int op = hb[b].op;
                cudaMemcpyAsync((DevCtl *)e->snaps.p + b, e->ctl.p, sizeof(DevCtl), cudaMemcpyDeviceToDevice, st);
                cudaMemsetAsync(dctl->queue + op, 0, sizeof(u64), st);
                A.blocks = (const BlockDesc *)e->blocks.p + b;
                A.nblocks = 1;
                A.total_items = hb[b].items;
                A.queue = dctl->queue + op;
                const int grid = (int)std::min<long long>(hb[b].items, max_grid_op[op]);
                if ((err = launch_op(op, A, grid, block_threads, st)) != cudaSuccess) return fail_cuda(e, err, res);
                ++launches;
            }
        }
        cudaEventRecord(e->ev_b, st);
        cudaMemcpyAsync(hc, e->ctl.p, sizeof(DevCtl), cudaMemcpyDeviceToHost, st);
        if (per_block && nb)
            cudaMemcpyAsync(e->h_snaps.p, e->snaps.p, nb * sizeof(DevCtl), cudaMemcpyDeviceToHost, st);
        if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, err, res);
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev_a, e->ev_b);
        device_ms += ms;
        dflags |= hc->status;
        const long long stored = std::min<long long>((long long)hc->row_count, cap_rows);
        // Reference-style candidate counting: whole blocks up to the one holding the find.
        uint64_t counted = level_cands;
        size_t nb_reported = nb;
        if (hc->found && !found) {
            const u64 p = hc->found & ~(1ull << 63);
            const int fop = parent_op(p);
            const long long l = (long long)parent_left(p), r = (long long)parent_right(p);
            int lc = cost_of_row(ls, l);
            if (fop == OP_U) lc = std::min(lc, cost_of_row(ls, r));
            counted = 0;
            nb_reported = 0;
            for (const Block &B : blocks) {
                counted += (uint64_t)B.candidates;
                ++nb_reported;
                if (B.op == fop && B.lcost == lc) break;
            }
        }
        if (per_block) {
            const DevCtl *sn = (const DevCtl *)e->h_snaps.p;
            uint64_t before = all;
            for (size_t b = 0; b < nb_reported; ++b) {
                ltlg_block_stat s{};
                s.cost = cost;
                s.op = blocks[b].op;
                s.left_cost = blocks[b].lcost;
                s.right_cost = blocks[b].rcost;
                s.stored_before = std::min<long long>((long long)sn[b].row_count, cap_rows);
                s.all_before = before;
                s.to_check = blocks[b].candidates;
                bstats.push_back(s);
                before += (uint64_t)blocks[b].candidates;
            }
        }
        all += counted;
        ltlg_level_stat L{};
        L.cost = cost;
        L.blocks = (int)nb;
        L.candidates = level_cands;
        L.uniques = (uint64_t)(stored - stored_before);
        L.ms = ms;
        lstats.push_back(L);
        if (hc->status & (ST_WAIT | ST_TMA)) {
            status = LTLG_DEVICE_WAIT;
            break;
        }
        if (hc->status & ST_TABLE) {
            status = LTLG_TABLE_FULL;
            break;
        }
        if (hc->found && !found) {
            found = true;
            found_word = hc->found;
            found_cost = cost;
            if (opt->stop_at_found) {
                ls[cost + 1] = stored;
                status = LTLG_FOUND;
                break;
            }
        }
        if (!on_the_fly) {
            if (hc->status & ST_OVERFLOW) {
                on_the_fly = true;
                hc->row_count = (u64)cap_rows;
            }
        }
        for (size_t k = (size_t)cost + 1; k < ls.size(); ++k) ls[k] = stored;
        if (last_round) break;
        if (on_the_fly && shortage == -1) shortage = cost;
        if (opt->time_limit_s > 0 && now_s() - t0 > opt->time_limit_s) {
            status = LTLG_TIMEOUT;
            break;
        }
    }
    if (cost == max_cost + 1) cost--;
    if (found && (status == LTLG_NOT_FOUND || status == LTLG_FOUND)) status = LTLG_FOUND;
    res->status = status;
    res->cost = found ? found_cost : cost;
    res->all_ltls = all;
    res->on_the_fly = on_the_fly ? 1 : 0;
    res->device_flags = dflags;
    res->device_ms = device_ms;
    res->evaluated = (uint64_t)nalpha + hc->evaluated;
    res->rows = std::min<long long>((long long)hc->row_count, cap_rows);

    std::string formula;
    if (letter_hit >= 0) {
        formula = std::string(1, alpha[letter_hit]);
        res->found_op = OP_ATOM;
    } else if (found) {
        const int cap = 1024;
        if ((err = launch_walk((const u64 *)e->parents.p, nalpha, found_word, (u64 *)e->walk.p, cap, st)) !=
            cudaSuccess)
            return fail_cuda(e, err, res);
        ++launches;
        cudaMemcpyAsync(e->h_walk.p, e->walk.p, (2 + 2 * cap) * 8, cudaMemcpyDeviceToHost, st);
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

LTLG_API int ltlg_learn(const ltlg_traces *t, const ltlg_options *opt, ltlg_result *res) {
    ltlg_engine_config cfg;
    ltlg_default_engine_config(&cfg);
    const int n = t ? t->num_pos + t->num_neg : 0;
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
    ScarletFile f;
    if (!path || !read_scarlet(path, f)) return LTLG_BAD_ARGS;
    std::vector<uint32_t> steps;
    std::vector<int32_t> offsets;
    std::string alpha;
    scarlet_to_masks(f, steps, offsets, alpha);
    uint32_t *s = (uint32_t *)malloc(std::max<size_t>(steps.size(), 1) * 4);
    int32_t *o = (int32_t *)malloc(offsets.size() * 4);
    char *a = strdup(alpha.c_str());
    if (!steps.empty()) memcpy(s, steps.data(), steps.size() * 4);
    memcpy(o, offsets.data(), offsets.size() * 4);
    out->num_pos = (int32_t)f.pos.size();
    out->num_neg = (int32_t)f.neg.size();
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
