// Evaluation of arbitrary formula strings on traces, on the device: the checker the
// divide-and-conquer driver applies to every sub-formula (the reference's dc.py does it on
// the host with bitarray, code/dc.py:136-187).  The string is parsed the way dc.py's bitVec
// reads it (code/dc.py:136-183): "~(f)", "X(f)", "F(f)", "G(f)", "(f)&(g)", "(f)|(g)",
// "(f)U(g)", single letters; the postfix program then runs on every trace in parallel with
// the enumerator's own operators (eval_formula_kernel in ltl_kernels.cu).
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "ltl_kernels.cuh"
#include "ltlgpu.h"
#include "traces.hpp"

namespace ltlg {
namespace {

struct Parser {
    const std::string &s;
    const std::string &alpha;
    std::vector<int> prog;  // (op, arg) pairs
    int depth = 0, max_depth = 0;

    void emit(int op, int arg, int push) {
        prog.push_back(op);
        prog.push_back(arg);
        depth += push;
        if (depth > max_depth) max_depth = depth;
    }

    // s[b, e) is one formula.
    bool parse(size_t b, size_t e) {
        if (b >= e) return false;
        size_t i = b;
        if (s[b] == '(') {  // skip the first parenthesised group: the operator follows it
            int p = 1;
            for (i = b + 1; i < e && p; ++i) p += s[i] == '(' ? 1 : s[i] == ')' ? -1 : 0;
            if (p) return false;
        }
        if (i >= e) return false;
        const char c = s[i];
        switch (c) {
        case '~':
        case 'X':
        case 'F':
        case 'G': {
            if (i != b || e - b < 4 || s[b + 1] != '(' || s[e - 1] != ')') return false;
            if (!parse(b + 2, e - 1)) return false;
            emit(c == '~' ? OP_NEG : c == 'X' ? OP_X : c == 'F' ? OP_F : OP_G, 0, 0);
            return true;
        }
        case '&':
        case '|':
        case 'U': {
            if (s[b] != '(' || i + 1 >= e || s[i + 1] != '(' || s[e - 1] != ')') return false;
            if (!parse(b + 1, i - 1) || !parse(i + 2, e - 1)) return false;
            emit(c == '&' ? OP_AND : c == '|' ? OP_OR : OP_U, 0, -1);
            return true;
        }
        default: {
            if (e - b != 1) return false;
            const size_t j = alpha.find(c);
            if (j == std::string::npos) return false;
            emit(OP_ATOM, (int)j, 1);
            return true;
        }
        }
    }
};

struct DevMem {
    std::vector<void *> p;
    ~DevMem() {
        for (void *q : p) cudaFree(q);
    }
    template <class T>
    T *get(size_t n, cudaError_t &err) {
        void *q = nullptr;
        if (err == cudaSuccess) err = cudaMalloc(&q, (n ? n : 1) * sizeof(T));
        if (err == cudaSuccess) p.push_back(q);
        return (T *)q;
    }
};

}  // namespace
}  // namespace ltlg

using namespace ltlg;

extern "C" LTLG_API int ltlg_evaluate(const ltlg_traces *t, const char *formula, uint64_t *cs, uint8_t *holds) {
    if (!formula || !traces_well_formed(t)) return LTLG_BAD_ARGS;
    const int n = t->num_pos + t->num_neg;
    const std::string alpha = t->alphabet ? t->alphabet : "";
    const std::string f = formula;
    Parser P{f, alpha, {}};
    if (!P.parse(0, f.size())) return LTLG_BAD_ARGS;
    if (n == 0) return 0;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LTLG_NO_DEVICE;
    // letters as CS words, per letter and trace
    std::vector<u64> atoms((size_t)alpha.size() * n, 0), lenmask(n, 0);
    for (int i = 0; i < n; ++i) {
        const int len = t->offsets[i + 1] - t->offsets[i];
        if (len < 0) return LTLG_BAD_ARGS;
        if (len > 63) return LTLG_INPUT_LIMITS;
        lenmask[i] = (1ull << len) - 1ull;
        for (int k = 0; k < len; ++k) {
            const uint32_t m = t->steps[t->offsets[i] + k];
            for (size_t j = 0; j < alpha.size(); ++j)
                if ((m >> (alpha[j] - 'a')) & 1u) atoms[j * n + i] |= 1ull << k;
        }
    }
    const int len = (int)P.prog.size() / 2;
    cudaError_t err = cudaSuccess;
    DevMem d;
    int *dprog = d.get<int>(P.prog.size(), err);
    u64 *datoms = d.get<u64>(atoms.size(), err);
    u64 *dmask = d.get<u64>(n, err);
    u64 *dstack = d.get<u64>((size_t)P.max_depth * n, err);
    u64 *dout = d.get<u64>(n, err);
    if (err == cudaSuccess) err = cudaMemcpy(dprog, P.prog.data(), P.prog.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (err == cudaSuccess && !atoms.empty())
        err = cudaMemcpy(datoms, atoms.data(), atoms.size() * sizeof(u64), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dmask, lenmask.data(), n * sizeof(u64), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = launch_eval_formula(dprog, len, datoms, dmask, n, dstack, dout, 0);
    std::vector<u64> out(n);
    if (err == cudaSuccess) err = cudaMemcpy(out.data(), dout, n * sizeof(u64), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return err == cudaErrorMemoryAllocation ? LTLG_NO_MEMORY : LTLG_CUDA_ERROR;
    for (int i = 0; i < n; ++i) {
        if (cs) cs[i] = out[i];
        if (holds) holds[i] = (uint8_t)(out[i] & 1ull);
    }
    return 0;
}
