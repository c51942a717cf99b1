// ltli6463-compatible command line (code/ltli6463.cu:1575-1680):
//   ltli6463 <input_file> c1 c2 c3 c4 c5 c6 c7 c8 maxCost RlxUnqChkTyp NegType [--flags]
// prints the traces, the cost function, the trace count, the measurement lines the
// reference prints under MEASUREMENT_MODE, and  LTL: "<formula>"  as the
// second-to-last line, which is what code/dc.py:194 and :278 parse.
//
// Trailing flags (new; the 12 positional arguments keep their meaning):
//   --exact           uniqueness on the full CS (default)
//   --reference-keys  the reference's relaxed keys of type RlxUnqChkTyp (ltli6463.cu:57-141)
//   --hash64          relaxed uniqueness on a 64-bit fingerprint of the full CS
//   --per-block       one launch per (operator, split) block, printing the reference's
//                     per-block progress lines
//   --limit-traces    refuse more than 64 traces, as the reference does
#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ltlgpu.h"
#include "scarlet.hpp"

int main(int argc, char *argv[]) {
    if (argc < 13) {
        printf("Arguments should be in the form of\n");
        printf("-----------------------------------------------------------------\n");
        printf("%s <input_file_address> <c1> <c2> <c3> <c4> <c5> <c6> <c7> <c8> <maxCost> <RlxUnqChkTyp> <NegType>\n",
               argv[0]);
        printf("-----------------------------------------------------------------\n");
        printf("\nFor example\n");
        printf("-----------------------------------------------------------------\n");
        printf("%s ./input.txt 1 1 1 1 1 1 1 1 500 3 2\n", argv[0]);
        printf("-----------------------------------------------------------------\n");
        return 0;
    }
    bool argError = false;
    for (int i = 2; i < 11; ++i) {
        if (std::atoi(argv[i]) <= 0 || std::atoi(argv[i]) > SHRT_MAX) {
            printf("Argument number %d, \"%s\", should be a positive short integer.\n", i, argv[i]);
            argError = true;
        }
    }
    if (std::atoi(argv[11]) < 1 || std::atoi(argv[11]) > 3) {
        printf("Argument number 11, RlxUnqChkTyp = \"%s\", should be 1, 2, or 3.\n", argv[11]);
        argError = true;
    }
    if (std::atoi(argv[12]) < 1 || std::atoi(argv[12]) > 2) {
        printf("Argument number 12, NegType = \"%s\", should be 1, or 2.\n", argv[12]);
        argError = true;
    }
    ltlg_options opt;
    ltlg_default_options(&opt);
    bool progress = false;
    for (int i = 13; i < argc; ++i) {
        const std::string f = argv[i];
        if (f == "--exact")
            opt.key_mode = LTLG_KEY_EXACT;
        else if (f == "--reference-keys")
            opt.key_mode = LTLG_KEY_REF;
        else if (f == "--hash64")
            opt.key_mode = LTLG_KEY_HASH64;
        else if (f == "--per-block") {
            opt.schedule = LTLG_SCHEDULE_PER_BLOCK;
            progress = true;
        } else if (f == "--limit-traces")
            opt.limit_traces = 1;
        else {
            printf("Unknown option \"%s\".\n", argv[i]);
            argError = true;
        }
    }
    if (argError) return 0;

    ltlg::ScarletFile file;
    if (!ltlg::read_scarlet(argv[1], file)) {
        printf("Failed to open the input file.\n");
        return 0;
    }
    for (int i = 0; i < 8; ++i) opt.cost_fun[i] = std::atoi(argv[i + 2]);
    opt.max_cost = std::atoi(argv[10]);
    opt.rlx_unq_chk_type = std::atoi(argv[11]);
    opt.neg_type = std::atoi(argv[12]);

    std::vector<uint32_t> steps;
    std::vector<int32_t> offsets;
    std::string alpha;
    ltlg::scarlet_to_masks(file, steps, offsets, alpha);
    ltlg_traces tr;
    tr.num_pos = (int32_t)file.pos.size();
    tr.num_neg = (int32_t)file.neg.size();
    tr.alphabet = alpha.c_str();
    tr.steps = steps.data();
    tr.offsets = offsets.data();

    const auto start = std::chrono::high_resolution_clock::now();
    ltlg_result res;
    ltlg_learn(&tr, &opt, &res);
    const auto stop = std::chrono::high_resolution_clock::now();

    if (res.status == LTLG_INPUT_LIMITS) {
        int maxlen = 0;
        for (size_t i = 0; i + 1 < offsets.size(); ++i) maxlen = std::max(maxlen, offsets[i + 1] - offsets[i]);
        printf("In this version, The input can have:\n");
        printf("1) At most %d traces. It is currently %d.\n", opt.limit_traces ? 64 : 8192,
               tr.num_pos + tr.num_neg);
        printf("2) Max(len(trace)) = %d. It is currently %d.\n", 63, maxlen);
        ltlg_result_free(&res);
        return 0;
    }
    if (progress) {
        // the letters' line, printed by the reference before its first level (ltli6463.cu:1095-1098)
        printf("Cost %-2d | (A) | AllLTLs: %-11lu | StoredLTLs: %-10d | ToBeChecked: %-10d \n", opt.cost_fun[0], 0ul,
               0, (int)alpha.size());
        for (int b = 0; b < res.num_blocks; ++b) {
            const ltlg_block_stat &s = res.blocks[b];
            static const char ops[] = "~&|XFGU";
            printf("Cost %-2d | (%c) | AllLTLs: %-11lu | StoredLTLs: %-10ld | ToBeChecked: %-10ld \n", s.cost,
                   ops[s.op], (unsigned long)s.all_before, (long)s.stored_before, (long)s.to_check);
        }
    }
    printf("\nPositive: \n");
    for (const auto &trace : file.pos) {
        printf("\t");
        for (const auto &t : trace) {
            std::string s;
            for (const auto &c : t) {
                s += c;
                s += ", ";
            }
            printf("{%s}\t", s.substr(0, s.length() >= 2 ? s.length() - 2 : 0).c_str());
        }
        printf("\n");
    }
    printf("\nNegative: \n");
    for (const auto &trace : file.neg) {
        printf("\t");
        for (const auto &t : trace) {
            std::string s;
            for (const auto &c : t) {
                s += c;
                s += ", ";
            }
            printf("{%s}\t", s.substr(0, s.length() >= 2 ? s.length() - 2 : 0).c_str());
        }
        printf("\n");
    }
    printf("\nCost Function: p:%u, ~:%u, &:%u, |:%u, X:%u, F:%u, G:%u, U:%u", opt.cost_fun[0], opt.cost_fun[1],
           opt.cost_fun[2], opt.cost_fun[3], opt.cost_fun[4], opt.cost_fun[5], opt.cost_fun[6], opt.cost_fun[7]);
    printf("\nNumber of Traces: %d", tr.num_pos + tr.num_neg);
    const auto us = std::chrono::duration_cast<std::chrono::microseconds>(stop - start).count();
    printf("\nNumber of All LTLs: %lu", (unsigned long)res.all_ltls);
    printf("\nCost of Final LTL: %d", res.cost);
    printf("\nRunning Time: %f s", (double)us * 0.000001);
    printf("\n\nLTL: \"%s\"\n", res.formula ? res.formula : "");
    ltlg_result_free(&res);
    return 0;
}
