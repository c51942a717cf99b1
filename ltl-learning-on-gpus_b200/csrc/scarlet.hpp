// Scarlet trace files, read with the reference's rules (code/ltli6463.cu:1500-1573).
#pragma once

#include <cstdint>
#include <set>
#include <string>
#include <vector>

namespace ltlg {

struct ScarletFile {
    std::string alpha;                             // letters of the last line, file order
    std::set<char> alphabet;                       // the same letters, sorted
    std::vector<std::vector<std::string>> pos;     // per trace, per step: letters holding
    std::vector<std::vector<std::string>> neg;
};

// Returns false when the file cannot be opened.
bool read_scarlet(const std::string &path, ScarletFile &out);

// Step masks (bit letter - 'a') and offsets, positives first.
void scarlet_to_masks(const ScarletFile &f, std::vector<uint32_t> &steps, std::vector<int32_t> &offsets,
                      std::string &sorted_alphabet);

// The same file read in one pass straight to step masks, with no per-step strings: what
// read_scarlet followed by scarlet_to_masks gives, for large trace files.
struct ScarletMasks {
    int32_t num_pos = 0, num_neg = 0;
    std::string sorted_alphabet;
    std::vector<uint32_t> steps;
    std::vector<int32_t> offsets;  // num_pos + num_neg + 1 entries
};
bool read_scarlet_masks(const std::string &path, ScarletMasks &out);

}  // namespace ltlg
