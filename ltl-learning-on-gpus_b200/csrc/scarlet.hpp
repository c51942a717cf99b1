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

}  // namespace ltlg
