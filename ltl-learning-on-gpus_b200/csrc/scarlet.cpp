// Scarlet reader restating code/ltli6463.cu:1500-1573: the last line of the file gives
// the letters (only 'a'..'z' kept; the file order maps a value's position in a step to
// a letter, the sorted set gives the letter indices); positive traces run until the
// first "---" line and negative traces until the next one.  Inside a trace line ';'
// ends a time step, ',' is skipped and every other character advances the value
// position, '1' adding the letter at that position.
#include "scarlet.hpp"

#include <fstream>
#include <iterator>
#include <sstream>

namespace ltlg {

static std::vector<std::string> parse_trace(const std::string &line, const std::string &alpha) {
    std::vector<std::string> trace;
    std::string token;
    size_t j = 0;
    for (char c : line) {
        if (c == ';') {
            trace.push_back(token);
            token.clear();
            j = 0;
        } else if (c == ',') {
            continue;
        } else {
            if (c == '1' && j < alpha.size()) token += alpha[j];
            ++j;
        }
    }
    trace.push_back(token);
    return trace;
}

bool read_scarlet(const std::string &path, ScarletFile &out) {
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) return false;
    std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    // The last line: the reference scans back from the second-to-last byte to the
    // previous newline, so one trailing newline is ignored.
    std::string body = text;
    if (!body.empty() && body.back() == '\n') body.pop_back();
    const size_t k = body.rfind('\n');
    const std::string last = k == std::string::npos ? body : body.substr(k + 1);
    out.alpha.clear();
    out.alphabet.clear();
    for (char c : last)
        if (c >= 'a' && c <= 'z') {
            out.alphabet.insert(c);
            out.alpha += c;
        }
    std::istringstream ss(text);
    std::string line;
    out.pos.clear();
    out.neg.clear();
    while (std::getline(ss, line)) {
        if (line == "---") break;
        out.pos.push_back(parse_trace(line, out.alpha));
    }
    while (std::getline(ss, line)) {
        if (line == "---") break;
        out.neg.push_back(parse_trace(line, out.alpha));
    }
    return true;
}

void scarlet_to_masks(const ScarletFile &f, std::vector<uint32_t> &steps, std::vector<int32_t> &offsets,
                      std::string &sorted_alphabet) {
    steps.clear();
    offsets.assign(1, 0);
    sorted_alphabet.assign(f.alphabet.begin(), f.alphabet.end());
    for (const auto *side : {&f.pos, &f.neg}) {
        for (const auto &trace : *side) {
            for (const auto &tok : trace) {
                uint32_t m = 0;
                for (char c : tok)
                    if (c >= 'a' && c <= 'z') m |= 1u << (c - 'a');
                steps.push_back(m);
            }
            offsets.push_back((int32_t)steps.size());
        }
    }
}

}  // namespace ltlg
