// Scarlet reader restating code/ltli6463.cu:1500-1573: the last line of the file gives
// the letters (only 'a'..'z' kept; the file order maps a value's position in a step to
// a letter, the sorted set gives the letter indices); positive traces run until the
// first "---" line and negative traces until the next one.  Inside a trace line ';'
// ends a time step, ',' is skipped and every other character advances the value
// position, '1' adding the letter at that position.
#include "scarlet.hpp"

#include <cstdio>
#include <cstring>
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

bool read_scarlet_masks(const std::string &path, ScarletMasks &out) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    std::string text;
    char buf[1 << 16];
    for (size_t k; (k = fread(buf, 1, sizeof(buf), f)) > 0;) text.append(buf, k);
    fclose(f);
    // letters: the last line, one trailing newline ignored (as read_scarlet)
    size_t end = text.size();
    if (end && text[end - 1] == '\n') --end;
    const size_t nl = text.rfind('\n', end ? end - 1 : 0);
    const size_t first = (nl == std::string::npos || nl >= end) ? 0 : nl + 1;
    std::vector<uint32_t> vbit;  // value position -> letter bit
    uint32_t letters = 0;
    for (size_t i = first; i < end; ++i) {
        const char c = text[i];
        if (c >= 'a' && c <= 'z') {
            vbit.push_back(1u << (c - 'a'));
            letters |= 1u << (c - 'a');
        }
    }
    out.sorted_alphabet.clear();
    for (int b = 0; b < 26; ++b)
        if ((letters >> b) & 1u) out.sorted_alphabet += (char)('a' + b);
    out.steps.clear();
    out.offsets.assign(1, 0);
    out.num_pos = out.num_neg = 0;
    // trace lines: positives up to the first "---" line, negatives up to the next one;
    // lines end at '\n' (a final line needs none, an empty segment after the last '\n' is
    // not a line), and a separator is exactly "---"
    const char *p = text.data(), *const e = p + text.size();
    int side = 0;
    while (p < e && side < 2) {
        const char *q = static_cast<const char *>(memchr(p, '\n', (size_t)(e - p)));
        if (!q) q = e;
        if (q - p == 3 && p[0] == '-' && p[1] == '-' && p[2] == '-') {
            ++side;
        } else {
            uint32_t m = 0;
            size_t j = 0;
            for (const char *c = p; c < q; ++c) {
                if (*c == ';') {
                    out.steps.push_back(m);
                    m = 0;
                    j = 0;
                } else if (*c != ',') {
                    if (*c == '1' && j < vbit.size()) m |= vbit[j];
                    ++j;
                }
            }
            out.steps.push_back(m);
            out.offsets.push_back((int32_t)out.steps.size());
            ++(side == 0 ? out.num_pos : out.num_neg);
        }
        p = q + 1;
    }
    return true;
}

}  // namespace ltlg
