// Host-side check of a trace set handed to the C ABI, before any of it is read as masks or
// shift counts: trace lengths come from differences of offsets and letters become bit
// positions (letter - 'a'), so offsets must not decrease and letters must be 'a'..'z'.
#pragma once

#include "ltlgpu.h"

namespace ltlg {

inline bool traces_well_formed(const ltlg_traces *t) {
    if (!t || t->num_pos < 0 || t->num_neg < 0 || t->num_pos > (1 << 30) || t->num_neg > (1 << 30)) return false;
    const int n = t->num_pos + t->num_neg;
    if (n > 0) {
        if (!t->offsets || t->offsets[0] < 0) return false;
        for (int i = 0; i < n; ++i)
            if (t->offsets[i + 1] < t->offsets[i]) return false;
        if (t->offsets[n] > t->offsets[0] && !t->steps) return false;
    }
    if (t->alphabet)
        for (const char *c = t->alphabet; *c; ++c)
            if (*c < 'a' || *c > 'z') return false;
    return true;
}

}  // namespace ltlg
