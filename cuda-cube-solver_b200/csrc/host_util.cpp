// Host helpers of libccs: search frames and canonical move prefixes.
#include <vector>

#include "ccs_internal.h"

namespace ccs {

void cube_frames(const uint32_t state[5], uint32_t out[30]) {
    Cubie g = unpack(state);
    Cubie f1 = conjugate(axis_rotation(), g);
    Cubie f2 = conjugate(axis_rotation(), f1);
    const Cubie fr[6] = {g, f1, f2, inverse(g), inverse(f1), inverse(f2)};
    for (int k = 0; k < 6; ++k) pack(fr[k], out + 5 * k);
}

std::vector<uint32_t> canonical_prefixes(int length) {
    // Breadth-first by length; each sequence's children in move order, so the result is the
    // lexicographic order of the canonical sequences.
    std::vector<uint32_t> seqs{0u};
    std::vector<int> last{-1};
    for (int len = 0; len < length; ++len) {
        std::vector<uint32_t> ns;
        std::vector<int> nl;
        for (size_t i = 0; i < seqs.size(); ++i) {
            for (int m = 0; m < 18; ++m) {
                int lf = last[i] / 3, mf = m / 3;
                if (last[i] >= 0 && (mf == lf || (lf >= 3 && mf == lf - 3))) continue;
                ns.push_back(seqs[i] | ((uint32_t)m << (5 * len)));
                nl.push_back(m);
            }
        }
        seqs.swap(ns);
        last.swap(nl);
    }
    return seqs;
}

}  // namespace ccs
