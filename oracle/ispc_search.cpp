/*
 * oracle/ispc_search.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Restatement of the 4-lane k-ary searches lower_bound_vec / upper_bound_vec of
 * kernels/upward-common.ispc:59-124, including their single-precision interval
 * arithmetic ((e - s) * 1.f / programCount and the + 0.499999f rounding).  Compiled
 * without -ffast-math so that the float expressions are evaluated as written.
 */
#include <algorithm>

typedef REAL realtype;

#include "upward-kernels.h"

namespace {
enum { LANES = 4 };

template <bool UPPER>
int kary_bound(int s, int e, const int val, const int keys[])
{
    int c = e - s;

    if (UPPER ? keys[s] > val : keys[s] >= val) return s;
    if (UPPER ? keys[e - 1] <= val : keys[e - 1] < val) return e;

    while (c) {
        int cs[LANES], ce[LANES];
        const float h = (float)(e - s) * 1.f / (float)LANES;
        for (int l = 0; l < LANES; ++l) {
            const float pos = (float)s + (float)l * h + 0.499999f;
            const int i = std::min(e - 1, (int)pos);
            const bool isless = UPPER ? keys[i] <= val : keys[i] < val;
            cs[l] = isless ? i : s;
            ce[l] = isless ? e : i;
        }
        s = std::max(std::max(cs[0], cs[1]), std::max(cs[2], cs[3]));
        e = std::min(std::min(ce[0], ce[1]), std::min(ce[2], ce[3]));
        c = std::min(c / LANES, e - s);
    }
    return s + 1;
}
} // namespace

/* kernels/upward-common.ispc:59-90 */
extern "C" int lower_bound_vec(int s, int e, const int val, const int keys[])
{
    return kary_bound<false>(s, e, val, keys);
}

/* kernels/upward-common.ispc:92-124 */
extern "C" int upper_bound_vec(int s, int e, const int val, const int keys[])
{
    return kary_bound<true>(s, e, val, keys);
}
