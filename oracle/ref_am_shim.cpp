// ref_am_shim.cpp -- TEST INFRASTRUCTURE ONLY: an extern "C" face over the reference's approximate pattern search
// (NikitaMishin/semilocal, source/cpu/approximate_matching/ApproximateMatching.h), compiled in place from the
// reference tree by oracle/build_ref.sh into oracle/_ref/libslcs_ref_am.so.  It pins the oracle's restatement
// (amatch_oracle.cpp) and generates tests/golden/ fixtures.  A separate library from libslcs_ref.so because these
// headers build on the reference's legacy permutation types.
#include <algorithm>
#include <cstdint>
#include <iostream>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "semi_local.h"
#include "approximate_matching/utils.h"
#include "approximate_matching/ApproximateMatching.h"

namespace {
template <class Search>
int run(const int32_t *p, int m, const int32_t *t, int n, double k, int32_t *starts, int32_t *ends, double *scores,
        int cap) {
    std::vector<int> pv(p, p + m), tv(t, t + n);
    std::vector<approximate_matching::utils::Interval> out;
    Search s;
    s.find(pv.data(), m, tv.data(), n, k, out);
    const int cnt = (int) out.size();
    for (int i = 0; i < cnt && i < cap; ++i) {
        starts[i] = out[i].start;
        ends[i] = out[i].end;
        scores[i] = out[i].score;
    }
    return cnt;
}
}  // namespace

extern "C" {
// InteractiveDuplicateSearchSemiDense::find / InteractiveDuplicateSearchSemiSparse::find on int symbols
int ref_dup_search_dense(const int32_t *p, int m, const int32_t *t, int n, double k, int32_t *starts, int32_t *ends,
                         double *scores, int cap) {
    return run<InteractiveDuplicateSearchSemiDense>(p, m, t, n, k, starts, ends, scores, cap);
}
int ref_dup_search_sparse(const int32_t *p, int m, const int32_t *t, int n, double k, int32_t *starts, int32_t *ends,
                          double *scores, int cap) {
    return run<InteractiveDuplicateSearchSemiSparse>(p, m, t, n, k, starts, ends, scores, cap);
}
}
