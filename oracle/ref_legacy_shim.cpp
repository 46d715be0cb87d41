// ref_legacy_shim.cpp -- TEST INFRASTRUCTURE ONLY: an extern "C" face over the reference's legacy implementations
// (NikitaMishin/semilocal, source/cpu/semi_local.h and source/cpu/unit_monge_mult/steady_ant.h), compiled in place
// from the reference tree by oracle/build_ref.sh into oracle/_ref/libslcs_ref_legacy.so.
//
// They are the reference's second, independent code for the same algorithms as the refactored headers that
// oracle/ref_shim.cpp wraps: anti-diagonal combing on AbstractPermutation, the nested-parallel steady ant with its
// n log n memory block, and the iterative hybrid on unsigned short strands.  The tests use them as a second oracle
// beside the first (tests/test_oracle.py).  Each wrapper calls the reference function it names, unmodified; only
// raw arrays are converted to and from the legacy Permutation type.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <iostream>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "semi_local.h"

namespace {
void to_array(const AbstractPermutation &p, int32_t *out) {
    for (int i = 0; i < p.row_size; ++i) out[i] = p.get_col_by_row(i);
}
PrecalcMap &precalc_map(int size) {
    static std::mutex mu;
    static PrecalcMap maps[8];
    static bool built[8] = {false};
    std::lock_guard<std::mutex> lk(mu);
    size = std::max(0, std::min(size, 7));
    if (!built[size]) {
        if (size > 0) precalc(maps[size], size);
        built[size] = true;
    }
    return maps[size];
}
}  // namespace

extern "C" {

// semi_local::sticky_braid_mpi<int, false, true> (R:semi_local.h:212-276): the legacy OpenMP anti-diagonal combing,
// with the barrier after every anti-diagonal (WithWait = true).  Without it (WithWait = false, R:semi_local.h:40-65
// leaves the loop `nowait`) the threads race across anti-diagonals; the reference uses that form with one thread
// only (its hybrid's leaves, R:semi_local.h:623).
int ref_legacy_sticky_braid_mpi(const int *a, int m, const int *b, int n, int threads, int32_t *out) {
    Permutation perm(m + n, m + n);
    semi_local::sticky_braid_mpi<int, false, true>(perm, a, m, b, n, threads);
    to_array(perm, out);
    return 0;
}

// distance_unit_monge_product::steady_ant::steady_ant_parallel_wrapper (R:unit_monge_mult/steady_ant.h:811-844):
// nested_lvls 0 = the sequential linear-memory form, > 0 = OpenMP tasks on the top levels; precalc of products up to
// precalc_size (the reference's precalc, steady_ant.h:860-894).
int ref_legacy_steady_ant(const int32_t *p, const int32_t *q, int n, int nested_lvls, int precalc_size, int32_t *out) {
    Permutation P(n, n), Q(n, n), R(n, n);
    for (int i = 0; i < n; ++i) {
        P.set_point(i, p[i]);
        Q.set_point(i, q[i]);
    }
    distance_unit_monge_product::steady_ant::steady_ant_parallel_wrapper(P, Q, R, precalc_map(precalc_size),
                                                                          nested_lvls);
    to_array(R, out);
    return 0;
}

// semi_local::hybrid_iterative_wrapper<false> (R:semi_local.h:740-790): tiles of at most 32000 rows or columns,
// combed by sticky_braid_mpi, glued by staggered_sticky_multiplication; unsigned short symbols.
int ref_legacy_hybrid_iterative(const int *a, int m, const int *b, int n, int threads, int precalc_size,
                                int32_t *out) {
    std::vector<unsigned short> av(a, a + m), bv(b, b + n);
    Permutation perm(m + n, m + n);
    semi_local::hybrid_iterative_wrapper<false>(perm, av.data(), m, bv.data(), n, precalc_map(precalc_size), threads);
    to_array(perm, out);
    return 0;
}

}  // extern "C"
