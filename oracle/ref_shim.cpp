// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// An extern "C" face over the reference's own C++ headers (NikitaMishin/semilocal, source/cpu/), compiled in
// place by oracle/build_ref.sh into oracle/_ref/libslcs_ref.so.  Used (1) to pin the C restatement in
// oracle/slcs_oracle.c, (2) to generate tests/golden/ vectors, (3) as the "reference" CPU baseline that
// bench.py times beside the GPU.  Nothing in the product library links or loads it.
//
// Each wrapper calls the reference class or function it names, unmodified; only argument marshalling
// (raw arrays <-> common::Permutation) is done here.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <unordered_map>
#include <unordered_set>
#include <iostream>
#include <vector>
#include <cstdint>
#include <cstdio>
#include <unistd.h>
#include <fcntl.h>
#include <omp.h>

#include "common/include/Permutations/Matrices.h"
#include "common/include/Permutations/MongeMultuplicationStrategy.h"
#include "include/SemiLocal/SemiLocalLCS.h"
#include "include/LCS/LCS.h"
#include "prefix_lcs/bitwise/encoders_and_decoders.h"
#include "prefix_lcs/bitwise/transposition_network_binary_alphabet.h"

// The reference declares these virtual members without a body (SemiLocalLCS.h:10, LCS.h:12); a shared
// library needs a definition for the base vtables.  They are never called.
template<> void semi_local::SemiLocalStrategy<int>::compute(const int *, int, const int *, int, common::Permutation &) noexcept {}
template<> int lcs::LCSStrategy<int>::compute(const int *, int, const int *, int) { return -1; }

namespace {
void to_array(const common::Permutation &p, int32_t *out) {
    for (int i = 0; i < p.rows; ++i) out[i] = p.getColByRow(i);
}
common::Permutation from_array(const int32_t *r2c, int n) {
    common::Permutation p(n, n);
    for (int i = 0; i < n; ++i) if (r2c[i] >= 0) p.set(i, r2c[i]);
    return p;
}
common::PrecalcMap &precalc(int size) {
    static common::PrecalcMap maps[8];
    static bool built[8] = {false};
    if (size < 0) size = 0;
    if (size > 7) size = 7;
    if (!built[size]) {
        common::NaiveBraidMultiplication naive;
        if (size > 0) common::StickyBraidMultiplication::buildPrecalcMap(&naive, maps[size], size);
        built[size] = true;
    }
    return maps[size];
}
// The n-ary bit routine prints its sizes to stdout (transposition_network_binary_alphabet.h:674);
// keep the caller's stdout clean.
struct QuietStdout {
    int saved = -1;
    QuietStdout() {
        fflush(stdout);
        std::cout.flush();
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        if (devnull >= 0) { dup2(devnull, 1); close(devnull); }
    }
    ~QuietStdout() {
        std::cout.flush();
        fflush(stdout);
        if (saved >= 0) { dup2(saved, 1); close(saved); }
    }
};
}  // namespace

extern "C" {

// SimpleIterativeCombing<int,false> (SemiLocalLCS.h:65-126).
int ref_comb_simple(const int *a, int m, const int *b, int n, int32_t *out) {
    semi_local::SimpleIterativeCombing<int, false> s;
    common::Permutation k;
    s.compute(a, m, b, n, k);
    to_array(k, out);
    return 0;
}

// OpenMPIterativeCombing<int,false>(threads) (SemiLocalLCS.h:231-306).
int ref_comb_openmp(const int *a, int m, const int *b, int n, int threads, int32_t *out) {
    semi_local::OpenMPIterativeCombing<int, false> s(threads);
    common::Permutation k;
    s.compute(a, m, b, n, k);
    to_array(k, out);
    return 0;
}

// DummyPrefixLCSStrategy<int>(-2) (SemiLocalLCS.h:13-63): the DP-defined kernel.
int ref_comb_dummy(const int *a, int m, const int *b, int n, int32_t *out) {
    semi_local::DummyPrefixLCSStrategy<int> s(-2);
    common::Permutation k;
    s.compute(a, m, b, n, k);
    to_array(k, out);
    return 0;
}

// OpenMPIterativeCombingCombined<int,false> (SemiLocalLCS.h:308-476) glued by the sequential steady ant.
int ref_comb_combined(const int *a, int m, const int *b, int n, int threads, int32_t *out) {
    common::PrecalcMap empty;
    common::SequentialMemoryOptimizedStickBraidMultiplication gluer(empty);
    common::StaggeredStickyBraidMultiplication staggered(&gluer);
    semi_local::OpenMPIterativeCombingCombined<int, false> s(threads, &staggered);
    common::Permutation k;
    s.compute(a, m, b, n, k);
    to_array(k, out);
    return 0;
}

// OpenMPHybridIterative<int,false>(threads, cols, rows, staggered, leaf OpenMPIterativeCombing(1))
// (SemiLocalLCS.h:594-794) with SequentialMemoryOptimizedStickBraidMultiplication glue.
int ref_hybrid_iterative(const int *a, int m, const int *b, int n, int threads, int cols, int rows, int precalc_size,
                         int32_t *out) {
    common::SequentialMemoryOptimizedStickBraidMultiplication gluer(precalc(precalc_size));
    common::StaggeredStickyBraidMultiplication staggered(&gluer);
    semi_local::OpenMPIterativeCombing<int, false> leaf(1);
    semi_local::OpenMPHybridIterative<int, false> s(threads, cols, rows, &staggered, &leaf);
    common::Permutation k;
    s.compute(a, m, b, n, k);
    to_array(k, out);
    return 0;
}

// OpenMPHybridRecursive<int,false,true,true>(parallel_depth, staggered, depth, sum_bound, leaf)
// (SemiLocalLCS.h:478-585).
int ref_hybrid_recursive(const int *a, int m, const int *b, int n, int parallel_depth, int depth, int sum_bound,
                         int32_t *out) {
    common::PrecalcMap empty;
    common::SequentialMemoryOptimizedStickBraidMultiplication gluer(empty);
    common::StaggeredStickyBraidMultiplication staggered(&gluer);
    semi_local::OpenMPIterativeCombing<int, false> leaf(1);
    semi_local::OpenMPHybridRecursive<int, false, true, true> s(parallel_depth, &staggered, depth, sum_bound, &leaf);
    common::Permutation k;
    s.compute(a, m, b, n, k);
    to_array(k, out);
    return 0;
}

// NaiveBraidMultiplication (MongeMultuplicationStrategy.h:28-55).
int ref_braid_naive(const int32_t *p, const int32_t *q, int n, int32_t *out) {
    common::NaiveBraidMultiplication s;
    common::Permutation res;
    s.multiply(from_array(p, n), from_array(q, n), res);
    to_array(res, out);
    return 0;
}

// SimpleStickyBraidMultiplication(precalc) (MongeMultuplicationStrategy.h:326-398).
int ref_braid_simple(const int32_t *p, const int32_t *q, int n, int precalc_size, int32_t *out) {
    common::SimpleStickyBraidMultiplication s(precalc(precalc_size));
    common::Permutation res;
    s.multiply(from_array(p, n), from_array(q, n), res);
    to_array(res, out);
    return 0;
}

// SequentialMemoryOptimizedStickBraidMultiplication(precalc) (MongeMultuplicationStrategy.h:548-594).
int ref_braid_seq(const int32_t *p, const int32_t *q, int n, int precalc_size, int32_t *out) {
    common::SequentialMemoryOptimizedStickBraidMultiplication s(precalc(precalc_size));
    common::Permutation res;
    s.multiply(from_array(p, n), from_array(q, n), res);
    to_array(res, out);
    return 0;
}

// OpenMPStickyBraid(depth, precalc) (MongeMultuplicationStrategy.h:597-673).
int ref_braid_omp(const int32_t *p, const int32_t *q, int n, int depth, int precalc_size, int32_t *out) {
    omp_set_nested(1);
    common::OpenMPStickyBraid s(depth, precalc(precalc_size));
    common::Permutation res;
    s.multiply(from_array(p, n), from_array(q, n), res);
    to_array(res, out);
    return 0;
}

// Build the precalc tables up front so that timing excludes them (the reference's drivers report the
// precalc time separately, e.g. cpu_impl/semi_local_hybrid_iterative.cpp:144-147).
int ref_precalc_warm(int size) { precalc(size); return 0; }

// StaggeredStickyBraidMultiplication::staggeredStickyMultiplication<RowGlue> (MongeMultuplicationStrategy.h:679-758).
int ref_staggered(const int32_t *p, int pm, int pn, const int32_t *q, int qm, int qn, int row_glue, int32_t *out) {
    common::PrecalcMap empty;
    common::SequentialMemoryOptimizedStickBraidMultiplication gluer(empty);
    common::StaggeredStickyBraidMultiplication s(&gluer);
    common::Permutation P = from_array(p, pm + pn), Q = from_array(q, qm + qn), R;
    P.m = pm; P.n = pn; Q.m = qm; Q.n = qn;
    if (row_glue) s.staggeredStickyMultiplication<true>(P, Q, pn, R);
    else s.staggeredStickyMultiplication<false>(P, Q, pm, R);
    to_array(R, out);
    return 0;
}

// SequentialMemLCS / DummyLCS / LCSBySemiLocal (LCS.h:16-80, 216-238).
int ref_lcs_seqmem(const int *a, int m, const int *b, int n) {
    lcs::SequentialMemLCS<int> s;
    return s.compute(a, m, b, n);
}
int ref_lcs_dummy(const int *a, int m, const int *b, int n) {
    lcs::DummyLCS<int> s;
    return s.compute(a, m, b, n);
}
int ref_lcs_by_semilocal(const int *a, int m, const int *b, int n) {
    semi_local::SimpleIterativeCombing<int, false> comb;
    lcs::LCSBySemiLocal<int> s(&comb);
    return s.compute(a, m, b, n);
}

// Bit-parallel LLCS on the reference's own packing (encode_reverse / encode, encoders_and_decoders.h:50-150):
// nary::llcs_nary_symbol_smart_combing<uint64_t> (transposition_network_binary_alphabet.h:668-736).
// Requires lengths that are multiples of 64/bps and |a| <= |b| (the reference's domain).
int ref_bit_nary_u64(const int *a, int m, const int *b, int n, int alphabet, int threads) {
    std::vector<int> av(a, a + m), bv(b, b + n);
    std::unordered_set<int> alpha;
    for (int s = 0; s < alphabet; ++s) alpha.insert(s);
    auto mappers = encode_alphabet<int, uint64_t>(alpha);
    // identity symbol mapping, so that packed codes equal the symbols
    std::unordered_map<int, uint64_t> fwd;
    std::unordered_map<uint64_t, int> rev;
    for (int s = 0; s < alphabet; ++s) { fwd[s] = (uint64_t) s; rev[(uint64_t) s] = s; }
    (void) mappers;
    auto ar = encode_reverse<int, uint64_t>(av, &fwd, &rev, alphabet);
    auto be = encode<int, uint64_t>(bv, &fwd, &rev, alphabet);
    int bps = int(std::ceil(std::log2(alphabet)));
    int res;
    {
        QuietStdout q;
        res = prefix_lcs_via_semi_local::nary::llcs_nary_symbol_smart_combing<uint64_t>(
                ar.first.first, ar.first.second, be.first.first, be.first.second, ar.second, bps, threads);
    }
    free(ar.first.first);
    free(be.first.first);
    return res;
}

// binary::llcs_2symbol_smart_combing<uint64_t> formula 2 (transposition_network_binary_alphabet.h:598-663).
int ref_bit_binary_u64(const int *a, int m, const int *b, int n, int threads) {
    std::vector<int> av(a, a + m), bv(b, b + n);
    std::unordered_map<int, uint64_t> fwd{{0, 0}, {1, 1}};
    std::unordered_map<uint64_t, int> rev{{0, 0}, {1, 1}};
    auto ar = encode_reverse<int, uint64_t>(av, &fwd, &rev, 2);
    auto be = encode<int, uint64_t>(bv, &fwd, &rev, 2);
    int res = prefix_lcs_via_semi_local::binary::llcs_2symbol_smart_combing<uint64_t>(
            ar.first.first, ar.first.second, be.first.first, be.first.second, ar.second, threads, false);
    free(ar.first.first);
    free(be.first.first);
    return res;
}

// lllcs_hyyro::preprocess + hyyro_magic<uint64_t> (threads == 1) or hyyro_magic_mpi_with_precalc (threads > 1)
// (transposition_network_binary_alphabet.h:749-914): the bit vector runs over `vec` (its lookup tables), the loop over
// `seq`.  The anti-diagonal form assumes more symbols in `seq` than words in `vec`.
int ref_hyyro_u64(const int *vec, int nv, const int *seq, int ns, int threads) {
    if (nv == 0 || ns == 0) return 0;
    std::unordered_set<int> alpha(vec, vec + nv);
    alpha.insert(seq, seq + ns);
    std::unordered_map<int, uint64_t *> lookup;
    lllcs_hyyro::preprocess<uint64_t>(vec, nv, alpha, lookup);
    const int words = (nv + 63) / 64;
    std::vector<int> sv(seq, seq + ns);
    int res = threads > 1 ? lllcs_hyyro::hyyro_magic_mpi_with_precalc<uint64_t>(sv.data(), ns, words, lookup, threads)
                          : lllcs_hyyro::hyyro_magic<uint64_t>(sv.data(), ns, words, lookup);
    for (auto &kv : lookup) delete[] kv.second;
    return res;
}

int ref_available(void) { return 1; }

}  // extern "C"
