// slcs.hpp -- header-only C++ adapter over the C ABI of libslcs.so (include/slcs.h).
//
// The classes have the shapes of the reference's strategy interfaces (NikitaMishin/semilocal, R: = source/cpu/):
//   GpuIterativeCombing / GpuHybridCombing::compute(a, aSize, b, bSize, kernel)
//                                   semi_local::SemiLocalStrategy<Input>::compute   R:include/SemiLocal/SemiLocalLCS.h:7-11
//   GpuSteadyAnt::multiply(p, q, res)
//                                   common::BraidMultiplicationStrategy::multiply   R:common/include/Permutations/MongeMultuplicationStrategy.h:18-21
//   GpuStaggeredGlue::glue(p, q, rowGlue, res)
//                                   StaggeredStickyBraidMultiplication::staggeredStickyMultiplication
//                                   R:common/include/Permutations/MongeMultuplicationStrategy.h:679-758
//   GpuLCS::compute(a, aSize, b, bSize) -> int
//                                   lcs::LCSStrategy<Input>::compute                 R:include/LCS/LCS.h:9-13
//   GpuBitParallelLCS::compute(...) -> int
//                                   prefix_lcs_via_semi_local::nary::llcs_nary_symbol_smart_combing
//                                   R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:668-736
// They are templates over the permutation type: slcs::Permutation below (the shape of common::Permutation,
// R:common/include/Permutations/Matrices.h:16-96) or the reference's own common::Permutation -- anything with
// a (rows, cols) constructor, public rows/cols/m/n, set(row, col) and getColByRow(row).  A reference subclass of
// SemiLocalStrategy / MemoryOptimizedStickBraidMultiplication forwards its virtual to these in a few lines
// (tests/cpp/reference_plugin.cpp does so).  Failures throw slcs::Error (status code + message); the engine never
// exits or aborts.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <algorithm>
#include <vector>

#include "slcs.h"

namespace slcs {

constexpr int kNoPoint = -1;   // the reference's NOPOINT

class Error : public std::runtime_error {
public:
    Error(int code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc) {
    if (rc != SLCS_OK) {
        const char *m = slcs_last_error();
        throw Error(rc, std::string("slcs status ") + std::to_string(rc) + ": " + (m ? m : ""));
    }
}

// Both maps of a permutation matrix, as the reference keeps them; m, n tag a braid's pair lengths.
class Permutation {
public:
    Permutation() = default;
    Permutation(int rows_, int cols_)
        : rows(rows_), cols(cols_), row_to_col_(rows_ > 0 ? rows_ : 0, kNoPoint),
          col_to_row_(cols_ > 0 ? cols_ : 0, kNoPoint) {}
    void set(int row, int col) {
        row_to_col_[row] = col;
        col_to_row_[col] = row;
    }
    int getColByRow(int row) const { return row_to_col_[row]; }
    int getRowByCol(int col) const { return col_to_row_[col]; }
    bool operator==(const Permutation &o) const {
        return rows == o.rows && cols == o.cols && row_to_col_ == o.row_to_col_ && col_to_row_ == o.col_to_row_;
    }
    bool operator!=(const Permutation &o) const { return !(*this == o); }
    const std::vector<int> &rowToCol() const { return row_to_col_; }
    const std::vector<int> &colToRow() const { return col_to_row_; }

    int m = 0;
    int n = 0;
    int rows = 0;
    int cols = 0;

private:
    std::vector<int> row_to_col_;
    std::vector<int> col_to_row_;
};

// Permutation-like <-> row->col arrays
template <class Perm>
std::vector<int32_t> row_to_col_of(const Perm &p) {
    std::vector<int32_t> r(p.rows > 0 ? p.rows : 0);
    for (int i = 0; i < p.rows; ++i) r[i] = p.getColByRow(i);
    return r;
}

template <class Perm>
void assign_from(Perm &out, const std::vector<int32_t> &r2c, int rows, int cols) {
    out = Perm(rows, cols);
    for (int i = 0; i < rows; ++i)
        if (r2c[i] != kNoPoint) out.set(i, r2c[i]);
}

template <class Perm>
void assign_braid(Perm &kernel, const std::vector<int32_t> &r2c, int m, int n) {
    assign_from(kernel, r2c, m + n, m + n);
    kernel.m = m;
    kernel.n = n;
}

namespace detail {
// Symbols as the C ABI takes them: uint8 as is, anything else widened to int32 (compared for equality only).
template <class Input>
int comb(const Input *a, int m, const Input *b, int n, int32_t *r2c, int32_t *score, const slcs_opts &o) {
    if (std::is_same<Input, uint8_t>::value || std::is_same<Input, unsigned char>::value)
        return slcs_comb_u8(reinterpret_cast<const uint8_t *>(a), m, reinterpret_cast<const uint8_t *>(b), n, r2c,
                            nullptr, score, &o);
    if (std::is_same<Input, int32_t>::value)
        return slcs_comb_i32(reinterpret_cast<const int32_t *>(a), m, reinterpret_cast<const int32_t *>(b), n, r2c,
                             nullptr, score, &o);
    std::vector<int32_t> aa(a, a + m), bb(b, b + n);
    return slcs_comb_i32(aa.data(), m, bb.data(), n, r2c, nullptr, score, &o);
}
}  // namespace detail

// Sticky-braid combing of (a, b) into the braid `kernel` (rows = cols = m+n, tags m, n), any algorithm.
template <class Input, class Perm = Permutation>
class GpuCombing {
public:
    explicit GpuCombing(int algo = SLCS_ALGO_AUTO, int band_rows = 0, int tile_rows = 0, int tile_cols = 0) {
        opts_ = slcs_opts{};
        opts_.algo = algo;
        opts_.band_rows = band_rows;
        opts_.tile_rows = tile_rows;
        opts_.tile_cols = tile_cols;
    }
    void compute(const Input *a, int aSize, const Input *b, int bSize, Perm &kernel) const {
        std::vector<int32_t> r2c((size_t) aSize + bSize > 0 ? (size_t) aSize + bSize : 1);
        int32_t score = 0;
        check(detail::comb(a, aSize, b, bSize, r2c.data(), &score, opts_));
        assign_braid(kernel, r2c, aSize, bSize);
    }
    // The global LLCS of the last pair is also available directly.
    int score(const Input *a, int aSize, const Input *b, int bSize) const {
        std::vector<int32_t> r2c((size_t) aSize + bSize > 0 ? (size_t) aSize + bSize : 1);
        int32_t s = 0;
        check(detail::comb(a, aSize, b, bSize, r2c.data(), &s, opts_));
        return s;
    }

private:
    slcs_opts opts_;
};

// The reference's AntidiagonalIterativeCombing / OpenMPIterativeCombing role (R:include/SemiLocal/SemiLocalLCS.h:128-304)
template <class Input, class Perm = Permutation>
class GpuIterativeCombing : public GpuCombing<Input, Perm> {
public:
    explicit GpuIterativeCombing(int band_rows = 0) : GpuCombing<Input, Perm>(SLCS_ALGO_WAVEFRONT, band_rows) {}
};

// The reference's OpenMPHybridIterative role (R:include/SemiLocal/SemiLocalLCS.h:594-792): tiles combed
// independently and glued by the steady ant.
template <class Input, class Perm = Permutation>
class GpuHybridCombing : public GpuCombing<Input, Perm> {
public:
    explicit GpuHybridCombing(int tile_rows = 0, int tile_cols = 0)
        : GpuCombing<Input, Perm>(SLCS_ALGO_HYBRID, 0, tile_rows, tile_cols) {}
};

// Unit-Monge (distance) product of two n x n permutations: the steady ant.
template <class Perm = Permutation>
class GpuSteadyAnt {
public:
    void multiply(const Perm &p, const Perm &q, Perm &res) const {
        if (p.rows != q.rows) throw Error(SLCS_ERR_ARG, "permutation sizes differ");
        const int n = p.rows;
        std::vector<int32_t> pp = row_to_col_of(p), qq = row_to_col_of(q), rr(n > 0 ? n : 1);
        check(slcs_steady_ant(pp.data(), qq.data(), n, rr.data(), nullptr));
        assign_from(res, rr, n, n);
    }
};

// Gluing of the braids of two adjacent grid blocks (tags m, n): rowGlue = p above q (sharing p.n = q.n column
// strands), else p left of q (sharing p.m = q.m row strands).  The result is the braid of the union.
template <class Perm = Permutation>
class GpuStaggeredGlue {
public:
    void glue(const Perm &p, const Perm &q, bool rowGlue, Perm &res) const {
        std::vector<int32_t> pp = row_to_col_of(p), qq = row_to_col_of(q);
        const int m = rowGlue ? p.m + q.m : p.m, n = rowGlue ? p.n : p.n + q.n;
        std::vector<int32_t> rr(m + n > 0 ? m + n : 1);
        check(slcs_staggered_glue(pp.data(), p.m, p.n, qq.data(), q.m, q.n, rowGlue ? 1 : 0, rr.data()));
        assign_braid(res, rr, m, n);
    }
};

// LCS length through the braid (the reference's LCSBySemiLocal, R:include/LCS/LCS.h:216-238).
template <class Input>
class GpuLCS {
public:
    int compute(const Input *a, int aSize, const Input *b, int bSize) const {
        return GpuCombing<Input>(SLCS_ALGO_AUTO).score(a, aSize, b, bSize);
    }
};

// LLCS by bit-parallel combing; symbols must be < 4.
class GpuBitParallelLCS {
public:
    template <class Input>
    int compute(const Input *a, int aSize, const Input *b, int bSize) const {
        std::vector<uint8_t> aa(a, a + aSize), bb(b, b + bSize);
        int32_t s = 0;
        check(slcs_bitcomb_llcs_u8(aa.data(), aSize, bb.data(), bSize, &s));
        return s;
    }
};

// An interval of the text and its score, the fields of the reference's approximate_matching::utils::Interval
// (R:approximate_matching/utils.h:233-253).
struct Interval {
    int start;
    int end;
    double score;
    int len() const { return end - start; }
};

// InteractiveDuplicateSearchSemiDense / ...SemiSparse shape (R:approximate_matching/ApproximateMatching.h:252-420):
// find(p, p_size, text, text_size, k, result) appends the same intervals the reference's find does.
template <bool Sparse>
class GpuDuplicateSearch {
public:
    template <class T>
    void find(const T *p, int p_size, const T *text, int text_size, double k, std::vector<Interval> &result) const {
        std::vector<int32_t> pp(p, p + p_size), tt(text, text + text_size);
        int cap = text_size / std::max(int(p_size * k), 1) + 2;   // picked intervals: disjoint, >= int(m k) long
        std::vector<slcs_interval> out;
        int cnt = 0;
        for (;;) {
            out.resize(cap);
            check(Sparse ? slcs_duplicate_search_sparse_i32(pp.data(), p_size, tt.data(), text_size, k, out.data(), cap,
                                                            &cnt)
                         : slcs_duplicate_search_i32(pp.data(), p_size, tt.data(), text_size, k, out.data(), cap, &cnt));
            if (cnt <= cap) break;
            cap = cnt;
        }
        for (int i = 0; i < cnt; ++i) result.push_back(Interval{out[i].start, out[i].end, out[i].score});
    }
};
using GpuDuplicateSearchSemiDense = GpuDuplicateSearch<false>;
using GpuDuplicateSearchSemiSparse = GpuDuplicateSearch<true>;

// Scores read from a braid: SLCS_Q_* queries (global, string-substring, prefix-suffix, ...).
template <class Perm>
std::vector<int32_t> scores(const Perm &braid, const std::vector<slcs_query> &qs) {
    std::vector<int32_t> r2c = row_to_col_of(braid), out(qs.empty() ? 1 : qs.size());
    check(slcs_scores(r2c.data(), braid.m, braid.n, qs.data(), (int) qs.size(), out.data()));
    out.resize(qs.size());
    return out;
}

}  // namespace slcs
