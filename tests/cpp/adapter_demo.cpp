// Drives the C++ adapter (include/slcs.hpp) the way the reference's tests drive its strategies
// (R:Google_tests/SemiLocalLCSTest.cpp:26-44, SteadyAntTest.cpp:26-40, LCSTest.cpp:35-60): inputs come from
// stdin, every result is printed for the Python side to compare with the oracle.
//
//   stdin: m n, a[0..m), b[0..n), k, p[0..k), q[0..k)
//   stdout: one line per result: "comb <r2c...>", "hybrid <r2c...>", "score <s>", "lcs <s>", "bit <s>",
//           "sa <r...>", "glue <r2c...>", "queries <q...>", "dup <start end score ...>"; or "error <code> <message>"
#include <algorithm>
#include <iostream>
#include <vector>

#include "slcs.hpp"

template <class V>
static void print(const char *tag, const V &v) {
    std::cout << tag;
    for (auto x : v) std::cout << ' ' << x;
    std::cout << '\n';
}

int main() {
    int m = 0, n = 0, k = 0;
    std::cin >> m >> n;
    std::vector<int> a(m), b(n);
    for (auto &x : a) std::cin >> x;
    for (auto &x : b) std::cin >> x;
    std::cin >> k;
    std::vector<int> p(k), q(k);
    for (auto &x : p) std::cin >> x;
    for (auto &x : q) std::cin >> x;
    try {
        slcs::Permutation braid, hyb;
        slcs::GpuIterativeCombing<int>().compute(a.data(), m, b.data(), n, braid);
        print("comb", slcs::row_to_col_of(braid));
        slcs::GpuHybridCombing<int>(256, 256).compute(a.data(), m, b.data(), n, hyb);
        print("hybrid", slcs::row_to_col_of(hyb));
        std::cout << "same " << (braid == hyb ? 1 : 0) << '\n';
        std::cout << "lcs " << slcs::GpuLCS<int>().compute(a.data(), m, b.data(), n) << '\n';
        std::cout << "bit " << slcs::GpuBitParallelLCS().compute(a.data(), m, b.data(), n) << '\n';
        auto qs = slcs::scores(braid, {{SLCS_Q_GLOBAL, 0, 0}, {SLCS_Q_STRING_SUBSTRING, n / 4, n / 2},
                                       {SLCS_Q_PREFIX_SUFFIX, m / 3, n / 5}});
        print("queries", qs);
        slcs::Permutation P, Q, R;
        std::vector<int32_t> pv(p.begin(), p.end()), qv(q.begin(), q.end());
        slcs::assign_from(P, pv, k, k);
        slcs::assign_from(Q, qv, k, k);
        slcs::GpuSteadyAnt<>().multiply(P, Q, R);
        print("sa", slcs::row_to_col_of(R));
        // glue the braids of the top and bottom halves of a back into the braid of the whole pair
        const int h = m / 2;
        slcs::Permutation top, bot, whole;
        slcs::GpuIterativeCombing<int>().compute(a.data(), h, b.data(), n, top);
        slcs::GpuIterativeCombing<int>().compute(a.data() + h, m - h, b.data(), n, bot);
        slcs::GpuStaggeredGlue<>().glue(top, bot, true, whole);
        print("glue", slcs::row_to_col_of(whole));
        // approximate copies of a's first 40 symbols in b (InteractiveDuplicateSearchSemiDense::find's shape)
        std::vector<slcs::Interval> dup;
        slcs::GpuDuplicateSearchSemiDense().find(a.data(), std::min(m, 40), b.data(), n, 0.8, dup);
        std::vector<long> flat;
        for (const auto &iv : dup) {
            flat.push_back(iv.start);
            flat.push_back(iv.end);
            flat.push_back(static_cast<long>(iv.score));
        }
        print("dup", flat);
    } catch (const slcs::Error &e) {
        std::cout << "error " << e.code() << ' ' << e.what() << '\n';
        return 3;
    }
    return 0;
}
