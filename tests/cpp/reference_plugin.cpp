// The binding a maintainer of the reference adds to run its own code on the GPU engine: subclasses of the
// reference's interfaces that forward to the C++ adapter (include/slcs.hpp), used inside the reference's own
// classes (LCSBySemiLocal, StaggeredStickyBraidMultiplication, OpenMPHybridIterative) and checked against the
// reference's CPU strategies on the same inputs.
//
// Built against the reference headers (R: = source/cpu/) by oracle/build_ref.sh into oracle/_ref/ -- it embeds
// reference code, so, like the compiled reference, it is test infrastructure and is not committed.
// Prints "ok <checks>" and exits 0 when every GPU result equals the reference's; "mismatch <what>" and 1 else.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "common/include/Permutations/Matrices.h"
#include "common/include/Permutations/MongeMultuplicationStrategy.h"
#include "include/SemiLocal/SemiLocalLCS.h"
#include "include/LCS/LCS.h"
#include "slcs.hpp"

namespace gpu_plugin {

// semi_local::SemiLocalStrategy (R:include/SemiLocal/SemiLocalLCS.h:7-11) on the GPU.  The interface is
// noexcept, as the reference's own strategies are: an engine error ends the process, like their abort().
template <class Input>
class GpuSemiLocal : public semi_local::SemiLocalStrategy<Input> {
public:
    explicit GpuSemiLocal(int algo = SLCS_ALGO_WAVEFRONT) : algo_(algo) {}
    void compute(const Input *a, int aSize, const Input *b, int bSize, common::Permutation &kernel) noexcept override {
        try {
            slcs::GpuCombing<Input, common::Permutation>(algo_, 0, 512, 512).compute(a, aSize, b, bSize, kernel);
        } catch (const slcs::Error &e) {
            std::cerr << e.what() << '\n';
            std::abort();
        }
    }

private:
    int algo_;
};

// A multiplier the reference's StaggeredStickyBraidMultiplication (and through it its hybrids) accepts
// (R:common/include/Permutations/MongeMultuplicationStrategy.h:401-405, 675-677).
class GpuBraidMultiplication : public common::MemoryOptimizedStickBraidMultiplication {
public:
    GpuBraidMultiplication() : common::MemoryOptimizedStickBraidMultiplication(common::PrecalcMap{}) {}
    void multiply(const common::Permutation &p, const common::Permutation &q, common::Permutation &res) override {
        slcs::GpuSteadyAnt<common::Permutation>().multiply(p, q, res);
    }
};

// lcs::LCSStrategy (R:include/LCS/LCS.h:9-13) by bit-parallel combing.
template <class Input>
class GpuBitLCS : public lcs::LCSStrategy<Input> {
public:
    int compute(const Input *a, int sizeA, const Input *b, int sizeB) override {
        return slcs::GpuBitParallelLCS().compute(a, sizeA, b, sizeB);
    }
};

}  // namespace gpu_plugin

namespace {

uint64_t mix(uint64_t &x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

std::vector<int> symbols(int len, uint64_t seed) {
    std::vector<int> v(len);
    for (auto &c : v) c = (int) (mix(seed) & 3);
    return v;
}

common::Permutation random_perm(int n, uint64_t seed) {
    std::vector<int> v(n);
    for (int i = 0; i < n; ++i) v[i] = i;
    for (int i = n - 1; i > 0; --i) std::swap(v[i], v[mix(seed) % (uint64_t) (i + 1)]);
    common::Permutation p(n, n);
    for (int i = 0; i < n; ++i) p.set(i, v[i]);
    return p;
}

int checks = 0;
bool expect(bool ok, const char *what, int x, int y) {
    ++checks;
    if (!ok) std::cout << "mismatch " << what << ' ' << x << ' ' << y << '\n';
    return ok;
}

}  // namespace

int main() {
    bool ok = true;
    gpu_plugin::GpuSemiLocal<int> gpu_wave(SLCS_ALGO_WAVEFRONT), gpu_hyb(SLCS_ALGO_HYBRID);
    semi_local::SimpleIterativeCombing<int, false> cpu_simple;
    const int sizes[][2] = {{1, 1}, {7, 3}, {3, 7}, {100, 130}, {513, 257}, {2000, 1999}, {3001, 2500}};
    uint64_t seed = 1;
    for (auto &mn : sizes) {
        const int m = mn[0], n = mn[1];
        auto a = symbols(m, ++seed), b = symbols(n, ++seed);
        common::Permutation g, h, c;
        gpu_wave.compute(a.data(), m, b.data(), n, g);
        gpu_hyb.compute(a.data(), m, b.data(), n, h);
        cpu_simple.compute(a.data(), m, b.data(), n, c);
        ok &= expect(g == c, "wavefront braid", m, n);
        ok &= expect(h == c, "hybrid braid", m, n);
        // the reference's own score readout on the GPU braid
        lcs::LCSBySemiLocal<int> via_gpu(&gpu_wave), via_cpu(&cpu_simple);
        const int sg = via_gpu.compute(a.data(), m, b.data(), n), sc = via_cpu.compute(a.data(), m, b.data(), n);
        ok &= expect(sg == sc, "LCSBySemiLocal", sg, sc);
        gpu_plugin::GpuBitLCS<int> bit;
        ok &= expect(bit.compute(a.data(), m, b.data(), n) == sc, "bit-parallel LLCS", m, n);
    }
    // the steady ant, alone and as the reference's staggered glue / hybrid multiplier
    gpu_plugin::GpuBraidMultiplication gpu_mult;
    common::SequentialMemoryOptimizedStickBraidMultiplication cpu_mult(common::PrecalcMap{});
    for (int n : {1, 2, 5, 64, 1000, 4096, 10007}) {
        auto p = random_perm(n, 100 + n), q = random_perm(n, 200 + n);
        common::Permutation rg, rc;
        gpu_mult.multiply(p, q, rg);
        cpu_mult.multiply(p, q, rc);
        ok &= expect(rg == rc, "steady ant", n, 0);
    }
    {
        common::StaggeredStickyBraidMultiplication glue_gpu(&gpu_mult), glue_cpu(&cpu_mult);
        semi_local::OpenMPIterativeCombing<int, false> leaf(1);
        semi_local::OpenMPHybridIterative<int, false> hyb_gpu(1, 300, 300, &glue_gpu, &leaf);
        semi_local::OpenMPHybridIterative<int, false> hyb_cpu(1, 300, 300, &glue_cpu, &leaf);
        auto a = symbols(1500, 777), b = symbols(1300, 778);
        common::Permutation kg, kc;
        hyb_gpu.compute(a.data(), 1500, b.data(), 1300, kg);
        hyb_cpu.compute(a.data(), 1500, b.data(), 1300, kc);
        ok &= expect(kg == kc, "reference hybrid with the GPU glue multiplier", 1500, 1300);
    }
    if (ok) std::cout << "ok " << checks << '\n';
    return ok ? 0 : 1;
}
