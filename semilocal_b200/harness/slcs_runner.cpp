// slcs_runner.cpp -- the engine behind the reference's benchmark harness.
//
// The reference times its implementations as executables driven by utils/runners.py (CombingRunner, LcsRunner:
// R:utils/runners.py:41-76): argv = [threads, path_a, path_b]; the input files are the .fna format of
// R:parsers.h:38-47 (line 1 name, line 2 length, line 3 comma-separated symbols); stdout is exactly seven lines
// without a trailing newline: preprocess ms, algorithm ms, result, |a|, |b|, name a, name b
// (R:cpu_impl/semi_local_hybrid_iterative.cpp:53-59).  The result is the braid's hash of R:test_utils.h:8-18
// (combing; col->row entries folded as h = (R h + x) mod M in 64-bit signed arithmetic) or the LCS score.
// Built twice: -DSLCS_RUNNER_LCS prints the score, otherwise the hash.  The thread count is accepted and ignored.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "slcs.h"

namespace {

struct Seq {
    std::string name;
    std::vector<int32_t> sym;
};

bool read_fna(const char *path, Seq &out) {
    std::ifstream f(path);
    if (!f) return false;
    std::string len, body;
    if (!std::getline(f, out.name) || !std::getline(f, len) || !std::getline(f, body)) return false;
    const long n = std::stol(len);
    out.sym.reserve(n > 0 ? n : 0);
    size_t i = 0;
    while (i < body.size() && (long) out.sym.size() < n) {
        size_t j = body.find(',', i);
        if (j == std::string::npos) j = body.size();
        if (j > i) out.sym.push_back((int32_t) std::stol(body.substr(i, j - i)));
        i = j + 1;
    }
    return (long) out.sym.size() == n;
}

// R:test_utils.h:8-18 with the reference's two's-complement wrap-around made explicit
long long braid_hash(const std::vector<int32_t> &col_to_row) {
    const long long R = 4294967279LL, M = 4294967291LL;
    long long h = 0;
    for (int32_t x : col_to_row) {
        const long long t = (long long) ((unsigned long long) R * (unsigned long long) h + (unsigned long long) (long long) x);
        h = t % M;
    }
    return h;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s threads path_a path_b\n", argv[0]);
        return 2;
    }
    Seq a, b;
    if (!read_fna(argv[2], a) || !read_fna(argv[3], b)) {
        std::fprintf(stderr, "cannot read the input files\n");
        return 2;
    }
    const int m = (int) a.sym.size(), n = (int) b.sym.size();
    std::vector<int32_t> r2c(m + n > 0 ? m + n : 1), c2r(m + n > 0 ? m + n : 1);
    int32_t score = 0;
    // the first call initialises the engine (context, pools): the preprocess time, as the reference reports
    // its own set-up (precalc) there
    const auto t0 = std::chrono::high_resolution_clock::now();
    int rc = slcs_comb_i32(a.sym.data(), m, b.sym.data(), n, r2c.data(), c2r.data(), &score, nullptr);
    const auto t1 = std::chrono::high_resolution_clock::now();
    if (rc == SLCS_OK) rc = slcs_comb_i32(a.sym.data(), m, b.sym.data(), n, r2c.data(), c2r.data(), &score, nullptr);
    const auto t2 = std::chrono::high_resolution_clock::now();
    if (rc != SLCS_OK) {
        const char *msg = slcs_last_error();
        std::fprintf(stderr, "slcs status %d: %s\n", rc, msg ? msg : "");
        return 1;
    }
    const long pre = (long) std::chrono::duration<double, std::milli>(t1 - t0).count();
    const long algo = (long) std::chrono::duration<double, std::milli>(t2 - t1).count();
    c2r.resize(m + n);
#ifdef SLCS_RUNNER_LCS
    const long long result = score;
#else
    const long long result = braid_hash(c2r);
#endif
    std::cout << pre << '\n' << algo << '\n' << result << '\n' << m << '\n' << n << '\n' << a.name << '\n' << b.name;
    return 0;
}
