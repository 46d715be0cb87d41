// CPU check of the int32 symbol map of the combing entry point (semilocal_b200/csrc/symbol_codes.h): it applies
// exactly when the symbols span at most 256 values, and then keeps every equality and inequality between symbols,
// with codes in 0..255.  Prints "ok <cases>" or the first mismatch.
#include <climits>
#include <cstdio>
#include <map>
#include <random>
#include <vector>

#include "symbol_codes.h"

int main() {
    std::mt19937_64 rng(7);
    int cases = 0;
    const int32_t bases[] = {0, -7, INT_MIN, INT_MAX - 255, INT_MAX - 300, -1000000, 123456789};
    for (int trial = 0; trial < 2000; ++trial) {
        const int m = static_cast<int>(rng() % 60), n = static_cast<int>(rng() % 60);
        const int32_t base = bases[rng() % 7];
        const int64_t span = trial % 3 == 0 ? 300 : 1 + static_cast<int64_t>(rng() % 256);   // values base .. base+span-1
        std::vector<int32_t> a(m), b(n);
        auto draw = [&]() {
            int64_t v = static_cast<int64_t>(base) + static_cast<int64_t>(rng() % static_cast<uint64_t>(span));
            return static_cast<int32_t>(std::min<int64_t>(v, INT_MAX));
        };
        for (auto &v : a) v = draw();
        for (auto &v : b) v = draw();
        int64_t lo = INT64_MAX, hi = INT64_MIN;
        for (int32_t v : a) lo = std::min<int64_t>(lo, v), hi = std::max<int64_t>(hi, v);
        for (int32_t v : b) lo = std::min<int64_t>(lo, v), hi = std::max<int64_t>(hi, v);
        const bool expect = m + n > 0 && hi - lo <= 255;
        std::vector<uint8_t> ca, cb;
        const bool got = slcs::range_codes_u8(a.data(), m, b.data(), n, &ca, &cb);
        if (got != expect) {
            printf("trial %d: applies %d, expected %d\n", trial, got, expect);
            return 1;
        }
        if (!got) {
            if (!ca.empty() || !cb.empty()) {
                printf("trial %d: outputs written although the map does not apply\n", trial);
                return 1;
            }
            continue;
        }
        std::map<int32_t, int> code_of;
        std::map<int, int32_t> value_of;
        for (int k = 0; k < m + n; ++k) {
            const int32_t v = k < m ? a[k] : b[k - m];
            const int c = k < m ? ca[k] : cb[k - m];
            if (code_of.count(v) && code_of[v] != c) {
                printf("trial %d: one value, two codes\n", trial);
                return 1;
            }
            if (value_of.count(c) && value_of[c] != v) {
                printf("trial %d: one code, two values\n", trial);
                return 1;
            }
            code_of[v] = c;
            value_of[c] = v;
        }
        ++cases;
    }
    printf("ok %d\n", cases);
    return 0;
}
