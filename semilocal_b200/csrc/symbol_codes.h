// symbol_codes.h -- host-side maps of int32 symbols to the codes the combing kernels take.  Symbols are only ever
// compared for equality (R:include/SemiLocal/SemiLocalLCS.h:153-174), so any one-to-one map of the values present
// gives the same braid.  Host-only C++, included by capi.cu and by the CPU check tests/cpp/symbol_codes_check.cpp.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

namespace slcs {

// When every symbol of a and b lies within 256 consecutive values, fills ca / cb with v - min (uint8) and returns
// true: one pass for the range and one for the codes, no sort.  Otherwise returns false and leaves them untouched.
inline bool range_codes_u8(const int32_t *a, int m, const int32_t *b, int n, std::vector<uint8_t> *ca,
                           std::vector<uint8_t> *cb) {
    if (m + n == 0) return false;
    int32_t lo = m ? a[0] : b[0], hi = lo;
    for (int i = 0; i < m; ++i) {
        lo = std::min(lo, a[i]);
        hi = std::max(hi, a[i]);
    }
    for (int i = 0; i < n; ++i) {
        lo = std::min(lo, b[i]);
        hi = std::max(hi, b[i]);
    }
    if (static_cast<int64_t>(hi) - lo > 255) return false;
    ca->resize(m);
    cb->resize(n);
    for (int i = 0; i < m; ++i) (*ca)[i] = static_cast<uint8_t>(static_cast<int64_t>(a[i]) - lo);
    for (int i = 0; i < n; ++i) (*cb)[i] = static_cast<uint8_t>(static_cast<int64_t>(b[i]) - lo);
    return true;
}

}  // namespace slcs
