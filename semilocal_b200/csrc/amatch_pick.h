// amatch_pick.h -- the host steps of the approximate pattern search after the device has produced, for every window
// start over the threshold, its best interval W(i): order by window start, keep the distinct intervals in the
// reference's order, sort them by (start, score descending) and pick greedily without overlap
// (R:approximate_matching/ApproximateMatching.h:186-200, 261-272, 346-406); and the map of int32 symbols away from the
// combing kernel's reserved codes.  Host-only C++, included by amatch.cu and by the CPU check of these steps
// (tests/cpp/amatch_pick_check.cpp).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <vector>

namespace slcs {
namespace am {

// One candidate as the device writes it (16 bytes, the layout of CUDA's int4): window start, interval start,
// interval end, interval score.  A window start appears at most once.
struct Cand {
    int i, start, end, score;
};
static_assert(sizeof(Cand) == 16, "Cand mirrors int4");

struct Iv {
    int start, end;
    double score;
};

// Orders candidates by window start.  The starts are distinct, so every correct sort gives the same order; this
// one is an LSD radix sort on the start (11 bits per pass) instead of a comparison sort.
inline void sort_by_window(std::vector<Cand> &c) {
    const size_t n = c.size();
    if (n < 2) return;
    int hi = 0;
    for (const Cand &x : c) hi = std::max(hi, x.i);
    std::vector<Cand> tmp(n);
    constexpr int kBits = 11, kBuckets = 1 << kBits;
    std::vector<uint32_t> cnt(kBuckets);
    for (int shift = 0; shift < 32; shift += kBits) {
        if (shift > 0 && (static_cast<uint32_t>(hi) >> shift) == 0) break;
        std::fill(cnt.begin(), cnt.end(), 0u);
        for (const Cand &x : c) cnt[(static_cast<uint32_t>(x.i) >> shift) & (kBuckets - 1)]++;
        uint32_t acc = 0;
        for (uint32_t &v : cnt) {
            const uint32_t t = v;
            v = acc;
            acc += t;
        }
        for (const Cand &x : c) tmp[cnt[(static_cast<uint32_t>(x.i) >> shift) & (kBuckets - 1)]++] = x;
        c.swap(tmp);
    }
}

// The set of (start, end) pairs seen so far: open addressing over a power-of-two table of 64-bit keys (start and
// end are non-negative, so -1 marks a free slot).  insert() is true when the pair is new.
class PairSet {
public:
    explicit PairSet(size_t expected) {
        size_t cap = 16;
        while (cap < 2 * expected) cap <<= 1;
        slots_.assign(cap, -1);
        mask_ = cap - 1;
    }
    bool insert(int start, int end) {
        const int64_t key = (static_cast<int64_t>(start) << 32) | static_cast<uint32_t>(end);
        const uint64_t h = static_cast<uint64_t>(key) * 0x9E3779B97F4A7C15ull;
        for (size_t p = (h >> 20) & mask_;; p = (p + 1) & mask_) {
            if (slots_[p] == key) return false;
            if (slots_[p] == -1) {
                slots_[p] = key;
                return true;
            }
        }
    }

private:
    std::vector<int64_t> slots_;
    size_t mask_ = 0;
};

// The dense search's candidate list: window starts from the last down to 0, each distinct (start, end) once (its
// first occurrence in that order), then reversed -- the list the reference builds.  c is ordered by window start.
inline std::vector<Iv> dense_candidates(const std::vector<Cand> &c) {
    std::vector<Iv> out;
    out.reserve(c.size());
    PairSet seen(c.size());
    for (size_t q = c.size(); q-- > 0;) {
        // neighbouring windows mostly share their best interval: a repeat of the one just seen is not new
        if (q + 1 < c.size() && c[q].start == c[q + 1].start && c[q].end == c[q + 1].end) continue;
        if (seen.insert(c[q].start, c[q].end)) out.push_back(Iv{c[q].start, c[q].end, static_cast<double>(c[q].score)});
    }
    std::reverse(out.begin(), out.end());
    return out;
}

// The sparse search's candidate list: the reference's first-phase walk over window ends (ApproximateMatching.h:
// 261-272), reading the window scores lcs[s] = LCS(p, t[s, s + w)); a visited window over the bar is one of the
// candidates in c (ordered by window start), each distinct (start, end) taken once.  False if a visited window over
// the bar is missing from c (the device and the walk disagree).
inline bool sparse_candidates(const std::vector<Cand> &c, const int32_t *lcs, int m, int n, int w, double kdi,
                              std::vector<Iv> *out) {
    PairSet seen(c.size());
    out->clear();
    for (int end = w; end < n + 1;) {
        const double dist = 2.0 * lcs[end - w] - m - w;
        if (dist >= kdi) {
            const auto it = std::lower_bound(c.begin(), c.end(), end - w, [](const Cand &x, int i) { return x.i < i; });
            if (it == c.end() || it->i != end - w) return false;
            if (seen.insert(it->start, it->end)) out->push_back(Iv{it->start, it->end, static_cast<double>(it->score)});
        }
        if (dist < kdi - 1) end += std::max(1, int((std::abs(dist) - std::abs(kdi)) / 2));
        else ++end;
    }
    return true;
}

// The greedy pick (R:approximate_matching/ApproximateMatching.h:186-200): sorted by (start, score descending) with
// the same std::sort the reference uses on the same list, so that equal keys land alike; an interval is taken when
// it starts after the last one taken and at or after every end taken.  Hands at most cap intervals to put(k, iv)
// and returns how many were picked.
template <typename Put>
int greedy_pick(std::vector<Iv> &cand, int cap, Put put) {
    std::sort(cand.begin(), cand.end(), [](const Iv &a, const Iv &b) {
        return (a.start < b.start) || (a.start == b.start && a.score > b.score);
    });
    int left = 0, right = 0, cnt = 0;
    for (const Iv &c : cand) {
        if (c.start > left && c.start >= right) {
            if (cnt < cap) put(cnt, c);
            ++cnt;
            left = c.start;
            right = std::max(right, c.end);
        }
    }
    return cnt;
}

// Symbols are only ever compared for equality, so any one-to-one map of the values keeps every result.  When p or
// t holds one of the two codes r0, r1 that the combing kernel reserves for padding, fills cp / ct with dense codes
// 0..k-1 (k = number of distinct values; equal values get equal codes) and returns true; otherwise returns false and
// leaves them untouched, and the caller passes its symbols as they are.
inline bool dense_codes_if_reserved(const int32_t *p, int m, const int32_t *t, int n, int32_t r0, int32_t r1,
                                    std::vector<int32_t> *cp, std::vector<int32_t> *ct) {
    bool hit = false;
    for (int i = 0; i < m && !hit; ++i) hit = p[i] == r0 || p[i] == r1;
    for (int i = 0; i < n && !hit; ++i) hit = t[i] == r0 || t[i] == r1;
    if (!hit) return false;
    std::vector<int32_t> vals(p, p + m);
    vals.insert(vals.end(), t, t + n);
    std::sort(vals.begin(), vals.end());
    vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
    auto code = [&](int32_t v) {
        return static_cast<int32_t>(std::lower_bound(vals.begin(), vals.end(), v) - vals.begin());
    };
    cp->resize(m);
    ct->resize(n);
    for (int i = 0; i < m; ++i) (*cp)[i] = code(p[i]);
    for (int i = 0; i < n; ++i) (*ct)[i] = code(t[i]);
    return true;
}

}  // namespace am
}  // namespace slcs
