// CPU check of the approximate search's host steps (semilocal_b200/csrc/amatch_pick.h) against a plain restatement of
// the reference's steps: a comparison sort by window start, std::unordered_set for the distinct intervals, the
// sort by (start, score descending) and the greedy pick (R:approximate_matching/ApproximateMatching.h:186-200,
// 261-272, 346-406).  Random candidate sets with many repeated intervals and ties of (start, score), in the arbitrary
// order the device's atomics leave them; and the map of int32 symbols away from the combing kernel's reserved codes.
// Prints "ok <cases>" or the first mismatch.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <unordered_set>
#include <vector>

#include "amatch_pick.h"

using slcs::am::Cand;
using slcs::am::Iv;

static std::vector<Iv> plain_dense(std::vector<Cand> c) {
    std::sort(c.begin(), c.end(), [](const Cand &x, const Cand &y) { return x.i < y.i; });
    std::vector<Iv> out;
    std::unordered_set<long long> seen;
    for (int q = static_cast<int>(c.size()) - 1; q >= 0; --q) {
        const long long key = (static_cast<long long>(c[q].start) << 32) | static_cast<unsigned>(c[q].end);
        if (seen.insert(key).second) out.push_back(Iv{c[q].start, c[q].end, static_cast<double>(c[q].score)});
    }
    std::reverse(out.begin(), out.end());
    return out;
}

static bool plain_sparse(std::vector<Cand> c, const std::vector<int> &lcs, int m, int n, int w, double kdi,
                         std::vector<Iv> *out) {
    std::sort(c.begin(), c.end(), [](const Cand &x, const Cand &y) { return x.i < y.i; });
    std::unordered_set<long long> seen;
    out->clear();
    for (int end = w; end < n + 1;) {
        const double dist = 2.0 * lcs[end - w] - m - w;
        if (dist >= kdi) {
            const Cand *hit = nullptr;
            for (const Cand &x : c)
                if (x.i == end - w) hit = &x;
            if (!hit) return false;
            const long long key = (static_cast<long long>(hit->start) << 32) | static_cast<unsigned>(hit->end);
            if (seen.insert(key).second) out->push_back(Iv{hit->start, hit->end, static_cast<double>(hit->score)});
        }
        if (dist < kdi - 1) end += std::max(1, int((std::abs(dist) - std::abs(kdi)) / 2));
        else ++end;
    }
    return true;
}

static std::vector<Iv> plain_pick(std::vector<Iv> cand) {
    std::sort(cand.begin(), cand.end(), [](const Iv &a, const Iv &b) {
        return (a.start < b.start) || (a.start == b.start && a.score > b.score);
    });
    std::vector<Iv> out;
    int left = 0, right = 0;
    for (const Iv &c : cand)
        if (c.start > left && c.start >= right) {
            out.push_back(c);
            left = c.start;
            right = std::max(right, c.end);
        }
    return out;
}

static bool same(const std::vector<Iv> &a, const std::vector<Iv> &b) {
    if (a.size() != b.size()) return false;
    for (size_t k = 0; k < a.size(); ++k)
        if (a[k].start != b[k].start || a[k].end != b[k].end || a[k].score != b[k].score) return false;
    return true;
}

int main() {
    std::mt19937_64 rng(12345);
    int cases = 0;
    for (int trial = 0; trial < 400; ++trial) {
        // window starts 0..N-1 (every tenth case past 2^22, so that the radix sort takes three passes)
        const int N = trial % 10 == 9 ? (1 << 22) + 77 : 1 + static_cast<int>(rng() % 20000);
        const int m = 5 + static_cast<int>(rng() % 40), w = m + static_cast<int>(rng() % 12);
        const double kdi = -static_cast<double>(rng() % 30);
        // a small pool of intervals, so that windows repeat intervals and (start, score) ties are common
        const int pool = 1 + static_cast<int>(rng() % 60);
        std::vector<Iv> ivs;
        for (int k = 0; k < pool; ++k) {
            const int st = static_cast<int>(rng() % 200), len = 1 + static_cast<int>(rng() % 9);
            ivs.push_back(Iv{st, st + len, static_cast<double>(static_cast<int>(rng() % 4))});
        }
        // window scores: most windows under the bar, runs of windows over it
        std::vector<int> lcs(N);
        for (int s = 0; s < N; ++s)
            lcs[s] = static_cast<int>(std::floor((m + w - 5.0 + kdi) / 2.0)) - static_cast<int>(rng() % 4);
        const int runs = static_cast<int>(rng() % 12);
        for (int r = 0; r < runs; ++r) {
            const int s0 = static_cast<int>(rng() % N), len = 1 + static_cast<int>(rng() % 300);
            for (int s = s0; s < std::min(N, s0 + len); ++s) lcs[s] = m;
        }
        std::vector<Cand> c;
        for (int s = 0; s < N; ++s)
            if (2.0 * lcs[s] - m - w >= kdi) {
                const Iv &v = ivs[rng() % ivs.size()];
                c.push_back(Cand{s, v.start, v.end, static_cast<int>(v.score)});
            }
        std::shuffle(c.begin(), c.end(), rng);
        std::vector<Cand> sorted = c;
        slcs::am::sort_by_window(sorted);
        for (size_t k = 1; k < sorted.size(); ++k)
            if (sorted[k - 1].i >= sorted[k].i) {
                printf("trial %d: window order broken at %zu\n", trial, k);
                return 1;
            }
        // dense: the candidate list itself, then the pick with a small output capacity
        const std::vector<Iv> got = slcs::am::dense_candidates(sorted), exp = plain_dense(c);
        if (!same(got, exp)) {
            printf("trial %d: dense candidate lists differ (%zu vs %zu)\n", trial, got.size(), exp.size());
            return 1;
        }
        std::vector<Iv> picked, gcopy = got;
        const int cap = static_cast<int>(rng() % 8);
        const int cnt = slcs::am::greedy_pick(gcopy, cap, [&](int, const Iv &v) { picked.push_back(v); });
        const std::vector<Iv> pexp = plain_pick(exp);
        if (cnt != static_cast<int>(pexp.size()) ||
            !same(picked, std::vector<Iv>(pexp.begin(), pexp.begin() + std::min<size_t>(cap, pexp.size())))) {
            printf("trial %d: dense pick differs\n", trial);
            return 1;
        }
        // sparse (the plain walk searches linearly, so only the smaller cases)
        if (N <= 20000) {
            const int n = N + w - 1;
            std::vector<Iv> gs, es;
            const bool okg = slcs::am::sparse_candidates(sorted, lcs.data(), m, n, w, kdi, &gs);
            const bool oke = plain_sparse(c, lcs, m, n, w, kdi, &es);
            if (okg != oke || !same(gs, es)) {
                printf("trial %d: sparse candidate lists differ\n", trial);
                return 1;
            }
            std::vector<Iv> ps;
            const int cs = slcs::am::greedy_pick(gs, 1 << 20, [&](int, const Iv &v) { ps.push_back(v); });
            if (cs != static_cast<int>(ps.size()) || !same(ps, plain_pick(es))) {
                printf("trial %d: sparse pick differs\n", trial);
                return 1;
            }
        }
        ++cases;
    }
    // the map away from the combing kernel's reserved codes: a no-op without them, one-to-one onto 0..k-1 with them
    const int32_t r0 = -0x40000000, r1 = -0x40000001;
    const int32_t pool[] = {r0, r1, r0 + 1, r1 - 1, 0, 7, -7, 2147483647, -2147483647 - 1};
    for (int trial = 0; trial < 200; ++trial) {
        const int m = 1 + static_cast<int>(rng() % 50), n = 1 + static_cast<int>(rng() % 200);
        std::vector<int32_t> p(m), t(n), cp, ct;   // odd trials may draw r0 / r1, even ones never do
        for (auto &v : p) v = pool[2 + rng() % 7];
        for (auto &v : t) v = pool[2 + rng() % 7];
        if (trial % 2) {
            for (int r = 0; r < 3; ++r) p[rng() % m] = pool[rng() % 9];
            for (int r = 0; r < 5; ++r) t[rng() % n] = pool[rng() % 9];
        }
        bool has = false;
        for (int32_t v : p) has |= v == r0 || v == r1;
        for (int32_t v : t) has |= v == r0 || v == r1;
        const bool mapped = slcs::am::dense_codes_if_reserved(p.data(), m, t.data(), n, r0, r1, &cp, &ct);
        if (mapped != has || (!mapped && (!cp.empty() || !ct.empty()))) {
            printf("remap trial %d: mapped %d, reserved codes present %d\n", trial, mapped, has);
            return 1;
        }
        if (!mapped) continue;
        std::vector<int32_t> all(p), codes(cp);
        all.insert(all.end(), t.begin(), t.end());
        codes.insert(codes.end(), ct.begin(), ct.end());
        int32_t hi = -1;
        for (size_t x = 0; x < all.size(); ++x) {
            hi = std::max(hi, codes[x]);
            if (codes[x] < 0 || codes[x] == r0 || codes[x] == r1) {
                printf("remap trial %d: code %d out of range\n", trial, codes[x]);
                return 1;
            }
            for (size_t y = 0; y < all.size(); ++y)
                if ((all[x] == all[y]) != (codes[x] == codes[y])) {
                    printf("remap trial %d: equality not kept\n", trial);
                    return 1;
                }
        }
        std::vector<int32_t> d(all);
        std::sort(d.begin(), d.end());
        if (hi + 1 != static_cast<int32_t>(std::unique(d.begin(), d.end()) - d.begin())) {
            printf("remap trial %d: codes not dense\n", trial);
            return 1;
        }
        ++cases;
    }
    printf("ok %d\n", cases);
    return 0;
}
