// amatch_oracle.cpp -- TEST INFRASTRUCTURE ONLY: host restatement of the reference's approximate pattern search,
// InteractiveDuplicateSearchSemiDense::find (R:approximate_matching/ApproximateMatching.h:320-420), step for step
// (and ...SemiSparse::find, :252-318, further down):
//   * one braid of the pattern against the text (row-major combing, slo_comb_rowmajor in slcs_oracle.c);
//   * the triangle of the last window (calculateTriangle, ApproximateMatching.h:137-184): for each interval end
//     j = n - kk, the best interval over starts walking down the column;
//   * the window sliding left one start at a time with the ring of per-end maxima (:346-406);
//   * the distinct candidates reversed, sorted and picked greedily (phase3, :186-200).
// Scores use the reference's fixed scheme (match 0, mismatch -2, gap -1; R:approximate_matching/utils.h:195-230)
// whose blow-up factor is 1: score(i, j) = 2 (j - i - D) - (m + j - i), with the dominance sum
// D = #{strands s >= m + i : row_to_col[s] < j} moved up, down and left as in
// R:unit_monge_mult/dominance_sum_queries.h:84-118.  C++ because the pick sorts with std::sort, whose order of
// equal keys the result depends on.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_set>
#include <vector>

extern "C" void slo_comb_rowmajor(const int32_t *a, int m, const int32_t *b, int n, int32_t *row_to_col);

namespace {

struct Iv {
    int start, end;
    double score;
    int len() const { return end - start; }
};

constexpr double kNegInf = -10000000.0;

// the reference's compare(): higher score, then longer
bool better(const Iv &a, const Iv &b) {
    if (a.score > b.score) return true;
    if (a.score < b.score) return false;
    return a.len() > b.len();
}

}  // namespace

// The greedy pick (phase3, ApproximateMatching.h:186-200); returns the number of intervals, writing at most cap.
static int pick(std::vector<Iv> &cands, int32_t *starts, int32_t *ends, double *scores, int cap) {
    std::sort(cands.begin(), cands.end(), [](const Iv &a, const Iv &b) {
        return (a.start < b.start) || (a.start == b.start && a.score > b.score);
    });
    int lb = 0, rb = 0, cnt = 0;
    for (const Iv &c : cands) {
        if (c.start > lb && c.start >= rb) {
            if (cnt < cap) {
                starts[cnt] = c.start;
                ends[cnt] = c.end;
                scores[cnt] = c.score;
            }
            ++cnt;
            lb = c.start;
            rb = std::max(rb, c.end);
        }
    }
    return cnt;
}

// The edit distance of the reference's first phase (DuplicateSearch::editDistance, ApproximateMatching.h:18-53):
// match 0, substitution 2, indel 1, negated.
static double edit_score(const int32_t *a, int na, const int32_t *b, int nb) {
    std::vector<double> prev(nb + 1), cur(nb + 1);
    for (int j = 0; j <= nb; ++j) prev[j] = j;
    for (int i = 1; i <= na; ++i) {
        cur[0] = i;
        for (int j = 1; j <= nb; ++j)
            cur[j] = std::min(a[i - 1] == b[j - 1] ? prev[j - 1] : 2.0 + prev[j - 1], 1.0 + std::min(prev[j], cur[j - 1]));
        std::swap(prev, cur);
    }
    return -prev[nb];
}

// InteractiveDuplicateSearchSemiSparse::find (ApproximateMatching.h:252-318): the first phase walks the window ends,
// skipping ahead by half the score deficit; each clone (a window scoring at least kdi) is combed against the
// pattern on its own and its triangle (calculateTriangle, offset 0, the whole clone) gives the clone's interval.
extern "C" int slo_duplicate_search_sparse(const int32_t *p, int m, const int32_t *t, int n, double k,
                                           int32_t *starts, int32_t *ends, double *scores, int cap) {
    if (m <= 0 || n <= 0 || !(k > 0.0 && k <= 1.0)) return -1;
    const int w = int(m / k);
    const int left_w = int(m * k) - 1;
    const double kdi = -(m * (1 / k + 1) * (1 - k * k));
    if (w > n) return -1;
    std::vector<Iv> clones;
    for (int end = w; end < n + 1;) {
        const double dist = edit_score(t + (end - w), w, p, m);
        if (dist >= kdi) clones.push_back(Iv{end - w, end, dist});
        if (dist < kdi - 1) end += std::max(1, int((std::abs(dist) - std::abs(kdi)) / 2));
        else ++end;
    }
    std::vector<Iv> cands;
    std::unordered_set<long long> seen;
    std::vector<int32_t> r2c(m + w), c2r(m + w);
    for (const Iv &cl : clones) {
        slo_comb_rowmajor(p, m, t + cl.start, w, r2c.data());
        for (int s = 0; s < m + w; ++s) c2r[r2c[s]] = s;
        // D(0, w) of the clone from its score: w - LCS, LCS = (score + m + w) / 2 (getRangeSumFromReverse)
        int dcol = static_cast<int>(std::lround(w - (cl.score + m + w) / 2.0));
        Iv wmax{0, 0, kNegInf};
        for (int kk = 0; kk < w - left_w; ++kk) {
            const int j = w - kk;
            int d = dcol;
            Iv best{0, 0, kNegInf};
            for (int tt = 0; tt < (w - kk) - left_w; ++tt) {
                const Iv c{tt, j, 2.0 * (j - tt - d) - (m + j - tt)};
                if (c.score > best.score || (c.score == best.score && c.len() > best.len())) best = c;
                if (r2c[m + tt] < j) --d;
            }
            if (better(best, wmax)) wmax = best;
            if (c2r[j - 1] >= m) --dcol;
        }
        const Iv shifted{wmax.start + cl.start, wmax.end + cl.start, wmax.score};
        const long long key = (static_cast<long long>(shifted.start) << 32) | static_cast<unsigned>(shifted.end);
        if (seen.insert(key).second) cands.push_back(shifted);
    }
    return pick(cands, starts, ends, scores, cap);
}

// Returns the number of intervals (writing at most cap of them), -1 for bad arguments.
extern "C" int slo_duplicate_search(const int32_t *p, int m, const int32_t *t, int n, double k, int32_t *starts,
                                    int32_t *ends, double *scores, int cap) {
    if (m <= 0 || n <= 0 || !(k > 0.0 && k <= 1.0)) return -1;
    const int w = int(m / k);
    const int left_w = int(m * k) - 1;
    const double kdi = -(m * (1 / k + 1) * (1 - k * k));
    if (w > n) return -1;
    const int S = w - left_w;
    std::vector<int32_t> r2c(m + n), c2r(m + n);
    slo_comb_rowmajor(p, m, t, n, r2c.data());
    for (int s = 0; s < m + n; ++s) c2r[r2c[s]] = s;
    // D(row, col) moves; rows are strand indices m + i
    auto down = [&](int row, int col, int v) { return (row < m + n && r2c[row] < col) ? v - 1 : v; };
    auto up = [&](int row, int col, int v) { return (row > 0 && r2c[row - 1] < col) ? v + 1 : v; };
    auto left = [&](int row, int col, int v) { return (col > 0 && c2r[col - 1] >= row) ? v - 1 : v; };
    auto score = [&](int i, int j, int d) { return 2.0 * (j - i - d) - (m + j - i); };

    std::vector<Iv> ring(S, Iv{0, 0, kNegInf});
    std::vector<Iv> cands;
    std::unordered_set<long long> seen;
    auto key = [](const Iv &v) { return (static_cast<long long>(v.start) << 32) | static_cast<unsigned>(v.end); };

    // ---- the last window [n - w, n): its triangle ----
    const int offset = n - w;
    int diag = 0;   // D(m + offset, n)
    for (int s = m + offset; s < m + n; ++s) diag += r2c[s] < n;
    Iv wmax{0, 0, kNegInf};
    {
        int dcol = diag;   // D(m + offset, j) for the column's end j
        for (int kk = 0; kk < S; ++kk) {
            const int j = n - kk;
            int d = dcol;
            Iv best{0, 0, kNegInf};
            for (int tt = 0; tt < (w - kk) - left_w; ++tt) {   // starts offset + tt, longest first
                const int i = offset + tt;
                const Iv c{i, j, score(i, j, d)};
                if (c.score > best.score || (c.score == best.score && c.len() > best.len())) best = c;
                d = down(m + i, j, d);
            }
            ring[kk] = best;
            if (better(best, wmax)) wmax = best;
            dcol = left(m + offset, j, dcol);
        }
    }
    if (score(offset, n, diag) >= kdi) {
        cands.push_back(wmax);
        seen.insert(key(wmax));
    }
    diag = left(m + offset - 1, n, up(m + offset, n, diag));   // the window [offset - 1, n - 1)

    // ---- windows [i, i + w) for i = offset - 1 .. 0 ----
    int head = 0;
    for (int start = 1; start <= n - w; ++start) {
        ring[head] = Iv{0, 0, kNegInf};
        head = (head + 1) % S;
        const int i = n - w - start, j = n - start;
        const double wdist = score(i, j, diag);
        int drow = diag;
        int r = j;
        Iv wm{0, 0, kNegInf};
        for (int mm = 0; mm < S; ++mm, --r) {
            Iv &slot = ring[(head + mm) % S];
            const Iv c{i, r, score(i, r, drow)};
            if (better(c, slot)) slot = c;
            if (better(slot, wm)) wm = slot;
            drow = left(m + i, r, drow);
        }
        if (wdist >= kdi && seen.insert(key(wm)).second) cands.push_back(wm);
        diag = left(m + i, j, diag);
        diag = up(m + i, j - 1, diag);
    }
    std::reverse(cands.begin(), cands.end());
    return pick(cands, starts, ends, scores, cap);
}
