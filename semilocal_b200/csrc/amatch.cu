// amatch.cu -- approximate pattern search (duplicate search) on the braid of a pattern against a text.
//
// The reference's InteractiveDuplicateSearchSemiDense::find (R:approximate_matching/ApproximateMatching.h:320-420)
// combs the pattern p (m symbols) against the whole text t (n symbols) once and slides a window of w = int(m / k)
// symbols over the text from its end to its start.  With the reference's fixed scoring (match 0, mismatch -2,
// gap -1: R:approximate_matching/utils.h:195-230, whose blow-up factor is 1) an interval's score is
//   score(i, j) = 2 LCS(p, t[i, j)) - m - (j - i)            (minus the indel distance of p and t[i, j)),
// read from the braid as LCS(p, t[i, j)) = (j - i) - D(i, j), D(i, j) = #{strands s >= m + i : row_to_col[s] < j}
// (the string-substring dominance sum, R:approximate_matching/utils.h:262-330).  At window start i (n - w down to
// 0) the reference keeps, for each interval end r of the window, the best interval ending at r (a ring of per-end
// maxima fed with the new start, ApproximateMatching.h:364-392) and takes the best of them; that is W(i), the
// interval inside [i, i + w] of length at least L = int(m k) that is largest by (score, length, end).  W(i) is a
// candidate when the window's own score(i, i + w) reaches kdi = -(m (1/k + 1)(1 - k^2)); the distinct candidates,
// in that order, are reversed, sorted by (start, score descending) and picked greedily without overlap
// (ApproximateMatching.h:186-200).
//
// Here the braid comes from the combing engine (the hybrid with one tile row: a short pattern against a long
// text), D(i, i + w) for every start from the window scan, and W(i) from am_window_kernel: the starts are cut into
// chunks and one warp walks its chunk from the top like the reference's ring, entering S - 1 starts above the
// chunk (S = w - L + 1 ends per window) so that every end's maximum is complete when the chunk begins.  Per end it
// keeps D(i, r) (one more strand per step: + [row_to_col[m + i] < r]; a new end from its neighbour:
// D(i, r) = D(i, r + 1) - [col_to_row[r] >= m + i]) and the best interval.  The candidates, their dedup, the sort
// and the greedy pick run on the host (amatch_pick.h), with the same sort as the reference so that equal keys land
// alike.
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "amatch_pick.h"
#include "slcs_internal.cuh"

namespace slcs {
namespace {

constexpr int kAmMaxEnds = 16384;   // ends a window can hold (w - L + 1): three ints each in shared memory
constexpr int kAmBits = 21;         // lengths and end offsets below 2^21 pack into the comparison key

// (score, length, end - i) packed so that integer order is the reference's order of intervals
__device__ __forceinline__ long long am_key(int score, int len, int rel) {
    return (static_cast<long long>(score) << (2 * kAmBits)) + (static_cast<long long>(len) << kAmBits) + rel;
}

__device__ __forceinline__ long long warp_max64(long long v) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v = max(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// W(i) of a start whose window reaches the threshold joins the candidate list (unordered: (i, start, end, score))
__device__ __forceinline__ void am_emit(const int32_t *wlcs, int m, int w, double kdi, int i, long long b,
                                        int *ncand, int4 *cand, int cap) {
    if (2.0 * wlcs[i] - m - w < kdi) return;   // the window's own score, as the reference computes it
    const int rel = static_cast<int>(b & ((1 << kAmBits) - 1));
    const int len = static_cast<int>((b >> kAmBits) & ((1 << kAmBits) - 1));
    const int pos = atomicAdd(ncand, 1);
    if (pos < cap) cand[pos] = make_int4(i, i + rel - len, i + rel, static_cast<int>(b >> (2 * kAmBits)));
}

// One warp per chunk of `chunk` window starts.  Shared memory: D, best start and best score of every end, indexed
// by end mod S.  Candidates (see am_emit) go to cand[0 .. *ncand).
__global__ void __launch_bounds__(32) am_window_kernel(const int32_t *__restrict__ r2c, const int32_t *__restrict__ c2r,
                                                       const int32_t *__restrict__ wlcs, int m, int n, int w, int L,
                                                       int chunk, double kdi, int *__restrict__ ncand,
                                                       int4 *__restrict__ cand, int cap) {
    extern __shared__ int am_smem[];
    const int S = w - L + 1;
    int *D = am_smem, *bs = am_smem + S, *bsc = am_smem + 2 * S;
    const int lane = threadIdx.x;
    const int nstart = n - w + 1;   // window starts 0 .. n - w
    const int i_lo = blockIdx.x * chunk;
    if (i_lo >= nstart) return;
    const int i_hi = min(i_lo + chunk, nstart) - 1;
    const int i_top = min(i_hi + S - 1, n - L);   // every end active at i_hi enters at or below i_top
    // ---- the state at i_top: ends [lo, hi], each with the one start i_top ----
    int lo = i_top + L;
    const int hi0 = min(i_top + w, n);
    int dtop;   // D(i_top, hi0)
    if (hi0 == i_top + w) {
        dtop = w - wlcs[i_top];   // the window scan: LCS(p, t[i, i + w)) = w - D(i, i + w)
    } else {                      // past the last window: strands s >= m + i_top leaving through the bottom
        dtop = 0;
        for (int s0 = m + i_top; s0 < m + n; s0 += 32) {
            const int s = s0 + lane;
            dtop += __popc(__ballot_sync(kFull, s < m + n && r2c[s] < n));
        }
    }
    long long best = LLONG_MIN;
    {
        // D(i_top, r) = dtop - #{c in [r, hi0) : col_to_row[c] >= m + i_top}, by 32 columns from the top
        int run = 0;
        for (int c0 = hi0; c0 >= lo; c0 -= 32) {
            const int c = c0 - lane;   // lane 0: column c0 (the end hi0 itself when c0 == hi0)
            const bool in = c >= lo;
            const bool q = in && c < hi0 && c2r[c] >= m + i_top;
            const unsigned msk = __ballot_sync(kFull, q);
            const int before = run + __popc(msk & ((1u << lane) - 1u));   // columns in (c, hi0) counted
            if (in) {
                const int d = dtop - before - (q ? 1 : 0);
                const int slot = c % S;
                const int sc = (c - i_top) - m - 2 * d;
                D[slot] = d;
                bs[slot] = i_top;
                bsc[slot] = sc;
                best = max(best, am_key(sc, c - i_top, c - i_top));
            }
            run += __popc(msk);
        }
    }
    if (i_top <= i_hi) {
        const long long b = warp_max64(best);
        if (lane == 0) am_emit(wlcs, m, w, kdi, i_top, b, ncand, cand, cap);
    }
    __syncwarp();
    // ---- steps i = i_top - 1 .. i_lo: strand m + i joins, end i + L enters, end i + 1 + w leaves ----
    int base = lo % S;   // ring slot of the lowest end
    int tv = 0, cv = 0;
    for (int i = i_top - 1, j = 32; i >= i_lo; --i, ++j) {
        if (j == 32) {   // the next 32 steps' strand ends and column starts, one per lane
            const int ii = i - lane;
            tv = ii >= 0 ? r2c[m + ii] : 0;
            cv = ii >= 0 ? c2r[ii + L] : 0;
            j = 0;
        }
        const int t = __shfl_sync(kFull, tv, j);    // row_to_col[m + i]
        const int cin = __shfl_sync(kFull, cv, j);  // col_to_row[i + L]
        lo = i + L;
        const int hi = min(i + w, n);
        base = base == 0 ? S - 1 : base - 1;
        const int d1 = D[base == S - 1 ? 0 : base + 1];   // D(i + 1, lo + 1), before this step's updates
        __syncwarp();
        best = LLONG_MIN;
        for (int q = lane; q < S; q += 32) {
            int rel = q - base;
            if (rel < 0) rel += S;
            const int r = lo + rel;
            if (r > hi) continue;
            int d, st, sc;
            if (rel == 0) {   // the entering end
                d = d1 + (t < lo + 1 ? 1 : 0) - (cin >= m + i ? 1 : 0);
                sc = (r - i) - m - 2 * d;
                st = i;
            } else {
                d = D[q] + (t < r ? 1 : 0);
                const int cand = (r - i) - m - 2 * d;
                sc = bsc[q];
                st = bs[q];
                if (cand >= sc) {   // equal scores: the new start gives the longer interval
                    sc = cand;
                    st = i;
                }
            }
            D[q] = d;
            bs[q] = st;
            bsc[q] = sc;
            best = max(best, am_key(sc, r - st, r - i));
        }
        __syncwarp();
        if (i <= i_hi) {
            const long long b = warp_max64(best);
            if (lane == 0) am_emit(wlcs, m, w, kdi, i, b, ncand, cand, cap);
        }
    }
}

// sparse = false: InteractiveDuplicateSearchSemiDense (every window start, from the end of the text);
// sparse = true: InteractiveDuplicateSearchSemiSparse (R:approximate_matching/ApproximateMatching.h:252-318): the
// windows its first phase visits (it skips ahead by half the score deficit), each a clone whose best interval is
// the triangle of the clone's own braid -- the same interval W(start), read here from the one braid of the text.
template <typename T>
int duplicate_search(const T *pattern, int m, const T *text, int n, double k, bool sparse, slcs_interval *out,
                     int cap, int *n_out) {
    if (!n_out || m <= 0 || n <= 0 || !pattern || !text || cap < 0 || (cap > 0 && !out))
        return fail(SLCS_ERR_ARG, "bad arguments");
    if (!(k > 0.0 && k <= 1.0)) return fail(SLCS_ERR_ARG, "k must lie in (0, 1]");
    *n_out = 0;
    // the reference's window and threshold (R:approximate_matching/ApproximateMatching.h:333-335)
    const int w = int(m / k);
    const int left_w = int(m * k) - 1;
    const double kdi = -(m * (1 / k + 1) * (1 - k * k));
    const int L = left_w + 1, S = w - L + 1;
    if (w > n) return fail(SLCS_ERR_ARG, "text shorter than the window int(m / k)");
    if (S > kAmMaxEnds || w >= (1 << kAmBits)) return fail(SLCS_ERR_TOO_LARGE, "window too wide");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = E->stream;
    NvtxRange nv("slcs: duplicate search");
    const int nstart = n - w + 1;
    DevBuf<T> dp, dt;
    DevBuf<int32_t> r2c, c2r, wl;
    DevBuf<int4> dc;
    DevBuf<int> dn;
    SLCS_TRY(dp.alloc(m, s));
    SLCS_TRY(dt.alloc(n, s));
    SLCS_TRY(r2c.alloc(m + n, s));
    SLCS_TRY(c2r.alloc(m + n, s));
    SLCS_TRY(wl.alloc(nstart, s));
    SLCS_TRY(dn.alloc(1, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(dn.p, 0, sizeof(int), s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(dp.p, pattern, sizeof(T) * m, cudaMemcpyHostToDevice, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(dt.p, text, sizeof(T) * n, cudaMemcpyHostToDevice, s));
    // a short pattern against a long text: one row of tiles, glued on the pattern's m strands
    slcs_opts o{};
    o.algo = SLCS_ALGO_HYBRID;
    o.tile_rows = m;
    o.tile_cols = 4096;
    SLCS_TRY(comb_dev<T>(E, dp.p, m, dt.p, n, r2c.p, c2r.p, nullptr, &o, s));
    SLCS_TRY(window_scores_dev(r2c.p, c2r.p, m, n, w, wl.p, s));
    const int chunk = std::max(1024, 4 * S);
    const size_t smem = sizeof(int) * 3 * (size_t) S;
    if (smem > 48 * 1024)
        SLCS_CUDA_TRY(cudaFuncSetAttribute(am_window_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    // candidate list: sized for the usual case, grown and rerun in the rare case of more windows over the bar
    int capc = std::min(nstart, 1 << 16), ncand = 0;
    std::vector<am::Cand> C;
    for (;;) {
        SLCS_TRY(dc.alloc(capc, s));
        am_window_kernel<<<(nstart + chunk - 1) / chunk, 32, smem, s>>>(r2c.p, c2r.p, wl.p, m, n, w, L, chunk, kdi,
                                                                        dn.p, dc.p, capc);
        SLCS_CUDA_TRY(cudaGetLastError());
        SLCS_CUDA_TRY(cudaMemcpyAsync(&ncand, dn.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        SLCS_CUDA_TRY(cudaStreamSynchronize(s));
        if (ncand <= capc) break;
        capc = ncand;
        dc.release();
        SLCS_CUDA_TRY(cudaMemsetAsync(dn.p, 0, sizeof(int), s));
    }
    C.resize(ncand);
    if (ncand) SLCS_CUDA_TRY(cudaMemcpyAsync(C.data(), dc.p, sizeof(int4) * ncand, cudaMemcpyDeviceToHost, s));
    std::vector<int32_t> lcs(sparse ? nstart : 0);   // the sparse walk reads every visited window's score
    if (sparse) SLCS_CUDA_TRY(cudaMemcpyAsync(lcs.data(), wl.p, sizeof(int32_t) * nstart, cudaMemcpyDeviceToHost, s));
    SLCS_CUDA_TRY(cudaStreamSynchronize(s));
    // candidates in the reference's order (dense: starts from n - w down; sparse: its first-phase walk), distinct by
    // (start, end), then the reference's sort and greedy pick
    am::sort_by_window(C);
    std::vector<am::Iv> cand;
    if (!sparse) cand = am::dense_candidates(C);
    else if (!am::sparse_candidates(C, lcs.data(), m, n, w, kdi, &cand))
        return fail(SLCS_ERR_INTERNAL, "window missing from the list");
    const int cnt =
        am::greedy_pick(cand, cap, [&](int k, const am::Iv &c) { out[k] = slcs_interval{c.start, c.end, c.score}; });
    *n_out = cnt;
    return SLCS_OK;
}

// int32 symbols go to the combing kernel as they are, unless they hold one of its two reserved padding codes: then
// pattern and text are mapped to dense codes (a one-to-one map, so every match and every result stays the same).
int duplicate_search_i32(const int32_t *pattern, int m, const int32_t *text, int n, double k, bool sparse,
                         slcs_interval *out, int cap, int *n_out) {
    if (m > 0 && n > 0 && pattern && text && (long long) m + n < (1ll << 30)) {
        std::vector<int32_t> cp, ct;
        if (am::dense_codes_if_reserved(pattern, m, text, n, kSymRowVirtual, kSymColVirtual, &cp, &ct))
            return duplicate_search<int32_t>(cp.data(), m, ct.data(), n, k, sparse, out, cap, n_out);
    }
    return duplicate_search<int32_t>(pattern, m, text, n, k, sparse, out, cap, n_out);
}

}  // namespace
}  // namespace slcs

using namespace slcs;

extern "C" {

int slcs_duplicate_search_u8(const uint8_t *pattern, int m, const uint8_t *text, int n, double k, slcs_interval *out,
                             int out_cap, int *n_out) {
    return duplicate_search<uint8_t>(pattern, m, text, n, k, false, out, out_cap, n_out);
}

int slcs_duplicate_search_i32(const int32_t *pattern, int m, const int32_t *text, int n, double k,
                              slcs_interval *out, int out_cap, int *n_out) {
    return duplicate_search_i32(pattern, m, text, n, k, false, out, out_cap, n_out);
}

int slcs_duplicate_search_sparse_u8(const uint8_t *pattern, int m, const uint8_t *text, int n, double k,
                                    slcs_interval *out, int out_cap, int *n_out) {
    return duplicate_search<uint8_t>(pattern, m, text, n, k, true, out, out_cap, n_out);
}

int slcs_duplicate_search_sparse_i32(const int32_t *pattern, int m, const int32_t *text, int n, double k,
                                     slcs_interval *out, int out_cap, int *n_out) {
    return duplicate_search_i32(pattern, m, text, n, k, true, out, out_cap, n_out);
}

}  // extern "C"
