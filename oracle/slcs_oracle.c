/*
 * slcs_oracle.c -- CPU ORACLE (test infrastructure only).
 *
 * A plain-C restatement of the algorithms of NikitaMishin/semilocal that lie on the accelerated path.
 * It is the parity checker for the CUDA engine (tests/, __graft_entry__.smoke()) and the "port" CPU
 * baseline timed by bench.py.  It is never linked into, loaded by, or called from the product library
 * (semilocal_b200/).  Every function names the reference file:line range it restates; paths are relative
 * to the reference project root, `R:` = source/cpu/.
 *
 * Parity of this restatement is pinned against the reference itself: oracle/build_ref.sh compiles the
 * reference's own headers (oracle/ref_shim.cpp) into oracle/_ref/libslcs_ref.so, tests/test_oracle_ref.py
 * compares the two on seeded inputs, and tests/golden/ holds vectors produced by that library.
 *
 * Conventions (shared with the reference):
 *   - a braid (strand permutation) of a pair (a[0..m), b[0..n)) is stored as row_to_col[m+n]:
 *     rows = strand starts (left strands 0..m-1, left strand l enters at row m-1-l of the grid;
 *     top strands m..m+n-1 enter at column r-m), cols = strand ends (bottom exits 0..n-1,
 *     right exits n..n+m-1, right exit n+l is row m-1-l).
 *   - permutations are int32 row->col maps, NOPOINT = -1.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NOPOINT (-1)

/* ------------------------------------------------------------------------------------------------ */
/* Integer sticky-braid combing                                                                     */
/* ------------------------------------------------------------------------------------------------ */

/* Row-major combing, the canonical definition of the braid.
 * Restates R:include/SemiLocal/SemiLocalLCS.h:65-126 (SimpleIterativeCombing::compute), branchless form
 * :97-98, output construction :117-121.  m == 0 or n == 0 give the identity (the reference indexes
 * top_strands[n-1] and is undefined for n == 0). */
void slo_comb_rowmajor(const int32_t *a, int m, const int32_t *b, int n, int32_t *row_to_col) {
    if (m == 0 || n == 0) {
        for (int i = 0; i < m + n; ++i) row_to_col[i] = i;
        return;
    }
    int32_t *top = (int32_t *) malloc(sizeof(int32_t) * (size_t) n);
    int32_t *left = (int32_t *) malloc(sizeof(int32_t) * (size_t) m);
    for (int l = 0; l < m; ++l) left[l] = l;
    for (int j = 0; j < n; ++j) top[j] = m + j;
    for (int i = 0; i < m; ++i) {
        int32_t ls = left[m - 1 - i];
        int32_t sym = a[i];
        for (int j = 0; j < n; ++j) {
            int32_t ts = top[j];
            int swap = (sym == b[j]) || (ls > ts);
            if (swap) { top[j] = ls; ls = ts; }
        }
        left[m - 1 - i] = ls;
    }
    for (int l = 0; l < m; ++l) row_to_col[left[l]] = n + l;
    for (int j = 0; j < n; ++j) row_to_col[top[j]] = j;
    free(top);
    free(left);
}

/* P_{b,a} from P_{a,b}: a 180-degree rotation of the permutation.
 * Restates R:include/SemiLocal/SemiLocalLCS.h:467-473 (fillPermutationBa, "theorem 5.21") and the
 * is_reverse branch of constructPermutation :208-219. */
void slo_rotate180(const int32_t *in, int size, int32_t *out) {
    for (int i = 0; i < size; ++i) {
        int c = in[i];
        if (c != NOPOINT) out[size - 1 - i] = size - 1 - c;
    }
}

/* Anti-diagonal combing with OpenMP threads (strand map of m+n entries, 3 phases, one barrier per
 * diagonal).  Restates R:include/SemiLocal/SemiLocalLCS.h:238-304 (OpenMPIterativeCombing::compute /
 * stickyBraidMpi), cell rule :147-179, initialisation :182-193, output :195-221, a reversed :223-228.
 * If m > n the pair is swapped and the result rotated (:252-255). */
void slo_comb_antidiag(const int32_t *a, int m, const int32_t *b, int n, int threads, int32_t *row_to_col) {
    if (m == 0 || n == 0) {
        for (int i = 0; i < m + n; ++i) row_to_col[i] = i;
        return;
    }
    int reverse = 0;
    if (m > n) {
        const int32_t *t = a; a = b; b = t;
        int tt = m; m = n; n = tt;
        reverse = 1;
    }
    int size = m + n;
    int32_t *strand = (int32_t *) malloc(sizeof(int32_t) * (size_t) size);
    int32_t *arev = (int32_t *) malloc(sizeof(int32_t) * (size_t) m);
    int ndiag = m + n - 1;
    if (threads < 1) threads = 1;
#pragma omp parallel num_threads(threads)
    {
#pragma omp for schedule(static)
        for (int k = 0; k < size; ++k) strand[k] = k;
#pragma omp for schedule(static)
        for (int i = 0; i < m; ++i) arev[i] = a[m - 1 - i];
        /* diagonal d covers cells (row i, col j) with i + j = d; in reversed-a indexing the cells are
         * k = 0..len-1 with left slot left0+k (arev index) and top slot m+top0+k (b index top0+k). */
        for (int d = 0; d < ndiag; ++d) {
            int left0, top0, len;
            if (d < m - 1) {            /* phase 1: growing */
                left0 = m - 1 - d; top0 = 0; len = d + 1;
            } else if (d <= n - 1) {    /* phase 2: full length m */
                left0 = 0; top0 = d - (m - 1); len = m;
            } else {                    /* phase 3: shrinking */
                left0 = 0; top0 = d - (m - 1); len = m - (d - (n - 1));
            }
#pragma omp for schedule(static)
            for (int k = 0; k < len; ++k) {
                int32_t ls = strand[left0 + k];
                int32_t ts = strand[m + top0 + k];
                int r = (arev[left0 + k] == b[top0 + k]) || (ls > ts);
                int32_t rm = (int32_t) r - 1, mr = -(int32_t) r;
                strand[left0 + k] = (ls & rm) | (mr & ts);
                strand[m + top0 + k] = (ts & rm) | (mr & ls);
            }
            /* implicit barrier at the end of the omp for */
        }
    }
    if (!reverse) {
        for (int r = m; r < m + n; ++r) row_to_col[strand[r]] = r - m;
        for (int l = 0; l < m; ++l) row_to_col[strand[l]] = n + l;
    } else {
        for (int r = m; r < m + n; ++r) row_to_col[size - 1 - strand[r]] = size - 1 - (r - m);
        for (int l = 0; l < m; ++l) row_to_col[size - 1 - strand[l]] = size - 1 - (n + l);
    }
    free(strand);
    free(arev);
}

/* ------------------------------------------------------------------------------------------------ */
/* Semi-local matrix from its definition (small sizes only)                                          */
/* ------------------------------------------------------------------------------------------------ */

/* H[i][j] = LCS(a, bExt[i .. j+m)) for bExt = ?^m b ?^m ('?' matches anything), i, j in [0, m+n];
 * entries with j <= i - m are j - i + m.  The braid is the cross-difference permutation of -H.
 * Restates R:include/SemiLocal/SemiLocalLCS.h:13-63 (DummyPrefixLCSStrategy) and
 * R:common/include/Permutations/Matrices.h:116-124 (getCrossDiffPermutation). */
void slo_semilocal_matrix(const int32_t *a, int m, const int32_t *b, int n, int32_t *H /* (m+n+1)^2 */) {
    int size = m + n + 1;
    int ext = m + n + m;
    int32_t *bext = (int32_t *) malloc(sizeof(int32_t) * (size_t) (ext > 0 ? ext : 1));
    int *wild = (int *) malloc(sizeof(int) * (size_t) (ext > 0 ? ext : 1));
    for (int i = 0; i < ext; ++i) { wild[i] = (i < m || i >= m + n); bext[i] = wild[i] ? 0 : b[i - m]; }
    int *row = (int *) malloc(sizeof(int) * (size_t) (ext + 1));
    int *prev = (int *) malloc(sizeof(int) * (size_t) (ext + 1));
    for (int i = 0; i < size; ++i) {
        /* LCS of a against bext[i..] prefixes, all end points at once */
        int len = ext - i;
        for (int j = 0; j <= len; ++j) prev[j] = 0;
        for (int x = 1; x <= m; ++x) {
            row[0] = 0;
            for (int j = 1; j <= len; ++j) {
                int s = i + j - 1;
                int match = wild[s] || a[x - 1] == bext[s];
                int v = prev[j] > row[j - 1] ? prev[j] : row[j - 1];
                int d = prev[j - 1] + (match ? 1 : 0);
                row[j] = v > d ? v : d;
            }
            int *t = prev; prev = row; row = t;
        }
        for (int j = 0; j < size; ++j) {
            if (j <= i - m) H[(size_t) i * size + j] = j - i + m;
            else H[(size_t) i * size + j] = prev[j + m - i];
        }
    }
    free(bext); free(wild); free(row); free(prev);
}

/* Kernel from the semi-local matrix: point (i, j) iff the cross difference of -H is 1. */
void slo_kernel_from_matrix(const int32_t *H, int m, int n, int32_t *row_to_col) {
    int size = m + n + 1;
    for (int i = 0; i < m + n; ++i) row_to_col[i] = NOPOINT;
    for (int i = 0; i + 1 < size; ++i)
        for (int j = 0; j + 1 < size; ++j) {
            int h00 = -H[(size_t) i * size + j], h01 = -H[(size_t) i * size + j + 1];
            int h10 = -H[(size_t) (i + 1) * size + j], h11 = -H[(size_t) (i + 1) * size + j + 1];
            if ((h01 + h10) - (h00 + h11) == 1) row_to_col[i] = j;
        }
}

/* ------------------------------------------------------------------------------------------------ */
/* Scores read from the braid                                                                        */
/* ------------------------------------------------------------------------------------------------ */

/* Global LLCS = m - #{left strands ending on the right border}.
 * Restates R:include/LCS/LCS.h:223-233 (LCSBySemiLocal::compute). */
int slo_global_score(const int32_t *row_to_col, int m, int n) {
    int acc = 0;
    for (int s = 0; s < m; ++s) if (row_to_col[s] >= n) acc++;
    return m - acc;
}

/* Dominance count #{(r, c) in P : r >= i, c < j}; the "top-right summator" of
 * R:common/include/Permutations/MongeMultuplicationStrategy.h:32-34 and
 * R:approximate_matching/utils.h:281-293 (dominanceSumRandom with v = 1). */
long slo_dominance(const int32_t *row_to_col, int size, int i, int j) {
    long cnt = 0;
    for (int r = i; r < size; ++r) if (row_to_col[r] != NOPOINT && row_to_col[r] < j) cnt++;
    return cnt;
}

/* Semi-local matrix entry H(i, j) = j + m - i - #{(r, c) : r >= i, c < j} for i, j in [0, m+n];
 * string-substring LCS(a, b[i..j)) = H(i + m, j) (R:approximate_matching/utils.h:331-334 with v = 1). */
int slo_semilocal_entry(const int32_t *row_to_col, int m, int n, int i, int j) {
    if (j <= i - m) return j - i + m;
    return j + m - i - (int) slo_dominance(row_to_col, m + n, i, j);
}

/* ------------------------------------------------------------------------------------------------ */
/* LCS by dynamic programming                                                                        */
/* ------------------------------------------------------------------------------------------------ */

/* Two-row DP.  Restates R:include/LCS/LCS.h:35-80 (SequentialMemLCS::compute). */
int slo_lcs_dp(const int32_t *a, int m, const int32_t *b, int n) {
    if (m == 0 || n == 0) return 0;
    int *prev = (int *) calloc((size_t) n + 1, sizeof(int));
    int *cur = (int *) calloc((size_t) n + 1, sizeof(int));
    for (int i = 1; i <= m; ++i) {
        int left = 0;
        cur[0] = 0;
        for (int j = 1; j <= n; ++j) {
            int v = prev[j] > left ? prev[j] : left;
            int d = prev[j - 1] + (a[i - 1] == b[j - 1]);
            cur[j] = v > d ? v : d;
            left = cur[j];
        }
        int *t = prev; prev = cur; cur = t;
    }
    int res = prev[n];
    free(prev); free(cur);
    return res;
}

/* ------------------------------------------------------------------------------------------------ */
/* Unit-Monge (sticky braid) multiplication                                                          */
/* ------------------------------------------------------------------------------------------------ */

/* O(n^3) distance product of the dominance ("top-right summator") matrices and its cross difference.
 * Restates R:common/include/Permutations/MongeMultuplicationStrategy.h:28-55 (NaiveBraidMultiplication)
 * with getDominanceSum R:common/include/Permutations/DominanceSum.h:304-320.  p, q: row->col (n). */
void slo_braid_mult_naive(const int32_t *p, const int32_t *q, int n, int32_t *r) {
    int s = n + 1;
    int32_t *dp = (int32_t *) calloc((size_t) s * s, sizeof(int32_t));
    int32_t *dq = (int32_t *) calloc((size_t) s * s, sizeof(int32_t));
    int32_t *dc = (int32_t *) calloc((size_t) s * s, sizeof(int32_t));
    /* D(i, j) = #{rows >= i with col < j}: suffix over rows of per-row prefix indicator */
    for (int i = n - 1; i >= 0; --i)
        for (int j = 0; j < s; ++j) {
            dp[(size_t) i * s + j] = dp[(size_t) (i + 1) * s + j] + (p[i] != NOPOINT && p[i] < j);
            dq[(size_t) i * s + j] = dq[(size_t) (i + 1) * s + j] + (q[i] != NOPOINT && q[i] < j);
        }
    for (int i = 0; i < s; ++i)
        for (int k = 0; k < s; ++k) {
            int best = 0x7fffffff;
            for (int j = 0; j < s; ++j) {
                int v = dp[(size_t) i * s + j] + dq[(size_t) j * s + k];
                if (v < best) best = v;
            }
            dc[(size_t) i * s + k] = best;
        }
    for (int i = 0; i < n; ++i) r[i] = NOPOINT;
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) {
            int cross = (dc[(size_t) i * s + k + 1] + dc[(size_t) (i + 1) * s + k]) -
                        (dc[(size_t) i * s + k] + dc[(size_t) (i + 1) * s + k + 1]);
            if (cross == 1) r[i] = k;
        }
    free(dp); free(dq); free(dc);
}

/* Bump allocator for the recursion scratch (the reference pre-allocates 16n ints likewise,
 * R:common/include/Permutations/MongeMultuplicationStrategy.h:532-545). */
typedef struct { int32_t *base; size_t top, cap; } slo_pool;

static int32_t *pool_take(slo_pool *pl, size_t cnt) {
    if (pl->top + cnt > pl->cap) return NULL;
    int32_t *p = pl->base + pl->top;
    pl->top += cnt;
    return p;
}

/* getVerticalSlice: rows of p (ascending) whose column lies in [lo, hi), compressed.
 * R:common/include/Permutations/MongeMultuplicationStrategy.h:165-176. */
static void slo_vslice(const int32_t *p_r2c, int rows, int lo, int hi, int32_t *rowmap, int32_t *out_r2c,
                       int32_t *out_c2r) {
    int k = 0;
    for (int row = 0; row < rows; ++row) {
        int c = p_r2c[row];
        if (c >= lo && c < hi) {
            rowmap[k] = row;
            out_r2c[k] = c - lo;
            out_c2r[c - lo] = k;
            k++;
        }
    }
}

/* getHorizontalSlice: columns of q (ascending) whose row lies in [lo, hi), compressed.
 * R:common/include/Permutations/MongeMultuplicationStrategy.h:187-198. */
static void slo_hslice(const int32_t *q_c2r, int cols, int lo, int hi, int32_t *colmap, int32_t *out_r2c,
                       int32_t *out_c2r) {
    int k = 0;
    for (int col = 0; col < cols; ++col) {
        int r = q_c2r[col];
        if (r >= lo && r < hi) {
            colmap[k] = col;
            out_r2c[r - lo] = k;
            out_c2r[k] = r - lo;
            k++;
        }
    }
}

/* Steady-ant recursion on square n x n permutations given by both maps.  Result written into
 * (out_r2c, out_c2r), with the reference's exact sequence of point sets (so that the column map the
 * parent reads is the one the reference reads).
 * Restates R:common/include/Permutations/MongeMultuplicationStrategy.h:569-593
 * (steadyAntWithPrecalcAndMemory) with initialPart :487-529 (base case n == 1 :494-501),
 * inverseMapping :208-220, antPassage :244-301 and restoreMatrixInRlo :304-323. */
static int slo_steady_ant_rec(int n, const int32_t *p_r2c, const int32_t *p_c2r, const int32_t *q_r2c,
                              const int32_t *q_c2r, int32_t *out_r2c, int32_t *out_c2r, slo_pool *pl) {
    (void) p_c2r; (void) q_r2c;
    if (n == 1) {
        out_r2c[0] = 0;
        out_c2r[0] = 0;
        return 0;
    }
    size_t mark = pl->top;
    int h = n / 2, h2 = n - h;
    int32_t *plo_r = pool_take(pl, h), *plo_c = pool_take(pl, h), *plo_map = pool_take(pl, h);
    int32_t *qlo_r = pool_take(pl, h), *qlo_c = pool_take(pl, h), *qlo_map = pool_take(pl, h);
    int32_t *phi_r = pool_take(pl, h2), *phi_c = pool_take(pl, h2), *phi_map = pool_take(pl, h2);
    int32_t *qhi_r = pool_take(pl, h2), *qhi_c = pool_take(pl, h2), *qhi_map = pool_take(pl, h2);
    int32_t *rlo_r = pool_take(pl, h), *rlo_c = pool_take(pl, h);
    int32_t *rhi_r = pool_take(pl, h2), *rhi_c = pool_take(pl, h2);
    int32_t *lo_r2c = pool_take(pl, n), *lo_c2r = pool_take(pl, n);
    int32_t *hi_r2c = pool_take(pl, n), *hi_c2r = pool_take(pl, n);
    if (!hi_c2r) return -1;
    slo_vslice(p_r2c, n, 0, h, plo_map, plo_r, plo_c);
    slo_hslice(q_c2r, n, 0, h, qlo_map, qlo_r, qlo_c);
    slo_vslice(p_r2c, n, h, n, phi_map, phi_r, phi_c);
    slo_hslice(q_c2r, n, h, n, qhi_map, qhi_r, qhi_c);
    if (slo_steady_ant_rec(h, plo_r, plo_c, qlo_r, qlo_c, rlo_r, rlo_c, pl)) return -1;
    if (slo_steady_ant_rec(h2, phi_r, phi_c, qhi_r, qhi_c, rhi_r, rhi_c, pl)) return -1;
    /* inverse mapping: iterate over the child's columns, read the child's column->row map */
    for (int i = 0; i < n; ++i) { lo_r2c[i] = lo_c2r[i] = hi_r2c[i] = hi_c2r[i] = NOPOINT; }
    for (int c = 0; c < h; ++c) {
        int oc = qlo_map[c], orow = plo_map[rlo_c[c]];
        lo_r2c[orow] = oc; lo_c2r[oc] = orow;
    }
    for (int c = 0; c < h2; ++c) {
        int oc = qhi_map[c], orow = phi_map[rhi_c[c]];
        hi_r2c[orow] = oc; hi_c2r[oc] = orow;
    }
    /* ant passage: walk the demarcation line from the bottom-left corner.  sh = #{hi points with
     * row < R, col < C} (BOTTOM_RIGHT arrow), sl = #{lo points with row >= R, col >= C} (TOP_LEFT),
     * both kept incrementally as in R:common/include/Permutations/DominanceSum.h:210-294. */
    int32_t *good_r = pool_take(pl, n), *good_c = pool_take(pl, n);
    if (!good_c) return -1;
    int ngood = 0;
    int row = n, col = -1, sh = 0, sl = 0, went_right = 0;
    for (;;) {
        if (row == 0 || col == n) break;
        int R = row - 1, C = col + 1;
        if (went_right) {           /* column C-1 joined the region */
            int rr = hi_c2r[C - 1];
            if (rr != NOPOINT && rr < R) sh++;
            rr = lo_c2r[C - 1];
            if (rr != NOPOINT && rr >= R) sl--;
        } else if (R + 1 != 0) {    /* row R left the hi region / joined the lo region */
            int cc = hi_r2c[R];
            if (cc != NOPOINT && cc < C) sh--;
            cc = lo_r2c[R];
            if (cc != NOPOINT && cc >= C) sl++;
        }
        if (sh - sl < 0) { went_right = 1; col++; }
        else if (sh - sl == 0) { went_right = 0; row--; }
        /* sh - sl > 0 does not occur for valid inputs (the reference prints "Impissble", :284) */
        if (C > 0) {
            int dal_h = sh, dal_l = sl, dbr_h = sh, dbr_l = sl;
            int rr = hi_c2r[C - 1];
            if (rr != NOPOINT && rr < R) dal_h--;
            rr = lo_c2r[C - 1];
            if (rr != NOPOINT && rr >= R) dal_l++;
            if (R < n) {
                int cc = hi_r2c[R];
                if (cc != NOPOINT && cc < C) dbr_h++;
                cc = lo_r2c[R];
                if (cc != NOPOINT && cc >= C) dbr_l--;
            } else { dbr_h = 0; dbr_l = 0; }
            if (dal_h - dal_l < 0 && dbr_h - dbr_l > 0) { good_r[ngood] = R; good_c[ngood] = C - 1; ngood++; }
        }
    }
    /* restore into lo: hi points overwrite, then the good points */
    for (int i = 0; i < n; ++i) {
        int c = hi_r2c[i];
        if (c == NOPOINT) continue;
        lo_r2c[i] = c; lo_c2r[c] = i;
    }
    for (int g = 0; g < ngood; ++g) { lo_r2c[good_r[g]] = good_c[g]; lo_c2r[good_c[g]] = good_r[g]; }
    memcpy(out_r2c, lo_r2c, sizeof(int32_t) * (size_t) n);
    memcpy(out_c2r, lo_c2r, sizeof(int32_t) * (size_t) n);
    pl->top = mark;
    return 0;
}

/* Sequential steady-ant product R = P (.) Q of two n x n permutations (row->col maps).
 * Restates R:common/include/Permutations/MongeMultuplicationStrategy.h:553-565
 * (SequentialMemoryOptimizedStickBraidMultiplication::multiply).  Returns 0 on success. */
int slo_steady_ant(const int32_t *p, const int32_t *q, int n, int32_t *r) {
    if (n <= 0) return 0;
    /* per level of size n: 12 half-size slices/maps (6n) + 2 half results (2n) + 4 full maps (4n)
     * + good points (2n) = 14n; nested levels halve, so 28n bounds the whole recursion */
    int levels = 1;
    for (int t = n; t > 1; t = (t + 1) / 2) levels++;
    size_t cap = (size_t) 14 * (size_t) n * 2 + (size_t) levels * 64;
    slo_pool pl = {(int32_t *) malloc(sizeof(int32_t) * cap), 0, cap};
    int32_t *p_c2r = (int32_t *) malloc(sizeof(int32_t) * (size_t) n);
    int32_t *q_c2r = (int32_t *) malloc(sizeof(int32_t) * (size_t) n);
    int32_t *o_c2r = (int32_t *) malloc(sizeof(int32_t) * (size_t) n);
    for (int i = 0; i < n; ++i) { p_c2r[p[i]] = i; q_c2r[q[i]] = i; }
    int rc = slo_steady_ant_rec(n, p, p_c2r, q, q_c2r, r, o_c2r, &pl);
    free(pl.base); free(p_c2r); free(q_c2r); free(o_c2r);
    return rc;
}

/* Glue two braids that share k strands.  row_glue != 0: P above Q, sharing the k = n columns
 * (P's bottom exits feed Q's top entries); row_glue == 0: P left of Q, sharing the k = m rows.
 * P is (pm, pn) with pm + pn strands, Q likewise; out has pm + pn + qm + qn - k strands.
 * Restates R:common/include/Permutations/MongeMultuplicationStrategy.h:679-758
 * (StaggeredStickyBraidMultiplication::staggeredStickyMultiplication) including k == 0 (:689-707). */
int slo_staggered(const int32_t *p, int p_size, const int32_t *q, int q_size, int k, int row_glue,
                  int32_t *out) {
    int out_size = p_size + q_size - k;
    for (int i = 0; i < out_size; ++i) out[i] = NOPOINT;
    if (k == p_size && k == q_size) return -1;     /* the reference aborts (:681-685) */
    if (k == 0) {
        for (int i = 0; i < p_size; ++i)
            if (p[i] != NOPOINT) { if (row_glue) out[i + q_size] = p[i] + q_size; else out[i] = p[i]; }
        for (int i = 0; i < q_size; ++i)
            if (q[i] != NOPOINT) { if (row_glue) out[i] = q[i]; else out[i + p_size] = q[i] + p_size; }
        return 0;
    }
    int32_t *p_c2r = (int32_t *) malloc(sizeof(int32_t) * (size_t) p_size);
    int32_t *q_c2r = (int32_t *) malloc(sizeof(int32_t) * (size_t) q_size);
    for (int i = 0; i < p_size; ++i) p_c2r[i] = NOPOINT;
    for (int i = 0; i < q_size; ++i) q_c2r[i] = NOPOINT;
    for (int i = 0; i < p_size; ++i) if (p[i] != NOPOINT) p_c2r[p[i]] = i;
    for (int i = 0; i < q_size; ++i) if (q[i] != NOPOINT) q_c2r[q[i]] = i;
    int32_t *mrow = (int32_t *) malloc(sizeof(int32_t) * (size_t) k);
    int32_t *mcol = (int32_t *) malloc(sizeof(int32_t) * (size_t) k);
    int32_t *pr = (int32_t *) malloc(sizeof(int32_t) * (size_t) k);
    int32_t *prc = (int32_t *) malloc(sizeof(int32_t) * (size_t) k);
    int32_t *qr = (int32_t *) malloc(sizeof(int32_t) * (size_t) k);
    int32_t *qrc = (int32_t *) malloc(sizeof(int32_t) * (size_t) k);
    int32_t *res = (int32_t *) malloc(sizeof(int32_t) * (size_t) k);
    if (row_glue) {
        slo_vslice(p, p_size, 0, k, mrow, pr, prc);
        slo_hslice(q_c2r, q_size, q_size - k, q_size, mcol, qr, qrc);
    } else {
        slo_vslice(p, p_size, p_size - k, p_size, mrow, pr, prc);
        slo_hslice(q_c2r, q_size, 0, k, mcol, qr, qrc);
    }
    int rc = slo_steady_ant(pr, qr, k, res);
    for (int i = 0; i < k && rc == 0; ++i) {
        int cc = mcol[res[i]], rr = mrow[i];
        if (row_glue) out[q_size - k + rr] = cc;
        else out[rr] = cc + p_size - k;
    }
    if (row_glue) {
        for (int j = k; j < p_size; ++j) { int r0 = p_c2r[j]; if (r0 != NOPOINT) out[r0 + q_size - k] = j + q_size - k; }
        for (int i = 0; i < q_size - k; ++i) if (q[i] != NOPOINT) out[i] = q[i];
    } else {
        for (int j = 0; j < p_size - k; ++j) { int r0 = p_c2r[j]; if (r0 != NOPOINT) out[r0] = j; }
        for (int i = k; i < q_size; ++i) if (q[i] != NOPOINT) out[i - k + p_size] = p_size - k + q[i];
    }
    free(p_c2r); free(q_c2r); free(mrow); free(mcol); free(pr); free(prc); free(qr); free(qrc); free(res);
    return rc;
}

/* Hybrid iterative scheme: tiles combed independently, then a bottom-up glue tree that alternates
 * row and column reductions.  Restates R:include/SemiLocal/SemiLocalLCS.h:602-647 (tile heuristic)
 * and :661-792 (hybridIterative); tile leaves use the anti-diagonal combing above. */
int slo_hybrid_iterative(const int32_t *a, int m, const int32_t *b, int n, int threads, int max_cols,
                         int max_rows, int32_t *row_to_col) {
    if (m == 0 || n == 0) {
        for (int i = 0; i < m + n; ++i) row_to_col[i] = i;
        return 0;
    }
    if (threads < 1) threads = 1;
    int cols = max_cols, rows = max_rows, total = cols + rows;
    int msmall, nsmall;
    if (rows >= m) { rows = m; msmall = 1; }
    else {
        int nums = (int) ceil((1.0 * m) / rows);
        rows = (int) ceil(1.0 * m / nums);
        msmall = (int) ceil((m * 1.0) / rows);
    }
    if (cols >= n) { cols = (int) ceil((n * 1.0) / threads); nsmall = threads; }
    else {
        int cpt = (int) ceil((1.0 * n) / threads);
        int rest = total - rows;
        if (cpt < rest) nsmall = threads;
        else nsmall = threads * (int) ceil(1.0 * cpt / rest);
    }
    int cpb = (int) ceil((double) n / nsmall);
    int rpb = (int) ceil((double) m / msmall);
    nsmall = (int) ceil((double) n / cpb);
    msmall = (int) ceil((double) m / rpb);
    int ntasks = msmall * nsmall;
    int32_t **cur = (int32_t **) calloc((size_t) ntasks, sizeof(int32_t *));
    int32_t **nxt = (int32_t **) calloc((size_t) ntasks, sizeof(int32_t *));
    int *tm = (int *) calloc((size_t) ntasks, sizeof(int)), *tn = (int *) calloc((size_t) ntasks, sizeof(int));
    int *nm = (int *) calloc((size_t) ntasks, sizeof(int)), *nn = (int *) calloc((size_t) ntasks, sizeof(int));
    int rc = 0;
#pragma omp parallel for num_threads(threads) schedule(dynamic)
    for (int i = 0; i < ntasks; ++i) {
        int sc = (i % nsmall) * cpb, ec = sc + cpb < n ? sc + cpb : n;
        int sr = (i / nsmall) * rpb, er = sr + rpb < m ? sr + rpb : m;
        if (i % nsmall == nsmall - 1) ec = n;
        if (i / nsmall == msmall - 1) er = m;
        int sa = er - sr, sb = ec - sc;
        cur[i] = (int32_t *) malloc(sizeof(int32_t) * (size_t) (sa + sb));
        slo_comb_antidiag(a + sr, sa, b + sc, sb, 1, cur[i]);
        tm[i] = sa; tn[i] = sb;
    }
    int steps = (int) ceil(log2(nsmall)) + (int) ceil(log2(msmall));
    int brows = rpb, bcols = cpb;
    for (int s = 0; s < steps; ++s) {
        int in_row = nsmall > msmall;
        if (nsmall > 1 && msmall > 1) in_row = brows >= 2 * bcols;
        if (in_row) bcols *= 2; else brows *= 2;
        int ncols = in_row ? (int) ceil(nsmall / 2.0) : nsmall;
        int nrows = !in_row ? (int) ceil(msmall / 2.0) : msmall;
#pragma omp parallel for num_threads(threads) schedule(dynamic)
        for (int i = 0; i < ncols * nrows; ++i) {
            int crow = i / ncols, ccol = i % ncols;
            int pi, qi;
            if (in_row) { pi = crow * nsmall + 2 * ccol; qi = (2 * ccol + 1 >= nsmall) ? -1 : pi + 1; }
            else { pi = 2 * crow * nsmall + ccol; qi = (2 * crow + 1 >= msmall) ? -1 : (2 * crow + 1) * nsmall + ccol; }
            if (qi < 0) { nxt[i] = cur[pi]; nm[i] = tm[pi]; nn[i] = tn[pi]; cur[pi] = NULL; continue; }
            int psz = tm[pi] + tn[pi], qsz = tm[qi] + tn[qi];
            int k = in_row ? tm[pi] : tn[pi];
            int32_t *prod = (int32_t *) malloc(sizeof(int32_t) * (size_t) (psz + qsz - k));
            if (slo_staggered(cur[pi], psz, cur[qi], qsz, k, !in_row, prod)) rc = -1;
            nm[i] = in_row ? tm[pi] : tm[pi] + tm[qi];
            nn[i] = in_row ? tn[pi] + tn[qi] : tn[pi];
            nxt[i] = prod;
            free(cur[pi]); free(cur[qi]); cur[pi] = cur[qi] = NULL;
        }
        int32_t **t = cur; cur = nxt; nxt = t;
        int *t2 = tm; tm = nm; nm = t2;
        t2 = tn; tn = nn; nn = t2;
        nsmall = ncols; msmall = nrows;
    }
    memcpy(row_to_col, cur[0], sizeof(int32_t) * (size_t) (m + n));
    free(cur[0]);
    free(cur); free(nxt); free(tm); free(tn); free(nm); free(nn);
    return rc;
}

/* ------------------------------------------------------------------------------------------------ */
/* Bit-parallel combing (score only)                                                                 */
/* ------------------------------------------------------------------------------------------------ */

/* Pack symbols LSB-first, bps bits each, S = 64 / bps per word (residue 64 % bps at the bottom).
 * Restates R:prefix_lcs/bitwise/encoders_and_decoders.h:50-87 (encode) for 64-bit words. */
int slo_encode_u64(const int32_t *s, int len, int bps, uint64_t *out) {
    int S = 64 / bps, residue = 64 % bps;
    int words = (len + S - 1) / S;
    for (int w = 0; w < words; ++w) {
        uint64_t word = 0;
        for (int k = 0; k < S && w * S + k < len; ++k)
            word |= ((uint64_t) s[w * S + k]) << (bps * k + residue);
        out[w] = word;
    }
    return words;
}

/* Pack a reversed: word n-1-i holds symbols i*S .. i*S+S-1, the first at the top.
 * Restates R:prefix_lcs/bitwise/encoders_and_decoders.h:100-139 (encode_reverse) for 64-bit words. */
int slo_encode_reverse_u64(const int32_t *s, int len, int bps, uint64_t *out) {
    int S = 64 / bps, residue = 64 % bps;
    int words = (len + S - 1) / S;
    for (int i = 0; i < words; ++i) {
        uint64_t word = 0;
        for (int k = 0; k < S && i * S + k < len; ++k)
            word |= ((uint64_t) s[i * S + k]) << (bps * (S - k - 1) + residue);
        out[words - 1 - i] = word;
    }
    return words;
}

/* One word cell of the n-ary bit combing: 2S-1 shifted steps.
 * Restates R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:329-411
 * (mpi_nary_size::process_antidiagonal, loop body). */
static void slo_nary_cell(uint64_t *lp, uint64_t *tp, uint64_t sa, uint64_t sb, int residue, int bps,
                          uint64_t ones) {
    uint64_t l = *lp, t = *tp, single = (uint64_t) 1 << residue, mask = single, cond, eq, lc, tc;
    int size = 64 - residue - bps;
    for (int sh = size; sh > 0; sh -= bps) {
        lc = l >> sh; tc = t << sh;
        cond = ~((sa >> sh) ^ sb); eq = cond;
        for (int i = 1; i < bps; ++i) cond &= eq >> i;
        t = (lc | (ones ^ mask)) & (t | (cond & mask));
        l = tc ^ (t << sh) ^ l;
        mask = (mask << bps) | single;
    }
    cond = ~(sa ^ sb); eq = cond;
    for (int i = 1; i < bps; ++i) cond &= eq >> i;
    lc = l; tc = t;
    t = lc & (t | (cond & ones));
    l = tc ^ t ^ l;
    mask = ones << bps;
    for (int sh = bps; sh <= size; sh += bps) {
        cond = ~((sa << sh) ^ sb); eq = cond;
        for (int i = 1; i < bps; ++i) cond &= eq >> i;
        lc = l << sh; tc = t >> sh;
        t = (lc | (ones ^ mask)) & (t | (cond & mask));
        l = tc ^ (t >> sh) ^ l;
        mask <<= bps;
    }
    *lp = l; *tp = t;
}

/* LLCS by n-ary bit combing over 64-bit words; a_rev = encode_reverse(a), b = encode(b), a_words <=
 * b_words, lengths multiples of the symbols per word (the reference's own domain).
 * Restates R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:668-736
 * (nary::llcs_nary_symbol_smart_combing): left strands = braid_ones, top = 0, three phases over word
 * diagonals, score = a_total_symbols - popcount(left strands). */
int slo_bit_llcs_nary_u64(const uint64_t *a_rev, int a_words, const uint64_t *b, int b_words,
                          int a_total_symbols, int bps) {
    int m = a_words, n = b_words;
    uint64_t *l = (uint64_t *) malloc(sizeof(uint64_t) * (size_t) m);
    uint64_t *t = (uint64_t *) malloc(sizeof(uint64_t) * (size_t) n);
    int residue = 64 % bps;
    uint64_t ones = (uint64_t) 1 << residue;
    for (int i = 0; i < 64; i += bps) ones |= ones << i;
    for (int k = 0; k < m; ++k) l[k] = ones;
    for (int k = 0; k < n; ++k) t[k] = 0;
    int same = (m + n - 1) - (m - 1) - (m - 1);
    for (int d = 0; d < m - 1; ++d)
        for (int j = 0; j < d + 1; ++j) slo_nary_cell(&l[m - 1 - d + j], &t[j], a_rev[m - 1 - d + j], b[j], residue, bps, ones);
    for (int k = 0; k < same; ++k)
        for (int j = 0; j < m; ++j) slo_nary_cell(&l[j], &t[k + j], a_rev[j], b[k + j], residue, bps, ones);
    int sj = same;
    for (int d = m - 1; d >= 1; --d, ++sj)
        for (int j = 0; j < d; ++j) slo_nary_cell(&l[j], &t[sj + j], a_rev[j], b[sj + j], residue, bps, ones);
    int dis = 0;
    for (int k = 0; k < m; ++k) dis += __builtin_popcountll(l[k]);
    free(l); free(t);
    return a_total_symbols - dis;
}

/* One word cell of binary combing, formula 2 (15 ops per step).
 * Restates R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:251-323. */
static void slo_binary_cell_u64(uint64_t *lp, uint64_t *tp, uint64_t sa, uint64_t sb) {
    uint64_t l = *lp, t = *tp, mask = 1, lc, tc, cond;
    for (int sh = 63; sh > 0; --sh) {
        lc = l >> sh; tc = t << sh;
        cond = ~((sa >> sh) ^ sb);
        t = (lc | ~mask) & (t | (cond & mask));
        l = tc ^ (t << sh) ^ l;
        mask = (mask << 1) | 1;
    }
    cond = ~(sa ^ sb);
    lc = l; tc = t;
    t = (lc | ~mask) & (t | (cond & mask));
    l = tc ^ t ^ l;
    mask = ~(uint64_t) 0;
    for (int sh = 1; sh < 64; ++sh) {
        mask <<= 1;
        lc = l << sh; tc = t >> sh;
        cond = ~((sa << sh) ^ sb);
        t = (lc | ~mask) & (t | (cond & mask));
        l = tc ^ (t >> sh) ^ l;
    }
    *lp = l; *tp = t;
}

/* LLCS of binary strings packed 64 per word, lengths multiples of 64, a_words <= b_words.
 * Restates R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:598-663
 * (binary::llcs_2symbol_smart_combing with formula 2). */
int slo_bit_llcs_binary_u64(const uint64_t *a_rev, int a_words, const uint64_t *b, int b_words,
                            int a_total_symbols) {
    int m = a_words, n = b_words;
    uint64_t *l = (uint64_t *) malloc(sizeof(uint64_t) * (size_t) m);
    uint64_t *t = (uint64_t *) malloc(sizeof(uint64_t) * (size_t) n);
    for (int k = 0; k < m; ++k) l[k] = ~(uint64_t) 0;
    for (int k = 0; k < n; ++k) t[k] = 0;
    int same = (m + n - 1) - (m - 1) - (m - 1);
    for (int d = 0; d < m - 1; ++d)
        for (int j = 0; j < d + 1; ++j) slo_binary_cell_u64(&l[m - 1 - d + j], &t[j], a_rev[m - 1 - d + j], b[j]);
    for (int k = 0; k < same; ++k)
        for (int j = 0; j < m; ++j) slo_binary_cell_u64(&l[j], &t[k + j], a_rev[j], b[k + j]);
    int sj = same;
    for (int d = m - 1; d >= 1; --d, ++sj)
        for (int j = 0; j < d; ++j) slo_binary_cell_u64(&l[j], &t[sj + j], a_rev[j], b[sj + j]);
    int dis = 0;
    for (int k = 0; k < m; ++k) dis += __builtin_popcountll(l[k]);
    free(l); free(t);
    return a_total_symbols - dis;
}

/* Convenience for the CPU baseline: global LLCS of one pair via anti-diagonal combing. */
int slo_comb_score(const int32_t *a, int m, const int32_t *b, int n, int threads) {
    int32_t *perm = (int32_t *) malloc(sizeof(int32_t) * (size_t) (m + n > 0 ? m + n : 1));
    slo_comb_antidiag(a, m, b, n, threads, perm);
    int s = slo_global_score(perm, m, n);
    free(perm);
    return s;
}

/* Bit-vector LLCS (R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:749-830, lllcs_hyyro::preprocess and
 * hyyro_magic): V over the symbols of `a` (bit i = a[i], 64-bit words), all ones; for every symbol c of b:
 * p = match(c) & V; V = (V ^ p) | (V + p + carry), the carry running from word to word; the score is the number
 * of zero bits of V over the real positions (padding bits never take a match, so they stay 1). */
int slo_hyyro_llcs(const int32_t *a, int m, const int32_t *b, int n) {
    if (m == 0 || n == 0) return 0;
    const int W = (m + 63) / 64;
    uint64_t *V = (uint64_t *) malloc(sizeof(uint64_t) * W);
    uint64_t *Mt = (uint64_t *) calloc((size_t) W, sizeof(uint64_t));
    for (int w = 0; w < W; ++w) V[w] = ~0ull;
    for (int j = 0; j < n; ++j) {
        for (int w = 0; w < W; ++w) {
            uint64_t x = 0;
            for (int i = 0; i < 64 && 64 * w + i < m; ++i)
                if (a[64 * w + i] == b[j]) x |= 1ull << i;
            Mt[w] = x;
        }
        uint64_t carry = 0;
        for (int w = 0; w < W; ++w) {
            const uint64_t v = V[w], p = Mt[w] & v;
            const uint64_t s1 = v + p;
            const uint64_t c1 = s1 < v;
            const uint64_t s2 = s1 + carry;
            const uint64_t c2 = s2 < s1;
            V[w] = (v ^ p) | s2;
            carry = c1 | c2;
        }
    }
    int zeros = 0;
    for (int w = 0; w < W; ++w) {
        const int bits = (64 * (w + 1) <= m) ? 64 : m - 64 * w;
        for (int i = 0; i < bits; ++i) zeros += !((V[w] >> i) & 1ull);
    }
    free(V);
    free(Mt);
    return zeros;
}

int slo_version(void) { return 1; }
