/*
 * slcs.h -- C ABI of the B200 semi-local LCS engine (libslcs.so).
 *
 * Plain C types only (no CUDA or torch types): pointers, sizes, status codes.  Streams are passed as
 * `void *` holding a cudaStream_t (NULL = the engine's own stream).  Every entry point returns an
 * SLCS_* status; on failure slcs_last_error() gives a message for the calling thread.  Nothing here
 * exits the process or falls back to the CPU: without a usable CUDA device every compute call returns
 * SLCS_ERR_NO_DEVICE.
 *
 * Braid layout (identical to the reference's common::Permutation, R:common/include/Permutations/
 * Matrices.h:16-96): a pair (a[0..m), b[0..n)) has m+n strands.  row_to_col[s] is the end of strand s:
 *   strand starts (rows): left strands 0..m-1 (strand l enters the grid at row m-1-l),
 *                         top strands m..m+n-1 (strand r enters at column r-m);
 *   strand ends (cols):   bottom exits 0..n-1 (column j), right exits n..n+m-1 (n+l is row m-1-l).
 * col_to_row is the inverse map.  Permutations for braid multiplication are n x n row->col maps.
 * Sizes: a pair's m + n, a glued braid's strands and a permutation's n must be below 2^30; larger sizes return
 * SLCS_ERR_TOO_LARGE before any device work.
 *
 * Reference interfaces replaced (paths relative to the reference project, R: = source/cpu/):
 *   semi_local::SemiLocalStrategy<Input>::compute          R:include/SemiLocal/SemiLocalLCS.h:7-11
 *   common::BraidMultiplicationStrategy::multiply           R:common/include/Permutations/MongeMultuplicationStrategy.h:18-21
 *   common::StaggeredStickyBraidMultiplication::staggeredStickyMultiplication
 *                                                           R:common/include/Permutations/MongeMultuplicationStrategy.h:679-758
 *   lcs::LCSStrategy<Input>::compute                        R:include/LCS/LCS.h:9-13
 *   prefix_lcs_via_semi_local::nary::llcs_nary_symbol_smart_combing
 *                                                           R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:668-736
 *   InteractiveDuplicateSearchSemiDense / ...SemiSparse::find
 *                                                           R:approximate_matching/ApproximateMatching.h:252-420
 */
#ifndef SLCS_H
#define SLCS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------------- */
#define SLCS_OK 0
#define SLCS_ERR_ARG 1          /* invalid argument (negative size, NULL pointer, bad option) */
#define SLCS_ERR_CUDA 2         /* a CUDA runtime call failed */
#define SLCS_ERR_OOM 3          /* device memory exhausted / admission budget exceeded */
#define SLCS_ERR_TIMEOUT 4      /* a bounded device-side wait gave up (error word set by a kernel) */
#define SLCS_ERR_TOO_LARGE 5    /* size beyond what the engine supports */
#define SLCS_ERR_NO_DEVICE 6    /* no usable CUDA device */
#define SLCS_ERR_INTERNAL 7     /* consistency check failed */
#define SLCS_ERR_BUSY 8         /* server queue full / request not finished */

/* ---- algorithm selection ------------------------------------------------------------------------ */
#define SLCS_ALGO_AUTO 0        /* engine chooses: wavefront; the hybrid once both lengths reach 2^17, tiles of about
                                   min(m, n) / 16 (a power of two in [16384, 65536]) */
#define SLCS_ALGO_WAVEFRONT 1   /* tiled wavefront combing over the whole grid */
#define SLCS_ALGO_HYBRID 2      /* tiles combed independently, glued by GPU steady ant */

typedef struct slcs_opts {
    int algo;            /* SLCS_ALGO_* */
    int tile_rows;       /* hybrid tile height (0 = default 4096) */
    int tile_cols;       /* hybrid tile width  (0 = default 4096) */
    int band_rows;       /* wavefront rows per warp band: 32*R, R in {1,2,4,8,16,32} (0 = auto) */
    int sa_cutoff;       /* steady-ant size below which sub-problems finish in shared memory (0 = default) */
    int lane_cols;       /* wavefront of a lone pair: columns a lane combs per step -- 4 or 8 = register tiles of
                            band_rows/32 x lane_cols cells (band_rows 64..512, else 256), 1 = one column per step
                            (the band kernel), 0 = auto: tiles of 8 x 4 (16 x 4 above 262144 rows) up to 524288
                            rows unless band_rows is given */
    int reserved[2];
} slcs_opts;

/* ---- library ------------------------------------------------------------------------------------ */
int slcs_version(void);
const char *slcs_last_error(void);
/* Select the CUDA device used by the calling thread's engine calls (default 0). */
int slcs_set_device(int device);
/* Release cached device memory and engine state of the current device. */
int slcs_release(void);

/* ---- semi-local combing: the braid of a pair -------------------------------------------------- */
/* Replaces semi_local::SemiLocalStrategy<Input>::compute (R:include/SemiLocal/SemiLocalLCS.h:7-11) for
 * uint8 symbols; outputs row_to_col (m+n).  col_to_row and score (global LLCS) are optional (NULL).
 * Host buffers; copies in and out are part of the call. */
int slcs_comb_u8(const uint8_t *a, int m, const uint8_t *b, int n, int32_t *row_to_col, int32_t *col_to_row,
                 int32_t *score, const slcs_opts *opts);
/* Same for int32 symbols (Input = int in the reference); symbols are compared for equality only. */
int slcs_comb_i32(const int32_t *a, int m, const int32_t *b, int n, int32_t *row_to_col, int32_t *col_to_row,
                  int32_t *score, const slcs_opts *opts);
/* Device-pointer variant: all pointers are device memory, work is ordered on `stream`.  d_row_to_col is
 * required; d_col_to_row and d_score are optional. */
int slcs_comb_u8_dev(const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_row_to_col,
                     int32_t *d_col_to_row, int32_t *d_score, const slcs_opts *opts, void *stream);
/* Allocation-free variant of slcs_comb_u8_dev, for callers that cannot let the engine allocate device
 * memory (a host that owns a fixed device-memory budget, a plugin in an application whose allocator
 * reserved the device memory up front, a serving loop that must not touch the allocator).
 * No counterpart in the reference.
 * Its scratch is one static device array of about 192 KiB per device (held until the process exits),
 * shared by every call and cleared by each call: calls that overlap on the GPU race, so serialise them.
 * The first call on a device resolves the array's address; make it before any stream capture, and do not
 * call this entry point again after cudaDeviceReset (the address belongs to the reset context).
 * The caller passes inputs and both outputs (d_col_to_row is required; it is also the band hand-off);
 * d_score is optional.  Limits: m <= 8388608 rows (8192 bands), m + n < 2^30, else SLCS_ERR_TOO_LARGE.
 * Above about 1.8 million rows the bands outnumber the resident warps and the call takes about twice as
 * long as slcs_comb_u8_dev; pass the shorter string as a. */
int slcs_comb_u8_dev_noalloc(const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_row_to_col,
                             int32_t *d_col_to_row, int32_t *d_score, void *stream);

/* ---- global LCS score ------------------------------------------------------------------------- */
/* Replaces lcs::LCSStrategy<Input>::compute (R:include/LCS/LCS.h:9-13) through the braid
 * (lcs::LCSBySemiLocal, R:include/LCS/LCS.h:216-238). */
int slcs_lcs_u8(const uint8_t *a, int m, const uint8_t *b, int n, int32_t *score);

/* ---- bit-parallel combing (score only) -------------------------------------------------------- */
/* LLCS by bit-parallel sticky-braid combing, one bit per strand; symbols must be < 4 (2-bit codes).
 * Replaces prefix_lcs_via_semi_local::nary::llcs_nary_symbol_smart_combing with bits_per_symbol = 2
 * (R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:668-736) and the binary variant
 * (:598-663) for symbols < 2; unlike the reference any lengths are accepted. */
int slcs_bitcomb_llcs_u8(const uint8_t *a, int m, const uint8_t *b, int n, int32_t *score);
int slcs_bitcomb_llcs_u8_dev(const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_score, void *stream);
/* LLCS by the bit-vector recurrence V' = (V + (V & match)) | (V & ~match) over one string's symbols (Allison-Dix,
 * Hyyro), the carry running through the whole vector; symbols must be < 4.  Replaces lllcs_hyyro::hyyro_magic and
 * hyyro_magic_mpi_with_precalc (R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:787-914, which build
 * the vector over their `b` and loop over `a`; the engine puts the vector over the longer string). */
int slcs_hyyro_llcs_u8(const uint8_t *a, int m, const uint8_t *b, int n, int32_t *score);
int slcs_hyyro_llcs_u8_dev(const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_score, void *stream);

/* ---- unit-Monge braid multiplication (steady ant) -------------------------------------------- */
/* r = p (.) q for n x n permutations given as row->col maps.
 * Replaces common::BraidMultiplicationStrategy::multiply
 * (R:common/include/Permutations/MongeMultuplicationStrategy.h:18-21). */
int slcs_steady_ant(const int32_t *p, const int32_t *q, int n, int32_t *r, const slcs_opts *opts);
int slcs_steady_ant_dev(const int32_t *d_p, const int32_t *d_q, int n, int32_t *d_r, const slcs_opts *opts,
                        void *stream);

/* Reusable steady-ant plan for size n (device-resident, graph-capturable): create() plans and allocates
 * all scratch, run() only launches kernels on `stream` (with use_graph != 0 the launch sequence is
 * captured once per (p, q, r) pointer triple and replayed), check() waits and reports the device error word. */
typedef struct slcs_sa_plan slcs_sa_plan;
int slcs_sa_plan_create(int n, slcs_sa_plan **out);
int slcs_sa_plan_run(slcs_sa_plan *pl, const int32_t *d_p, const int32_t *d_q, int32_t *d_r, int use_graph,
                     void *stream);
int slcs_sa_plan_check(slcs_sa_plan *pl, void *stream);
int slcs_sa_plan_launches(slcs_sa_plan *pl, int32_t *launches);
int slcs_sa_plan_destroy(slcs_sa_plan *pl);

/* Glue braid p (pm rows of a, pn columns of b) with braid q sharing k strands.
 * row_glue != 0: p above q (k = pn = qn); row_glue == 0: p left of q (k = pm = qm).
 * Replaces common::StaggeredStickyBraidMultiplication::staggeredStickyMultiplication<RowGlue>
 * (R:common/include/Permutations/MongeMultuplicationStrategy.h:679-758).  out has pm+pn+qm+qn-k entries. */
int slcs_staggered_glue(const int32_t *p, int pm, int pn, const int32_t *q, int qm, int qn, int row_glue,
                        int32_t *out);

/* ---- scores read from a braid ----------------------------------------------------------------- */
#define SLCS_Q_GLOBAL 0             /* LCS(a, b) */
#define SLCS_Q_STRING_SUBSTRING 1   /* LCS(a, b[i..j)) */
#define SLCS_Q_PREFIX_SUFFIX 2      /* LCS(a[0..i), b[j..n)) */
#define SLCS_Q_SUFFIX_PREFIX 3      /* LCS(a[i..m), b[0..j)) */
#define SLCS_Q_SUBSTRING_STRING 4   /* LCS(a[i..j), b) */
#define SLCS_Q_MATRIX 5             /* raw semi-local matrix entry H(i, j), i, j in [0, m+n] */
typedef struct slcs_query {
    int32_t kind;
    int32_t i;
    int32_t j;
} slcs_query;
/* Answers nq queries against a braid (host row_to_col of m+n entries).  Semantics follow the
 * semi-local matrix of R:include/SemiLocal/SemiLocalLCS.h:13-63 and the string-substring readout of
 * R:approximate_matching/utils.h:281-334. */
int slcs_scores(const int32_t *row_to_col, int m, int n, const slcs_query *q, int nq, int32_t *out);
int slcs_scores_dev(const int32_t *d_row_to_col, int m, int n, const slcs_query *d_q, int nq, int32_t *d_out,
                    void *stream);

/* Window scan: out[s] = LCS(a, b[s..s+w)) for every s = 0..n-w (n-w+1 values), in O(m+n) for all windows:
 * the incremental dominance moves of the reference's window matcher (R:approximate_matching/WindowAMatch.h:
 * 26-71) as one prefix sum.  The _dev form takes an optional col_to_row (NULL: computed on the device). */
int slcs_window_scores(const int32_t *row_to_col, int m, int n, int w, int32_t *out);
int slcs_window_scores_dev(const int32_t *d_row_to_col, const int32_t *d_col_to_row, int m, int n, int w,
                           int32_t *d_out, void *stream);

/* ---- approximate pattern search ----------------------------------------------------------------- */
/* An interval [start, end) of the text and its score: minus the indel distance (substitution = 2 indels) of the
 * pattern and the interval, the reference's approximate_matching::utils::Interval
 * (R:approximate_matching/utils.h:233-253) with the fixed scoring scheme (0, -2, -1). */
typedef struct slcs_interval {
    int32_t start;
    int32_t end;
    double score;
} slcs_interval;

/* Approximate copies of `pattern` (m symbols) in `text` (n >= int(m / k) symbols), 0 < k <= 1: replaces
 * InteractiveDuplicateSearchSemiDense::find (R:approximate_matching/ApproximateMatching.h:320-420) with the same
 * result vector.  One braid of the pattern against the text (the combing engine), every window's score by the
 * window scan, every window's best interval by a warp kernel; the dedup, sort and greedy pick on the host.
 * Writes the first min(count, out_cap) intervals to out and the count to *n_out.  SLCS_ERR_ARG for a text shorter
 * than the window, SLCS_ERR_TOO_LARGE for a window of more than 16384 interval ends or 2^21 symbols. */
int slcs_duplicate_search_u8(const uint8_t *pattern, int m, const uint8_t *text, int n, double k, slcs_interval *out,
                             int out_cap, int *n_out);
int slcs_duplicate_search_i32(const int32_t *pattern, int m, const int32_t *text, int n, double k,
                              slcs_interval *out, int out_cap, int *n_out);
/* The same search with the reference's InteractiveDuplicateSearchSemiSparse::find
 * (R:approximate_matching/ApproximateMatching.h:252-318): only the windows its first phase visits (it skips ahead
 * by half the score deficit) are clones; each clone's best interval is the one the dense search finds for that
 * window start (the reference reads it from the clone's own braid). */
int slcs_duplicate_search_sparse_u8(const uint8_t *pattern, int m, const uint8_t *text, int n, double k,
                                    slcs_interval *out, int out_cap, int *n_out);
int slcs_duplicate_search_sparse_i32(const int32_t *pattern, int m, const int32_t *text, int n, double k,
                                     slcs_interval *out, int out_cap, int *n_out);

/* ---- batched combing -------------------------------------------------------------------------- */
/* Braids of npairs independent pairs in one persistent, length-bucketed launch.  a_cat / b_cat hold the
 * concatenated symbols, a_off / b_off (npairs) the start of each string, m / n (npairs) the lengths;
 * row_to_col_cat receives the concatenated braids (pair i at offset sum_{j<i} m_j + n_j); scores
 * (npairs, optional) the global LLCS.  The reference has no batch API: this replaces a loop of
 * SemiLocalStrategy::compute calls.  mode 0 = persistent batched launch, 1 = one launch per pair. */
int slcs_batch_comb_u8(const uint8_t *a_cat, const int64_t *a_off, const int32_t *m, const uint8_t *b_cat,
                       const int64_t *b_off, const int32_t *n, int npairs, int32_t *row_to_col_cat,
                       int32_t *scores, int mode, const slcs_opts *opts);

/* ---- batch plans (device-resident batches, reusable, graph-capturable) ------------------------- */
/* A plan fixes the pair lengths and owns the device buffers of one batch.  run() is the device-only
 * step: one persistent length-bucketed launch (mode 0) or one launch per pair (mode 1), then the
 * end->start inversion; with use_graph != 0 the step is captured once into a CUDA graph and replayed. */
typedef struct slcs_batch slcs_batch;
int slcs_batch_create(const int32_t *m, const int32_t *n, int npairs, int mode, const slcs_opts *opts,
                      slcs_batch **out);
int slcs_batch_upload(slcs_batch *bt, const uint8_t *a_cat, const int64_t *a_off, const uint8_t *b_cat,
                      const int64_t *b_off, void *stream);
int slcs_batch_run(slcs_batch *bt, int use_graph, void *stream);
int slcs_batch_download(slcs_batch *bt, int32_t *row_to_col_cat, int32_t *scores, void *stream);
/* Device time (ms) of the last run's combing kernel(s), measured with CUDA events on the run's stream. */
int slcs_batch_kernel_ms(slcs_batch *bt, float *ms);
/* Total cells (sum m*n) and launch count of one run. */
int slcs_batch_info(slcs_batch *bt, int64_t *cells, int32_t *launches, int64_t *h2d_bytes, int64_t *d2h_bytes);
int slcs_batch_destroy(slcs_batch *bt);

/* ---- single-pair plans (device-resident, reusable, graph-capturable) -------------------------- */
/* kind: SLCS_ALGO_WAVEFRONT, SLCS_ALGO_HYBRID (braid + score), SLCS_PLAN_BITPARALLEL or SLCS_PLAN_HYYRO (score only).
 * create() plans and allocates everything for an m x n pair; run() launches kernels on `stream` (uint8
 * device strings; with use_graph != 0 the launch sequence is captured once per buffer set and replayed);
 * check() waits and reports the device error word; kernel_ms() is the device time of the last run's
 * combing kernel (CUDA events on the run's stream). */
#define SLCS_PLAN_BITPARALLEL 3
#define SLCS_PLAN_HYYRO 4
typedef struct slcs_pair_plan slcs_pair_plan;
int slcs_pair_plan_create(int m, int n, int kind, const slcs_opts *opts, slcs_pair_plan **out);
int slcs_pair_plan_run(slcs_pair_plan *pl, const uint8_t *d_a, const uint8_t *d_b, int32_t *d_row_to_col,
                       int32_t *d_score, int use_graph, void *stream);
int slcs_pair_plan_check(slcs_pair_plan *pl, void *stream);
int slcs_pair_plan_kernel_ms(slcs_pair_plan *pl, float *ms);
int slcs_pair_plan_launches(slcs_pair_plan *pl, int32_t *launches);
int slcs_pair_plan_destroy(slcs_pair_plan *pl);

/* ---- serving loop (no counterpart in the reference) ---------------------------------------------- */
/* Continuous batching of comparison requests on one GPU.  A request is a pair (a, b) plus one score query
 * on its braid; the result is what SemiLocalStrategy::compute (R:include/SemiLocal/SemiLocalLCS.h:7-11)
 * followed by the score readout (R:include/LCS/LCS.h:223-233, R:approximate_matching/utils.h:281-334)
 * gives.  A worker thread admits requests by a device-memory budget, batches the small ones into
 * persistent combing launches on several streams (requests at or above big_cells cells run alone on the
 * big streams), overlaps the launches on the device, and keeps every finished braid resident for further
 * queries until it is released or evicted (least recently used first) to make room.  Results do not
 * depend on what else runs. */
typedef struct slcs_server slcs_server;
typedef struct slcs_server_opts {
    int64_t mem_budget;     /* device bytes for in-flight requests and resident braids (0: half the free memory) */
    int32_t max_pending;    /* submitted but not admitted; beyond it submit returns SLCS_ERR_BUSY (0: 65536) */
    int32_t small_streams;  /* concurrent batches of small requests (0: 2, at most 16) */
    int64_t big_cells;      /* m*n at or above which a request runs alone on the big stream (0: 2^32) */
    int32_t big_warps;      /* persistent-grid cap of a big launch, in warps (0: half the resident warps) */
    int32_t small_warps;    /* persistent-grid cap of a small batch (0: a quarter of the resident warps) */
    int32_t max_batch;      /* requests per small batch (0: 1024) */
    int32_t band_rows;      /* rows per band (0: chosen per request) */
    int32_t big_streams;    /* concurrent big requests (0: 2, at most 8) */
    int32_t reserved[7];
} slcs_server_opts;
typedef struct slcs_result {
    uint64_t ticket;
    int32_t status;         /* SLCS_OK, or the error that ended the request (SLCS_ERR_BUSY: cancelled) */
    int32_t score;          /* the query's answer */
    int32_t m, n;
    slcs_query query;
    int32_t pad;
    double t_submit, t_admit, t_done;   /* seconds on the server's clock (slcs_server_now) */
} slcs_result;
typedef struct slcs_server_stats {
    int64_t submitted, completed, rejected, evicted;
    int64_t resident, resident_bytes, used_bytes, peak_bytes, budget;
    int64_t launches, cells;
    int32_t pending, inflight;
} slcs_server_stats;
int slcs_server_create(const slcs_server_opts *opts, slcs_server **out);
/* Copies a and b (borrowed for the call only); q NULL = global score.  SLCS_ERR_BUSY when the queue is full,
 * SLCS_ERR_OOM when the request alone exceeds the budget. */
int slcs_server_submit(slcs_server *srv, const uint8_t *a, int m, const uint8_t *b, int n, const slcs_query *q,
                       uint64_t *ticket);
/* Up to cap finished results (waits up to timeout_ms for the first one). */
int slcs_server_poll(slcs_server *srv, slcs_result *out, int cap, int *count, int timeout_ms);
/* More queries on a finished request's resident braid (synchronous). */
int slcs_server_query(slcs_server *srv, uint64_t ticket, const slcs_query *q, int nq, int32_t *out);
/* Window scan of a resident braid: out[s] = LCS(a, b[s..s+w)), s = 0..n-w (synchronous). */
int slcs_server_window(slcs_server *srv, uint64_t ticket, int w, int32_t *out);
/* Copies a resident braid (row_to_col, m+n entries) to the host. */
int slcs_server_braid(slcs_server *srv, uint64_t ticket, int32_t *row_to_col);
int slcs_server_release(slcs_server *srv, uint64_t ticket);
int slcs_server_stats_get(slcs_server *srv, slcs_server_stats *st);
double slcs_server_now(slcs_server *srv);
/* Cancels requests not yet admitted, finishes those on the device, frees everything. */
int slcs_server_destroy(slcs_server *srv);

/* ---- autotuner (no counterpart in the reference) ------------------------------------------------- */
/* Per device, the parameters an entry point uses when the caller passes 0: band heights by row-count class
 * (for pairs that share a launch -- batches, hybrid tiles, serving -- and for one pair alone), the hybrid
 * tile edge and the steady-ant shared-memory cutoff.  slcs_autotune() times the candidates on synthetic
 * inputs (a few seconds) and installs the fastest; get/set let a caller persist and restore a table
 * (set(NULL) restores the built-in defaults).  Zero entries mean "built-in default". */
typedef struct slcs_tuning {
    int32_t band_rows_batch[32];    /* rows per band (32 R) for a pair with ceil(log2 m) = k in a shared launch */
    int32_t band_rows_single[32];   /* the same for one pair alone on the device (wavefront plans) */
    int32_t tile;                   /* hybrid tile edge */
    int32_t sa_cutoff;              /* steady-ant sub-problem size finished in shared memory (<= 4096) */
    int32_t reserved[6];
} slcs_tuning;
#define SLCS_TUNE_BANDS_BATCH 1
#define SLCS_TUNE_BANDS_SINGLE 2
#define SLCS_TUNE_TILE 4
#define SLCS_TUNE_SA_CUTOFF 8
#define SLCS_TUNE_ALL 15
int slcs_autotune(int flags, slcs_tuning *out);
int slcs_tuning_get(slcs_tuning *out);
int slcs_tuning_set(const slcs_tuning *in);

/* ---- failure-path self-test (no counterpart in the reference) ------------------------------------ */
/* Runs the combing kernel on a band whose upstream band is never launched, so its bounded wait (about 2 s of
 * the GPU timer) gives up: *status receives the status the engine reports for it (SLCS_ERR_TIMEOUT when the
 * failure path works).  Nothing faults; the engine stays usable.  Returns SLCS_OK if the test could run. */
int slcs_selftest_wait_timeout(int32_t *status);
/* Debug check of a braid or product (no counterpart in the reference): every entry of perm[0..size) is in range
 * and no value repeats.  SLCS_OK if so, else SLCS_ERR_INTERNAL; *bad_entries (optional) counts the offenders. */
int slcs_check_permutation(const int32_t *perm, int size, int32_t *bad_entries);
int slcs_check_permutation_dev(const int32_t *d_perm, int size, int32_t *bad_entries, void *stream);

/* ---- measurement helper (no counterpart in the reference) --------------------------------------- */
/* Issue-rate ceiling of the combing cell's instruction mix on this device, in cells per second
 * (independent cells at full occupancy): the denominator of the combing kernels' roofline fraction. */
int slcs_probe_cell_peak(double *cells_per_sec);

#ifdef __cplusplus
}
#endif
#endif /* SLCS_H */
