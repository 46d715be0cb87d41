// slcs_internal.cuh -- shared helpers of the B200 semi-local LCS engine (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>
#include <cuda/atomic>
#include <cstdint>
#include <cstdio>
#include <string>

#include <nvtx3/nvToolsExt.h>
#include <vector>

#include "../../include/slcs.h"

namespace slcs {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarp = 32;

// Device-side error word values (the first failing kernel wins; the host maps them to SLCS_ERR_*).
constexpr int kDevErrNone = 0;
constexpr int kDevErrTimeout = 1;     // a bounded spin gave up
constexpr int kDevErrBadState = 2;    // an internal consistency check failed

// Spin limits: each wait gives up after kWaitLimitNs of the GPU's global timer (sleeping ~kSpinSleepNs
// between polls), sets the error word and returns; waiters also leave as soon as the word is set.  Legitimate
// waits (a band waiting for the band above it to publish 32 columns) last microseconds.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;
constexpr unsigned kSpinSleepNs = 100;
constexpr int kSpinPolls = 64;   // polls without sleeping before the sleeping ones

// NVTX range for the host side of a stage (visible in Nsight timelines; no cost without a tool attached).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// ------------------------------------------------------------------------------------------------
// host error plumbing
// ------------------------------------------------------------------------------------------------
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);

#define SLCS_CUDA_TRY(expr)                                                                          \
    do {                                                                                             \
        cudaError_t _e = (expr);                                                                     \
        if (_e != cudaSuccess) {                                                                     \
            return ::slcs::fail(_e == cudaErrorMemoryAllocation ? SLCS_ERR_OOM : SLCS_ERR_CUDA,      \
                                std::string(#expr) + ": " + cudaGetErrorString(_e));                 \
        }                                                                                            \
    } while (0)

#define SLCS_TRY(expr)                    \
    do {                                  \
        int _rc = (expr);                 \
        if (_rc != SLCS_OK) return _rc;   \
    } while (0)

// ------------------------------------------------------------------------------------------------
// device helpers
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire(const int *p) {
    cuda::atomic_ref<int, cuda::thread_scope_device> r(*const_cast<int *>(p));
    return r.load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void st_release(int *p, int v) {
    cuda::atomic_ref<int, cuda::thread_scope_device> r(*p);
    r.store(v, cuda::memory_order_release);
}
__device__ __forceinline__ int ld_relaxed(const int *p) {
    cuda::atomic_ref<int, cuda::thread_scope_device> r(*const_cast<int *>(p));
    return r.load(cuda::memory_order_relaxed);
}
__device__ __forceinline__ void raise_error(int *err, int code) { atomicCAS(err, kDevErrNone, code); }

// Wait until *p >= need.  Returns false (after setting *err) when the bounded spin gives up or when
// another thread already reported an error.  Called by one lane; the caller broadcasts the outcome.
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool wait_at_least(const int *p, int need, int *err,
                                              unsigned long long limit_ns = kWaitLimitNs) {
    if (ld_acquire(p) >= need) return true;
    const unsigned long long t0 = global_ns();
    // the first polls follow each other without sleeping (a band usually waits for the band above to publish
    // its next chunk, well under a microsecond; a sleep there would add its own granularity to every hand-off);
    // then one poll every ~kSpinSleepNs.  The iteration cap is a second bound in case the timer does not advance
    // (at >= 100 ns per poll it is never the first to trigger while the timer runs).
#pragma unroll 1
    for (int it = 0; it < kSpinPolls; ++it) {
        if (ld_acquire(p) >= need) return true;
    }
    for (long long it = 0; it < (1ll << 26); ++it) {
        __nanosleep(kSpinSleepNs);
        if (ld_acquire(p) >= need) return true;
        if (ld_relaxed(err) != kDevErrNone) return false;
        if (global_ns() - t0 > limit_ns) break;
    }
    raise_error(err, kDevErrTimeout);
    return false;
}

// Hand-off words that carry a value and the tag of the band that wrote it in one 64-bit store: a reader that sees
// the expected tag has the value, with no fence between them.
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*const_cast<unsigned long long *>(p));
    return r.load(cuda::memory_order_relaxed);
}
__device__ __forceinline__ void st_relaxed64(unsigned long long *p, unsigned long long v) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*p);
    r.store(v, cuda::memory_order_relaxed);
}
// Until the hand-off word *p (already read into v) carries `tag` in its high half: re-reads it, polling without
// sleeping first, bounded like wait_at_least (the error word is set when it gives up).  Data and tag travel in one
// 64-bit store, so a word with the right tag is the right word.
__device__ __forceinline__ bool wait_tag(const unsigned long long *p, unsigned long long &v, unsigned tag, int *err) {
    if ((unsigned) (v >> 32) == tag) return true;
    const unsigned long long t0 = global_ns();
    for (long long it = 0; it < (1ll << 26); ++it) {
        if (it >= kSpinPolls) __nanosleep(kSpinSleepNs);
        v = ld_relaxed64(p);
        if ((unsigned) (v >> 32) == tag) return true;
        if ((it & 15) == 15) {
            if (ld_relaxed(err) != kDevErrNone) return false;
            if (global_ns() - t0 > kWaitLimitNs) break;
        }
    }
    raise_error(err, kDevErrTimeout);
    return false;
}

// ------------------------------------------------------------------------------------------------
// per-device engine state: stream, error word, scratch arena
// ------------------------------------------------------------------------------------------------
struct Engine {
    int device = -1;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    bool ready = false;
};

// Returns the calling thread's engine for its current device, initialising it on first use.
int engine(Engine **out);
// Stream-ordered scratch allocation (cudaMallocAsync on the engine's memory pool).
int dalloc(void **p, size_t bytes, cudaStream_t s);
void dfree(void *p, cudaStream_t s);
// Waits for the stream, then maps the device error word to an SLCS_* status.
int check_dev_err(const int *d_err, cudaStream_t s);

template <typename T>
struct DevBuf {
    T *p = nullptr;
    cudaStream_t s = nullptr;
    size_t count = 0;
    int alloc(size_t cnt, cudaStream_t st) {
        s = st;
        count = cnt;
        return dalloc(reinterpret_cast<void **>(&p), (cnt ? cnt : 1) * sizeof(T), st);
    }
    void release() {
        if (p) dfree(p, s);
        p = nullptr;
    }
    ~DevBuf() { release(); }
};

// ------------------------------------------------------------------------------------------------
// tuning table of the current device (tune.cu): what a caller that passes 0 for a parameter gets
// ------------------------------------------------------------------------------------------------
int pick_rows_batch(int rows);    // rows per lane (band height / 32) for a pair sharing a launch
int pick_rows_single(int rows);   // the same for one pair alone on the device
int pick_tile();                  // hybrid tile edge
int pick_sa_cutoff();             // steady-ant size finished in shared memory

// ------------------------------------------------------------------------------------------------
// combing (comb.cu)
// ------------------------------------------------------------------------------------------------
// Symbol codes the combing kernel reserves for its padding rows and columns (they match nothing).  int32 symbols
// handed to it must differ from both: the host entry points map inputs that hold them to dense codes first.
constexpr int kSymRowVirtual = -0x40000000;   // a-symbol of a padding row
constexpr int kSymColVirtual = -0x40000001;   // b-symbol of a padding column

struct CombPair {
    const void *a;        // symbols of the row string (T)
    const void *b;        // symbols of the column string (T)
    int32_t *c2r;         // out: strand end -> strand start (m+n); also the band-to-band hand-off of the
                          //      top strands (entries 0..n-1)
    int32_t *progress;    // per band: number of leading columns whose hand-off value is final
    int32_t *score;       // out (optional): global LLCS
    int m, n;
    unsigned long long *hand;   // tile kernel only: n hand-off words (band tag << 32 | strand), zeroed per launch
};

struct CombItem {
    int pair;
    int band;    // band index inside the pair
    int r0;      // first row of the band
    int R;       // rows per lane (band height 32 R), in {1, 2, 4, 8, 16, 32}
    int last;    // 1 if this is the pair's last band (its bottom outputs are final)
};

// Plans the bands of one pair: appends items with the given default R (the last band uses the smallest
// R that still covers its rows).  Returns the number of bands.
int plan_bands(int pair, int m, int R, std::vector<CombItem> &items);
// Launch the persistent combing kernel over items (device arrays).  T = uint8_t or int32_t.
template <typename T>
int launch_comb(const CombPair *d_pairs, const CombItem *d_items, int nitems, int *d_next, int *d_err,
                int grid_warps, cudaStream_t s);
// The same for the bands of one pair alone on the device: two dependency chains per lane (comb.cu).
template <typename T>
int launch_comb_lone(const CombPair *d_pairs, const CombItem *d_items, int nitems, int *d_next, int *d_err,
                     int grid_warps, cudaStream_t s);
// Register-tile kernel for one pair alone on the device (comb.cu): a lane combs C columns of its R rows per step,
// bands hand strands down through the pair's `hand` words (zeroed before every launch).  Bands come from
// plan_tile_bands (one height for all, the last padded with rows that never swap); R in {2, 4, 8, 16}, C in {4, 8}.
constexpr int kTileRows = 8;                  // default tile: kTileRows x kTileCols cells per lane and step
constexpr int kTileCols = 4;
constexpr int kTileAutoMaxRows = 1 << 19;     // lone pairs up to this many rows take the tile kernel by default
int plan_tile_bands(int pair, int m, int R, std::vector<CombItem> &items);
template <typename T>
int launch_comb_tile(const CombPair *d_pairs, const CombItem *d_items, int nitems, int *d_next, int *d_err,
                     int grid_warps, int C, cudaStream_t s);
// The tile a lone pair of `rows` rows is combed with; R = 0: the band kernel.  lane_cols is the caller's choice
// (slcs_opts.lane_cols): 4 or 8 = the tile kernel with that width, band_rows 64..512 giving its height (else
// kTileRows); 1 = the band kernel; 0 = automatic: the band kernel when band_rows is given, else the tile kernel up
// to kTileAutoMaxRows rows (8 x 4 tiles, 16 x 4 above 2^18 rows), the band kernel above.
struct TileShape {
    int R = 0, C = 0;
};
TileShape tile_shape_for(int rows, int band_rows, int lane_cols);
// Warps that fit on the device at once for the combing kernel.
int comb_resident_warps(Engine *E);
int comb_resident_warps_sm(int num_sms);
// c2r -> r2c for one pair (optionally rotated by 180 degrees), and the batched version.
int launch_invert(const int32_t *c2r, int size, int32_t *r2c, bool rot180, int *d_err, cudaStream_t s);

// ------------------------------------------------------------------------------------------------
// steady ant (steady_ant.cu)
// ------------------------------------------------------------------------------------------------
// Batched unit-Monge products on device memory: problem i occupies [off[i], off[i] + n[i]) of the
// concatenated row->col arrays d_P, d_Q and d_R (out).
int steady_ant_batch_dev(const int32_t *d_P, const int32_t *d_Q, const std::vector<int64_t> &off,
                         const std::vector<int> &n, int32_t *d_R, int *d_err, cudaStream_t s, int cutoff = 0);
int steady_ant_max_small();
// Reusable plans: create() plans and allocates, run() only launches kernels on s (capturable).
struct SaPlan;
// Per-element scratch that several plans run one after another can share (owned by the caller).
struct SaScratch {
    int32_t *b[11] = {};   // 11 arrays of `elems` int32
    int32_t *tabp = nullptr, *vecp = nullptr, *cstp = nullptr;
    int64_t elems = 0, tab = 0, vec = 0, cst = 0;
};
int sa_plan_create(const std::vector<int64_t> &off, const std::vector<int> &n, SaPlan **out, cudaStream_t s,
                   const SaScratch *shared, int cutoff = 0);   // cutoff 0: the tuned / default cutoff
// shared != nullptr: the plan uses the caller's scratch; shared->elems < 0 defers the binding to sa_plan_bind.
int sa_plan_bind(SaPlan *P, const SaScratch *shared);
// Scratch sizes a plan needs (for building a shared SaScratch).
void sa_plan_needs(const SaPlan *P, int64_t *elems, int64_t *tab, int64_t *vec, int64_t *cst);
int sa_plan_run(SaPlan *P, const int32_t *d_P, const int32_t *d_Q, int32_t *d_R, int *d_err, cudaStream_t s);
int sa_plan_run_ex(SaPlan *P, const int32_t *d_P, const int32_t *d_leafP, const int32_t *d_Q, int32_t *d_R,
                   int32_t *d_PLout, int32_t *d_QLout, int *d_err, cudaStream_t s);
void sa_plan_destroy(SaPlan *P);
// The stream the plan's buffers are freed on; only for a plan whose work on its old stream has completed.
void sa_plan_set_stream(SaPlan *P, cudaStream_t s);
int sa_plan_launches(const SaPlan *P);
int64_t sa_plan_total(const SaPlan *P);

// ------------------------------------------------------------------------------------------------
// hybrid (hybrid.cu)
// ------------------------------------------------------------------------------------------------
struct HybridPlan;
int hybrid_plan_create(int m, int n, int tile_rows, int tile_cols, Engine *E, cudaStream_t s, HybridPlan **out);
template <typename T>
int hybrid_plan_run(HybridPlan *H, const T *d_a, const T *d_b, int *d_err, cudaStream_t s);
void hybrid_plan_destroy(HybridPlan *H);
// Moves the plan (and its steady-ant plans) onto stream s for its later frees; only once the work queued on the
// stream it was created on has completed.  A plan that outlives the call that made it is moved onto the engine's
// own stream, since the caller's stream may be destroyed before the plan is.
void hybrid_plan_set_stream(HybridPlan *H, cudaStream_t s);
int32_t *hybrid_result_r2c(HybridPlan *H);
int32_t *hybrid_result_c2r(HybridPlan *H);
int hybrid_score(HybridPlan *H, int32_t *d_score, cudaStream_t s);
int hybrid_launches(const HybridPlan *H);
int hybrid_enable_timing(HybridPlan *H);
void hybrid_set_capturing(HybridPlan *H, bool c);
int hybrid_comb_ms(HybridPlan *H, float *ms);

// ------------------------------------------------------------------------------------------------
// bit-parallel combing (bitcomb.cu)
// ------------------------------------------------------------------------------------------------
struct BitPlan;
int bit_plan_create(Engine *E, int m, int n, cudaStream_t s, BitPlan **out);
int bit_plan_run(BitPlan *B, const uint8_t *d_a, const uint8_t *d_b, int32_t *d_score, int *d_err, cudaStream_t s,
                 bool capturing);
int bit_plan_kernel_ms(BitPlan *B, float *ms);
void bit_plan_destroy(BitPlan *B);

// ------------------------------------------------------------------------------------------------
// bit-vector LLCS, Hyyro recurrence (hyyro.cu)
// ------------------------------------------------------------------------------------------------
struct HyyroPlan;
int hyyro_plan_create(Engine *E, int m, int n, cudaStream_t s, HyyroPlan **out);
int hyyro_plan_run(HyyroPlan *H, const uint8_t *d_a, const uint8_t *d_b, int32_t *d_score, int *d_err,
                   cudaStream_t s, bool capturing);
int hyyro_plan_kernel_ms(HyyroPlan *H, float *ms);
void hyyro_plan_destroy(HyyroPlan *H);
int hyyro_dev(Engine *E, const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_score, cudaStream_t s);

// ------------------------------------------------------------------------------------------------
// scores (scores.cu)
// ------------------------------------------------------------------------------------------------
// Maps a query to the semi-local matrix entry H(i, j) it reads and the offset added to it; ok = false for
// arguments out of range.  Semantics: R:include/SemiLocal/SemiLocalLCS.h:13-63, R:approximate_matching/
// utils.h:281-334.
__device__ __forceinline__ void query_to_matrix(const slcs_query &q, int m, int n, int &i, int &j, int &offset,
                                                bool &ok) {
    ok = true;
    offset = 0;
    switch (q.kind) {
        case SLCS_Q_GLOBAL: i = m; j = n; break;
        case SLCS_Q_STRING_SUBSTRING:   // LCS(a, b[i..j)) = H(i + m, j)
            ok = 0 <= q.i && q.i <= q.j && q.j <= n;
            i = q.i + m; j = q.j; break;
        case SLCS_Q_PREFIX_SUFFIX:      // LCS(a[0..i), b[j..n)) = H(j + m, n + m - i) - (m - i)
            ok = 0 <= q.i && q.i <= m && 0 <= q.j && q.j <= n;
            i = q.j + m; j = n + m - q.i; offset = -(m - q.i); break;
        case SLCS_Q_SUFFIX_PREFIX:      // LCS(a[i..m), b[0..j)) = H(m - i, j) - i
            ok = 0 <= q.i && q.i <= m && 0 <= q.j && q.j <= n;
            i = m - q.i; j = q.j; offset = -q.i; break;
        case SLCS_Q_SUBSTRING_STRING:   // LCS(a[i..j), b) = H(m - i, n + m - j) - i - (m - j)
            ok = 0 <= q.i && q.i <= q.j && q.j <= m;
            i = m - q.i; j = n + m - q.j; offset = -q.i - (m - q.j); break;
        case SLCS_Q_MATRIX:
            ok = 0 <= q.i && q.i <= m + n && 0 <= q.j && q.j <= m + n;
            i = q.i; j = q.j; break;
        default: ok = false; i = j = 0;
    }
}

int launch_scores(const int32_t *d_r2c, int m, int n, const slcs_query *d_q, int nq, int32_t *d_out, int *d_err,
                  cudaStream_t s);
// LCS(a, b[s..s+w)) for every window s = 0..n-w of a braid (d_c2r optional: computed when NULL); synchronous.
int window_scores_dev(const int32_t *d_r2c, const int32_t *d_c2r, int m, int n, int w, int32_t *d_out, cudaStream_t s);
// The braid of one pair on the device (capi.cu): wavefront, or the hybrid when opts ask for it.
template <typename T>
int comb_dev(Engine *E, const T *d_a, int m, const T *d_b, int n, int32_t *d_r2c, int32_t *d_c2r, int32_t *d_score,
             const slcs_opts *opts, cudaStream_t s);
// The same for host queries / answers (synchronous on s).
int launch_scores_host(const int32_t *d_r2c, int m, int n, const slcs_query *q, int nq, int32_t *out,
                       cudaStream_t s);

}  // namespace slcs
