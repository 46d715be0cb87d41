// capi.cu -- the extern "C" entry points of libslcs.so and the per-device engine state.
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>

#include "slcs_internal.cuh"
#include "symbol_codes.h"

namespace slcs {

namespace {
thread_local std::string g_last_error;
thread_local int g_device = 0;
std::mutex g_mu;
Engine g_engines[64];
}  // namespace

void set_error(const std::string &msg) { g_last_error = msg; }
int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int engine(Engine **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return fail(SLCS_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (g_device < 0 || g_device >= count || g_device >= 64)
        return fail(SLCS_ERR_ARG, "device index out of range");
    Engine &E = g_engines[g_device];
    SLCS_CUDA_TRY(cudaSetDevice(g_device));
    if (!E.ready) {
        cudaDeviceProp prop;
        SLCS_CUDA_TRY(cudaGetDeviceProperties(&prop, g_device));
        if (prop.major < 10)
            return fail(SLCS_ERR_NO_DEVICE, "libslcs is built for sm_100a (B200); device " +
                                                std::string(prop.name) + " is not supported");
        E.num_sms = prop.multiProcessorCount;
        SLCS_CUDA_TRY(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking));
        cudaMemPool_t pool;
        SLCS_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, g_device));
        uint64_t threshold = ~0ull;   // keep freed blocks cached in this process
        SLCS_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
        E.device = g_device;
        E.ready = true;
    }
    *out = &E;
    return SLCS_OK;
}

int dalloc(void **p, size_t bytes, cudaStream_t s) {
    *p = nullptr;
    cudaError_t e = cudaMallocAsync(p, bytes, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(e == cudaErrorMemoryAllocation ? SLCS_ERR_OOM : SLCS_ERR_CUDA,
                    std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " +
                        cudaGetErrorString(e));
    }
    return SLCS_OK;
}
void dfree(void *p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

int check_dev_err(const int *d_err, cudaStream_t s) {
    int h = 0;
    SLCS_CUDA_TRY(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    SLCS_CUDA_TRY(cudaStreamSynchronize(s));
    if (h == kDevErrTimeout) return fail(SLCS_ERR_TIMEOUT, "a device-side bounded wait gave up");
    if (h != kDevErrNone) return fail(SLCS_ERR_INTERNAL, "device consistency check failed");
    return SLCS_OK;
}

namespace {


// Combing of one pair on device memory: d_r2c (m+n) receives row->col, d_c2r (optional) col->row,
// d_score (optional, must be zeroed by the caller) the global LLCS.
template <typename T>
int comb_wavefront_dev(Engine *E, const T *d_a, int m, const T *d_b, int n, int32_t *d_r2c, int32_t *d_c2r,
                       int32_t *d_score, const slcs_opts *opts, cudaStream_t s) {
    const int size = m + n;
    // orientation: rows = the string giving the shorter pipeline (64 steps per band + columns)
    const int Ra = (opts && opts->band_rows) ? std::max(1, opts->band_rows / 32) : pick_rows_single(m);
    const int Rb = (opts && opts->band_rows) ? std::max(1, opts->band_rows / 32) : pick_rows_single(n);
    const long long cost_ab = 64ll * ((m + 32 * Ra - 1) / (32 * Ra)) + n;
    const long long cost_ba = 64ll * ((n + 32 * Rb - 1) / (32 * Rb)) + m;
    const bool swap = cost_ba < cost_ab;
    const T *rows_s = swap ? d_b : d_a;
    const T *cols_s = swap ? d_a : d_b;
    const int rows = swap ? n : m, cols = swap ? m : n;

    std::vector<CombItem> items;
    const TileShape ts = tile_shape_for(rows, opts ? opts->band_rows : 0, opts ? opts->lane_cols : 0);
    const int Rt = ts.R;
    const int bands = Rt > 0 ? plan_tile_bands(0, rows, Rt, items) : plan_bands(0, rows, swap ? Rb : Ra, items);
    DevBuf<unsigned long long> hand;
    DevBuf<int32_t> c2r_tmp, prog, err;
    DevBuf<CombPair> dpair;
    DevBuf<CombItem> ditems;
    DevBuf<int> next;
    int32_t *c2r_work = d_c2r;
    if (swap || c2r_work == nullptr) {
        SLCS_TRY(c2r_tmp.alloc(size, s));
        c2r_work = c2r_tmp.p;
    }
    SLCS_TRY(prog.alloc(bands, s));
    if (Rt > 0) {
        SLCS_TRY(hand.alloc(cols, s));
        SLCS_CUDA_TRY(cudaMemsetAsync(hand.p, 0, sizeof(unsigned long long) * cols, s));
    }
    SLCS_TRY(err.alloc(1, s));
    SLCS_TRY(dpair.alloc(1, s));
    SLCS_TRY(ditems.alloc(items.size(), s));
    SLCS_TRY(next.alloc(1, s));
    CombPair hp{rows_s, cols_s, c2r_work, prog.p, d_score, rows, cols, hand.p};
    SLCS_CUDA_TRY(cudaMemsetAsync(prog.p, 0, sizeof(int32_t) * bands, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    SLCS_CUDA_TRY(cudaMemsetAsync(next.p, 0, sizeof(int), s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(dpair.p, &hp, sizeof(hp), cudaMemcpyHostToDevice, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(ditems.p, items.data(), sizeof(CombItem) * items.size(),
                                  cudaMemcpyHostToDevice, s));
    if (Rt > 0)
        SLCS_TRY(launch_comb_tile<T>(dpair.p, ditems.p, (int) items.size(), next.p, err.p, comb_resident_warps(E),
                                     ts.C, s));
    else
        SLCS_TRY(launch_comb_lone<T>(dpair.p, ditems.p, (int) items.size(), next.p, err.p, comb_resident_warps(E), s));
    SLCS_TRY(launch_invert(c2r_work, size, d_r2c, swap, err.p, s));
    if (d_c2r != nullptr && swap) SLCS_TRY(launch_invert(d_r2c, size, d_c2r, false, err.p, s));
    return check_dev_err(err.p, s);
}

constexpr int kAutoHybridMin = 1 << 17;    // both lengths at least this: AUTO takes the hybrid

// Tile edge of the hybrid the engine chooses by itself: about a sixteenth of the shorter length, a power of two in
// [2^14, 2^16] -- enough tiles to fill the device with bands, few enough glue levels.
int auto_tile(int m, int n) {
    const int want = std::min(m, n) / 16;
    int t = 1 << 14;
    while (t < want && t < (1 << 16)) t <<= 1;
    return t;
}

// The last hybrid plan of each device, kept for the next call of the same shape (planning a hybrid -- tile
// descriptors, glue levels, steady-ant plans, scratch -- costs far more host time than running a small one).  A
// call that finds it busy or of another shape plans afresh and then offers its plan in its place.
struct HybridCache {
    std::mutex mu;
    HybridPlan *H = nullptr;
    int m = -1, n = -1, tr = -1, tc = -1, elem = 0;
    bool busy = false;
};
HybridCache g_hcache[64];

template <typename T>
int comb_hybrid_dev(Engine *E, const T *d_a, int m, const T *d_b, int n, int32_t *d_r2c, int32_t *d_c2r,
                    int32_t *d_score, const slcs_opts *opts, cudaStream_t s) {
    // tiles: the caller's, else for the engine's own choice of the hybrid (AUTO, large pairs) auto_tile, else the
    // tuned edge
    const bool chosen = !opts || opts->algo == SLCS_ALGO_AUTO;
    const int at = auto_tile(m, n);
    const int tr = (opts && opts->tile_rows > 0) ? opts->tile_rows : (chosen ? at : pick_tile());
    const int tc = (opts && opts->tile_cols > 0) ? opts->tile_cols : (chosen ? at : pick_tile());
    HybridCache &C = g_hcache[E->device];
    HybridPlan *H = nullptr;
    bool from_cache = false;
    {
        std::lock_guard<std::mutex> lk(C.mu);
        if (!C.busy && C.H && C.m == m && C.n == n && C.tr == tr && C.tc == tc && C.elem == (int) sizeof(T)) {
            H = C.H;
            C.busy = true;
            from_cache = true;
        }
    }
    if (!H) SLCS_TRY(hybrid_plan_create(m, n, tr, tc, E, s, &H));
    DevBuf<int> err;
    int rc = err.alloc(1, s);
    if (rc == SLCS_OK && cudaMemsetAsync(err.p, 0, sizeof(int), s) != cudaSuccess) rc = fail(SLCS_ERR_CUDA, "memset");
    if (rc == SLCS_OK) rc = hybrid_plan_run<T>(H, d_a, d_b, err.p, s);
    if (rc == SLCS_OK && cudaMemcpyAsync(d_r2c, hybrid_result_r2c(H), sizeof(int32_t) * (m + n),
                                         cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        rc = fail(SLCS_ERR_CUDA, "result copy");
    if (rc == SLCS_OK && d_c2r && cudaMemcpyAsync(d_c2r, hybrid_result_c2r(H), sizeof(int32_t) * (m + n),
                                                  cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        rc = fail(SLCS_ERR_CUDA, "result copy");
    if (rc == SLCS_OK && d_score) rc = hybrid_score(H, d_score, s);
    if (rc == SLCS_OK) rc = check_dev_err(err.p, s);   // the plan's work is over when this returns
    HybridPlan *drop = nullptr;
    {
        std::lock_guard<std::mutex> lk(C.mu);
        if (from_cache) {
            C.busy = false;
            if (rc != SLCS_OK) {   // a failed run leaves no plan behind
                drop = C.H;
                C.H = nullptr;
            }
        } else if (rc == SLCS_OK && !C.busy) {
            // check_dev_err synchronised s, so nothing of this plan is queued on it any more; later frees go to
            // the engine's stream, which lives until the process exits (the caller's may not)
            hybrid_plan_set_stream(H, E->stream);
            drop = C.H;
            C.H = H;
            C.m = m;
            C.n = n;
            C.tr = tr;
            C.tc = tc;
            C.elem = (int) sizeof(T);
        } else {
            drop = H;
        }
    }
    if (drop) hybrid_plan_destroy(drop);
    return rc;
}

// Algorithm choice: the hybrid when asked for, or (AUTO) for grids large in both dimensions, with tiles of
// auto_tile(m, n): few enough glue levels that the full occupancy of the tile combing outweighs them.  Measured on
// B200 (event-timed, random and similar-string pairs alike): 2^17 pair wavefront 9.6 ms, 16384-tiles 7.2 (8192:
// 7.9, 32768: 8.9); 2^18 pair 28.8 ms, 16384-tiles 18.9 (65536: 19.5); 2^19 pair 81.6 ms, 32768-tiles 58.0
// (16384: 61.0, 65536: 61.3); 2^20 pair 300 ms, 65536-tiles 207, 4096-tiles 309 (16 glue levels).
bool use_hybrid(const slcs_opts *opts, int m, int n) {
    const int algo = opts ? opts->algo : SLCS_ALGO_AUTO;
    if (algo == SLCS_ALGO_HYBRID) return true;
    if (algo == SLCS_ALGO_WAVEFRONT) return false;
    return std::min(m, n) >= kAutoHybridMin;
}

}  // namespace

template <typename T>
int comb_dev(Engine *E, const T *d_a, int m, const T *d_b, int n, int32_t *d_r2c, int32_t *d_c2r, int32_t *d_score,
             const slcs_opts *opts, cudaStream_t s) {
    NvtxRange nv("slcs: combing");
    if (use_hybrid(opts, m, n)) return comb_hybrid_dev<T>(E, d_a, m, d_b, n, d_r2c, d_c2r, d_score, opts, s);
    return comb_wavefront_dev<T>(E, d_a, m, d_b, n, d_r2c, d_c2r, d_score, opts, s);
}
template int comb_dev<uint8_t>(Engine *, const uint8_t *, int, const uint8_t *, int, int32_t *, int32_t *, int32_t *,
                               const slcs_opts *, cudaStream_t);
template int comb_dev<int32_t>(Engine *, const int32_t *, int, const int32_t *, int, int32_t *, int32_t *, int32_t *,
                               const slcs_opts *, cudaStream_t);

namespace {

int identity_host(int size, int32_t *r2c, int32_t *c2r, int32_t *score) {
    for (int i = 0; i < size; ++i) {
        if (r2c) r2c[i] = i;
        if (c2r) c2r[i] = i;
    }
    if (score) *score = 0;
    return SLCS_OK;
}

template <typename T>
int comb_host(const T *a, int m, const T *b, int n, int32_t *row_to_col, int32_t *col_to_row, int32_t *score,
              const slcs_opts *opts) {
    if (m < 0 || n < 0) return fail(SLCS_ERR_ARG, "negative length");
    if ((m > 0 && !a) || (n > 0 && !b) || !row_to_col) return fail(SLCS_ERR_ARG, "NULL buffer");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    Engine *E;
    SLCS_TRY(engine(&E));
    if (m == 0 || n == 0) return identity_host(m + n, row_to_col, col_to_row, score);
    cudaStream_t s = E->stream;
    DevBuf<T> da, db;
    DevBuf<int32_t> dr, dc, dsc;
    SLCS_TRY(da.alloc(m, s));
    SLCS_TRY(db.alloc(n, s));
    SLCS_TRY(dr.alloc(m + n, s));
    if (col_to_row) SLCS_TRY(dc.alloc(m + n, s));
    SLCS_TRY(dsc.alloc(1, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(da.p, a, sizeof(T) * m, cudaMemcpyHostToDevice, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(db.p, b, sizeof(T) * n, cudaMemcpyHostToDevice, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(dsc.p, 0, sizeof(int32_t), s));
    SLCS_TRY(comb_dev<T>(E, da.p, m, db.p, n, dr.p, col_to_row ? dc.p : nullptr, dsc.p, opts, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(row_to_col, dr.p, sizeof(int32_t) * (m + n), cudaMemcpyDeviceToHost, s));
    if (col_to_row)
        SLCS_CUDA_TRY(cudaMemcpyAsync(col_to_row, dc.p, sizeof(int32_t) * (m + n), cudaMemcpyDeviceToHost, s));
    int32_t hscore = 0;
    SLCS_CUDA_TRY(cudaMemcpyAsync(&hscore, dsc.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SLCS_CUDA_TRY(cudaStreamSynchronize(s));
    if (score) *score = hscore;
    return SLCS_OK;
}

}  // namespace
}  // namespace slcs

using namespace slcs;

extern "C" {

int slcs_version(void) { return 100; }

const char *slcs_last_error(void) { return g_last_error.c_str(); }

int slcs_set_device(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return fail(SLCS_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= count) return fail(SLCS_ERR_ARG, "device index out of range");
    g_device = device;
    return SLCS_OK;
}

int slcs_release(void) {
    Engine *E;
    SLCS_TRY(engine(&E));
    {
        HybridCache &C = g_hcache[E->device];
        HybridPlan *drop = nullptr;
        {
            std::lock_guard<std::mutex> lk(C.mu);
            if (!C.busy) {
                drop = C.H;
                C.H = nullptr;
            }
        }
        if (drop) hybrid_plan_destroy(drop);
    }
    SLCS_CUDA_TRY(cudaStreamSynchronize(E->stream));
    cudaMemPool_t pool;
    SLCS_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, E->device));
    SLCS_CUDA_TRY(cudaMemPoolTrimTo(pool, 0));
    return SLCS_OK;
}

int slcs_comb_u8(const uint8_t *a, int m, const uint8_t *b, int n, int32_t *row_to_col, int32_t *col_to_row,
                 int32_t *score, const slcs_opts *opts) {
    return comb_host<uint8_t>(a, m, b, n, row_to_col, col_to_row, score, opts);
}

int slcs_comb_i32(const int32_t *a, int m, const int32_t *b, int n, int32_t *row_to_col, int32_t *col_to_row,
                  int32_t *score, const slcs_opts *opts) {
    if (m < 0 || n < 0) return fail(SLCS_ERR_ARG, "negative length");
    if ((m > 0 && !a) || (n > 0 && !b) || !row_to_col) return fail(SLCS_ERR_ARG, "NULL buffer");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    // symbols are compared for equality only: map them to codes >= 0 (the kernel reserves negative codes for
    // padding) -- v - min as uint8 when the symbols span at most 256 values, else dense codes, narrowed to uint8
    // when at most 256 values occur
    {
        std::vector<uint8_t> ca, cb;
        if (range_codes_u8(a, m, b, n, &ca, &cb))
            return comb_host<uint8_t>(ca.data(), m, cb.data(), n, row_to_col, col_to_row, score, opts);
    }
    std::vector<int32_t> all;
    all.reserve((size_t) m + n);
    if (m) all.insert(all.end(), a, a + m);
    if (n) all.insert(all.end(), b, b + n);
    std::vector<int32_t> uniq(all);
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    auto code = [&](int32_t v) { return (int32_t) (std::lower_bound(uniq.begin(), uniq.end(), v) - uniq.begin()); };
    if (uniq.size() <= 256) {
        std::vector<uint8_t> ca(m), cb(n);
        for (int i = 0; i < m; ++i) ca[i] = (uint8_t) code(a[i]);
        for (int i = 0; i < n; ++i) cb[i] = (uint8_t) code(b[i]);
        return comb_host<uint8_t>(ca.data(), m, cb.data(), n, row_to_col, col_to_row, score, opts);
    }
    std::vector<int32_t> ca(m), cb(n);
    for (int i = 0; i < m; ++i) ca[i] = code(a[i]);
    for (int i = 0; i < n; ++i) cb[i] = code(b[i]);
    return comb_host<int32_t>(ca.data(), m, cb.data(), n, row_to_col, col_to_row, score, opts);
}

int slcs_comb_u8_dev(const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_row_to_col,
                     int32_t *d_col_to_row, int32_t *d_score, const slcs_opts *opts, void *stream) {
    if (m < 0 || n < 0) return fail(SLCS_ERR_ARG, "negative length");
    if ((m > 0 && !d_a) || (n > 0 && !d_b) || (m + n > 0 && !d_row_to_col))
        return fail(SLCS_ERR_ARG, "NULL buffer (d_row_to_col is required)");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    if (d_score) SLCS_CUDA_TRY(cudaMemsetAsync(d_score, 0, sizeof(int32_t), s));
    if (m == 0 || n == 0) {
        std::vector<int32_t> id(m + n);
        std::iota(id.begin(), id.end(), 0);
        if (m + n > 0) {
            SLCS_CUDA_TRY(cudaMemcpyAsync(d_row_to_col, id.data(), sizeof(int32_t) * (m + n), cudaMemcpyHostToDevice, s));
            if (d_col_to_row)
                SLCS_CUDA_TRY(cudaMemcpyAsync(d_col_to_row, id.data(), sizeof(int32_t) * (m + n), cudaMemcpyHostToDevice, s));
            SLCS_CUDA_TRY(cudaStreamSynchronize(s));
        }
        return SLCS_OK;
    }
    return comb_dev<uint8_t>(E, d_a, m, d_b, n, d_row_to_col, d_col_to_row, d_score, opts, s);
}

int slcs_lcs_u8(const uint8_t *a, int m, const uint8_t *b, int n, int32_t *score) {
    if (!score) return fail(SLCS_ERR_ARG, "NULL score");
    if (m < 0 || n < 0) return fail(SLCS_ERR_ARG, "negative length");
    if ((m > 0 && !a) || (n > 0 && !b)) return fail(SLCS_ERR_ARG, "NULL buffer");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    if (m == 0 || n == 0) {   // no cells: the score is 0 (still only with a usable device, like every call)
        Engine *E;
        SLCS_TRY(engine(&E));
        *score = 0;
        return SLCS_OK;
    }
    std::vector<int32_t> r2c((size_t) m + n);
    return slcs_comb_u8(a, m, b, n, r2c.data(), nullptr, score, nullptr);
}

}  // extern "C"
