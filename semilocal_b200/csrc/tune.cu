// tune.cu -- the autotuner.  Per device it chooses, by timing the candidates on synthetic inputs with CUDA
// events on the engine's stream:
//   * the band height (32 R rows per warp band) per row-count class 2^k, for pairs that share a launch
//     (batches, hybrid tiles, serving) and for a pair alone on the device (wavefront plans);
//   * the hybrid tile edge;
//   * the steady-ant cutoff (sub-problems of at most this many common indices finish in shared memory).
// Every entry point that receives 0 for one of these parameters takes the tuned value, or the built-in
// default before any tuning.  The reference fixes these by hand in its callers (tile sizes and thread counts
// of OpenMPHybridIterative, R:include/SemiLocal/SemiLocalLCS.h:602-647; the precalc depth of the steady ant,
// R:common/include/Permutations/MongeMultuplicationStrategy.h:80-111); it has no tuner.
#include <algorithm>
#include <mutex>
#include <vector>

#include "slcs_internal.cuh"

namespace slcs {
namespace {

std::mutex g_tmu;
slcs_tuning g_tab[64];   // all zero = untuned

int cur_device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) {
        cudaGetLastError();
        d = 0;
    }
    return (d < 0 || d >= 64) ? 0 : d;
}

int log2_class(int rows) {   // ceil(log2(rows)), rows >= 1
    int k = 0;
    while (k < 31 && (1 << k) < rows) ++k;
    return k;
}

int default_rows_single(int rows) {
    // enough bands to spread one pair over the device, but long bands for throughput
    int R = 1;
    while (R < 32 && 32 * 64 * R * 2 <= rows) R *= 2;
    return R;
}

struct Rng {
    uint64_t x;
    uint64_t next() {
        uint64_t z = (x += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
};

void random_symbols(std::vector<uint8_t> &v, size_t len, uint64_t seed) {
    Rng r{seed};
    v.resize(len);
    for (size_t i = 0; i < len; ++i) v[i] = (uint8_t) (r.next() & 3);
}

// b = a with every position substituted by a different letter with probability 1/10
void mutated(const std::vector<uint8_t> &a, std::vector<uint8_t> &b, uint64_t seed) {
    Rng r{seed};
    b = a;
    for (auto &c : b)
        if (r.next() % 10 == 0) c = (uint8_t) ((c + 1 + r.next() % 3) & 3);
}

struct Timer {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    Timer() {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
    }
    ~Timer() {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
};

// the fastest of three timed runs of fn (CUDA events on s)
template <typename F>
int best_of(cudaStream_t s, float *ms, F fn) {
    Timer T;
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        float t = 0;
        if (cudaEventRecord(T.e0, s) != cudaSuccess) return fail(SLCS_ERR_CUDA, "tuning timing failed");
        SLCS_TRY(fn());
        if (cudaEventRecord(T.e1, s) != cudaSuccess || cudaEventSynchronize(T.e1) != cudaSuccess ||
            cudaEventElapsedTime(&t, T.e0, T.e1) != cudaSuccess)
            return fail(SLCS_ERR_CUDA, "tuning timing failed");
        best = std::min(best, t);
    }
    *ms = best;
    return SLCS_OK;
}

// The candidate to install: the fastest, unless the built-in default is within 3 % of it (timing noise must
// not move a parameter away from its default).
int choose(const std::vector<std::pair<int, float>> &timed, int dflt) {
    float best = 1e30f, tdef = -1;
    int arg = dflt;
    for (const auto &c : timed) {
        if (c.second < best) {
            best = c.second;
            arg = c.first;
        }
        if (c.first == dflt) tdef = c.second;
    }
    return (tdef >= 0 && tdef <= 1.03f * best) ? dflt : arg;
}

// Warps of the combing kernel resident on the current device at once (cached per device).
int resident_warps_now() {
    static int cache[64] = {0};
    const int d = cur_device();
    if (!cache[d]) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d) != cudaSuccess || sms <= 0) {
            cudaGetLastError();
            return 1 << 30;
        }
        cache[d] = comb_resident_warps_sm(sms);
    }
    return cache[d];
}

// ms of one batched run of np pairs of L x L cells at band height 32 R (the fastest of three)
int time_batch(int L, int np, int R, cudaStream_t s, float *ms) {
    std::vector<int32_t> m(np, L), n(np, L);
    std::vector<int64_t> off(np);
    std::vector<uint8_t> a, b, acat, bcat;
    acat.reserve((size_t) L * np);
    bcat.reserve((size_t) L * np);
    for (int i = 0; i < np; ++i) {
        random_symbols(a, L, 1000 + i);
        mutated(a, b, 2000 + i);
        off[i] = (int64_t) i * L;
        acat.insert(acat.end(), a.begin(), a.end());
        bcat.insert(bcat.end(), b.begin(), b.end());
    }
    slcs_opts o{};
    o.band_rows = 32 * R;
    slcs_batch *bt = nullptr;
    SLCS_TRY(slcs_batch_create(m.data(), n.data(), np, 0, &o, &bt));
    int rc = slcs_batch_upload(bt, acat.data(), off.data(), bcat.data(), off.data(), s);
    if (rc == SLCS_OK) rc = slcs_batch_run(bt, 0, s);   // warm-up
    if (rc == SLCS_OK) rc = best_of(s, ms, [&] { return slcs_batch_run(bt, 0, s); });
    slcs_batch_destroy(bt);
    return rc;
}

// ms of one single-pair plan run (kind, opts) on an L x L pair (the fastest of three)
int time_pair(int L, int kind, const slcs_opts &o, cudaStream_t s, float *ms) {
    std::vector<uint8_t> a, b;
    random_symbols(a, L, 77);
    mutated(a, b, 78);
    slcs_pair_plan *pl = nullptr;
    SLCS_TRY(slcs_pair_plan_create(L, L, kind, &o, &pl));
    int rc = SLCS_OK;
    uint8_t *da = nullptr, *db = nullptr;
    int32_t *dr = nullptr, *dsc = nullptr;
    if ((rc = dalloc(reinterpret_cast<void **>(&da), L, s)) == SLCS_OK &&
        (rc = dalloc(reinterpret_cast<void **>(&db), L, s)) == SLCS_OK &&
        (rc = dalloc(reinterpret_cast<void **>(&dr), sizeof(int32_t) * 2 * (size_t) L, s)) == SLCS_OK &&
        (rc = dalloc(reinterpret_cast<void **>(&dsc), sizeof(int32_t), s)) == SLCS_OK) {
        if (cudaMemcpyAsync(da, a.data(), L, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(db, b.data(), L, cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = fail(SLCS_ERR_CUDA, "tuning upload failed");
        if (rc == SLCS_OK) rc = slcs_pair_plan_run(pl, da, db, dr, dsc, 0, s);   // warm-up
        if (rc == SLCS_OK) rc = best_of(s, ms, [&] { return slcs_pair_plan_run(pl, da, db, dr, dsc, 0, s); });
        if (rc == SLCS_OK) rc = slcs_pair_plan_check(pl, s);
    }
    dfree(da, s);
    dfree(db, s);
    dfree(dr, s);
    dfree(dsc, s);
    slcs_pair_plan_destroy(pl);
    return rc;
}

// ms of one steady-ant product of two random n x n permutations with the given cutoff
int time_sa(int n, int cutoff, cudaStream_t s, float *ms) {
    std::vector<int32_t> p(n), q(n);
    for (int i = 0; i < n; ++i) p[i] = q[i] = i;
    Rng r{99};
    for (int i = n - 1; i > 0; --i) {
        std::swap(p[i], p[r.next() % (uint64_t) (i + 1)]);
        std::swap(q[i], q[r.next() % (uint64_t) (i + 1)]);
    }
    int32_t *dp = nullptr, *dq = nullptr, *dr = nullptr;
    int *derr = nullptr;
    SaPlan *P = nullptr;
    int rc = SLCS_OK;
    if ((rc = dalloc(reinterpret_cast<void **>(&dp), sizeof(int32_t) * n, s)) == SLCS_OK &&
        (rc = dalloc(reinterpret_cast<void **>(&dq), sizeof(int32_t) * n, s)) == SLCS_OK &&
        (rc = dalloc(reinterpret_cast<void **>(&dr), sizeof(int32_t) * n, s)) == SLCS_OK &&
        (rc = dalloc(reinterpret_cast<void **>(&derr), sizeof(int), s)) == SLCS_OK &&
        (rc = sa_plan_create(std::vector<int64_t>{0}, std::vector<int>{n}, &P, s, nullptr, cutoff)) == SLCS_OK) {
        if (cudaMemcpyAsync(dp, p.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(dq, q.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemsetAsync(derr, 0, sizeof(int), s) != cudaSuccess)
            rc = fail(SLCS_ERR_CUDA, "tuning upload failed");
        if (rc == SLCS_OK) rc = sa_plan_run(P, dp, dq, dr, derr, s);   // warm-up
        if (rc == SLCS_OK) rc = best_of(s, ms, [&] { return sa_plan_run(P, dp, dq, dr, derr, s); });
        if (rc == SLCS_OK) rc = check_dev_err(derr, s);
    }
    if (P) sa_plan_destroy(P);
    dfree(dp, s);
    dfree(dq, s);
    dfree(dr, s);
    dfree(derr, s);
    return rc;
}

}  // namespace

int pick_rows_batch(int rows) {
    std::lock_guard<std::mutex> lk(g_tmu);
    const int v = g_tab[cur_device()].band_rows_batch[log2_class(std::max(rows, 1))];
    return v > 0 ? std::max(1, std::min(32, v / 32)) : 32;
}

int pick_rows_single(int rows) {
    int R;
    {
        std::lock_guard<std::mutex> lk(g_tmu);
        const int v = g_tab[cur_device()].band_rows_single[log2_class(std::max(rows, 1))];
        R = v > 0 ? std::max(1, std::min(32, v / 32)) : default_rows_single(rows);
    }
    // a lone pair's bands must all be resident at once: a band beyond the resident warps starts only when
    // a warp finishes a whole band, which doubles the time
    const int64_t W = resident_warps_now();
    while (R < 32 && ((int64_t) rows + 32 * R - 1) / (32 * R) > W) R *= 2;
    return R;
}

int pick_tile() {
    std::lock_guard<std::mutex> lk(g_tmu);
    const int v = g_tab[cur_device()].tile;
    return v > 0 ? v : 4096;
}

int pick_sa_cutoff() {
    std::lock_guard<std::mutex> lk(g_tmu);
    const int v = g_tab[cur_device()].sa_cutoff;
    return v > 0 ? v : steady_ant_max_small();
}

}  // namespace slcs

using namespace slcs;

extern "C" {

int slcs_tuning_get(slcs_tuning *out) {
    if (!out) return fail(SLCS_ERR_ARG, "NULL output");
    std::lock_guard<std::mutex> lk(g_tmu);
    *out = g_tab[cur_device()];
    return SLCS_OK;
}

int slcs_tuning_set(const slcs_tuning *in) {
    std::lock_guard<std::mutex> lk(g_tmu);
    slcs_tuning t{};
    if (in) {
        t = *in;
        for (int k = 0; k < 32; ++k) {
            const int vb = t.band_rows_batch[k], vs = t.band_rows_single[k];
            if (vb < 0 || vs < 0 || vb > 1024 || vs > 1024) return fail(SLCS_ERR_ARG, "band_rows out of range");
        }
        if (t.tile < 0 || t.sa_cutoff < 0) return fail(SLCS_ERR_ARG, "negative tuning value");
    }
    g_tab[cur_device()] = t;
    return SLCS_OK;
}

int slcs_autotune(int flags, slcs_tuning *out) {
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = E->stream;
    if (flags == 0) flags = SLCS_TUNE_ALL;
    slcs_tuning T{};
    {
        std::lock_guard<std::mutex> lk(g_tmu);
        T = g_tab[E->device];
    }
    const int W = comb_resident_warps(E);
    // 1. band height for pairs sharing a launch, classes 2^8 .. 2^14: L x L pairs, enough of them for at least
    //    four waves of bands (a tuned height must hold in a launch much larger than the device); longer pairs
    //    keep the default (32 rows per lane)
    if (flags & SLCS_TUNE_BANDS_BATCH) {
        for (int k = 8; k <= 14; ++k) {
            const int L = 1 << k;
            const int bands32 = (L + 1023) / 1024;
            const int np = (int) std::min<int64_t>(32768, std::max<int64_t>((4ll * W + bands32 - 1) / bands32,
                                                                            (1ll << 31) / ((int64_t) L * L)));
            std::vector<std::pair<int, float>> timed;
            for (int R = 1; R <= 32; R *= 2) {
                if (32 * R > 2 * L || (L >= 4096 && R < 4)) continue;
                float ms = 0;
                SLCS_TRY(time_batch(L, np, R, s, &ms));
                timed.emplace_back(R, ms);
            }
            T.band_rows_batch[k] = 32 * choose(timed, 32);
        }
        for (int k = 0; k < 8; ++k) T.band_rows_batch[k] = T.band_rows_batch[8];
        for (int k = 15; k < 32; ++k) T.band_rows_batch[k] = 32 * 32;
    }
    // 2. band height for one pair alone: L x L, classes 2^10 .. 2^19; each longer class doubles the height
    //    (the same number of bands), and pick_rows_single keeps every band resident
    if (flags & SLCS_TUNE_BANDS_SINGLE) {
        for (int k = 10; k <= 19; ++k) {
            const int L = 1 << k;
            std::vector<std::pair<int, float>> timed;
            for (int R = 1; R <= 32; R *= 2) {
                if (32 * R > L || (k == 19 && R < 8)) continue;
                slcs_opts o{};
                o.algo = SLCS_ALGO_WAVEFRONT;
                o.band_rows = 32 * R;
                float ms = 0;
                SLCS_TRY(time_pair(L, SLCS_ALGO_WAVEFRONT, o, s, &ms));
                timed.emplace_back(R, ms);
            }
            T.band_rows_single[k] = 32 * choose(timed, default_rows_single(L));
        }
        for (int k = 0; k < 10; ++k) T.band_rows_single[k] = T.band_rows_single[10];
        for (int k = 20; k < 32; ++k) T.band_rows_single[k] = std::min(1024, T.band_rows_single[k - 1] * 2);
    }
    // 3. hybrid tile edge on a 2^17 x 2^17 pair
    if (flags & SLCS_TUNE_TILE) {
        std::vector<std::pair<int, float>> timed;
        for (int tile : {2048, 4096, 8192}) {
            slcs_opts o{};
            o.algo = SLCS_ALGO_HYBRID;
            o.tile_rows = o.tile_cols = tile;
            float ms = 0;
            SLCS_TRY(time_pair(1 << 17, SLCS_ALGO_HYBRID, o, s, &ms));
            timed.emplace_back(tile, ms);
        }
        T.tile = choose(timed, 4096);
    }
    // 4. steady-ant cutoff on two random 2^20 permutations
    if (flags & SLCS_TUNE_SA_CUTOFF) {
        std::vector<std::pair<int, float>> timed;
        for (int c = 1024; c <= steady_ant_max_small(); c *= 2) {
            float ms = 0;
            SLCS_TRY(time_sa(1 << 20, c, s, &ms));
            timed.emplace_back(c, ms);
        }
        T.sa_cutoff = choose(timed, steady_ant_max_small());
    }
    {
        std::lock_guard<std::mutex> lk(g_tmu);
        g_tab[E->device] = T;
    }
    if (out) *out = T;
    return SLCS_OK;
}

}  // extern "C"
