// plans.cu -- reusable single-pair plans: wavefront, hybrid or bit-parallel behind one handle.
//
// create() does all host planning and device allocation; run() only launches kernels (the first run on a
// new pair of string pointers also writes the descriptors that point into them), so from the second run on
// a run can be captured once into a CUDA graph and replayed.
#include <algorithm>

#include "slcs_internal.cuh"

using namespace slcs;

struct slcs_pair_plan {
    int kind = SLCS_ALGO_WAVEFRONT;
    int m = 0, n = 0, device = 0;
    int *d_err = nullptr;
    // wavefront
    std::vector<CombItem> items;
    CombItem *d_items = nullptr;
    CombPair *d_pair = nullptr;
    int32_t *d_prog = nullptr, *d_c2r = nullptr;
    int *d_next = nullptr;
    int bands = 0, resident = 0;
    bool tile = false;                       // the register-tile kernel (else the band kernel)
    int tile_cols = 0;
    unsigned long long *d_hand = nullptr;    // its hand-off words (n)
    const void *ba = nullptr, *bb = nullptr, *bscore = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // hybrid / bit
    HybridPlan *hyb = nullptr;
    BitPlan *bit = nullptr;
    HyyroPlan *hy = nullptr;
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const void *ga = nullptr, *gb = nullptr, *gr = nullptr, *gs = nullptr;
};

namespace {

int wave_run(slcs_pair_plan *P, const uint8_t *d_a, const uint8_t *d_b, int32_t *d_r2c, int32_t *d_score,
             cudaStream_t s, bool capturing) {
    if (P->ba != d_a || P->bb != d_b || P->bscore != d_score) {
        if (capturing) return fail(SLCS_ERR_ARG, "plan must run once on these buffers before capture");
        CombPair hp{d_a, d_b, P->d_c2r, P->d_prog, d_score, P->m, P->n, P->d_hand};
        SLCS_CUDA_TRY(cudaMemcpyAsync(P->d_pair, &hp, sizeof(hp), cudaMemcpyHostToDevice, s));
        SLCS_CUDA_TRY(cudaStreamSynchronize(s));
        P->ba = d_a;
        P->bb = d_b;
        P->bscore = d_score;
    }
    if (P->tile)
        SLCS_CUDA_TRY(cudaMemsetAsync(P->d_hand, 0, sizeof(unsigned long long) * P->n, s));
    else
        SLCS_CUDA_TRY(cudaMemsetAsync(P->d_prog, 0, sizeof(int32_t) * std::max(P->bands, 1), s));
    SLCS_CUDA_TRY(cudaMemsetAsync(P->d_next, 0, sizeof(int), s));
    if (d_score) SLCS_CUDA_TRY(cudaMemsetAsync(d_score, 0, sizeof(int32_t), s));
    const unsigned fl = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    SLCS_CUDA_TRY(cudaEventRecordWithFlags(P->ev0, s, fl));
    if (P->tile)
        SLCS_TRY(launch_comb_tile<uint8_t>(P->d_pair, P->d_items, (int) P->items.size(), P->d_next, P->d_err,
                                           P->resident, P->tile_cols, s));
    else
        SLCS_TRY(launch_comb_lone<uint8_t>(P->d_pair, P->d_items, (int) P->items.size(), P->d_next, P->d_err,
                                           P->resident, s));
    SLCS_CUDA_TRY(cudaEventRecordWithFlags(P->ev1, s, fl));
    SLCS_TRY(launch_invert(P->d_c2r, P->m + P->n, d_r2c, false, P->d_err, s));
    return SLCS_OK;
}

int plan_run(slcs_pair_plan *P, const uint8_t *d_a, const uint8_t *d_b, int32_t *d_r2c, int32_t *d_score,
             cudaStream_t s, bool capturing) {
    if (P->kind == SLCS_ALGO_WAVEFRONT) return wave_run(P, d_a, d_b, d_r2c, d_score, s, capturing);
    if (P->kind == SLCS_ALGO_HYBRID) {
        hybrid_set_capturing(P->hyb, capturing);
        SLCS_TRY(hybrid_plan_run<uint8_t>(P->hyb, d_a, d_b, P->d_err, s));
        if (d_r2c)
            SLCS_CUDA_TRY(cudaMemcpyAsync(d_r2c, hybrid_result_r2c(P->hyb), sizeof(int32_t) * (P->m + P->n),
                                          cudaMemcpyDeviceToDevice, s));
        if (d_score) SLCS_TRY(hybrid_score(P->hyb, d_score, s));
        return SLCS_OK;
    }
    if (P->kind == SLCS_PLAN_HYYRO) return hyyro_plan_run(P->hy, d_a, d_b, d_score, P->d_err, s, capturing);
    return bit_plan_run(P->bit, d_a, d_b, d_score, P->d_err, s, capturing);
}

}  // namespace

extern "C" {

int slcs_pair_plan_destroy(slcs_pair_plan *P) {
    if (!P) return SLCS_OK;
    cudaSetDevice(P->device);
    Engine *E = nullptr;
    cudaStream_t s = nullptr;
    if (engine(&E) == SLCS_OK) s = E->stream;
    if (s) cudaStreamSynchronize(s);
    if (P->gexec) cudaGraphExecDestroy(P->gexec);
    if (P->graph) cudaGraphDestroy(P->graph);
    if (P->ev0) cudaEventDestroy(P->ev0);
    if (P->ev1) cudaEventDestroy(P->ev1);
    if (P->hyb) hybrid_plan_destroy(P->hyb);
    if (P->bit) bit_plan_destroy(P->bit);
    if (P->hy) hyyro_plan_destroy(P->hy);
    void *ps[] = {P->d_err, P->d_items, P->d_pair, P->d_prog, P->d_c2r, P->d_next, P->d_hand};
    for (void *p : ps) dfree(p, s);
    if (s) cudaStreamSynchronize(s);
    delete P;
    return SLCS_OK;
}

int slcs_pair_plan_create(int m, int n, int kind, const slcs_opts *opts, slcs_pair_plan **out) {
    if (!out || m < 1 || n < 1 || (long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_ARG, "bad plan arguments");
    if (kind != SLCS_ALGO_WAVEFRONT && kind != SLCS_ALGO_HYBRID && kind != SLCS_PLAN_BITPARALLEL &&
        kind != SLCS_PLAN_HYYRO)
        return fail(SLCS_ERR_ARG, "unknown plan kind");
    *out = nullptr;
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = E->stream;
    auto P = new slcs_pair_plan();
    P->kind = kind;
    P->m = m;
    P->n = n;
    P->device = E->device;
    auto bail = [&](int rc) {
        slcs_pair_plan_destroy(P);
        return rc;
    };
    int rc;
    if ((rc = dalloc(reinterpret_cast<void **>(&P->d_err), sizeof(int), s))) return bail(rc);
    if (cudaMemsetAsync(P->d_err, 0, sizeof(int), s) != cudaSuccess) return bail(fail(SLCS_ERR_CUDA, "memset"));
    if (kind == SLCS_ALGO_WAVEFRONT) {
        const int band_rows = opts ? opts->band_rows : 0;
        const TileShape ts = tile_shape_for(m, band_rows, opts ? opts->lane_cols : 0);
        P->tile = ts.R > 0;
        P->tile_cols = ts.C;
        if (P->tile) {
            P->bands = plan_tile_bands(0, m, ts.R, P->items);
            if ((rc = dalloc(reinterpret_cast<void **>(&P->d_hand), sizeof(unsigned long long) * n, s)))
                return bail(rc);
        } else {
            const int R = band_rows > 0 ? std::max(1, band_rows / 32) : pick_rows_single(m);
            P->bands = plan_bands(0, m, R, P->items);
        }
        P->resident = comb_resident_warps(E);
        if ((rc = dalloc(reinterpret_cast<void **>(&P->d_items), sizeof(CombItem) * P->items.size(), s)) ||
            (rc = dalloc(reinterpret_cast<void **>(&P->d_pair), sizeof(CombPair), s)) ||
            (rc = dalloc(reinterpret_cast<void **>(&P->d_prog), sizeof(int32_t) * P->bands, s)) ||
            (rc = dalloc(reinterpret_cast<void **>(&P->d_c2r), sizeof(int32_t) * (m + n), s)) ||
            (rc = dalloc(reinterpret_cast<void **>(&P->d_next), sizeof(int), s)))
            return bail(rc);
        if (cudaMemcpyAsync(P->d_items, P->items.data(), sizeof(CombItem) * P->items.size(), cudaMemcpyHostToDevice, s) !=
                cudaSuccess ||
            cudaEventCreate(&P->ev0) != cudaSuccess || cudaEventCreate(&P->ev1) != cudaSuccess)
            return bail(fail(SLCS_ERR_CUDA, "plan setup failed"));
    } else if (kind == SLCS_ALGO_HYBRID) {
        const int tr = (opts && opts->tile_rows > 0) ? opts->tile_rows : pick_tile();
        const int tc = (opts && opts->tile_cols > 0) ? opts->tile_cols : pick_tile();
        if ((rc = hybrid_plan_create(m, n, tr, tc, E, s, &P->hyb)) || (rc = hybrid_enable_timing(P->hyb)))
            return bail(rc);
    } else {
        if (kind == SLCS_PLAN_HYYRO) {
            if ((rc = hyyro_plan_create(E, m, n, s, &P->hy))) return bail(rc);
        } else if ((rc = bit_plan_create(E, m, n, s, &P->bit))) {
            return bail(rc);
        }
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(SLCS_ERR_CUDA, "plan setup failed"));
    *out = P;
    return SLCS_OK;
}

int slcs_pair_plan_run(slcs_pair_plan *P, const uint8_t *d_a, const uint8_t *d_b, int32_t *d_row_to_col,
                       int32_t *d_score, int use_graph, void *stream) {
    if (!P || !d_a || !d_b) return fail(SLCS_ERR_ARG, "NULL argument");
    const bool score_only = P->kind == SLCS_PLAN_BITPARALLEL || P->kind == SLCS_PLAN_HYYRO;
    if (!score_only && !d_row_to_col) return fail(SLCS_ERR_ARG, "NULL row_to_col");
    if (score_only && !d_score) return fail(SLCS_ERR_ARG, "NULL score");
    SLCS_CUDA_TRY(cudaSetDevice(P->device));
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    if (!use_graph) return plan_run(P, d_a, d_b, d_row_to_col, d_score, s, false);
    if (!P->gexec || P->ga != d_a || P->gb != d_b || P->gr != d_row_to_col || P->gs != d_score) {
        // bind the descriptors outside the capture, then capture a pure launch sequence
        SLCS_TRY(plan_run(P, d_a, d_b, d_row_to_col, d_score, s, false));
        SLCS_CUDA_TRY(cudaStreamSynchronize(s));
        if (P->gexec) cudaGraphExecDestroy(P->gexec);
        if (P->graph) cudaGraphDestroy(P->graph);
        P->gexec = nullptr;
        P->graph = nullptr;
        cudaStream_t cap;
        SLCS_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        SLCS_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        const int rc = plan_run(P, d_a, d_b, d_row_to_col, d_score, cap, true);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc != SLCS_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return rc != SLCS_OK ? rc : fail(SLCS_ERR_CUDA, std::string("capture failed: ") + cudaGetErrorString(e));
        }
        P->graph = g;
        SLCS_CUDA_TRY(cudaGraphInstantiate(&P->gexec, g, 0));
        P->ga = d_a;
        P->gb = d_b;
        P->gr = d_row_to_col;
        P->gs = d_score;
    }
    SLCS_CUDA_TRY(cudaGraphLaunch(P->gexec, s));
    return SLCS_OK;
}

int slcs_pair_plan_check(slcs_pair_plan *P, void *stream) {
    if (!P) return fail(SLCS_ERR_ARG, "NULL plan");
    Engine *E;
    SLCS_TRY(engine(&E));
    return check_dev_err(P->d_err, stream ? (cudaStream_t) stream : E->stream);
}

int slcs_pair_plan_kernel_ms(slcs_pair_plan *P, float *ms) {
    if (!P || !ms) return fail(SLCS_ERR_ARG, "NULL argument");
    if (P->kind == SLCS_ALGO_HYBRID) return hybrid_comb_ms(P->hyb, ms);
    if (P->kind == SLCS_PLAN_BITPARALLEL) return bit_plan_kernel_ms(P->bit, ms);
    if (P->kind == SLCS_PLAN_HYYRO) return hyyro_plan_kernel_ms(P->hy, ms);
    SLCS_CUDA_TRY(cudaEventSynchronize(P->ev1));
    SLCS_CUDA_TRY(cudaEventElapsedTime(ms, P->ev0, P->ev1));
    return SLCS_OK;
}

int slcs_pair_plan_launches(slcs_pair_plan *P, int32_t *launches) {
    if (!P || !launches) return fail(SLCS_ERR_ARG, "NULL argument");
    if (P->kind == SLCS_ALGO_HYBRID) *launches = hybrid_launches(P->hyb) + 1;
    else if (P->kind == SLCS_PLAN_BITPARALLEL || P->kind == SLCS_PLAN_HYYRO) *launches = 3;
    else *launches = 2;
    return SLCS_OK;
}

}  // extern "C"
