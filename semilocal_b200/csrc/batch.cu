// batch.cu -- batched combing of many independent pairs: one persistent, length-bucketed launch.
//
// Work items are (pair, band) with a per-item band height 32*R (R from the pair's length: long pairs use
// R = 32, the last band of a pair the smallest height covering it); items are ordered by a target start time
// (band k of a pair at k times its share of the launch, first bands by decreasing pair cost), and persistent
// warps dequeue them in that order.  The device step
// (counter resets, the combing launch, the end->start inversion) can be captured once in a CUDA graph and
// replayed.  Mode 1 issues one launch per pair instead (the per-pair baseline on the same plan).
#include <algorithm>
#include <numeric>

#include "slcs_internal.cuh"

namespace slcs {
namespace {

__global__ void invert_batch_kernel(const int32_t *__restrict__ c2r_cat, const int64_t *__restrict__ out_off,
                                    int32_t *__restrict__ r2c_cat, int *err) {
    const int p = blockIdx.x;
    const int64_t o = out_off[p];
    const int size = (int) (out_off[p + 1] - o);
    for (int i = threadIdx.x; i < size; i += blockDim.x) {
        const int r = c2r_cat[o + i];
        if (r < 0 || r >= size) {   // never expected: report instead of writing out of bounds
            raise_error(err, kDevErrBadState);
            continue;
        }
        r2c_cat[o + r] = i;
    }
}

__global__ void identity_fill_kernel(int32_t *__restrict__ c2r_cat, const int64_t *__restrict__ out_off,
                                     const int32_t *__restrict__ empty_pairs, int nempty) {
    const int k = blockIdx.x;
    if (k >= nempty) return;
    const int p = empty_pairs[k];
    const int64_t o = out_off[p];
    const int size = (int) (out_off[p + 1] - o);
    for (int i = threadIdx.x; i < size; i += blockDim.x) c2r_cat[o + i] = i;
}

}  // namespace
}  // namespace slcs

using namespace slcs;

struct slcs_batch {
    int device = 0;
    int npairs = 0;
    int mode = 0;
    std::vector<int32_t> m, n;
    std::vector<int64_t> out_off;
    std::vector<CombItem> items;
    std::vector<int> item_begin;    // per launch (mode 1: per pair in LPT order)
    std::vector<int> empty;
    int64_t a_len = 0, b_len = 0, total = 0, prog_total = 0, cells = 0;
    int resident = 0;
    // device
    uint8_t *da = nullptr, *db = nullptr;
    int32_t *dc2r = nullptr, *dr2c = nullptr, *dprog = nullptr, *dsc = nullptr, *derr = nullptr, *dempty = nullptr;
    int64_t *doff = nullptr;
    CombPair *dpairs = nullptr;
    CombItem *ditems = nullptr;
    int *dnext = nullptr;
    std::vector<int64_t> a_off, b_off;
    bool pairs_ready = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t graph_stream = nullptr;
};

namespace {

int batch_step(slcs_batch *bt, cudaStream_t s, bool capturing) {
    NvtxRange nv("slcs: batch step");
    // inside a capture the timing events must become external event-record nodes of the graph
    const unsigned evflags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    const int np = bt->npairs;
    SLCS_CUDA_TRY(cudaMemsetAsync(bt->dprog, 0, sizeof(int32_t) * std::max<int64_t>(bt->prog_total, 1), s));
    SLCS_CUDA_TRY(cudaMemsetAsync(bt->dsc, 0, sizeof(int32_t) * np, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(bt->derr, 0, sizeof(int), s));
    SLCS_CUDA_TRY(cudaMemsetAsync(bt->dnext, 0, sizeof(int) * (np + 1), s));
    if (!bt->empty.empty()) {
        identity_fill_kernel<<<(int) bt->empty.size(), 256, 0, s>>>(bt->dc2r, bt->doff, bt->dempty,
                                                                   (int) bt->empty.size());
        SLCS_CUDA_TRY(cudaGetLastError());
    }
    SLCS_CUDA_TRY(cudaEventRecordWithFlags(bt->ev0, s, evflags));
    const int nl = (int) bt->item_begin.size() - 1;
    for (int l = 0; l < nl; ++l) {
        const int cnt = bt->item_begin[l + 1] - bt->item_begin[l];
        if (cnt == 0) continue;
        SLCS_TRY(launch_comb<uint8_t>(bt->dpairs, bt->ditems + bt->item_begin[l], cnt, bt->dnext + l, bt->derr,
                                      bt->resident, s));
    }
    SLCS_CUDA_TRY(cudaEventRecordWithFlags(bt->ev1, s, evflags));
    invert_batch_kernel<<<np, 256, 0, s>>>(bt->dc2r, bt->doff, bt->dr2c, bt->derr);
    SLCS_CUDA_TRY(cudaGetLastError());
    return SLCS_OK;
}

}  // namespace

extern "C" {

int slcs_batch_create(const int32_t *m, const int32_t *n, int npairs, int mode, const slcs_opts *opts,
                      slcs_batch **out) {
    if (!out || npairs < 0 || (npairs > 0 && (!m || !n))) return fail(SLCS_ERR_ARG, "bad batch arguments");
    if (mode != 0 && mode != 1) return fail(SLCS_ERR_ARG, "mode must be 0 (batched) or 1 (per pair)");
    *out = nullptr;
    Engine *E;
    SLCS_TRY(engine(&E));
    auto bt = new slcs_batch();
    bt->device = E->device;
    bt->npairs = npairs;
    bt->mode = mode;
    bt->m.assign(m, m + npairs);
    bt->n.assign(n, n + npairs);
    bt->out_off.assign(npairs + 1, 0);
    for (int i = 0; i < npairs; ++i) {
        if (m[i] < 0 || n[i] < 0 || (long long) m[i] + n[i] >= (1ll << 30)) {
            delete bt;
            return fail(SLCS_ERR_ARG, "pair length out of range");
        }
        bt->out_off[i + 1] = bt->out_off[i] + m[i] + n[i];
        bt->cells += (int64_t) m[i] * n[i];
        if (m[i] == 0 || n[i] == 0) bt->empty.push_back(i);
    }
    bt->total = bt->out_off[npairs];
    // length buckets: every pair gets the band height tuned for its row count (or the caller's)
    const int Rforce = (opts && opts->band_rows) ? std::max(1, opts->band_rows / 32) : 0;
    std::vector<int> order(npairs);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return (long long) m[x] * n[x] > (long long) m[y] * n[y]; });
    bt->item_begin.push_back(0);
    for (int oi = 0; oi < npairs; ++oi) {
        const int p = order[oi];
        if (m[p] > 0 && n[p] > 0) {
            // mode 1 launches every pair alone, so it takes the band height tuned for a lone pair
            const int R = Rforce ? Rforce : (mode == 1 ? pick_rows_single(m[p]) : pick_rows_batch(m[p]));
            bt->prog_total += plan_bands(p, m[p], R, bt->items);
            if (mode == 1) bt->item_begin.push_back((int) bt->items.size());
        }
    }
    if (mode == 0) {
        // Work order: band k of pair p gets the target start k (T - D_p) / B_p, with D_p the time of its longest
        // band (columns x band height), B_p its band count and T the launch's work over the resident warps; ties by
        // band index, then by decreasing pair cost (every pair's first band comes first).  A pair's bands are
        // spread over the launch so that its last band starts early enough to end with it (plain band-major order
        // leaves the late bands of the longest pairs, each a long item, for the very end), while consecutive bands
        // of a pair stay far apart in the order, so a warp takes band k only after band k-1 is well under way
        // instead of polling behind it.  A band still waits only on a band taken earlier: no assumption about
        // co-residency is added.
        const double W = std::max(1, comb_resident_warps(E));
        std::vector<int> nb(npairs, 0);
        std::vector<double> gap(npairs, 0.0);
        double work = 0;
        for (const CombItem &it : bt->items) {
            const double d = (double) (bt->n[it.pair] + 32) * 32.0 * it.R;
            nb[it.pair]++;
            gap[it.pair] = std::max(gap[it.pair], d);
            work += d;
        }
        for (int p = 0; p < npairs; ++p)
            if (nb[p]) gap[p] = std::max(work / W - gap[p], 0.0) / nb[p];
        std::stable_sort(bt->items.begin(), bt->items.end(), [&](const CombItem &x, const CombItem &y) {
            const double kx = x.band * gap[x.pair], ky = y.band * gap[y.pair];
            if (kx != ky) return kx < ky;
            return x.band < y.band;
        });
        bt->item_begin.push_back((int) bt->items.size());
    }
    bt->resident = comb_resident_warps(E);
    cudaStream_t s = E->stream;
    auto cleanup_fail = [&](int rc) {
        slcs_batch_destroy(bt);
        return rc;
    };
    int rc;
#define BT_ALLOC(ptr, count) \
    if ((rc = dalloc(reinterpret_cast<void **>(&bt->ptr), sizeof(*bt->ptr) * std::max<int64_t>((count), 1), s)) != SLCS_OK) \
        return cleanup_fail(rc);
    BT_ALLOC(dc2r, bt->total);
    BT_ALLOC(dr2c, bt->total);
    BT_ALLOC(dprog, bt->prog_total);
    BT_ALLOC(dsc, npairs);
    BT_ALLOC(derr, 1);
    BT_ALLOC(doff, npairs + 1);
    BT_ALLOC(dpairs, npairs);
    BT_ALLOC(ditems, bt->items.size());
    BT_ALLOC(dnext, npairs + 1);
    BT_ALLOC(dempty, bt->empty.size());
#undef BT_ALLOC
    if (cudaEventCreate(&bt->ev0) != cudaSuccess || cudaEventCreate(&bt->ev1) != cudaSuccess)
        return cleanup_fail(fail(SLCS_ERR_CUDA, "cudaEventCreate failed"));
    if (cudaMemcpyAsync(bt->doff, bt->out_off.data(), sizeof(int64_t) * (npairs + 1), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        (!bt->items.empty() && cudaMemcpyAsync(bt->ditems, bt->items.data(), sizeof(CombItem) * bt->items.size(),
                                               cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        (!bt->empty.empty() && cudaMemcpyAsync(bt->dempty, bt->empty.data(), sizeof(int32_t) * bt->empty.size(),
                                               cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return cleanup_fail(fail(SLCS_ERR_CUDA, "batch plan upload failed"));
    // the pair descriptors need the device string pointers: they are written by slcs_batch_upload
    bt->pairs_ready = false;
    *out = bt;
    return SLCS_OK;
}

int slcs_batch_upload(slcs_batch *bt, const uint8_t *a_cat, const int64_t *a_off, const uint8_t *b_cat,
                      const int64_t *b_off, void *stream) {
    if (!bt || (bt->npairs > 0 && (!a_off || !b_off))) return fail(SLCS_ERR_ARG, "bad upload arguments");
    SLCS_CUDA_TRY(cudaSetDevice(bt->device));
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    const int np = bt->npairs;
    int64_t a_len = 0, b_len = 0;
    for (int i = 0; i < np; ++i) {
        if (a_off[i] < 0 || b_off[i] < 0) return fail(SLCS_ERR_ARG, "negative offset");
        a_len = std::max<int64_t>(a_len, a_off[i] + bt->m[i]);
        b_len = std::max<int64_t>(b_len, b_off[i] + bt->n[i]);
    }
    if ((a_len > 0 && !a_cat) || (b_len > 0 && !b_cat)) return fail(SLCS_ERR_ARG, "NULL strings");
    if (a_len > bt->a_len || !bt->da) {
        if (bt->da) dfree(bt->da, s);
        bt->da = nullptr;
        SLCS_TRY(dalloc(reinterpret_cast<void **>(&bt->da), std::max<int64_t>(a_len, 1), s));
        bt->a_len = a_len;
        bt->pairs_ready = false;
    }
    if (b_len > bt->b_len || !bt->db) {
        if (bt->db) dfree(bt->db, s);
        bt->db = nullptr;
        SLCS_TRY(dalloc(reinterpret_cast<void **>(&bt->db), std::max<int64_t>(b_len, 1), s));
        bt->b_len = b_len;
        bt->pairs_ready = false;
    }
    if (a_len) SLCS_CUDA_TRY(cudaMemcpyAsync(bt->da, a_cat, a_len, cudaMemcpyHostToDevice, s));
    if (b_len) SLCS_CUDA_TRY(cudaMemcpyAsync(bt->db, b_cat, b_len, cudaMemcpyHostToDevice, s));
    bool same = bt->pairs_ready;
    for (int i = 0; i < np && same; ++i) same = bt->a_off[i] == a_off[i] && bt->b_off[i] == b_off[i];
    if (!same) {
        // one progress slot per band: pair p's slots are a contiguous range (whatever the items' order)
        std::vector<int64_t> prog_off(np + 1, 0);
        for (const CombItem &it : bt->items) prog_off[it.pair + 1]++;
        for (int p = 0; p < np; ++p) prog_off[p + 1] += prog_off[p];
        std::vector<CombPair> hp(np);
        for (int p = 0; p < np; ++p)
            hp[p] = CombPair{bt->da + a_off[p], bt->db + b_off[p], bt->dc2r + bt->out_off[p], bt->dprog + prog_off[p],
                             bt->dsc + p, bt->m[p], bt->n[p]};
        SLCS_CUDA_TRY(cudaMemcpyAsync(bt->dpairs, hp.data(), sizeof(CombPair) * std::max(np, 1), cudaMemcpyHostToDevice, s));
        SLCS_CUDA_TRY(cudaStreamSynchronize(s));
        bt->a_off.assign(a_off, a_off + np);
        bt->b_off.assign(b_off, b_off + np);
        bt->pairs_ready = true;
        if (bt->gexec) {
            cudaGraphExecDestroy(bt->gexec);
            bt->gexec = nullptr;
        }
        if (bt->graph) {
            cudaGraphDestroy(bt->graph);
            bt->graph = nullptr;
        }
    }
    return SLCS_OK;
}

int slcs_batch_run(slcs_batch *bt, int use_graph, void *stream) {
    if (!bt || !bt->pairs_ready) return fail(SLCS_ERR_ARG, "batch not uploaded");
    SLCS_CUDA_TRY(cudaSetDevice(bt->device));
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    if (!use_graph) return batch_step(bt, s, false);
    if (!bt->gexec) {
        cudaStream_t cap;
        SLCS_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        SLCS_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        int rc = batch_step(bt, cap, true);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc != SLCS_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return fail(SLCS_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(e));
        bt->graph = g;
        SLCS_CUDA_TRY(cudaGraphInstantiate(&bt->gexec, g, 0));
    }
    SLCS_CUDA_TRY(cudaGraphLaunch(bt->gexec, s));
    return SLCS_OK;
}

int slcs_batch_download(slcs_batch *bt, int32_t *row_to_col_cat, int32_t *scores, void *stream) {
    if (!bt) return fail(SLCS_ERR_ARG, "NULL batch");
    SLCS_CUDA_TRY(cudaSetDevice(bt->device));
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    if (row_to_col_cat && bt->total)
        SLCS_CUDA_TRY(cudaMemcpyAsync(row_to_col_cat, bt->dr2c, sizeof(int32_t) * bt->total, cudaMemcpyDeviceToHost, s));
    if (scores && bt->npairs)
        SLCS_CUDA_TRY(cudaMemcpyAsync(scores, bt->dsc, sizeof(int32_t) * bt->npairs, cudaMemcpyDeviceToHost, s));
    return check_dev_err(bt->derr, s);
}

int slcs_batch_kernel_ms(slcs_batch *bt, float *ms) {
    if (!bt || !ms) return fail(SLCS_ERR_ARG, "NULL argument");
    SLCS_CUDA_TRY(cudaEventSynchronize(bt->ev1));
    SLCS_CUDA_TRY(cudaEventElapsedTime(ms, bt->ev0, bt->ev1));
    return SLCS_OK;
}

int slcs_batch_info(slcs_batch *bt, int64_t *cells, int32_t *launches, int64_t *h2d_bytes, int64_t *d2h_bytes) {
    if (!bt) return fail(SLCS_ERR_ARG, "NULL batch");
    if (cells) *cells = bt->cells;
    if (launches) {
        int nl = 0;
        for (size_t l = 0; l + 1 < bt->item_begin.size(); ++l) nl += bt->item_begin[l + 1] > bt->item_begin[l];
        *launches = nl + 1 + (bt->empty.empty() ? 0 : 1);   // combing launch(es) + inversion (+ identity fill)
    }
    int64_t in = 0;
    for (int i = 0; i < bt->npairs; ++i) in += bt->m[i] + bt->n[i];
    if (h2d_bytes) *h2d_bytes = in;
    if (d2h_bytes) *d2h_bytes = 4 * bt->total + 4ll * bt->npairs;
    return SLCS_OK;
}

int slcs_batch_destroy(slcs_batch *bt) {
    if (!bt) return SLCS_OK;
    cudaSetDevice(bt->device);
    Engine *E = nullptr;
    cudaStream_t s = nullptr;
    if (engine(&E) == SLCS_OK) s = E->stream;
    if (s) cudaStreamSynchronize(s);
    if (bt->gexec) cudaGraphExecDestroy(bt->gexec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    if (bt->ev0) cudaEventDestroy(bt->ev0);
    if (bt->ev1) cudaEventDestroy(bt->ev1);
    void *ptrs[] = {bt->da, bt->db, bt->dc2r, bt->dr2c, bt->dprog, bt->dsc, bt->derr, bt->dempty,
                    bt->doff, bt->dpairs, bt->ditems, bt->dnext};
    for (void *p : ptrs) dfree(p, s);
    if (s) cudaStreamSynchronize(s);
    delete bt;
    return SLCS_OK;
}

int slcs_batch_comb_u8(const uint8_t *a_cat, const int64_t *a_off, const int32_t *m, const uint8_t *b_cat,
                       const int64_t *b_off, const int32_t *n, int npairs, int32_t *row_to_col_cat,
                       int32_t *scores, int mode, const slcs_opts *opts) {
    if (npairs < 0) return fail(SLCS_ERR_ARG, "negative pair count");
    if (npairs == 0) return SLCS_OK;
    if (!a_cat || !a_off || !m || !b_cat || !b_off || !n || !row_to_col_cat) return fail(SLCS_ERR_ARG, "NULL buffer");
    slcs_batch *bt = nullptr;
    SLCS_TRY(slcs_batch_create(m, n, npairs, mode, opts, &bt));
    int rc = slcs_batch_upload(bt, a_cat, a_off, b_cat, b_off, nullptr);
    if (rc == SLCS_OK) rc = slcs_batch_run(bt, 0, nullptr);
    if (rc == SLCS_OK) rc = slcs_batch_download(bt, row_to_col_cat, scores, nullptr);
    slcs_batch_destroy(bt);
    return rc;
}

}  // extern "C"
