// server.cu -- the serving loop: continuous batching of comparison requests on one GPU.
//
// A request is one pair (a, b) plus one score query on its braid.  The caller submits requests at any time;
// a worker thread owned by the server
//   * admits them by a device-memory budget (inputs, strands and scratch while in flight, the braid while
//     resident), evicting least recently used resident braids when the budget is short;
//   * launches admitted requests as soon as a stream is free: requests of at least big_cells cells run on one
//     of the big streams (two by default; alone, or with other pending big requests when several wait), the
//     others are batched (largest first) into one persistent
//     combing launch on one of the small streams.  Each launch caps its persistent grid (big: half the
//     resident warps, small: a quarter), so long big launches leave SMs to the small batches and their work
//     overlaps on the device; requests that arrive while launches run are admitted into the next launch of a
//     stream that frees up;
//     A launch of big requests whose rows are all at most kTileAutoMaxRows combs them with the register-tile kernel
//     (hand-off words per request, zeroed per launch), otherwise with the band kernel;
//   * after each launch: c2r -> r2c, the request's query, 4 bytes back to the host per request;
//   * keeps every finished braid resident (r2c, m+n int32) for further queries until it is released or
//     evicted.
// The combing of a pair does not depend on what else shares its launch (the bands of a pair only exchange
// data with each other), so a result is the same alone and in any mix.
// The reference has no serving layer; its per-pair entry point is SemiLocalStrategy::compute
// (R:include/SemiLocal/SemiLocalLCS.h:7-11) followed by a score readout (R:include/LCS/LCS.h:223-233,
// R:approximate_matching/utils.h:281-334).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "slcs_internal.cuh"

namespace slcs {
namespace {

struct SrvPair {   // one request of a launch, as the invert / query kernels see it
    const int32_t *c2r;
    int32_t *r2c;
    int m, n;
    slcs_query q;
};

// c2r -> r2c of every request of a launch (blockIdx.y = request); an empty pair's braid is the identity
__global__ void srv_invert_kernel(const SrvPair *__restrict__ pairs, int *err) {
    const SrvPair P = pairs[blockIdx.y];
    const int size = P.m + P.n;
    const bool empty = P.m == 0 || P.n == 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x) {
        if (empty) {
            P.r2c[i] = i;
            continue;
        }
        const int r = P.c2r[i];
        if (r < 0 || r >= size) {   // never expected: report instead of writing out of bounds
            raise_error(err, kDevErrBadState);
            continue;
        }
        P.r2c[r] = i;
    }
}

// the query of every request (one block each): H(i, j) = j + m - i - #{r >= i : r2c[r] < j}
__global__ void __launch_bounds__(256) srv_query_kernel(const SrvPair *__restrict__ pairs, int32_t *__restrict__ out,
                                                        int *err) {
    __shared__ int warp_cnt[8];
    const SrvPair P = pairs[blockIdx.x];
    int i, j, offset;
    bool ok;
    query_to_matrix(P.q, P.m, P.n, i, j, offset, ok);
    if (!ok) {
        if (threadIdx.x == 0) {
            out[blockIdx.x] = INT32_MIN;
            raise_error(err, kDevErrBadState);
        }
        return;
    }
    int cnt = 0;
    if (!(j <= i - P.m))
        for (int r = i + threadIdx.x; r < P.m + P.n; r += blockDim.x) cnt += P.r2c[r] < j;
    cnt = __reduce_add_sync(kFull, cnt);
    if ((threadIdx.x & 31) == 0) warp_cnt[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int total = 0;
        for (int w = 0; w < 8; ++w) total += warp_cnt[w];
        out[blockIdx.x] = ((j <= i - P.m) ? (j - i + P.m) : (j + P.m - i - total)) + offset;
    }
}

bool query_valid(const slcs_query &q, int m, int n) {
    switch (q.kind) {
        case SLCS_Q_GLOBAL: return true;
        case SLCS_Q_STRING_SUBSTRING: return 0 <= q.i && q.i <= q.j && q.j <= n;
        case SLCS_Q_PREFIX_SUFFIX:
        case SLCS_Q_SUFFIX_PREFIX: return 0 <= q.i && q.i <= m && 0 <= q.j && q.j <= n;
        case SLCS_Q_SUBSTRING_STRING: return 0 <= q.i && q.i <= q.j && q.j <= m;
        case SLCS_Q_MATRIX: return 0 <= q.i && q.i <= m + n && 0 <= q.j && q.j <= m + n;
        default: return false;
    }
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Page-locked host blocks in power-of-two size classes, reused across requests.
struct PinnedPool {
    std::mutex mu;
    std::map<size_t, std::vector<void *>> free_blocks;
    std::vector<void *> all;
    void *get(size_t bytes, size_t *cap) {
        size_t c = 4096;
        while (c < bytes) c <<= 1;
        *cap = c;
        {
            std::lock_guard<std::mutex> lk(mu);
            auto &v = free_blocks[c];
            if (!v.empty()) {
                void *p = v.back();
                v.pop_back();
                return p;
            }
        }
        void *p = nullptr;
        if (cudaMallocHost(&p, c) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        std::lock_guard<std::mutex> lk(mu);
        all.push_back(p);
        return p;
    }
    void put(void *p, size_t cap) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(mu);
        free_blocks[cap].push_back(p);
    }
    ~PinnedPool() {
        for (void *p : all) cudaFreeHost(p);
    }
};

struct Req {
    uint64_t ticket = 0;
    int m = 0, n = 0;
    slcs_query q{};
    int64_t cells = 0;
    int64_t need = 0;   // device bytes while in flight
    int64_t keep = 0;   // device bytes of the resident braid
    int R = 32;         // rows per lane of the request's bands
    int tileR = 0;      // rows per lane when a launch of big requests combs it with the register-tile kernel
    int nbands = 0;
    int retries = 0;    // launches of this request that ended in a device-side wait timeout
    double t_submit = 0, t_admit = 0;
    uint8_t *ha = nullptr;   // pinned staging: a then b
    size_t hcap = 0;
    uint8_t *dab = nullptr;   // device: a | b | c2r
    int32_t *dr2c = nullptr;  // device: the braid (resident after the launch)
};

struct Launch {
    cudaStream_t s = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<Req *> reqs;
    void *dmeta = nullptr;   // device: CombPair[np] | CombItem[ni] | SrvPair[np] | progress | out[np] | err | next
    void *dhand = nullptr;   // device: the tile kernel's hand-off words (n per request), when it runs
    void *hmeta = nullptr;   // pinned mirror (out and err come back into it)
    size_t hcap = 0;
    int32_t *hout = nullptr;
    int *herr = nullptr;
};

struct Resident {
    int32_t *r2c = nullptr;
    int m = 0, n = 0;
    int64_t bytes = 0;
    uint64_t lru = 0;
    int pins = 0;
};

}  // namespace
}  // namespace slcs

using namespace slcs;

struct slcs_server {
    int device = 0;
    slcs_server_opts o{};
    int64_t budget = 0;
    int resident_warps = 0;
    std::chrono::steady_clock::time_point t0;
    // client <-> worker
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req *> submitq;
    std::deque<slcs_result> done;
    bool stop = false;
    int64_t submitted = 0, completed = 0, rejected = 0, launches = 0, cells = 0;
    int pending_count = 0, inflight_count = 0;
    // worker-owned
    std::thread worker;
    std::deque<Req *> pending;
    int nbig = 1;
    std::vector<cudaStream_t> streams;   // [0, nbig) big, [nbig, ..) small
    std::vector<Launch *> inflight;      // one launch per stream at most
    // resident braids and the budget
    std::mutex rmu;
    std::unordered_map<uint64_t, Resident> resident;
    uint64_t lru_clock = 0;
    int64_t used = 0, peak = 0, evicted = 0, resident_bytes = 0;
    std::atomic<uint64_t> next_ticket{1};
    PinnedPool pinned;
    // synchronous queries on resident braids
    std::mutex qmu;
    cudaStream_t qstream = nullptr;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

int64_t req_need(int m, int n, int nbands) {
    const size_t ab = align_up((size_t) m + n, 256);
    return (int64_t) (ab + align_up(sizeof(int32_t) * (size_t) (m + n), 256) +   // inputs, c2r
                      align_up(sizeof(int32_t) * (size_t) std::max(m + n, 1), 256) +   // r2c
                      sizeof(int32_t) * (size_t) nbands + sizeof(CombItem) * (size_t) nbands + 512);
}

// Makes room for need bytes (evicting unpinned resident braids, oldest first); false if it cannot.
bool reserve(slcs_server *S, int64_t need, cudaStream_t s) {
    std::lock_guard<std::mutex> lk(S->rmu);
    while (S->used + need > S->budget) {
        auto victim = S->resident.end();
        for (auto it = S->resident.begin(); it != S->resident.end(); ++it)
            if (it->second.pins == 0 && (victim == S->resident.end() || it->second.lru < victim->second.lru)) victim = it;
        if (victim == S->resident.end()) return false;
        dfree(victim->second.r2c, s);
        S->used -= victim->second.bytes;
        S->resident_bytes -= victim->second.bytes;
        S->resident.erase(victim);
        ++S->evicted;
    }
    S->used += need;
    S->peak = std::max(S->peak, S->used);
    return true;
}

void unreserve(slcs_server *S, int64_t bytes) {
    std::lock_guard<std::mutex> lk(S->rmu);
    S->used -= bytes;
}

void finish_req(slcs_server *S, Req *r, int status, int32_t score, double t_done) {
    slcs_result res{};
    res.ticket = r->ticket;
    res.status = status;
    res.score = score;
    res.m = r->m;
    res.n = r->n;
    res.query = r->q;
    res.t_submit = r->t_submit;
    res.t_admit = r->t_admit;
    res.t_done = t_done;
    S->pinned.put(r->ha, r->hcap);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->done.push_back(res);
        ++S->completed;
        if (status == SLCS_OK) S->cells += r->cells;
    }
    S->cv_done.notify_all();
    delete r;
}

// Builds and enqueues one launch of the requests on stream idx.  Their budget is already reserved.
int launch_group(slcs_server *S, int idx, std::vector<Req *> &reqs, int warp_cap, bool lone = false) {
    NvtxRange nv("slcs: server launch");
    cudaStream_t s = S->streams[idx];
    std::sort(reqs.begin(), reqs.end(), [](const Req *x, const Req *y) { return x->cells > y->cells; });
    const int np = (int) reqs.size();
    // big requests of at most kTileAutoMaxRows rows comb with the register-tile kernel (few bands per request, so
    // a warp's own latency is the bound); a launch takes it only when all its requests qualify
    bool tile = np > 0;
    for (const Req *r : reqs) tile = tile && r->tileR > 0;
    std::vector<CombItem> items;
    std::vector<int> prog_off(np + 1, 0);
    std::vector<size_t> hand_off(np + 1, 0);
    for (int i = 0; i < np; ++i) {
        Req *r = reqs[i];
        int nb = 0;
        if (r->m > 0 && r->n > 0) nb = tile ? plan_tile_bands(i, r->m, r->tileR, items) : plan_bands(i, r->m, r->R, items);
        prog_off[i + 1] = prog_off[i] + nb;
        hand_off[i + 1] = hand_off[i] + (tile ? (size_t) r->n : 0);
    }
    // band-major order: a request's band k is taken once its band k-1 is under way (slots are per request)
    std::stable_sort(items.begin(), items.end(), [](const CombItem &x, const CombItem &y) { return x.band < y.band; });
    const int ni = (int) items.size();
    // meta layout
    size_t off = 0;
    const size_t o_pairs = off; off = align_up(off + sizeof(CombPair) * np, 16);
    const size_t o_items = off; off = align_up(off + sizeof(CombItem) * std::max(ni, 1), 16);
    const size_t o_sp = off;    off = align_up(off + sizeof(SrvPair) * np, 16);
    const size_t o_prog = off;  off = align_up(off + sizeof(int32_t) * std::max(prog_off[np], 1), 16);
    const size_t o_out = off;   off = align_up(off + sizeof(int32_t) * np, 16);
    const size_t o_err = off;   off += 16;   // err, next
    const size_t bytes = off;
    auto L = new Launch();
    L->s = s;
    L->hmeta = S->pinned.get(bytes, &L->hcap);
    auto fail_all = [&](int rc) {
        for (Req *r : reqs) {
            dfree(r->dab, s);
            dfree(r->dr2c, s);
            unreserve(S, r->need);
            finish_req(S, r, rc, 0, S->now());
        }
        reqs.clear();
        if (L->dmeta) dfree(L->dmeta, s);
        if (L->dhand) dfree(L->dhand, s);
        S->pinned.put(L->hmeta, L->hcap);
        if (L->done) cudaEventDestroy(L->done);
        delete L;
        return rc;
    };
    if (!L->hmeta) return fail_all(fail(SLCS_ERR_OOM, "pinned host allocation failed"));
    if (dalloc(&L->dmeta, bytes, s) != SLCS_OK) return fail_all(SLCS_ERR_OOM);
    if (tile) {
        const size_t hb = sizeof(unsigned long long) * std::max<size_t>(hand_off[np], 1);
        if (dalloc(&L->dhand, hb, s) != SLCS_OK) return fail_all(SLCS_ERR_OOM);
        if (cudaMemsetAsync(L->dhand, 0, hb, s) != cudaSuccess) return fail_all(fail(SLCS_ERR_CUDA, "memset failed"));
    }
    if (cudaEventCreateWithFlags(&L->done, cudaEventDisableTiming) != cudaSuccess)
        return fail_all(fail(SLCS_ERR_CUDA, "cudaEventCreate failed"));
    unsigned char *H = static_cast<unsigned char *>(L->hmeta);
    unsigned char *D = static_cast<unsigned char *>(L->dmeta);
    std::memset(H, 0, bytes);
    auto *hp = reinterpret_cast<CombPair *>(H + o_pairs);
    auto *hsp = reinterpret_cast<SrvPair *>(H + o_sp);
    int32_t *dprog = reinterpret_cast<int32_t *>(D + o_prog);
    const double t_admit = S->now();
    for (int i = 0; i < np; ++i) {
        Req *r = reqs[i];
        r->t_admit = t_admit;
        const size_t ab = align_up((size_t) r->m + r->n, 256);
        if (dalloc(reinterpret_cast<void **>(&r->dab), ab + sizeof(int32_t) * (size_t) (r->m + r->n) + 16, s) != SLCS_OK ||
            dalloc(reinterpret_cast<void **>(&r->dr2c), sizeof(int32_t) * (size_t) std::max(r->m + r->n, 1), s) != SLCS_OK)
            return fail_all(SLCS_ERR_OOM);
        if (r->m + r->n > 0 &&
            cudaMemcpyAsync(r->dab, r->ha, (size_t) r->m + r->n, cudaMemcpyHostToDevice, s) != cudaSuccess)
            return fail_all(fail(SLCS_ERR_CUDA, "input upload failed"));
        int32_t *c2r = reinterpret_cast<int32_t *>(r->dab + ab);
        unsigned long long *hand = tile ? static_cast<unsigned long long *>(L->dhand) + hand_off[i] : nullptr;
        hp[i] = CombPair{r->dab, r->dab + r->m, c2r, dprog + prog_off[i], nullptr, r->m, r->n, hand};
        hsp[i] = SrvPair{c2r, r->dr2c, r->m, r->n, r->q};
    }
    if (ni) std::memcpy(H + o_items, items.data(), sizeof(CombItem) * ni);
    if (cudaMemcpyAsync(D, H, o_out, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemsetAsync(D + o_out, 0, bytes - o_out, s) != cudaSuccess)
        return fail_all(fail(SLCS_ERR_CUDA, "launch metadata upload failed"));
    int *derr = reinterpret_cast<int *>(D + o_err);
    // a launch of one big request that has the device to itself combs with two dependency chains per lane
    const auto *dpairs = reinterpret_cast<const CombPair *>(D + o_pairs);
    const auto *ditems = reinterpret_cast<const CombItem *>(D + o_items);
    int rc = tile ? launch_comb_tile<uint8_t>(dpairs, ditems, ni, derr + 1, derr, std::max(1, warp_cap), kTileCols, s)
                  : (lone ? launch_comb_lone<uint8_t> : launch_comb<uint8_t>)(dpairs, ditems, ni, derr + 1, derr,
                                                                              std::max(1, warp_cap), s);
    if (rc != SLCS_OK) return fail_all(rc);
    int maxsize = 1;
    for (Req *r : reqs) maxsize = std::max(maxsize, r->m + r->n);
    const SrvPair *dsp = reinterpret_cast<const SrvPair *>(D + o_sp);
    srv_invert_kernel<<<dim3((unsigned) std::min(1024, (maxsize + 255) / 256), (unsigned) np), 256, 0, s>>>(dsp, derr);
    srv_query_kernel<<<np, 256, 0, s>>>(dsp, reinterpret_cast<int32_t *>(D + o_out), derr);
    if (cudaGetLastError() != cudaSuccess) return fail_all(fail(SLCS_ERR_CUDA, "server kernel launch failed"));
    if (cudaMemcpyAsync(H + o_out, D + o_out, bytes - o_out, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaEventRecord(L->done, s) != cudaSuccess)
        return fail_all(fail(SLCS_ERR_CUDA, "result download failed"));
    L->hout = reinterpret_cast<int32_t *>(H + o_out);
    L->herr = reinterpret_cast<int *>(H + o_err);
    L->reqs = std::move(reqs);
    S->inflight[idx] = L;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        ++S->launches;
        S->inflight_count += (int) L->reqs.size();
    }
    return SLCS_OK;
}

bool retire(slcs_server *S) {
    bool did = false;
    for (size_t idx = 0; idx < S->inflight.size(); ++idx) {
        Launch *L = S->inflight[idx];
        if (!L) continue;
        const cudaError_t e = cudaEventQuery(L->done);
        if (e == cudaErrorNotReady) continue;
        did = true;
        int st = SLCS_OK;
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = SLCS_ERR_CUDA;
        } else if (*L->herr == kDevErrTimeout) {
            st = SLCS_ERR_TIMEOUT;
        } else if (*L->herr != kDevErrNone) {
            st = SLCS_ERR_INTERNAL;
        }
        const double t = S->now();
        std::vector<Req *> again;
        for (size_t i = 0; i < L->reqs.size(); ++i) {
            Req *r = L->reqs[i];
            dfree(r->dab, L->s);
            if (st == SLCS_ERR_TIMEOUT && r->retries == 0) {
                // a bounded wait gave up (the context was held off the GPU for seconds, e.g. time-sliced with
                // another process): the launch's work is incomplete, so the request goes back to the front of
                // the queue once, with its staged inputs, and is admitted again like a new one
                dfree(r->dr2c, L->s);
                r->dab = nullptr;
                r->dr2c = nullptr;
                ++r->retries;
                unreserve(S, r->need);
                again.push_back(r);
                continue;
            }
            {
                std::lock_guard<std::mutex> lk(S->rmu);
                S->used -= r->need - r->keep;
                if (st == SLCS_OK) {
                    Resident &R = S->resident[r->ticket];
                    R = Resident{r->dr2c, r->m, r->n, r->keep, ++S->lru_clock, 0};
                    S->resident_bytes += r->keep;
                } else {
                    dfree(r->dr2c, L->s);
                    S->used -= r->keep;
                }
            }
            finish_req(S, r, st, st == SLCS_OK ? L->hout[i] : 0, t);
        }
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->inflight_count -= (int) L->reqs.size();
        }
        for (auto it = again.rbegin(); it != again.rend(); ++it) S->pending.push_front(*it);
        dfree(L->dmeta, L->s);
        if (L->dhand) dfree(L->dhand, L->s);
        S->pinned.put(L->hmeta, L->hcap);
        cudaEventDestroy(L->done);
        delete L;
        S->inflight[idx] = nullptr;
    }
    return did;
}

// Cells per second a request is assumed to comb at when the scheduler orders big requests (B200, batched rate).
constexpr double kServeCellsPerSec = 5.0e12;

bool schedule(slcs_server *S) {
    bool did = false;
    const int W = S->resident_warps;
    auto big = [&](const Req *r) { return r->cells >= S->o.big_cells; };
    // big streams: the oldest big requests that fit; when several are pending each free big stream takes its
    // share (at most 8) in one launch, whose band-major work order keeps the device busy across them
    int pending_big = 0;
    for (const Req *r : S->pending) pending_big += big(r);
    for (int idx = 0; idx < S->nbig && pending_big > 0; ++idx) {
        if (S->inflight[idx]) continue;
        int free_big = 0;
        for (int j = idx; j < S->nbig; ++j) free_big += S->inflight[j] == nullptr;
        const int share = std::min(8, std::max(1, (pending_big + free_big - 1) / free_big));
        // which big requests first: the least remaining time, i.e. the request's own combing time (at the
        // device's batched rate) minus the time it has already waited -- short requests overtake long ones, and a
        // long one that has waited as long as its own work takes goes first (so none starves)
        const double now = S->now();
        std::vector<std::pair<double, Req *>> cand;
        for (Req *r : S->pending)
            if (big(r)) cand.emplace_back((double) r->cells / kServeCellsPerSec - (now - r->t_submit), r);
        std::stable_sort(cand.begin(), cand.end(),
                         [](const std::pair<double, Req *> &x, const std::pair<double, Req *> &y) {
                             return x.first < y.first;
                         });
        std::vector<Req *> g;
        for (const auto &c : cand) {
            if ((int) g.size() >= share) break;
            if (!reserve(S, c.second->need, S->streams[idx])) break;
            g.push_back(c.second);
            S->pending.erase(std::find(S->pending.begin(), S->pending.end(), c.second));
        }
        if (g.empty()) break;
        pending_big -= (int) g.size();
        // the grid cap: half the resident warps while big launches may overlap; when this launch is the only
        // big work (one request on an otherwise idle big side, nothing big pending) three quarters of them and
        // two chains per lane, since a 1M-row request has ~1000 bands and a half grid would run its later bands
        // only after whole earlier ones.  A quarter always stays free for a small batch.
        bool alone = g.size() == 1 && pending_big == 0;
        for (int j = 0; j < S->nbig && alone; ++j) alone = j == idx || S->inflight[j] == nullptr;
        const int cap = S->o.big_warps > 0 ? S->o.big_warps : (alone ? W - W / 4 : W / 2);
        launch_group(S, idx, g, cap, alone);
        did = true;
    }
    // small streams: everything small that fits, oldest first, up to max_batch per launch
    for (size_t idx = S->nbig; idx < S->streams.size(); ++idx) {
        if (S->inflight[idx]) continue;
        std::vector<Req *> g;
        for (auto it = S->pending.begin(); it != S->pending.end() && (int) g.size() < S->o.max_batch;) {
            if (big(*it)) {
                ++it;
                continue;
            }
            if (!reserve(S, (*it)->need, S->streams[idx])) break;
            g.push_back(*it);
            it = S->pending.erase(it);
        }
        if (g.empty()) break;
        launch_group(S, (int) idx, g, S->o.small_warps > 0 ? S->o.small_warps : W / 4);
        did = true;
    }
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->pending_count = (int) S->pending.size() + (int) S->submitq.size();
    }
    return did;
}

void worker_main(slcs_server *S) {
    cudaSetDevice(S->device);
    for (;;) {
        bool did = false;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            while (!S->submitq.empty()) {
                S->pending.push_back(S->submitq.front());
                S->submitq.pop_front();
                did = true;
            }
            if (S->stop) {
                // cancel what was never admitted, finish what is on the device
                while (!S->pending.empty()) {
                    Req *r = S->pending.front();
                    S->pending.pop_front();
                    S->done.push_back(slcs_result{r->ticket, SLCS_ERR_BUSY, 0, r->m, r->n, r->q, 0, r->t_submit, 0, 0});
                    S->pinned.put(r->ha, r->hcap);
                    delete r;
                }
            }
        }
        did |= retire(S);
        bool busy = false;
        for (Launch *L : S->inflight) busy |= L != nullptr;
        if (S->stop && !busy) break;
        if (!S->stop) did |= schedule(S);
        busy = false;
        for (Launch *L : S->inflight) busy |= L != nullptr;
        if (!did) {
            if (!busy) {
                std::unique_lock<std::mutex> lk(S->mu);
                S->cv_work.wait_for(lk, std::chrono::milliseconds(2), [&] { return !S->submitq.empty() || S->stop; });
            } else {
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
        }
    }
}


}  // namespace

extern "C" {

int slcs_server_create(const slcs_server_opts *opts, slcs_server **out) {
    if (!out) return fail(SLCS_ERR_ARG, "NULL output");
    *out = nullptr;
    Engine *E;
    SLCS_TRY(engine(&E));
    auto S = new slcs_server();
    if (opts) S->o = *opts;
    if (S->o.max_pending <= 0) S->o.max_pending = 65536;
    if (S->o.small_streams <= 0) S->o.small_streams = 2;
    if (S->o.small_streams > 16) S->o.small_streams = 16;
    if (S->o.big_cells <= 0) S->o.big_cells = (int64_t) 1 << 32;
    if (S->o.max_batch <= 0) S->o.max_batch = 1024;
    S->nbig = S->o.big_streams > 0 ? std::min(S->o.big_streams, 8) : 2;
    S->device = E->device;
    S->t0 = std::chrono::steady_clock::now();
    S->resident_warps = comb_resident_warps(E);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        delete S;
        return fail(SLCS_ERR_CUDA, "cudaMemGetInfo failed");
    }
    S->budget = S->o.mem_budget > 0 ? S->o.mem_budget : (int64_t) (free_b / 2);
    S->streams.assign(S->nbig + S->o.small_streams, nullptr);
    S->inflight.assign(S->streams.size(), nullptr);
    for (auto &s : S->streams)
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
            for (auto &t : S->streams)
                if (t) cudaStreamDestroy(t);
            delete S;
            return fail(SLCS_ERR_CUDA, "cudaStreamCreate failed");
        }
    if (cudaStreamCreateWithFlags(&S->qstream, cudaStreamNonBlocking) != cudaSuccess) {
        for (auto &t : S->streams) cudaStreamDestroy(t);
        delete S;
        return fail(SLCS_ERR_CUDA, "cudaStreamCreate failed");
    }
    S->worker = std::thread(worker_main, S);
    *out = S;
    return SLCS_OK;
}

int slcs_server_submit(slcs_server *S, const uint8_t *a, int m, const uint8_t *b, int n, const slcs_query *q,
                       uint64_t *ticket) {
    if (!S || !ticket || m < 0 || n < 0 || (m > 0 && !a) || (n > 0 && !b)) return fail(SLCS_ERR_ARG, "bad request");
    if ((int64_t) m + n >= (1ll << 30) || m > (1 << 23)) return fail(SLCS_ERR_TOO_LARGE, "pair too large");
    slcs_query qq{SLCS_Q_GLOBAL, 0, 0};
    if (q) qq = *q;
    if (!query_valid(qq, m, n)) return fail(SLCS_ERR_ARG, "query out of range");
    auto r = new Req();
    r->m = m;
    r->n = n;
    r->q = qq;
    r->cells = (int64_t) m * n;
    r->R = S->o.band_rows > 0 ? std::max(1, std::min(32, S->o.band_rows / 32)) : pick_rows_batch(m);
    r->nbands = (m > 0 && n > 0) ? (m + 32 * r->R - 1) / (32 * r->R) + 1 : 0;
    if (S->o.band_rows <= 0 && m > 0 && n > 0 && r->cells >= S->o.big_cells) {
        r->tileR = tile_shape_for(m, 0, 0).R;
        if (r->tileR > 0) r->nbands = std::max(r->nbands, (m + 32 * r->tileR - 1) / (32 * r->tileR));
    }
    r->need = req_need(m, n, r->nbands) + (r->tileR > 0 ? (int64_t) sizeof(unsigned long long) * n + 256 : 0);
    r->keep = (int64_t) align_up(sizeof(int32_t) * (size_t) std::max(m + n, 1), 256);
    if (r->need > S->budget) {
        delete r;
        std::lock_guard<std::mutex> lk(S->mu);
        ++S->rejected;
        return fail(SLCS_ERR_OOM, "request exceeds the server's memory budget");
    }
    r->ha = static_cast<uint8_t *>(S->pinned.get((size_t) m + n + 1, &r->hcap));
    if (!r->ha) {
        delete r;
        return fail(SLCS_ERR_OOM, "pinned host allocation failed");
    }
    if (m) std::memcpy(r->ha, a, (size_t) m);
    if (n) std::memcpy(r->ha + m, b, (size_t) n);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stop || S->pending_count + (int64_t) S->submitq.size() >= S->o.max_pending) {
            S->pinned.put(r->ha, r->hcap);
            delete r;
            ++S->rejected;
            return fail(SLCS_ERR_BUSY, "server queue full");
        }
        r->ticket = S->next_ticket++;
        r->t_submit = S->now();
        *ticket = r->ticket;
        S->submitq.push_back(r);
        ++S->submitted;
    }
    S->cv_work.notify_one();
    return SLCS_OK;
}

int slcs_server_poll(slcs_server *S, slcs_result *out, int cap, int *count, int timeout_ms) {
    if (!S || !count || cap < 0 || (cap > 0 && !out)) return fail(SLCS_ERR_ARG, "bad poll arguments");
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->done.empty() && timeout_ms > 0)
        S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !S->done.empty(); });
    int c = 0;
    while (c < cap && !S->done.empty()) {
        out[c++] = S->done.front();
        S->done.pop_front();
    }
    *count = c;
    return SLCS_OK;
}

int slcs_server_query(slcs_server *S, uint64_t ticket, const slcs_query *q, int nq, int32_t *out) {
    if (!S || nq < 0 || (nq > 0 && (!q || !out))) return fail(SLCS_ERR_ARG, "bad query arguments");
    Resident R;
    {
        std::lock_guard<std::mutex> lk(S->rmu);
        auto it = S->resident.find(ticket);
        if (it == S->resident.end()) return fail(SLCS_ERR_ARG, "braid not resident (unknown, pending, released or evicted)");
        it->second.pins++;
        it->second.lru = ++S->lru_clock;
        R = it->second;
    }
    for (int x = 0; x < nq; ++x)
        if (!query_valid(q[x], R.m, R.n)) {
            std::lock_guard<std::mutex> lk(S->rmu);
            S->resident[ticket].pins--;
            return fail(SLCS_ERR_ARG, "query out of range");
        }
    int rc = SLCS_OK;
    {
        std::lock_guard<std::mutex> lk(S->qmu);
        rc = launch_scores_host(R.r2c, R.m, R.n, q, nq, out, S->qstream);
    }
    std::lock_guard<std::mutex> lk(S->rmu);
    S->resident[ticket].pins--;
    return rc;
}

int slcs_server_braid(slcs_server *S, uint64_t ticket, int32_t *row_to_col) {
    if (!S || !row_to_col) return fail(SLCS_ERR_ARG, "bad arguments");
    Resident R;
    {
        std::lock_guard<std::mutex> lk(S->rmu);
        auto it = S->resident.find(ticket);
        if (it == S->resident.end()) return fail(SLCS_ERR_ARG, "braid not resident (unknown, pending, released or evicted)");
        it->second.pins++;
        R = it->second;
    }
    int rc = SLCS_OK;
    {
        std::lock_guard<std::mutex> lk(S->qmu);
        if (R.m + R.n > 0 &&
            (cudaMemcpyAsync(row_to_col, R.r2c, sizeof(int32_t) * (size_t) (R.m + R.n), cudaMemcpyDeviceToHost,
                             S->qstream) != cudaSuccess ||
             cudaStreamSynchronize(S->qstream) != cudaSuccess))
            rc = fail(SLCS_ERR_CUDA, "braid download failed");
    }
    std::lock_guard<std::mutex> lk(S->rmu);
    S->resident[ticket].pins--;
    return rc;
}

int slcs_server_window(slcs_server *S, uint64_t ticket, int w, int32_t *out) {
    if (!S || !out) return fail(SLCS_ERR_ARG, "bad arguments");
    Resident R;
    {
        std::lock_guard<std::mutex> lk(S->rmu);
        auto it = S->resident.find(ticket);
        if (it == S->resident.end()) return fail(SLCS_ERR_ARG, "braid not resident (unknown, pending, released or evicted)");
        it->second.pins++;
        it->second.lru = ++S->lru_clock;
        R = it->second;
    }
    int rc = SLCS_OK;
    if (w < 1 || w > R.n) rc = fail(SLCS_ERR_ARG, "window length must be in [1, n]");
    if (rc == SLCS_OK) {
        std::lock_guard<std::mutex> lk(S->qmu);
        DevBuf<int32_t> dout;
        rc = dout.alloc(R.n - w + 1, S->qstream);
        if (rc == SLCS_OK) rc = window_scores_dev(R.r2c, nullptr, R.m, R.n, w, dout.p, S->qstream);
        if (rc == SLCS_OK &&
            (cudaMemcpyAsync(out, dout.p, sizeof(int32_t) * (size_t) (R.n - w + 1), cudaMemcpyDeviceToHost,
                             S->qstream) != cudaSuccess ||
             cudaStreamSynchronize(S->qstream) != cudaSuccess))
            rc = fail(SLCS_ERR_CUDA, "window download failed");
    }
    std::lock_guard<std::mutex> lk(S->rmu);
    S->resident[ticket].pins--;
    return rc;
}

int slcs_server_release(slcs_server *S, uint64_t ticket) {
    if (!S) return fail(SLCS_ERR_ARG, "NULL server");
    std::lock_guard<std::mutex> lk(S->rmu);
    auto it = S->resident.find(ticket);
    if (it == S->resident.end()) return fail(SLCS_ERR_ARG, "braid not resident");
    if (it->second.pins) return fail(SLCS_ERR_BUSY, "braid in use");
    dfree(it->second.r2c, S->qstream);
    S->used -= it->second.bytes;
    S->resident_bytes -= it->second.bytes;
    S->resident.erase(it);
    return SLCS_OK;
}

int slcs_server_stats_get(slcs_server *S, slcs_server_stats *st) {
    if (!S || !st) return fail(SLCS_ERR_ARG, "bad arguments");
    slcs_server_stats x{};
    {
        std::lock_guard<std::mutex> lk(S->mu);
        x.submitted = S->submitted;
        x.completed = S->completed;
        x.rejected = S->rejected;
        x.launches = S->launches;
        x.cells = S->cells;
        x.pending = S->pending_count;
        x.inflight = S->inflight_count;
    }
    {
        std::lock_guard<std::mutex> lk(S->rmu);
        x.evicted = S->evicted;
        x.resident = (int64_t) S->resident.size();
        x.resident_bytes = S->resident_bytes;
        x.used_bytes = S->used;
        x.peak_bytes = S->peak;
        x.budget = S->budget;
    }
    *st = x;
    return SLCS_OK;
}

double slcs_server_now(slcs_server *S) { return S ? S->now() : 0.0; }

int slcs_server_destroy(slcs_server *S) {
    if (!S) return SLCS_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    if (S->worker.joinable()) S->worker.join();
    cudaSetDevice(S->device);
    for (auto &kv : S->resident) dfree(kv.second.r2c, S->qstream);
    S->resident.clear();
    for (auto s : S->streams) cudaStreamSynchronize(s);
    cudaStreamSynchronize(S->qstream);
    for (auto s : S->streams) cudaStreamDestroy(s);
    cudaStreamDestroy(S->qstream);
    delete S;
    return SLCS_OK;
}

}  // extern "C"
