// hyyro.cu -- bit-vector LLCS (Allison-Dix / Hyyro recurrence) on sm_100a.
//
// The reference carries it beside its bit-parallel combing (R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:
// 743-914, lllcs_hyyro::hyyro_magic and the anti-diagonal OpenMP form hyyro_magic_mpi_with_precalc): a bit vector V
// over the rows (one string), all ones at first, takes every column symbol c of the other string in turn:
//     U = V & match(c);   V' = (V + U) | (V & ~match(c))
// where the addition runs over the whole vector, carries moving from row 0 upwards; LLCS = number of zero bits of
// the final V over the real rows.  (The reference counts zero bits over whole words: its padding bits never match
// and stay ones.  Here padding rows hold symbol 0 and may change, above every real row, and are masked out.)
//
// Layout: a warp is a band of 32 words (1024 rows), lane l owning word 32 band + l (its two symbol bit planes and its
// V in registers).  The warp is a 32-stage systolic array over the carries: at step s lane l adds column group
// s - l (C columns), taking each column's carry-in from lane l - 1, which produced it one step earlier, by one
// shuffle per column; lane 0 takes it from the band below (rows below = lower words) and lane 31's carry-outs go
// to the band above.  The 32-bit adder propagates a carry through a whole word in one instruction, so a band is
// 32 steps deep for its 1024 rows, and each column costs a lane about ten instructions for 32 cells.
//   * column symbols: a ring of 256 columns in shared memory holding, per column, the two symbol planes as all-ones
//     or zero masks and a "real column" mask (0 for padding columns beyond n, whose cells then change nothing:
//     U = 0 and no carry); one column per lane per sub-chunk of 32 columns, loaded a sub-chunk ahead;
//   * bands: carry bits of 32 columns travel in one 64-bit word together with the writing band's tag (band + 1),
//     polled (bounded) only while the tag is not there yet, requested two sub-chunks ahead; persistent warps
//     dequeue bands in order, so a band only waits for a band a running warp owns.
#include <algorithm>

#include "slcs_internal.cuh"

namespace slcs {
namespace {

constexpr int kHyC = 4;                 // columns a lane adds per step
constexpr int kHyK = 32 / kHyC;         // steps per sub-chunk of 32 columns
constexpr int kHyRing = 256;            // column ring (covers 31 kHyC + 64 columns)

struct HyPair {
    const uint32_t *a0, *a1;            // row planes: word w = rows [32 w, 32 w + 32), bit i = row 32 w + i
    const uint8_t *b;                   // column symbols (< 4)
    unsigned long long *hand;           // carry words between bands: word q = columns [32 q, 32 q + 32) in the low
                                        // half, (index of the writing band) + 1 in the high half
    int32_t *ones;                      // out: ones of the final vectors over the real rows
    int m, n, words;
};

struct HyShared {
    int s0[kHyRing], s1[kHyRing], real[kHyRing];
};

__device__ __forceinline__ void lds4(const int *p, int (&o)[4]) {
    const int4 v = *reinterpret_cast<const int4 *>(p);
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
}

__device__ __forceinline__ void hyyro_band(const HyPair &P, int band, bool last_band, int *err, int lane,
                                           HyShared &S) {
    constexpr int C = kHyC, K = kHyK;
    const int n = P.n;
    const int w = band * 32 + lane;
    const uint32_t a0 = w < P.words ? P.a0[w] : 0u;
    const uint32_t a1 = w < P.words ? P.a1[w] : 0u;
    uint32_t V = ~0u;
    const int G = (n + C - 1) / C;            // column groups; lane l adds group s - l at step s
    const int nsub = (G + 31 + K - 1) / K;    // sub-chunks of steps
    const int Q = (n + 31) >> 5;              // carry words
    const bool has_below = band > 0;
    const unsigned tag_below = (unsigned) band;
    const unsigned long long my_tag = (unsigned long long) (band + 1) << 32;

    __syncwarp();   // the previous band's last reads of S are done
    for (int i = lane; i < kHyRing; i += 32) {
        S.s0[i] = 0;
        S.s1[i] = 0;
        S.real[i] = 0;
    }
    // The carry word and the column symbols of sub-chunk j are requested two sub-chunks ahead, into one of two
    // registers each that the sub-chunk loop, unrolled by two, names statically: a register is never read while
    // its load is in flight (a load of a word another SM wrote outlasts a sub-chunk of steps; measured: with one
    // register, read by a shuffle every sub-chunk, a band below another ran at 105 ns per step instead of 65).
    unsigned long long pwA = (has_below && 0 < Q) ? ld_relaxed64(P.hand) : 0ull;
    unsigned long long pwB = (has_below && 1 < Q) ? ld_relaxed64(P.hand + 1) : 0ull;
    int pbA = lane < n ? (int) P.b[lane] : 0;
    int pbB = 32 + lane < n ? (int) P.b[32 + lane] : 0;
    // carry-ins from the lane below for the next step: each column's carry-out is shuffled up as soon as it is
    // computed, so the shuffle's latency overlaps the lane's later columns instead of opening the next step
    int cup[C];
#pragma unroll
    for (int c = 0; c < C; ++c) cup[c] = 0;
    // lane 31's carry-outs: at step k of sub-chunk j, column (j K + k - 31) C + c is bit (k C + c + C) mod 32 of word
    // j - C + (k C + c + C) / 32.  Steps k < K - 1 finish word j - C (collected in wdone), the last step starts word
    // j - C + 1 (wnext); the finished word is published after the step loop, outside the unrolled steps (a branch
    // among them would cut them into separately scheduled blocks: measured 75 against 45 ns per step)
    uint32_t wdone = 0, wnext = 0;
    int qpub = 0;        // next carry word to publish

    // one sub-chunk of steps; false: a wait gave up (the error word is set)
    auto sub = [&](int j, unsigned long long &pw, int &pb) -> bool {
        // carry-ins of columns [32 j, 32 j + 32) from the band below, one word for all lanes
        uint32_t win = 0;
        if (has_below && j < Q) {
            unsigned long long v = pw;
            const bool ok = wait_tag(P.hand + j, v, tag_below, err);
            if (!__all_sync(kFull, ok)) return false;
            win = (uint32_t) v;
            if (j + 2 < Q) pw = ld_relaxed64(P.hand + j + 2);
        }
        const int col = (j << 5) + lane;
        if (pb > 3) raise_error(err, kDevErrBadState);
        S.s0[col & (kHyRing - 1)] = -(pb & 1);
        S.s1[col & (kHyRing - 1)] = -((pb >> 1) & 1);
        S.real[col & (kHyRing - 1)] = col < n ? -1 : 0;
        pb = col + 64 < n ? (int) P.b[col + 64] : 0;
        __syncwarp();
        const int base = (j * K - lane) * C;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            int s0[C], s1[C], re[C];
            const int idx = (base + k * C) & (kHyRing - 1);
            lds4(S.s0 + idx, s0);
            lds4(S.s1 + idx, s1);
            lds4(S.real + idx, re);
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const int cin = lane == 0 ? (int) ((win >> (k * C + c)) & 1u) : cup[c];
                const uint32_t M = (a0 ^ (uint32_t) s0[c]) | (a1 ^ (uint32_t) s1[c]);   // rows not matching
                const uint32_t U = V & ~M & (uint32_t) re[c];
                const unsigned long long sum = (unsigned long long) V + U + (unsigned) cin;
                V = (uint32_t) sum | (V & M);
                const int cout = (int) (sum >> 32);
                cup[c] = __shfl_up_sync(kFull, cout, 1);
                if (k * C + c + C < 32) wdone |= (uint32_t) cout << (k * C + c + C);
                else wnext |= (uint32_t) cout << (k * C + c + C - 32);
            }
        }
        // word j - C (columns [32 q, 32 q + 32)) is complete: its last column left lane 31 at step K - 2
        {
            const int q = j - C;
            if (q >= 0 && q < Q) {
                if (!last_band && lane == 31) st_relaxed64(P.hand + q, my_tag | wdone);
                qpub = q + 1;
            }
            wdone = wnext;
            wnext = 0;
        }
        __syncwarp();
        return true;
    };
    for (int j = 0; j < nsub; j += 2) {
        if (!sub(j, pwA, pbA)) return;
        if (j + 1 < nsub && !sub(j + 1, pwB, pbB)) return;
    }
    // a last word whose groups ended before its regular publication
    if (!last_band && lane == 31)
        for (int q = qpub; q < Q; ++q) st_relaxed64(P.hand + q, my_tag | (q == qpub ? wdone : 0u));
    // ones over the real rows
    const int r0 = 32 * w;
    uint32_t real_rows = 0u;
    if (r0 < P.m) real_rows = P.m - r0 >= 32 ? ~0u : ((1u << (P.m - r0)) - 1u);
    const int cnt = __reduce_add_sync(kFull, __popc(V & real_rows));
    if (lane == 0 && cnt) atomicAdd(P.ones, cnt);
}

__global__ void __launch_bounds__(32) hyyro_kernel(const HyPair *__restrict__ pp, int bands, int *next, int *err) {
    __shared__ __align__(16) HyShared S;
    const int lane = threadIdx.x & 31;
    const HyPair P = *pp;
    for (;;) {
        int it = bands;
        if (lane == 0 && ld_relaxed(err) == kDevErrNone) it = atomicAdd(next, 1);
        it = __shfl_sync(kFull, it, 0);
        if (it >= bands) return;
        hyyro_band(P, it, it == bands - 1, err, lane, S);
    }
}

// row planes: one warp per word
__global__ void hyyro_pack_kernel(const uint8_t *__restrict__ a, int m, int words, uint32_t *a0, uint32_t *a1,
                                  int *err) {
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int w = wid; w < words; w += nwarps) {
        const int row = 32 * w + lane;
        const int sym = row < m ? a[row] : 0;
        if (sym > 3) raise_error(err, kDevErrBadState);
        const unsigned h = __ballot_sync(kFull, (sym >> 1) & 1), l = __ballot_sync(kFull, sym & 1);
        if (lane == 0) {
            a1[w] = h;
            a0[w] = l;
        }
    }
}

__global__ void hyyro_score_kernel(const int32_t *ones, int m, int32_t *score) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *score = m - *ones;
}

}  // namespace

struct HyyroPlan {
    int m = 0, n = 0, words = 0, bands = 0, warps = 0, Q = 0;
    bool swap = false;   // rows are the second string (the longer one)
    uint32_t *a0 = nullptr, *a1 = nullptr;
    unsigned long long *hand = nullptr;
    int32_t *ones = nullptr;
    int *next = nullptr;
    HyPair *dp = nullptr;
    const uint8_t *ba = nullptr, *bb = nullptr;   // string pointers the descriptor holds
    cudaStream_t s = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

void hyyro_plan_destroy(HyyroPlan *H) {
    if (!H) return;
    void *ps[] = {H->a0, H->a1, H->hand, H->ones, H->next, H->dp};
    for (void *p : ps) dfree(p, H->s);
    if (H->ev0) cudaEventDestroy(H->ev0);
    if (H->ev1) cudaEventDestroy(H->ev1);
    delete H;
}

int hyyro_plan_create(Engine *E, int m, int n, cudaStream_t s, HyyroPlan **out) {
    *out = nullptr;
    auto H = new HyyroPlan();
    // rows = the longer string: the run is about (columns / kHyC + 47 per band) steps
    H->swap = n > m;
    H->m = H->swap ? n : m;
    H->n = H->swap ? m : n;
    H->s = s;
    H->words = (H->m + 31) / 32;
    H->bands = std::max(1, (H->words + 31) / 32);
    H->Q = (H->n + 31) / 32;
    auto bail = [&](int rc) {
        hyyro_plan_destroy(H);
        return rc;
    };
    int rc;
#define HY_ALLOC(ptr, cnt) \
    if ((rc = dalloc(reinterpret_cast<void **>(&H->ptr), sizeof(*H->ptr) * std::max<int64_t>((cnt), 1), s))) return bail(rc);
    HY_ALLOC(a0, H->words);
    HY_ALLOC(a1, H->words);
    HY_ALLOC(hand, H->Q);
    HY_ALLOC(ones, 1);
    HY_ALLOC(next, 1);
    HY_ALLOC(dp, 1);
#undef HY_ALLOC
    if (cudaEventCreate(&H->ev0) != cudaSuccess || cudaEventCreate(&H->ev1) != cudaSuccess)
        return bail(fail(SLCS_ERR_CUDA, "hyyro plan setup failed"));
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hyyro_kernel, 32, 0) != cudaSuccess)
        return bail(fail(SLCS_ERR_CUDA, "occupancy query failed"));
    H->warps = std::min(H->bands, std::max(1, per_sm) * E->num_sms);
    *out = H;
    return SLCS_OK;
}

// Kernels only (capturable once the plan has run on these string pointers): pack the rows, run the bands, write
// the score (device int32).
int hyyro_plan_run(HyyroPlan *H, const uint8_t *d_a, const uint8_t *d_b, int32_t *d_score, int *d_err,
                   cudaStream_t s, bool capturing) {
    if (H->m == 0 || H->n == 0) {
        SLCS_CUDA_TRY(cudaMemsetAsync(d_score, 0, sizeof(int32_t), s));
        return SLCS_OK;
    }
    const uint8_t *rows = H->swap ? d_b : d_a;
    const uint8_t *cols = H->swap ? d_a : d_b;
    if (H->ba != rows || H->bb != cols) {
        if (capturing) return fail(SLCS_ERR_ARG, "plan must run once on these buffers before capture");
        HyPair hp{H->a0, H->a1, cols, H->hand, H->ones, H->m, H->n, H->words};
        SLCS_CUDA_TRY(cudaMemcpyAsync(H->dp, &hp, sizeof(hp), cudaMemcpyHostToDevice, s));
        SLCS_CUDA_TRY(cudaStreamSynchronize(s));
        H->ba = rows;
        H->bb = cols;
    }
    SLCS_CUDA_TRY(cudaMemsetAsync(H->ones, 0, sizeof(int32_t), s));
    SLCS_CUDA_TRY(cudaMemsetAsync(H->next, 0, sizeof(int), s));
    SLCS_CUDA_TRY(cudaMemsetAsync(H->hand, 0, sizeof(unsigned long long) * std::max(H->Q, 1), s));
    hyyro_pack_kernel<<<std::min(4096, (H->words + 7) / 8), 256, 0, s>>>(rows, H->m, H->words, H->a0, H->a1, d_err);
    const unsigned fl = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    SLCS_CUDA_TRY(cudaEventRecordWithFlags(H->ev0, s, fl));
    hyyro_kernel<<<H->warps, 32, 0, s>>>(H->dp, H->bands, H->next, d_err);
    SLCS_CUDA_TRY(cudaEventRecordWithFlags(H->ev1, s, fl));
    hyyro_score_kernel<<<1, 32, 0, s>>>(H->ones, H->m, d_score);
    SLCS_CUDA_TRY(cudaGetLastError());
    return SLCS_OK;
}

int hyyro_plan_kernel_ms(HyyroPlan *H, float *ms) {
    SLCS_CUDA_TRY(cudaEventSynchronize(H->ev1));
    SLCS_CUDA_TRY(cudaEventElapsedTime(ms, H->ev0, H->ev1));
    return SLCS_OK;
}

int hyyro_dev(Engine *E, const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_score, cudaStream_t s) {
    HyyroPlan *H = nullptr;
    SLCS_TRY(hyyro_plan_create(E, m, n, s, &H));
    DevBuf<int> err;
    int rc = err.alloc(1, s);
    if (rc == SLCS_OK && cudaMemsetAsync(err.p, 0, sizeof(int), s) != cudaSuccess) rc = fail(SLCS_ERR_CUDA, "memset");
    if (rc == SLCS_OK) rc = hyyro_plan_run(H, d_a, d_b, d_score, err.p, s, false);
    if (rc == SLCS_OK) rc = check_dev_err(err.p, s);
    hyyro_plan_destroy(H);
    return rc;
}

}  // namespace slcs

using namespace slcs;

extern "C" {

int slcs_hyyro_llcs_u8_dev(const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_score, void *stream) {
    if (m < 0 || n < 0) return fail(SLCS_ERR_ARG, "negative length");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    if ((m > 0 && !d_a) || (n > 0 && !d_b) || !d_score) return fail(SLCS_ERR_ARG, "NULL buffer");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    return hyyro_dev(E, d_a, m, d_b, n, d_score, s);
}

int slcs_hyyro_llcs_u8(const uint8_t *a, int m, const uint8_t *b, int n, int32_t *score) {
    if (m < 0 || n < 0) return fail(SLCS_ERR_ARG, "negative length");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    if ((m > 0 && !a) || (n > 0 && !b) || !score) return fail(SLCS_ERR_ARG, "NULL buffer");
    for (int i = 0; i < m; ++i)
        if (a[i] > 3) return fail(SLCS_ERR_ARG, "the bit-vector LLCS needs symbols < 4");
    for (int i = 0; i < n; ++i)
        if (b[i] > 3) return fail(SLCS_ERR_ARG, "the bit-vector LLCS needs symbols < 4");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = E->stream;
    DevBuf<uint8_t> da, db;
    DevBuf<int32_t> ds;
    SLCS_TRY(da.alloc(m, s));
    SLCS_TRY(db.alloc(n, s));
    SLCS_TRY(ds.alloc(1, s));
    if (m) SLCS_CUDA_TRY(cudaMemcpyAsync(da.p, a, m, cudaMemcpyHostToDevice, s));
    if (n) SLCS_CUDA_TRY(cudaMemcpyAsync(db.p, b, n, cudaMemcpyHostToDevice, s));
    SLCS_TRY(hyyro_dev(E, da.p, m, db.p, n, ds.p, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(score, ds.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SLCS_CUDA_TRY(cudaStreamSynchronize(s));
    return SLCS_OK;
}

}  // extern "C"
