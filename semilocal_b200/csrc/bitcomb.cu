// bitcomb.cu -- bit-parallel sticky-braid combing (LLCS only) on sm_100a.
//
// The reference's bit-parallel combing (R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:329-411,
// 668-736) keeps one bit per strand: left strands are 1, top strands 0, and a cell swaps its two strands when
// the symbols match or a top strand sits in the left slot (the integer rule "swap iff match or left > top",
// R:include/SemiLocal/SemiLocalLCS.h:158, restricted to the two strand classes).  In bits:
//     new_top  = left & (top | match)          new_left = top | (left & ~match)
// and LLCS = m - popcount(final left strands).
//
// Layout here: a lane owns strips of 32 rows; a strip's 32 left strands, a-symbol bit planes and the 32 top
// strands in flight are one 32-bit word each (bit i = row i).  Row i of a strip works on column s - i at
// step s, so the 32 cells of a step lie on an anti-diagonal and are independent.  Per step and strip:
//   * T is shifted down one row, the new row-0 strand entering from the strip above (1 funnel shift);
//   * the b-planes are read as windows "bit i = plane[s - i]" of MSB-first column words (3 funnel shifts:
//     two symbol bit planes and an "outside the string" plane that turns padding columns into non-matches);
//   * match and update are 4 three-input logic ops.
// About 8 instructions per 32 cells.  A lane's strips follow each other one 32-step block apart and update
// independently; lanes are (strips per lane + 1) blocks apart and pass one word per block by shuffle; warps
// (bands of 32 x RS strips) are chained through an array of hand-off words, each stored together with the tag of
// the band that wrote it in one 64-bit word: the band below polls the words it needs until they carry the tag of
// the band above, so no release fence or progress counter sits between them.
#include <algorithm>
#include <cstdlib>

#include "slcs_internal.cuh"

namespace slcs {
namespace {

struct BitPair {
    const uint32_t *a1, *a0;        // row planes, word w = rows [32 w, 32 w + 32), bit i = row 32 w + i
    const uint32_t *b1, *b0, *b2;   // column planes, index q + 2 = columns [32 q, 32 q + 32), MSB first;
                                    // b2 = 1 outside [0, n); indices 0, 1 are leading pad words
    unsigned long long *hand;       // hand-off words between bands: word q = columns [32 q, 32 q + 32) in the low
                                    // half, (index of the band that wrote it) + 1 in the high half
    int32_t *ones;                  // out: popcount of the final left strands over real rows
    int m, n, nstrips, nblocks;
};

struct BitItem {
    int pair, band, s0, last;
};

constexpr int kChunk = 8;   // hand-off words a band requests together (one chunk ahead of their use)

// One band (warp).  Lane k owns strips s0 + k RS + r, r = 0..RS-1.  The strips of a lane form one systolic
// chain: strip r works one 32-step block behind strip r-1 and takes its input bit, each step, straight from
// strip r-1's bottom row (so the RS strips of a lane update independently every step); lanes are RS+1 blocks
// apart and hand one 32-bit word per block to the next lane by shuffle.  Strips outside their real blocks keep
// running on padding columns, whose "outside" plane forces non-matches, so the loop has no per-strip branches.
constexpr int kRing = 256;   // column-plane words a warp keeps in shared memory (a ring, index & 255)

template <int RS>
__device__ __forceinline__ void bit_band(const BitPair &P, const BitItem &I, int *err, int lane,
                                         uint32_t (*ring)[kRing]) {
    uint32_t A1[RS], A0[RS], L[RS], T[RS], V[RS];
    bool live[RS];
#pragma unroll
    for (int r = 0; r < RS; ++r) {
        const int s = I.s0 + lane * RS + r;
        live[r] = s < P.nstrips;
        A1[r] = live[r] ? P.a1[s] : 0u;
        A0[r] = live[r] ? P.a0[s] : 0u;
        const int rows = live[r] ? min(32, P.m - 32 * s) : 0;
        V[r] = rows >= 32 ? 0xffffffffu : ((1u << rows) - 1u);
        L[r] = 0xffffffffu;
        T[r] = 0u;
    }
    const int nb = P.nblocks;
    const int lag = lane * (RS + 1);
    const int gmax = 31 * (RS + 1) + RS - 1 + nb;
    uint32_t carry = 0u;    // input word of strip 0, from the lane above (previous iteration)
    uint32_t chunkw = 0u;   // lanes 0..kChunk-1: the current chunk of hand-off words from the band above
    unsigned long long nextw = 0ull;   // lanes 0..kChunk-1: the next chunk, requested one chunk ahead
    const unsigned tag_above = (unsigned) I.band;   // tag of the band above: its index + 1
    // Column-plane words (index 0 .. nb + 2) reach the lanes through a ring in shared memory: the warp loads
    // 32 words per plane every 32 iterations, 64 words ahead, and stores them one iteration later, so no load
    // latency sits on the loop.  At iteration g the lanes read words >= g - 31 (RS + 1) - RS + 1 and <= g + 3;
    // the ring then holds words [g - 161, g + 94] (RS <= 4), so nothing live is overwritten.
    const int last = nb + 2;
    __syncwarp();
    for (int idx = lane; idx < 64; idx += 32)
        if (idx <= last) {
            ring[0][idx & (kRing - 1)] = __ldg(P.b1 + idx);
            ring[1][idx & (kRing - 1)] = __ldg(P.b0 + idx);
            ring[2][idx & (kRing - 1)] = __ldg(P.b2 + idx);
        }
    __syncwarp();
    uint32_t s1 = 0u, s0 = 0u, s2 = 0u;   // words loaded at g % 32 == 0, stored at g % 32 == 1
    uint32_t p1[RS], pl1[RS], p0[RS], pl0[RS], p2[RS], pl2[RS];   // plane words of the next iteration
#pragma unroll
    for (int r = 0; r < RS; ++r) {
        const int q = min(max(-lag - r, -1), nb);
        p1[r] = ring[0][(q + 1) & (kRing - 1)];
        pl1[r] = ring[0][(q + 2) & (kRing - 1)];
        p0[r] = ring[1][(q + 1) & (kRing - 1)];
        pl0[r] = ring[1][(q + 2) & (kRing - 1)];
        p2[r] = ring[2][(q + 1) & (kRing - 1)];
        pl2[r] = ring[2][(q + 2) & (kRing - 1)];
    }
    for (int g = 0; g < gmax; ++g) {
        if ((g & 31) == 1) {
            const int idx = g - 1 + 64 + lane;
            if (idx <= last) {
                ring[0][idx & (kRing - 1)] = s1;
                ring[1][idx & (kRing - 1)] = s0;
                ring[2][idx & (kRing - 1)] = s2;
            }
            __syncwarp();
        } else if ((g & 31) == 0) {
            const int idx = g + 64 + lane;
            if (idx <= last) {
                s1 = __ldg(P.b1 + idx);
                s0 = __ldg(P.b0 + idx);
                s2 = __ldg(P.b2 + idx);
            }
        }
        // lane 0's input word: from the band above (zero strands for the first band).  Lanes 0..kChunk-1 read one
        // word each of the next chunk a chunk ahead; at the chunk's start each waits until its word carries the
        // band above's tag, and the words reach lane 0 by shuffle, one per iteration.
        // The band above writes words 0 .. nb - 2 (block nb - 1 lies wholly past the string's end and leaves its
        // last strip after the band's final iteration): the last word is taken as zero strands, unwaited.
        if (I.band > 0 && g < nb && (g % kChunk) == 0) {
            const bool mine = lane < kChunk && g + lane < nb - 1;
            if (g == 0 && mine) nextw = ld_relaxed64(P.hand + lane);
            unsigned long long v = nextw;
            const bool ok = !mine || wait_tag(P.hand + g + lane, v, tag_above, err);
            if (!__all_sync(kFull, ok)) return;   // a bounded wait gave up (error word set)
            chunkw = mine ? (uint32_t) v : 0u;
            nextw = (lane < kChunk && g + kChunk + lane < nb - 1) ? ld_relaxed64(P.hand + g + kChunk + lane) : 0ull;
        }
        const uint32_t hw = __shfl_sync(kFull, chunkw, g % kChunk);
        uint32_t io = lane == 0 ? ((I.band > 0 && g < nb) ? hw : 0u) : carry;
        // column-plane words of every strip's block (loaded one iteration ahead; q clamped to [-1, nb]:
        // words q - 1 and q sit at indices q + 1, q + 2 in [0, nb + 2])
        uint32_t h1[RS], l1[RS], h0[RS], l0[RS], h2[RS], l2[RS];
#pragma unroll
        for (int r = 0; r < RS; ++r) {
            h1[r] = p1[r]; l1[r] = pl1[r]; h0[r] = p0[r]; l0[r] = pl0[r]; h2[r] = p2[r]; l2[r] = pl2[r];
            const int q = min(max(g + 1 - lag - r, -1), nb);
            p1[r] = ring[0][(q + 1) & (kRing - 1)];
            pl1[r] = ring[0][(q + 2) & (kRing - 1)];
            p0[r] = ring[1][(q + 1) & (kRing - 1)];
            pl0[r] = ring[1][(q + 2) & (kRing - 1)];
            p2[r] = ring[2][(q + 1) & (kRing - 1)];
            pl2[r] = ring[2][(q + 2) & (kRing - 1)];
        }
        uint32_t out = 0u;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            // rotate every strip's top strands down one row; the new row-0 bit comes from the strip above
            // (strip 0: the lane's input word), the bottom row of the last strip leaves into `out`
            uint32_t nt[RS];
            out = __funnelshift_l(T[RS - 1], out, 1);
#pragma unroll
            for (int r = RS - 1; r >= 1; --r) nt[r] = __funnelshift_l(T[r - 1], T[r], 1);
            nt[0] = __funnelshift_l(io, T[0], 1);
            io <<= 1;
#pragma unroll
            for (int r = 0; r < RS; ++r) {
                const uint32_t w1 = __funnelshift_r(l1[r], h1[r], 31 - j);
                const uint32_t w0 = __funnelshift_r(l0[r], h0[r], 31 - j);
                const uint32_t w2 = __funnelshift_r(l2[r], h2[r], 31 - j);
                const uint32_t y = (A1[r] ^ w1) | w2;
                const uint32_t mt = ~(y | (A0[r] ^ w0));
                const uint32_t l = L[r];
                T[r] = l & (nt[r] | mt);
                L[r] = nt[r] | (l & ~mt);
            }
        }
        // `out` holds the last strip's bottom-row outputs of its block g - lag - (RS - 1) minus one
        const int w = g - lag - RS;
        if (lane == 31 && !I.last && w >= 0 && w < nb)
            st_relaxed64(P.hand + w, ((unsigned long long) (I.band + 1) << 32) | out);
        carry = __shfl_up_sync(kFull, out, 1);
    }
    int ones = 0;
#pragma unroll
    for (int r = 0; r < RS; ++r)
        if (live[r]) ones += __popc(L[r] & V[r]);
    ones = __reduce_add_sync(kFull, ones);
    if (lane == 0 && ones) atomicAdd(P.ones, ones);
}

template <int RS>
__global__ void __launch_bounds__(32) bit_kernel(const BitPair *__restrict__ pairs, const BitItem *__restrict__ items,
                                                  int nitems, int *next, int *err) {
    const int lane = threadIdx.x & 31;
    __shared__ uint32_t ring[3][kRing];
    for (;;) {
        int it = nitems;
        if (lane == 0 && ld_relaxed(err) == kDevErrNone) it = atomicAdd(next, 1);
        it = __shfl_sync(kFull, it, 0);
        if (it >= nitems) return;
        const BitItem I = items[it];
        const BitPair P = pairs[I.pair];   // by value: no field reloads after the loop's global stores
        bit_band<RS>(P, I, err, lane, ring);
    }
}

// a -> row planes (LSB first per strip); b -> MSB-first column planes with two leading pad words.
__global__ void bit_pack_kernel(const uint8_t *__restrict__ a, int m, const uint8_t *__restrict__ b, int n,
                                int nstrips, int nbw, uint32_t *a1, uint32_t *a0, uint32_t *b1, uint32_t *b0,
                                uint32_t *b2, int *err) {
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int w = wid; w < nstrips + nbw; w += nwarps) {
        if (w < nstrips) {
            const int row = 32 * w + lane;
            const int sym = row < m ? a[row] : 0;
            if (sym > 3) raise_error(err, kDevErrBadState);
            const unsigned h = __ballot_sync(kFull, (sym >> 1) & 1), l = __ballot_sync(kFull, sym & 1);
            if (lane == 0) {
                a1[w] = h;
                a0[w] = l;
            }
        } else {
            const int q = w - nstrips - 2;   // word index q + 2 = w - nstrips
            const int col = 32 * q + lane;
            const bool in = q >= 0 && col < n;
            const int sym = in ? b[col] : 0;
            if (sym > 3) raise_error(err, kDevErrBadState);
            const unsigned h = __brev(__ballot_sync(kFull, (sym >> 1) & 1));
            const unsigned l = __brev(__ballot_sync(kFull, sym & 1));
            const unsigned o = __brev(__ballot_sync(kFull, !in));
            if (lane == 0) {
                b1[w - nstrips] = h;
                b0[w - nstrips] = l;
                b2[w - nstrips] = o;
            }
        }
    }
}

int strips_per_lane(int nstrips) {
    // tuning override (1, 2 or 4 strips of 32 rows per lane), e.g. for the autotuner
    if (const char *env = getenv("SLCS_BIT_STRIPS_PER_LANE")) {
        const int v = atoi(env);
        if (v == 1 || v == 2 || v == 4) return v;
    }
    // more strips per lane = fewer bands and more independent work per warp, but a longer fill; one pair has
    // only ~n / (32 * skew) strips in flight, so small pairs keep one strip per lane (measured on B200: a
    // 2^20-row pair runs 7% faster with two, a 2^18-row pair is faster with one)
    if (nstrips >= 32 * 1024) return 2;
    return 1;
}

__global__ void bit_score_kernel(const int32_t *ones, int m, int32_t *score) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *score = m - *ones;
}

}  // namespace

struct BitPlan {
    int m = 0, n = 0, nstrips = 0, nblocks = 0, nbw = 0, RS = 1, bands = 0, warps = 0;
    uint32_t *a1 = nullptr, *a0 = nullptr, *b1 = nullptr, *b0 = nullptr, *b2 = nullptr;
    unsigned long long *hand = nullptr;
    int32_t *ones = nullptr;
    int *next = nullptr;
    BitPair *dp = nullptr;
    BitItem *di = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

void bit_plan_destroy(BitPlan *B) {
    if (!B) return;
    void *ps[] = {B->a1, B->a0, B->b1, B->b0, B->b2, B->hand, B->ones, B->next, B->dp, B->di};
    for (void *p : ps) dfree(p, B->s);
    if (B->ev0) cudaEventDestroy(B->ev0);
    if (B->ev1) cudaEventDestroy(B->ev1);
    delete B;
}

int bit_plan_create(Engine *E, int m, int n, cudaStream_t s, BitPlan **out) {
    *out = nullptr;
    auto B = new BitPlan();
    B->m = m;
    B->n = n;
    B->s = s;
    B->nstrips = (m + 31) / 32;
    B->nblocks = (n + 63) / 32;
    B->nbw = B->nblocks + 3;   // two leading pads, nblocks words, one trailing pad
    B->RS = strips_per_lane(B->nstrips);
    const int per_band = 32 * B->RS;
    B->bands = std::max(1, (B->nstrips + per_band - 1) / per_band);
    auto bail = [&](int rc) {
        bit_plan_destroy(B);
        return rc;
    };
    int rc;
#define BP_ALLOC(ptr, cnt) \
    if ((rc = dalloc(reinterpret_cast<void **>(&B->ptr), sizeof(*B->ptr) * std::max<int64_t>((cnt), 1), s))) return bail(rc);
    BP_ALLOC(a1, B->nstrips);
    BP_ALLOC(a0, B->nstrips);
    BP_ALLOC(b1, B->nbw);
    BP_ALLOC(b0, B->nbw);
    BP_ALLOC(b2, B->nbw);
    BP_ALLOC(hand, B->nblocks + 1);
    BP_ALLOC(ones, 1);
    BP_ALLOC(next, 1);
    BP_ALLOC(dp, 1);
    BP_ALLOC(di, B->bands);
#undef BP_ALLOC
    BitPair hp{B->a1, B->a0, B->b1, B->b0, B->b2, B->hand, B->ones, m, n, B->nstrips, B->nblocks};
    std::vector<BitItem> items(B->bands);
    for (int b = 0; b < B->bands; ++b) items[b] = BitItem{0, b, b * per_band, b == B->bands - 1 ? 1 : 0};
    if (cudaMemcpyAsync(B->dp, &hp, sizeof(hp), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(B->di, items.data(), sizeof(BitItem) * B->bands, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaEventCreate(&B->ev0) != cudaSuccess || cudaEventCreate(&B->ev1) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return bail(fail(SLCS_ERR_CUDA, "bit plan setup failed"));
    int per_sm = 0;
    cudaError_t e = B->RS == 4 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bit_kernel<4>, 32, 0)
                  : B->RS == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bit_kernel<2>, 32, 0)
                               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bit_kernel<1>, 32, 0);
    if (e != cudaSuccess) return bail(fail(SLCS_ERR_CUDA, "occupancy query failed"));
    B->warps = std::min(B->bands, std::max(1, per_sm) * E->num_sms);
    *out = B;
    return SLCS_OK;
}

// Kernels only: pack the strings, comb, write the score (device int32) -- capturable.
int bit_plan_run(BitPlan *B, const uint8_t *d_a, const uint8_t *d_b, int32_t *d_score, int *d_err, cudaStream_t s,
                 bool capturing) {
    if (B->m == 0 || B->n == 0) {
        SLCS_CUDA_TRY(cudaMemsetAsync(d_score, 0, sizeof(int32_t), s));
        return SLCS_OK;
    }
    SLCS_CUDA_TRY(cudaMemsetAsync(B->ones, 0, sizeof(int32_t), s));
    SLCS_CUDA_TRY(cudaMemsetAsync(B->next, 0, sizeof(int), s));
    SLCS_CUDA_TRY(cudaMemsetAsync(B->hand, 0, sizeof(unsigned long long) * (B->nblocks + 1), s));
    const int pack_warps = B->nstrips + B->nbw;
    bit_pack_kernel<<<std::min(4096, (pack_warps + 7) / 8), 256, 0, s>>>(d_a, B->m, d_b, B->n, B->nstrips, B->nbw, B->a1,
                                                                         B->a0, B->b1, B->b0, B->b2, d_err);
    const unsigned fl = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    SLCS_CUDA_TRY(cudaEventRecordWithFlags(B->ev0, s, fl));
    // one warp per block, so that the bands spread over every SM
    const int blocks = B->warps;
    if (B->RS == 4) bit_kernel<4><<<blocks, 32, 0, s>>>(B->dp, B->di, B->bands, B->next, d_err);
    else if (B->RS == 2) bit_kernel<2><<<blocks, 32, 0, s>>>(B->dp, B->di, B->bands, B->next, d_err);
    else bit_kernel<1><<<blocks, 32, 0, s>>>(B->dp, B->di, B->bands, B->next, d_err);
    SLCS_CUDA_TRY(cudaEventRecordWithFlags(B->ev1, s, fl));
    bit_score_kernel<<<1, 32, 0, s>>>(B->ones, B->m, d_score);
    SLCS_CUDA_TRY(cudaGetLastError());
    return SLCS_OK;
}

int bit_plan_kernel_ms(BitPlan *B, float *ms) {
    SLCS_CUDA_TRY(cudaEventSynchronize(B->ev1));
    SLCS_CUDA_TRY(cudaEventElapsedTime(ms, B->ev0, B->ev1));
    return SLCS_OK;
}

int bitcomb_dev(Engine *E, const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_score, cudaStream_t s) {
    BitPlan *B = nullptr;
    SLCS_TRY(bit_plan_create(E, m, n, s, &B));
    DevBuf<int> err;
    int rc = err.alloc(1, s);
    if (rc == SLCS_OK && cudaMemsetAsync(err.p, 0, sizeof(int), s) != cudaSuccess) rc = fail(SLCS_ERR_CUDA, "memset");
    if (rc == SLCS_OK) rc = bit_plan_run(B, d_a, d_b, d_score, err.p, s, false);
    if (rc == SLCS_OK) rc = check_dev_err(err.p, s);
    bit_plan_destroy(B);
    return rc;
}

}  // namespace slcs

using namespace slcs;

extern "C" {

int slcs_bitcomb_llcs_u8_dev(const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_score, void *stream) {
    if (m < 0 || n < 0) return fail(SLCS_ERR_ARG, "negative length");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    if ((m > 0 && !d_a) || (n > 0 && !d_b) || !d_score) return fail(SLCS_ERR_ARG, "NULL buffer");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    return bitcomb_dev(E, d_a, m, d_b, n, d_score, s);
}

int slcs_bitcomb_llcs_u8(const uint8_t *a, int m, const uint8_t *b, int n, int32_t *score) {
    if (m < 0 || n < 0) return fail(SLCS_ERR_ARG, "negative length");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    if ((m > 0 && !a) || (n > 0 && !b) || !score) return fail(SLCS_ERR_ARG, "NULL buffer");
    for (int i = 0; i < m; ++i)
        if (a[i] > 3) return fail(SLCS_ERR_ARG, "bit-parallel combing needs symbols < 4");
    for (int i = 0; i < n; ++i)
        if (b[i] > 3) return fail(SLCS_ERR_ARG, "bit-parallel combing needs symbols < 4");
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
    SLCS_TRY(bitcomb_dev(E, da.p, m, db.p, n, ds.p, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(score, ds.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SLCS_CUDA_TRY(cudaStreamSynchronize(s));
    return SLCS_OK;
}

}  // extern "C"
