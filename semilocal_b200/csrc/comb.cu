// comb.cu -- integer sticky-braid combing on sm_100a.
//
// The grid of a pair (rows = symbols of a, columns = symbols of b) is cut into horizontal bands of 32*R rows.
// One warp combs one band: lane l owns R consecutive rows (their left strands and a-symbols stay in
// registers for the whole band) and the warp is a 32-stage systolic array: at step s lane l processes
// column s - l, the strand leaving a lane's last row goes down to the next lane by a warp shuffle.
// The warp exchanges 32 columns at a time with the band above / below through the pair's output array
// (entries 0..n-1 hold the top strands handed down band by band, in place), synchronised by a per-band
// progress counter (release/acquire, bounded spins that give up into the device error word).
// Work items (pair, band) are dequeued in order by persistent warps, so a band only ever waits for a band
// that an already-running warp owns: no co-residency assumption, no deadlock.
//
// Cell rule (R:include/SemiLocal/SemiLocalLCS.h:153-174, canonical form :81-114): the strands swap iff the
// symbols match or the left strand's id is larger than the top strand's.
// Output (ends -> starts, R:include/SemiLocal/SemiLocalLCS.h:117-121): column j < n receives the strand
// leaving the bottom of column j, column n+l the strand leaving the right side of row m-1-l.
#include "slcs_internal.cuh"

namespace slcs {
namespace {

constexpr int kStrandPad = 0x7fffffff;        // strand of a padding column: never smaller than a left strand

// One cell: the strands swap iff the symbols match or the left strand's id is larger than the top strand's.
// The two strands leave the cell as they entered it, possibly swapped, so the left strand's new id is
// (L + t) - nt.  That sum and difference are two IMADs with multipliers `one` = 1 and `neg1` = -1 passed in as
// kernel parameters (the compiler cannot fold them into additions), which run on the FMA pipe; the compares and
// the select stay on the ALU pipe.  Three ALU ops per cell instead of four (two compares, two selects): the ALU
// pipe is the bound at full occupancy, and the FMA pipe is otherwise idle.
__device__ __forceinline__ void comb_cell(int A, int bs, int &L, int &t, int one, int neg1) {
    const int sum = L * one + t;
    const bool sw = (A == bs) | (L > t);
    const int nt = sw ? L : t;
    L = nt * neg1 + sum;
    t = nt;
}

template <typename T, int R, int CH>
__device__ __forceinline__ void comb_band(const CombPair &P, const CombItem &I, int *err, int lane, int one,
                                          int neg1) {
    static_assert(CH == 1 || (CH == 2 && R >= 2), "two chains need at least two rows per lane");
    const T *__restrict__ a = static_cast<const T *>(P.a);
    const T *__restrict__ b = static_cast<const T *>(P.b);
    const int m = P.m, n = P.n;
    const int rbase = I.r0 + lane * R;

    int A[R], L[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int row = rbase + k;
        if (row < m) {
            A[k] = static_cast<int>(a[row]);
            L[k] = m - 1 - row;
        } else {
            A[k] = kSymRowVirtual;
            L[k] = -1;
        }
    }

    const bool has_prev = I.band > 0;
    const int *prev_prog = has_prev ? P.progress + (I.band - 1) : nullptr;
    int *my_prog = P.progress + I.band;
    // steps 0 .. n+32*CH-1 (column n-1 leaves the warp's last stage at step n+32*CH-1)
    const int nchunks = (n + 32 * CH + 31) >> 5;

    int io_t = kStrandPad, io_b = kSymColVirtual;
    // b-symbols are read one chunk ahead of their use (they do not depend on the band above), so the load's
    // latency is not exposed at every chunk boundary of a band that has the SM to itself
    int pre_b = lane < n ? static_cast<int>(b[lane]) : kSymColVirtual;
    // Loads the top strands and b-symbols of columns [32q, 32q+32) into io (lane j <- column 32q+j).
    auto load = [&](int q) -> bool {
        const int c0 = q << 5;
        io_b = pre_b;
        pre_b = c0 + 32 + lane < n ? static_cast<int>(b[c0 + 32 + lane]) : kSymColVirtual;
        if (has_prev && c0 < n) {
            int ok = 1;
            if (lane == 0) ok = wait_at_least(prev_prog, min(n, c0 + 32), err) ? 1 : 0;
            ok = __shfl_sync(kFull, ok, 0);
            if (!ok) return false;
        }
        const int c = c0 + lane;
        io_t = c < n ? (has_prev ? __ldcg(P.c2r + c) : (m + c)) : kStrandPad;
        return true;
    };

    if (!load(0)) return;
    // t / bs: the strand and symbol entering the lane's first row; with two chains (CH = 2) the lane is two
    // systolic stages, rows [0, R/2) and [R/2, R): tm / bm carry the upper stage's output to the lower stage one
    // step later, so the two halves work on neighbouring columns at once (two independent dependency chains).
    int t = kStrandPad, bs = kSymColVirtual;
    int tm = kStrandPad, bm = kSymColVirtual;
    const int src_dn = (lane + 31) & 31, src_up = (lane + 1) & 31;
    for (int q = 0; q < nchunks; ++q) {
#pragma unroll 4
        for (int k = 0; k < 32; ++k) {
            // systolic shift: lane l takes the strand (and symbol) lane l-1 produced one step ago;
            // lane 0 receives the warp's bottom output instead, parks it in io and takes the next input.
            t = __shfl_sync(kFull, t, src_dn);
            bs = __shfl_sync(kFull, bs, src_dn);
            if (lane == 0) {
                const int x = t;
                t = io_t;
                io_t = x;
                bs = io_b;
            }
            if (CH == 1) {
#pragma unroll
                for (int r = 0; r < R; ++r) comb_cell(A[r], bs, L[r], t, one, neg1);
            } else {
                int u = t, w = tm;
                const int bw = bm;
#pragma unroll
                for (int r = 0; r < R / 2; ++r) {
                    comb_cell(A[r], bs, L[r], u, one, neg1);
                    comb_cell(A[R / 2 + r], bw, L[R / 2 + r], w, one, neg1);
                }
                tm = u;
                bm = bs;
                t = w;
                bs = bw;
            }
            io_t = __shfl_sync(kFull, io_t, src_up);
            io_b = __shfl_sync(kFull, io_b, src_up);
        }
        // io_t of lane j now holds the strand that left the band's bottom in column 32(q-CH)+j.
        const int col = ((q - CH) << 5) + lane;
        const bool valid = col >= 0 && col < n;
        if (valid) __stcg(P.c2r + col, io_t);
        if (I.last && P.score != nullptr) {
            const unsigned bal = __ballot_sync(kFull, valid && io_t < m);
            if (lane == 0 && bal) atomicAdd(P.score, __popc(bal));
        }
        __syncwarp();
        if (!I.last && lane == 0 && q >= CH - 1) st_release(my_prog, min(n, (q - CH + 1) << 5));
        if (q + 1 < nchunks && !load(q + 1)) return;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int row = rbase + k;
        if (row < m) P.c2r[n + (m - 1 - row)] = L[k];
    }
}

// CH = 1: one dependency chain per lane (pairs that share the device with many others: the ALU pipe is the
// bound, and the shorter pipeline costs 32 fewer steps per band).  CH = 2: two chains per lane, for a lone pair
// whose few bands leave the SMs short of warps, where the chain's latency is the bound.  one = 1, neg1 = -1.
template <typename T, int CH>
__global__ void __launch_bounds__(32, 12) comb_kernel(const CombPair *__restrict__ pairs,
                                                   const CombItem *__restrict__ items, int nitems, int *next,
                                                   int *err, int one, int neg1) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int it = nitems;
        if (lane == 0 && ld_relaxed(err) == kDevErrNone) it = atomicAdd(next, 1);
        it = __shfl_sync(kFull, it, 0);
        if (it >= nitems) return;
        const CombItem I = items[it];
        const CombPair P = pairs[I.pair];
        switch (I.R) {
            case 32: comb_band<T, 32, CH>(P, I, err, lane, one, neg1); break;
            case 16: comb_band<T, 16, CH>(P, I, err, lane, one, neg1); break;
            case 8: comb_band<T, 8, CH>(P, I, err, lane, one, neg1); break;
            case 4: comb_band<T, 4, CH>(P, I, err, lane, one, neg1); break;
            case 2: comb_band<T, 2, CH>(P, I, err, lane, one, neg1); break;
            default: comb_band<T, 1, 1>(P, I, err, lane, one, neg1); break;
        }
    }
}

// ---- lone pairs: register tiles ----
//
// A pair alone on the device gets few bands, one warp each, and a warp alone on its SM sub-partition is bound by
// its own latency, not by issue: each step of the band kernel above waits for the shuffle bringing the strand from
// the lane above, so a step costs a shuffle's latency however few rows the lane combs.  Here a lane combs a tile
// of R rows x C columns per step: the C strands arriving from the lane above travel in C independent shuffles
// (one latency per step), and the R x C cells form a small wavefront with C-fold parallelism.  Everything
// else works per sub-chunk of 32 columns (K = 32 / C steps):
//   * b-symbols go through a ring of 256 (C = 4) or 512 (C = 8) columns in shared memory (as ints, padding columns
//     kSymColVirtual), one column per lane per sub-chunk, loaded one sub-chunk ahead; each step reads its C
//     symbols in 16-byte accesses;
//   * lane 0's input strands of sub-chunk j come from the band above through the pair's hand-off words, each
//     carrying the writing band's tag (band + 1) beside the strand in one 64-bit word: loaded one sub-chunk ahead
//     and polled (bounded) only while the tag is not there yet;
//   * lane 31's bottom strands are staged in shared memory and published 32 words at a time (coalesced) as soon
//     as a sub-chunk is complete, two steps after its last group left the warp.  The last band writes them to c2r
//     instead (they are final) and counts the score.
// The band kernel's persistent in-order dequeue is kept: a band only waits for a band a running warp owns.
// Measured on B200 (8192 x 8192, one warp per band): a step of an 8 x 4 tile takes ~330 cycles against ~240 for
// 4 x 4 and ~76 for the band kernel's one column of four rows, and a band starts ~47 steps after the one above
// (32 for the lanes, the rest the hand-off); the whole pair takes 0.61 ms against 0.86-1.0 ms.
// C consecutive ints of shared memory in 16-byte accesses (C a multiple of 4, the address 16-byte aligned)
template <int C>
__device__ __forceinline__ void lds_ints(const int *p, int (&o)[C]) {
#pragma unroll
    for (int i = 0; i < C; i += 4) {
        const int4 v = *reinterpret_cast<const int4 *>(p + i);
        o[i] = v.x;
        o[i + 1] = v.y;
        o[i + 2] = v.z;
        o[i + 3] = v.w;
    }
}
template <int C>
__device__ __forceinline__ void sts_ints(int *p, const int (&v)[C]) {
#pragma unroll
    for (int i = 0; i < C; i += 4) *reinterpret_cast<int4 *>(p + i) = make_int4(v[i], v[i + 1], v[i + 2], v[i + 3]);
}

// symbol ring: the columns a step can read span 31 C + 32 behind the newest sub-chunk, plus the sub-chunk
// written ahead; a power of two above that
template <int C>
struct TileShared {
    static constexpr int kRing = C <= 4 ? 256 : 512;
    int sym[kRing];   // b-symbols of columns c (at c & (kRing - 1)) as ints
    int tin[64];      // lane 0's input strands of two sub-chunks (column c at c & 63)
    int tout[64];     // lane 31's output strands of two sub-chunks (column c at c & 63)
};

template <typename T, int R, int C>
__device__ __forceinline__ void comb_tile_band(const CombPair &P, const CombItem &I, int *err, int lane, int one,
                                               int neg1, TileShared<C> &S) {
    static_assert(C == 4 || C == 8, "tile widths 4 and 8");
    constexpr int K = 32 / C;   // steps per sub-chunk of 32 columns
    constexpr int SB = TileShared<C>::kRing;
    const T *__restrict__ a = static_cast<const T *>(P.a);
    const T *__restrict__ b = static_cast<const T *>(P.b);
    const int m = P.m, n = P.n;
    const int rbase = I.r0 + lane * R;

    int A[R], L[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int row = rbase + k;
        if (row < m) {
            A[k] = static_cast<int>(a[row]);
            L[k] = m - 1 - row;
        } else {
            A[k] = kSymRowVirtual;
            L[k] = -1;
        }
    }
    const int G = (n + C - 1) / C;               // column groups; lane l combs group s - l at step s
    const int nsub = (G + 31 + K - 1) / K;       // sub-chunks of steps
    const int Q = (n + 31) >> 5;                 // sub-chunks of columns
    const bool has_prev = I.band > 0;
    const unsigned tag_above = (unsigned) I.band;                                  // the band above: its index + 1
    const unsigned long long my_tag = (unsigned long long) (I.band + 1) << 32;

    __syncwarp();   // the previous band's last reads of S are done
    for (int i = lane; i < SB; i += 32) S.sym[i] = kSymColVirtual;
    int pb = lane < n ? static_cast<int>(b[lane]) : kSymColVirtual;
    unsigned long long pw = (has_prev && lane < n) ? ld_relaxed64(P.hand + lane) : 0ull;

    int t[C];
#pragma unroll
    for (int c = 0; c < C; ++c) t[c] = kStrandPad;
    int cnt = 0;   // last band: bottom strands < m (the score)
    int qpub = 0;  // next sub-chunk of columns to publish

    // publishes every column sub-chunk whose groups all left the warp before step `done` (exclusive)
    auto publish = [&](int done) {
        while (qpub < Q && min((qpub + 1) * K, G) + 31 <= done) {
            const int col = (qpub << 5) + lane;
            if (col < n) {
                const int v = S.tout[col & 63];
                if (I.last) {
                    P.c2r[col] = v;
                    cnt += v < m;
                } else {
                    st_relaxed64(P.hand + col, my_tag | (unsigned) v);
                }
            }
            ++qpub;
        }
    };

    for (int j = 0; j < nsub; ++j) {
        const int col = (j << 5) + lane;
        int in = kStrandPad;
        bool ok = true;
        if (col < n) {
            if (!has_prev) in = m + col;
            else {
                ok = wait_tag(P.hand + col, pw, tag_above, err);
                in = (int) (unsigned) pw;
            }
        }
        if (!__all_sync(kFull, ok)) return;
        publish(j * K);   // reads S.tout written before the last __syncwarp
        S.tin[col & 63] = in;
        S.sym[col & (SB - 1)] = pb;
        const int ncol = col + 32;
        pb = ncol < n ? static_cast<int>(b[ncol]) : kSymColVirtual;
        if (has_prev && ncol < n) pw = ld_relaxed64(P.hand + ncol);
        __syncwarp();
        const int tin_base = (j & 1) << 5;
        const int sym_base = (j * K - lane) * C;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            int x[C], bs[C];
            lds_ints<C>(S.tin + tin_base + k * C, x);
            lds_ints<C>(S.sym + ((sym_base + k * C) & (SB - 1)), bs);
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const int u = __shfl_up_sync(kFull, t[c], 1);
                t[c] = lane == 0 ? x[c] : u;
            }
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int c = 0; c < C; ++c) comb_cell(A[r], bs[c], L[r], t[c], one, neg1);
            const int g = j * K + k - 31;
            if (lane == 31 && g >= 0 && g < G) sts_ints<C>(S.tout + ((g * C) & 63), t);
        }
        __syncwarp();
    }
    publish(nsub * K);
    if (I.last && P.score != nullptr) {
        const int tot = __reduce_add_sync(kFull, cnt);
        if (lane == 0 && tot) atomicAdd(P.score, tot);
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int row = rbase + k;
        if (row < m) P.c2r[n + (m - 1 - row)] = L[k];
    }
}

template <typename T, int C>
__global__ void __launch_bounds__(32, 1) comb_tile_kernel(const CombPair *__restrict__ pairs,
                                                         const CombItem *__restrict__ items, int nitems, int *next,
                                                         int *err, int one, int neg1) {
    __shared__ __align__(16) TileShared<C> S;
    const int lane = threadIdx.x & 31;
    for (;;) {
        int it = nitems;
        if (lane == 0 && ld_relaxed(err) == kDevErrNone) it = atomicAdd(next, 1);
        it = __shfl_sync(kFull, it, 0);
        if (it >= nitems) return;
        const CombItem I = items[it];
        const CombPair P = pairs[I.pair];
        switch (I.R) {
            case 16: comb_tile_band<T, 16, C>(P, I, err, lane, one, neg1, S); break;
            case 8: comb_tile_band<T, 8, C>(P, I, err, lane, one, neg1, S); break;
            case 2: comb_tile_band<T, 2, C>(P, I, err, lane, one, neg1, S); break;
            default: comb_tile_band<T, 4, C>(P, I, err, lane, one, neg1, S); break;
        }
    }
}

__global__ void invert_kernel(const int32_t *__restrict__ c2r, int size, int32_t *__restrict__ r2c, int rot,
                              int *err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x) {
        const int r = c2r[i];
        if (r < 0 || r >= size) {   // never expected: report instead of writing out of bounds
            raise_error(err, kDevErrBadState);
            continue;
        }
        if (rot) r2c[size - 1 - r] = size - 1 - i;
        else r2c[r] = i;
    }
}

}  // namespace

int plan_bands(int pair, int m, int R, std::vector<CombItem> &items) {
    int Rmax = 1;
    while (Rmax * 2 <= R && Rmax < 32) Rmax *= 2;
    const size_t first = items.size();
    int r0 = 0, band = 0;
    while (r0 < m) {
        const int rem = m - r0;
        // smallest band height covering the rest; taken when it pads by at most a third
        int Rc = 1;
        while (32 * Rc < rem) Rc *= 2;
        if (Rc <= Rmax && (3 * 32 * Rc <= 4 * rem || rem <= 32)) {
            items.push_back(CombItem{pair, band++, r0, Rc, 0});
            break;
        }
        // otherwise the largest band height the rest fills completely
        int Rf = 1;
        while (Rf * 2 <= Rmax && 32 * Rf * 2 <= rem) Rf *= 2;
        items.push_back(CombItem{pair, band++, r0, Rf, 0});
        r0 += 32 * Rf;
    }
    if (items.size() > first) items.back().last = 1;
    return band;
}

template <typename T>
int launch_comb(const CombPair *d_pairs, const CombItem *d_items, int nitems, int *d_next, int *d_err,
                int grid_warps, cudaStream_t s) {
    if (nitems <= 0) return SLCS_OK;
    // one warp per block (the warps are independent workers), so that few items still spread over all SMs
    const int warps = grid_warps < nitems ? grid_warps : nitems;
    comb_kernel<T, 1><<<warps, 32, 0, s>>>(d_pairs, d_items, nitems, d_next, d_err, 1, -1);
    SLCS_CUDA_TRY(cudaGetLastError());
    return SLCS_OK;
}
template int launch_comb<uint8_t>(const CombPair *, const CombItem *, int, int *, int *, int, cudaStream_t);
template int launch_comb<int32_t>(const CombPair *, const CombItem *, int, int *, int *, int, cudaStream_t);

template <typename T>
int launch_comb_lone(const CombPair *d_pairs, const CombItem *d_items, int nitems, int *d_next, int *d_err,
                     int grid_warps, cudaStream_t s) {
    if (nitems <= 0) return SLCS_OK;
    const int warps = grid_warps < nitems ? grid_warps : nitems;
    // two chains per lane only while the bands fill at most half the resident warps (measured on B200: 8192^2,
    // up to 256 bands, 1.09 -> 0.92 ms; the 2^20 pair's 1024 bands gain nothing from it)
    if (2 * nitems <= grid_warps)
        comb_kernel<T, 2><<<warps, 32, 0, s>>>(d_pairs, d_items, nitems, d_next, d_err, 1, -1);
    else
        comb_kernel<T, 1><<<warps, 32, 0, s>>>(d_pairs, d_items, nitems, d_next, d_err, 1, -1);
    SLCS_CUDA_TRY(cudaGetLastError());
    return SLCS_OK;
}
template int launch_comb_lone<uint8_t>(const CombPair *, const CombItem *, int, int *, int *, int, cudaStream_t);
template int launch_comb_lone<int32_t>(const CombPair *, const CombItem *, int, int *, int *, int, cudaStream_t);

int plan_tile_bands(int pair, int m, int R, std::vector<CombItem> &items) {
    const int h = 32 * R;
    const int bands = (m + h - 1) / h;
    for (int i = 0; i < bands; ++i) items.push_back(CombItem{pair, i, i * h, R, i == bands - 1 ? 1 : 0});
    return bands;
}

template <typename T>
int launch_comb_tile(const CombPair *d_pairs, const CombItem *d_items, int nitems, int *d_next, int *d_err,
                     int grid_warps, int C, cudaStream_t s) {
    if (nitems <= 0) return SLCS_OK;
    const int warps = grid_warps < nitems ? grid_warps : nitems;
    if (C == 8)
        comb_tile_kernel<T, 8><<<warps, 32, 0, s>>>(d_pairs, d_items, nitems, d_next, d_err, 1, -1);
    else
        comb_tile_kernel<T, 4><<<warps, 32, 0, s>>>(d_pairs, d_items, nitems, d_next, d_err, 1, -1);
    SLCS_CUDA_TRY(cudaGetLastError());
    return SLCS_OK;
}
template int launch_comb_tile<uint8_t>(const CombPair *, const CombItem *, int, int *, int *, int, int, cudaStream_t);
template int launch_comb_tile<int32_t>(const CombPair *, const CombItem *, int, int *, int *, int, int, cudaStream_t);

TileShape tile_shape_for(int rows, int band_rows, int lane_cols) {
    if (lane_cols == 4 || lane_cols == 8) {
        const bool given = band_rows == 64 || band_rows == 128 || band_rows == 256 || band_rows == 512;
        return TileShape{given ? band_rows / 32 : kTileRows, lane_cols};
    }
    if (lane_cols != 0 || band_rows > 0) return TileShape{};   // one column per step / the band kernel's height
    // automatic: 8 x 4 tiles, 16 x 4 above 2^18 rows, so that a pair keeps about 1024 bands or fewer (measured on
    // B200, square pairs: 8192 0.61 ms against 1.0 for the band kernel, 2^18 28.8 against 46.5, 2^19 81.8 (16 x 4)
    // against 143; at 2^20 the band kernel's 1024 bands of 1024 rows are faster: 294 against 312 or more)
    if (rows > kTileAutoMaxRows) return TileShape{};
    return TileShape{rows > (1 << 18) ? 16 : kTileRows, kTileCols};
}

int comb_resident_warps_sm(int num_sms) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, comb_kernel<uint8_t, 1>, 32, 0) != cudaSuccess ||
        per_sm <= 0) {
        cudaGetLastError();
        per_sm = 12;
    }
    return per_sm * num_sms;
}

int comb_resident_warps(Engine *E) { return comb_resident_warps_sm(E->num_sms); }

int launch_invert(const int32_t *c2r, int size, int32_t *r2c, bool rot180, int *d_err, cudaStream_t s) {
    if (size <= 0) return SLCS_OK;
    int blocks = (size + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    invert_kernel<<<blocks, 256, 0, s>>>(c2r, size, r2c, rot180 ? 1 : 0, d_err);
    SLCS_CUDA_TRY(cudaGetLastError());
    return SLCS_OK;
}

}  // namespace slcs
