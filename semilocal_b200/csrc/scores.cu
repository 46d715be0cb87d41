// scores.cu -- semi-local scores read from a resident braid.
//
// The braid P of (a, b) (row_to_col of m+n strands) determines the whole semi-local LCS matrix
// (R:include/SemiLocal/SemiLocalLCS.h:13-63 defines it over bExt = ?^m b ?^m; the braid is its cross
// difference, R:common/include/Permutations/Matrices.h:116-124):
//     H(i, j) = j - i + m                                    for j <= i - m,
//     H(i, j) = j + m - i - #{(r, c) in P : r >= i, c < j}   otherwise,          i, j in [0, m+n].
// The dominance count is the reference's top-right summator (R:common/include/Permutations/
// MongeMultuplicationStrategy.h:32-34; R:approximate_matching/utils.h:281-293).  Each query is one block-wide
// count over the rows r >= i (coalesced reads of row_to_col).
#include "slcs_internal.cuh"

namespace slcs {
namespace {

__global__ void __launch_bounds__(256) scores_kernel(const int32_t *__restrict__ r2c, int m, int n,
                                                     const slcs_query *__restrict__ qs, int nq,
                                                     int32_t *__restrict__ out, int *err) {
    __shared__ int warp_cnt[8];
    for (int qi = blockIdx.x; qi < nq; qi += gridDim.x) {
        const slcs_query q = qs[qi];
        int i, j, offset;
        bool ok;
        query_to_matrix(q, m, n, i, j, offset, ok);
        if (!ok) {
            if (threadIdx.x == 0) {
                out[qi] = INT32_MIN;
                raise_error(err, kDevErrBadState);
            }
            continue;
        }
        int cnt = 0;
        if (!(j <= i - m))
            for (int r = i + threadIdx.x; r < m + n; r += blockDim.x) cnt += r2c[r] < j;
        cnt = __reduce_add_sync(kFull, cnt);
        if ((threadIdx.x & 31) == 0) warp_cnt[threadIdx.x >> 5] = cnt;
        __syncthreads();
        if (threadIdx.x == 0) {
            int total = 0;
            for (int w = 0; w < (int) (blockDim.x >> 5); ++w) total += warp_cnt[w];
            const int h = (j <= i - m) ? (j - i + m) : (j + m - i - total);
            out[qi] = h + offset;
        }
        __syncthreads();
    }
}

int scores_dev(const int32_t *d_r2c, int m, int n, const slcs_query *d_q, int nq, int32_t *d_out, int *d_err,
               cudaStream_t s) {
    if (nq <= 0) return SLCS_OK;
    scores_kernel<<<std::min(nq, 65535), 256, 0, s>>>(d_r2c, m, n, d_q, nq, d_out, d_err);
    SLCS_CUDA_TRY(cudaGetLastError());
    return SLCS_OK;
}

}  // namespace

int launch_scores(const int32_t *d_r2c, int m, int n, const slcs_query *d_q, int nq, int32_t *d_out, int *d_err,
                  cudaStream_t s) {
    return scores_dev(d_r2c, m, n, d_q, nq, d_out, d_err, s);
}

int launch_scores_host(const int32_t *d_r2c, int m, int n, const slcs_query *q, int nq, int32_t *out,
                       cudaStream_t s) {
    if (nq <= 0) return SLCS_OK;
    DevBuf<slcs_query> dq;
    DevBuf<int32_t> dout;
    DevBuf<int> err;
    SLCS_TRY(dq.alloc(nq, s));
    SLCS_TRY(dout.alloc(nq, s));
    SLCS_TRY(err.alloc(1, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(dq.p, q, sizeof(slcs_query) * nq, cudaMemcpyHostToDevice, s));
    SLCS_TRY(scores_dev(d_r2c, m, n, dq.p, nq, dout.p, err.p, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(out, dout.p, sizeof(int32_t) * nq, cudaMemcpyDeviceToHost, s));
    return check_dev_err(err.p, s);
}

// ---- window scans: LCS(a, b[s..s+w)) for every window s = 0..n-w --------------------------------------
// string-substring score of window s: H(s + m, s + w) = w - D(s), D(s) = #{r >= s + m : r2c[r] < s + w}.
// Moving the window by one drops row s + m and adds column s + w:
//     D(s + 1) = D(s) - [r2c[s + m] < s + w] + [c2r[s + w] >= s + m + 1],
// the incremental dominance moves of the reference's window matcher (R:approximate_matching/WindowAMatch.h:
// 58-71, R:common/include/Permutations/DominanceSum.h:210-294) made data-parallel: one count for D(0), one
// delta per window, one prefix sum.
constexpr int kWinPer = 2048;   // windows per scan block (256 threads x 8)

__global__ void win_invert_kernel(const int32_t *__restrict__ r2c, int size, int32_t *__restrict__ c2r, int *err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x) {
        const int c = r2c[i];
        if (c < 0 || c >= size) {
            raise_error(err, kDevErrBadState);
            continue;
        }
        c2r[c] = i;
    }
}

__global__ void win_d0_kernel(const int32_t *__restrict__ r2c, int m, int n, int w, int *d0) {
    int cnt = 0;
    for (int r = m + blockIdx.x * blockDim.x + threadIdx.x; r < m + n; r += gridDim.x * blockDim.x) cnt += r2c[r] < w;
    cnt = __reduce_add_sync(kFull, cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(d0, cnt);
}

__device__ __forceinline__ int win_delta(const int32_t *r2c, const int32_t *c2r, int m, int w, int s) {
    return (c2r[s + w] >= s + m + 1 ? 1 : 0) - (r2c[s + m] < s + w ? 1 : 0);
}

// per block: the sum of its windows' deltas (deltas of windows 0..nwin-2 lead from D(s) to D(s+1))
__global__ void __launch_bounds__(256) win_block_sums_kernel(const int32_t *__restrict__ r2c,
                                                             const int32_t *__restrict__ c2r, int m, int w, int nd,
                                                             int *__restrict__ bsum) {
    const int s0 = blockIdx.x * kWinPer;
    int acc = 0;
    for (int s = s0 + threadIdx.x; s < min(s0 + kWinPer, nd); s += blockDim.x) acc += win_delta(r2c, c2r, m, w, s);
    acc = __reduce_add_sync(kFull, acc);
    __shared__ int ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int i = 0; i < 8; ++i) t += ws[i];
        bsum[blockIdx.x] = t;
    }
}

// exclusive prefix of the block sums in place (one block of 1024 threads, each a contiguous chunk)
__global__ void __launch_bounds__(1024) win_scan_sums_kernel(int *bsum, int nb) {
    const int per = (nb + 1023) / 1024;
    const int b0 = min(nb, (int) threadIdx.x * per), b1 = min(nb, b0 + per);
    int t = 0;
    for (int b = b0; b < b1; ++b) t += bsum[b];
    __shared__ int part[1024];
    part[threadIdx.x] = t;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        const int v = threadIdx.x >= (unsigned) d ? part[threadIdx.x - d] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int run = part[threadIdx.x] - t;
    for (int b = b0; b < b1; ++b) {
        const int v = bsum[b];
        bsum[b] = run;
        run += v;
    }
}

// out[s] = w - D(s): each block scans its windows (8 per thread, then across threads)
__global__ void __launch_bounds__(256) win_out_kernel(const int32_t *__restrict__ r2c, const int32_t *__restrict__ c2r,
                                                      int m, int w, int nwin, const int *__restrict__ bsum,
                                                      const int *__restrict__ d0, int32_t *__restrict__ out) {
    const int s0 = blockIdx.x * kWinPer + threadIdx.x * 8;
    int d[8], t = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int s = s0 + i;   // delta leading from window s to s + 1
        d[i] = (s < nwin - 1) ? win_delta(r2c, c2r, m, w, s) : 0;
        t += d[i];
    }
    // exclusive prefix of the thread totals
    __shared__ int part[256];
    part[threadIdx.x] = t;
    __syncthreads();
    for (int k = 1; k < 256; k <<= 1) {
        const int v = threadIdx.x >= (unsigned) k ? part[threadIdx.x - k] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int D = *d0 + bsum[blockIdx.x] + part[threadIdx.x] - t;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int s = s0 + i;
        if (s < nwin) out[s] = w - D;
        D += d[i];
    }
}

int window_scores_dev(const int32_t *d_r2c, const int32_t *d_c2r, int m, int n, int w, int32_t *d_out, cudaStream_t s) {
    NvtxRange nv("slcs: window scan");
    const int size = m + n, nwin = n - w + 1;
    if (nwin <= 0) return SLCS_OK;
    const int nblk = (nwin + kWinPer - 1) / kWinPer;
    DevBuf<int> scratch;   // err, d0, block sums
    SLCS_TRY(scratch.alloc(2 + nblk, s));
    int *err = scratch.p, *d0 = scratch.p + 1, *bsum = scratch.p + 2;
    SLCS_CUDA_TRY(cudaMemsetAsync(scratch.p, 0, sizeof(int) * 2, s));
    DevBuf<int32_t> inv;
    if (!d_c2r) {
        SLCS_TRY(inv.alloc(std::max(size, 1), s));
        win_invert_kernel<<<std::min(4096, (size + 255) / 256), 256, 0, s>>>(d_r2c, size, inv.p, err);
        d_c2r = inv.p;
    }
    win_d0_kernel<<<std::max(1, std::min(1024, (n + 255) / 256)), 256, 0, s>>>(d_r2c, m, n, w, d0);
    win_block_sums_kernel<<<nblk, 256, 0, s>>>(d_r2c, d_c2r, m, w, nwin - 1, bsum);
    win_scan_sums_kernel<<<1, 1024, 0, s>>>(bsum, nblk);
    win_out_kernel<<<nblk, 256, 0, s>>>(d_r2c, d_c2r, m, w, nwin, bsum, d0, d_out);
    SLCS_CUDA_TRY(cudaGetLastError());
    return check_dev_err(err, s);
}

}  // namespace slcs

using namespace slcs;

extern "C" {

int slcs_scores_dev(const int32_t *d_row_to_col, int m, int n, const slcs_query *d_q, int nq, int32_t *d_out,
                    void *stream) {
    if (m < 0 || n < 0 || nq < 0) return fail(SLCS_ERR_ARG, "negative size");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    if (nq > 0 && (!d_q || !d_out || (m + n > 0 && !d_row_to_col))) return fail(SLCS_ERR_ARG, "NULL buffer");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    DevBuf<int> err;
    SLCS_TRY(err.alloc(1, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    SLCS_TRY(scores_dev(d_row_to_col, m, n, d_q, nq, d_out, err.p, s));
    const int rc = check_dev_err(err.p, s);
    if (rc == SLCS_ERR_INTERNAL) return fail(SLCS_ERR_ARG, "a query is out of range (its answer is INT32_MIN)");
    return rc;
}

int slcs_scores(const int32_t *row_to_col, int m, int n, const slcs_query *q, int nq, int32_t *out) {
    if (m < 0 || n < 0 || nq < 0) return fail(SLCS_ERR_ARG, "negative size");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    if (nq == 0) return SLCS_OK;
    if (!q || !out || (m + n > 0 && !row_to_col)) return fail(SLCS_ERR_ARG, "NULL buffer");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = E->stream;
    DevBuf<int32_t> dr, dout;
    DevBuf<slcs_query> dq;
    SLCS_TRY(dr.alloc(m + n, s));
    SLCS_TRY(dq.alloc(nq, s));
    SLCS_TRY(dout.alloc(nq, s));
    if (m + n) SLCS_CUDA_TRY(cudaMemcpyAsync(dr.p, row_to_col, sizeof(int32_t) * (m + n), cudaMemcpyHostToDevice, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(dq.p, q, sizeof(slcs_query) * nq, cudaMemcpyHostToDevice, s));
    const int rc = slcs_scores_dev(dr.p, m, n, dq.p, nq, dout.p, s);
    SLCS_CUDA_TRY(cudaMemcpyAsync(out, dout.p, sizeof(int32_t) * nq, cudaMemcpyDeviceToHost, s));
    SLCS_CUDA_TRY(cudaStreamSynchronize(s));
    return rc;
}

int slcs_window_scores_dev(const int32_t *d_row_to_col, const int32_t *d_col_to_row, int m, int n, int w,
                           int32_t *d_out, void *stream) {
    if (m < 0 || n < 0 || w < 1 || w > n) return fail(SLCS_ERR_ARG, "window length must be in [1, n]");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    if (!d_row_to_col || !d_out) return fail(SLCS_ERR_ARG, "NULL buffer");
    Engine *E;
    SLCS_TRY(engine(&E));
    return window_scores_dev(d_row_to_col, d_col_to_row, m, n, w, d_out,
                             stream ? (cudaStream_t) stream : E->stream);
}

int slcs_window_scores(const int32_t *row_to_col, int m, int n, int w, int32_t *out) {
    if (m < 0 || n < 0 || w < 1 || w > n) return fail(SLCS_ERR_ARG, "window length must be in [1, n]");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    if (!row_to_col || !out) return fail(SLCS_ERR_ARG, "NULL buffer");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = E->stream;
    DevBuf<int32_t> dr, dout;
    SLCS_TRY(dr.alloc(m + n, s));
    SLCS_TRY(dout.alloc(n - w + 1, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(dr.p, row_to_col, sizeof(int32_t) * (m + n), cudaMemcpyHostToDevice, s));
    SLCS_TRY(window_scores_dev(dr.p, nullptr, m, n, w, dout.p, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(out, dout.p, sizeof(int32_t) * (n - w + 1), cudaMemcpyDeviceToHost, s));
    SLCS_CUDA_TRY(cudaStreamSynchronize(s));
    return SLCS_OK;
}

}  // extern "C"
