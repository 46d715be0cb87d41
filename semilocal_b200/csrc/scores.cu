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

}  // namespace slcs

using namespace slcs;

extern "C" {

int slcs_scores_dev(const int32_t *d_row_to_col, int m, int n, const slcs_query *d_q, int nq, int32_t *d_out,
                    void *stream) {
    if (m < 0 || n < 0 || nq < 0) return fail(SLCS_ERR_ARG, "negative size");
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

}  // extern "C"
