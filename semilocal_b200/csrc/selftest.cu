// selftest.cu -- failure-path self-test of the bounded device waits.
//
// The combing kernels chain warps through progress counters; every wait on one is bounded by kWaitLimitNs of
// the GPU's global timer, after which the waiting warp sets the device error word and returns, and the host
// maps the word to SLCS_ERR_TIMEOUT.  This entry point makes exactly that happen on purpose, without faulting
// anything: it launches the real combing kernel on the second band of a 64 x 64 pair and never launches the
// first, so the progress counter the band waits on is never set.  The reference has no counterpart (its
// failures end the process).
#include "slcs_internal.cuh"

using namespace slcs;

extern "C" int slcs_selftest_wait_timeout(int32_t *status) {
    if (!status) return fail(SLCS_ERR_ARG, "NULL status");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = E->stream;
    const int m = 64, n = 64;
    DevBuf<uint8_t> ab;
    DevBuf<int32_t> c2r, prog;
    DevBuf<CombPair> pair;
    DevBuf<CombItem> item;
    DevBuf<int> words;   // error word, work counter
    SLCS_TRY(ab.alloc(m + n, s));
    SLCS_TRY(c2r.alloc(m + n, s));
    SLCS_TRY(prog.alloc(2, s));
    SLCS_TRY(pair.alloc(1, s));
    SLCS_TRY(item.alloc(1, s));
    SLCS_TRY(words.alloc(2, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(ab.p, 0, m + n, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(prog.p, 0, sizeof(int32_t) * 2, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(words.p, 0, sizeof(int) * 2, s));
    const CombPair hp{ab.p, ab.p + m, c2r.p, prog.p, nullptr, m, n};
    const CombItem hi{0, 1, 32, 1, 1};   // band 1 (rows 32..63); band 0 is never launched
    SLCS_CUDA_TRY(cudaMemcpyAsync(pair.p, &hp, sizeof(hp), cudaMemcpyHostToDevice, s));
    SLCS_CUDA_TRY(cudaMemcpyAsync(item.p, &hi, sizeof(hi), cudaMemcpyHostToDevice, s));
    SLCS_TRY(launch_comb<uint8_t>(pair.p, item.p, 1, words.p + 1, words.p, 1, s));
    *status = check_dev_err(words.p, s);   // SLCS_ERR_TIMEOUT expected
    return SLCS_OK;
}

// ---- permutation validity check --------------------------------------------------------------------------
// Every value of perm[0..size) in range and hit once: a bitmap with atomicOr finds repeats; with size values
// and no repeat or out-of-range value the map is a bijection.
namespace {
__global__ void perm_check_kernel(const int32_t *__restrict__ perm, int size, unsigned *__restrict__ bits,
                                  int *__restrict__ bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x) {
        const int v = perm[i];
        if (v < 0 || v >= size) {
            atomicAdd(bad, 1);
            continue;
        }
        const unsigned bit = 1u << (v & 31);
        if (atomicOr(bits + (v >> 5), bit) & bit) atomicAdd(bad, 1);
    }
}
}  // namespace

extern "C" int slcs_check_permutation_dev(const int32_t *d_perm, int size, int32_t *bad_entries, void *stream) {
    if (size < 0 || (size > 0 && !d_perm)) return fail(SLCS_ERR_ARG, "bad arguments");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = stream ? (cudaStream_t) stream : E->stream;
    const int words = (size + 31) / 32;
    DevBuf<unsigned> bits;
    DevBuf<int> bad;
    SLCS_TRY(bits.alloc(std::max(words, 1), s));
    SLCS_TRY(bad.alloc(1, s));
    SLCS_CUDA_TRY(cudaMemsetAsync(bits.p, 0, sizeof(unsigned) * std::max(words, 1), s));
    SLCS_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    if (size > 0) perm_check_kernel<<<std::min(4096, (size + 255) / 256), 256, 0, s>>>(d_perm, size, bits.p, bad.p);
    SLCS_CUDA_TRY(cudaGetLastError());
    int h = 0;
    SLCS_CUDA_TRY(cudaMemcpyAsync(&h, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SLCS_CUDA_TRY(cudaStreamSynchronize(s));
    if (bad_entries) *bad_entries = h;
    return h == 0 ? SLCS_OK : fail(SLCS_ERR_INTERNAL, std::to_string(h) + " entries are repeated or out of range");
}

extern "C" int slcs_check_permutation(const int32_t *perm, int size, int32_t *bad_entries) {
    if (size < 0 || (size > 0 && !perm)) return fail(SLCS_ERR_ARG, "bad arguments");
    Engine *E;
    SLCS_TRY(engine(&E));
    cudaStream_t s = E->stream;
    DevBuf<int32_t> d;
    SLCS_TRY(d.alloc(std::max(size, 1), s));
    if (size > 0) SLCS_CUDA_TRY(cudaMemcpyAsync(d.p, perm, sizeof(int32_t) * size, cudaMemcpyHostToDevice, s));
    return slcs_check_permutation_dev(d.p, size, bad_entries, s);
}
