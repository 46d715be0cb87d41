// comb_noalloc.cu -- an allocation-free entry point for single-pair combing on device memory.
//
// Some callers cannot allocate device memory on the engine's behalf: a host that hands the engine a fixed
// device-memory budget and owns every allocation itself, a plugin inside an application whose own
// allocator reserved the device memory up front, or a latency-bound serving loop that must never touch
// the allocator (cudaMalloc may synchronise the device and can fail under fragmentation).  For them,
// slcs_comb_u8_dev_noalloc runs the same wavefront combing as slcs_comb_u8_dev but keeps all of its
// scratch (band progress counters, work items, the pair descriptor, the dequeue counter and the error
// word) in one file-scope __device__ array of fixed size, kNoAllocScratchBytes below.  The caller still
// provides the inputs and all outputs, including col_to_row, which doubles as the band-to-band hand-off.
//
// Facts a caller must know:
//  * The array is a single static buffer per device that loads this library; it stays allocated until the
//    process exits.  Every call on a device shares it and it keeps the previous call's contents: the set-up
//    kernel clears everything that must start at zero.  Calls that overlap on the GPU (two streams, or two
//    host threads on one device) race on it: serialise them.
//  * The first call on a device resolves the array's device address (cudaGetSymbolAddress) with that
//    device current and caches it; make that first call before any stream capture.
//  * The cached address belongs to the device's current context: after cudaDeviceReset (or any teardown of the
//    primary context) the process must not call this entry point again.
//  * Limits: at most kNoAllocMaxBands bands of 32*R rows (R = 32 for long strings), i.e. m <= 8,388,608
//    rows; m + n < 2^30.  Larger inputs are rejected with SLCS_ERR_TOO_LARGE.  The strings keep the
//    orientation given (rows = a).
//  * Speed: above about 1.8 million rows (m / 1024 bands beyond the ~1776 warps resident on a B200) the later
//    bands start only when a warp has finished a whole band, which roughly doubles the time; pass the shorter
//    string as a, or use slcs_comb_u8_dev, for such pairs.
#include <mutex>

#include "slcs_internal.cuh"

namespace slcs {
namespace {

constexpr int kNoAllocMaxBands = 8192;

struct NoAllocScratch {
    int err;
    int next;
    int pad[2];
    CombPair pair;
    CombItem items[kNoAllocMaxBands];
    int32_t progress[kNoAllocMaxBands];
};

constexpr size_t kNoAllocScratchBytes = sizeof(NoAllocScratch);

// The scratch.  In host code this name is only a host-side stand-in for the symbol, never a device address.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

struct DeviceSetup {
    NoAllocScratch *scratch = nullptr;   // device address of g_noalloc_scratch on this device
    int num_sms = 0;
    int resident_warps = 0;
    bool ready = false;
};
std::mutex g_setup_mu;
DeviceSetup g_setup[64];

// Writes the pair descriptor and the band items, clears counters, progress and the score.
__global__ void noalloc_setup_kernel(NoAllocScratch *sc, const uint8_t *a, int m, const uint8_t *b, int n,
                                     int32_t *c2r, int32_t *score, int R, int bands) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) {
        sc->err = kDevErrNone;
        sc->next = 0;
        sc->pair = CombPair{a, b, c2r, sc->progress, score, m, n};
        if (score) *score = 0;
    }
    for (int k = tid; k < bands; k += gridDim.x * blockDim.x) {
        sc->items[k] = CombItem{0, k, k * 32 * R, R, k == bands - 1 ? 1 : 0};
        sc->progress[k] = 0;
    }
}

__global__ void noalloc_identity_kernel(int32_t *r2c, int32_t *c2r, int32_t *score, int size) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < size) {
        r2c[i] = i;
        c2r[i] = i;
    }
    if (i == 0 && score) *score = 0;
}

int setup_device(DeviceSetup **out) {
    int dev = 0;
    SLCS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(SLCS_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    DeviceSetup &S = g_setup[dev];
    if (!S.ready) {
        int major = 0;
        SLCS_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
        if (major < 10) return fail(SLCS_ERR_NO_DEVICE, "libslcs is built for sm_100a (B200)");
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr) {
            cudaGetLastError();
            return fail(SLCS_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") +
                                           cudaGetErrorString(e));
        }
        SLCS_CUDA_TRY(cudaDeviceGetAttribute(&S.num_sms, cudaDevAttrMultiProcessorCount, dev));
        S.scratch = static_cast<NoAllocScratch *>(ptr);
        S.resident_warps = comb_resident_warps_sm(S.num_sms);
        S.ready = true;
    }
    *out = &S;
    return SLCS_OK;
}

int rows_per_lane(int rows) {
    int R = 1;
    while (R < 32 && 32 * 64 * R * 2 <= rows) R *= 2;
    return R;
}

}  // namespace
}  // namespace slcs

using namespace slcs;

extern "C" int slcs_comb_u8_dev_noalloc(const uint8_t *d_a, int m, const uint8_t *d_b, int n, int32_t *d_row_to_col,
                                        int32_t *d_col_to_row, int32_t *d_score, void *stream) {
    if (m < 0 || n < 0) return fail(SLCS_ERR_ARG, "negative length");
    if ((m > 0 && !d_a) || (n > 0 && !d_b) || (m + n > 0 && (!d_row_to_col || !d_col_to_row)))
        return fail(SLCS_ERR_ARG, "NULL buffer (row_to_col and col_to_row are both required)");
    if ((long long) m + n >= (1ll << 30)) return fail(SLCS_ERR_TOO_LARGE, "m + n must be below 2^30");
    const int R = rows_per_lane(m);
    const long long bands = (m + 32ll * R - 1) / (32ll * R);
    if (bands > kNoAllocMaxBands)
        return fail(SLCS_ERR_TOO_LARGE, "slcs_comb_u8_dev_noalloc: m = " + std::to_string(m) +
                                            " needs " + std::to_string(bands) + " bands; the static scratch holds " +
                                            std::to_string(kNoAllocMaxBands) + " (m <= 8388608)");
    DeviceSetup *S;
    SLCS_TRY(setup_device(&S));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (m + n == 0) {   // no strands: only the score (0), as the regular entry point writes it
        if (d_score) {
            SLCS_CUDA_TRY(cudaMemsetAsync(d_score, 0, sizeof(int32_t), s));
            SLCS_CUDA_TRY(cudaStreamSynchronize(s));
        }
        return SLCS_OK;
    }
    if (m == 0 || n == 0) {   // the identity braid needs no scratch
        noalloc_identity_kernel<<<(m + n + 255) / 256, 256, 0, s>>>(d_row_to_col, d_col_to_row, d_score, m + n);
        SLCS_CUDA_TRY(cudaGetLastError());
        SLCS_CUDA_TRY(cudaStreamSynchronize(s));
        return SLCS_OK;
    }
    NoAllocScratch *sc = S->scratch;
    noalloc_setup_kernel<<<((int) bands + 255) / 256, 256, 0, s>>>(sc, d_a, m, d_b, n, d_col_to_row, d_score, R,
                                                                  (int) bands);
    SLCS_CUDA_TRY(cudaGetLastError());
    SLCS_TRY(launch_comb<uint8_t>(&sc->pair, sc->items, (int) bands, &sc->next, &sc->err, S->resident_warps, s));
    SLCS_TRY(launch_invert(d_col_to_row, m + n, d_row_to_col, false, &sc->err, s));
    return check_dev_err(&sc->err, s);
}
