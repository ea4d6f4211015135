// noalloc.cu -- F_s(q) reduction that allocates nothing on the device.
//
// bd_fself_isotropic (mirror.cu) keeps its FP64 partial sums in a per-device
// workspace that is cudaMalloc'd on first use.  Some callers cannot allocate
// device memory at the moment they sample F_s: real-time sampling loops whose
// rules forbid allocation after start-up, and host programs whose device
// memory is fully reserved up front by another allocator (a pool that owns
// the GPU), where a late cudaMalloc fails or fragments the pool.  For them,
// bd_fself_isotropic_noalloc does the same reduction with its scratch in the
// fixed array below.
//
// Scratch: kFselfScratchBlocks FP64 per-block partial sums (32 KB), held by
// every GPU that loads this library until process exit.  One block covers 256
// particles, so ngrain is limited to kFselfScratchBlocks * 256 = 1,048,576;
// larger calls are rejected with BD_ERR_ARG before any work is queued.
// The partial sums are overwritten by every call (nothing accumulates into
// the array, so nothing needs clearing).  All calls on a GPU share the one
// array: calls that overlap on the GPU (two streams, or two host threads)
// race on it, so callers must serialise them.
//
// Set-up: host code cannot use the array's name as a device address, so the
// first call on each device (with that device current) looks the address up
// with cudaGetSymbolAddress and caches it for that device's context; a device
// reset, which destroys the context, makes the next call look it up again.
// Make that first call on a device before a global-mode stream capture
// starts anywhere in the process (the lookup is a runtime call such a
// capture refuses).  The entry point synchronises its stream to read the sum
// back, so it cannot itself be captured.
#include <mutex>

#include "runtime.cuh"

namespace bd {

constexpr int kFselfScratchBlocks = 4096;
constexpr int kFselfThreads = 256;

static __device__ __align__(256) double g_fself_scratch[kFselfScratchBlocks];

// one FP64 partial per block: sum of sin(q|dr|)/(q|dr|) over its particles,
// per-particle float terms as in fself_isotropic (fself.cu:3-21)
__global__ void __launch_bounds__(kFselfThreads) k_fself_partials(const float *__restrict__ raw,
                                                                  const float *__restrict__ r0, int n, float q,
                                                                  double *part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s = 0.0;
    if (i < n) {
        const float dx = raw[3 * i] - r0[3 * i], dy = raw[3 * i + 1] - r0[3 * i + 1],
                    dz = raw[3 * i + 2] - r0[3 * i + 2];
        const float mag = __fsqrt_rn(dist2_rn(dx, dy, dz));
        s = (double)(sinf(q * mag) / (q * mag));
    }
    for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ double red[kFselfThreads / 32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kFselfThreads / 32; w++) t += red[w];
        part[blockIdx.x] = t;
    }
}

// sum of the partials in a fixed order; the result goes to part[0]
__global__ void k_fself_finish(double *part, int nblocks) {
    __shared__ double red[256];
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += part[b];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[0] = red[0];
}

// device address of g_fself_scratch, looked up once per device and context
static double *fself_scratch_address(int *rc) {
    static std::mutex mu;
    static double *addr[64] = {nullptr};
    static unsigned long long ctx_of[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        *rc = BD_ERR_CUDA;
        return nullptr;
    }
    const unsigned long long ctx = current_context_id();
    if (!ctx) {
        *rc = BD_ERR_CUDA;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev] || ctx_of[dev] != ctx) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_fself_scratch);
        if (e != cudaSuccess || !p) {
            *rc = BD_ERR_CUDA;
            return nullptr;
        }
        addr[dev] = (double *)p;
        ctx_of[dev] = ctx;
    }
    *rc = BD_OK;
    return addr[dev];
}

}  // namespace bd

using namespace bd;

extern "C" int bd_fself_isotropic_noalloc(const float *rr_raw, const float *rr0, int ngrain, float *fself_host,
                                          int sample_number, float qmax, void *stream) {
    if (ngrain <= 0 || !rr_raw || !rr0 || !fself_host || sample_number < 0) return BD_ERR_ARG;
    if (ngrain > kFselfScratchBlocks * kFselfThreads) return BD_ERR_ARG;  // beyond the fixed scratch
    int rc = BD_OK;
    double *part = fself_scratch_address(&rc);
    if (!part) return rc;
    cudaStream_t s = as_stream(stream);
    const int nblocks = div_up(ngrain, kFselfThreads);
    k_fself_partials<<<nblocks, kFselfThreads, 0, s>>>(rr_raw, rr0, ngrain, qmax, part);
    BD_LAUNCH_CHECK();
    k_fself_finish<<<1, 256, 0, s>>>(part, nblocks);
    BD_LAUNCH_CHECK();
    double sum = 0.0;
    BD_CUDA_TRY(cudaMemcpyAsync(&sum, part, sizeof(double), cudaMemcpyDeviceToHost, s));
    BD_CUDA_TRY(cudaStreamSynchronize(s));
    fself_host[sample_number] += (float)(sum / ngrain);
    return BD_OK;
}
