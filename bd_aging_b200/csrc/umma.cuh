// umma.cuh -- BF16 GEMM on the sm_100a tensor cores (tcgen05 / UMMA) for the
// surrogate network's weight gradients: C[M][N] = sum_k A[M][k] B[N][k] (both
// operands K-major, BF16; FP32 accumulation in tensor memory), written
// transposed as FP32 split-K partials.  The PTX helpers here are shared with
// the fused forward / input-gradient kernel (mlp_chain.cuh).
//
// One CTA (8 warps) computes a 128 x 64 tile over a K range of at most 256:
//   * thread 0 issues every TMA load of the range at once (64-wide K chunks,
//     128-byte swizzle, one mbarrier per chunk, no multicast);
//   * one lane of warp 1 issues tcgen05.mma (M=128, N=64, K=16) per 16-wide
//     slice as each chunk lands, then tcgen05.commit to the "done" barrier;
//   * all eight warps read accumulator rows with tcgen05.ld (warp w: lanes
//     32 (w % 4) .. + 31, the column half w / 4) and store them.
// Every mbarrier wait is bounded: on expiry the CTA records an error flag,
// waits (bounded) for its own copies, frees its tensor memory and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace bd {
namespace umma {

constexpr int kBM = 128, kBN = 64, kBK = 64;  // kBK bf16 = one 128-byte swizzle row
constexpr int kMaxChunks = 4;                  // K range per CTA <= 256
constexpr int kThreads = 256;  // 8 warps: warp w reads TMEM lanes 32 (w % 4), columns kBN / 2 (w / 4)
constexpr int kStageA = kBM * kBK * 2;         // 16 KB per A tile
constexpr int kStageB = kBN * kBK * 2;         // 8 KB per B tile
constexpr int kSmemBytes = kMaxChunks * (kStageA + kStageB) + 1024 /* align */ + 256 /* barriers */;
static_assert(kBN % 64 == 0, "two column halves of whole 32-column groups");
constexpr long kSpinLimit = 1L << 20;

struct GemmArgs {
    int M, N, K;          // logical sizes (rows of A, rows of B, reduction)
    int k_split;          // K range per blockIdx.z (multiple of 64, <= 256)
    // split-K partials stored transposed, [splits][N][M]: the epilogue thread
    // owns one row m, so consecutive lanes touch consecutive addresses
    float *out_f32;
    unsigned *err;
};

// ----------------------------------------------------------------- PTX
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false (and the error flag set) when the barrier never flips
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned *err, unsigned code) {
    for (long i = 0; i < kSpinLimit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(err, code);
    return false;
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), leading offset 1 (unused for swizzled K-major),
// descriptor version 1 (bits 46-47), layout type 2 = SWIZZLE_128B (bits 61-63)
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// instruction descriptor, kind::f16: D f32 (bits 4-5 = 1), A and B bf16
// (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    tmem_ld16(taddr, v);
    tmem_ld16(taddr + 16, v + 16);
}

// ----------------------------------------------------------------- math
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678f)) + z * 0.39894228f * expf(-0.5f * z * z);
}

// ----------------------------------------------------------------- kernel
__global__ void __launch_bounds__(kThreads, 1)
    k_umma_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem =
        reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char *sA = smem;                          // [kMaxChunks][kStageA]
    unsigned char *sB = smem + kMaxChunks * kStageA;   // [kMaxChunks][kStageB]
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + kMaxChunks * (kStageA + kStageB));
    uint64_t *done = full + kMaxChunks;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
    const int kb = blockIdx.z * g.k_split;
    const int nk = max(0, min(kMaxChunks, (min(g.k_split, g.K - kb) + kBK - 1) / kBK));

    if (threadIdx.x == 0) {
        for (int c = 0; c < kMaxChunks; c++) mbar_init(&full[c], 1);
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (threadIdx.x == 0) {
        for (int c = 0; c < nk; c++) {
            mbar_expect_tx(&full[c], kStageA + kStageB);
            tma_load_2d(sA + c * kStageA, &tmA, &full[c], kb + c * kBK, m0);
            tma_load_2d(sB + c * kStageB, &tmB, &full[c], kb + c * kBK, n0);
        }
    }
    if (warp == 1 && lane == 0) {
        bool ok = true;
        for (int c = 0; c < nk && ok; c++) {
            ok = mbar_wait(&full[c], 0, g.err, 1u);
            if (!ok) break;
            tc_fence_after();
            const uint64_t ad = smem_desc_sw128(smem_u32(sA + c * kStageA));
            const uint64_t bd = smem_desc_sw128(smem_u32(sB + c * kStageB));
#pragma unroll
            for (int kk = 0; kk < kBK / 16; kk++)  // 16 bf16 = 32 bytes = 2 descriptor units
                umma_bf16(tmem, ad + 2 * kk, bd + 2 * kk, (c | kk) ? 1u : 0u);
        }
        umma_commit(done);  // arrives once every issued MMA has completed
    }
    __syncwarp();
    const bool have = mbar_wait(done, 0, g.err, 2u) && nk > 0;
    tc_fence_after();

    const int quad = warp & 3, half = warp >> 2;
    const int m = m0 + quad * 32 + lane;
    if (have) {
#pragma unroll 1
        for (int cc = half * (kBN / 64); cc < (half + 1) * (kBN / 64); cc++) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(cc * 32), v);
            const int nb = n0 + cc * 32;
            // lane = row m: outputs indexed [n][m] are coalesced across lanes
#pragma unroll
            for (int j = 0; j < 32; j++) {
                const int n = nb + j;
                if (m < g.M && n < g.N) g.out_f32[(size_t)blockIdx.z * g.M * g.N + (size_t)n * g.M + m] = v[j];
            }
        }
    } else if (threadIdx.x == 0) {
        // bounded wait for this CTA's own copies before its memory goes away
        for (int c = 0; c < nk; c++) mbar_wait(&full[c], 0, g.err, 4u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kBN));
    }
}

}  // namespace umma
}  // namespace bd
