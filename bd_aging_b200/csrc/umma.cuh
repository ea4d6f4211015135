// umma.cuh -- BF16 GEMM on the sm_100a tensor cores (tcgen05 / UMMA) for the
// surrogate network: C[M][N] = sum_k A[M][k] B[N][k] (both operands
// K-major, BF16; FP32 accumulation in tensor memory) with fused epilogues.
//
// One CTA (8 warps) computes a 128 x 64 tile over a K range of at most 256:
//   * thread 0 issues every TMA load of the range at once (64-wide K chunks,
//     128-byte swizzle, one mbarrier per chunk, no multicast);
//   * one lane of warp 1 issues tcgen05.mma (M=128, N=64, K=16) per 16-wide
//     slice as each chunk lands, then tcgen05.commit to the "done" barrier;
//   * all eight warps read accumulator rows with tcgen05.ld (warp w: lanes
//     32 (w % 4) .. + 31, the column half w / 4) and apply the epilogue.
// The 64-wide N tile gives the small surrogate GEMMs (N = 256) four column
// tiles, so 128 CTAs share the epilogue work instead of 64.
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

enum Epilogue {
    kEpiF32 = 0,      // out_f32[z][n][m] = acc (split-K partials, transposed)
    kEpiFwdGelu = 1,  // z = acc + bias -> out_f32 [n][m]; gelu(z) -> out_bf [m][n] and out_bfT [n][m]
    kEpiFwdOut = 2,   // y = acc + bias -> out_f32 [n][m]; with a target [n][m]: loss gradient -> out_bf / out_bfT
    kEpiBwdGelu = 3,  // dz = acc * gelu'(zin [n][m]) -> out_bf / out_bfT
};

struct GemmArgs {
    int M, N, K;          // logical sizes (rows of A, rows of B, reduction)
    int k_split;          // K range per blockIdx.z (multiple of 64, <= 256)
    const float *bias;    // [N]
    // FP32 outputs and inputs are stored transposed ([N][M]): the epilogue
    // thread owns one row m, so consecutive lanes touch consecutive addresses
    float *out_f32;       // kEpiF32: [splits][N][M]; kEpiFwdGelu: z [N][M]; kEpiFwdOut: y [N][M]
    __nv_bfloat16 *out_bf;   // [M][N]
    __nv_bfloat16 *out_bfT;  // [N][M]
    const float *zin;     // kEpiBwdGelu: pre-activation [N][M]
    const float *target;  // kEpiFwdOut: [N][M] or null (inference)
    const float *tweight; // [N] loss weight per output
    int m_valid;          // rows that count in the loss
    int n_valid;          // outputs that count in the loss
    float grad_scale;     // d loss / d y = grad_scale * w (y - t)
    float *loss_part;     // [grid x * grid y] sum w (y - t)^2 per CTA
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
template <int EPI>
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
    __shared__ float red[kThreads / 32];
    __shared__ float stage[kThreads / 32][32][33];  // per-warp 32 x 32 tile, padded against bank conflicts

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
    const bool mrow = m < g.M;
    float loss = 0.f;
    float(*st)[33] = stage[warp];
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
                const bool ok = mrow && n < g.N;
                const size_t nm = (size_t)n * g.M + m;
                float r = 0.f;  // value of the row-major BF16 output
                if (EPI == kEpiF32) {
                    if (ok) g.out_f32[(size_t)blockIdx.z * g.M * g.N + nm] = v[j];
                } else if (EPI == kEpiFwdGelu) {
                    if (ok) {
                        const float z = v[j] + g.bias[n];
                        g.out_f32[nm] = z;
                        r = gelu(z);
                        g.out_bfT[nm] = __float2bfloat16_rn(r);
                    }
                } else if (EPI == kEpiFwdOut) {
                    if (ok) {
                        const float y = v[j] + g.bias[n];
                        g.out_f32[nm] = y;
                        if (g.target) {
                            if (n < g.n_valid && m < g.m_valid) {
                                const float e = y - g.target[nm];
                                loss += g.tweight[n] * e * e;
                                r = g.grad_scale * g.tweight[n] * e;
                            }
                            g.out_bfT[nm] = __float2bfloat16_rn(r);
                        }
                    }
                } else {  // kEpiBwdGelu
                    if (ok) {
                        r = v[j] * gelu_grad(g.zin[nm]);
                        g.out_bfT[nm] = __float2bfloat16_rn(r);
                    }
                }
                st[lane][j] = r;
            }
            // row-major BF16 output [m][n]: through the padded tile, one row per
            // instruction (lane = column)
            const bool rowmajor = EPI == kEpiFwdGelu || EPI == kEpiBwdGelu || (EPI == kEpiFwdOut && g.target);
            if (rowmajor) {
                __syncwarp();
                const int n = nb + lane;
#pragma unroll 4
                for (int rr = 0; rr < 32; rr++) {
                    const int mr = m0 + quad * 32 + rr;
                    if (mr < g.M && n < g.N) g.out_bf[(size_t)mr * g.N + n] = __float2bfloat16_rn(st[rr][lane]);
                }
                __syncwarp();
            }
        }
    } else if (threadIdx.x == 0) {
        // bounded wait for this CTA's own copies before its memory goes away
        for (int c = 0; c < nk; c++) mbar_wait(&full[c], 0, g.err, 4u);
    }
    if (EPI == kEpiFwdOut && g.target && g.loss_part) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, off);
        if (lane == 0) red[warp] = loss;
    }
    tc_fence_before();
    __syncthreads();
    if (EPI == kEpiFwdOut && g.target && g.loss_part && threadIdx.x == 0)
        g.loss_part[blockIdx.x * gridDim.y + blockIdx.y] =
            ((red[0] + red[1]) + (red[2] + red[3])) + ((red[4] + red[5]) + (red[6] + red[7]));
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kBN));
    }
}

}  // namespace umma
}  // namespace bd
