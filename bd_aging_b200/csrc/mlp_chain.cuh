// mlp_chain.cuh -- the surrogate's forward pass and its input-gradient chain
// in one kernel, on the sm_100a tensor cores (tcgen05, BF16 in, FP32 in
// tensor memory).
//
// Rows of the batch never mix in these GEMMs, so a cluster of four CTAs
// takes a block of 128 rows through every layer without leaving the chip:
//   forward   Z_l = H_{l-1} W_l^T + b_l, H_l = gelu(Z_l)        (l = 0 .. L-1)
//   backward  dZ_{l-1} = (dZ_l W_l) * gelu'(Z_{l-1})             (l = L-1 .. 1)
// Each GEMM is M = 128 rows by N <= 256 columns over K <= 256; CTA q of the
// cluster computes columns [q N / 4, (q + 1) N / 4).  The A operand (the
// block's activations or gradients, [128][K]) sits in every CTA's shared
// memory in the 128-byte-swizzled K-major layout the MMA descriptor reads,
// double-buffered; the B operand (the CTA's N / 4 rows of W_l for the forward
// GEMMs, of W_l^T for the backward ones) comes by TMA (no multicast); the
// accumulator is 128 lanes x N / 4 columns of tensor memory.  The epilogue of
// each GEMM writes its slice of the next GEMM's A operand into the other
// buffer of all four CTAs, and the transposed copies the weight-gradient
// GEMMs need (H_l^T, dZ_l^T, both [N][M], lane = row so stores coalesce) plus
// Z_l to global memory.  When N = 256 a CTA's slice is one whole 16 KB chunk
// of the A operand: the epilogue writes it locally and one thread copies it
// to the three peers with shared-to-shared bulk copies that complete on the
// peer's mbarrier.  A peer's buffer is free by then: the copy follows this
// CTA's MMA, which needed the peer's slice of the current operand, which the
// peer sent after its own MMA of the previous GEMM had read the buffer.
// Other shapes use per-thread distributed shared-memory stores and one
// cluster barrier per GEMM.  The weight-gradient GEMMs reduce over the batch
// and stay separate launches.  The next GEMM's weights are loaded while the
// epilogue of the current one runs.  Every mbarrier wait is bounded: on
// expiry the CTA records an error flag and skips its remaining MMAs and
// epilogues while still passing every barrier of the cluster, then waits
// (bounded) for its own copies and frees its tensor memory.
#pragma once
#include "umma.cuh"

namespace bd {
namespace umma {

constexpr int kChainThreads = 256;          // 8 warps: warp w reads TMEM lanes 32 (w % 4), column half w / 4
constexpr int kChainCluster = 4;            // CTAs per 128-row block, each a quarter of every GEMM's columns
constexpr int kChainMaxLayers = 9;
constexpr int kChainMaxDim = 256;           // K and N of every GEMM (N a multiple of 64)
constexpr int kChainMaxNc = kChainMaxDim / kChainCluster;     // columns per CTA
constexpr int kChainA = kBM * kChainMaxDim * 2;               // one A buffer: 4 chunks of [128][64] BF16
constexpr int kChainB = kChainMaxNc * kChainMaxDim * 2;       // B operand: up to 4 chunks of [64][64] BF16
constexpr int kChainSmem = 2 * kChainA + kChainB + 1024 /* align */ + 64 /* barriers, TMEM slot */;
static_assert(kChainSmem <= 227 * 1024, "shared memory of one CTA");

struct ChainLayer {
    int K, N;                   // padded sizes of W_l [N][K]: multiples of 64, at most 256
    const float *bias;          // [N]
    float *z;                   // hidden layer: Z_l [N][M]; output layer: Y [N][M]
    __nv_bfloat16 *ht;          // hidden layer: H_l^T [N][M] (the next layer's input, transposed)
    __nv_bfloat16 *dzt;         // dZ_l^T [N][M] (training)
};

struct ChainArgs {
    int L;                      // weight layers
    int M;                      // batch rows (a multiple of 128)
    int backward;               // 1: training (loss gradient and the input-gradient chain)
    ChainLayer lay[kChainMaxLayers];
    const float *target;        // training: targets [N_out][M]
    const float *tweight;       // [N_out] loss weight per output
    int n_valid;                // live outputs
    float grad_scale;           // d loss / d y = grad_scale * w (y - t)
    float *loss_part;           // [4 M / 128]: sum w (y - t)^2 per CTA
    unsigned *err;
};

struct ChainMaps {
    CUtensorMap x;                          // X0 [M][K_0], box 64 x 128
    CUtensorMap w[kChainMaxLayers];         // W_l [N_l][K_l], box 64 x N_l / 4
    CUtensorMap wt[kChainMaxLayers];        // W_l^T [K_l][N_l], box 64 x K_l / 4
};

// instruction descriptor of kind::f16 for M = 128 and N columns (BF16 in,
// FP32 accumulate, both operands K-major), as kIdesc
__device__ __forceinline__ uint32_t chain_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16_n(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// tcgen05.ld of 8 columns without the wait (several in flight, then
// tmem_wait_ld once)
__device__ __forceinline__ void tmem_ld8_issue(uint32_t taddr, uint32_t *r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset in an A buffer of row r, columns n0 .. n0 + 7 (n0 a multiple of
// 8): chunk n0 / 64 of [128][64] (16 KB), row r at 128 bytes, its 16-byte
// unit (n0 % 64) / 8 at position unit ^ (r % 8) -- the 128-byte swizzle TMA
// applies to a box in a 1024-byte-aligned buffer.
__device__ __forceinline__ uint32_t chain_a_offset(int r, int n0) {
    const int unit = ((n0 & 63) >> 3) ^ (r & 7);
    return (uint32_t)((n0 >> 6) * (kBM * 128) + r * 128 + unit * 16);
}
// Eight values as BF16 into the A buffer at shared-memory address `a` of every
// CTA of the cluster (the same offset in each).
__device__ __forceinline__ void chain_put8_cluster(uint32_t a, const float *v) {
    __nv_bfloat162 p0 = __floats2bfloat162_rn(v[0], v[1]), p1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(v[4], v[5]), p3 = __floats2bfloat162_rn(v[6], v[7]);
    const uint32_t q0 = *reinterpret_cast<uint32_t *>(&p0), q1 = *reinterpret_cast<uint32_t *>(&p1);
    const uint32_t q2 = *reinterpret_cast<uint32_t *>(&p2), q3 = *reinterpret_cast<uint32_t *>(&p3);
#pragma unroll
    for (int p = 0; p < kChainCluster; p++) {
        uint32_t ra;
        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(a), "r"(p));
        asm volatile("st.shared::cluster.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(ra), "r"(q0), "r"(q1), "r"(q2), "r"(q3)
                     : "memory");
    }
}
// Eight values as BF16 into this CTA's A buffer (`a` points at their unit).
__device__ __forceinline__ void chain_put8_local(unsigned char *a, const float *v) {
    __nv_bfloat162 p0 = __floats2bfloat162_rn(v[0], v[1]), p1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(v[4], v[5]), p3 = __floats2bfloat162_rn(v[6], v[7]);
    uint4 q;
    q.x = *reinterpret_cast<uint32_t *>(&p0);
    q.y = *reinterpret_cast<uint32_t *>(&p1);
    q.z = *reinterpret_cast<uint32_t *>(&p2);
    q.w = *reinterpret_cast<uint32_t *>(&p3);
    *reinterpret_cast<uint4 *>(a) = q;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// GEMM gi of the chain: forward layer gi for gi < L, then backward layer
// 2L - 1 - gi (L - 1 down to 1).  GEMM sizes: forward K_l x N_l with B = W_l;
// backward N_l x K_l (reduction over the layer's outputs) with B = W_l^T.
struct ChainStep {
    bool fwd;
    int l, K, N;
};
__device__ __forceinline__ ChainStep chain_step(const ChainArgs &g, int gi) {
    ChainStep c;
    c.fwd = gi < g.L;
    c.l = c.fwd ? gi : 2 * g.L - 1 - gi;
    c.K = c.fwd ? g.lay[c.l].K : g.lay[c.l].N;
    c.N = c.fwd ? g.lay[c.l].N : g.lay[c.l].K;
    return c;
}

__global__ void __launch_bounds__(kChainThreads, 1)
    k_mlp_chain(const __grid_constant__ ChainMaps maps, const __grid_constant__ ChainArgs g) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem =
        reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char *sA0 = smem;               // A buffers [2][K / 64][128][64] BF16, swizzled
    unsigned char *sB = smem + 2 * kChainA;  // [K / 64][N / 4][64] BF16, swizzled
    uint64_t *bar_x = reinterpret_cast<uint64_t *>(smem + 2 * kChainA + kChainB);  // X0 landed
    uint64_t *bar_b = bar_x + 1;             // B of the current GEMM landed (one phase per GEMM)
    uint64_t *bar_d = bar_x + 2;             // MMAs of the current GEMM completed (one phase per GEMM)
    uint64_t *bar_a = bar_x + 3;             // [2]: the peers' chunks of A buffer b landed (bulk copies)
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar_x + 5);
    __shared__ float red[kChainThreads / 32];
    __shared__ float s_bias[kChainMaxNc], s_tw[kChainMaxNc];  // per-column epilogue inputs of the GEMM

    unsigned q;  // rank in the cluster: the quarter of every GEMM's columns this CTA computes
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(q));
    const int blk = blockIdx.x / kChainCluster;  // the cluster's block of 128 rows
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quad = warp & 3, half = warp >> 2;
    const int r = quad * 32 + lane;  // this thread's row of the block in every epilogue
    const int m = blk * kBM + r;     // ... and of the batch
    const bool mrow = m < g.M;
    const int nG = g.L + (g.backward ? g.L - 1 : 0);

    if (tid == 0) {
        mbar_init(bar_x, 1);
        mbar_init(bar_b, 1);
        mbar_init(bar_d, 1);
        mbar_init(&bar_a[0], 1);
        mbar_init(&bar_a[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kChainMaxNc));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    cluster_sync_all();  // every CTA of the cluster is set up before shared memory crosses CTAs
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // thread 0: this CTA's rows of the B operand of GEMM gi, one box per
    // 64-wide K chunk
    int nb = 0;  // B loads issued (thread 0)
    auto load_b = [&](int gi) {
        nb++;
        const ChainStep c = chain_step(g, gi);
        const int nc = c.N / kChainCluster;
        const CUtensorMap *map = c.fwd ? &maps.w[c.l] : &maps.wt[c.l];
        const int kc = c.K / kBK;
        mbar_expect_tx(bar_b, (uint32_t)(kc * nc * 128));
        for (int k = 0; k < kc; k++) tma_load_2d(sB + k * nc * 128, map, bar_b, k * kBK, (int)q * nc);
    };
    if (tid == 0) {
        const int kc0 = g.lay[0].K / kBK;
        mbar_expect_tx(bar_x, (uint32_t)(kc0 * kBM * 128));
        for (int k = 0; k < kc0; k++) tma_load_2d(sA0 + k * kBM * 128, &maps.x, bar_x, k * kBK, blk * kBM);
        load_b(0);
    }

    bool failed = false;   // uniform over the CTA
    bool bulk_in = false;  // this GEMM's A operand came from the peers by bulk copy
    int na0 = 0, na1 = 0;  // bulk-filled uses of A buffers 0 and 1 (bar_a phases)
    float loss = 0.f;
    for (int gi = 0; gi < nG; gi++) {
        const ChainStep c = chain_step(g, gi);
        const int nc = c.N / kChainCluster;
        const uint32_t ph = (uint32_t)(gi & 1);
        unsigned char *sA = sA0 + (gi & 1) * kChainA;  // this GEMM's A operand
        const uint32_t a_next = smem_u32(sA0 + ((gi + 1) & 1) * kChainA);
        bool issued = true;
        if (warp == 1 && lane == 0) {  // one thread issues the MMAs of the GEMM
            bool go = !failed && (gi > 0 || mbar_wait(bar_x, 0, g.err, 1u));
            go = go && mbar_wait(bar_b, ph, g.err, 1u);
            go = go && (!bulk_in || mbar_wait(&bar_a[gi & 1], (uint32_t)(((gi & 1) ? na1 : na0) & 1), g.err, 3u));
            issued = go;
            if (go) {
                tc_fence_after();
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the A operand came from generic stores
                const uint32_t idesc = chain_idesc(nc);
                for (int k = 0; k < c.K / kBK; k++) {
                    const uint64_t ad = smem_desc_sw128(smem_u32(sA + k * kBM * 128));
                    const uint64_t bd = smem_desc_sw128(smem_u32(sB + k * nc * 128));
#pragma unroll
                    for (int kk = 0; kk < kBK / 16; kk++)  // 16 BF16 = 32 bytes = 2 descriptor units
                        umma_bf16_n(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (k | kk) ? 1u : 0u);
                }
            }
            umma_commit(bar_d);  // arrives when every MMA issued so far has completed
        }
        __syncwarp();
        if (bulk_in) {
            if (gi & 1) na1++;
            else na0++;
        }
        // the epilogue's inputs that do not depend on the MMAs load under them:
        // per-column bias and loss weight to shared memory, per-element Z_{l-1}
        // (backward) or targets (output layer) to registers
        const bool out_layer = c.fwd && c.l == g.L - 1;
        const int cw = nc / 2, c0 = half * cw, nbase = (int)q * nc + c0;  // this warp's columns
        if (tid < nc) {
            s_bias[tid] = c.fwd ? g.lay[c.l].bias[(int)q * nc + tid] : 0.f;
            s_tw[tid] = out_layer && g.backward ? g.tweight[(int)q * nc + tid] : 0.f;
        }
        float pre[32];
        {
            const float *src = !c.fwd ? g.lay[c.l - 1].z : (out_layer && g.backward ? g.target : nullptr);
#pragma unroll
            for (int j = 0; j < 32; j++)
                pre[j] = (src && j < cw && mrow) ? src[(size_t)(nbase + j) * g.M + m] : 0.f;
        }
        const bool done = mbar_wait(bar_d, ph, g.err, 2u) && issued;  // the commit arrives even when nothing was issued
        tc_fence_after();
        // this CTA's earlier bulk copies have read their source (the A buffer
        // this epilogue writes was the source two GEMMs ago)
        if (tid == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        const bool ok = __syncthreads_and(done) != 0;
        failed = failed || !ok;
        // the B buffer is free: the next GEMM's weights load under this epilogue
        if (tid == 0 && gi + 1 < nG && !failed) load_b(gi + 1);
        const bool next_a = gi + 1 < nG;  // a GEMM follows that reads the A operand written here
        // a CTA's columns of an N = 256 GEMM are one whole 16 KB chunk of the next
        // A operand: written locally, then bulk-copied to the three peers;
        // otherwise every thread stores its values into all four CTAs
        const bool bulk_next = next_a && nc == kBK;
        const uint32_t trow = tmem + ((uint32_t)(quad * 32) << 16);
        if (ok) {  // warp (quad, half): rows 32 quad .. + 31 (lane = row), half of the CTA's columns
            float v[32];
            {
                uint32_t raw[32];
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (u * 8 < cw) tmem_ld8_issue(trow + (uint32_t)(c0 + 8 * u), raw + 8 * u);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 32; j++) v[j] = __uint_as_float(raw[j]);
            }
            if (c.fwd && !out_layer) {  // hidden layer: bias, GELU
                const ChainLayer &Ly = g.lay[c.l];
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    if (j < cw) {
                        const int n = nbase + j;
                        const float zv = v[j] + s_bias[c0 + j];
                        const float h = gelu(zv);
                        if (mrow) {
                            Ly.z[(size_t)n * g.M + m] = zv;
                            Ly.ht[(size_t)n * g.M + m] = __float2bfloat16_rn(h);
                        }
                        v[j] = h;
                    }
                }
            } else if (c.fwd) {  // output layer: y and, in training, the loss gradient
                const ChainLayer &Ly = g.lay[c.l];
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    if (j < cw) {
                        const int n = nbase + j;
                        const float y = v[j] + s_bias[c0 + j];
                        float gr = 0.f;
                        if (mrow) {
                            Ly.z[(size_t)n * g.M + m] = y;
                            if (g.backward) {
                                if (n < g.n_valid) {
                                    const float e = y - pre[j];
                                    loss += s_tw[c0 + j] * e * e;
                                    gr = g.grad_scale * s_tw[c0 + j] * e;
                                }
                                Ly.dzt[(size_t)n * g.M + m] = __float2bfloat16_rn(gr);
                            }
                        }
                        v[j] = gr;
                    }
                }
            } else {  // backward: dZ_{l-1} = (dZ_l W_l) * gelu'(Z_{l-1})
                const ChainLayer &Lp = g.lay[c.l - 1];
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    if (j < cw) {
                        const int n = nbase + j;
                        float d = 0.f;
                        if (mrow) {
                            d = v[j] * gelu_grad(pre[j]);
                            Lp.dzt[(size_t)n * g.M + m] = __float2bfloat16_rn(d);
                        }
                        v[j] = d;
                    }
                }
            }
            if (next_a)
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (u * 8 < cw) {
                        if (bulk_next) chain_put8_local(sA0 + ((gi + 1) & 1) * kChainA + chain_a_offset(r, nbase + 8 * u), v + 8 * u);
                        else chain_put8_cluster(a_next + chain_a_offset(r, nbase + 8 * u), v + 8 * u);
                    }
        }
        // publish the next A operand: the chunk by bulk copy under the peers'
        // mbarriers, or the stores by a cluster barrier (which also frees this one)
        if (bulk_next) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        else asm volatile("fence.proxy.async.shared::cluster;" ::: "memory");
        tc_fence_before();
        if (bulk_next) __syncthreads();
        else cluster_sync_all();
        tc_fence_after();
        if (bulk_next && tid == 0 && !failed) {
            uint64_t *ba = &bar_a[(gi + 1) & 1];
            mbar_expect_tx(ba, (uint32_t)((kChainCluster - 1) * kBM * 128));  // the peers' chunks
            const uint32_t src = a_next + q * (uint32_t)(kBM * 128);
            for (int p = 1; p < kChainCluster; p++) {
                const uint32_t dq = (q + (uint32_t)p) % kChainCluster;
                uint32_t dst, mb;
                asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(dst) : "r"(src), "r"(dq));
                asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(mb) : "r"(smem_u32(ba)), "r"(dq));
                asm volatile(
                    "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                    "r"(src), "r"((uint32_t)(kBM * 128)), "r"(mb)
                    : "memory");
            }
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
        bulk_in = bulk_next;
    }
    if (tid == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");  // sources read
    cluster_sync_all();  // no shared-memory traffic between the CTAs is left when any of them exits
    if (failed && tid == 0) {  // bounded wait for this CTA's own copies before its memory goes away
        mbar_wait(bar_x, 0, g.err, 4u);
        if (nb > 0) mbar_wait(bar_b, (uint32_t)((nb - 1) & 1), g.err, 4u);
    }
    if (g.backward && g.loss_part) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, off);
        if (lane == 0) red[warp] = loss;
    }
    tc_fence_before();
    __syncthreads();
    if (g.backward && g.loss_part && tid == 0)
        g.loss_part[blockIdx.x] = ((red[0] + red[1]) + (red[2] + red[3])) + ((red[4] + red[5]) + (red[6] + red[7]));
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kChainMaxNc));
    }
}

}  // namespace umma
}  // namespace bd
