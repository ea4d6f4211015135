// surrogate.cu -- the learned surrogate: an MLP n_in -> width (GELU) x depth
// -> n_out trained and evaluated by hand-written tcgen05 BF16 GEMMs with FP32
// accumulation, Adam in FP32 on FP32 master weights.
//
// Per layer l (K_l inputs, N_l outputs, batch B) every GEMM has both
// operands K-major; the transposed copies it needs are written by the
// epilogue or the optimizer that produces them:
//   forward   Z_l  = H_{l-1} W_l^T + b_l        A = H_{l-1} [B][K_l], B = W_l  [N_l][K_l]
//   input     dH_{l-1} = dZ_l W_l               A = dZ_l    [B][N_l], B = W_l^T [K_l][N_l]
//   weights   dW_l = dZ_l^T H_{l-1}             A = dZ_l^T  [N_l][B], B = H_{l-1}^T [K_l][B]
// The forward and input-gradient GEMMs of a training step run in one launch
// of the fused kernel (mlp_chain.cuh), which keeps each 128-row block's
// activations and gradients in shared memory and writes H_l^T and dZ_l^T for
// the weight-gradient GEMMs (umma.cuh).  dW is split over the batch (256
// rows per CTA) into FP32 partials that the Adam kernel adds in a fixed
// order, so a training step is deterministic.
#include <cuda.h>
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "mlp_chain.cuh"
#include "runtime.cuh"
#include "umma.cuh"

namespace bd {
namespace {

using umma::GemmArgs;
using umma::kBK;
using umma::kBM;
using umma::kBN;

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 2-D BF16 row-major matrix [rows][cols] as a TMA map with a box of 64
// columns (128 bytes, 128-byte swizzle) by box_rows rows (kBM for A
// operands, kBN for B operands); out-of-range rows and columns read as zero.
int make_tmap(CUtensorMap *map, const void *ptr, int rows, int cols, int box_rows) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return BD_ERR_CUDA;
    if ((reinterpret_cast<uintptr_t>(ptr) & 15) || (cols % 8)) return BD_ERR_ARG;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? BD_OK : BD_ERR_ARG;
}

// dynamic shared memory above 48 KB for the GEMM and the fused kernel;
// called outside stream capture (create, direct GEMM)
int set_gemm_attrs() {
    BD_CUDA_TRY(cudaFuncSetAttribute(umma::k_umma_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     umma::kSmemBytes));
    BD_CUDA_TRY(cudaFuncSetAttribute(umma::k_mlp_chain, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     umma::kChainSmem));
    return BD_OK;
}

int launch_gemm(const CUtensorMap &a, const CUtensorMap &b, const GemmArgs &g, cudaStream_t st) {
    if (g.k_split % kBK || g.k_split > umma::kMaxChunks * kBK || g.k_split < kBK) return BD_ERR_ARG;
    dim3 grid(div_up(g.M, kBM), div_up(g.N, kBN), div_up(g.K, g.k_split));
    umma::k_umma_gemm<<<grid, umma::kThreads, umma::kSmemBytes, st>>>(a, b, g);
    BD_LAUNCH_CHECK();
    return BD_OK;
}

// ---------------------------------------------------------------- kernels
__global__ void k_sum_splits(const float *part, int splits, size_t n, float *out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.f;
    for (int k = 0; k < splits; k++) s += part[(size_t)k * n + i];
    out[i] = s;
}

// counter-based sample index (splitmix64 of seed, step, row)
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

// minibatch rows: x (FP32 [n_data][n_in]) -> X0 [B][k0] and X0^T [k0][B]
// (BF16, zero padded), targets -> T [n_out_pad][B].  A block takes 32 rows
// (lane = row), its warps split the columns: the transposed writes of a warp
// are 32 consecutive rows.
constexpr int kGatherRows = 32;
__global__ void k_gather(const float *x, const float *y, int n_data, int n_in, int n_out, int k0, int n_out_pad,
                         int B, const int *rows, const long long *step, unsigned long long seed, __nv_bfloat16 *X0,
                         __nv_bfloat16 *X0t, float *T) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int r = blockIdx.x * kGatherRows + lane;
    if (r >= B) return;
    int src;
    if (rows) {
        src = rows[r];
    } else {
        src = (int)(mix64(seed ^ mix64((unsigned long long)*step * 1315423911ULL + (unsigned long long)r)) %
                    (unsigned long long)n_data);
    }
    const bool valid = src >= 0 && src < n_data;
    for (int k = warp; k < k0; k += nw) {
        const float v = (valid && k < n_in) ? x[(size_t)src * n_in + k] : 0.f;
        const __nv_bfloat16 b = __float2bfloat16_rn(v);
        X0[(size_t)r * k0 + k] = b;
        X0t[(size_t)k * B + r] = b;
    }
    if (T)  // targets transposed [n_out_pad][B], as the loss epilogue reads them
        for (int k = warp; k < n_out_pad; k += nw)
            T[(size_t)k * B + r] = (valid && k < n_out) ? y[(size_t)src * n_out + k] : 0.f;
}

// Bias gradients of every layer in one launch: block `row` of the layer
// table sums dZ_l^T[n][:] over the batch (16-byte loads, a fixed order: the
// thread's strided slice, then the warp, then the block's warps).
struct BiasGradArgs {
    const __nv_bfloat16 *dzt[umma::kChainMaxLayers];  // [N_l][B]
    float *db[umma::kChainMaxLayers];                 // [N_l]
    int first[umma::kChainMaxLayers + 1];             // first block of each layer
    int L, B;                                         // B a multiple of 8
};
__global__ void k_bias_grads(const __grid_constant__ BiasGradArgs a) {
    const int row = blockIdx.x;
    int l = 0;
    while (l + 1 < a.L && row >= a.first[l + 1]) l++;
    const int n = row - a.first[l];
    const uint4 *src = reinterpret_cast<const uint4 *>(a.dzt[l] + (size_t)n * a.B);
    float sum = 0.f;
    for (int i = threadIdx.x; i < a.B / 8; i += blockDim.x) {
        const uint4 v = src[i];
        const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float2 f = __bfloat1622float2(h[j]);
            sum += f.x;
            sum += f.y;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off);
    __shared__ float red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        a.db[l][n] = t;
    }
}

struct AdamArgs {
    float lr, b1, b2, eps;
    const long long *step;  // number of updates so far (incremented by the caller's counter kernel)
};
// Every layer's weights and biases in one launch: element i of the table
// (weights of layer 0, 1, ... then biases of layer 0, 1, ...).  Weights are
// updated in [k][n] order (the gradient is the sum of the split partials,
// stored [splits][K][N] by the weight-gradient GEMM); the FP32 master weights
// and the moments are kept in that order too, so every FP32 access is
// coalesced.  Writes the BF16 copies W [N][K] and W^T [K][N].  The
// bias-correction denominators 1 - b^t are computed once per block.
struct AdamTable {
    float *w[umma::kChainMaxLayers], *wm[umma::kChainMaxLayers], *wv[umma::kChainMaxLayers];
    const float *part[umma::kChainMaxLayers];
    __nv_bfloat16 *wb[umma::kChainMaxLayers], *wbt[umma::kChainMaxLayers];
    float *b[umma::kChainMaxLayers], *bm[umma::kChainMaxLayers], *bv[umma::kChainMaxLayers];
    const float *db[umma::kChainMaxLayers];
    int N[umma::kChainMaxLayers], K[umma::kChainMaxLayers];
    int n_live[umma::kChainMaxLayers], k_live[umma::kChainMaxLayers];
    long long first_w[umma::kChainMaxLayers + 1];  // prefix of N K over the layers
    int first_b[umma::kChainMaxLayers + 1];        // prefix of N over the layers
    int L, splits;
};
__global__ void k_adam_all(const __grid_constant__ AdamTable t, AdamArgs a) {
    __shared__ float corr[2];
    if (threadIdx.x == 0) {
        const float tt = (float)(*a.step + 1);
        corr[0] = 1.f - powf(a.b1, tt);
        corr[1] = 1.f - powf(a.b2, tt);
    }
    __syncthreads();
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nw = t.first_w[t.L];
    if (e < nw) {
        int l = 0;
        while (l + 1 < t.L && e >= t.first_w[l + 1]) l++;
        const size_t i = (size_t)(e - t.first_w[l]);  // [k][n] order
        const int N = t.N[l], K = t.K[l];
        const int k = (int)(i / N), n = (int)(i % N);
        float gsum = 0.f;
        for (int s = 0; s < t.splits; s++) gsum += t.part[l][(size_t)s * N * K + i];
        float wv = t.w[l][i];
        if (n < t.n_live[l] && k < t.k_live[l]) {
            const float mm = a.b1 * t.wm[l][i] + (1.f - a.b1) * gsum;
            const float vv = a.b2 * t.wv[l][i] + (1.f - a.b2) * gsum * gsum;
            t.wm[l][i] = mm;
            t.wv[l][i] = vv;
            const float mh = mm / corr[0], vh = vv / corr[1];
            wv -= a.lr * mh / (sqrtf(vh) + a.eps);
            t.w[l][i] = wv;
        }
        const __nv_bfloat16 bv = __float2bfloat16_rn(wv);
        t.wb[l][(size_t)n * K + k] = bv;
        t.wbt[l][i] = bv;
        return;
    }
    const long long j = e - nw;
    if (j >= t.first_b[t.L]) return;
    int l = 0;
    while (l + 1 < t.L && j >= t.first_b[l + 1]) l++;
    const int n = (int)(j - t.first_b[l]);
    if (n >= t.n_live[l]) return;
    const float g = t.db[l][n];
    const float mm = a.b1 * t.bm[l][n] + (1.f - a.b1) * g;
    const float vv = a.b2 * t.bv[l][n] + (1.f - a.b2) * g * g;
    t.bm[l][n] = mm;
    t.bv[l][n] = vv;
    t.b[l][n] -= a.lr * (mm / corr[0]) / (sqrtf(vv / corr[1]) + a.eps);
}
__global__ void k_count(long long *step) { *step += 1; }
// BF16 copies W [N][K] and W^T [K][N] of the FP32 master weights (kept [K][N])
__global__ void k_to_bf16(const float *w, int N, int K, __nv_bfloat16 *wb, __nv_bfloat16 *wbt) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // [k][n] order
    if (i >= (size_t)N * K) return;
    const int k = (int)(i / N), n = (int)(i % N);
    const __nv_bfloat16 b = __float2bfloat16_rn(w[i]);
    wb[(size_t)n * K + k] = b;
    wbt[i] = b;
}

}  // namespace
}  // namespace bd

using namespace bd;

// ---------------------------------------------------------------- state
struct bd_surrogate {
    int n_in = 0, n_out = 0, width = 0, depth = 0, batch = 0;
    int L = 0;                        // weight layers = depth + 1
    std::vector<int> Kp, Np;          // padded input / output sizes per layer
    std::vector<int> Kl, Nl;          // live sizes
    cudaStream_t stream = nullptr;
    // parameters (FP32 master weights [K][N] and Adam moments in that order, biases), BF16 copies
    std::vector<float *> w, b, wm, wv, bm, bv;
    std::vector<__nv_bfloat16 *> wb, wbt;
    // activations (BF16 row-major and transposed), pre-activations FP32
    __nv_bfloat16 *x0 = nullptr;          // input X0 [B][K_0]
    std::vector<__nv_bfloat16 *> ht;      // ht[0] = X0^T; ht[l+1] = H_l^T, output of hidden layer l [N_l][B]
    std::vector<float *> z;               // z[l] pre-activation of layer l, transposed [N_l][B]
    std::vector<__nv_bfloat16 *> dzt;     // dZ_l^T, gradient w.r.t. z[l] [N_l][B]
    float *y = nullptr, *t = nullptr, *tw = nullptr;  // output [128][B], target [128][B] (transposed), weights
    float *part = nullptr;            // weight-gradient split partials [splits][K_l][N_l] per layer
    std::vector<float *> db;          // bias gradients
    float *loss_part = nullptr;
    long long *step = nullptr;
    unsigned *err = nullptr;
    float *data_x = nullptr, *data_y = nullptr;
    int n_data = 0;
    unsigned long long seed = 1;
    // TMA maps: X0 (box 128 rows), the weight-gradient GEMMs' operands dZ_l^T and
    // H_{l-1}^T, and W_l, W_l^T in boxes of a quarter of their rows (one CTA of a
    // fused kernel's cluster each)
    CUtensorMap tm_x;
    std::vector<CUtensorMap> tm_ht, tm_dzt, tm_w, tm_wt;
    cudaGraphExec_t graph = nullptr;
    float lr = 1e-3f;
    int loss_cells = 0;
    int ksplit = 256;
};

namespace {

void free_surrogate(bd_surrogate *s) {
    if (s->graph) cudaGraphExecDestroy(s->graph);
    auto F = [](void *p) {
        if (p) cudaFree(p);
    };
    for (auto *p : s->w) F(p);
    for (auto *p : s->b) F(p);
    for (auto *p : s->wm) F(p);
    for (auto *p : s->wv) F(p);
    for (auto *p : s->bm) F(p);
    for (auto *p : s->bv) F(p);
    for (auto *p : s->wb) F(p);
    for (auto *p : s->wbt) F(p);
    for (auto *p : s->ht) F(p);
    for (auto *p : s->z) F(p);
    for (auto *p : s->dzt) F(p);
    for (auto *p : s->db) F(p);
    F(s->x0); F(s->y); F(s->t); F(s->tw); F(s->part); F(s->loss_part); F(s->step); F(s->err); F(s->data_x);
    F(s->data_y);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int sg_status(bd_surrogate *s) {
    unsigned e = 0;
    BD_CUDA_TRY(cudaMemcpyAsync(&e, s->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
    BD_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return e ? BD_ERR_TIMEOUT : BD_OK;
}

GemmArgs base_args(bd_surrogate *s) {
    GemmArgs g;
    std::memset(&g, 0, sizeof(g));
    g.err = s->err;
    g.k_split = 256;
    return g;
}

// The forward pass of every 128-row block of the batch, and in training its
// loss gradient and input-gradient chain (dZ_l for every layer), in one
// launch of k_mlp_chain (a cluster of four CTAs per block).
int chain_launch(bd_surrogate *s, bool train) {
    umma::ChainMaps maps;
    std::memset(&maps, 0, sizeof(maps));
    maps.x = s->tm_x;
    umma::ChainArgs g;
    std::memset(&g, 0, sizeof(g));
    g.L = s->L;
    g.M = s->batch;
    g.backward = train ? 1 : 0;
    for (int l = 0; l < s->L; l++) {
        maps.w[l] = s->tm_w[l];
        maps.wt[l] = s->tm_wt[l];
        const bool hidden = l < s->L - 1;
        g.lay[l] = {s->Kp[l], s->Np[l], s->b[l], hidden ? s->z[l] : s->y, hidden ? s->ht[l + 1] : nullptr, s->dzt[l]};
    }
    if (train) {
        g.target = s->t;
        g.tweight = s->tw;
        g.n_valid = s->n_out;
        g.grad_scale = 2.0f / ((float)s->batch * (float)s->n_out);
        g.loss_part = s->loss_part;
    }
    g.err = s->err;
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((s->batch / kBM) * umma::kChainCluster);
    cfg.blockDim = dim3(umma::kChainThreads);
    cfg.dynamicSmemBytes = umma::kChainSmem;
    cfg.stream = s->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = umma::kChainCluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    BD_CUDA_TRY(cudaLaunchKernelEx(&cfg, umma::k_mlp_chain, maps, g));
    return BD_OK;
}

// forward of the whole network on the batch in h[0]; with a target also the
// loss gradient and every dZ_l (the fused kernel's input-gradient chain)
int forward(bd_surrogate *s, bool with_target) { return chain_launch(s, with_target); }

// gradients of every layer into the split partials and db; dW_l partials go
// to part + offset(l)
size_t part_offset(const bd_surrogate *s, int l) {
    size_t off = 0;
    for (int i = 0; i < l; i++) off += (size_t)(s->batch / s->ksplit) * s->Np[i] * s->Kp[i];
    return off;
}

// weight and bias gradients from the dZ_l^T and H_{l-1}^T the forward
// launch wrote
int backward(bd_surrogate *s) {
    const int B = s->batch;
    for (int l = s->L - 1; l >= 0; l--) {
        // dW_l = dZ_l^T H_{l-1}
        GemmArgs g = base_args(s);
        g.M = s->Np[l];
        g.N = s->Kp[l];
        g.K = B;
        g.k_split = s->ksplit;
        g.out_f32 = s->part + part_offset(s, l);
        int rc = launch_gemm(s->tm_dzt[l], s->tm_ht[l], g, s->stream);
        if (rc) return rc;
    }
    BiasGradArgs a;
    std::memset(&a, 0, sizeof(a));
    a.L = s->L;
    a.B = B;
    for (int l = 0; l < s->L; l++) {
        a.dzt[l] = s->dzt[l];
        a.db[l] = s->db[l];
        a.first[l + 1] = a.first[l] + s->Np[l];
    }
    k_bias_grads<<<a.first[s->L], 256, 0, s->stream>>>(a);
    BD_LAUNCH_CHECK();
    return BD_OK;
}

int adam(bd_surrogate *s) {
    AdamArgs a{s->lr, 0.9f, 0.999f, 1e-8f, s->step};
    AdamTable t;
    std::memset(&t, 0, sizeof(t));
    t.L = s->L;
    t.splits = s->batch / s->ksplit;
    for (int l = 0; l < s->L; l++) {
        t.w[l] = s->w[l];
        t.wm[l] = s->wm[l];
        t.wv[l] = s->wv[l];
        t.part[l] = s->part + part_offset(s, l);
        t.wb[l] = s->wb[l];
        t.wbt[l] = s->wbt[l];
        t.b[l] = s->b[l];
        t.bm[l] = s->bm[l];
        t.bv[l] = s->bv[l];
        t.db[l] = s->db[l];
        t.N[l] = s->Np[l];
        t.K[l] = s->Kp[l];
        t.n_live[l] = s->Nl[l];
        t.k_live[l] = s->Kl[l];
        t.first_w[l + 1] = t.first_w[l] + (long long)s->Np[l] * s->Kp[l];
        t.first_b[l + 1] = t.first_b[l] + s->Np[l];
    }
    const long long total = t.first_w[s->L] + t.first_b[s->L];
    k_adam_all<<<(unsigned)div_up(total, 256), 256, 0, s->stream>>>(t, a);
    k_count<<<1, 1, 0, s->stream>>>(s->step);
    BD_LAUNCH_CHECK();
    return BD_OK;
}

int train_step_launches(bd_surrogate *s) {
    k_gather<<<div_up(s->batch, kGatherRows), 256, 0, s->stream>>>(
        s->data_x, s->data_y, s->n_data, s->n_in, s->n_out, s->Kp[0], s->Np[s->L - 1], s->batch, nullptr, s->step,
        s->seed, s->x0, s->ht[0], s->t);
    BD_LAUNCH_CHECK();
    int rc = forward(s, true);
    if (!rc) rc = backward(s);
    if (!rc) rc = adam(s);
    return rc;
}

}  // namespace

extern "C" {

int bd_surrogate_create(int n_in, int n_out, int width, int depth, int batch, unsigned long long seed,
                        bd_surrogate **out) {
    if (!out || n_in < 1 || n_in > 64 || n_out < 1 || n_out > 128 || width < 64 || width > 256 || width % 64 ||
        depth < 1 || depth > 8 || batch < 256 || batch % 256)
        return BD_ERR_ARG;
    bd_surrogate *s = new (std::nothrow) bd_surrogate();
    if (!s) return BD_ERR_NOMEM;
    s->n_in = n_in;
    s->n_out = n_out;
    s->width = width;
    s->depth = depth;
    s->batch = batch;
    s->seed = seed;
    s->L = depth + 1;
    for (int l = 0; l < s->L; l++) {
        s->Kl.push_back(l == 0 ? n_in : width);
        s->Kp.push_back(l == 0 ? 64 : width);
        s->Nl.push_back(l == s->L - 1 ? n_out : width);
        s->Np.push_back(l == s->L - 1 ? 128 : width);
    }
    // the fused forward / input-gradient kernel covers every shape accepted here
    static_assert(8 + 1 <= umma::kChainMaxLayers && 256 % kBM == 0, "depth <= 8, batch a multiple of 256");
    if (set_gemm_attrs() != BD_OK || cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete s;
        return BD_ERR_CUDA;
    }
    bool ok = true;
    auto A = [&](void **p, size_t bytes) {
        if (ok && cudaMalloc(p, bytes) != cudaSuccess) ok = false;
        if (ok) cudaMemsetAsync(*p, 0, bytes, s->stream);
    };
    size_t part_total = 0;
    for (int l = 0; l < s->L; l++) {
        const size_t nk = (size_t)s->Np[l] * s->Kp[l];
        float *p;
        __nv_bfloat16 *q;
        A((void **)&p, nk * 4); s->w.push_back(p);
        A((void **)&p, nk * 4); s->wm.push_back(p);
        A((void **)&p, nk * 4); s->wv.push_back(p);
        A((void **)&p, s->Np[l] * 4); s->b.push_back(p);
        A((void **)&p, s->Np[l] * 4); s->bm.push_back(p);
        A((void **)&p, s->Np[l] * 4); s->bv.push_back(p);
        A((void **)&p, s->Np[l] * 4); s->db.push_back(p);
        A((void **)&q, nk * 2); s->wb.push_back(q);
        A((void **)&q, nk * 2); s->wbt.push_back(q);
        if (l == 0) A((void **)&s->x0, (size_t)batch * s->Kp[0] * 2);
        A((void **)&q, (size_t)batch * s->Kp[l] * 2); s->ht.push_back(q);
        A((void **)&p, (size_t)batch * s->Np[l] * 4); s->z.push_back(p);
        A((void **)&q, (size_t)batch * s->Np[l] * 2); s->dzt.push_back(q);
        part_total += (size_t)(batch / s->ksplit) * nk;
    }
    A((void **)&s->y, (size_t)batch * 128 * 4);
    A((void **)&s->t, (size_t)batch * 128 * 4);
    A((void **)&s->tw, 128 * 4);
    A((void **)&s->part, part_total * 4);
    // loss partials: one per CTA of the fused kernel
    s->loss_cells = (batch / kBM) * umma::kChainCluster;
    A((void **)&s->loss_part, (size_t)s->loss_cells * 4);
    A((void **)&s->step, sizeof(long long));
    A((void **)&s->err, sizeof(unsigned));
    if (!ok) {
        free_surrogate(s);
        return BD_ERR_NOMEM;
    }
    // He-style initialisation on the host (deterministic), biases zero
    unsigned long long st = seed * 6364136223846793005ULL + 1442695040888963407ULL;
    auto rnd = [&]() {
        st = st * 6364136223846793005ULL + 1442695040888963407ULL;
        return ((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;  // uniform(-1, 1)
    };
    for (int l = 0; l < s->L; l++) {
        std::vector<float> hw((size_t)s->Np[l] * s->Kp[l], 0.f);
        const double scale = std::sqrt(6.0 / (double)s->Kl[l]);
        for (int n = 0; n < s->Nl[l]; n++)
            for (int k = 0; k < s->Kl[l]; k++) hw[(size_t)k * s->Np[l] + n] = (float)(scale * rnd() * 0.5);
        cudaMemcpyAsync(s->w[l], hw.data(), hw.size() * 4, cudaMemcpyHostToDevice, s->stream);
        k_to_bf16<<<div_up((long)hw.size(), 256), 256, 0, s->stream>>>(s->w[l], s->Np[l], s->Kp[l], s->wb[l],
                                                                       s->wbt[l]);
    }
    std::vector<float> ones(128, 1.f);
    cudaMemcpyAsync(s->tw, ones.data(), 128 * 4, cudaMemcpyHostToDevice, s->stream);
    // tensor maps
    int rc = BD_OK;
    s->tm_ht.resize(s->L);
    s->tm_dzt.resize(s->L);
    s->tm_w.resize(s->L);
    s->tm_wt.resize(s->L);
    rc |= make_tmap(&s->tm_x, s->x0, batch, s->Kp[0], kBM);
    for (int l = 0; l < s->L && !rc; l++) {
        // weight gradient: A = dZ_l^T, B = H_{l-1}^T; fused kernel: W_l and W_l^T,
        // a quarter of the rows per CTA of a cluster
        rc |= make_tmap(&s->tm_dzt[l], s->dzt[l], s->Np[l], batch, kBM);
        rc |= make_tmap(&s->tm_ht[l], s->ht[l], s->Kp[l], batch, kBN);
        rc |= make_tmap(&s->tm_w[l], s->wb[l], s->Np[l], s->Kp[l], s->Np[l] / umma::kChainCluster);
        rc |= make_tmap(&s->tm_wt[l], s->wbt[l], s->Kp[l], s->Np[l], s->Kp[l] / umma::kChainCluster);
    }
    if (rc || cudaStreamSynchronize(s->stream) != cudaSuccess) {
        free_surrogate(s);
        return rc ? rc : BD_ERR_CUDA;
    }
    *out = s;
    return BD_OK;
}

int bd_surrogate_destroy(bd_surrogate *s) {
    if (!s) return BD_ERR_ARG;
    cudaStreamSynchronize(s->stream);
    free_surrogate(s);
    return BD_OK;
}

int bd_surrogate_get_stream(const bd_surrogate *s, void **stream) {
    if (!s || !stream) return BD_ERR_ARG;
    *stream = (void *)s->stream;
    return BD_OK;
}

int bd_surrogate_param_count(const bd_surrogate *s, long long *count) {
    if (!s || !count) return BD_ERR_ARG;
    long long c = 0;
    for (int l = 0; l < s->L; l++) c += (long long)s->Nl[l] * s->Kl[l] + s->Nl[l];
    *count = c;
    return BD_OK;
}

// Parameters as a flat FP32 vector: for each layer W [N_l][K_l] then b [N_l].
int bd_surrogate_get_params(bd_surrogate *s, float *out) {
    if (!s || !out) return BD_ERR_ARG;
    size_t off = 0;
    for (int l = 0; l < s->L; l++) {
        std::vector<float> hw((size_t)s->Np[l] * s->Kp[l]), hb(s->Np[l]);
        BD_CUDA_TRY(cudaMemcpyAsync(hw.data(), s->w[l], hw.size() * 4, cudaMemcpyDeviceToHost, s->stream));
        BD_CUDA_TRY(cudaMemcpyAsync(hb.data(), s->b[l], hb.size() * 4, cudaMemcpyDeviceToHost, s->stream));
        BD_CUDA_TRY(cudaStreamSynchronize(s->stream));
        for (int n = 0; n < s->Nl[l]; n++)
            for (int k = 0; k < s->Kl[l]; k++) out[off++] = hw[(size_t)k * s->Np[l] + n];  // master kept [K][N]
        for (int n = 0; n < s->Nl[l]; n++) out[off++] = hb[n];
    }
    return BD_OK;
}

int bd_surrogate_set_params(bd_surrogate *s, const float *in) {
    if (!s || !in) return BD_ERR_ARG;
    size_t off = 0;
    for (int l = 0; l < s->L; l++) {
        std::vector<float> hw((size_t)s->Np[l] * s->Kp[l], 0.f), hb(s->Np[l], 0.f);
        for (int n = 0; n < s->Nl[l]; n++)
            for (int k = 0; k < s->Kl[l]; k++) hw[(size_t)k * s->Np[l] + n] = in[off++];  // master kept [K][N]
        for (int n = 0; n < s->Nl[l]; n++) hb[n] = in[off++];
        BD_CUDA_TRY(cudaMemcpyAsync(s->w[l], hw.data(), hw.size() * 4, cudaMemcpyHostToDevice, s->stream));
        BD_CUDA_TRY(cudaMemcpyAsync(s->b[l], hb.data(), hb.size() * 4, cudaMemcpyHostToDevice, s->stream));
        k_to_bf16<<<div_up((long)hw.size(), 256), 256, 0, s->stream>>>(s->w[l], s->Np[l], s->Kp[l], s->wb[l],
                                                                       s->wbt[l]);
        BD_LAUNCH_CHECK();
    }
    BD_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return BD_OK;
}

// Loss weight per output (default 1).
int bd_surrogate_set_output_weights(bd_surrogate *s, const float *w) {
    if (!s || !w) return BD_ERR_ARG;
    std::vector<float> hw(128, 0.f);
    for (int i = 0; i < s->n_out; i++) hw[i] = w[i];
    BD_CUDA_TRY(cudaMemcpyAsync(s->tw, hw.data(), 128 * 4, cudaMemcpyHostToDevice, s->stream));
    BD_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return BD_OK;
}

// Training set on the device: x [n][n_in], y [n][n_out] (host, FP32).
int bd_surrogate_set_data(bd_surrogate *s, const float *x, const float *y, int n) {
    if (!s || !x || !y || n < 1) return BD_ERR_ARG;
    if (s->graph) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }
    if (s->data_x) cudaFree(s->data_x);
    if (s->data_y) cudaFree(s->data_y);
    s->data_x = s->data_y = nullptr;
    BD_CUDA_TRY(cudaMalloc(&s->data_x, (size_t)n * s->n_in * 4));
    BD_CUDA_TRY(cudaMalloc(&s->data_y, (size_t)n * s->n_out * 4));
    BD_CUDA_TRY(cudaMemcpyAsync(s->data_x, x, (size_t)n * s->n_in * 4, cudaMemcpyHostToDevice, s->stream));
    BD_CUDA_TRY(cudaMemcpyAsync(s->data_y, y, (size_t)n * s->n_out * 4, cudaMemcpyHostToDevice, s->stream));
    BD_CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->n_data = n;
    return BD_OK;
}

// `steps` Adam steps on random minibatches (with replacement) of the
// training set, captured once as a CUDA graph; mean loss of the last step.
int bd_surrogate_train(bd_surrogate *s, int steps, float lr, float *last_loss) {
    if (!s || steps < 0 || !(lr > 0.f)) return BD_ERR_ARG;
    if (!s->data_x) return BD_ERR_STATE;
    if (lr != s->lr && s->graph) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }
    s->lr = lr;
    if (!s->graph && steps > 0) {
        cudaGraph_t g;
        BD_CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        int rc = train_step_launches(s);
        cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
        if (rc) return rc;
        BD_CUDA_TRY(ce);
        BD_CUDA_TRY(cudaGraphInstantiate(&s->graph, g, 0));
        cudaGraphDestroy(g);
    }
    for (int i = 0; i < steps; i++) BD_CUDA_TRY(cudaGraphLaunch(s->graph, s->stream));
    if (last_loss) {
        std::vector<float> lp(s->loss_cells);
        BD_CUDA_TRY(cudaMemcpyAsync(lp.data(), s->loss_part, lp.size() * 4, cudaMemcpyDeviceToHost, s->stream));
        BD_CUDA_TRY(cudaStreamSynchronize(s->stream));
        double sum = 0;
        for (float v : lp) sum += v;
        *last_loss = (float)(sum / ((double)s->batch * s->n_out));
    }
    return sg_status(s);
}

// Gradients of the mean loss over one batch (x [batch][n_in], y
// [batch][n_out], host) without an update, flat like bd_surrogate_get_params;
// loss = (1 / (batch n_out)) sum w (y_pred - y)^2.
int bd_surrogate_gradients(bd_surrogate *s, const float *x, const float *y, float *grad, float *loss) {
    if (!s || !x || !y || !grad) return BD_ERR_ARG;
    const int B = s->batch;
    float *dx = nullptr, *dy = nullptr;
    BD_CUDA_TRY(cudaMalloc(&dx, (size_t)B * s->n_in * 4));
    BD_CUDA_TRY(cudaMalloc(&dy, (size_t)B * s->n_out * 4));
    cudaMemcpyAsync(dx, x, (size_t)B * s->n_in * 4, cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(dy, y, (size_t)B * s->n_out * 4, cudaMemcpyHostToDevice, s->stream);
    std::vector<int> rows(B);
    for (int i = 0; i < B; i++) rows[i] = i;
    int *drows = nullptr;
    BD_CUDA_TRY(cudaMalloc(&drows, B * 4));
    cudaMemcpyAsync(drows, rows.data(), B * 4, cudaMemcpyHostToDevice, s->stream);
    k_gather<<<div_up(B, kGatherRows), 256, 0, s->stream>>>(dx, dy, B, s->n_in, s->n_out, s->Kp[0],
                                                             s->Np[s->L - 1], B, drows, s->step, s->seed, s->x0,
                                                             s->ht[0], s->t);
    int rc = forward(s, true);
    if (!rc) rc = backward(s);
    const int splits = B / s->ksplit;
    size_t off = 0;
    std::vector<float> lp(s->loss_cells);
    if (!rc) {
        for (int l = 0; l < s->L && !rc; l++) {
            const size_t n = (size_t)s->Np[l] * s->Kp[l];
            float *gsum = nullptr;
            if (cudaMalloc(&gsum, n * 4) != cudaSuccess) { rc = BD_ERR_NOMEM; break; }
            k_sum_splits<<<div_up((long)n, 256), 256, 0, s->stream>>>(s->part + part_offset(s, l), splits, n, gsum);
            std::vector<float> hg(n), hb(s->Np[l]);
            cudaMemcpyAsync(hg.data(), gsum, n * 4, cudaMemcpyDeviceToHost, s->stream);
            cudaMemcpyAsync(hb.data(), s->db[l], s->Np[l] * 4, cudaMemcpyDeviceToHost, s->stream);
            cudaStreamSynchronize(s->stream);
            cudaFree(gsum);
            for (int nn = 0; nn < s->Nl[l]; nn++)  // partial sums are [K][N]
                for (int k = 0; k < s->Kl[l]; k++) grad[off++] = hg[(size_t)k * s->Np[l] + nn];
            for (int nn = 0; nn < s->Nl[l]; nn++) grad[off++] = hb[nn];
        }
        cudaMemcpyAsync(lp.data(), s->loss_part, lp.size() * 4, cudaMemcpyDeviceToHost, s->stream);
    }
    cudaStreamSynchronize(s->stream);
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(drows);
    if (rc) return rc;
    if (loss) {
        double sum = 0;
        for (float v : lp) sum += v;
        *loss = (float)(sum / ((double)B * s->n_out));
    }
    return sg_status(s);
}

// Network outputs for n inputs (host x [n][n_in] -> y [n][n_out]).
int bd_surrogate_predict(bd_surrogate *s, const float *x, int n, float *y) {
    if (!s || !x || !y || n < 0) return BD_ERR_ARG;
    const int B = s->batch;
    float *dx = nullptr;
    int *drows = nullptr;
    BD_CUDA_TRY(cudaMalloc(&dx, (size_t)std::max(n, 1) * s->n_in * 4));
    BD_CUDA_TRY(cudaMalloc(&drows, B * 4));
    BD_CUDA_TRY(cudaMemcpyAsync(dx, x, (size_t)n * s->n_in * 4, cudaMemcpyHostToDevice, s->stream));
    std::vector<int> rows(B);
    std::vector<float> hy((size_t)B * 128);
    int rc = BD_OK;
    for (int r0 = 0; r0 < n && !rc; r0 += B) {
        const int cnt = std::min(B, n - r0);
        for (int i = 0; i < B; i++) rows[i] = i < cnt ? r0 + i : -1;
        cudaMemcpyAsync(drows, rows.data(), B * 4, cudaMemcpyHostToDevice, s->stream);
        k_gather<<<div_up(B, kGatherRows), 256, 0, s->stream>>>(dx, nullptr, n, s->n_in, s->n_out, s->Kp[0],
                                                                 s->Np[s->L - 1], B, drows, s->step, s->seed,
                                                                 s->x0, s->ht[0], nullptr);
        rc = forward(s, false);
        if (rc) break;
        cudaMemcpyAsync(hy.data(), s->y, hy.size() * 4, cudaMemcpyDeviceToHost, s->stream);
        if (cudaStreamSynchronize(s->stream) != cudaSuccess) rc = BD_ERR_CUDA;
        for (int i = 0; i < cnt; i++)  // outputs are [128][B]
            for (int k = 0; k < s->n_out; k++) y[(size_t)(r0 + i) * s->n_out + k] = hy[(size_t)k * B + i];
    }
    cudaFree(dx);
    cudaFree(drows);
    if (rc) return rc;
    return sg_status(s);
}

// Plain GEMM through the same kernel, for tests and measurement:
// C [M][N] (FP32) = A [M][K] B [N][K]^T with BF16 inputs given as raw bits.
int bd_umma_gemm_bf16(const unsigned short *a, const unsigned short *b, int M, int N, int K, float *c) {
    if (!a || !b || !c || M < 1 || N < 1 || K < 8 || K % 8) return BD_ERR_ARG;
    __nv_bfloat16 *da = nullptr, *db = nullptr;
    float *dc = nullptr, *part = nullptr;
    unsigned *err = nullptr;
    const int ks = 256, splits = div_up(K, ks);
    int rc = BD_OK;
    cudaStream_t st = nullptr;
    if (set_gemm_attrs() != BD_OK) return BD_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return BD_ERR_CUDA;
    if (cudaMalloc(&da, (size_t)M * K * 2) != cudaSuccess || cudaMalloc(&db, (size_t)N * K * 2) != cudaSuccess ||
        cudaMalloc(&part, (size_t)splits * M * N * 4) != cudaSuccess || cudaMalloc(&dc, (size_t)M * N * 4) != cudaSuccess ||
        cudaMalloc(&err, 4) != cudaSuccess)
        rc = BD_ERR_NOMEM;
    CUtensorMap ta, tb;
    if (!rc) {
        cudaMemcpyAsync(da, a, (size_t)M * K * 2, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(db, b, (size_t)N * K * 2, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(err, 0, 4, st);
        rc = make_tmap(&ta, da, M, K, kBM);
        if (!rc) rc = make_tmap(&tb, db, N, K, kBN);
    }
    if (!rc) {
        GemmArgs g;
        std::memset(&g, 0, sizeof(g));
        g.M = M;
        g.N = N;
        g.K = K;
        g.k_split = ks;
        g.out_f32 = part;
        g.err = err;
        rc = launch_gemm(ta, tb, g, st);
    }
    if (!rc) {
        k_sum_splits<<<div_up((long)M * N, 256), 256, 0, st>>>(part, splits, (size_t)M * N, dc);
        std::vector<float> ct((size_t)M * N);  // the kernel writes C transposed
        cudaMemcpyAsync(ct.data(), dc, (size_t)M * N * 4, cudaMemcpyDeviceToHost, st);
        unsigned e = 0;
        cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = BD_ERR_CUDA;
        else if (e) rc = BD_ERR_TIMEOUT;
        for (int i = 0; i < M && !rc; i++)
            for (int j = 0; j < N; j++) c[(size_t)i * N + j] = ct[(size_t)j * M + i];
    }
    cudaFree(da);
    cudaFree(db);
    cudaFree(dc);
    cudaFree(part);
    cudaFree(err);
    cudaStreamDestroy(st);
    return rc;
}

}  // extern "C"
