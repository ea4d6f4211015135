// cv3d.cu -- Contracting_Vector3D (Contracting_Vector3D.cuh:39-75) on the GPU.
//
// add_statistics (Contracting_Vector3D.cu:57-164): for every particle m, the
// per-bin sums h_b(m) of unit vectors d/|d| towards its neighbours closer than
// `range` (d = r_m - r_n, optional minimum image with floor() of the double
// sum, Contracting_Vector3D.cu:101-105), then per Cartesian component c the
// normal equations A^T A_c += h_c h_c^T and A^T b_c += h_c f_c.
//   kernel 1 (k_cv_hits): one warp per particle, lanes stride over partners,
//     bins accumulated in shared memory -> H[c][m][b] (float, like the
//     reference's hit_vec);
//   kernel 2 (k_cv_normal): A^T A_c = H_c^T H_c and A^T b_c = H_c^T f_c
//     accumulated in FP64 (the reference accumulates in float), tiled over m.
// calculate_vector (Contracting_Vector3D.cu:166-297): per component the SVD
// pseudo-inverse x = V diag(1/w) U^T b with 1/w dropped where
// |w / w_max| <= 1e-6, averaged over the three components.  The matrices are
// bins x bins, so the FP64 one-sided Jacobi SVD runs on the host.
#include <cmath>
#include <cstring>
#include <vector>

#include "runtime.cuh"

namespace bd {

constexpr int kCvNeighsMax = 10000;  // Contracting_Vector3D.cuh:36

__global__ void k_cv_hits(const float *__restrict__ rr, int n, float side, float range, int bins, float *H,
                          unsigned *st) {
    extern __shared__ float sh[];  // [warps][3][bins]
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float *hw = sh + (size_t)wid * 3 * bins;
    const int m = blockIdx.x * (blockDim.x >> 5) + wid;
    for (int b = lane; b < 3 * bins; b += 32) hw[b] = 0.f;
    __syncwarp();
    if (m >= n) return;
    const float bin_size = __fdiv_rn(range, (float)bins);
    const float bin_size_inv = __fdiv_rn(1.0f, bin_size);
    const float range_sq = __fmul_rn(range, range);
    const bool pbc = side > 0.f;
    const float side_inv = pbc ? __fdiv_rn(1.0f, side) : 0.f;
    const float xm = rr[3 * m], ym = rr[3 * m + 1], zm = rr[3 * m + 2];
    int neighs = 0;
    for (int j = lane; j < n; j += 32) {
        if (j == m) continue;
        float dx = __fsub_rn(xm, rr[3 * j]), dy = __fsub_rn(ym, rr[3 * j + 1]), dz = __fsub_rn(zm, rr[3 * j + 2]);
        if (pbc) {
            dx = __fsub_rn(dx, __fmul_rn(side, (float)floor(__dadd_rn((double)__fmul_rn(side_inv, dx), 0.5))));
            dy = __fsub_rn(dy, __fmul_rn(side, (float)floor(__dadd_rn((double)__fmul_rn(side_inv, dy), 0.5))));
            dz = __fsub_rn(dz, __fmul_rn(side, (float)floor(__dadd_rn((double)__fmul_rn(side_inv, dz), 0.5))));
        }
        float d2 = dist2_rn(dx, dy, dz);
        if (d2 < range_sq) {
            float dist = __fsqrt_rn(d2);
            int nb = (int)__fmul_rn(bin_size_inv, dist);
            if (nb >= bins) nb = bins - 1;  // the reference indexes hit_vec[bins] here
            atomicAdd(&hw[nb], __fdiv_rn(dx, dist));
            atomicAdd(&hw[bins + nb], __fdiv_rn(dy, dist));
            atomicAdd(&hw[2 * bins + nb], __fdiv_rn(dz, dist));
            neighs++;
        }
    }
    for (int o = 16; o; o >>= 1) neighs += __shfl_down_sync(0xffffffffu, neighs, o);
    if (lane == 0 && neighs >= kCvNeighsMax) set_status(st, kStatCellOverflow);
    __syncwarp();
    for (int b = lane; b < bins; b += 32) {
        H[(size_t)0 * n * bins + (size_t)m * bins + b] = hw[b];
        H[(size_t)1 * n * bins + (size_t)m * bins + b] = hw[bins + b];
        H[(size_t)2 * n * bins + (size_t)m * bins + b] = hw[2 * bins + b];
    }
}

// A^T A_c[i][j] += sum_m H_c[m][i] H_c[m][j];  A^T b_c[i] += sum_m H_c[m][i] f_c[m]
// grid: (ceil(bins/16), ceil(bins/16), 3), block 16x16, m tiled by 64.
__global__ void k_cv_normal(const float *__restrict__ H, const float *__restrict__ xx, int n, int bins, double *ata,
                            double *atb) {
    __shared__ float hi[64][17], hj[64][17], fc[64];
    const int c = blockIdx.z;
    const int i = blockIdx.y * 16 + threadIdx.y, j = blockIdx.x * 16 + threadIdx.x;
    const float *Hc = H + (size_t)c * n * bins;
    double acc = 0.0, accb = 0.0;
    const int tid = threadIdx.y * 16 + threadIdx.x;
    for (int m0 = 0; m0 < n; m0 += 64) {
        __syncthreads();
        for (int t = tid; t < 64 * 16; t += 256) {
            int mm = t / 16, kk = t % 16;
            int m = m0 + mm;
            int ii = blockIdx.y * 16 + kk, jj = blockIdx.x * 16 + kk;
            hi[mm][kk] = (m < n && ii < bins) ? Hc[(size_t)m * bins + ii] : 0.f;
            hj[mm][kk] = (m < n && jj < bins) ? Hc[(size_t)m * bins + jj] : 0.f;
        }
        if (tid < 64) fc[tid] = (m0 + tid < n) ? xx[3 * (size_t)(m0 + tid) + c] : 0.f;
        __syncthreads();
#pragma unroll 8
        for (int mm = 0; mm < 64; mm++) {
            acc += (double)hi[mm][threadIdx.y] * (double)hj[mm][threadIdx.x];
            if (blockIdx.x == 0 && threadIdx.x == 0) accb += (double)hi[mm][threadIdx.y] * (double)fc[mm];
        }
    }
    if (i < bins && j < bins) ata[(size_t)c * bins * bins + (size_t)i * bins + j] += acc;
    if (blockIdx.x == 0 && threadIdx.x == 0 && i < bins) atb[(size_t)c * bins + i] += accb;
}

// One-sided Jacobi SVD of a symmetric bins x bins matrix in FP64 (host).
static void jacobi_svd(int N, std::vector<double> &a, std::vector<double> &v, std::vector<double> &w) {
    v.assign((size_t)N * N, 0.0);
    for (int i = 0; i < N; i++) v[(size_t)i * N + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (int p = 0; p + 1 < N; p++)
            for (int q = p + 1; q < N; q++) {
                double al = 0, be = 0, ga = 0;
                for (int i = 0; i < N; i++) {
                    double ap = a[(size_t)i * N + p], aq = a[(size_t)i * N + q];
                    al += ap * ap; be += aq * aq; ga += ap * aq;
                }
                if (ga == 0.0) continue;
                double den = std::sqrt(al * be);
                if (den == 0.0) continue;
                double co = std::fabs(ga) / den;
                off = std::max(off, co);
                if (co < 1e-15) continue;
                double zeta = (be - al) / (2.0 * ga);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                double cs = 1.0 / std::sqrt(1.0 + t * t), sn = cs * t;
                for (int i = 0; i < N; i++) {
                    double ap = a[(size_t)i * N + p], aq = a[(size_t)i * N + q];
                    a[(size_t)i * N + p] = cs * ap - sn * aq;
                    a[(size_t)i * N + q] = sn * ap + cs * aq;
                    double vp = v[(size_t)i * N + p], vq = v[(size_t)i * N + q];
                    v[(size_t)i * N + p] = cs * vp - sn * vq;
                    v[(size_t)i * N + q] = sn * vp + cs * vq;
                }
            }
        if (off < 1e-15) break;
    }
    w.assign(N, 0.0);
    for (int j = 0; j < N; j++) {
        double s = 0;
        for (int i = 0; i < N; i++) s += a[(size_t)i * N + j] * a[(size_t)i * N + j];
        s = std::sqrt(s);
        w[j] = s;
        if (s > 0)
            for (int i = 0; i < N; i++) a[(size_t)i * N + j] /= s;
    }
}

}  // namespace bd

using namespace bd;

struct bd_cv3d {
    int bins = 0;
    float range = 0.f;
    int samples = 0;
    bool calculated = false;
    double *d_ata = nullptr, *d_atb = nullptr;
    float *d_H = nullptr;
    size_t H_cap = 0;
    unsigned *d_status = nullptr;
    std::vector<float> result;
};

extern "C" {

int bd_cv3d_create(int bins, float range, bd_cv3d **out) {
    if (!out || bins < 1 || bins > 1024 || !(range > 0)) return BD_ERR_ARG;
    bd_cv3d *cv = new bd_cv3d();
    cv->bins = bins;
    cv->range = range;
    cv->result.assign(bins, 0.f);
    if (cudaMalloc(&cv->d_ata, sizeof(double) * 3 * bins * bins) != cudaSuccess ||
        cudaMalloc(&cv->d_atb, sizeof(double) * 3 * bins) != cudaSuccess ||
        cudaMalloc(&cv->d_status, sizeof(unsigned)) != cudaSuccess) {
        bd_cv3d_destroy(cv);
        return BD_ERR_NOMEM;
    }
    cudaMemset(cv->d_ata, 0, sizeof(double) * 3 * bins * bins);
    cudaMemset(cv->d_atb, 0, sizeof(double) * 3 * bins);
    cudaMemset(cv->d_status, 0, sizeof(unsigned));
    *out = cv;
    return BD_OK;
}

int bd_cv3d_add_statistics(bd_cv3d *cv, const float *rr, const float *xx, int n, float side, void *stream) {
    if (!cv || n <= 0 || !rr || !xx) return BD_ERR_ARG;  // DEBUG_ASSERT(nparticles > 0) in the reference
    cudaStream_t s = as_stream(stream);
    const size_t need = (size_t)3 * n * cv->bins;
    if (need > cv->H_cap) {
        if (cv->d_H) cudaFree(cv->d_H);
        cv->d_H = nullptr;
        cv->H_cap = 0;
        if (cudaMalloc(&cv->d_H, need * sizeof(float)) != cudaSuccess) return BD_ERR_NOMEM;
        cv->H_cap = need;
    }
    const int warps = 8;
    const size_t sm = (size_t)warps * 3 * cv->bins * sizeof(float);
    if (sm > 200 * 1024) return BD_ERR_ARG;
    BD_CUDA_TRY(cudaFuncSetAttribute(k_cv_hits, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    BD_CUDA_TRY(cudaMemsetAsync(cv->d_status, 0, sizeof(unsigned), s));
    k_cv_hits<<<div_up(n, warps), warps * 32, sm, s>>>(rr, n, side, cv->range, cv->bins, cv->d_H, cv->d_status);
    BD_LAUNCH_CHECK();
    dim3 grid(div_up(cv->bins, 16), div_up(cv->bins, 16), 3);
    k_cv_normal<<<grid, dim3(16, 16), 0, s>>>(cv->d_H, xx, n, cv->bins, cv->d_ata, cv->d_atb);
    BD_LAUNCH_CHECK();
    unsigned bits = 0;
    BD_CUDA_TRY(cudaMemcpyAsync(&bits, cv->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    BD_CUDA_TRY(cudaStreamSynchronize(s));
    cv->samples++;
    return status_from_bits(bits);
}

int bd_cv3d_calculate_vector(bd_cv3d *cv) {
    if (!cv) return BD_ERR_ARG;
    if (cv->samples <= 0) return BD_ERR_STATE;  // the reference throws runtime_error
    const int N = cv->bins;
    std::vector<double> ata((size_t)3 * N * N), atb((size_t)3 * N);
    BD_CUDA_TRY(cudaMemcpy(ata.data(), cv->d_ata, sizeof(double) * ata.size(), cudaMemcpyDeviceToHost));
    BD_CUDA_TRY(cudaMemcpy(atb.data(), cv->d_atb, sizeof(double) * atb.size(), cudaMemcpyDeviceToHost));
    std::vector<double> acc(N, 0.0), a, v, w;
    for (int c = 0; c < 3; c++) {
        a.assign(ata.begin() + (size_t)c * N * N, ata.begin() + (size_t)(c + 1) * N * N);
        jacobi_svd(N, a, v, w);  // a <- U
        double wmax = 0;
        for (double x : w) wmax = std::max(wmax, std::fabs(x));
        std::vector<double> aux(N, 0.0);
        for (int j = 0; j < N; j++) {
            double s = 0;
            for (int i = 0; i < N; i++) s += a[(size_t)i * N + j] * atb[(size_t)c * N + i];
            double winv = (wmax > 0 && std::fabs(w[j] / wmax) > 1e-6) ? 1.0 / w[j] : 0.0;
            aux[j] = s * winv;
        }
        for (int i = 0; i < N; i++) {
            double s = 0;
            for (int k = 0; k < N; k++) s += v[(size_t)i * N + k] * aux[k];
            acc[i] += s;
        }
    }
    for (int i = 0; i < N; i++) cv->result[i] = (float)(acc[i] / 3.0);
    cv->calculated = true;
    return BD_OK;
}

int bd_cv3d_get_vector(const bd_cv3d *cv, float *out) {
    if (!cv || !out) return BD_ERR_ARG;
    if (!cv->calculated) return BD_ERR_STATE;  // the reference throws runtime_error
    std::memcpy(out, cv->result.data(), sizeof(float) * cv->bins);
    return BD_OK;
}

int bd_cv3d_destroy(bd_cv3d *cv) {
    if (!cv) return BD_ERR_ARG;
    if (cv->d_ata) cudaFree(cv->d_ata);
    if (cv->d_atb) cudaFree(cv->d_atb);
    if (cv->d_H) cudaFree(cv->d_H);
    if (cv->d_status) cudaFree(cv->d_status);
    delete cv;
    return BD_OK;
}

}  // extern "C"
