// engine_kernels.cuh -- device code of the batched replica engine: the fused
// force + Ermak-McCammon + re-binning step over cell bricks, initial load,
// export and reference-stream set-up.  Included by engine.cu (host driver).
#pragma once
//
// One time step of the reference (main.cu:494-588: update_ermak_dev x2, cell
// clears + cell_locate_dev x2, force clears + get_forces_*_dev x4, three
// device synchronisations) becomes ONE launch here:
//   1. stage the cells of a brick plus a one-cell halo into shared memory
//      (counts -> block scan -> compact copy, each cell sorted by storage id
//      so the force sum order is fixed),
//   2. sweep the 27 neighbour cells of every home particle with the
//      per-species-pair cut distances (bb, bs, ss) in one pass,
//   3. apply the Ermak-McCammon update with counter-based Gaussians and the
//      compensated FP32 position + FP64 displacement,
//   4. bin the new position into the next count/position buffer (atomic slot)
//      and clear the third count buffer for the brick's own cells.
// Forces never touch HBM.
#include <curand_kernel.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "engine.cuh"
#include "runtime.cuh"

namespace bd {

// ------------------------------------------------------------- schedules
__device__ __forceinline__ float temp_protocol(const SysDev &S, float t) {
    if (S.protocol == 0) return temp_linear(S.T0, S.Tf, S.t0, S.tf, t);
    if (S.protocol == 1) {  // set_temp.cu:14-23
        if (t < S.t0) return S.T0;
        if (t > S.tf) return S.Tf;
        float a = __double2float_rn(0.5 * (double)__fadd_rn(S.T0, S.Tf));
        float b = __double2float_rn(0.5 * (double)__fsub_rn(S.Tf, S.T0));
        float arg = __double2float_rn((double)(2.0f * kRefPi) * ((double)__fdiv_rn(t, S.period) - 0.25));
        return __fadd_rn(a, __fmul_rn(b, sinf(arg)));
    }
    return S.T0;
}
// Temperature seen by the update of reference step ni: temp_set was last set
// after the update of step ni-1 with time = dt * (1 + (float)(ni-1))
// (main.cu:520-524); the first step of a run uses T0 (main.cu:156).
__device__ __forceinline__ float step_temperature(const SysDev &S, long long ni, long long ni_first) {
    if (ni == ni_first) return S.T0;
    float t = __double2float_rn(__dmul_rn(S.dt_d, __dadd_rn(1.0, (double)(float)(ni - 1))));
    return temp_protocol(S, t);
}
// update_ermak.cu:114 with the mobility in place of 1/sigma
__device__ __forceinline__ float amplitude(float T, float mob, float dt) {
    return __double2float_rn(__dsqrt_rn(__dmul_rn(__dmul_rn(__dmul_rn(2.0, (double)T), (double)mob), (double)dt)));
}

// ------------------------------------------------------------- block scan
// Exclusive scan of a[0..n) and b[0..n) in place; a[n], b[n] get the totals.
__device__ void block_scan2(int *a, int *b, int n, int *tmp) {
    const int T = blockDim.x, tid = threadIdx.x;
    const int per = (n + T - 1) / T, beg = min(n, tid * per), end = min(n, beg + per);
    int sa = 0, sb = 0;
    for (int i = beg; i < end; i++) { sa += a[i]; sb += b[i]; }
    const int lane = tid & 31, wid = tid >> 5, nw = (T + 31) >> 5;
    int ia = sa, ib = sb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int ua = __shfl_up_sync(0xffffffffu, ia, o), ub = __shfl_up_sync(0xffffffffu, ib, o);
        if (lane >= o) { ia += ua; ib += ub; }
    }
    if (lane == 31) { tmp[wid] = ia; tmp[32 + wid] = ib; }
    __syncthreads();
    if (tid == 0) {
        int ra = 0, rb = 0;
        for (int w = 0; w < nw; w++) {
            int va = tmp[w], vb = tmp[32 + w];
            tmp[w] = ra; tmp[32 + w] = rb;
            ra += va; rb += vb;
        }
        a[n] = ra;
        b[n] = rb;
    }
    __syncthreads();
    int oa = tmp[wid] + ia - sa, ob = tmp[32 + wid] + ib - sb;
    for (int i = beg; i < end; i++) {
        int va = a[i], vb = b[i];
        a[i] = oa; b[i] = ob;
        oa += va; ob += vb;
    }
    __syncthreads();
}

__device__ __forceinline__ double block_sum(double v, double *red) {
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < nw; w++) s += red[w];
    return s;  // valid in thread 0
}

}  // namespace bd
#include "step.cuh"
#include "nlist.cuh"
namespace bd {

__global__ void k_advance_counter(long long *ni_base, int k) { *ni_base += k; }

// ------------------------------------------------------------- load/export
// Bin particles given in storage order (float4 w = sid | species << 31).
__global__ void k_load(const float4 *__restrict__ staged, int P, const int *__restrict__ rep_of_sid,
                       const SysDev *sys, int *cnt, float4 *pos, int cap, double *x0, const int *gid_of,
                       unsigned *st, float4 *pos_sid) {
    int sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= P) return;
    float4 v = staged[sid];
    if (pos_sid) pos_sid[sid] = v;  // neighbour-list mode keeps positions by storage id
    const SysDev &S = sys[rep_of_sid[sid]];
    int nc = S.ncell;
    int ix = (int)__fmul_rn(v.x, S.cinv), iy = (int)__fmul_rn(v.y, S.cinv), iz = (int)__fmul_rn(v.z, S.cinv);
    if (!(v.x >= 0.f && v.x <= S.L && v.y >= 0.f && v.y <= S.L && v.z >= 0.f && v.z <= S.L)) set_status(st, kStatArg);
    ix = min(max(ix, 0), nc - 1);
    iy = min(max(iy, 0), nc - 1);
    iz = min(max(iz, 0), nc - 1);
    int cell = S.cell_base + ix + nc * (iy + nc * iz);
    int slot = atomicAdd(cnt + cell, 1);
    if (slot < cap) pos[(size_t)cell * cap + slot] = v;
    else set_status(st, kStatCellOverflow);
    int gid = gid_of[sid];
    x0[3 * (size_t)gid] = v.x;
    x0[3 * (size_t)gid + 1] = v.y;
    x0[3 * (size_t)gid + 2] = v.z;
}
// Export current positions by global index: wrapped (hi) and unwrapped
// (origin + displacement) float3.
__global__ void k_export(const int *__restrict__ cnt, const float4 *__restrict__ pos, int C, int cap, int P,
                         const int *__restrict__ gid_of, const double *__restrict__ x0,
                         const double *__restrict__ dx, const double *__restrict__ dy, const double *__restrict__ dz,
                         float *out_pos, float *out_raw, float4 *snap) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    int k = min(cnt[c], cap);
    for (int s = 0; s < k; s++) {
        float4 v = pos[(size_t)c * cap + s];
        unsigned w = __float_as_uint(v.w);
        int sid = w & 0x7fffffff;
        if (sid >= P) continue;  // never true for consistent buffers
        int gid = gid_of[sid];
        if (out_pos) { out_pos[3 * (size_t)gid] = v.x; out_pos[3 * (size_t)gid + 1] = v.y; out_pos[3 * (size_t)gid + 2] = v.z; }
        if (out_raw) {
            out_raw[3 * (size_t)gid] = (float)(x0[3 * (size_t)gid] + dx[sid]);
            out_raw[3 * (size_t)gid + 1] = (float)(x0[3 * (size_t)gid + 1] + dy[sid]);
            out_raw[3 * (size_t)gid + 2] = (float)(x0[3 * (size_t)gid + 2] + dz[sid]);
        }
        if (snap) snap[gid] = make_float4(v.x, v.y, v.z, __int_as_float((int)(w >> 31)));
    }
}
// Per-particle rannew64 seeding (rannew64.cu, first call): particle pid of a
// replica with seed S uses idum = S + pid (absolute value), 1000 warm-up LCG
// steps, then 250 ring words; the second LCG starts from the last word.
__global__ void k_rannew64_seed(unsigned long long *ring, unsigned long long *lcg, const SysDev *sys,
                                const int *rep_of_sid, const int *gid_of, int P) {
    const int sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= P) return;
    const SysDev &S = sys[rep_of_sid[sid]];
    long long idum = (long long)S.seed + (long long)(gid_of[sid] - S.part_base);
    if (idum < 0) idum = -idum;
    unsigned long long u = (unsigned long long)idum;
    for (int i = 0; i < 1000; i++) u = u * kRnSeedA + kRnSeedC;
    for (int i = 0; i < kRnWords; i++) {
        u = u * kRnSeedA + kRnSeedC;
        ring[(size_t)i * P + sid] = u;
    }
    lcg[sid] = u;
}

__global__ void k_curand_setup(curandState *st, const SysDev *sys, const int *rep_of_gid, int P) {
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= P) return;
    const SysDev &S = sys[rep_of_gid[gid]];
    int pid = gid - S.part_base;
    // reference: big seeded with idum, small with idum + 1, subsequence = index
    // within the species (main.cu:483-484, update_ermak.cu:85-89)
    if (pid < S.n_big) curand_init(S.seed, pid, 0, &st[gid]);
    else curand_init(S.seed + 1, pid - S.n_big, 0, &st[gid]);
}

}  // namespace bd
