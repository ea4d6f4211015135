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
// (main.cu:520-524); the first step of a run uses the temp_set the run
// starts with: T0 (main.cu:156), or the caller's T_first.
__device__ __forceinline__ float step_temperature(const SysDev &S, long long ni, long long ni_first) {
    if (ni == ni_first) return S.T_first;
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

// ------------------------------------------------------------- storage order
// set_positions on the device.  A particle's slot is (replica, brick, cell
// within the brick) numbered in the order of the brick table; storage ids
// run over the slots in order and, within a slot, by reference index.
constexpr int kScanThreads = 1024, kScanPer = 4, kScanBlock = kScanThreads * kScanPer;

// slot of every particle (reference order) and the particle count per slot;
// a position outside [0, L] (or NaN) sets *bad and gets no slot
__global__ void k_order_keys(const float *__restrict__ pos3, int P, const int *__restrict__ rep_of_gid,
                             const SysDev *__restrict__ sys, int bx, int by, int bz, int *__restrict__ slot_of,
                             int *__restrict__ slot_cnt, unsigned *bad) {
    const int V = bx * by * bz;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < P; g += gridDim.x * blockDim.x) {
        const SysDev &S = sys[rep_of_gid[g]];
        const float x = pos3[3 * (size_t)g], y = pos3[3 * (size_t)g + 1], z = pos3[3 * (size_t)g + 2];
        if (!(x >= 0.f && x <= S.L && y >= 0.f && y <= S.L && z >= 0.f && z <= S.L)) {
            atomicOr(bad, 1u);
            slot_of[g] = -1;
            continue;
        }
        const int nc = S.ncell;
        const int ix = min(max((int)__fmul_rn(x, S.cinv), 0), nc - 1);
        const int iy = min(max((int)__fmul_rn(y, S.cinv), 0), nc - 1);
        const int iz = min(max((int)__fmul_rn(z, S.cinv), 0), nc - 1);
        const int b = ix / bx + S.nbx * (iy / by + S.nby * (iz / bz));
        const int c = ix % bx + bx * (iy % by + by * (iz % bz));
        const int sp = (g - S.part_base) < S.n_big ? 0 : 1;
        const int slot = ((S.brick_base + b) * 2 + sp) * V + c;  // brick, species, cell
        slot_of[g] = slot;
        atomicAdd(slot_cnt + slot, 1);
    }
}

// exclusive scan, pass 1: each block scans kScanBlock entries in place and
// writes its total
__global__ void __launch_bounds__(kScanThreads) k_scan_local(int *__restrict__ v, int n, int *__restrict__ bsum) {
    __shared__ int wsum[kScanThreads / 32];
    const int base = blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
    int x[kScanPer], t = 0;
#pragma unroll
    for (int i = 0; i < kScanPer; i++) {
        x[i] = base + i < n ? v[base + i] : 0;
        t += x[i];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = t;  // inclusive warp scan of the thread totals
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += y;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kScanThreads / 32 ? wsum[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        wsum[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    int run = inc - t + (warp ? wsum[warp - 1] : 0);
#pragma unroll
    for (int i = 0; i < kScanPer; i++) {
        if (base + i < n) v[base + i] = run;
        run += x[i];
    }
    if (threadIdx.x == kScanThreads - 1) bsum[blockIdx.x] = run;
}
// pass 2 (one block): exclusive scan of the block totals
__global__ void __launch_bounds__(kScanThreads) k_scan_totals(int *bsum, int nb) {
    __shared__ int carry;
    __shared__ int wsum[kScanThreads / 32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b0 = 0; b0 < nb; b0 += kScanThreads) {
        const int i = b0 + threadIdx.x;
        const int t = i < nb ? bsum[i] : 0;
        int inc = t;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, off);
            if (lane >= off) inc += y;
        }
        if (lane == 31) wsum[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            int w = wsum[lane];
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, off);
                if (lane >= off) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        const int excl = carry + inc - t + (warp ? wsum[warp - 1] : 0);
        if (i < nb) bsum[i] = excl;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry = excl + t;
        __syncthreads();
    }
}
// pass 3: add the scanned block totals
__global__ void k_scan_add(int *__restrict__ v, int n, const int *__restrict__ bsum) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] += bsum[i / kScanBlock];
}

// particles into their slots (order within a slot still arbitrary); counts
// run down to zero
__global__ void k_order_fill(const int *__restrict__ slot_of, int P, const int *__restrict__ start,
                             int *__restrict__ slot_cnt, int *__restrict__ bucket) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < P; g += gridDim.x * blockDim.x) {
        const int s = slot_of[g];
        if (s < 0) continue;
        const int k = atomicSub(slot_cnt + s, 1) - 1;
        bucket[start[s] + k] = g;
    }
}

// each slot sorted by reference index (slots above `cap` particles stay
// unsorted: the binning that follows reports them as cell overflow), then
// the storage-order arrays
__global__ void k_order_emit(const int *__restrict__ start, int T, int P, int cap, int *__restrict__ bucket,
                             const float *__restrict__ pos3, const int *__restrict__ rep_of_gid,
                             const SysDev *__restrict__ sys, float4 *__restrict__ staged, int *__restrict__ gid_of,
                             int *__restrict__ rep_of_sid) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < T; s += gridDim.x * blockDim.x) {
        const int a = start[s], n = (s + 1 < T ? start[s + 1] : P) - a;
        int *bk = bucket + a;
        if (n <= cap)
            for (int i = 1; i < n; i++) {  // insertion sort: a cell holds a few particles
                const int g = bk[i];
                int j = i - 1;
                while (j >= 0 && bk[j] > g) {
                    bk[j + 1] = bk[j];
                    j--;
                }
                bk[j + 1] = g;
            }
        for (int i = 0; i < n; i++) {
            const int sid = a + i, g = bk[i];
            const int r = rep_of_gid[g];
            const SysDev &S = sys[r];
            const unsigned w = (unsigned)sid | ((g - S.part_base) < S.n_big ? 0u : 1u) << 31;
            staged[sid] = make_float4(pos3[3 * (size_t)g], pos3[3 * (size_t)g + 1], pos3[3 * (size_t)g + 2],
                                      __uint_as_float(w));
            gid_of[sid] = g;
            rep_of_sid[sid] = r;
        }
    }
}

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
