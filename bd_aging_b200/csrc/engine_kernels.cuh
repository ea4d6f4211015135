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

// shared-memory carve for a brick with nh halo cells and smax staged particles
struct BrickSmem {
    int *start, *hstart, *gc, *home;
    unsigned char *code;
    float4 *sp;
    double *red;
    int *tmp;
    float *amp;
};
__host__ __device__ inline size_t brick_smem_bytes(int nh, int smax) {
    size_t b = 0;
    b += (size_t)(nh + 1) * 4 * 2;        // start, hstart
    b += (size_t)nh * 4;                  // gc
    b += (size_t)smax * 4;                // home
    b += ((size_t)nh + 15) & ~(size_t)15; // code
    b = (b + 15) & ~(size_t)15;
    b += (size_t)smax * 16;               // sp
    b += 32 * 8 + 64 * 4 + 16;            // red, tmp, amp
    return b;
}
__device__ inline BrickSmem carve(unsigned char *base, int nh, int smax) {
    BrickSmem s;
    unsigned char *p = base;
    s.start = (int *)p; p += (size_t)(nh + 1) * 4;
    s.hstart = (int *)p; p += (size_t)(nh + 1) * 4;
    s.gc = (int *)p; p += (size_t)nh * 4;
    s.home = (int *)p; p += (size_t)smax * 4;
    s.code = p; p += ((size_t)nh + 15) & ~(size_t)15;
    p = (unsigned char *)(((uintptr_t)p + 15) & ~(uintptr_t)15);
    s.sp = (float4 *)p; p += (size_t)smax * 16;
    s.red = (double *)p; p += 32 * 8;
    s.tmp = (int *)p; p += 64 * 4;
    s.amp = (float *)p;
    return s;
}

// ------------------------------------------------------------- the step
template <int RNG, bool OBS, bool CENSUS>
__device__ void process_brick(const StepArgs &a, int bidx, long long ni, unsigned char *smem_raw) {
    const int4 br = a.bricks[bidx];
    const SysDev &S = a.sys[br.x];
    const int nc = S.ncell;
    const int ox = br.y, oy = br.z, oz = br.w;
    const int wx = min(a.bx, nc - ox), wy = min(a.by, nc - oy), wz = min(a.bz, nc - oz);
    const int hx = wx + 2, hy = wy + 2, hz = wz + 2, nh = hx * hy * hz;
    BrickSmem sm = carve(smem_raw, (a.bx + 2) * (a.by + 2) * (a.bz + 2), a.smax);
    const int tid = threadIdx.x, T = blockDim.x;
    const float L = S.L;

    if (tid == 0) {
        float Tm = step_temperature(S, ni, a.ni_first);
        sm.amp[0] = amplitude(Tm, S.mob[0], S.dt);
        sm.amp[1] = amplitude(Tm, S.mob[1], S.dt);
    }
    // 1. halo cells: global index, clamped count, periodic shift code
    for (int h = tid; h < nh; h += T) {
        int lx = h % hx, ly = (h / hx) % hy, lz = h / (hx * hy);
        int gx = ox + lx - 1, gy = oy + ly - 1, gz = oz + lz - 1;
        int sx = 0, sy = 0, sz = 0;
        if (gx < 0) { gx += nc; sx = 1; } else if (gx >= nc) { gx -= nc; sx = -1; }
        if (gy < 0) { gy += nc; sy = 1; } else if (gy >= nc) { gy -= nc; sy = -1; }
        if (gz < 0) { gz += nc; sz = 1; } else if (gz >= nc) { gz -= nc; sz = -1; }
        int gc = S.cell_base + gx + nc * (gy + nc * gz);
        int c = __ldcg(a.cnt_in + gc);
        if (c > a.cap) { set_status(a.status, kStatCellOverflow); c = a.cap; }
        bool home = lx >= 1 && lx <= wx && ly >= 1 && ly <= wy && lz >= 1 && lz <= wz;
        sm.gc[h] = gc;
        sm.start[h] = c;
        sm.hstart[h] = home ? c : 0;
        sm.code[h] = (unsigned char)((sx + 1) | ((sy + 1) << 2) | ((sz + 1) << 4));
    }
    __syncthreads();
    block_scan2(sm.start, sm.hstart, nh, sm.tmp);
    const int M = sm.start[nh], MH = sm.hstart[nh];
    if (M > a.smax) {  // staging capacity exceeded: flag and leave the brick
        if (tid == 0) set_status(a.status, kStatCellOverflow);
        return;
    }
    // 2. stage positions; sort each cell by storage id; list home particles
    for (int h = tid; h < nh; h += T) {
        const int st = sm.start[h], c = sm.start[h + 1] - st;
        const float4 *src = a.pos_in + (size_t)sm.gc[h] * a.cap;
        for (int k = 0; k < c; k++) {
            float4 v = __ldcg(src + k);
            unsigned key = __float_as_uint(v.w) & 0x7fffffffu;
            int j = st + k - 1;
            while (j >= st && (__float_as_uint(sm.sp[j].w) & 0x7fffffffu) > key) { sm.sp[j + 1] = sm.sp[j]; j--; }
            sm.sp[j + 1] = v;
        }
        const int hs = sm.hstart[h];
        if (sm.hstart[h + 1] > hs)
            for (int k = 0; k < c; k++) sm.home[hs + k] = (st + k) | (h << 16);
    }
    __syncthreads();

    // 3. forces + update per home particle
    const float c2bb = S.cut2[0], c2bs = S.cut2[1], c2ss = S.cut2[2];
    const float sgbb = S.sig[0], sgbs = S.sig[1], sgss = S.sig[2];
    double acc_pb = 0, acc_ps = 0, acc_v = 0, acc_mb = 0, acc_ms = 0, acc_fs = 0, acc_nb = 0;
    for (int q = tid; q < MH; q += T) {
        const int packed = sm.home[q];
        const int si = packed & 0xffff, h = packed >> 16;
        float4 m = sm.sp[si];
        const unsigned wm = __float_as_uint(m.w);
        const int tm = wm >> 31;
        float fx = 0.f, fy = 0.f, fz = 0.f, pot = 0.f, vir = 0.f;
        int nbr = 0;
        unsigned long long nh_hash = 0;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const int hh = h + dx + hx * (dy + hy * dz);
                    const int st = sm.start[hh], en = sm.start[hh + 1];
                    if (st == en) continue;
                    const unsigned cd = sm.code[hh];
                    const int cx = (int)(cd & 3) - 1, cy = (int)((cd >> 2) & 3) - 1, cz = (int)((cd >> 4) & 3) - 1;
                    const float shx = cx == 0 ? 0.f : (cx > 0 ? L : -L);
                    const float shy = cy == 0 ? 0.f : (cy > 0 ? L : -L);
                    const float shz = cz == 0 ? 0.f : (cz > 0 ? L : -L);
                    for (int j = st; j < en; j++) {
                        const float4 n = sm.sp[j];
                        const unsigned wn = __float_as_uint(n.w);
                        if (wn == wm) continue;
                        const float ddx = __fsub_rn(__fsub_rn(n.x, m.x), shx);
                        const float ddy = __fsub_rn(__fsub_rn(n.y, m.y), shy);
                        const float ddz = __fsub_rn(__fsub_rn(n.z, m.z), shz);
                        const float d2 = dist2_rn(ddx, ddy, ddz);
                        const int pt = tm + (int)(wn >> 31);
                        const float c2 = pt == 0 ? c2bb : (pt == 1 ? c2bs : c2ss);
                        if (d2 < c2) {
                            const float sg = pt == 0 ? sgbb : (pt == 1 ? sgbs : sgss);
                            PairOut o = wca_modified_pair(sg, d2, ddx, ddy, ddz);
                            fx += o.fx;
                            fy += o.fy;
                            fz += o.fz;
                            if (OBS) { pot += o.pot; vir += o.vir; }
                            if (CENSUS) {
                                nbr++;
                                int gidn = __ldg(a.gid_of + (wn & 0x7fffffffu)) - S.part_base;
                                nh_hash += (unsigned long long)(gidn + 1) * 0x9E3779B97F4A7C15ull;
                            }
                        }
                    }
                }
        if (S.fcap > 0.f) {  // capped forces for the initial relaxation
            float fmx = fmaxf(fabsf(fx), fmaxf(fabsf(fy), fabsf(fz)));
            if (fmx > 0.f && isfinite(fmx)) {
                float gx = fx / fmx, gy = fy / fmx, gz = fz / fmx;
                float ng = sqrtf(gx * gx + gy * gy + gz * gz);
                if (fmx * ng > S.fcap) {
                    float sc = S.fcap / ng;
                    fx = gx * sc; fy = gy * sc; fz = gz * sc;
                }
            } else if (!isfinite(fmx)) {
                fx = fy = fz = 0.f;
            }
        }
        const int sid = wm & 0x7fffffff;
        const int gid = __ldg(a.gid_of + sid);
        const int pid = gid - S.part_base;
        float lx = __ldcg(a.lo_x + sid), ly = __ldcg(a.lo_y + sid), lz = __ldcg(a.lo_z + sid);
        double qx = __ldcg(a.dsp_x + sid), qy = __ldcg(a.dsp_y + sid), qz = __ldcg(a.dsp_z + sid);
        if (OBS) {
            if (tm == 0) acc_pb += pot; else acc_ps += pot;
            acc_v += vir;
            double r2 = qx * qx + qy * qy + qz * qz;
            if (tm == 0) {
                acc_mb += r2;
                double r = sqrt(r2), qr = (double)a.qmax * r;
                acc_fs += (r > 0.0) ? sin(qr) / qr : 1.0;
            } else {
                acc_ms += r2;
            }
            a.snap[gid] = make_float4(m.x, m.y, m.z, __int_as_float(tm));
        }
        if (CENSUS) {
            acc_nb += nbr;
            a.nbr_count[gid] = nbr;
            a.nbr_hash[gid] = nh_hash;
        }
        if (!a.do_update) continue;
        if (ni == 0) {  // origin of the unwrapped positions (main.cu:497-506)
            qx = qy = qz = 0.0;
            a.x0[3 * (size_t)gid] = (double)m.x + (double)lx;
            a.x0[3 * (size_t)gid + 1] = (double)m.y + (double)ly;
            a.x0[3 * (size_t)gid + 2] = (double)m.z + (double)lz;
        }
        float3 xi;
        if (RNG == kRngPhilox) {
            xi = gauss3(S.seed, (uint32_t)pid, (uint64_t)ni, a.rng_stream);
        } else if (RNG == kRngCurand) {
            curandState *stp = (curandState *)a.curand_states + gid;
            curandState st = *stp;
            xi.x = curand_normal(&st);
            xi.y = curand_normal(&st);
            xi.z = curand_normal(&st);
            *stp = st;
        } else {
            xi = make_float3(a.noise[3 * (size_t)gid], a.noise[3 * (size_t)gid + 1], a.noise[3 * (size_t)gid + 2]);
        }
        const float mob = S.mob[tm], amp = sm.amp[tm], dt = S.dt;
        // displacement: F*mob*dt + amp*xi (update_ermak.cu:122-134), rounded as written
        const float ex = __fadd_rn(__fmul_rn(__fmul_rn(fx, mob), dt), __fmul_rn(amp, xi.x));
        const float ey = __fadd_rn(__fmul_rn(__fmul_rn(fy, mob), dt), __fmul_rn(amp, xi.y));
        const float ez = __fadd_rn(__fmul_rn(__fmul_rn(fz, mob), dt), __fmul_rn(amp, xi.z));
        float x = m.x, y = m.y, z = m.z;
        advance_wrap(x, lx, ex, L, S.Linv);
        advance_wrap(y, ly, ey, L, S.Linv);
        advance_wrap(z, lz, ez, L, S.Linv);
        qx += (double)ex;
        qy += (double)ey;
        qz += (double)ez;
        __stcg(a.lo_x + sid, lx);
        __stcg(a.lo_y + sid, ly);
        __stcg(a.lo_z + sid, lz);
        __stcg(a.dsp_x + sid, qx);
        __stcg(a.dsp_y + sid, qy);
        __stcg(a.dsp_z + sid, qz);
        int ix = (int)__fmul_rn(x, S.cinv), iy = (int)__fmul_rn(y, S.cinv), iz = (int)__fmul_rn(z, S.cinv);
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) {
            set_status(a.status, kStatNumeric);
            ix = iy = iz = 0;
        }
        ix = min(max(ix, 0), nc - 1);
        iy = min(max(iy, 0), nc - 1);
        iz = min(max(iz, 0), nc - 1);
        const int cell = S.cell_base + ix + nc * (iy + nc * iz);
        const int slot = atomicAdd(a.cnt_out + cell, 1);
        if (slot < a.cap)
            __stcg(a.pos_out + (size_t)cell * a.cap + slot, make_float4(x, y, z, m.w));
        else
            set_status(a.status, kStatCellOverflow);
    }
    if (OBS || CENSUS) {
        double *o = a.obs + (size_t)br.x * kObsCount;
        double v;
        if (OBS) {
            v = block_sum(acc_pb, sm.red); if (tid == 0 && v != 0.0) atomicAdd(o + kObsPotBig, v);
            v = block_sum(acc_ps, sm.red); if (tid == 0 && v != 0.0) atomicAdd(o + kObsPotSml, v);
            v = block_sum(acc_v, sm.red); if (tid == 0 && v != 0.0) atomicAdd(o + kObsVir, v);
            v = block_sum(acc_mb, sm.red); if (tid == 0 && v != 0.0) atomicAdd(o + kObsMsdBig, v);
            v = block_sum(acc_ms, sm.red); if (tid == 0 && v != 0.0) atomicAdd(o + kObsMsdSml, v);
            v = block_sum(acc_fs, sm.red); if (tid == 0 && v != 0.0) atomicAdd(o + kObsFsBig, v);
        }
        if (CENSUS) { v = block_sum(acc_nb, sm.red); if (tid == 0 && v != 0.0) atomicAdd(o + kObsNbr, v); }
    }
    // 4. clear the third count buffer for this brick's own cells
    if (a.do_update)
        for (int h = tid; h < nh; h += T) {
            int lx = h % hx, ly = (h / hx) % hy, lz = h / (hx * hy);
            if (lx >= 1 && lx <= wx && ly >= 1 && ly <= wy && lz >= 1 && lz <= wz) a.cnt_clr[sm.gc[h]] = 0;
        }
}

template <int RNG, bool OBS, bool CENSUS>
__global__ void __launch_bounds__(256) k_step(StepArgs a, const long long *ni_base, int ni_off) {
    extern __shared__ __align__(16) unsigned char smem[];
    const long long ni = *ni_base + ni_off;
    process_brick<RNG, OBS, CENSUS>(a, blockIdx.x, ni, smem);
}

__global__ void k_advance_counter(long long *ni_base, int k) { *ni_base += k; }

// ------------------------------------------------------------- load/export
// Bin particles given in storage order (float4 w = sid | species << 31).
__global__ void k_load(const float4 *__restrict__ staged, int P, const int *__restrict__ rep_of_sid,
                       const SysDev *sys, int *cnt, float4 *pos, int cap, double *x0, const int *gid_of,
                       unsigned *st) {
    int sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= P) return;
    float4 v = staged[sid];
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
__global__ void k_export(const int *__restrict__ cnt, const float4 *__restrict__ pos, int C, int cap,
                         const int *__restrict__ gid_of, const double *__restrict__ x0,
                         const double *__restrict__ dx, const double *__restrict__ dy, const double *__restrict__ dz,
                         float *out_pos, float *out_raw, float4 *snap) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    int k = min(cnt[c], cap);
    for (int s = 0; s < k; s++) {
        float4 v = pos[(size_t)c * cap + s];
        unsigned w = __float_as_uint(v.w);
        int sid = w & 0x7fffffff, gid = gid_of[sid];
        if (out_pos) { out_pos[3 * (size_t)gid] = v.x; out_pos[3 * (size_t)gid + 1] = v.y; out_pos[3 * (size_t)gid + 2] = v.z; }
        if (out_raw) {
            out_raw[3 * (size_t)gid] = (float)(x0[3 * (size_t)gid] + dx[sid]);
            out_raw[3 * (size_t)gid + 1] = (float)(x0[3 * (size_t)gid + 1] + dy[sid]);
            out_raw[3 * (size_t)gid + 2] = (float)(x0[3 * (size_t)gid + 2] + dz[sid]);
        }
        if (snap) snap[gid] = make_float4(v.x, v.y, v.z, __int_as_float((int)(w >> 31)));
    }
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
