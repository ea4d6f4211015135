// nlist.cuh -- neighbour-list mode of the batched engine.
//
// The 27-cell sweep of step.cuh visits ~64 candidates per particle and step,
// of which ~10 interact.  In list mode the same staged sweep runs only when a
// rebuild is needed and records, per particle, every partner closer than the
// cut distance plus a skin (in sweep order); each time step then walks that
// list.  A pair enters the force sum when its exact squared distance (the
// reference's minimum image and rounding, get_forces.cu:383-396) is below the
// squared cut distance, the same test as the sweep, so the interacting set is
// unchanged as long as no particle has moved more than half the skin since
// the list was built.  The step kernel checks that for every particle and
// raises a device flag; the rebuild kernels of the next step run only when the
// flag is set (they exit at once otherwise), so CUDA graphs need no host
// decision.
//
// State by storage id: pos[2][P] float4 (double-buffered: x, y, z and
// w = storage id | species << 31), positions at the last build, the lists
// [kMaxNbr][P] (slot-major: the threads of a warp read consecutive words),
// list lengths, plus the compensated remainder and FP64 displacement shared
// with the sweep path.  Cell buckets (cnt / pos of buffer 0) are rebuilt
// from the by-id positions for list builds and observation passes.
#pragma once

namespace bd {

constexpr int kMaxNbr = 64;
#ifndef BD_LIST_GATHER
#define BD_LIST_GATHER 4  // list partners whose positions are in flight together
#endif
#ifndef BD_LIST_PIPE
#define BD_LIST_PIPE 1       // load the next chunk's list words under this chunk's gathers
#endif
#ifndef BD_LIST_THREADS
#define BD_LIST_THREADS 256  // CTA size of the list step
#endif
#ifndef BD_LIST_MINB
#define BD_LIST_MINB 4       // resident CTAs per SM asked of the register allocator (64 registers)
#endif

struct ListArgs {
    const SysDev *sys;
    const int *rep_of_sid;
    const int *gid_of;
    int np;
    const float4 *pos_in;   // by storage id, this step
    float4 *pos_out;        // by storage id, next step
    float *lo_x, *lo_y, *lo_z;
    double *dsp_x, *dsp_y, *dsp_z;
    const int *nbr;         // [kMaxNbr][np]
    const int *nnb;         // [np]
    const float4 *pbuild;   // positions at the last build
    int *flag;              // [R + 1]: flag[r] replica r needs a rebuild, flag[R] any does
    int nrep;
    double *x0;
    void *curand_states;
    const float *noise;
    unsigned long long *rn_ring, *rn_lcg;
    long long rn_ni0;
    unsigned *status;
    long long ni_first;
    uint32_t rng_stream;
    int *nbr_count;              // census: interacting partners per gid
    unsigned long long *nbr_hash;
};

// minimum image of the reference (d - L floor(d / L + 1/2), float), exact
// shortcut when |d / L| < 0.49
__device__ __forceinline__ float min_image_fast(float d, float L, float Linv) {
    return fabsf(__fmul_rn(Linv, d)) < 0.49f ? d : min_image_f(d, L, Linv);
}

// ------------------------------------------------------------- rebuild
__global__ void k_list_clear(int *cnt, long long C, const int *flag) {
    if (*flag == 0) return;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < C; c += (long long)gridDim.x * blockDim.x)
        cnt[c] = 0;
}

// cell buckets from the by-id positions (same binning as the step kernels)
// of the replicas whose flag is set (every replica when rflag is null)
__global__ void k_list_bin(const float4 *__restrict__ pos_sid, int P, const int *__restrict__ rep_of_sid,
                           const SysDev *sys, int *cnt, float4 *pos, int cap, unsigned *status, const int *flag,
                           const int *rflag) {
    if (*flag == 0) return;
    for (int sid = blockIdx.x * blockDim.x + threadIdx.x; sid < P; sid += gridDim.x * blockDim.x) {
        const int r = rep_of_sid[sid];
        if (rflag && rflag[r] == 0) continue;
        const float4 v = pos_sid[sid];
        const SysDev &S = sys[r];
        const int nc = S.ncell;
        int ix = (int)__fmul_rn(v.x, S.cinv), iy = (int)__fmul_rn(v.y, S.cinv), iz = (int)__fmul_rn(v.z, S.cinv);
        ix = min(max(ix, 0), nc - 1);
        iy = min(max(iy, 0), nc - 1);
        iz = min(max(iz, 0), nc - 1);
        const int cell = S.cell_base + ix + nc * (iy + nc * iz);
        const int slot = atomicAdd(cnt + cell, 1);
        if (slot < cap) pos[(size_t)cell * cap + slot] = v;
        else set_status(status, kStatCellOverflow);
    }
}

struct ListBuild {
    int *nbr;
    int *nnb;
    float4 *pbuild;
    const float4 *pos_sid;
    const int *flag;  // [R + 1] as in ListArgs
    int nrep;
};

// Lists of every home particle of each brick (grid-stride over bricks):
// the staged sweep with the squared list cut distances (sigma + skin)^2,
// partners recorded by storage id in sweep order.
__global__ void __launch_bounds__(192, 4) k_list_build(StepArgs a, ListBuild lb) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (lb.flag[lb.nrep] == 0) return;
    const int tid = threadIdx.x, T = blockDim.x;
    for (int b = blockIdx.x; b < a.nbricks; b += gridDim.x) {
        const int4 br = a.bricks[b];
        if (lb.flag[br.x] == 0) continue;  // this replica's lists are still valid (uniform over the block)
        const SysDev &S = a.sys[br.x];
        const int nc = S.ncell;
        const int wx = min(a.bx, nc - br.y), wy = min(a.by, nc - br.z), wz = min(a.bz, nc - br.w);
        const int hx = wx + 2, hy = wy + 2, nh = hx * hy * (wz + 2);
        BrickSmem sm;
        brick_smem_layout((a.bx + 2) * (a.by + 2) * (a.bz + 2), a.smax, T, &sm, smem);
        const float L = S.L;
        const int vstride = a.smax + 2;
        if (stage_brick(a, br, S, sm, S.lcut2[0], S.lcut2[1], S.lcut2[2])) {
            const int MH = sm.hstart[nh];
            for (int q = tid; q < MH; q += T) {
                const int packed = sm.home[q];
                const int si = packed & 0xffff, h = packed >> 16;
                const float mx = sm.xs[si], my = sm.ys[si], mz = sm.zs[si];
                const int tm = (int)(sm.tc[si] & 1u);
                const float *view = sm.c2v + tm * vstride;
                const f2 mxx = f2_bcast(mx), myy = f2_bcast(my), mzz = f2_bcast(mz);
                const int home_sid = sm.ssid[si];
                const bool ok_sid = (unsigned)home_sid < (unsigned)a.np;
                int cnt = 0, nq = 0;
                auto flush = [&]() {
                    for (int e = 0; e < nq; e++) {
                        if (cnt < kMaxNbr) {
                            if (ok_sid) lb.nbr[(size_t)cnt * a.np + home_sid] = sm.ssid[sm.queue[e * T + tid]];
                        } else {
                            set_status(a.status, kStatCellOverflow);
                        }
                        cnt++;
                    }
                    nq = 0;
                };
                for (int dz = -1; dz <= 1; dz++)
                    for (int dy = -1; dy <= 1; dy++) {
                        const int hr = h - 1 + hx * (dy + hy * dz);
                        const int j0 = sm.start[hr], j1 = sm.start[hr + 3];
                        if (nq + (j1 - j0) > kQueue) flush();
                        const bool wrap =
                            sm.code[hr] != kNoShift || sm.code[hr + 1] != kNoShift || sm.code[hr + 2] != kNoShift;
                        if (dy == 0 && dz == 0)
                            sweep_row<true>(sm, view, j0, j1, si, wrap, mx, my, mz, mxx, myy, mzz, L, nq);
                        else
                            sweep_row<false>(sm, view, j0, j1, si, wrap, mx, my, mz, mxx, myy, mzz, L, nq);
                    }
                flush();
                if (ok_sid) {
                    lb.nnb[home_sid] = min(cnt, kMaxNbr);
                    lb.pbuild[home_sid] = lb.pos_sid[home_sid];
                } else {
                    set_status(a.status, kStatArg);
                }
            }
        }
        __syncthreads();  // the next brick reuses the staging memory
    }
}

// clear the flags after a rebuild; builds counts replica rebuilds
__global__ void k_list_done(int *flag, int nrep, long long *builds) {
    if (flag[nrep] == 0) return;
    __syncthreads();
    for (int r = threadIdx.x; r < nrep; r += blockDim.x)
        if (flag[r]) {
            atomicAdd((unsigned long long *)builds, 1ull);
            flag[r] = 0;
        }
    __syncthreads();
    if (threadIdx.x == 0) flag[nrep] = 0;
}

// ------------------------------------------------------------- step
// One time step of every particle from its list (thread per storage id).
// Force sum in list order; update, compensated position and FP64
// displacement exactly as process_brick.
// EXTRA: some replica of the batch uses a potential other than the modified
// WCA (instantiated separately so the default kernel keeps its registers).
template <int RNG, bool EXTRA>
__global__ void __launch_bounds__(BD_LIST_THREADS, BD_LIST_MINB) k_step_list(ListArgs a, const long long *ni_base,
                                                                          int ni_off) {
    const int sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= a.np) return;
    const long long ni = *ni_base + ni_off;
    const SysDev &S = a.sys[a.rep_of_sid[sid]];
    const float L = S.L, Linv = S.Linv;
    const float4 pi = a.pos_in[sid];
    const unsigned wi = __float_as_uint(pi.w);
    const int tm = (int)(wi >> 31);
    const float sg0 = tm ? S.sig[1] : S.sig[0], sg1 = tm ? S.sig[2] : S.sig[1];
    const float c0 = tm ? S.cut2[1] : S.cut2[0], c1 = tm ? S.cut2[2] : S.cut2[1];
    // own state early: its latency overlaps the force loop
    const int gid = __ldg(a.gid_of + sid);
    float lx = a.lo_x[sid], ly = a.lo_y[sid], lz = a.lo_z[sid];
    double qx = a.dsp_x[sid], qy = a.dsp_y[sid], qz = a.dsp_z[sid];
    const float4 pb = __ldg(a.pbuild + sid);
    float fx = 0.f, fy = 0.f, fz = 0.f;
    const int n = min(a.nnb[sid], kMaxNbr);
    // partners in chunks of kGather: all list words, then all positions in
    // flight, then the pair arithmetic in list order
    constexpr int kGather = BD_LIST_GATHER;
    // the list words of the next chunk load while this chunk's positions do
    int jn[kGather];
#pragma unroll
    for (int u = 0; u < kGather; u++) jn[u] = (u < n) ? __ldg(a.nbr + (size_t)u * a.np + sid) : -1;
    for (int k0 = 0; k0 < n; k0 += kGather) {
        int jj[kGather];
        float4 pj[kGather];
#pragma unroll
        for (int u = 0; u < kGather; u++) {
            jj[u] = jn[u];
            const bool ok = (unsigned)jj[u] < (unsigned)a.np;
            if (jj[u] >= 0 && !ok) set_status(a.status, kStatArg);  // never true for consistent lists
            pj[u] = ok ? __ldg(a.pos_in + jj[u]) : make_float4(0.f, 0.f, 0.f, 0.f);
            if (!ok) jj[u] = -1;
        }
#if BD_LIST_PIPE
#pragma unroll
        for (int u = 0; u < kGather; u++) {
            const int k = k0 + kGather + u;
            jn[u] = (k < n) ? __ldg(a.nbr + (size_t)k * a.np + sid) : -1;
        }
#endif
#pragma unroll
        for (int u = 0; u < kGather; u++) {
            if (jj[u] < 0) continue;
            const float dx = min_image_fast(__fsub_rn(pj[u].x, pi.x), L, Linv);
            const float dy = min_image_fast(__fsub_rn(pj[u].y, pi.y), L, Linv);
            const float dz = min_image_fast(__fsub_rn(pj[u].z, pi.z), L, Linv);
            const float d2 = dist2_rn(dx, dy, dz);
            const bool tj = (__float_as_uint(pj[u].w) >> 31) != 0u;
            if (d2 < (tj ? c1 : c0)) {
                const float sg = tj ? sg1 : sg0;
                const float di = rsqrtf(d2);
                float g;
                if (!EXTRA || S.pot == kPotWcaModified) {
                    const float sor = di * sg;
                    const float s2 = sor * sor;
                    const float s6 = s2 * s2 * s2;
                    const float s12 = s6 * s6;
                    g = -12.0f * (s12 - s6) * (di * di);
                } else {
                    float u = 0.f;
                    g = pair_extra(S.pot, S.pp, sg, di, &u);
                }
                fx = fmaf(g, dx, fx);
                fy = fmaf(g, dy, fy);
                fz = fmaf(g, dz, fz);
            }
        }
#if !BD_LIST_PIPE
#pragma unroll
        for (int u = 0; u < kGather; u++) {
            const int k = k0 + kGather + u;
            jn[u] = (k < n) ? __ldg(a.nbr + (size_t)k * a.np + sid) : -1;
        }
#endif
    }
    if (S.fcap > 0.f) {  // capped forces for the initial relaxation
        const float fmx = fmaxf(fabsf(fx), fmaxf(fabsf(fy), fabsf(fz)));
        if (fmx > 0.f && isfinite(fmx)) {
            const float gx = fx / fmx, gy = fy / fmx, gz = fz / fmx;
            const float ng = sqrtf(gx * gx + gy * gy + gz * gz);
            if (fmx * ng > S.fcap) {
                const float sc = S.fcap / ng;
                fx = gx * sc; fy = gy * sc; fz = gz * sc;
            }
        } else if (!isfinite(fmx)) {
            fx = fy = fz = 0.f;
        }
    }
    const int pid = gid - S.part_base;
    if (ni == 0) {  // origin of the unwrapped positions (main.cu:497-506)
        qx = qy = qz = 0.0;
        a.x0[3 * (size_t)gid] = (double)pi.x + (double)lx;
        a.x0[3 * (size_t)gid + 1] = (double)pi.y + (double)ly;
        a.x0[3 * (size_t)gid + 2] = (double)pi.z + (double)lz;
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
    } else if (RNG == kRngRannew64) {
        xi = rannew64_gauss3(a.rn_ring, a.rn_lcg, sid, (size_t)a.np, ni - a.rn_ni0);
    } else {
        xi = make_float3(a.noise[3 * (size_t)gid], a.noise[3 * (size_t)gid + 1], a.noise[3 * (size_t)gid + 2]);
    }
    const float mob = S.mob[tm], dt = S.dt;
    const float amp = amplitude(step_temperature(S, ni, a.ni_first), mob, dt);
    const float ex = __fadd_rn(__fmul_rn(__fmul_rn(fx, mob), dt), __fmul_rn(amp, xi.x));
    const float ey = __fadd_rn(__fmul_rn(__fmul_rn(fy, mob), dt), __fmul_rn(amp, xi.y));
    const float ez = __fadd_rn(__fmul_rn(__fmul_rn(fz, mob), dt), __fmul_rn(amp, xi.z));
    float x = pi.x, y = pi.y, z = pi.z;
    advance_wrap(x, lx, ex, L, Linv);
    advance_wrap(y, ly, ey, L, Linv);
    advance_wrap(z, lz, ez, L, Linv);
    qx += (double)ex;
    qy += (double)ey;
    qz += (double)ez;
    a.lo_x[sid] = lx;
    a.lo_y[sid] = ly;
    a.lo_z[sid] = lz;
    a.dsp_x[sid] = qx;
    a.dsp_y[sid] = qy;
    a.dsp_z[sid] = qz;
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) set_status(a.status, kStatNumeric);
    a.pos_out[sid] = make_float4(x, y, z, pi.w);
    // skin check against the positions at the last build
    const float bx = min_image_fast(__fsub_rn(x, pb.x), L, Linv);
    const float by = min_image_fast(__fsub_rn(y, pb.y), L, Linv);
    const float bz = min_image_fast(__fsub_rn(z, pb.z), L, Linv);
    if (!(dist2_rn(bx, by, bz) <= S.skin_half2)) {
        a.flag[a.rep_of_sid[sid]] = 1;
        a.flag[a.nrep] = 1;
    }
}

// Census from the lists: interacting partners per particle and a hash of
// their reference indices, as the sweep's census pass computes them.
__global__ void k_census_list(ListArgs a, double *obs) {
    const int sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= a.np) return;
    const int r = a.rep_of_sid[sid];
    const SysDev &S = a.sys[r];
    const float L = S.L, Linv = S.Linv;
    const float4 pi = a.pos_in[sid];
    const int tm = (int)(__float_as_uint(pi.w) >> 31);
    int cnt = 0;
    unsigned long long h = 0;
    const int n = min(a.nnb[sid], kMaxNbr);
    for (int k = 0; k < n; k++) {
        const int j = a.nbr[(size_t)k * a.np + sid];
        if ((unsigned)j >= (unsigned)a.np) continue;
        const float4 pj = a.pos_in[j];
        const float dx = min_image_fast(__fsub_rn(pj.x, pi.x), L, Linv);
        const float dy = min_image_fast(__fsub_rn(pj.y, pi.y), L, Linv);
        const float dz = min_image_fast(__fsub_rn(pj.z, pi.z), L, Linv);
        const int pt = tm + (int)(__float_as_uint(pj.w) >> 31);
        if (dist2_rn(dx, dy, dz) < S.cut2[pt]) {
            cnt++;
            h += (unsigned long long)(a.gid_of[j] - S.part_base + 1) * 0x9E3779B97F4A7C15ull;
        }
    }
    const int gid = a.gid_of[sid];
    a.nbr_count[gid] = cnt;
    a.nbr_hash[gid] = h;
    atomicAdd(obs + (size_t)r * kObsCount + kObsNbr, (double)cnt);
}

}  // namespace bd
