// step.cuh -- the fused per-step kernel of the batched engine.
//
// One CTA per brick of cells of one replica.  One reference time step
// (main.cu:494-588: update_ermak_dev x2, cell clears + cell_locate_dev x2,
// force clears + get_forces_*_dev x4) becomes one pass over the brick:
//   1. stage the brick's cells plus a one-cell halo into shared memory: cell
//      counts -> block scan -> one independent load per staged particle ->
//      scatter to its rank within the cell by storage id (every force sum then
//      has a fixed order, independent of brick shape and batching);
//   2. every home particle sweeps the 9 rows of 3 contiguous neighbour cells
//      two candidates at a time with packed f32x2 arithmetic; the cut-off
//      test rounds like the reference (get_forces.cu:383-396) and reads the
//      squared cut distance from a per-home-species view of the staged
//      particles (bb, bs, ss without a per-candidate select); interacting
//      partners are queued and evaluated after the sweep;
//   3. Ermak-McCammon update of that particle with counter-based Gaussians,
//      compensated FP32 position + FP64 displacement;
//   4. the new position is binned into the next count/position buffer and
//      the third count buffer is cleared for the brick's own cells.
// Forces never touch global memory.
#pragma once

namespace bd {

constexpr int kQueue = 72;            // queue length per thread; >= one row (3 cells x 24 slots)
constexpr unsigned kNoShift = 0x15u;  // shift code of a halo cell that did not wrap

typedef unsigned long long f2;  // two floats in one 64-bit register (lo, hi)
__device__ __forceinline__ f2 f2_bcast(float v) {
    f2 r;
    asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(v));
    return r;
}
__device__ __forceinline__ void f2_split(f2 v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
    f2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 f2_sub(f2 a, f2 b) {
    f2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 f2_make(float lo, float hi) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

struct BrickSmem {
    int *start;             // [nh+1] staged-particle prefix over halo cells
    int *hstart;            // [nh+1] home-particle prefix over halo cells
    int *gc;                // [nh]   global cell index
    unsigned char *code;    // [nh]   periodic shift code (2 bits per axis)
    float *xs, *ys, *zs;    // [smax+2] staged positions, sorted by storage id in each cell
    float *c2v;             // [2][smax+2] squared cut distance towards each staged
                            //   particle, seen from a big / a small home particle
    unsigned char *tc;      // [smax] species | shift code << 1
    int *ssid;              // [smax] storage id
    int *home;              // [smax] staged index | halo cell << 16, per home particle
    float4 *raw;            // [smax] unsorted staging   (shares memory with queue)
    unsigned short *queue;  // [kQueue][threads]          (shares memory with raw)
    unsigned short *hslot;  // [smax] halo cell of each unsorted slot
    double *red;
    int *tmp;
    float *amp;
};

// Layout shared by host (size) and device (carve).
__host__ __device__ inline size_t brick_smem_layout(int nh, int smax, int threads, BrickSmem *s,
                                                    unsigned char *base) {
    size_t off = 0;
    auto take = [&](size_t bytes, size_t align) -> unsigned char * {
        off = (off + align - 1) & ~(align - 1);
        unsigned char *q = base ? base + off : nullptr;
        off += bytes;
        return q;
    };
    const size_t ns = (size_t)smax + 2;
    size_t uni = (size_t)smax * 16;
    if ((size_t)kQueue * threads * 2 > uni) uni = (size_t)kQueue * threads * 2;
    unsigned char *p_uni = take(uni, 16);
    unsigned char *p_xs = take(ns * 4, 16);
    unsigned char *p_ys = take(ns * 4, 16);
    unsigned char *p_zs = take(ns * 4, 16);
    unsigned char *p_c2 = take(2 * ns * 4, 16);
    unsigned char *p_start = take((size_t)(nh + 1) * 4, 4);
    unsigned char *p_hstart = take((size_t)(nh + 1) * 4, 4);
    unsigned char *p_gc = take((size_t)nh * 4, 4);
    unsigned char *p_ssid = take((size_t)smax * 4, 4);
    unsigned char *p_home = take((size_t)smax * 4, 4);
    unsigned char *p_hslot = take((size_t)smax * 2, 4);
    unsigned char *p_tc = take((size_t)smax, 4);
    unsigned char *p_code = take((size_t)nh, 4);
    unsigned char *p_red = take(32 * 8, 8);
    unsigned char *p_tmp = take(64 * 4, 4);
    unsigned char *p_amp = take(16, 4);
    if (s) {
        s->raw = (float4 *)p_uni; s->queue = (unsigned short *)p_uni;
        s->xs = (float *)p_xs; s->ys = (float *)p_ys; s->zs = (float *)p_zs; s->c2v = (float *)p_c2;
        s->start = (int *)p_start; s->hstart = (int *)p_hstart; s->gc = (int *)p_gc; s->ssid = (int *)p_ssid;
        s->home = (int *)p_home; s->hslot = (unsigned short *)p_hslot; s->tc = p_tc; s->code = p_code;
        s->red = (double *)p_red; s->tmp = (int *)p_tmp; s->amp = (float *)p_amp;
    }
    return off;
}
__host__ __device__ inline size_t brick_smem_bytes(int nh, int smax, int threads) {
    return brick_smem_layout(nh, smax, threads, nullptr, nullptr);
}

// periodic shift of a staged particle along one axis: code bits -> -L, 0, +L
__device__ __forceinline__ float axis_shift(unsigned tc, int axis, float L) {
    const int c = (int)((tc >> (1 + 2 * axis)) & 3u) - 1;
    return __int2float_rn(c) * L;  // exact: c in {-1, 0, 1}
}

struct PairSums {
    float fx = 0.f, fy = 0.f, fz = 0.f, pot = 0.f, vir = 0.f;
    int nbr = 0;
    unsigned long long hsh = 0;
};

// Evaluate the queued partners of one home particle in queue order.
template <bool OBS, bool CENSUS>
__device__ __forceinline__ void flush_queue(const BrickSmem &sm, const StepArgs &a, int nq, float mx, float my,
                                            float mz, int tm, float L, float sgbb, float sgbs, float sgss,
                                            int part_base, int pot, const float *pp, PairSums &ps) {
    const int T = blockDim.x, tid = threadIdx.x;
    for (int e = 0; e < nq; e++) {
        const int j = sm.queue[e * T + tid];
        const unsigned tcj = sm.tc[j];
        const float dx = __fsub_rn(__fsub_rn(sm.xs[j], mx), axis_shift(tcj, 0, L));
        const float dy = __fsub_rn(__fsub_rn(sm.ys[j], my), axis_shift(tcj, 1, L));
        const float dz = __fsub_rn(__fsub_rn(sm.zs[j], mz), axis_shift(tcj, 2, L));
        const float d2 = dist2_rn(dx, dy, dz);
        const int pt = tm + (int)(tcj & 1u);
        const float sg = pt == 0 ? sgbb : (pt == 1 ? sgbs : sgss);
        // WCA-modified pair (potentials.cu:137-147) in terms of 1/r, or the
        // replica's other potential
        const float di = rsqrtf(d2);
        float g, u = 0.f;
        if (pot == kPotWcaModified) {
            const float sor = di * sg;
            const float s2 = sor * sor;
            const float s6 = s2 * s2 * s2;
            const float s12 = s6 * s6;
            g = -12.0f * (s12 - s6) * (di * di);  // pair force = g d
            u = s12 - 2.0f * s6 + 1.0f;
        } else {
            g = pair_extra(pot, pp, sg, di, &u);
        }
        ps.fx = fmaf(g, dx, ps.fx);
        ps.fy = fmaf(g, dy, ps.fy);
        ps.fz = fmaf(g, dz, ps.fz);
        if (OBS) {
            ps.pot += u;
            ps.vir = fmaf(-0.5f * g, d2, ps.vir);
        }
        if (CENSUS) {
            ps.nbr++;
            const int sj = sm.ssid[j];
            const int gidn = ((unsigned)sj < (unsigned)a.np ? __ldg(a.gid_of + sj) : part_base) - part_base;
            ps.hsh += (unsigned long long)(gidn + 1) * 0x9E3779B97F4A7C15ull;
        }
    }
}

// One row of candidates [j0, j1) against home particle si.  MID: the row
// holding the home particle itself (excluded by index, like the reference's
// nn == mm test).  Rows that cross the periodic box take the scalar path with
// the per-candidate shift; all others are swept two candidates at a time.
template <bool MID>
__device__ __forceinline__ void sweep_row(const BrickSmem &sm, const float *view, int j0, int j1, int si, bool wrap,
                                          float mx, float my, float mz, f2 mxx, f2 myy, f2 mzz, float L, int &nq) {
    const int T = blockDim.x, tid = threadIdx.x;
    unsigned short *q = sm.queue + tid;
    if (wrap) {
        for (int j = j0; j < j1; j++) {
            const unsigned tcj = sm.tc[j];
            const float dx = __fsub_rn(__fsub_rn(sm.xs[j], mx), axis_shift(tcj, 0, L));
            const float dy = __fsub_rn(__fsub_rn(sm.ys[j], my), axis_shift(tcj, 1, L));
            const float dz = __fsub_rn(__fsub_rn(sm.zs[j], mz), axis_shift(tcj, 2, L));
            const bool hit = dist2_rn(dx, dy, dz) < view[j] && (!MID || j != si);
            if (hit) q[(nq++) * T] = (unsigned short)j;
        }
        return;
    }
#pragma unroll 2
    for (int j = j0 & ~1; j < j1; j += 2) {
        const f2 dx = f2_sub(*reinterpret_cast<const f2 *>(sm.xs + j), mxx);
        const f2 dy = f2_sub(*reinterpret_cast<const f2 *>(sm.ys + j), myy);
        const f2 dz = f2_sub(*reinterpret_cast<const f2 *>(sm.zs + j), mzz);
        const f2 d2 = f2_add(f2_add(f2_mul(dx, dx), f2_mul(dy, dy)), f2_mul(dz, dz));
        float d2a, d2b, ca, cb;
        f2_split(d2, d2a, d2b);
        f2_split(*reinterpret_cast<const f2 *>(view + j), ca, cb);
        const bool ha = d2a < ca && j >= j0 && (!MID || j != si);
        const bool hb = d2b < cb && j + 1 < j1 && (!MID || j + 1 != si);
        if (ha) q[(nq++) * T] = (unsigned short)j;
        if (hb) q[(nq++) * T] = (unsigned short)(j + 1);
    }
}

// Stage the cells of brick `br` plus a one-cell halo into shared memory
// (steps 1-2 above) with the squared cut distances c2bb, c2bs, c2ss in the
// per-home-species views.  Returns false (status set) when the staging
// capacity is exceeded.  On return the block is synchronised and sm.start /
// sm.hstart hold the staged and home prefixes (totals M, MH at [nh]).
__device__ __forceinline__ bool stage_brick(const StepArgs &a, const int4 br, const SysDev &S, const BrickSmem &sm,
                                            float c2bb, float c2bs, float c2ss) {
    const int nc = S.ncell;
    const int ox = br.y, oy = br.z, oz = br.w;
    const int wx = min(a.bx, nc - ox), wy = min(a.by, nc - oy), wz = min(a.bz, nc - oz);
    const int hx = wx + 2, hy = wy + 2, hz = wz + 2, nh = hx * hy * hz;
    const int tid = threadIdx.x, T = blockDim.x;
    const int vstride = a.smax + 2;
    const int cell_base = S.cell_base;
    // 1. halo cells: global index, clamped count, periodic shift code
    for (int h = tid; h < nh; h += T) {
        const int lx = h % hx, ly = (h / hx) % hy, lz = h / (hx * hy);
        int gx = ox + lx - 1, gy = oy + ly - 1, gz = oz + lz - 1;
        int sx = 0, sy = 0, sz = 0;
        if (gx < 0) { gx += nc; sx = 1; } else if (gx >= nc) { gx -= nc; sx = -1; }
        if (gy < 0) { gy += nc; sy = 1; } else if (gy >= nc) { gy -= nc; sy = -1; }
        if (gz < 0) { gz += nc; sz = 1; } else if (gz >= nc) { gz -= nc; sz = -1; }
        const int gc = cell_base + gx + nc * (gy + nc * gz);
        int c = __ldcg(a.cnt_in + gc);
        if (c > a.cap) { set_status(a.status, kStatCellOverflow); c = a.cap; }
        if (c < 0) { set_status(a.status, kStatArg); c = 0; }  // never true for consistent buffers
        const bool home = lx >= 1 && lx <= wx && ly >= 1 && ly <= wy && lz >= 1 && lz <= wz;
        sm.gc[h] = gc;
        sm.start[h] = c;
        sm.hstart[h] = home ? c : 0;
        sm.code[h] = (unsigned char)((sx + 1) | ((sy + 1) << 2) | ((sz + 1) << 4));
    }
    __syncthreads();
    block_scan2(sm.start, sm.hstart, nh, sm.tmp);
    const int M = sm.start[nh];
    if (M > a.smax) {  // staging capacity exceeded: flag and leave the brick
        if (tid == 0) set_status(a.status, kStatCellOverflow);
        return false;
    }
    // 2a. one independent load per staged particle (unsorted)
    for (int t = tid; t < M; t += T) {
        int lo = 0, hi = nh - 1;  // last halo cell with start <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sm.start[mid] <= t) lo = mid; else hi = mid - 1;
        }
        sm.raw[t] = __ldcg(a.pos_in + (size_t)sm.gc[lo] * a.cap + (t - sm.start[lo]));
        sm.hslot[t] = (unsigned short)lo;
    }
    if (tid < 2) {  // padding read by the paired sweep past the last staged particle
        sm.xs[M + tid] = 1e30f; sm.ys[M + tid] = 1e30f; sm.zs[M + tid] = 1e30f;
        sm.c2v[M + tid] = 0.f; sm.c2v[vstride + M + tid] = 0.f;
    }
    __syncthreads();
    // 2b. scatter to the rank within the cell by storage id; list home particles
    for (int t = tid; t < M; t += T) {
        const int h = sm.hslot[t];
        const int st = sm.start[h], c = sm.start[h + 1] - st;
        const float4 v = sm.raw[t];
        const unsigned w = __float_as_uint(v.w), key = w & 0x7fffffffu;
        int rank = 0;
        for (int k = 0; k < c; k++) rank += (__float_as_uint(sm.raw[st + k].w) & 0x7fffffffu) < key;
        const int d = st + rank;
        const unsigned tn = w >> 31;
        sm.xs[d] = v.x;
        sm.ys[d] = v.y;
        sm.zs[d] = v.z;
        sm.c2v[d] = tn ? c2bs : c2bb;
        sm.c2v[vstride + d] = tn ? c2ss : c2bs;
        sm.tc[d] = (unsigned char)(tn | ((unsigned)sm.code[h] << 1));
        sm.ssid[d] = (int)key;
        const int hs = sm.hstart[h];
        if (sm.hstart[h + 1] > hs) sm.home[hs + rank] = d | (h << 16);
    }
    __syncthreads();

    return true;
}

template <int RNG, bool OBS, bool CENSUS>
__device__ void process_brick(const StepArgs &a, int bidx, long long ni, unsigned char *smem_raw) {
    const int4 br = a.bricks[bidx];
    const SysDev &S = a.sys[br.x];
    const int nc = S.ncell;
    const int ox = br.y, oy = br.z, oz = br.w;
    const int wx = min(a.bx, nc - ox), wy = min(a.by, nc - oy), wz = min(a.bz, nc - oz);
    const int hx = wx + 2, hy = wy + 2, hz = wz + 2, nh = hx * hy * hz;
    BrickSmem sm;
    brick_smem_layout((a.bx + 2) * (a.by + 2) * (a.bz + 2), a.smax, blockDim.x, &sm, smem_raw);
    const int tid = threadIdx.x, T = blockDim.x;
    const int vstride = a.smax + 2;
    const float L = S.L, Linv = S.Linv, cinv = S.cinv;
    const int cell_base = S.cell_base, part_base = S.part_base;
    const float c2bb = S.cut2[0], c2bs = S.cut2[1], c2ss = S.cut2[2];
    const float sgbb = S.sig[0], sgbs = S.sig[1], sgss = S.sig[2];

    if (tid == 0) {
        const float Tm = step_temperature(S, ni, a.ni_first);
        sm.amp[0] = amplitude(Tm, S.mob[0], S.dt);
        sm.amp[1] = amplitude(Tm, S.mob[1], S.dt);
    }
    if (!stage_brick(a, br, S, sm, c2bb, c2bs, c2ss)) return;
    const int MH = sm.hstart[nh];
    // 3. forces and update, one thread per home particle
    double acc_pb = 0, acc_ps = 0, acc_v = 0, acc_mb = 0, acc_ms = 0, acc_fs = 0, acc_nb = 0;
    for (int q = tid; q < MH; q += T) {
        const int packed = sm.home[q];
        const int si = packed & 0xffff, h = packed >> 16;
        const float mx = sm.xs[si], my = sm.ys[si], mz = sm.zs[si];
        const int tm = (int)(sm.tc[si] & 1u);
        const float *view = sm.c2v + tm * vstride;
        const f2 mxx = f2_bcast(mx), myy = f2_bcast(my), mzz = f2_bcast(mz);
        PairSums ps;
        int nq = 0;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++) {
                const int hr = h - 1 + hx * (dy + hy * dz);  // row of 3 contiguous halo cells
                const int j0 = sm.start[hr], j1 = sm.start[hr + 3];
                if (nq + (j1 - j0) > kQueue) {
                    flush_queue<OBS, CENSUS>(sm, a, nq, mx, my, mz, tm, L, sgbb, sgbs, sgss, part_base, S.pot, S.pp, ps);
                    nq = 0;
                }
                const bool wrap =
                    sm.code[hr] != kNoShift || sm.code[hr + 1] != kNoShift || sm.code[hr + 2] != kNoShift;
                if (dy == 0 && dz == 0)
                    sweep_row<true>(sm, view, j0, j1, si, wrap, mx, my, mz, mxx, myy, mzz, L, nq);
                else
                    sweep_row<false>(sm, view, j0, j1, si, wrap, mx, my, mz, mxx, myy, mzz, L, nq);
            }
        flush_queue<OBS, CENSUS>(sm, a, nq, mx, my, mz, tm, L, sgbb, sgbs, sgss, part_base, S.pot, S.pp, ps);
        float fx = ps.fx, fy = ps.fy, fz = ps.fz;
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
        const int sid = sm.ssid[si];
        if ((unsigned)sid >= (unsigned)a.np) {  // never true for consistent buffers
            set_status(a.status, kStatArg);
            continue;
        }
        const int gid = __ldg(a.gid_of + sid);
        const int pid = gid - part_base;
        float lx = __ldcg(a.lo_x + sid), ly = __ldcg(a.lo_y + sid), lz = __ldcg(a.lo_z + sid);
        double qx = __ldcg(a.dsp_x + sid), qy = __ldcg(a.dsp_y + sid), qz = __ldcg(a.dsp_z + sid);
        if (OBS) {
            if (tm == 0) acc_pb += ps.pot; else acc_ps += ps.pot;
            acc_v += ps.vir;
            const double r2 = qx * qx + qy * qy + qz * qz;
            if (tm == 0) {
                acc_mb += r2;
                const double r = sqrt(r2), qr = (double)a.qmax * r;
                acc_fs += (r > 0.0) ? sin(qr) / qr : 1.0;
            } else {
                acc_ms += r2;
            }
            a.snap[gid] = make_float4(mx, my, mz, __int_as_float(tm));
        }
        if (CENSUS) {
            acc_nb += ps.nbr;
            a.nbr_count[gid] = ps.nbr;
            a.nbr_hash[gid] = ps.hsh;
        }
        if (!a.do_update) continue;
        if (ni == 0) {  // origin of the unwrapped positions (main.cu:497-506)
            qx = qy = qz = 0.0;
            a.x0[3 * (size_t)gid] = (double)mx + (double)lx;
            a.x0[3 * (size_t)gid + 1] = (double)my + (double)ly;
            a.x0[3 * (size_t)gid + 2] = (double)mz + (double)lz;
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
        const float mob = S.mob[tm], amp = sm.amp[tm], dt = S.dt;
        // displacement: F*mob*dt + amp*xi (update_ermak.cu:122-134), rounded as written
        const float ex = __fadd_rn(__fmul_rn(__fmul_rn(fx, mob), dt), __fmul_rn(amp, xi.x));
        const float ey = __fadd_rn(__fmul_rn(__fmul_rn(fy, mob), dt), __fmul_rn(amp, xi.y));
        const float ez = __fadd_rn(__fmul_rn(__fmul_rn(fz, mob), dt), __fmul_rn(amp, xi.z));
        float x = mx, y = my, z = mz;
        advance_wrap(x, lx, ex, L, Linv);
        advance_wrap(y, ly, ey, L, Linv);
        advance_wrap(z, lz, ez, L, Linv);
        qx += (double)ex;
        qy += (double)ey;
        qz += (double)ez;
        __stcg(a.lo_x + sid, lx);
        __stcg(a.lo_y + sid, ly);
        __stcg(a.lo_z + sid, lz);
        __stcg(a.dsp_x + sid, qx);
        __stcg(a.dsp_y + sid, qy);
        __stcg(a.dsp_z + sid, qz);
        int ix = (int)__fmul_rn(x, cinv), iy = (int)__fmul_rn(y, cinv), iz = (int)__fmul_rn(z, cinv);
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) {
            set_status(a.status, kStatNumeric);
            ix = iy = iz = 0;
        }
        ix = min(max(ix, 0), nc - 1);
        iy = min(max(iy, 0), nc - 1);
        iz = min(max(iz, 0), nc - 1);
        const int cell = cell_base + ix + nc * (iy + nc * iz);
        const int slot = atomicAdd(a.cnt_out + cell, 1);
        const unsigned wout = (unsigned)sid | ((unsigned)tm << 31);
        if (slot < a.cap)
            __stcg(a.pos_out + (size_t)cell * a.cap + slot, make_float4(x, y, z, __uint_as_float(wout)));
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
    // clear the third count buffer for this brick's own cells
    if (a.do_update)
        for (int h = tid; h < nh; h += T) {
            const int lx = h % hx, ly = (h / hx) % hy, lz = h / (hx * hy);
            if (lx >= 1 && lx <= wx && ly >= 1 && ly <= wy && lz >= 1 && lz <= wz) a.cnt_clr[sm.gc[h]] = 0;
        }
}

template <int RNG, bool OBS, bool CENSUS>
__global__ void __launch_bounds__(192, 4) k_step(StepArgs a, const long long *ni_base, int ni_off) {
    extern __shared__ __align__(16) unsigned char smem[];
    const long long ni = *ni_base + ni_off;
    process_brick<RNG, OBS, CENSUS>(a, blockIdx.x, ni, smem);
}

// Persistent mode: each thread-block cluster owns the bricks of a bin of
// replicas and advances them `nsteps` time steps in one launch; between
// steps the cluster synchronises with the hardware cluster barrier
// (release/acquire at cluster scope orders the global-memory count and
// position buffers, which are read and written at L2 with .cg accesses).
// Replicas never span clusters, so no other synchronisation is needed.
// Every CTA of a cluster executes the same number of barriers.
template <int RNG>
__global__ void __launch_bounds__(192, 4) k_step_persistent(StepArgs a, const long long *ni_base, int nsteps) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned cid, rank, csz;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(cid));
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(csz));
    const long long ni0 = *ni_base;
    const int b0 = a.cl_start[cid], b1 = a.cl_start[cid + 1];
    for (int s = 0; s < nsteps; s++) {
        StepArgs as = a;
        const int c = (a.cur0 + s) % 3;
        as.cnt_in = a.cnt3[c];
        as.pos_in = a.pos3[c];
        as.cnt_out = a.cnt3[(c + 1) % 3];
        as.pos_out = a.pos3[(c + 1) % 3];
        as.cnt_clr = a.cnt3[(c + 2) % 3];
        for (int b = b0 + (int)rank; b < b1; b += (int)csz) {
            process_brick<RNG, false, false>(as, a.cl_bricks[b], ni0 + s, smem);
            __syncthreads();
        }
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
}

}  // namespace bd
