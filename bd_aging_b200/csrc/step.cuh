// step.cuh -- the fused per-step kernel of the batched engine.
//
// One CTA per brick of cells of one replica.  One reference time step
// (main.cu:494-588: update_ermak_dev x2, cell clears + cell_locate_dev x2,
// force clears + get_forces_*_dev x4) becomes one pass over the brick:
//   1. stage the brick's cells plus a one-cell halo into shared memory: cell
//      counts -> block scan -> one independent load per staged particle ->
//      each cell sorted by storage id (so every force sum has a fixed order);
//   2. every home particle sweeps the 9 rows of 3 contiguous neighbour cells
//      with the per-species-pair cut distances (bb, bs, ss) in one pass; the
//      cut-off test rounds like the reference (get_forces.cu:383-396) and
//      interacting partners are queued, then evaluated after the sweep so the
//      pair arithmetic runs only for lanes that need it;
//   3. Ermak-McCammon update of that particle with counter-based Gaussians,
//      compensated FP32 position + FP64 displacement;
//   4. the new position is binned into the next count/position buffer and
//      the third count buffer is cleared for the brick's own cells.
// Forces never touch global memory.
#pragma once

namespace bd {

constexpr int kQueue = 32;  // queued interacting partners per thread before a flush

struct BrickSmem {
    int *start;            // [nh+1] staged-particle prefix over halo cells
    int *hstart;           // [nh+1] home-particle prefix over halo cells
    int *gc;               // [nh]   global cell index
    unsigned char *code;   // [nh]   periodic shift code (2 bits per axis)
    float4 *sp;            // [smax] staged particles: x, y, z, w = species | code << 1
    int *ssid;             // [smax] storage id of each staged particle
    int *home;             // [smax] staged index | halo cell << 16, per home particle
    unsigned short *queue; // [kQueue][threads] interacting partners (staged index)
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
    unsigned char *p_sp = take((size_t)smax * 16, 16);
    unsigned char *p_start = take((size_t)(nh + 1) * 4, 4);
    unsigned char *p_hstart = take((size_t)(nh + 1) * 4, 4);
    unsigned char *p_gc = take((size_t)nh * 4, 4);
    unsigned char *p_ssid = take((size_t)smax * 4, 4);
    unsigned char *p_home = take((size_t)smax * 4, 4);
    unsigned char *p_queue = take((size_t)kQueue * threads * 2, 4);
    unsigned char *p_code = take((size_t)nh, 4);
    unsigned char *p_red = take(32 * 8, 8);
    unsigned char *p_tmp = take(64 * 4, 4);
    unsigned char *p_amp = take(16, 4);
    if (s) {
        s->sp = (float4 *)p_sp; s->start = (int *)p_start; s->hstart = (int *)p_hstart; s->gc = (int *)p_gc;
        s->ssid = (int *)p_ssid; s->home = (int *)p_home; s->queue = (unsigned short *)p_queue; s->code = p_code;
        s->red = (double *)p_red; s->tmp = (int *)p_tmp; s->amp = (float *)p_amp;
    }
    return off;
}
__host__ __device__ inline size_t brick_smem_bytes(int nh, int smax, int threads) {
    return brick_smem_layout(nh, smax, threads, nullptr, nullptr);
}

// periodic shift of a staged particle along one axis: code bits -> -L, 0, +L
__device__ __forceinline__ float axis_shift(unsigned w, int axis, float L) {
    const int c = (int)((w >> (1 + 2 * axis)) & 3u) - 1;
    return __int2float_rn(c) * L;  // exact: c in {-1, 0, 1}
}

struct PairSums {
    float fx = 0.f, fy = 0.f, fz = 0.f, pot = 0.f, vir = 0.f;
    int nbr = 0;
    unsigned long long hsh = 0;
};

// Evaluate the queued partners of home particle m (staged index list in
// queue column `tid`), in queue order.
template <bool OBS, bool CENSUS>
__device__ __forceinline__ void flush_queue(const BrickSmem &sm, const StepArgs &a, int nq, float4 m, int tm,
                                            bool wrapx, bool wrapy, bool wrapz, float L, float sgbb, float sgbs,
                                            float sgss, int part_base, PairSums &ps) {
    const int T = blockDim.x, tid = threadIdx.x;
    for (int e = 0; e < nq; e++) {
        const int j = sm.queue[e * T + tid];
        const float4 n = sm.sp[j];
        const unsigned wn = __float_as_uint(n.w);
        float dx = __fsub_rn(n.x, m.x), dy = __fsub_rn(n.y, m.y), dz = __fsub_rn(n.z, m.z);
        if (wrapx) dx = __fsub_rn(dx, axis_shift(wn, 0, L));
        if (wrapy) dy = __fsub_rn(dy, axis_shift(wn, 1, L));
        if (wrapz) dz = __fsub_rn(dz, axis_shift(wn, 2, L));
        const float d2 = dist2_rn(dx, dy, dz);
        const int pt = tm + (int)(wn & 1u);
        const float sg = pt == 0 ? sgbb : (pt == 1 ? sgbs : sgss);
        // WCA-modified pair (potentials.cu:137-147) in terms of 1/r
        const float di = rsqrtf(d2);
        const float sor = di * sg;
        const float s2 = sor * sor;
        const float s6 = s2 * s2 * s2;
        const float s12 = s6 * s6;
        const float g = -12.0f * (s12 - s6) * (di * di);  // pair force = g d
        ps.fx = fmaf(g, dx, ps.fx);
        ps.fy = fmaf(g, dy, ps.fy);
        ps.fz = fmaf(g, dz, ps.fz);
        if (OBS) {
            ps.pot += s12 - 2.0f * s6 + 1.0f;
            ps.vir = fmaf(-0.5f * g, d2, ps.vir);
        }
        if (CENSUS) {
            ps.nbr++;
            const int gidn = __ldg(a.gid_of + sm.ssid[j]) - part_base;
            ps.hsh += (unsigned long long)(gidn + 1) * 0x9E3779B97F4A7C15ull;
        }
    }
}

template <int RNG, bool OBS, bool CENSUS>
__device__ void process_brick(const StepArgs &a, int bidx, long long ni, unsigned char *smem_raw) {
    const int4 br = a.bricks[bidx];
    const SysDev &S = a.sys[br.x];
    const int nc = S.ncell;
    const int ox = br.y, oy = br.z, oz = br.w;
    const int wx = min(a.bx, nc - ox), wy = min(a.by, nc - oy), wz = min(a.bz, nc - oz);
    const int hx = wx + 2, hy = wy + 2, hz = wz + 2, nh = hx * hy * hz;
    const bool wrapx = ox == 0 || ox + wx == nc, wrapy = oy == 0 || oy + wy == nc, wrapz = oz == 0 || oz + wz == nc;
    BrickSmem sm;
    brick_smem_layout((a.bx + 2) * (a.by + 2) * (a.bz + 2), a.smax, blockDim.x, &sm, smem_raw);
    const int tid = threadIdx.x, T = blockDim.x;
    const float L = S.L, Linv = S.Linv, cinv = S.cinv;
    const int cell_base = S.cell_base, part_base = S.part_base;
    const float c2bb = S.cut2[0], c2bs = S.cut2[1], c2ss = S.cut2[2];
    const float sgbb = S.sig[0], sgbs = S.sig[1], sgss = S.sig[2];

    if (tid == 0) {
        const float Tm = step_temperature(S, ni, a.ni_first);
        sm.amp[0] = amplitude(Tm, S.mob[0], S.dt);
        sm.amp[1] = amplitude(Tm, S.mob[1], S.dt);
    }
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
        const bool home = lx >= 1 && lx <= wx && ly >= 1 && ly <= wy && lz >= 1 && lz <= wz;
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
    // 2. one independent load per staged particle
    for (int t = tid; t < M; t += T) {
        int lo = 0, hi = nh - 1;  // last halo cell with start <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sm.start[mid] <= t) lo = mid; else hi = mid - 1;
        }
        const float4 v = __ldcg(a.pos_in + (size_t)sm.gc[lo] * a.cap + (t - sm.start[lo]));
        const unsigned w = __float_as_uint(v.w);
        sm.sp[t] = make_float4(v.x, v.y, v.z, __uint_as_float((w >> 31) | ((unsigned)sm.code[lo] << 1)));
        sm.ssid[t] = (int)(w & 0x7fffffffu);
    }
    __syncthreads();
    // 3. sort each cell by storage id; list the home particles
    for (int h = tid; h < nh; h += T) {
        const int st = sm.start[h], c = sm.start[h + 1] - st;
        for (int k = 1; k < c; k++) {
            const int key = sm.ssid[st + k];
            const float4 v = sm.sp[st + k];
            int j = st + k - 1;
            while (j >= st && sm.ssid[j] > key) { sm.ssid[j + 1] = sm.ssid[j]; sm.sp[j + 1] = sm.sp[j]; j--; }
            sm.ssid[j + 1] = key;
            sm.sp[j + 1] = v;
        }
        const int hs = sm.hstart[h];
        if (sm.hstart[h + 1] > hs)
            for (int k = 0; k < c; k++) sm.home[hs + k] = (st + k) | (h << 16);
    }
    __syncthreads();

    // 4. forces and update, one thread per home particle
    double acc_pb = 0, acc_ps = 0, acc_v = 0, acc_mb = 0, acc_ms = 0, acc_fs = 0, acc_nb = 0;
    for (int q = tid; q < MH; q += T) {
        const int packed = sm.home[q];
        const int si = packed & 0xffff, h = packed >> 16;
        const float4 m = sm.sp[si];
        const int tm = (int)(__float_as_uint(m.w) & 1u);
        // does this particle's 27-cell neighbourhood cross the periodic box?
        const int hlx = h % hx, hly = (h / hx) % hy, hlz = h / (hx * hy);
        const bool px = wrapx && (hlx == 1 || hlx == wx), py = wrapy && (hly == 1 || hly == wy),
                   pz = wrapz && (hlz == 1 || hlz == wz);
        // cut distances squared towards a partner of the same / the other species
        const float c2same = tm == 0 ? c2bb : c2ss;
        const unsigned tmu = (unsigned)tm;
        PairSums ps;
        int nq = 0;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++) {
                const int hr = h - 1 + hx * (dy + hy * dz);  // row of 3 contiguous halo cells
                const int j0 = sm.start[hr], j1 = sm.start[hr + 3];
#pragma unroll 2
                for (int j = j0; j < j1; j++) {
                    const float4 n = sm.sp[j];
                    const unsigned wn = __float_as_uint(n.w);
                    float dx = __fsub_rn(n.x, m.x), dy_ = __fsub_rn(n.y, m.y), dz_ = __fsub_rn(n.z, m.z);
                    if (px) dx = __fsub_rn(dx, axis_shift(wn, 0, L));
                    if (py) dy_ = __fsub_rn(dy_, axis_shift(wn, 1, L));
                    if (pz) dz_ = __fsub_rn(dz_, axis_shift(wn, 2, L));
                    const float d2 = dist2_rn(dx, dy_, dz_);
                    const float c2 = ((wn ^ tmu) & 1u) ? c2bs : c2same;
                    if (d2 < c2 && j != si) {
                        sm.queue[nq * T + tid] = (unsigned short)j;
                        if (++nq == kQueue) {
                            flush_queue<OBS, CENSUS>(sm, a, nq, m, tm, px, py, pz, L, sgbb, sgbs, sgss, part_base, ps);
                            nq = 0;
                        }
                    }
                }
            }
        flush_queue<OBS, CENSUS>(sm, a, nq, m, tm, px, py, pz, L, sgbb, sgbs, sgss, part_base, ps);
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
            a.snap[gid] = make_float4(m.x, m.y, m.z, __int_as_float(tm));
        }
        if (CENSUS) {
            acc_nb += ps.nbr;
            a.nbr_count[gid] = ps.nbr;
            a.nbr_hash[gid] = ps.hsh;
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

}  // namespace bd
