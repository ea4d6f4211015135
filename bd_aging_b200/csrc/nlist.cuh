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
// decision.  (Conditional graph nodes around the rebuild kernels, switched on
// by the step kernel, measured 2% slower than these early exits.)
//
// State by storage id: pos[2][P + 1] float4 (double-buffered: x, y, z and
// w = storage id | species << 31; entry P is the zero position that list
// padding gathers), positions at the last build, the lists
// [kMaxNbr / 4][P][4] (chunks of four words per particle: a thread reads a
// gather chunk in one load, the threads of a warp consecutive chunks; padded
// to whole chunks), list lengths, the compensated remainder shared with the
// sweep path, and face crossings per axis [3][P] in place of a per-step FP64
// displacement (k_list_dsp rebuilds it for observations).  Cell buckets
// (cnt / pos of buffer 0) are rebuilt from the by-id positions for list
// builds and observation passes.
#pragma once

namespace bd {

constexpr int kMaxNbr = 64;
#ifndef BD_LIST_GATHER
#define BD_LIST_GATHER 4  // list partners whose positions are in flight together
#endif
constexpr int kGather = BD_LIST_GATHER;
// Launch variants of the list step, chosen per engine by the autotuner:
// CTA size, resident CTAs per SM asked of the register allocator (9 x 128
// threads: 56 registers; 8 x 128: 64), and whether the particle's own state
// (remainder, build position, reference index) is loaded after the force
// loop (fewer registers live in the loop, so more warps hide the gathers)
// or before it (its latency hidden under the gathers).  Each particle's
// arithmetic is the same in every variant, so results do not depend on the
// choice.  Variant 0, the default, measured fastest on the aging workload.
template <int V> struct ListVariant;
template <> struct ListVariant<0> { static constexpr int kThreads = 128, kMinBlocks = 9; static constexpr bool kLate = true; };
template <> struct ListVariant<1> { static constexpr int kThreads = 128, kMinBlocks = 8; static constexpr bool kLate = false; };
template <> struct ListVariant<2> { static constexpr int kThreads = 256, kMinBlocks = 4; static constexpr bool kLate = false; };
// 3-5: one block per replica running a whole batch of steps (k_list_replica)
template <> struct ListVariant<3> { static constexpr int kThreads = 256, kMinBlocks = 4; static constexpr bool kLate = true; };
template <> struct ListVariant<4> { static constexpr int kThreads = 512, kMinBlocks = 2; static constexpr bool kLate = true; };
template <> struct ListVariant<5> { static constexpr int kThreads = 1024, kMinBlocks = 1; static constexpr bool kLate = true; };
constexpr int kListVariants = 6;
constexpr int kListFirstPersistent = 3;
constexpr int kListBuildThreads = 256;  // CTA size of the list build
static_assert(kGather % 2 == 0 && kMaxNbr % kGather == 0, "partners are paired for f32x2 arithmetic");
static_assert(kGather == 4, "the list words of a gather chunk are one int4");
// Word k of particle sid's list.  Lists are stored in chunks of four words
// per particle, [k / 4][sid][k % 4]: a gather chunk is one 16-byte load per
// thread, consecutive threads reading consecutive chunks.
__device__ __forceinline__ size_t list_slot(int k, int sid, int np) {
    return ((size_t)(k >> 2) * np + sid) * 4 + (k & 3);
}

struct ListArgs {
    const SysDev *sys;
    const int *rep_of_sid;
    const int *gid_of;
    int np;
    const float4 *pos_in;   // by storage id, this step
    float4 *pos_out;        // by storage id, next step
    float *lo_x, *lo_y, *lo_z;
    int *img;               // [3][np]: box lengths crossed per axis since the origin
    const int *nbr;         // [kMaxNbr / 4][np][4] (list_slot)
    const int *nnb;         // [np]
    const float *amp_tab;   // [step in launch batch][R][species] noise amplitudes (k_amp_table)
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
// Work over the flagged replicas only: s_first[r] = number of work items of
// the flagged replicas before r (per replica: its particles, cells or
// bricks), built in shared memory by the block; returns the total.
constexpr int kSchedMaxRep = 1024;
enum SchedItem { kItemParticle = 0, kItemCell = 1, kItemBrick = 2 };
__device__ __forceinline__ int sched_count(const SysDev &S, int item) {
    return item == kItemParticle ? S.n : item == kItemCell ? S.ncell * S.ncell * S.ncell : S.nbx * S.nby * S.nbz;
}
__device__ __forceinline__ int sched_first(const SysDev &S, int item) {
    return item == kItemParticle ? S.part_base : item == kItemCell ? S.cell_base : S.brick_base;
}
__device__ int flagged_prefix(const int *__restrict__ rflag, int nrep, const SysDev *__restrict__ sys, int item,
                              int *s_first) {
    const int tid = threadIdx.x, T = blockDim.x;
    for (int r = tid; r < nrep; r += T) s_first[r + 1] = rflag[r] ? sched_count(sys[r], item) : 0;
    if (tid == 0) s_first[0] = 0;
    __syncthreads();
    if (tid < 32) {  // inclusive scan of s_first[1 .. nrep] by warp 0
        int carry = 0;
        for (int base = 1; base <= nrep; base += 32) {
            const int i = base + tid;
            int v = i <= nrep ? s_first[i] : 0;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, v, off);
                if (tid >= off) v += y;
            }
            if (i <= nrep) s_first[i] = v + carry;
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
    }
    __syncthreads();
    return s_first[nrep];
}
// replica of work item w (s_first[r] <= w < s_first[r + 1]) and the item's
// global index (storage id, cell or brick); the storage ids of a replica are
// contiguous from its part_base
__device__ __forceinline__ int sched_item(const int *s_first, int nrep, const SysDev *__restrict__ sys, int item,
                                          int w, int *rep) {
    int lo = 0, hi = nrep - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_first[mid] <= w) lo = mid;
        else hi = mid - 1;
    }
    *rep = lo;
    return sched_first(sys[lo], item) + (w - s_first[lo]);
}

// cell counts of the flagged replicas (all C cells when rflag is null)
__global__ void k_list_clear(int *cnt, long long C, const int *flag, const int *rflag, int nrep, const SysDev *sys) {
    __shared__ int s_first[kSchedMaxRep + 1];
    if (*flag == 0) return;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x, nt = (long long)gridDim.x * blockDim.x;
    if (rflag && nrep <= kSchedMaxRep) {
        const int total = flagged_prefix(rflag, nrep, sys, kItemCell, s_first);
        for (long long w = t0; w < total; w += nt) {
            int r;
            cnt[sched_item(s_first, nrep, sys, kItemCell, (int)w, &r)] = 0;
        }
        return;
    }
    for (long long c = t0; c < C; c += nt) cnt[c] = 0;
}

__device__ __forceinline__ void bin_particle(const float4 *__restrict__ pos_sid, int sid, const SysDev &S, int *cnt,
                                             float4 *pos, int cap, unsigned *status) {
    const float4 v = pos_sid[sid];
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

// cell buckets from the by-id positions (same binning as the step kernels)
// of the replicas whose flag is set (every replica when rflag is null)
__global__ void k_list_bin(const float4 *__restrict__ pos_sid, int P, const int *__restrict__ rep_of_sid,
                           const SysDev *sys, int *cnt, float4 *pos, int cap, unsigned *status, const int *flag,
                           const int *rflag, int nrep) {
    __shared__ int s_first[kSchedMaxRep + 1];
    if (*flag == 0) return;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    if (rflag && nrep <= kSchedMaxRep) {
        const int total = flagged_prefix(rflag, nrep, sys, kItemParticle, s_first);
        for (int w = t0; w < total; w += nt) {
            int r;
            const int sid = sched_item(s_first, nrep, sys, kItemParticle, w, &r);
            bin_particle(pos_sid, sid, sys[r], cnt, pos, cap, status);
        }
        return;
    }
    for (int sid = t0; sid < P; sid += nt) {
        const int r = rep_of_sid[sid];
        if (rflag && rflag[r] == 0) continue;
        bin_particle(pos_sid, sid, sys[r], cnt, pos, cap, status);
    }
}

struct ListBuild {
    int *nbr;
    int *nnb;
    float4 *pbuild;
    const float4 *pos_sid;
    int *flag;                // [R + 1] as in ListArgs; cleared by the build's last block
    int nrep;
    long long *builds;        // [0] replica list builds, [1] steps that rebuilt
    unsigned *blocks_done;    // blocks of this launch that have finished (reset by the last one)
};

// Lists of every home particle of each brick (grid-stride over bricks):
// the staged sweep with the squared list cut distances (sigma + skin)^2,
// partners recorded by storage id in sweep order.
// Only the bricks of flagged replicas are visited: each block numbers them
// (flagged_prefix) and takes every gridDim.x-th one, so no block walks the
// bricks of unflagged replicas.
// One thread per home particle of a brick in one round (a brick holds about
// 170 particles at phi = 0.58): a rebuild of a few replicas runs one brick
// per SM, so its time is one CTA's staging plus one particle's sweep.  The
// lists do not depend on the CTA size (each particle's sweep order is fixed).
__global__ void __launch_bounds__(kListBuildThreads, 2) k_list_build(StepArgs a, ListBuild lb) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_first[kSchedMaxRep + 1];
    if (lb.flag[lb.nrep] == 0) return;
    const int tid = threadIdx.x, T = blockDim.x;
    const int nrep = lb.nrep;
    const bool sched = nrep <= kSchedMaxRep;
    const int total = sched ? flagged_prefix(lb.flag, nrep, a.sys, kItemBrick, s_first) : a.nbricks;
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
        int r;
        const int b = sched ? sched_item(s_first, nrep, a.sys, kItemBrick, w, &r) : w;
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
                            if (ok_sid) lb.nbr[list_slot(cnt, home_sid, a.np)] = sm.ssid[sm.queue[e * T + tid]];
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
                    const int nl = min(cnt, kMaxNbr);
                    // pad to whole gather chunks with storage id np (the zero position)
                    for (int k = nl; k < kMaxNbr && (k % kGather) != 0; k++) lb.nbr[list_slot(k, home_sid, a.np)] = a.np;
                    lb.nnb[home_sid] = nl;
                    lb.pbuild[home_sid] = lb.pos_sid[home_sid];
                } else {
                    set_status(a.status, kStatArg);
                }
            }
        }
        __syncthreads();  // the next brick reuses the staging memory
    }
    // The last block to finish clears the flags, every block having read
    // them (one launch per step fewer than a separate clearing kernel);
    // builds[0] counts replica rebuilds, builds[1] the steps that rebuilt.
    __shared__ bool last;
    if (tid == 0) {
        __threadfence();
        last = atomicAdd(lb.blocks_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
        __threadfence();
        if (tid == 0) atomicAdd((unsigned long long *)(lb.builds + 1), 1ull);
        for (int r = tid; r < nrep; r += T)
            if (lb.flag[r]) {
                atomicAdd((unsigned long long *)lb.builds, 1ull);
                lb.flag[r] = 0;
            }
        __syncthreads();
        if (tid == 0) {
            lb.flag[nrep] = 0;
            *lb.blocks_done = 0;
        }
    }
}

// ------------------------------------------------------------- step
// Partners go in chunks of kGather: the chunk's list words (loaded one chunk
// ahead), then all its positions in flight, then the next chunk's list words
// under those gathers, then the pair arithmetic in list order.  Lists are
// padded to whole chunks with storage id np, whose position entry is zero and
// never written, so a chunk needs no per-entry length test.

// Loads of the list state: through the read-only path in the per-step
// kernels (NC), plain loads in the per-replica persistent kernel, which
// rewrites positions and lists during its launch (a block sees its own
// writes after a barrier; the read-only path gives no such guarantee).
template <bool NC, typename T>
__device__ __forceinline__ T ld_state(const T *p) {
    if constexpr (NC) return __ldg(p);
    else return *p;
}

// list words k0 .. k0 + kGather - 1 (k0 < kMaxNbr)
template <bool NC = true>
__device__ __forceinline__ void list_words(const ListArgs &a, int sid, int k0, int (&jn)[kGather]) {
    const int4 w = ld_state<NC>(reinterpret_cast<const int4 *>(a.nbr) + (size_t)(k0 >> 2) * a.np + sid);
    jn[0] = w.x;
    jn[1] = w.y;
    jn[2] = w.z;
    jn[3] = w.w;
}
// positions of the chunk's partners: an entry outside [0, np) reads the zero
// position at np and counts as absent (jj = np)
template <bool NC = true>
__device__ __forceinline__ void gather_chunk(const ListArgs &a, const int (&jn)[kGather], int (&jj)[kGather],
                                             float4 (&pj)[kGather]) {
#pragma unroll
    for (int u = 0; u < kGather; u++) {
        jj[u] = (int)min((unsigned)jn[u], (unsigned)a.np);
        pj[u] = ld_state<NC>(a.pos_in + jj[u]);
    }
}

// The reference's minimum image d - L floor(d / L + 1/2) (get_forces.cu)
// of two list partners at once.  A list partner lies within cut + 2 skin of
// the particle, and a box holds at least three cells of side cut + skin with
// skin at most 0.9 of the largest cut (checked at engine creation), so d / L
// is within 0.492 of an integer k: then
// floor(d / L + 1/2) = rint(d / L) = k, L k is exact, and one rounded
// fma(k, -L, d) is the reference's rounded difference.  (A pair whose
// quotient lay near a half integer would sit near L / 2, beyond every cut
// distance, and fail the cut test with either rounding.)
__device__ __forceinline__ f2 min_image_pair(f2 d, f2 linv, f2 neg_l) {
    float ta, tb;
    f2_split(f2_mul(d, linv), ta, tb);
    return f2_fma(f2_make(rintf(ta), rintf(tb)), neg_l, d);
}

// Modified-WCA force on one particle from its list, two partners per f32x2
// operation (each lane rounds as the scalar operation does).  WRAP: a
// partner may lie across the periodic boundary, so each displacement takes
// the reference minimum image; otherwise every partner is within the box
// around the particle and the minimum image would return the plain
// difference.  The force is summed in two interleaved partial sums (even and
// odd list positions) that are added at the end.
template <bool WRAP, bool NC = true>
__device__ __forceinline__ void list_forces_wca(const ListArgs &a, int sid, int n, float4 pi, float L, float Linv,
                                                float sg0, float sg1, float c0, float c1, float &fx, float &fy,
                                                float &fz) {
    const f2 PX = f2_bcast(pi.x), PY = f2_bcast(pi.y), PZ = f2_bcast(pi.z), M12 = f2_bcast(-12.0f);
    const float sq0 = sg0 * sg0, sq1 = sg1 * sg1;
    const f2 LINV = f2_bcast(Linv), NEGL = f2_bcast(-L);
    f2 FX = 0ull, FY = 0ull, FZ = 0ull;  // (0.f, 0.f)
    const int np = a.np;
    int jn[kGather];
    if (n > 0) list_words<NC>(a, sid, 0, jn);
    for (int k0 = 0; k0 < n; k0 += kGather) {
        int jj[kGather];
        float4 pj[kGather];
        gather_chunk<NC>(a, jn, jj, pj);
        if (k0 + kGather < n) list_words<NC>(a, sid, k0 + kGather, jn);
#pragma unroll
        for (int u = 0; u < kGather; u += 2) {
            const float4 qa = pj[u], qb = pj[u + 1];
            f2 dX = f2_sub(f2_make(qa.x, qb.x), PX);
            f2 dY = f2_sub(f2_make(qa.y, qb.y), PY);
            f2 dZ = f2_sub(f2_make(qa.z, qb.z), PZ);
            if (WRAP) {
                dX = min_image_pair(dX, LINV, NEGL);
                dY = min_image_pair(dY, LINV, NEGL);
                dZ = min_image_pair(dZ, LINV, NEGL);
            }
            // dist2_rn in each lane
            const f2 D2 = f2_add(f2_add(f2_mul(dX, dX), f2_mul(dY, dY)), f2_mul(dZ, dZ));
            float d2a, d2b;
            f2_split(D2, d2a, d2b);
            const bool ta = (__float_as_uint(qa.w) >> 31) != 0u, tb = (__float_as_uint(qb.w) >> 31) != 0u;
            // without WRAP the particle is farther than every cut distance from
            // the origin, where the padding entries sit
            const bool oka = (!WRAP || jj[u] != np) && d2a < (ta ? c1 : c0);
            const bool okb = (!WRAP || jj[u + 1] != np) && d2b < (tb ? c1 : c0);
            if (oka || okb) {
                // (s / r)^2 from one approximate reciprocal of r^2 (one
                // multiply pair fewer than from 1 / r)
                float ra, rb;
                asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(ra) : "f"(d2a));
                asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rb) : "f"(d2b));
                const f2 R2 = f2_make(ra, rb);
                const f2 S2 = f2_mul(R2, f2_make(ta ? sq1 : sq0, tb ? sq1 : sq0));
                const f2 S6 = f2_mul(f2_mul(S2, S2), S2);
                // -12 (s^12 - s^6) / r^2
                const f2 G = f2_mul(f2_mul(M12, f2_sub(f2_mul(S6, S6), S6)), R2);
                float ga, gb;
                f2_split(G, ga, gb);
                const f2 GM = f2_make(oka ? ga : 0.f, okb ? gb : 0.f);
                FX = f2_fma(GM, dX, FX);
                FY = f2_fma(GM, dY, FY);
                FZ = f2_fma(GM, dZ, FZ);
            }
        }
    }
    float ea, eb;
    f2_split(FX, ea, eb);
    fx = __fadd_rn(ea, eb);
    f2_split(FY, ea, eb);
    fy = __fadd_rn(ea, eb);
    f2_split(FZ, ea, eb);
    fz = __fadd_rn(ea, eb);
}

// Force from the list for a replica with another potential of PotKind
// (scalar, list order).
template <bool NC = true>
__device__ __forceinline__ void list_forces_extra(const ListArgs &a, const SysDev &S, int sid, int n, float4 pi, int tm,
                                               float &fx, float &fy, float &fz) {
    const float L = S.L, Linv = S.Linv;
    const float sg0 = tm ? S.sig[1] : S.sig[0], sg1 = tm ? S.sig[2] : S.sig[1];
    const float c0 = tm ? S.cut2[1] : S.cut2[0], c1 = tm ? S.cut2[2] : S.cut2[1];
    fx = fy = fz = 0.f;
    int jn[kGather];
    if (n > 0) list_words<NC>(a, sid, 0, jn);
    for (int k0 = 0; k0 < n; k0 += kGather) {
        int jj[kGather];
        float4 pj[kGather];
        gather_chunk<NC>(a, jn, jj, pj);
        if (k0 + kGather < n) list_words<NC>(a, sid, k0 + kGather, jn);
#pragma unroll
        for (int u = 0; u < kGather; u++) {
            if (jj[u] == a.np) continue;
            const float dx = min_image_fast(__fsub_rn(pj[u].x, pi.x), L, Linv);
            const float dy = min_image_fast(__fsub_rn(pj[u].y, pi.y), L, Linv);
            const float dz = min_image_fast(__fsub_rn(pj[u].z, pi.z), L, Linv);
            const float d2 = dist2_rn(dx, dy, dz);
            const bool tj = (__float_as_uint(pj[u].w) >> 31) != 0u;
            if (d2 < (tj ? c1 : c0)) {
                const float sg = tj ? sg1 : sg0;
                const float di = rsqrtf(d2);
                float uu = 0.f;
                const float g = pair_extra(S.pot, S.pp, sg, di, &uu);
                fx = fmaf(g, dx, fx);
                fy = fmaf(g, dy, fy);
                fz = fmaf(g, dz, fz);
            }
        }
    }
}

// One time step of particle sid from its list: force sum in list order;
// update, compensated position and FP64 displacement exactly as
// process_brick.  Returns true when the particle has moved more than half
// the skin since the last build (its replica's lists must be rebuilt).
// EXTRA: some replica of the batch uses a potential other than the modified
// WCA (instantiated separately so the default kernel keeps its registers).
// LATE: the particle's own state is loaded after the force loop.  NC: loads
// through the read-only path (ld_state).
template <int RNG, bool EXTRA, bool LATE, bool NC>
__device__ __forceinline__ bool list_particle_step(const ListArgs &a, int sid, int rep, long long ni, int ni_off) {
    const SysDev &S = a.sys[rep];
    const float L = S.L, Linv = S.Linv;
    const float4 pi = a.pos_in[sid];
    const unsigned wi = __float_as_uint(pi.w);
    const int tm = (int)(wi >> 31);
    const float sg0 = tm ? S.sig[1] : S.sig[0], sg1 = tm ? S.sig[2] : S.sig[1];
    const float c0 = tm ? S.cut2[1] : S.cut2[0], c1 = tm ? S.cut2[2] : S.cut2[1];
    int gid;
    float lx, ly, lz;
    float4 pb;
    if constexpr (!LATE) {  // own state early: its latency overlaps the force loop
        gid = __ldg(a.gid_of + sid);
        lx = a.lo_x[sid], ly = a.lo_y[sid], lz = a.lo_z[sid];
        pb = ld_state<NC>(a.pbuild + sid);
    }
    float fx, fy, fz;
    const int n = min(ld_state<NC>(a.nnb + sid), kMaxNbr);
    if (EXTRA && S.pot != kPotWcaModified) {
        list_forces_extra<NC>(a, S, sid, n, pi, tm, fx, fy, fz);
    } else {  // the same arithmetic in either instantiation: a replica's result does not depend on its batch
        // a warp whose particles all sit away from the faces needs no
        // minimum image for any partner
        const float lo_edge = S.interior, hi_edge = L - S.interior;
        const bool inner = pi.x >= lo_edge && pi.x <= hi_edge && pi.y >= lo_edge && pi.y <= hi_edge &&
                           pi.z >= lo_edge && pi.z <= hi_edge;
        if (__all_sync(__activemask(), inner))
            list_forces_wca<false, NC>(a, sid, n, pi, L, Linv, sg0, sg1, c0, c1, fx, fy, fz);
        else
            list_forces_wca<true, NC>(a, sid, n, pi, L, Linv, sg0, sg1, c0, c1, fx, fy, fz);
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
    if constexpr (LATE) {
        gid = __ldg(a.gid_of + sid);
        lx = a.lo_x[sid], ly = a.lo_y[sid], lz = a.lo_z[sid];
        pb = ld_state<NC>(a.pbuild + sid);
    }
    const int pid = gid - S.part_base;
    if (ni == 0) {  // origin of the unwrapped positions (main.cu:497-506)
        a.x0[3 * (size_t)gid] = (double)pi.x + (double)lx;
        a.x0[3 * (size_t)gid + 1] = (double)pi.y + (double)ly;
        a.x0[3 * (size_t)gid + 2] = (double)pi.z + (double)lz;
        a.img[sid] = a.img[a.np + sid] = a.img[2 * a.np + sid] = 0;
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
    const float amp = a.amp_tab[((size_t)ni_off * a.nrep + rep) * 2 + tm];
    const float ex = __fadd_rn(__fmul_rn(__fmul_rn(fx, mob), dt), __fmul_rn(amp, xi.x));
    const float ey = __fadd_rn(__fmul_rn(__fmul_rn(fy, mob), dt), __fmul_rn(amp, xi.y));
    const float ez = __fadd_rn(__fmul_rn(__fmul_rn(fz, mob), dt), __fmul_rn(amp, xi.z));
    float x = pi.x, y = pi.y, z = pi.z;
    // the displacement is not stored per step: crossings of a face are
    // counted, and k_list_dsp rebuilds the FP64 displacement exactly from
    // hi + lo + L * crossings - origin when an observation needs it
    const float kx = advance_wrap(x, lx, ex, L, Linv);
    const float ky = advance_wrap(y, ly, ey, L, Linv);
    const float kz = advance_wrap(z, lz, ez, L, Linv);
    if (kx != 0.f) a.img[sid] += (int)kx;
    if (ky != 0.f) a.img[a.np + sid] += (int)ky;
    if (kz != 0.f) a.img[2 * a.np + sid] += (int)kz;
    a.lo_x[sid] = lx;
    a.lo_y[sid] = ly;
    a.lo_z[sid] = lz;
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) set_status(a.status, kStatNumeric);
    a.pos_out[sid] = make_float4(x, y, z, pi.w);
    // skin check against the positions at the last build: the minimum image
    // as in min_image_pair (a displacement near L / 2 raises the flag with
    // either rounding of the image)
    const float dbx = __fsub_rn(x, pb.x), dby = __fsub_rn(y, pb.y), dbz = __fsub_rn(z, pb.z);
    const float bx = fmaf(rintf(__fmul_rn(Linv, dbx)), -L, dbx);
    const float by = fmaf(rintf(__fmul_rn(Linv, dby)), -L, dby);
    const float bz = fmaf(rintf(__fmul_rn(Linv, dbz)), -L, dbz);
    return !(dist2_rn(bx, by, bz) <= S.skin_half2);
}

// One time step of every particle (thread per storage id); a particle beyond
// half the skin flags its replica for a rebuild before the next step.
template <int RNG, bool EXTRA, int V>
__global__ void __launch_bounds__(ListVariant<V>::kThreads, ListVariant<V>::kMinBlocks)
    k_step_list(ListArgs a, const long long *ni_base, int ni_off) {
    const int sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= a.np) return;
    const int rep = a.rep_of_sid[sid];
    if (list_particle_step<RNG, EXTRA, ListVariant<V>::kLate, true>(a, sid, rep, *ni_base + ni_off, ni_off)) {
        a.flag[rep] = 1;
        a.flag[a.nrep] = 1;
    }
}

// ------------------------------------------------------------- per-replica persistent launch
// Launch variants 3-5 run a whole batch of steps in one launch, one block
// per replica: the block steps its replica's particles, decides at a block
// barrier whether any of them left half the skin, and if so rebuilds the
// replica's cell buckets and lists itself before the next step.  Replicas
// never interact, so blocks never wait on one another; a block's own writes
// (positions, buckets, lists) are visible to its threads after each barrier,
// which is why these kernels read the list state with plain loads.
// The lists are the ones k_list_build writes: partners in the staged
// sweep's order (rows dz, dy of three cells dx, each cell in storage-id
// order), the same shifted differences and the same list cut test, so a
// replica's trajectory does not depend on the variant.
struct ListPersist {
    float4 *pos[2];        // by-id positions, the two buffers
    int cur0;              // buffer holding the input of the launch's first step
    int *cnt;              // cell counts of the buckets (buffer 0)
    float4 *bucket;        // [C][cap] cell buckets
    int cap;
    int *nbr;              // lists (list_slot), lengths and build positions:
    int *nnb;              //   the writable views of ListArgs' nbr, nnb, pbuild
    float4 *pbuild;
    const int *order;      // replica of each block, most particles first
    long long *builds;     // [0] replica list builds, [1] steps that rebuilt
    int *step_rebuilt;     // [step of the launch]: some replica rebuilt before it
    int shared_build;      // variant 5: rebuild from shared memory (replica_rebuild_shared)
};

// cell of a by-id position, as bin_particle and the step kernels bin it
__device__ __forceinline__ int3 list_cell_of(const float4 v, const SysDev &S) {
    const int nc = S.ncell;
    int ix = (int)__fmul_rn(v.x, S.cinv), iy = (int)__fmul_rn(v.y, S.cinv), iz = (int)__fmul_rn(v.z, S.cinv);
    return make_int3(min(max(ix, 0), nc - 1), min(max(iy, 0), nc - 1), min(max(iz, 0), nc - 1));
}
// neighbour cell index along one axis (periodic) and the staged sweep's
// shift of its particles (+L when the cell wrapped below 0, -L above nc - 1)
__device__ __forceinline__ int wrap_cell(int g, int nc, float L, float &shift) {
    int sgn = 0;
    if (g < 0) { g += nc; sgn = 1; } else if (g >= nc) { g -= nc; sgn = -1; }
    shift = __int2float_rn(sgn) * L;  // exact: sgn in {-1, 0, 1}
    return g;
}

// A replica's cells for the in-block list build, each in storage-id order:
// the bucket buffer in global memory (cap slots per cell), or a compact
// cell-sorted copy in shared memory.
struct CellsGlobal {
    const int *cnt;
    const float4 *bucket;
    int cap, cell_base;
    __device__ __forceinline__ const float4 *cell(int c, int &m) const {
        const int gc = cell_base + c;
        m = min(cnt[gc], cap);
        return bucket + (size_t)gc * cap;
    }
};
struct CellsShared {
    const int *start;  // [cells + 1]
    const float4 *pos;
    __device__ __forceinline__ const float4 *cell(int c, int &m) const {
        m = start[c + 1] - start[c];
        return pos + start[c];
    }
};

// List of particle sid from the sorted cells of its replica.
template <class CELLS>
__device__ __forceinline__ void replica_list(const ListArgs &a, const ListPersist &lp, const SysDev &S, int sid,
                                             const CELLS &cells) {
    const float4 v = a.pos_in[sid];
    const int np = a.np, nc = S.ncell;
    const int tm = (int)(__float_as_uint(v.w) >> 31);
    const float cut_b = S.lcut2[tm], cut_s = S.lcut2[tm + 1];  // towards a big / a small partner
    const float L = S.L;
    const int3 c = list_cell_of(v, S);
    int cnt = 0;
    for (int dz = -1; dz <= 1; dz++) {
        float shz;
        const int gz = wrap_cell(c.z + dz, nc, L, shz);
        for (int dy = -1; dy <= 1; dy++) {
            float shy;
            const int gy = wrap_cell(c.y + dy, nc, L, shy);
            for (int dx = -1; dx <= 1; dx++) {
                float shx;
                const int gx = wrap_cell(c.x + dx, nc, L, shx);
                int m;
                const float4 *b = cells.cell(gx + nc * (gy + nc * gz), m);
                for (int k = 0; k < m; k++) {
                    const float4 q = b[k];
                    const unsigned wq = __float_as_uint(q.w);
                    const int sj = (int)(wq & 0x7fffffffu);
                    if (sj == sid) continue;
                    const float ex = __fsub_rn(__fsub_rn(q.x, v.x), shx);
                    const float ey = __fsub_rn(__fsub_rn(q.y, v.y), shy);
                    const float ez = __fsub_rn(__fsub_rn(q.z, v.z), shz);
                    if (dist2_rn(ex, ey, ez) < ((wq >> 31) ? cut_s : cut_b)) {
                        if (cnt < kMaxNbr) lp.nbr[list_slot(cnt, sid, np)] = sj;
                        else set_status(a.status, kStatCellOverflow);
                        cnt++;
                    }
                }
            }
        }
    }
    const int nl = min(cnt, kMaxNbr);
    for (int k = nl; k < kMaxNbr && (k % kGather) != 0; k++) lp.nbr[list_slot(k, sid, np)] = np;
    lp.nnb[sid] = nl;
    lp.pbuild[sid] = v;
}

// Buckets and lists of replica S from a.pos_in, by the whole block.
__device__ __forceinline__ void replica_rebuild(const ListArgs &a, const ListPersist &lp, const SysDev &S) {
    const int tid = threadIdx.x, T = blockDim.x;
    const int nc = S.ncell, ncell = nc * nc * nc, cb = S.cell_base, cap = lp.cap;
    const int base = S.part_base, end = S.part_base + S.n;
    for (int c = tid; c < ncell; c += T) lp.cnt[cb + c] = 0;
    __syncthreads();
    for (int sid = base + tid; sid < end; sid += T) {
        const float4 v = a.pos_in[sid];
        const int3 c = list_cell_of(v, S);
        const int cell = cb + c.x + nc * (c.y + nc * c.z);
        const int slot = atomicAdd(lp.cnt + cell, 1);
        if (slot < cap) lp.bucket[(size_t)cell * cap + slot] = v;
        else set_status(a.status, kStatCellOverflow);
    }
    __syncthreads();
    // each cell in storage-id order (insertion sort, a thread per cell)
    for (int c = tid; c < ncell; c += T) {
        float4 *b = lp.bucket + (size_t)(cb + c) * cap;
        const int m = min(lp.cnt[cb + c], cap);
        for (int i = 1; i < m; i++) {
            const float4 v = b[i];
            const unsigned key = __float_as_uint(v.w) & 0x7fffffffu;
            int j = i - 1;
            while (j >= 0 && (__float_as_uint(b[j].w) & 0x7fffffffu) > key) {
                b[j + 1] = b[j];
                j--;
            }
            b[j + 1] = v;
        }
    }
    __syncthreads();
    const CellsGlobal cells{lp.cnt, lp.bucket, cap, cb};
    for (int sid = base + tid; sid < end; sid += T) replica_list(a, lp, S, sid, cells);
    __syncthreads();
}

// Shared-memory bytes of the in-block rebuild from shared memory for a
// replica of n particles in c cells: exclusive cell starts [c + 1] and fill
// counters [c], then the positions sorted by cell.
__host__ __device__ inline size_t replica_shared_build_bytes(int n, int c) {
    return (((size_t)(2 * c + 1) * 4 + 15) & ~(size_t)15) + (size_t)n * 16;
}

// The same lists as replica_rebuild, from a compact copy of the replica
// sorted by cell (a counting sort, then each cell by storage id) in the
// block's dynamic shared memory `dsm` (replica_shared_build_bytes).  Cells
// above the bucket capacity raise the overflow status as the bucket build
// does.
__device__ __forceinline__ void replica_rebuild_shared(const ListArgs &a, const ListPersist &lp, const SysDev &S,
                                                       unsigned char *dsm) {
    const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const int nc = S.ncell, ncell = nc * nc * nc;
    const int base = S.part_base, n = S.n;
    int *s_start = reinterpret_cast<int *>(dsm);  // [ncell + 1]
    int *s_fill = s_start + ncell + 1;            // [ncell]
    float4 *s_pos = reinterpret_cast<float4 *>(dsm + (((size_t)(2 * ncell + 1) * 4 + 15) & ~(size_t)15));
    __shared__ int s_warp[32];
    for (int c = tid; c < ncell; c += T) s_fill[c] = 0;
    __syncthreads();
    for (int i = tid; i < n; i += T) {
        const int3 c = list_cell_of(a.pos_in[base + i], S);
        atomicAdd(&s_fill[c.x + nc * (c.y + nc * c.z)], 1);
    }
    __syncthreads();
    // exclusive scan of the counts: a segment per thread, then the warps
    const int per = (ncell + T - 1) / T, c0 = min(tid * per, ncell), c1 = min(c0 + per, ncell);
    int local = 0;
    for (int c = c0; c < c1; c++) local += s_fill[c];
    int incl = local;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (T >> 5) ? s_warp[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        s_warp[lane] = w;
    }
    __syncthreads();
    int run = incl - local + (warp > 0 ? s_warp[warp - 1] : 0);
    for (int c = c0; c < c1; c++) {
        const int k = s_fill[c];
        if (k > lp.cap) set_status(a.status, kStatCellOverflow);
        s_start[c] = run;
        s_fill[c] = run;
        run += k;
    }
    if (tid == 0) s_start[ncell] = n;
    __syncthreads();
    for (int i = tid; i < n; i += T) {
        const float4 v = a.pos_in[base + i];
        const int3 c = list_cell_of(v, S);
        s_pos[atomicAdd(&s_fill[c.x + nc * (c.y + nc * c.z)], 1)] = v;
    }
    __syncthreads();
    // each cell in storage-id order (insertion sort, a thread per cell)
    for (int c = tid; c < ncell; c += T) {
        float4 *b = s_pos + s_start[c];
        const int m = s_start[c + 1] - s_start[c];
        for (int i = 1; i < m; i++) {
            const float4 v = b[i];
            const unsigned key = __float_as_uint(v.w) & 0x7fffffffu;
            int j = i - 1;
            while (j >= 0 && (__float_as_uint(b[j].w) & 0x7fffffffu) > key) {
                b[j + 1] = b[j];
                j--;
            }
            b[j + 1] = v;
        }
    }
    __syncthreads();
    const CellsShared cells{s_start, s_pos};
    for (int sid = base + tid; sid < base + n; sid += T) replica_list(a, lp, S, sid, cells);
    __syncthreads();
}

// nsteps steps of replica order[blockIdx.x] (Philox noise; nsteps at most the
// amplitude table's batch).  The replica's flag on entry asks for a rebuild
// before the first step; on exit it holds the last step's decision.
template <bool EXTRA, int V>
__global__ void __launch_bounds__(ListVariant<V>::kThreads, ListVariant<V>::kMinBlocks)
    k_list_replica(ListArgs a, ListPersist lp, const long long *ni_base, int nsteps) {
    extern __shared__ __align__(16) unsigned char dsm[];
    const int rep = lp.order[blockIdx.x];
    const SysDev &S = a.sys[rep];
    const int base = S.part_base, end = S.part_base + S.n;
    const long long ni0 = *ni_base;
    bool need = a.flag[rep] != 0;
    for (int s = 0; s < nsteps; s++) {
        ListArgs as = a;
        const bool odd = ((lp.cur0 + s) & 1) != 0;  // a select, not an indexed (local-memory) copy
        as.pos_in = odd ? lp.pos[1] : lp.pos[0];
        as.pos_out = odd ? lp.pos[0] : lp.pos[1];
        if (need) {
            bool done = false;
            if constexpr (V == 5) {
                if (lp.shared_build) {
                    replica_rebuild_shared(as, lp, S, dsm);
                    done = true;
                }
            }
            if (!done) replica_rebuild(as, lp, S);
            if (threadIdx.x == 0) {
                atomicAdd((unsigned long long *)lp.builds, 1ull);
                lp.step_rebuilt[s] = 1;
            }
        }
        bool beyond = false;
        for (int sid = base + (int)threadIdx.x; sid < end; sid += blockDim.x)
            beyond |= list_particle_step<kRngPhilox, EXTRA, ListVariant<V>::kLate, false>(as, sid, rep, ni0 + s, s);
        need = __syncthreads_or(beyond) != 0;
    }
    if (threadIdx.x == 0) a.flag[rep] = need ? 1 : 0;
}

// After a per-replica launch: the any-replica flag from the per-replica
// flags, and the launch's steps that rebuilt some replica counted.
__global__ void k_list_replica_done(int *flag, int nrep, int *step_rebuilt, int nsteps, long long *builds) {
    __shared__ int s_any, s_steps;
    if (threadIdx.x == 0) s_any = s_steps = 0;
    __syncthreads();
    int any = 0, steps = 0;
    for (int r = threadIdx.x; r < nrep; r += blockDim.x) any |= flag[r];
    for (int s = threadIdx.x; s < nsteps; s += blockDim.x) {
        steps += step_rebuilt[s] != 0;
        step_rebuilt[s] = 0;
    }
    if (any) atomicOr(&s_any, 1);
    if (steps) atomicAdd(&s_steps, steps);
    __syncthreads();
    if (threadIdx.x == 0) {
        flag[nrep] = s_any;
        if (s_steps) atomicAdd((unsigned long long *)(builds + 1), (unsigned long long)s_steps);
    }
}

// FP64 displacement since the origin, rebuilt from the state of list mode:
// (hi + lo) and L * crossings are exact in FP64; their sum is exact while few
// crossings have accumulated (otherwise it rounds once, about 1e-13 in a box
// of side 30 after tens of crossings), and the subtraction of the origin
// rounds once.
__global__ void k_list_dsp(const float4 *__restrict__ pos, const float *__restrict__ lo_x,
                           const float *__restrict__ lo_y, const float *__restrict__ lo_z, const int *__restrict__ img,
                           const double *__restrict__ x0, const int *__restrict__ gid_of,
                           const int *__restrict__ rep_of_sid, const SysDev *__restrict__ sys, int np, double *dx,
                           double *dy, double *dz) {
    const int sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= np) return;
    const double L = (double)sys[rep_of_sid[sid]].L;
    const float4 v = pos[sid];
    const size_t g = 3 * (size_t)gid_of[sid];
    dx[sid] = (((double)v.x + (double)lo_x[sid]) + L * (double)img[sid]) - x0[g];
    dy[sid] = (((double)v.y + (double)lo_y[sid]) + L * (double)img[np + sid]) - x0[g + 1];
    dz[sid] = (((double)v.z + (double)lo_z[sid]) + L * (double)img[2 * (size_t)np + sid]) - x0[g + 2];
}

// Noise amplitude of every replica and species for `count` consecutive steps
// from *ni_base (the same temperature and amplitude arithmetic as the
// sweep's update), once per launch batch instead of once per particle:
// tab[(j * nrep + r) * 2 + species].
__global__ void k_amp_table(const SysDev *sys, int nrep, const long long *ni_base, long long ni_first, int count,
                            float *tab) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count * nrep) return;
    const int j = t / nrep, r = t % nrep;
    const SysDev &S = sys[r];
    const float T = step_temperature(S, *ni_base + j, ni_first);
    tab[2 * (size_t)t] = amplitude(T, S.mob[0], S.dt);
    tab[2 * (size_t)t + 1] = amplitude(T, S.mob[1], S.dt);
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
        const int j = a.nbr[list_slot(k, sid, a.np)];
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
