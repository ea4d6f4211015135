// engine.cu -- host driver of the batched replica engine (bd_engine_* ABI):
// geometry, buffers, initial load, CUDA-graph stepping, observation passes,
// export, and the batch g(r) kernel.
#include "engine_kernels.cuh"
#include "engine_state.cuh"

namespace bd {

// ------------------------------------------------------------- batch g(r)
// get_gder_dev (get_gder.cu:69-127) for all four species pairs of one
// replica in one pass over unordered pairs i < j: the forward distance
// (r_i - r_j) counts for (type_i, type_j), the reverse one for (type_j,
// type_i), recomputed when the minimum-image rounding can differ.  Big
// particles come first, so i < j gives bb, bs and ss forward and bb, sb, ss
// in reverse.
// g(r) bin thresholds (gr_bin_thr): thr[k], k = 0 .. nbins + 1
__global__ void k_gr_thresholds(float range, int nbins, float *thr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > nbins + 1) return;
    if (k == 0) { thr[0] = 0.f; return; }
    const float bin_size = __fdiv_rn(range, (float)nbins);
    unsigned lo = 0u, hi = 0x7f800000u;  // +0 .. +inf
    while (lo < hi) {
        const unsigned mid = lo + ((hi - lo) >> 1);
        const float x = __uint_as_float(mid);
        const bool reach = k <= nbins ? gr_bin_exact(x, bin_size) >= k : !(__fsqrt_rn(x) < range);
        if (reach) hi = mid;
        else lo = mid + 1;
    }
    thr[k] = __uint_as_float(lo);
}
constexpr int kGrTile = 1024;
__device__ __forceinline__ int gr_bin(float dx, float dy, float dz, float side, float side_inv, const float *thr,
                                      float inv_bin_size, int nbins) {
    dx = min_image_gder_fast(dx, side, side_inv);
    dy = min_image_gder_fast(dy, side, side_inv);
    dz = min_image_gder_fast(dz, side, side_inv);
    return gr_bin_thr(dist2_rn(dx, dy, dz), thr, inv_bin_size, nbins);
}
// One launch for every replica that needs all pairs (blockIdx.z indexes
// `reps`).  Histogram: with `copies` > 1 each pair of warps adds into its own
// copy in shared memory with plain atomics (bins spread over the lanes rarely
// collide), and the copies are summed at the end; with one copy, lanes of
// equal bins are combined by __match_any_sync first.
__global__ void __launch_bounds__(256) k_gr_batch(const float4 *__restrict__ snap_all, const SysDev *__restrict__ sys,
                                                  const int *__restrict__ reps, float range,
                                                  const float *__restrict__ thr_g, int nbins, int jchunk, int copies,
                                                  unsigned long long *counts_all) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int r = reps[blockIdx.z];
    const SysDev &S = sys[r];
    const int n = S.n, n_big = S.n_big;
    const int j0 = max(blockIdx.y * jchunk, (int)(blockIdx.x * blockDim.x) + 1), j1 = min(n, (int)(blockIdx.y + 1) * jchunk);
    if (j0 >= j1) return;  // uniform over the block: no pair of this replica here
    const float4 *snap = snap_all + S.part_base;
    unsigned long long *counts = counts_all + (size_t)r * 4 * nbins;
    const float side = S.L;
    float4 *tile = reinterpret_cast<float4 *>(smem);
    float *thr = reinterpret_cast<float *>(tile + kGrTile);          // [nbins + 2] bin thresholds
    unsigned *hist0 = reinterpret_cast<unsigned *>(thr + nbins + 2);  // [copies][4][nbins]
    for (int b = threadIdx.x; b < copies * 4 * nbins; b += blockDim.x) hist0[b] = 0;
    for (int b = threadIdx.x; b < nbins + 2; b += blockDim.x) thr[b] = thr_g[b];
    const int per_copy = (blockDim.x / 32 + copies - 1) / copies;  // warps per copy
    unsigned *hist = hist0 + ((threadIdx.x >> 5) / per_copy) * 4 * nbins;
    const float side_inv = __double2float_rn(1.0 / (double)side);
    const float inv_bin_size = 1.0f / __fdiv_rn(range, (float)nbins);  // estimate only (gr_bin_thr)
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool vi = i < n;
    float4 pi = vi ? snap[i] : make_float4(0, 0, 0, 0);
    const int ti = i < n_big ? 0 : 1;
    __syncthreads();
    for (int t0 = j0; t0 < j1; t0 += kGrTile) {
        const int tn = min(kGrTile, j1 - t0);
        __syncthreads();
        for (int t = threadIdx.x; t < tn; t += blockDim.x) tile[t] = snap[t0 + t];
        __syncthreads();
        for (int t = 0; t < tn; t++) {
            const int j = t0 + t;
            const int tj = j < n_big ? 0 : 1;
            int kf = -1, kr = -1;
            if (vi && j > i) {
                float4 pj = tile[t];
                float dx = __fsub_rn(pi.x, pj.x), dy = __fsub_rn(pi.y, pj.y), dz = __fsub_rn(pi.z, pj.z);
                int bf = gr_bin(dx, dy, dz, side, side_inv, thr, inv_bin_size, nbins);
                // below 0.49 the minimum image returns d itself for both signs
                // (min_image_gder_fast), so the reverse distance is the same
                bool sym = fabsf(__fmul_rn(side_inv, dx)) < 0.49f && fabsf(__fmul_rn(side_inv, dy)) < 0.49f &&
                           fabsf(__fmul_rn(side_inv, dz)) < 0.49f;
                int bb = sym ? bf : gr_bin(-dx, -dy, -dz, side, side_inv, thr, inv_bin_size, nbins);
                if (bf >= 0) kf = (ti * 2 + tj) * nbins + bf;
                if (bb >= 0) kr = (tj * 2 + ti) * nbins + bb;
            }
            if (copies > 1) {
                if (kf >= 0) atomicAdd(&hist[kf], 1u);
                if (kr >= 0) atomicAdd(&hist[kr], 1u);
            } else {
                unsigned s1 = __match_any_sync(0xffffffffu, kf);
                if (kf >= 0 && (threadIdx.x & 31) == __ffs(s1) - 1) atomicAdd(&hist[kf], (unsigned)__popc(s1));
                unsigned s2 = __match_any_sync(0xffffffffu, kr);
                if (kr >= 0 && (threadIdx.x & 31) == __ffs(s2) - 1) atomicAdd(&hist[kr], (unsigned)__popc(s2));
            }
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 4 * nbins; b += blockDim.x) {
        unsigned long long v = 0;
        for (int c = 0; c < copies; c++) v += hist0[c * 4 * nbins + b];
        if (v) atomicAdd(&counts[b], v);
    }
}

}  // namespace bd

using namespace bd;

namespace {

StepArgs make_args(bd_engine *e, int buf, int do_update) {
    StepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.sys = e->d_sys;
    a.bricks = e->d_bricks;
    a.nbricks = e->nbricks;
    a.bx = e->bx; a.by = e->by; a.bz = e->bz;
    a.cap = e->cap;
    a.smax = e->smax;
    a.cnt_in = e->cnt[buf % 3];
    a.pos_in = e->pos[buf % 3];
    a.cnt_out = e->cnt[(buf + 1) % 3];
    a.pos_out = e->pos[(buf + 1) % 3];
    a.cnt_clr = e->cnt[(buf + 2) % 3];
    a.lo_x = e->lo[0]; a.lo_y = e->lo[1]; a.lo_z = e->lo[2];
    a.dsp_x = e->dsp[0]; a.dsp_y = e->dsp[1]; a.dsp_z = e->dsp[2];
    a.gid_of = e->gid_of;
    a.np = (int)e->P;
    a.x0 = e->x0;
    a.snap = e->snap;
    a.obs = e->obs;
    a.nbr_count = e->nbr_count;
    a.nbr_hash = e->nbr_hash;
    a.curand_states = e->cr;
    a.noise = e->noise;
    a.rn_ring = e->rn_ring;
    a.rn_lcg = e->rn_lcg;
    a.rn_ni0 = e->rn_ni0;
    a.status = e->status;
    a.ni_first = e->ni_first;
    a.qmax = e->qmax;
    a.do_update = do_update;
    a.rng_stream = e->rng_stream;
    for (int k = 0; k < 3; k++) { a.cnt3[k] = e->cnt[k]; a.pos3[k] = e->pos[k]; }
    a.cur0 = buf % 3;
    a.cl_start = e->d_cl_start;
    a.cl_bricks = e->d_cl_bricks;
    return a;
}

// Dynamic shared memory above 48 KB needs a per-kernel attribute; it is set
// outside stream capture (launch_step_t with attr_only) before any graph is
// recorded.
template <int RNG, bool OBS, bool CENSUS>
int launch_step_t(bd_engine *e, const StepArgs &a, int ni_off, bool attr_only = false) {
    auto kern = k_step<RNG, OBS, CENSUS>;
    if (attr_only) {
        BD_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(CENSUS ? e->smem_census : e->smem)));
        return BD_OK;
    }
    kern<<<e->nbricks, e->threads, CENSUS ? e->smem_census : e->smem, e->stream>>>(a, e->d_ni, ni_off);
    BD_LAUNCH_CHECK();
    return BD_OK;
}

template <int RNG>
int launch_persistent_t(bd_engine *e, const StepArgs &a, int nsteps, bool attr_only = false) {
    auto kern = k_step_persistent<RNG>;
    if (attr_only) {
        BD_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e->smem));
        return BD_OK;
    }
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(e->nclusters * e->cluster);
    cfg.blockDim = dim3(e->threads);
    cfg.dynamicSmemBytes = e->smem;
    cfg.stream = e->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = e->cluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    BD_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, a, (const long long *)e->d_ni, nsteps));
    return BD_OK;
}
int launch_persistent(bd_engine *e, const StepArgs &a, int nsteps) {
    switch (e->rng) {
        case BD_RNG_CURAND: return launch_persistent_t<kRngCurand>(e, a, nsteps);
        case BD_RNG_NOISE: return launch_persistent_t<kRngNoise>(e, a, nsteps);
        case BD_RNG_RANNEW64: return launch_persistent_t<kRngRannew64>(e, a, nsteps);
        default: return launch_persistent_t<kRngPhilox>(e, a, nsteps);
    }
}
// Clusters of e->cluster CTAs that can be resident at once (0 if none).
int max_active_clusters(bd_engine *e) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(e->cluster);
    cfg.blockDim = dim3(e->threads);
    cfg.dynamicSmemBytes = e->smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = e->cluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_step_persistent<kRngPhilox>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int configure_kernels(bd_engine *e) {
    StepArgs a;
    std::memset(&a, 0, sizeof(a));
    int rc = 0;
    rc |= launch_persistent_t<kRngPhilox>(e, a, 0, true);
    rc |= launch_persistent_t<kRngCurand>(e, a, 0, true);
    rc |= launch_persistent_t<kRngNoise>(e, a, 0, true);
    rc |= launch_persistent_t<kRngRannew64>(e, a, 0, true);
#define BD_ATTR(R)                                                 \
    rc |= launch_step_t<R, false, false>(e, a, 0, true);           \
    rc |= launch_step_t<R, true, false>(e, a, 0, true);            \
    rc |= launch_step_t<R, false, true>(e, a, 0, true);
    BD_ATTR(kRngPhilox)
    BD_ATTR(kRngCurand)
    BD_ATTR(kRngNoise)
    BD_ATTR(kRngRannew64)
#undef BD_ATTR
    if (cudaFuncSetAttribute(k_list_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e->lsmem) != cudaSuccess)
        rc = 1;
    if (e->lrep_smem > 0) {  // variant 5 rebuilds from shared memory
        if (cudaFuncSetAttribute(k_list_replica<false, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)e->lrep_smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_list_replica<true, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)e->lrep_smem) != cudaSuccess)
            rc = 1;
    }
    return rc ? BD_ERR_CUDA : BD_OK;
}

template <bool OBS, bool CENSUS>
int launch_step_rng(bd_engine *e, const StepArgs &a, int ni_off) {
    switch (e->rng) {
        case BD_RNG_CURAND: return launch_step_t<kRngCurand, OBS, CENSUS>(e, a, ni_off);
        case BD_RNG_NOISE: return launch_step_t<kRngNoise, OBS, CENSUS>(e, a, ni_off);
        case BD_RNG_RANNEW64: return launch_step_t<kRngRannew64, OBS, CENSUS>(e, a, ni_off);
        default: return launch_step_t<kRngPhilox, OBS, CENSUS>(e, a, ni_off);
    }
}
int launch_step(bd_engine *e, const StepArgs &a, int ni_off, bool obs, bool census) {
    if (census) return launch_step_rng<false, true>(e, a, ni_off);
    if (obs) return launch_step_rng<true, false>(e, a, ni_off);
    return launch_step_rng<false, false>(e, a, ni_off);
}

// ---- neighbour-list mode
ListArgs make_largs(bd_engine *e, int cur) {
    ListArgs a;
    std::memset(&a, 0, sizeof(a));
    a.sys = e->d_sys;
    a.rep_of_sid = e->rep_of_sid;
    a.gid_of = e->gid_of;
    a.np = (int)e->P;
    a.pos_in = e->lpos[cur & 1];
    a.pos_out = e->lpos[(cur + 1) & 1];
    a.lo_x = e->lo[0]; a.lo_y = e->lo[1]; a.lo_z = e->lo[2];
    a.img = e->img;
    a.nbr = e->nbr;
    a.nnb = e->nnb;
    a.pbuild = e->pbuild;
    a.amp_tab = e->amp_tab;
    a.flag = e->lflag;
    a.nrep = e->R;
    a.x0 = e->x0;
    a.curand_states = e->cr;
    a.noise = e->noise;
    a.rn_ring = e->rn_ring;
    a.rn_lcg = e->rn_lcg;
    a.rn_ni0 = e->rn_ni0;
    a.status = e->status;
    a.ni_first = e->ni_first;
    a.rng_stream = e->rng_stream;
    a.nbr_count = e->nbr_count;
    a.nbr_hash = e->nbr_hash;
    return a;
}
int rebuild_grid(bd_engine *e, long long work) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->dev);
    return (int)std::max(1LL, std::min(work, (long long)sms * 4));
}
// Cell buckets (buffer 0) from the by-id positions of phase `cur`: `any`
// gates the work, `rflag` (per replica, or null for all) selects replicas
// (e->lflag inside steps; e->d_one and null for observation passes).
int list_bin(bd_engine *e, int cur, const int *any, const int *rflag) {
    cudaStream_t st = e->stream;
    // with rflag only the flagged replicas' cells are cleared and binned: a
    // build stages cells of its own replica only
    k_list_clear<<<rebuild_grid(e, div_up(e->C, 256)), 256, 0, st>>>(e->cnt[0], e->C, any, rflag, e->R, e->d_sys);
    k_list_bin<<<rebuild_grid(e, div_up(e->P, 256)), 256, 0, st>>>(e->lpos[cur & 1], (int)e->P, e->rep_of_sid,
                                                                 e->d_sys, e->cnt[0], e->pos[0], e->cap, e->status,
                                                                 any, rflag, e->R);
    BD_LAUNCH_CHECK();
    return BD_OK;
}
// Rebuild the lists of the flagged replicas (every kernel exits at once when
// no replica is flagged).  Rebuild decisions are per replica, so a replica
// gets the same lists alone as in any batch.
int list_rebuild(bd_engine *e, int cur) {
    cudaStream_t st = e->stream;
    int rc = list_bin(e, cur, e->lflag + e->R, e->lflag);
    if (rc) return rc;
    ListBuild lb{e->nbr, e->nnb, e->pbuild, e->lpos[cur & 1], e->lflag, e->R, e->d_builds,
                 reinterpret_cast<unsigned *>(e->d_builds + 2)};
    k_list_build<<<rebuild_grid(e, e->nbricks), kListBuildThreads, e->lsmem, st>>>(make_args(e, 0, 0), lb);
    BD_LAUNCH_CHECK();
    return BD_OK;
}
template <int RNG, int V>
int launch_list_step_v(bd_engine *e, const ListArgs &a, int ni_off) {
    constexpr int T = ListVariant<V>::kThreads;
    if (e->extra_pot)
        k_step_list<RNG, true, V><<<div_up(e->P, T), T, 0, e->stream>>>(a, e->d_ni, ni_off);
    else
        k_step_list<RNG, false, V><<<div_up(e->P, T), T, 0, e->stream>>>(a, e->d_ni, ni_off);
    BD_LAUNCH_CHECK();
    return BD_OK;
}
// every variant for the default (Philox) noise; the compatibility streams
// run variant 0
int launch_list_step(bd_engine *e, const ListArgs &a, int ni_off) {
    switch (e->rng) {
        case BD_RNG_CURAND: return launch_list_step_v<kRngCurand, 0>(e, a, ni_off);
        case BD_RNG_RANNEW64: return launch_list_step_v<kRngRannew64, 0>(e, a, ni_off);
        default:
            switch (e->lvar) {
                case 1: return launch_list_step_v<kRngPhilox, 1>(e, a, ni_off);
                case 2: return launch_list_step_v<kRngPhilox, 2>(e, a, ni_off);
                default: return launch_list_step_v<kRngPhilox, 0>(e, a, ni_off);
            }
    }
}
// Launch variants 3-5: one block per replica runs `nsteps` steps (the
// Philox noise only; other noise streams take variant 0).
bool list_per_replica(const bd_engine *e) {
    return e->list && e->lvar >= kListFirstPersistent && e->rng == BD_RNG_PHILOX;
}
template <int V>
int launch_list_replica_v(bd_engine *e, int cur, int nsteps) {
    constexpr int T = ListVariant<V>::kThreads;
    const ListArgs a = make_largs(e, cur);
    const bool shared_build = V == 5 && e->lrep_smem > 0;
    const ListPersist lp{{e->lpos[0], e->lpos[1]}, cur & 1, e->cnt[0], e->pos[0], e->cap, e->nbr, e->nnb,
                         e->pbuild, e->d_rep_order, e->d_builds, e->d_step_rebuilt, shared_build ? 1 : 0};
    const size_t sm = shared_build ? e->lrep_smem : 0;
    if (e->extra_pot) k_list_replica<true, V><<<e->R, T, sm, e->stream>>>(a, lp, e->d_ni, nsteps);
    else k_list_replica<false, V><<<e->R, T, sm, e->stream>>>(a, lp, e->d_ni, nsteps);
    BD_LAUNCH_CHECK();
    k_list_replica_done<<<1, 256, 0, e->stream>>>(e->lflag, e->R, e->d_step_rebuilt, nsteps, e->d_builds);
    BD_LAUNCH_CHECK();
    return BD_OK;
}
int list_replica_steps(bd_engine *e, int cur, int nsteps) {
    if (nsteps > e->graph_steps) return BD_ERR_ARG;  // the amplitude table holds one batch
    switch (e->lvar) {
        case 3: return launch_list_replica_v<3>(e, cur, nsteps);
        case 4: return launch_list_replica_v<4>(e, cur, nsteps);
        default: return launch_list_replica_v<5>(e, cur, nsteps);
    }
}
// one list-mode step in phase `cur`: gated rebuild, then the step
int list_step(bd_engine *e, int cur, int ni_off) {
    int rc = list_rebuild(e, cur);
    if (rc) return rc;
    return launch_list_step(e, make_largs(e, cur), ni_off);
}
}  // namespace

// displacement of list mode rebuilt from positions, remainders and crossings
int bd::sync_dsp(bd_engine *e) {
    if (!e->list) return BD_OK;
    const int c = e->cur & 1;
    k_list_dsp<<<div_up(e->P, 256), 256, 0, e->stream>>>(e->lpos[c], e->lo[0], e->lo[1], e->lo[2], e->img, e->x0,
                                                         e->gid_of, e->rep_of_sid, e->d_sys, (int)e->P, e->dsp[0],
                                                         e->dsp[1], e->dsp[2]);
    BD_LAUNCH_CHECK();
    return BD_OK;
}

namespace {
// observation passes read cell buckets and displacements: rebuild them from
// the by-id state
int sync_buckets(bd_engine *e) {
    if (!e->list) return BD_OK;
    int rc = sync_dsp(e);
    return rc ? rc : list_bin(e, e->cur, e->d_one, nullptr);
}

// noise amplitudes of the next `count` list steps (count <= graph_steps)
int list_amplitudes(bd_engine *e, int count) {
    const int n = count * e->R;
    k_amp_table<<<div_up(n, 256), 256, 0, e->stream>>>(e->d_sys, e->R, e->d_ni, e->ni_first, count, e->amp_tab);
    BD_LAUNCH_CHECK();
    return BD_OK;
}

// k steps outside graphs (k = 1 in plain mode): launch, advance the counter
int direct_steps(bd_engine *e, int k) {
    if (e->list) {
        if (k > e->graph_steps) return BD_ERR_ARG;  // the amplitude table holds one batch
        if (int rc = list_amplitudes(e, k)) return rc;
        if (list_per_replica(e)) {
            if (int rc = list_replica_steps(e, e->cur, k)) return rc;
        } else {
            for (int i = 0; i < k; i++) {
                int rc = list_step(e, e->cur + i, i);
                if (rc) return rc;
            }
        }
        k_advance_counter<<<1, 1, 0, e->stream>>>(e->d_ni, k);
        BD_LAUNCH_CHECK();
        e->cur = (e->cur + k) & 1;
        e->ni += k;
        return BD_OK;
    }
    StepArgs a = make_args(e, e->cur, 1);
    int rc = e->mode == BD_MODE_PERSISTENT ? launch_persistent(e, a, k) : launch_step(e, a, 0, false, false);
    if (rc) return rc;
    k_advance_counter<<<1, 1, 0, e->stream>>>(e->d_ni, k);
    BD_LAUNCH_CHECK();
    e->cur = (e->cur + k) % 3;
    e->ni += k;
    return BD_OK;
}

int build_graph(bd_engine *e) {
    // The recorded launches bake in the buffer rotation of e->cur, so each
    // rotation phase gets its own graph.
    if (e->gexec[e->cur]) return BD_OK;
    cudaGraph_t g;
    BD_CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int rc = BD_OK;
    if (e->list) {
        rc = list_amplitudes(e, e->graph_steps);
        if (rc == BD_OK && list_per_replica(e)) rc = list_replica_steps(e, e->cur, e->graph_steps);
        else
            for (int j = 0; j < e->graph_steps && rc == BD_OK; j++) rc = list_step(e, e->cur + j, j);
    } else if (e->mode == BD_MODE_PERSISTENT) {
        StepArgs a = make_args(e, e->cur, 1);
        rc = launch_persistent(e, a, e->graph_steps);
    } else {
        for (int j = 0; j < e->graph_steps && rc == BD_OK; j++) {
            StepArgs a = make_args(e, e->cur + j, 1);
            rc = launch_step(e, a, j, false, false);
        }
    }
    if (rc == BD_OK) k_advance_counter<<<1, 1, 0, e->stream>>>(e->d_ni, e->graph_steps);
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (rc) return rc;
    BD_CUDA_TRY(ce);
    BD_CUDA_TRY(cudaGraphInstantiate(&e->gexec[e->cur], g, 0));
    cudaGraphDestroy(g);
    return BD_OK;
}

void free_engine(bd_engine *e) {
    for (int k = 0; k < 3; k++)
        if (e->gexec[k]) cudaGraphExecDestroy(e->gexec[k]);
    void *ptrs[] = {e->d_sys, e->d_bricks, e->cnt[0], e->cnt[1], e->cnt[2], e->pos[0], e->pos[1], e->pos[2],
                    e->lo[0], e->lo[1], e->lo[2], e->dsp[0], e->dsp[1], e->dsp[2], e->gid_of, e->rep_of_sid,
                    e->rep_of_gid, e->x0, e->obs, e->snap, e->nbr_count, e->nbr_hash, e->cr, e->noise,
                    e->status, e->d_ni, e->out_pos, e->out_raw, e->d_cl_start, e->d_cl_bricks, e->rn_ring, e->rn_lcg,
                    e->snaps, e->d_segs, e->d_seg_first, e->corr_part, e->corr_out, e->lpos[0], e->lpos[1],
                    e->pbuild, e->nbr, e->nnb, e->lflag, e->d_one, e->d_builds, e->ld_in, e->ld_staged,
                    e->ld_slot, e->ld_bucket, e->ld_cnt, e->ld_start, e->ld_bsum, e->ld_bad, e->img, e->amp_tab,
                    e->d_rep_order, e->d_step_rebuilt};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

// Brick decomposition of every replica for the current brick shape and CTA
// size; in persistent mode also the packing of replicas into cluster bins
// (longest-processing-time first by brick count).  Host side only.
int rebuild_bricks(bd_engine *e) {
    e->bricks_h.clear();
    for (int r = 0; r < e->R; r++) {
        SysDev &S = e->sysh[r];
        const int nc = S.ncell;
        S.nbx = (nc + e->bx - 1) / e->bx;
        S.nby = (nc + e->by - 1) / e->by;
        S.nbz = (nc + e->bz - 1) / e->bz;
        S.brick_base = (int)e->bricks_h.size();
        for (int z = 0; z < S.nbz; z++)
            for (int y = 0; y < S.nby; y++)
                for (int x = 0; x < S.nbx; x++) e->bricks_h.push_back(make_int4(r, x * e->bx, y * e->by, z * e->bz));
    }
    e->nbricks = (int)e->bricks_h.size();
    const int nh = (e->bx + 2) * (e->by + 2) * (e->bz + 2);
    // Staging capacity: the densest replica's mean cell occupancy over the
    // halo block with 25% + 32 slots of headroom (a liquid's particle count
    // in a few hundred cells varies by a few percent; a uniform random start
    // by ~4%), never above what the cells can hold.
    double occ = 0.0;
    for (int r = 0; r < e->R; r++) {
        const SysDev &S = e->sysh[r];
        occ = std::max(occ, (double)S.n / ((double)S.ncell * S.ncell * S.ncell));
    }
    const long long want = (long long)std::ceil(occ * nh * 1.25) + 32;
    e->smax = (int)std::min<long long>(std::min<long long>(65534, (long long)nh * e->cap), std::max(256LL, want)) & ~1;
    e->smem = brick_smem_bytes(nh, e->smax, e->threads);
    e->smem_census = e->smem;
    e->lsmem = brick_smem_bytes(nh, e->smax, kListBuildThreads);
    if (e->smem > 227 * 1024 || e->lsmem > 227 * 1024 || nh > 65535) return BD_ERR_ARG;
    e->cl_start_h.clear();
    e->cl_bricks_h.clear();
    if (e->mode == BD_MODE_PERSISTENT) {
        const int G = std::max(1, std::min(e->R, e->max_clusters > 0 ? e->max_clusters : e->R));
        std::vector<int> order(e->R);
        std::iota(order.begin(), order.end(), 0);
        auto nb_of = [&](int r) { const SysDev &S = e->sysh[r]; return S.nbx * S.nby * S.nbz; };
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return nb_of(a) > nb_of(b); });
        std::vector<long long> load(G, 0);
        std::vector<std::vector<int>> bins(G);
        for (int r : order) {
            int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            bins[g].push_back(r);
            load[g] += nb_of(r);
        }
        e->cl_start_h.push_back(0);
        for (int g = 0; g < G; g++) {
            std::sort(bins[g].begin(), bins[g].end());
            for (int r : bins[g]) {
                const SysDev &S = e->sysh[r];
                for (int b = 0; b < nb_of(r); b++) e->cl_bricks_h.push_back(S.brick_base + b);
            }
            e->cl_start_h.push_back((int)e->cl_bricks_h.size());
        }
        e->nclusters = G;
    }
    return BD_OK;
}

// Upload the brick layout (after rebuild_bricks) and drop graphs recorded
// for the previous layout.
int upload_layout(bd_engine *e) {
    for (int k = 0; k < 3; k++)
        if (e->gexec[k]) { cudaGraphExecDestroy(e->gexec[k]); e->gexec[k] = nullptr; }
    if (e->d_bricks) cudaFree(e->d_bricks);
    e->d_bricks = nullptr;
    BD_CUDA_TRY(cudaMalloc(&e->d_bricks, sizeof(int4) * e->nbricks));
    BD_CUDA_TRY(cudaMemcpyAsync(e->d_bricks, e->bricks_h.data(), sizeof(int4) * e->nbricks, cudaMemcpyHostToDevice,
                                e->stream));
    BD_CUDA_TRY(cudaMemcpyAsync(e->d_sys, e->sysh.data(), sizeof(SysDev) * e->R, cudaMemcpyHostToDevice, e->stream));
    if (e->d_cl_start) cudaFree(e->d_cl_start);
    if (e->d_cl_bricks) cudaFree(e->d_cl_bricks);
    e->d_cl_start = e->d_cl_bricks = nullptr;
    if (e->mode == BD_MODE_PERSISTENT) {
        BD_CUDA_TRY(cudaMalloc(&e->d_cl_start, sizeof(int) * e->cl_start_h.size()));
        BD_CUDA_TRY(cudaMalloc(&e->d_cl_bricks, sizeof(int) * std::max<size_t>(1, e->cl_bricks_h.size())));
        BD_CUDA_TRY(cudaMemcpyAsync(e->d_cl_start, e->cl_start_h.data(), sizeof(int) * e->cl_start_h.size(),
                                    cudaMemcpyHostToDevice, e->stream));
        BD_CUDA_TRY(cudaMemcpyAsync(e->d_cl_bricks, e->cl_bricks_h.data(), sizeof(int) * e->cl_bricks_h.size(),
                                    cudaMemcpyHostToDevice, e->stream));
    }
    BD_CUDA_TRY(cudaStreamSynchronize(e->stream));
    return configure_kernels(e);
}

int setup_geometry(bd_engine *e) {
    e->sysh.resize(e->R);
    long long cell_base = 0, part_base = 0;
    e->bricks_h.clear();
    for (int r = 0; r < e->R; r++) {
        const bd_system_desc &d = e->desc[r];
        SysDev &S = e->sysh[r];
        std::memset(&S, 0, sizeof(S));
        if (d.n_big < 0 || d.n_sml < 0 || d.n_big + d.n_sml < 1 || !(d.side > 0) || !(d.sigma_big > 0) ||
            !(d.sigma_sml > 0) || !(d.dt > 0))
            return BD_ERR_ARG;
        S.L = d.side;
        S.Linv = 1.0f / d.side;
        S.sig[0] = d.sigma_big;
        S.sig[1] = 0.5f * (d.sigma_big + d.sigma_sml);  // get_forces.cu:441
        S.sig[2] = d.sigma_sml;
        S.pot = d.potential;
        if (d.potential != kPotWcaModified) e->extra_pot = true;
        for (int k = 0; k < 4; k++) S.pp[k] = d.pot_param[k];
        if (S.pot < kPotWcaModified || S.pot > kPotHsay) return BD_ERR_ARG;
        if (S.pot == kPotAO && !(S.pp[2] > 0.f)) return BD_ERR_ARG;
        if (S.pot == kPotHsay && !(S.pp[1] >= 1.0f && S.pp[1] <= 4.0f)) return BD_ERR_ARG;
        float cut[3];
        for (int k = 0; k < 3; k++) {
            cut[k] = S.pot == kPotWcaModified ? S.sig[k] : S.sig[k] * pot_cut_factor(S.pot, S.pp, S.sig[k]);
            S.cut2[k] = cut[k] * cut[k];
        }
        float rcmax = std::max(cut[0], std::max(cut[1], cut[2]));
        const float skin = e->list ? e->skin : 0.f;  // list builds sweep cut + skin
        for (int k = 0; k < 3; k++) S.lcut2[k] = (cut[k] + skin) * (cut[k] + skin);
        S.skin_half2 = 0.25f * skin * skin;
        // list partners are within rcmax + skin at the build and each end has
        // moved at most skin / 2 since
        S.interior = rcmax + 2.0f * skin + 0.01f;
        int nc = (int)std::floor((double)d.side / ((double)(rcmax + skin) * (1.0 + 1e-5)));
        if (nc < 3) return BD_ERR_ARG;  // box too small for a 27-cell sweep
        // the list step's minimum image (min_image_pair) needs every list
        // partner well within L / 2 of the particle: with skin at most 0.9 of
        // the largest cut distance and three cells per side, within 0.492 L
        if (e->list && skin > 0.9f * rcmax) return BD_ERR_ARG;
        S.ncell = nc;
        S.cinv = (float)nc / d.side;
        S.cell_base = (int)cell_base;
        S.n = d.n_big + d.n_sml;
        S.n_big = d.n_big;
        S.part_base = (int)part_base;
        S.mob[0] = d.mob_big;
        S.mob[1] = d.mob_sml;
        S.dt = (float)d.dt;
        S.dt_d = d.dt;
        S.fcap = d.force_cap;
        S.protocol = d.temp_protocol;
        S.T0 = d.T0; S.Tf = d.Tf; S.t0 = d.t0; S.tf = d.tf; S.period = d.period;
        S.T_first = d.first_temp_set ? d.T_first : d.T0;
        S.seed = d.seed;
        cell_base += (long long)nc * nc * nc;
        part_base += S.n;
        if (cell_base > (1ll << 31) / e->cap || part_base >= (1ll << 31)) return BD_ERR_ARG;
    }
    e->C = cell_base;
    e->P = part_base;
    return rebuild_bricks(e);
}

}  // namespace

extern "C" {

void bd_engine_opts_default(bd_engine_opts *o) {
    std::memset(o, 0, sizeof(*o));
    o->rng = BD_RNG_PHILOX;
    o->cell_capacity = 16;
    o->mode = BD_MODE_AUTO;
    o->cluster = 8;
    o->graph_steps = 96;
    o->qmax = 6.2831853f;
    o->neighbor_skin = 0.25f;
    o->list_variant = -1;
}

int bd_engine_create(const bd_system_desc *systems, int nsys, const bd_engine_opts *opts_in, bd_engine **out) {
    if (!systems || nsys < 1 || !out) return BD_ERR_ARG;
    *out = nullptr;
    bd_engine_opts opts;
    if (opts_in) opts = *opts_in; else bd_engine_opts_default(&opts);
    bd_engine *e = new (std::nothrow) bd_engine();
    if (!e) return BD_ERR_NOMEM;
    if (cudaGetDevice(&e->dev) != cudaSuccess) { delete e; return BD_ERR_CUDA; }
    e->R = nsys;
    e->desc.assign(systems, systems + nsys);
    e->rng = opts.rng;
    if (e->rng < BD_RNG_PHILOX || e->rng > BD_RNG_RANNEW64) { delete e; return BD_ERR_ARG; }
    // list mode's cells are sized for cut + skin and hold about 1.7x more particles
    const bool want_list = opts.neighbor_skin > 0.f && opts.mode != BD_MODE_PERSISTENT && opts.rng != BD_RNG_NOISE;
    e->cap = opts.cell_capacity > 0 ? opts.cell_capacity : (want_list ? 24 : 16);
    if (e->cap > kQueue / 3) { delete e; return BD_ERR_ARG; }  // a row of 3 cells must fit one queue
    if (opts.brick[0] > 0 && opts.brick[1] > 0 && opts.brick[2] > 0) {
        e->bx = opts.brick[0]; e->by = opts.brick[1]; e->bz = opts.brick[2];
    }
    e->threads = opts.threads > 0 ? opts.threads : 128;
    if (e->threads % 32 || e->threads > 192) { delete e; return BD_ERR_ARG; }  // k_step launch bounds
    e->mode = opts.mode == BD_MODE_AUTO ? BD_MODE_PLAIN : opts.mode;
    e->cluster = opts.cluster > 0 ? opts.cluster : 8;
    e->graph_steps = opts.graph_steps > 0 ? ((opts.graph_steps + 2) / 3) * 3 : 96;
    e->qmax = opts.qmax != 0.f ? opts.qmax : 6.2831853f;
    e->ni = e->ni_first = opts.ni_start;
    e->rng_stream = opts.rng_stream;
    e->autotune = opts.autotune;
    if (opts.list_variant < -1 || opts.list_variant >= kListVariants) { delete e; return BD_ERR_ARG; }
    e->lvar = opts.list_variant >= 0 ? opts.list_variant : 0;
    e->tune_lvar = opts.list_variant < 0;
    if (!(opts.neighbor_skin >= 0.f) || opts.neighbor_skin > 1.0f) { delete e; return BD_ERR_ARG; }
    // lists serve plain mode with generated noise; a box too small for the
    // enlarged cells keeps the sweep
    e->list = opts.neighbor_skin > 0.f && e->mode == BD_MODE_PLAIN && e->rng != BD_RNG_NOISE;
    e->skin = e->list ? opts.neighbor_skin : 0.f;
    if (e->list) e->graph_steps = ((e->graph_steps + 5) / 6) * 6;  // keeps both buffer rotations in phase
    int rc = setup_geometry(e);
    if (rc == BD_ERR_ARG && e->list) {
        e->list = false;
        e->skin = 0.f;
        rc = setup_geometry(e);
    }
    if (rc) { delete e; return rc; }
    if (opts.cell_capacity <= 0) {
        // default capacity: room for twice the densest replica's mean cell
        // occupancy plus 8 (long cut distances make large cells)
        double occ = 0.0;
        for (const SysDev &S : e->sysh) occ = std::max(occ, (double)S.n / ((double)S.ncell * S.ncell * S.ncell));
        const int want = std::min(kQueue / 3, (int)std::ceil(2.0 * occ + 8.0));
        if (want > e->cap) {
            e->cap = want;
            if ((rc = setup_geometry(e))) { delete e; return rc; }
        }
    }
#define ALLOC(ptr, bytes)                                                    \
    do {                                                                     \
        if (cudaMalloc((void **)&(ptr), (bytes)) != cudaSuccess) {          \
            free_engine(e);                                                  \
            return BD_ERR_NOMEM;                                             \
        }                                                                    \
    } while (0)
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) { delete e; return BD_ERR_CUDA; }
    const size_t P = (size_t)e->P, C = (size_t)e->C;
    ALLOC(e->d_sys, sizeof(SysDev) * e->R);
    ALLOC(e->d_bricks, sizeof(int4) * e->nbricks);
    for (int k = 0; k < 3; k++) {
        ALLOC(e->cnt[k], sizeof(int) * C);
        ALLOC(e->pos[k], sizeof(float4) * C * e->cap);
        ALLOC(e->lo[k], sizeof(float) * P);
        ALLOC(e->dsp[k], sizeof(double) * P);
    }
    ALLOC(e->gid_of, sizeof(int) * P);
    ALLOC(e->rep_of_sid, sizeof(int) * P);
    ALLOC(e->rep_of_gid, sizeof(int) * P);
    ALLOC(e->x0, sizeof(double) * 3 * P);
    ALLOC(e->snap, sizeof(float4) * P);
    ALLOC(e->obs, sizeof(double) * kObsCount * e->R);
    ALLOC(e->status, 256);
    ALLOC(e->d_ni, sizeof(long long));
    if (e->rng == BD_RNG_CURAND) ALLOC(e->cr, sizeof(curandState) * P);
    if (e->rng == BD_RNG_NOISE) ALLOC(e->noise, sizeof(float) * 3 * P);
    if (e->rng == BD_RNG_RANNEW64) {
        ALLOC(e->rn_ring, sizeof(unsigned long long) * kRnWords * P);
        ALLOC(e->rn_lcg, sizeof(unsigned long long) * P);
    }
    if (e->list) {
        // one more entry: storage id P is the zero position that padded list
        // entries gather (never written after this)
        ALLOC(e->lpos[0], sizeof(float4) * (P + 1));
        ALLOC(e->lpos[1], sizeof(float4) * (P + 1));
        cudaMemsetAsync(e->lpos[0], 0, sizeof(float4) * (P + 1), e->stream);
        cudaMemsetAsync(e->lpos[1], 0, sizeof(float4) * (P + 1), e->stream);
        ALLOC(e->pbuild, sizeof(float4) * P);
        ALLOC(e->nbr, sizeof(int) * (size_t)kMaxNbr * P);
        ALLOC(e->nnb, sizeof(int) * P);
        ALLOC(e->img, sizeof(int) * 3 * P);
        ALLOC(e->amp_tab, sizeof(float) * 2 * (size_t)e->R * e->graph_steps);
        ALLOC(e->lflag, sizeof(int) * (e->R + 1));
        ALLOC(e->d_one, sizeof(int));
        ALLOC(e->d_builds, 3 * sizeof(long long));  // + the build's finished-block counter
        cudaMemsetAsync(e->d_builds, 0, 3 * sizeof(long long), e->stream);
        ALLOC(e->d_step_rebuilt, sizeof(int) * e->graph_steps);
        cudaMemsetAsync(e->d_step_rebuilt, 0, sizeof(int) * e->graph_steps, e->stream);
        ALLOC(e->d_rep_order, sizeof(int) * e->R);
        {  // blocks of a per-replica launch start with the largest replicas
            std::vector<int> order(e->R);
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(),
                             [&](int a, int b) { return e->sysh[a].n > e->sysh[b].n; });
            cudaMemcpyAsync(e->d_rep_order, order.data(), sizeof(int) * e->R, cudaMemcpyHostToDevice, e->stream);
            size_t need = 0;  // the largest in-block rebuild from shared memory
            for (int r = 0; r < e->R; r++) {
                const SysDev &S = e->sysh[r];
                need = std::max(need, replica_shared_build_bytes(S.n, S.ncell * S.ncell * S.ncell));
            }
            e->lrep_smem = need <= (size_t)227 * 1024 ? need : 0;
            cudaStreamSynchronize(e->stream);  // the host vector goes out of scope
        }
        const int one = 1;
        cudaMemcpyAsync(e->d_one, &one, sizeof(int), cudaMemcpyHostToDevice, e->stream);
    }
#undef ALLOC
    cudaMemcpyAsync(e->d_sys, e->sysh.data(), sizeof(SysDev) * e->R, cudaMemcpyHostToDevice, e->stream);
    cudaMemcpyAsync(e->d_bricks, e->bricks_h.data(), sizeof(int4) * e->nbricks, cudaMemcpyHostToDevice, e->stream);
    cudaMemsetAsync(e->status, 0, 256, e->stream);
    cudaMemcpyAsync(e->d_ni, &e->ni, sizeof(long long), cudaMemcpyHostToDevice, e->stream);
    std::vector<int> rog(P);
    for (int r = 0; r < e->R; r++)
        for (int i = 0; i < e->sysh[r].n; i++) rog[e->sysh[r].part_base + i] = r;
    cudaMemcpyAsync(e->rep_of_gid, rog.data(), sizeof(int) * P, cudaMemcpyHostToDevice, e->stream);
    if (e->rng == BD_RNG_CURAND) {
        k_curand_setup<<<div_up((long)P, 128), 128, 0, e->stream>>>(e->cr, e->d_sys, e->rep_of_gid, (int)P);
    }
    if (configure_kernels(e) != BD_OK) {
        free_engine(e);
        return BD_ERR_CUDA;
    }
    if (e->mode == BD_MODE_PERSISTENT) {  // as many cluster bins as can be resident at once
        if (e->cluster < 1 || e->cluster > 8) { free_engine(e); return BD_ERR_ARG; }
        e->max_clusters = max_active_clusters(e);
        if (e->max_clusters < 1) { free_engine(e); return BD_ERR_ARG; }
        if (rebuild_bricks(e) != BD_OK || upload_layout(e) != BD_OK) { free_engine(e); return BD_ERR_CUDA; }
    }
    if (cudaStreamSynchronize(e->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        free_engine(e);
        return BD_ERR_CUDA;
    }
    *out = e;
    return BD_OK;
}

int bd_engine_destroy(bd_engine *e) {
    if (!e) return BD_ERR_ARG;
    cudaStreamSynchronize(e->stream);
    free_engine(e);
    return BD_OK;
}

int bd_engine_get_info(const bd_engine *e, bd_engine_info *info) {
    if (!e || !info) return BD_ERR_ARG;
    std::memset(info, 0, sizeof(*info));
    info->nsys = e->R;
    info->n_particles = e->P;
    info->n_cells = e->C;
    info->brick[0] = e->bx; info->brick[1] = e->by; info->brick[2] = e->bz;
    info->threads = e->threads;
    info->cell_capacity = e->cap;
    info->staging_capacity = e->smax;
    info->mode = e->mode;
    info->cluster = e->cluster;
    info->smem_bytes = e->smem;
    info->next_step = e->ni;
    info->neighbor_skin = e->list ? e->skin : 0.f;
    if (e->list) {
        long long b[2];
        BD_CUDA_TRY(cudaMemcpyAsync(b, e->d_builds, sizeof(b), cudaMemcpyDeviceToHost, e->stream));
        BD_CUDA_TRY(cudaStreamSynchronize(e->stream));
        info->list_builds = b[0];
        info->list_rebuild_steps = b[1];
    }
    info->list_variant = e->list ? e->lvar : -1;
    info->tuned_ms = e->tuned ? e->tuned_ms : 0.f;
    return BD_OK;
}

int bd_engine_get_stream(const bd_engine *e, void **stream) {
    if (!e || !stream) return BD_ERR_ARG;
    *stream = (void *)e->stream;
    return BD_OK;
}

int bd_engine_set_positions(bd_engine *e, const float *pos) {
    if (!e || !pos) return BD_ERR_ARG;
    const size_t P = (size_t)e->P;
    // storage order: replica, brick, species, cell within brick, reference
    // index -- computed on the device (keys, counting sort over the slots,
    // per-slot sort by reference index).  Inside a cell the order is that of
    // the reference index either way (big particles come first), so the
    // species split changes no sweep or list order; it gives the list step
    // warps of one species, whose list lengths are alike.
    const long long V = (long long)e->bx * e->by * e->bz, T = (long long)e->nbricks * V * 2;
    if (T > INT_MAX) return BD_ERR_ARG;
    if (!e->ld_in) {
        BD_CUDA_TRY(cudaMalloc(&e->ld_in, sizeof(float) * 3 * P));
        BD_CUDA_TRY(cudaMalloc(&e->ld_staged, sizeof(float4) * P));
        BD_CUDA_TRY(cudaMalloc(&e->ld_slot, sizeof(int) * P));
        BD_CUDA_TRY(cudaMalloc(&e->ld_bucket, sizeof(int) * P));
        BD_CUDA_TRY(cudaMalloc(&e->ld_bad, sizeof(unsigned)));
    }
    if (T > e->ld_slots) {  // the brick shape sets the slot count
        if (e->ld_cnt) cudaFree(e->ld_cnt);
        if (e->ld_start) cudaFree(e->ld_start);
        if (e->ld_bsum) cudaFree(e->ld_bsum);
        e->ld_cnt = e->ld_start = e->ld_bsum = nullptr;
        e->ld_slots = 0;
        BD_CUDA_TRY(cudaMalloc(&e->ld_cnt, sizeof(int) * T));
        BD_CUDA_TRY(cudaMalloc(&e->ld_start, sizeof(int) * T));
        BD_CUDA_TRY(cudaMalloc(&e->ld_bsum, sizeof(int) * (T / kScanBlock + 1)));
        e->ld_slots = T;
    }
    const int n = (int)T, nb = (int)div_up(T, kScanBlock);
    const int gp = rebuild_grid(e, div_up((long long)P, 256)), gt = rebuild_grid(e, div_up(T, 256));
    BD_CUDA_TRY(cudaMemcpyAsync(e->ld_in, pos, sizeof(float) * 3 * P, cudaMemcpyHostToDevice, e->stream));
    cudaMemsetAsync(e->ld_cnt, 0, sizeof(int) * T, e->stream);
    cudaMemsetAsync(e->ld_bad, 0, sizeof(unsigned), e->stream);
    k_order_keys<<<gp, 256, 0, e->stream>>>(e->ld_in, (int)P, e->rep_of_gid, e->d_sys, e->bx, e->by, e->bz,
                                            e->ld_slot, e->ld_cnt, e->ld_bad);
    BD_LAUNCH_CHECK();
    unsigned bad = 0;
    BD_CUDA_TRY(cudaMemcpyAsync(&bad, e->ld_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    BD_CUDA_TRY(cudaStreamSynchronize(e->stream));
    if (bad) return BD_ERR_ARG;  // nothing of the engine state has changed
    int *start = e->ld_start;  // the scan runs on a copy of the counts
    cudaMemcpyAsync(start, e->ld_cnt, sizeof(int) * T, cudaMemcpyDeviceToDevice, e->stream);
    k_scan_local<<<nb, kScanThreads, 0, e->stream>>>(start, n, e->ld_bsum);
    k_scan_totals<<<1, kScanThreads, 0, e->stream>>>(e->ld_bsum, nb);
    k_scan_add<<<div_up(T, 256), 256, 0, e->stream>>>(start, n, e->ld_bsum);
    k_order_fill<<<gp, 256, 0, e->stream>>>(e->ld_slot, (int)P, start, e->ld_cnt, e->ld_bucket);
    k_order_emit<<<gt, 256, 0, e->stream>>>(start, n, (int)P, e->cap, e->ld_bucket, e->ld_in, e->rep_of_gid,
                                            e->d_sys, e->ld_staged, e->gid_of, e->rep_of_sid);
    BD_LAUNCH_CHECK();
    for (int k = 0; k < 3; k++) {
        cudaMemsetAsync(e->cnt[k], 0, sizeof(int) * e->C, e->stream);
        cudaMemsetAsync(e->lo[k], 0, sizeof(float) * P, e->stream);
        cudaMemsetAsync(e->dsp[k], 0, sizeof(double) * P, e->stream);
    }
    if (e->img) cudaMemsetAsync(e->img, 0, sizeof(int) * 3 * P, e->stream);
    cudaMemsetAsync(e->status, 0, 256, e->stream);
    e->cur = 0;
    e->generation++;  // displacement snapshots of earlier positions are void
    if (e->rng == BD_RNG_RANNEW64) {  // streams keyed by particle, stored by storage id
        e->rn_ni0 = e->ni;
        for (int g = 0; g < 3; g++)
            if (e->gexec[g]) { cudaGraphExecDestroy(e->gexec[g]); e->gexec[g] = nullptr; }
    }
    k_load<<<div_up((long)P, 256), 256, 0, e->stream>>>(e->ld_staged, (int)P, e->rep_of_sid, e->d_sys, e->cnt[0],
                                                        e->pos[0], e->cap, e->x0, e->gid_of, e->status,
                                                        e->list ? e->lpos[0] : nullptr);
    if (e->list) {  // every replica's lists are built before its first step
        std::vector<int> ones(e->R + 1, 1);
        cudaMemcpyAsync(e->lflag, ones.data(), sizeof(int) * (e->R + 1), cudaMemcpyHostToDevice, e->stream);
    }
    if (e->rng == BD_RNG_RANNEW64)
        k_rannew64_seed<<<div_up((long)P, 128), 128, 0, e->stream>>>(e->rn_ring, e->rn_lcg, e->d_sys, e->rep_of_sid,
                                                                     e->gid_of, (int)P);
    cudaError_t le = cudaGetLastError();
    cudaStreamSynchronize(e->stream);
    if (le != cudaSuccess) return BD_ERR_CUDA;

    e->loaded = true;
    return engine_status(e);
}

}  // extern "C"

namespace {
// Steps issued directly (no graph): one persistent launch, or k plain launches.
int run_direct(bd_engine *e, int k) {
    if (k <= 0) return BD_OK;
    if (e->mode == BD_MODE_PERSISTENT) return direct_steps(e, k);
    for (int i = 0; i < k; i++) {
        int rc = direct_steps(e, 1);
        if (rc) return rc;
    }
    return BD_OK;
}

// Project autotuner: times brick shapes x CTA sizes (and cluster sizes in
// persistent mode) on the live batch and keeps the fastest.  The steps it
// takes are real steps of the run; results do not depend on the layout
// (every force sum has a fixed order), only the speed does.
// List mode, in two stages, on the live batch with rebuilds as they come:
// 1. the list-build brick shape and the per-step launch variant (0-2), each
//    pair over 2 + 12 steps launched one by one;
// 2. the winner of stage 1 against the per-replica variants (3-5), each over
//    one whole graph batch (graph_steps steps, graph instantiated before the
//    timer starts) after 2 warm-up steps: a per-replica launch pays each
//    block's cold start and in-block rebuilds once per launch, so a
//    12-step window does not rank it (it ranks the per-step variants
//    correctly, whose launches are the same in and out of graphs).
// Neither choice changes a list or a force sum, so the tuned run's results
// are those of an untuned run.
int autotune_list(bd_engine *e, long long &nsteps) {
    static const int shapes[][3] = {{4, 4, 3}, {4, 4, 4}, {3, 3, 3}, {5, 4, 4}, {4, 4, 2}};
    struct Cand { int bx, by, bz, v; };
    std::vector<Cand> stage1, stage2;
    for (int v = 0; v < kListVariants; v++) {
        if (!(e->tune_lvar || v == e->lvar)) continue;
        if (v >= kListFirstPersistent) {  // builds its lists in the block: no brick shape to choose
            if (e->rng == BD_RNG_PHILOX) stage2.push_back({e->bx, e->by, e->bz, v});
            continue;
        }
        for (auto &sh : shapes) stage1.push_back({sh[0], sh[1], sh[2], v});
    }
    const int warm = 2, timed = 12;
    const int n2 = (int)stage2.size() + (stage1.empty() || stage2.empty() ? 0 : 1);
    const long long need = (long long)stage1.size() * (warm + timed) + (long long)n2 * (warm + e->graph_steps) + 1;
    if (nsteps < need) return BD_OK;  // too short to tune now
    cudaEvent_t t0, t1;
    BD_CUDA_TRY(cudaEventCreate(&t0));
    BD_CUDA_TRY(cudaEventCreate(&t1));
    int rc = BD_OK;
    auto apply = [&](const Cand &c) -> int {
        e->bx = c.bx; e->by = c.by; e->bz = c.bz; e->lvar = c.v;
        if (rebuild_bricks(e) != BD_OK) return -1;  // staging of this shape does not fit
        int r = configure_kernels(e);
        return r ? r : upload_layout(e);
    };
    auto elapsed = [&](float &ms) -> int {
        BD_CUDA_TRY(cudaEventRecord(t1, e->stream));
        if (int r = engine_status(e)) return r;
        BD_CUDA_TRY(cudaEventElapsedTime(&ms, t0, t1));
        return BD_OK;
    };
    Cand best = {e->bx, e->by, e->bz, e->lvar};
    float best_ms = 1e30f;  // per step
    for (const Cand &c : stage1) {
        const int a = apply(c);
        if (a < 0) continue;
        if ((rc = a) != BD_OK) break;
        if ((rc = direct_steps(e, warm)) != BD_OK) break;
        BD_CUDA_TRY(cudaEventRecord(t0, e->stream));
        if ((rc = direct_steps(e, timed)) != BD_OK) break;
        float ms = 0.f;
        if ((rc = elapsed(ms)) != BD_OK) break;
        nsteps -= warm + timed;
        if (ms / timed < best_ms) { best_ms = ms / timed; best = c; }
    }
    if (rc == BD_OK && !stage2.empty()) {
        if (!stage1.empty()) stage2.insert(stage2.begin(), best);
        best_ms = 1e30f;
        for (const Cand &c : stage2) {
            const int a = apply(c);
            if (a < 0) continue;
            if ((rc = a) != BD_OK) break;
            if ((rc = direct_steps(e, warm)) != BD_OK) break;
            if ((rc = build_graph(e)) != BD_OK) break;
            BD_CUDA_TRY(cudaEventRecord(t0, e->stream));
            BD_CUDA_TRY(cudaGraphLaunch(e->gexec[e->cur], e->stream));
            e->ni += e->graph_steps;  // cur unchanged: graph_steps is a multiple of 6 in list mode
            float ms = 0.f;
            if ((rc = elapsed(ms)) != BD_OK) break;
            nsteps -= warm + e->graph_steps;
            if (ms / e->graph_steps < best_ms) { best_ms = ms / e->graph_steps; best = c; }
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc) return rc;
    if ((rc = apply(best)) != BD_OK) return rc < 0 ? BD_ERR_CUDA : rc;
    e->tuned = true;
    e->tuned_ms = best_ms;
    return BD_OK;
}

int autotune_layout(bd_engine *e, long long &nsteps) {
    if (e->list) return autotune_list(e, nsteps);
    struct Cand { int bx, by, bz, t, cl; };
    static const int shapes[][4] = {{4, 4, 3, 128}, {4, 4, 4, 160}, {5, 4, 4, 192}, {4, 3, 3, 96}, {3, 3, 3, 64},
                                    {4, 4, 2, 96},  {2, 2, 2, 64},  {3, 3, 2, 64},  {6, 4, 3, 192}};
    std::vector<Cand> cands;
    for (auto &s : shapes) {
        if (e->mode == BD_MODE_PERSISTENT) {
            for (int cl : {8, 4, 2}) cands.push_back({s[0], s[1], s[2], s[3], cl});
        } else {
            cands.push_back({s[0], s[1], s[2], s[3], e->cluster});
        }
    }
    const int warm = 2, timed = 6;
    if (nsteps < (long long)cands.size() * (warm + timed) + 1) return BD_OK;  // too short to tune now
    cudaEvent_t t0, t1;
    BD_CUDA_TRY(cudaEventCreate(&t0));
    BD_CUDA_TRY(cudaEventCreate(&t1));
    const Cand orig = {e->bx, e->by, e->bz, e->threads, e->cluster};
    Cand best = orig;
    float best_ms = 1e30f;
    int rc = BD_OK;
    for (const Cand &c : cands) {
        e->bx = c.bx; e->by = c.by; e->bz = c.bz; e->threads = c.t; e->cluster = c.cl;
        if (rebuild_bricks(e) != BD_OK) continue;
        if (e->mode == BD_MODE_PERSISTENT) {
            if ((rc = configure_kernels(e)) != BD_OK) break;
            e->max_clusters = max_active_clusters(e);
            if (e->max_clusters < 1 || rebuild_bricks(e) != BD_OK) continue;
        }
        if ((rc = upload_layout(e)) != BD_OK) break;
        if ((rc = run_direct(e, warm)) != BD_OK) break;
        BD_CUDA_TRY(cudaEventRecord(t0, e->stream));
        if ((rc = run_direct(e, timed)) != BD_OK) break;
        BD_CUDA_TRY(cudaEventRecord(t1, e->stream));
        if ((rc = engine_status(e)) != BD_OK) break;
        float ms = 0.f;
        BD_CUDA_TRY(cudaEventElapsedTime(&ms, t0, t1));
        nsteps -= warm + timed;
        if (ms < best_ms) { best_ms = ms; best = c; }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc) return rc;
    e->bx = best.bx; e->by = best.by; e->bz = best.bz; e->threads = best.t; e->cluster = best.cl;
    if ((rc = rebuild_bricks(e)) != BD_OK) return rc;
    if (e->mode == BD_MODE_PERSISTENT) {
        if ((rc = configure_kernels(e)) != BD_OK) return rc;
        e->max_clusters = max_active_clusters(e);
        if ((rc = rebuild_bricks(e)) != BD_OK) return rc;
    }
    if ((rc = upload_layout(e)) != BD_OK) return rc;
    e->tuned = true;
    e->tuned_ms = best_ms / timed;
    return BD_OK;
}
}  // namespace

extern "C" {

int bd_engine_run(bd_engine *e, long long nsteps) {
    if (!e || nsteps < 0) return BD_ERR_ARG;
    if (!e->loaded) return BD_ERR_STATE;
    if (e->rng == BD_RNG_NOISE && nsteps > 1) return BD_ERR_ARG;  // one injected step at a time
    if (e->autotune && !e->tuned && e->rng != BD_RNG_NOISE) {
        int rc = autotune_layout(e, nsteps);
        if (rc) return rc;
    }
    while (nsteps > 0) {
        if (nsteps >= e->graph_steps && e->rng != BD_RNG_NOISE) {
            int rc = build_graph(e);
            if (rc) return rc;
            BD_CUDA_TRY(cudaGraphLaunch(e->gexec[e->cur], e->stream));
            e->ni += e->graph_steps;  // cur unchanged: graph_steps is a multiple of 3
            nsteps -= e->graph_steps;
        } else {
            int rc = run_direct(e, (int)nsteps);
            if (rc) return rc;
            nsteps = 0;
        }
    }
    return engine_status(e);
}

int bd_engine_observe(bd_engine *e, bd_observables *out) {
    if (!e || !out) return BD_ERR_ARG;
    if (!e->loaded) return BD_ERR_STATE;
    BD_CUDA_TRY(cudaMemsetAsync(e->obs, 0, sizeof(double) * kObsCount * e->R, e->stream));
    int rc0 = sync_buckets(e);
    if (rc0) return rc0;
    StepArgs a = make_args(e, obs_buf(e), 0);
    int rc = launch_step(e, a, 0, true, false);
    if (rc) return rc;
    std::vector<double> h((size_t)kObsCount * e->R);
    BD_CUDA_TRY(cudaMemcpyAsync(h.data(), e->obs, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, e->stream));
    rc = engine_status(e);
    for (int r = 0; r < e->R; r++) {
        const SysDev &S = e->sysh[r];
        const double *o = h.data() + (size_t)r * kObsCount;
        const int nb = S.n_big, ns = S.n - S.n_big;
        bd_observables &v = out[r];
        v.energy_big = nb ? 0.5 * o[kObsPotBig] / nb : 0.0;
        v.energy_sml = ns ? 0.5 * o[kObsPotSml] / ns : 0.0;
        v.virial = o[kObsVir];
        v.msd_big = nb ? o[kObsMsdBig] / nb : 0.0;
        v.msd_sml = ns ? o[kObsMsdSml] / ns : 0.0;
        v.fself_big = nb ? o[kObsFsBig] / nb : 0.0;
        v.nbr_pairs = 0.0;
        // temp_set after the last completed step ni-1: time = dt (1 + (float)(ni-1))
        const bd_system_desc &d = e->desc[r];
        float t = (float)(d.dt * (1.0 + (float)(e->ni - 1)));
        float T = d.T0;
        if (e->ni > e->ni_first) {
            if (d.temp_protocol == BD_PROTOCOL_LINEAR) T = bd_calculate_temp_linear(d.T0, d.Tf, d.t0, d.tf, t);
            else if (d.temp_protocol == BD_PROTOCOL_SINE) T = bd_calculate_temp_sine(d.T0, d.Tf, d.t0, d.tf, d.period, t);
        }
        v.temperature = T;
    }
    return rc;
}

int bd_engine_get_positions(bd_engine *e, float *pos_host, float *raw_host) {
    if (!e) return BD_ERR_ARG;
    if (!e->loaded) return BD_ERR_STATE;
    const size_t P = (size_t)e->P;
    if (!e->out_pos) {
        if (cudaMalloc(&e->out_pos, sizeof(float) * 3 * P) != cudaSuccess) return BD_ERR_NOMEM;
        if (cudaMalloc(&e->out_raw, sizeof(float) * 3 * P) != cudaSuccess) return BD_ERR_NOMEM;
    }
    {
        int rcb = sync_buckets(e);
        if (rcb) return rcb;
    }
    k_export<<<div_up(e->C, 128), 128, 0, e->stream>>>(e->cnt[obs_buf(e)], e->pos[obs_buf(e)], (int)e->C, e->cap, (int)e->P, e->gid_of,
                                                       e->x0, e->dsp[0], e->dsp[1], e->dsp[2], e->out_pos,
                                                       e->out_raw, e->snap);
    BD_LAUNCH_CHECK();
    if (pos_host) BD_CUDA_TRY(cudaMemcpyAsync(pos_host, e->out_pos, sizeof(float) * 3 * P, cudaMemcpyDeviceToHost, e->stream));
    if (raw_host) BD_CUDA_TRY(cudaMemcpyAsync(raw_host, e->out_raw, sizeof(float) * 3 * P, cudaMemcpyDeviceToHost, e->stream));
    return engine_status(e);
}

int bd_engine_gder_method(bd_engine *e, int nbins, float range, int method, unsigned long long *counts_host) {
    if (!e || !counts_host || nbins < 1 || nbins > 4096 || !(range > 0)) return BD_ERR_ARG;
    if (method != BD_GDER_AUTO && method != BD_GDER_ALL_PAIRS && method != BD_GDER_CELLS) return BD_ERR_ARG;
    if (!e->loaded) return BD_ERR_STATE;
    if (int rcb = sync_buckets(e)) return rcb;
    // per replica: cell-bounded whenever the stencil applies (it skips cells
    // beyond the range and evaluates each unordered pair once; on the aging
    // boxes, a region as large as the box, it measured 90 ms against 220 ms
    // of all pairs for 64 x 32768 particles, 400 bins to 15)
    std::vector<int> m_of(e->R, -1);
    bool any_all = false;
    for (int r = 0; r < e->R; r++) {
        const SysDev &S = e->sysh[r];
        const int m = gder_cell_reach(S, range);
        if (method == BD_GDER_CELLS && m < 0) return BD_ERR_ARG;
        const bool cells = m >= 0 && (method == BD_GDER_CELLS || method == BD_GDER_AUTO);
        m_of[r] = cells ? m : -1;
        any_all |= !cells;
    }
    unsigned long long *d_counts = nullptr;
    const size_t per = (size_t)4 * nbins;
    // counts, then the nbins + 2 bin thresholds (gr_bin_thr)
    BD_CUDA_TRY(cudaMalloc(&d_counts, sizeof(unsigned long long) * per * e->R + sizeof(float) * (nbins + 2)));
    float *d_thr = reinterpret_cast<float *>(d_counts + per * e->R);
    cudaMemsetAsync(d_counts, 0, sizeof(unsigned long long) * per * e->R, e->stream);
    k_gr_thresholds<<<div_up(nbins + 2, 128), 128, 0, e->stream>>>(range, nbins, d_thr);
    int rc = launch_gder_cells(e, m_of, nbins, range, d_thr, d_counts);  // may hand replicas back
    for (int r = 0; r < e->R; r++) any_all |= m_of[r] < 0;
    cudaError_t le = cudaSuccess;
    if (rc == BD_OK && any_all) {
        k_export<<<div_up(e->C, 128), 128, 0, e->stream>>>(e->cnt[obs_buf(e)], e->pos[obs_buf(e)], (int)e->C, e->cap, (int)e->P,
                                                           e->gid_of, e->x0, e->dsp[0], e->dsp[1], e->dsp[2], nullptr,
                                                           nullptr, e->snap);
        // one histogram copy per two warps when 4 of them fit beside the tile
        const int copies = (size_t)4 * per * sizeof(unsigned) <= 96 * 1024 ? 4 : 1;
        const size_t sm = kGrTile * sizeof(float4) + sizeof(float) * (nbins + 2) + copies * per * sizeof(unsigned);
        cudaFuncSetAttribute(k_gr_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        const int jchunk = 8192;
        std::vector<int> reps;
        int nmax = 0;
        for (int r = 0; r < e->R; r++)
            if (m_of[r] < 0) {
                reps.push_back(r);
                nmax = std::max(nmax, e->sysh[r].n);
            }
        int *d_reps = nullptr;
        le = cudaMalloc(&d_reps, sizeof(int) * reps.size());
        if (le == cudaSuccess)
            le = cudaMemcpyAsync(d_reps, reps.data(), sizeof(int) * reps.size(), cudaMemcpyHostToDevice, e->stream);
        if (le == cudaSuccess && nmax > 0) {
            dim3 grid(div_up(nmax, 256), div_up(nmax, jchunk), (unsigned)reps.size());
            k_gr_batch<<<grid, 256, sm, e->stream>>>(e->snap, e->d_sys, d_reps, range, d_thr, nbins, jchunk, copies,
                                                     d_counts);
        }
        if (le == cudaSuccess) le = cudaStreamSynchronize(e->stream);
        if (d_reps) cudaFree(d_reps);
        if (le != cudaSuccess) rc = BD_ERR_CUDA;
        le = cudaGetLastError();
        if (le != cudaSuccess) rc = BD_ERR_CUDA;
    }
    cudaMemcpyAsync(counts_host, d_counts, sizeof(unsigned long long) * per * e->R, cudaMemcpyDeviceToHost, e->stream);
    cudaStreamSynchronize(e->stream);
    cudaFree(d_counts);
    if (rc) return rc;
    return engine_status(e);
}

int bd_engine_gder(bd_engine *e, int nbins, float range, unsigned long long *counts_host) {
    return bd_engine_gder_method(e, nbins, range, BD_GDER_AUTO, counts_host);
}

int bd_engine_set_noise(bd_engine *e, const float *noise_host) {
    if (!e || !noise_host || e->rng != BD_RNG_NOISE) return BD_ERR_ARG;
    BD_CUDA_TRY(cudaMemcpyAsync(e->noise, noise_host, sizeof(float) * 3 * e->P, cudaMemcpyHostToDevice, e->stream));
    return BD_OK;
}

int bd_engine_census(bd_engine *e, int *nbr_count, unsigned long long *nbr_hash) {
    if (!e || !nbr_count || !nbr_hash) return BD_ERR_ARG;
    if (!e->loaded) return BD_ERR_STATE;
    if (!e->nbr_count) {
        if (cudaMalloc(&e->nbr_count, sizeof(int) * e->P) != cudaSuccess) return BD_ERR_NOMEM;
        if (cudaMalloc(&e->nbr_hash, sizeof(unsigned long long) * e->P) != cudaSuccess) return BD_ERR_NOMEM;
    }
    BD_CUDA_TRY(cudaMemsetAsync(e->obs, 0, sizeof(double) * kObsCount * e->R, e->stream));
    int rc;
    if (e->list) {  // from the lists themselves (rebuilt first if they are stale)
        if ((rc = list_rebuild(e, e->cur))) return rc;
        k_census_list<<<div_up(e->P, 256), 256, 0, e->stream>>>(make_largs(e, e->cur), e->obs);
        BD_LAUNCH_CHECK();
    } else {
        StepArgs a = make_args(e, e->cur, 0);
        a.nbr_count = e->nbr_count;
        a.nbr_hash = e->nbr_hash;
        if ((rc = launch_step(e, a, 0, false, true))) return rc;
    }
    BD_CUDA_TRY(cudaMemcpyAsync(nbr_count, e->nbr_count, sizeof(int) * e->P, cudaMemcpyDeviceToHost, e->stream));
    BD_CUDA_TRY(cudaMemcpyAsync(nbr_hash, e->nbr_hash, sizeof(unsigned long long) * e->P, cudaMemcpyDeviceToHost, e->stream));
    return engine_status(e);
}

}  // extern "C"
