// correlate.cu -- waiting-time correlations of the batched replica engine:
// displacement snapshots kept on the device and one batched reduction of
// F_s(q; t_w, t_w + tau), MSD and the fourth moment of the displacement for
// every (snapshot, replica) pair.
//
// The reference measures aging by restarting the program from the
// configuration saved at each waiting time (main.cu:809-835, decade loop of
// run-fself.sh:149-197) and evaluating fself_isotropic (fself.cu:3-21) and
// the MSD loop (main.cu:776-797) on the host against the restart origin
// (main.cu:497-506).  Here every waiting time is a snapshot slot of the same
// run: slot k holds the FP64 displacement of every particle at t_w(k), and
// a correlation of slot k at time t reduces dr = dsp(t) - dsp(t_w(k)).
//
// Reduction layout: a replica's storage ids are contiguous, so the batch is
// cut into segments of kCorrChunk ids that never straddle two replicas.
// k_corr_partial writes one partial sum per (segment, slot, field);
// k_corr_finish adds a replica's segments in index order.  No atomics: the
// result is bit-reproducible.
#include <climits>
#include <vector>

#include "engine_state.cuh"

namespace bd {

constexpr int kCorrThreads = 256;
constexpr int kCorrPerThread = 4;
constexpr int kCorrChunk = kCorrThreads * kCorrPerThread;
constexpr int kCorrFields = 6;  // msd, r4, fs of big; msd, r4, fs of small
constexpr int kMaxCorrSlots = 64;

struct SlotList {
    int n;
    int slot[kMaxCorrSlots];
};

__global__ void __launch_bounds__(kCorrThreads) k_corr_partial(const int2 *__restrict__ segs,
                                                               const SysDev *__restrict__ sys,
                                                               const int *__restrict__ gid_of,
                                                               const double *__restrict__ dx,
                                                               const double *__restrict__ dy,
                                                               const double *__restrict__ dz,
                                                               const double *__restrict__ snaps, long long P,
                                                               SlotList sl, double q, double *__restrict__ part) {
    // per-warp partial sums of every slot; one barrier, then a fixed-order
    // reduction over the warps
    __shared__ double red[kMaxCorrSlots][kCorrThreads / 32][kCorrFields];
    const int2 sg = segs[blockIdx.x];  // (replica, first storage id)
    const SysDev &S = sys[sg.x];
    const int end = min(sg.y + kCorrChunk, S.part_base + S.n);
    double px[kCorrPerThread], py[kCorrPerThread], pz[kCorrPerThread];
    int sid[kCorrPerThread];
    bool big[kCorrPerThread];
#pragma unroll
    for (int i = 0; i < kCorrPerThread; i++) {
        sid[i] = sg.y + threadIdx.x + kCorrThreads * i;
        px[i] = py[i] = pz[i] = 0.0;
        big[i] = false;
        if (sid[i] < end) {
            px[i] = dx[sid[i]];
            py[i] = dy[sid[i]];
            pz[i] = dz[sid[i]];
            big[i] = gid_of[sid[i]] - S.part_base < S.n_big;
        } else {
            sid[i] = -1;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll 2
    for (int j = 0; j < sl.n; j++) {
        const double *bx = snaps + (size_t)sl.slot[j] * 3 * (size_t)P;
        const double *by = bx + P, *bz = by + P;
        double acc[kCorrFields];
#pragma unroll
        for (int f = 0; f < kCorrFields; f++) acc[f] = 0.0;
#pragma unroll
        for (int i = 0; i < kCorrPerThread; i++) {
            if (sid[i] < 0) continue;
            const double ex = px[i] - bx[sid[i]], ey = py[i] - by[sid[i]], ez = pz[i] - bz[sid[i]];
            const double r2 = ex * ex + ey * ey + ez * ez;
            const double qr = q * sqrt(r2);
            const double fs = qr > 0.0 ? sin(qr) / qr : 1.0;
            const int o = big[i] ? 0 : 3;
            acc[o] += r2;
            acc[o + 1] += r2 * r2;
            acc[o + 2] += fs;
        }
#pragma unroll
        for (int f = 0; f < kCorrFields; f++) {
            double v = acc[f];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0) red[j][warp][f] = v;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < sl.n * kCorrFields; t += kCorrThreads) {
        const int j = t / kCorrFields, f = t % kCorrFields;
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kCorrThreads / 32; w++) v += red[j][w][f];
        part[((size_t)blockIdx.x * sl.n + j) * kCorrFields + f] = v;
    }
}

// out[(j * R + r) * kCorrFields + f] = sum over the segments of replica r
__global__ void k_corr_finish(const int *__restrict__ seg_first, const double *__restrict__ part, int nslot, int R,
                              double *__restrict__ out) {
    const int r = blockIdx.x, t = threadIdx.x;
    if (t >= nslot * kCorrFields) return;
    const int j = t / kCorrFields, f = t % kCorrFields;
    double v = 0.0;
    for (int s = seg_first[r]; s < seg_first[r + 1]; s++) v += part[((size_t)s * nslot + j) * kCorrFields + f];
    out[((size_t)j * R + r) * kCorrFields + f] = v;
}

// out[3 * gid + k] = displacement component k of the particle with global index gid
__global__ void k_export_dsp(const int *__restrict__ gid_of, const double *__restrict__ dx,
                             const double *__restrict__ dy, const double *__restrict__ dz, int P,
                             double *__restrict__ out) {
    const int sid = blockIdx.x * blockDim.x + threadIdx.x;
    if (sid >= P) return;
    const int g = gid_of[sid];
    out[3 * (size_t)g] = dx[sid];
    out[3 * (size_t)g + 1] = dy[sid];
    out[3 * (size_t)g + 2] = dz[sid];
}

namespace {

int ensure_segments(bd_engine *e) {
    if (e->d_segs) return BD_OK;
    std::vector<int2> segs;
    std::vector<int> first(1, 0);
    for (int r = 0; r < e->R; r++) {
        const SysDev &S = e->sysh[r];
        for (int s = 0; s < S.n; s += kCorrChunk) segs.push_back(make_int2(r, S.part_base + s));
        first.push_back((int)segs.size());
    }
    e->nsegs = (int)segs.size();
    BD_CUDA_TRY(cudaMalloc(&e->d_segs, sizeof(int2) * segs.size()));
    BD_CUDA_TRY(cudaMalloc(&e->d_seg_first, sizeof(int) * first.size()));
    BD_CUDA_TRY(cudaMemcpyAsync(e->d_segs, segs.data(), sizeof(int2) * segs.size(), cudaMemcpyHostToDevice,
                                e->stream));
    BD_CUDA_TRY(cudaMemcpyAsync(e->d_seg_first, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice,
                                e->stream));
    return BD_OK;
}

int ensure_scratch(double *&buf, size_t &cap, size_t n) {
    if (cap >= n) return BD_OK;
    if (buf) cudaFree(buf);
    buf = nullptr;
    cap = 0;
    BD_CUDA_TRY(cudaMalloc(&buf, sizeof(double) * n));
    cap = n;
    return BD_OK;
}

}  // namespace
}  // namespace bd

using namespace bd;

extern "C" {

int bd_engine_reserve_snapshots(bd_engine *e, int nslots) {
    if (!e || nslots < 0) return BD_ERR_ARG;
    if (nslots <= e->nslots) return BD_OK;
    const size_t per = 3 * (size_t)e->P;
    double *buf = nullptr;
    BD_CUDA_TRY(cudaMalloc(&buf, sizeof(double) * per * nslots));
    if (e->snaps) {
        BD_CUDA_TRY(cudaMemcpyAsync(buf, e->snaps, sizeof(double) * per * e->nslots, cudaMemcpyDeviceToDevice,
                                    e->stream));
        BD_CUDA_TRY(cudaStreamSynchronize(e->stream));
        cudaFree(e->snaps);
    }
    e->snaps = buf;
    e->nslots = nslots;
    e->snap_ni.resize(nslots, LLONG_MIN);
    e->snap_gen.resize(nslots, -1);
    return BD_OK;
}

int bd_engine_snapshot(bd_engine *e, int slot) {
    if (!e || slot < 0 || slot >= e->nslots) return BD_ERR_ARG;
    if (!e->loaded) return BD_ERR_STATE;
    const size_t P = (size_t)e->P;
    double *dst = e->snaps + (size_t)slot * 3 * P;
    if (e->ni == 0) {
        // the next update re-bases every displacement to zero (main.cu:497-506):
        // a snapshot taken here is that origin
        BD_CUDA_TRY(cudaMemsetAsync(dst, 0, sizeof(double) * 3 * P, e->stream));
    } else {
        if (int rc = sync_dsp(e)) return rc;
        for (int k = 0; k < 3; k++)
            BD_CUDA_TRY(cudaMemcpyAsync(dst + k * P, e->dsp[k], sizeof(double) * P, cudaMemcpyDeviceToDevice,
                                        e->stream));
    }
    e->snap_ni[slot] = e->ni;
    e->snap_gen[slot] = e->generation;
    return engine_status(e);
}

int bd_engine_correlate(bd_engine *e, const int *slots, int nslots, double q, bd_correlation *out) {
    if (!e || !slots || !out || nslots < 1 || nslots > kMaxCorrSlots || !(q > 0.0)) return BD_ERR_ARG;
    if (!e->loaded) return BD_ERR_STATE;
    SlotList sl;
    sl.n = nslots;
    for (int j = 0; j < nslots; j++) {
        const int k = slots[j];
        if (k < 0 || k >= e->nslots) return BD_ERR_ARG;
        if (e->snap_gen[k] != e->generation || e->snap_ni[k] == LLONG_MIN) return BD_ERR_STATE;
        if (e->snap_ni[k] < 0 && e->ni > 0) return BD_ERR_STATE;  // the origin was re-based since
        sl.slot[j] = k;
    }
    int rc = ensure_segments(e);
    if (rc) return rc;
    if ((rc = ensure_scratch(e->corr_part, e->corr_part_cap, (size_t)e->nsegs * nslots * kCorrFields))) return rc;
    if ((rc = ensure_scratch(e->corr_out, e->corr_out_cap, (size_t)e->R * nslots * kCorrFields))) return rc;
    if ((rc = sync_dsp(e))) return rc;
    k_corr_partial<<<e->nsegs, kCorrThreads, 0, e->stream>>>(e->d_segs, e->d_sys, e->gid_of, e->dsp[0], e->dsp[1],
                                                             e->dsp[2], e->snaps, e->P, sl, q, e->corr_part);
    BD_LAUNCH_CHECK();
    const int nt = (nslots * kCorrFields + 31) / 32 * 32;
    k_corr_finish<<<e->R, nt, 0, e->stream>>>(e->d_seg_first, e->corr_part, nslots, e->R, e->corr_out);
    BD_LAUNCH_CHECK();
    std::vector<double> h((size_t)e->R * nslots * kCorrFields);
    BD_CUDA_TRY(cudaMemcpyAsync(h.data(), e->corr_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, e->stream));
    if ((rc = engine_status(e))) return rc;
    for (int j = 0; j < nslots; j++) {
        for (int r = 0; r < e->R; r++) {
            const SysDev &S = e->sysh[r];
            const double *v = h.data() + ((size_t)j * e->R + r) * kCorrFields;
            const int nb = S.n_big, ns = S.n - S.n_big;
            bd_correlation &c = out[(size_t)j * e->R + r];
            c.lag_steps = e->ni - e->snap_ni[slots[j]];
            c.msd_big = nb ? v[0] / nb : 0.0;
            c.r4_big = nb ? v[1] / nb : 0.0;
            c.fself_big = nb ? v[2] / nb : 0.0;
            c.msd_sml = ns ? v[3] / ns : 0.0;
            c.r4_sml = ns ? v[4] / ns : 0.0;
            c.fself_sml = ns ? v[5] / ns : 0.0;
        }
    }
    return BD_OK;
}

int bd_engine_get_displacements(bd_engine *e, double *dsp_host) {
    if (!e || !dsp_host) return BD_ERR_ARG;
    if (!e->loaded) return BD_ERR_STATE;
    const size_t n = 3 * (size_t)e->P;
    double *d = nullptr;
    BD_CUDA_TRY(cudaMalloc(&d, sizeof(double) * n));
    if (int rc = sync_dsp(e)) return rc;
    k_export_dsp<<<div_up((long)e->P, 256), 256, 0, e->stream>>>(e->gid_of, e->dsp[0], e->dsp[1], e->dsp[2],
                                                                 (int)e->P, d);
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(dsp_host, d, sizeof(double) * n, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    cudaFree(d);
    if (ce != cudaSuccess) return BD_ERR_CUDA;
    return engine_status(e);
}

}  // extern "C"
