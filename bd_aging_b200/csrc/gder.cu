// gder.cu -- cell-bounded g(r) counts of the batched replica engine.
//
// get_gder_dev (get_gder.cu:69-127) tests every ordered pair (i, j) of two
// species against `range` with the minimum-image distance (r_i - r_j) and
// adds one count to bin (int)(dist / bin_size).  That is O(N^2) per sample;
// only pairs closer than `range` count, so when the range covers a small part
// of the box the candidates can be bounded by the engine's own cell buckets.
//
// A CTA owns a brick of kGrBrick^3 cells (its "home" particles) and sweeps
// every cell within m = ceil(range / cell side) cells of the brick in tiles
// of kGrTileCells cells, skipping cells whose nearest point lies farther than
// `range` from the brick.  Every unordered pair is evaluated once: a
// candidate counts when its brick comes after the home brick in brick order,
// and within the home brick when its storage id is larger; the pair then adds
// one count to each of its two ordered bins (two to one bin for equal
// species).  Inside the range the minimum-image distance of (j, i) is the
// exact negation of that of (i, j), so the ordered counts are those of the
// reference.  Bins use the reference's rounding; counts go to a shared-memory
// histogram and then to 64-bit global counters, so the result is the exact
// integer histogram of the all-pairs kernel.  The candidate region
// (kGrBrick + 2m cells per axis) must not wrap onto itself, so every cell
// appears at most once.
//
// Pair loop: a warp holds 32 home particles in registers and walks a quarter
// of the staged candidates, all lanes reading the same candidate (a
// shared-memory broadcast).  A candidate cell that the region reaches across
// a face of the box carries the periodic shift s = L k (k = -1, 0, 1 per
// axis) of its image next to the brick, and the difference is taken as
// (x_i - x_j) - s, both roundings the reference's minimum image makes
// (d - L floor(d / L + 1/2), get_gder.cu:113-115) when its floor equals k.
// For a pair within range that is always the case: a separation below the
// range is below L / 2, so the region's image of the cell is the minimum
// image; and a pair whose minimum image lies within range has its cell in
// the region at that image.  Pairs out of range are not counted either way.
//
// The bound assumes every particle lies in its cell to within
// kGrTol * cell side.  The engine's wrap keeps positions in [0, L], but a
// blown-up state can leave a coordinate outside the box by the rounding of
// x - L floor(x / L); each home particle checks its cell, and a replica with
// a misplaced particle is flagged and recounted by the all-pairs kernel.
#include "engine_state.cuh"

namespace bd {

constexpr int kGrBrick = 4;
constexpr int kGrThreads = 256;
constexpr int kGrTileCells = 96;
constexpr int kGrMaxCap = 24;
constexpr int kGrHomeMax = kGrBrick * kGrBrick * kGrBrick * kGrMaxCap;
constexpr int kGrTileMax = kGrTileCells * kGrMaxCap;
constexpr int kGrQuarters = 4;  // candidate slices per warp task
constexpr double kGrTol = 1e-3;  // allowed stick-out of a particle from its cell, in cell sides

struct GrArgs {
    const SysDev *sys;
    const int *cnt;
    const float4 *pos;
    const int4 *bricks;  // (replica, ox, oy, oz)
    int cap;
    int nbins;
    float range;
    const float *thr;            // [nbins + 2] bin thresholds (gr_bin_thr)
    unsigned long long *counts;  // [R][4][nbins]
    const int *m_of;             // stencil reach in cells, per replica
    int *misplaced;              // per replica: a particle lies outside its cell
    unsigned *status;
};

// Exclusive scan of a[0..n) in place (n <= 4 * kGrThreads); returns the total.
__device__ int gr_scan(int *a, int n, int *wsum) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    int v[4], s = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int i = 4 * t + k;
        v[k] = i < n ? a[i] : 0;
        s += v[k];
    }
    int incl = s;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int nw = kGrThreads / 32;
        int w = lane < nw ? wsum[lane] : 0, wi = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wi, off);
            if (lane >= off) wi += y;
        }
        if (lane < nw) wsum[lane] = wi - w;
        if (lane == nw - 1) wsum[nw] = wi;
    }
    __syncthreads();
    int base = wsum[warp] + incl - s;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int i = 4 * t + k;
        if (i < n) a[i] = base;
        base += v[k];
    }
    const int total = wsum[kGrThreads / 32];
    __syncthreads();
    return total;
}

// last index c in [0, n) with start[c] <= t
// one unordered pair (i, j), j at periodic shift s of its stored position:
// both ordered counts when the pair is within range (range2_hi = the
// smallest squared distance at or beyond the range, thr[nbins + 1])
__device__ __forceinline__ void gr_count_shifted(float4 pi, float4 pj, float4 s, float range2_hi, const float *thr,
                                                 float inv_bin_size, int nbins, unsigned *hist) {
    const float dx = __fsub_rn(__fsub_rn(pi.x, pj.x), s.x);
    const float dy = __fsub_rn(__fsub_rn(pi.y, pj.y), s.y);
    const float dz = __fsub_rn(__fsub_rn(pi.z, pj.z), s.z);
    const float d2 = dist2_rn(dx, dy, dz);
    if (!(d2 < range2_hi)) return;
    int b = (int)fmaxf(0.f, __fmul_rn(__fmul_rn(d2, rsqrtf(d2)), inv_bin_size));
    b = min(b, nbins);
    if (b < nbins && d2 >= thr[b + 1]) b++;
    else if (b > 0 && d2 < thr[b]) b--;
    const int bin = min(b, nbins - 1);
    // species pair bb 0, bs 1, ss 2: an equal-species pair adds its two
    // ordered counts to one bin; a mixed pair one count to bs and one to sb
    // at the same bin, so bs and sb are one histogram (copied at the end)
    const unsigned ti = __float_as_uint(pi.w) >> 31, tj = __float_as_uint(pj.w) >> 31;
    atomicAdd(&hist[(ti + tj) * nbins + bin], ti == tj ? 2u : 1u);
}

__device__ __forceinline__ int gr_find(const int *start, int n, int t);

// Warp tasks over (32 home particles) x (a quarter of the candidates
// cand[0, nc)): the lanes keep their home particle in registers and read
// each candidate together.  HOME: the candidates are the home particles
// themselves and a pair counts once (smaller storage id first); otherwise
// the candidates of tile cell k are cand[start[k], start[k + 1]) and carry
// the cell's periodic shift cshift[k] (the cell index advances with the
// candidate index, the same in every lane).
template <bool HOME>
__device__ __forceinline__ void gr_warp_tasks(const float4 *home, int H, const float4 *cand, const int *start,
                                              const float4 *cshift, int ncells, int nc, float range2_hi,
                                              const float *thr, float inv_bin_size, int nbins, unsigned *hist) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int groups = (H + 31) >> 5;
    const int per = (nc + kGrQuarters - 1) / kGrQuarters;
    for (int task = warp; task < groups * kGrQuarters; task += nwarps) {
        const int g = task / kGrQuarters, q = task % kGrQuarters;
        const int h = (g << 5) + lane;
        const bool live = h < H;
        const float4 pi = home[live ? h : 0];
        const unsigned si = __float_as_uint(pi.w) & 0x7fffffffu;
        const int c0 = q * per, c1 = min(nc, (q + 1) * per);
        if (c0 >= c1) continue;
        int cell = 0, cend = nc;
        float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!HOME) {
            cell = gr_find(start, ncells, c0);
            cend = start[cell + 1];
            s = cshift[cell];
        }
        for (int c = c0; c < c1; c++) {
            if (!HOME && c >= cend) {  // next non-empty cell (uniform over the warp)
                do { cell++; cend = start[cell + 1]; } while (c >= cend);
                s = cshift[cell];
            }
            const float4 pj = cand[c];
            if (HOME) {
                if (live && si < (__float_as_uint(pj.w) & 0x7fffffffu))
                    gr_count_shifted(pi, pj, s, range2_hi, thr, inv_bin_size, nbins, hist);
            } else if (live) {
                gr_count_shifted(pi, pj, s, range2_hi, thr, inv_bin_size, nbins, hist);
            }
        }
    }
}

__device__ __forceinline__ int gr_find(const int *start, int n, int t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kGrThreads) k_gr_cells(GrArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    float4 *home = reinterpret_cast<float4 *>(smem);
    float4 *tile = home + kGrHomeMax;
    int *cstart = reinterpret_cast<int *>(tile + kGrTileMax);  // [kGrTileCells + 1]
    int *cgc = cstart + kGrTileCells + 1;                       // [kGrTileCells]
    __shared__ float4 cshift[kGrTileCells];                     // periodic shift of each tile cell
    int *wsum = cgc + kGrTileCells;                             // [kGrThreads / 32 + 1]
    unsigned *hist = reinterpret_cast<unsigned *>(wsum + kGrThreads / 32 + 4);  // [4][nbins]
    float *thr = reinterpret_cast<float *>(hist + 3 * a.nbins);                   // [nbins + 2]
    const int tid = threadIdx.x;
    const int4 br = a.bricks[blockIdx.x];
    const SysDev &S = a.sys[br.x];
    const int nc = S.ncell, m = a.m_of[br.x];
    const int ox = br.y, oy = br.z, oz = br.w;
    const int wx = min(kGrBrick, nc - ox), wy = min(kGrBrick, nc - oy), wz = min(kGrBrick, nc - oz);
    const int nbins = a.nbins;
    const float side = S.L;
    const float range = a.range;
    const float inv_bin_size = 1.0f / __fdiv_rn(range, (float)nbins);  // estimate only (gr_bin_thr)
    // cells whose nearest point is farther than range: gap g (cells) with
    // g cs - 4 tol > range (cell units, with margin)
    const float cs = side / (float)nc;
    const float tol = (float)kGrTol * cs;
    const float lim = (range / cs) * 1.00001f + 4.0f * (float)kGrTol;
    const float lim2 = lim * lim;
    for (int b = tid; b < 3 * nbins; b += kGrThreads) hist[b] = 0;
    for (int b = tid; b < nbins + 2; b += kGrThreads) thr[b] = a.thr[b];

    // 1. home particles of the brick
    const int nhc = wx * wy * wz;
    for (int c = tid; c < nhc; c += kGrThreads) {
        const int gx = ox + c % wx, gy = oy + (c / wx) % wy, gz = oz + c / (wx * wy);
        const int gc = S.cell_base + gx + nc * (gy + nc * gz);
        int k = a.cnt[gc];
        if (k > a.cap) { set_status(a.status, kStatCellOverflow); k = a.cap; }
        cstart[c] = max(k, 0);
        cgc[c] = gc;
    }
    __syncthreads();
    const int H = gr_scan(cstart, nhc, wsum);
    if (tid == 0) cstart[nhc] = H;
    __syncthreads();
    bool bad = false;
    for (int t = tid; t < H; t += kGrThreads) {
        const int c = gr_find(cstart, nhc, t);
        const float4 v = a.pos[(size_t)cgc[c] * a.cap + (t - cstart[c])];
        home[t] = v;
        const int lx = c % wx, ly = (c / wx) % wy, lz = c / (wx * wy);
        const float x0 = (float)(ox + lx) * cs, y0 = (float)(oy + ly) * cs, z0 = (float)(oz + lz) * cs;
        bad |= !(v.x >= x0 - tol && v.x <= x0 + cs + tol && v.y >= y0 - tol && v.y <= y0 + cs + tol &&
                 v.z >= z0 - tol && v.z <= z0 + cs + tol);
    }
    if (__syncthreads_or(bad)) {
        if (tid == 0) a.misplaced[br.x] = 1;
        return;
    }

    const float range2_hi = thr[nbins + 1];  // thr was filled before the home staging barriers
    if (H > 0) {
        // 2. pairs inside the home brick, each once (smaller storage id
        // first); the brick does not wrap, so no shift
        gr_warp_tasks<true>(home, H, home, nullptr, nullptr, 0, H, range2_hi, thr, inv_bin_size, nbins, hist);
        // 3. candidate region, tile by tile: only cells of bricks after the
        // home brick (brick order of the grid this kernel tiles with)
        const int nbr = (nc + kGrBrick - 1) / kGrBrick;
        const int hb = ox / kGrBrick + nbr * (oy / kGrBrick + nbr * (oz / kGrBrick));
        const int rx = wx + 2 * m, ry = wy + 2 * m, rz = wz + 2 * m;
        const int nreg = rx * ry * rz;
        for (int c0 = 0; c0 < nreg; c0 += kGrTileCells) {
            const int ntc = min(kGrTileCells, nreg - c0);
            for (int q = tid; q < ntc; q += kGrThreads) {
                const int qq = c0 + q;
                const int lx = qq % rx, ly = (qq / rx) % ry, lz = qq / (rx * ry);
                // cell distance to the brick along each axis, minus one
                const int kx = max(0, max(m - lx, lx - (m + wx - 1)) - 1);
                const int ky = max(0, max(m - ly, ly - (m + wy - 1)) - 1);
                const int kz = max(0, max(m - lz, lz - (m + wz - 1)) - 1);
                int k = 0, gc = 0;
                if ((float)(kx * kx + ky * ky + kz * kz) <= lim2) {
                    int gx = ox - m + lx, gy = oy - m + ly, gz = oz - m + lz;
                    // a cell reached across a face: its image next to the
                    // brick is the stored position minus L (k = -1) or plus L
                    const float sx = gx < 0 ? -side : (gx >= nc ? side : 0.f);
                    const float sy = gy < 0 ? -side : (gy >= nc ? side : 0.f);
                    const float sz = gz < 0 ? -side : (gz >= nc ? side : 0.f);
                    cshift[q] = make_float4(sx, sy, sz, 0.f);
                    gx += gx < 0 ? nc : 0; gx -= gx >= nc ? nc : 0;
                    gy += gy < 0 ? nc : 0; gy -= gy >= nc ? nc : 0;
                    gz += gz < 0 ? nc : 0; gz -= gz >= nc ? nc : 0;
                    gc = S.cell_base + gx + nc * (gy + nc * gz);
                    const int cb = gx / kGrBrick + nbr * (gy / kGrBrick + nbr * (gz / kGrBrick));
                    if (cb > hb) k = min(max(a.cnt[gc], 0), a.cap);
                }
                cstart[q] = k;
                cgc[q] = gc;
            }
            __syncthreads();
            const int Tn = gr_scan(cstart, ntc, wsum);
            if (tid == 0) cstart[ntc] = Tn;
            __syncthreads();
            for (int t = tid; t < Tn; t += kGrThreads) {
                const int c = gr_find(cstart, ntc, t);
                tile[t] = a.pos[(size_t)cgc[c] * a.cap + (t - cstart[c])];
            }
            __syncthreads();
            // pairs (home h, candidate c) of different bricks
            gr_warp_tasks<false>(home, H, tile, cstart, cshift, ntc, Tn, range2_hi, thr, inv_bin_size, nbins, hist);
            __syncthreads();
        }
    }
    __syncthreads();
    unsigned long long *out = a.counts + (size_t)br.x * 4 * nbins;  // bb, bs, sb, ss
    for (int b = tid; b < 3 * nbins; b += kGrThreads) {
        const unsigned v = hist[b];
        if (!v) continue;
        atomicAdd(&out[b < 2 * nbins ? b : b + nbins], (unsigned long long)v);  // bb, bs / ss
        if (b >= nbins && b < 2 * nbins) atomicAdd(&out[b + nbins], (unsigned long long)v);  // sb = bs
    }
}

// Stencil reach of replica r for `range`, or -1 when the candidate region
// would wrap onto itself (the all-pairs kernel handles that replica).
int gder_cell_reach(const SysDev &S, float range) {
    const double cs = (double)S.L / S.ncell;
    // a pair closer than range can sit m cells apart when both particles
    // stick out of their cells by the tolerance
    const int m = (int)std::ceil(((double)range * (1.0 + 1e-5) + 2.0 * kGrTol * cs) / (cs * (1.0 - 1e-5)));
    if (kGrBrick + 2 * m > S.ncell) return -1;
    return m;
}

size_t gder_cells_smem(int nbins) {
    return sizeof(float4) * (kGrHomeMax + kGrTileMax) + sizeof(int) * (2 * kGrTileCells + 1 + kGrThreads / 32 + 4) +
           sizeof(unsigned) * 3 * (size_t)nbins + sizeof(float) * (nbins + 2);
}

// Counts of the replicas with m_of[r] >= 0 into d_counts.  A replica whose
// particles are not all inside their cells gets m_of[r] = -1 and zero counts
// (the caller recounts it with all pairs).
int launch_gder_cells(bd_engine *e, std::vector<int> &m_of, int nbins, float range, const float *d_thr,
                      unsigned long long *d_counts) {
    std::vector<int4> bricks;
    for (int r = 0; r < e->R; r++) {
        if (m_of[r] < 0) continue;
        const int nc = e->sysh[r].ncell;
        for (int z = 0; z < nc; z += kGrBrick)
            for (int y = 0; y < nc; y += kGrBrick)
                for (int x = 0; x < nc; x += kGrBrick) bricks.push_back(make_int4(r, x, y, z));
    }
    if (bricks.empty()) return BD_OK;
    if (e->cap > kGrMaxCap) return BD_ERR_ARG;
    int4 *d_bricks = nullptr;
    int *d_m = nullptr, *d_bad = nullptr;
    BD_CUDA_TRY(cudaMalloc(&d_bricks, sizeof(int4) * bricks.size()));
    cudaError_t ce = cudaMalloc(&d_m, sizeof(int) * 2 * e->R);
    if (ce == cudaSuccess) {
        d_bad = d_m + e->R;
        ce = cudaMemsetAsync(d_bad, 0, sizeof(int) * e->R, e->stream);
    }
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(d_bricks, bricks.data(), sizeof(int4) * bricks.size(), cudaMemcpyHostToDevice, e->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(d_m, m_of.data(), sizeof(int) * e->R, cudaMemcpyHostToDevice, e->stream);
    const size_t sm = gder_cells_smem(nbins);
    if (ce == cudaSuccess) ce = cudaFuncSetAttribute(k_gr_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (ce == cudaSuccess) {
        GrArgs a;
        a.sys = e->d_sys;
        a.cnt = e->cnt[obs_buf(e)];
        a.pos = e->pos[obs_buf(e)];
        a.bricks = d_bricks;
        a.cap = e->cap;
        a.nbins = nbins;
        a.range = range;
        a.thr = d_thr;
        a.counts = d_counts;
        a.m_of = d_m;
        a.misplaced = d_bad;
        a.status = e->status;
        k_gr_cells<<<(unsigned)bricks.size(), kGrThreads, sm, e->stream>>>(a);
        ce = cudaGetLastError();
    }
    std::vector<int> bad(e->R, 0);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(bad.data(), d_bad, sizeof(int) * e->R, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    const size_t per = (size_t)4 * nbins;
    for (int r = 0; r < e->R && ce == cudaSuccess; r++) {
        if (!bad[r]) continue;
        m_of[r] = -1;
        ce = cudaMemsetAsync(d_counts + per * r, 0, sizeof(unsigned long long) * per, e->stream);
    }
    cudaFree(d_bricks);
    if (d_m) cudaFree(d_m);
    return ce == cudaSuccess ? BD_OK : BD_ERR_CUDA;
}

}  // namespace bd
