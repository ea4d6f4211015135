// mirror.cu -- the reference's entry points (encabezados.h:86-158) as sm_100a
// kernels behind the C ABI of include/bd_aging.h.  Same argument meaning and
// float3 array-of-structs layout as the reference; status codes instead of
// exit(); explicit streams; no write ever leaves its buffer.
#include <cuda.h>
#include <curand_kernel.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "runtime.cuh"

namespace bd {

// ------------------------------------------------------------ workspace
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (GetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (GetId)f;
    });
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    if (get_current(&c) != CUDA_SUCCESS || !c) {
        int dev = 0;  // no context yet on this thread: make the device's primary context current
        if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess) return 0;
        if (get_current(&c) != CUDA_SUCCESS || !c) return 0;
    }
    unsigned long long id = 0;
    return get_id(c, &id) == CUDA_SUCCESS ? id + 1 : 0;  // +1: a valid id is never 0 here
}

DeviceWork *device_work() {
    static std::mutex mu;
    static DeviceWork works[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    const unsigned long long ctx = current_context_id();
    if (!ctx) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    DeviceWork &w = works[dev];
    if (w.ctx != ctx) {  // first use, or the context was destroyed (its memory with it)
        w = DeviceWork{};
        if (cudaMalloc(&w.status, 256) != cudaSuccess) return nullptr;
        if (cudaMalloc(&w.accum, kWorkAccum * sizeof(double)) != cudaSuccess) return nullptr;
        if (cudaMemset(w.status, 0, 256) != cudaSuccess) return nullptr;
        w.ctx = ctx;
    }
    return &w;
}

// Reset the status word, run nothing else; read it back after the kernels.
static int read_status(DeviceWork *w, cudaStream_t s) {
    unsigned bits = 0;
    BD_CUDA_TRY(cudaMemcpyAsync(&bits, w->status, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    BD_CUDA_TRY(cudaStreamSynchronize(s));
    return status_from_bits(bits);
}

// ------------------------------------------------------------ cell list
// cell_locate_dev (cell_locate.cu:155-209): cell (int)(cell_side_inv * x)
// with the inverse side a double division narrowed to float, ==ncell clamp,
// linear index i + n(j + n k), slot by atomic increment of nocup.
__global__ void k_cell_bin(const float *__restrict__ rr, int n, float csi, int ncell, int ntags, int *nocup,
                           int *cell_vec, unsigned *st) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    float x = rr[3 * m], y = rr[3 * m + 1], z = rr[3 * m + 2];
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) set_status(st, kStatNumeric);
    int ii = (int)__fmul_rn(csi, x), jj = (int)__fmul_rn(csi, y), kk = (int)__fmul_rn(csi, z);
    if (ii == ncell) ii--;
    if (jj == ncell) jj--;
    if (kk == ncell) kk--;
    if ((unsigned)ii >= (unsigned)ncell || (unsigned)jj >= (unsigned)ncell || (unsigned)kk >= (unsigned)ncell) {
        // outside the box: the reference would write out of bounds here
        set_status(st, kStatArg);
        ii = min(max(ii, 0), ncell - 1);
        jj = min(max(jj, 0), ncell - 1);
        kk = min(max(kk, 0), ncell - 1);
    }
    int c = ii + ncell * (jj + ncell * kk);
    int s = atomicAdd(&nocup[c], 1);
    if (s < ntags) cell_vec[(long)c * ntags + s] = m;
    if (s + 1 >= ntags) set_status(st, kStatCellOverflow);  // main.cu:655 (nocup_max >= ntags)
}
// Slots in ascending particle order (the order cell_locate_hst produces).
__global__ void k_cell_sort(const int *nocup, int *cell_vec, int nc3, int ntags) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc3) return;
    int k = min(nocup[c], ntags);
    int *v = cell_vec + (long)c * ntags;
    for (int a = 1; a < k; a++) {
        int key = v[a], b = a - 1;
        while (b >= 0 && v[b] > key) { v[b + 1] = v[b]; b--; }
        v[b + 1] = key;
    }
}

// ------------------------------------------------------------ forces
// get_forces_same_dev / get_forces_diff_dev (get_forces.cu:297-558): one
// thread per particle over the (2 nrange + 1)^3 cells around its own cell of
// the partner species; pair selection with the reference's rounding
// (min_image_f, dist2_rn), WCA-modified pair; results ADDED to ff/vir/pot.
template <bool SAME>
__global__ void k_forces(const float *__restrict__ rr, float *ff, float *vir, float *pot,
                         const float *__restrict__ rr_o, const int *__restrict__ nocup,
                         const int *__restrict__ cell_vec, int n, int ncell, int ntags, int nrange, float csi,
                         float sigma, float side, unsigned *st) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    const float side_inv = __fdiv_rn(1.0f, side);
    const float cut2 = __fmul_rn(sigma, sigma);
    float rx = rr[3 * m], ry = rr[3 * m + 1], rz = rr[3 * m + 2];
    int ii = (int)__fmul_rn(csi, rx), jj = (int)__fmul_rn(csi, ry), kk = (int)__fmul_rn(csi, rz);
    if (ii == ncell) ii--;
    if (jj == ncell) jj--;
    if (kk == ncell) kk--;
    if ((unsigned)ii >= (unsigned)ncell || (unsigned)jj >= (unsigned)ncell || (unsigned)kk >= (unsigned)ncell) {
        set_status(st, kStatArg);
        ii = min(max(ii, 0), ncell - 1);
        jj = min(max(jj, 0), ncell - 1);
        kk = min(max(kk, 0), ncell - 1);
    }
    float fx = ff[3 * m], fy = ff[3 * m + 1], fz = ff[3 * m + 2], v = vir[m], p = pot[m];
    for (int di = -nrange; di <= nrange; di++)
        for (int dj = -nrange; dj <= nrange; dj++)
            for (int dk = -nrange; dk <= nrange; dk++) {
                int ip = (ii + di + ncell) % ncell, jp = (jj + dj + ncell) % ncell, kp = (kk + dk + ncell) % ncell;
                int c = ip + ncell * (jp + ncell * kp);
                int occ = min(nocup[c], ntags);
                const int *cv = cell_vec + (long)c * ntags;
                for (int t = 0; t < occ; t++) {
                    int nn = cv[t];
                    if (SAME && nn == m) continue;
                    float dx = min_image_f(__fsub_rn(rr_o[3 * nn], rx), side, side_inv);
                    float dy = min_image_f(__fsub_rn(rr_o[3 * nn + 1], ry), side, side_inv);
                    float dz = min_image_f(__fsub_rn(rr_o[3 * nn + 2], rz), side, side_inv);
                    float d2 = dist2_rn(dx, dy, dz);
                    if (d2 < cut2) {
                        PairOut o = wca_modified_pair(sigma, d2, dx, dy, dz);
                        fx += o.fx;
                        fy += o.fy;
                        fz += o.fz;
                        p += o.pot;
                        v += o.vir;
                    }
                }
            }
    ff[3 * m] = fx;
    ff[3 * m + 1] = fy;
    ff[3 * m + 2] = fz;
    vir[m] = v;
    pot[m] = p;
}

// ------------------------------------------------------------ update
__global__ void k_setup_rng(curandState *states, unsigned long long seed, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) curand_init(seed, i, 0, &states[i]);
}
// update_ermak_dev (update_ermak.cu:91-160) with the reference's cuRAND
// stream; the expression is the reference's, so the compiler treats it alike.
__global__ void k_update_curand(float *rr, float *raw, const float *__restrict__ ff, curandState *states, int n,
                                float side, float side_inv, float dinv, float dt, float amplitude) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    curandState s = states[m];
    float rx = amplitude * curand_normal(&s);
    float ry = amplitude * curand_normal(&s);
    float rz = amplitude * curand_normal(&s);
    states[m] = s;
    float tx = ff[3 * m] * dinv * dt + rx;
    float ty = ff[3 * m + 1] * dinv * dt + ry;
    float tz = ff[3 * m + 2] * dinv * dt + rz;
    float x = rr[3 * m] + tx, y = rr[3 * m + 1] + ty, z = rr[3 * m + 2] + tz;
    raw[3 * m] += tx;
    raw[3 * m + 1] += ty;
    raw[3 * m + 2] += tz;
    x -= side * floorf(side_inv * x);
    y -= side * floorf(side_inv * y);
    z -= side * floorf(side_inv * z);
    rr[3 * m] = x;
    rr[3 * m + 1] = y;
    rr[3 * m + 2] = z;
}
// update_ermak_hst (update_ermak.cu:8-77) with injected N(0,1) values, every
// operation rounded separately as on the host: bit-identical to it.
__global__ void k_update_noise(float *rr, float *raw, const float *__restrict__ ff, const float *__restrict__ noise,
                               int n, float side, float side_inv, float dinv, float dt, float amplitude) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float rnd = __fmul_rn(amplitude, noise[3 * m + k]);
        float tot = __fadd_rn(__fmul_rn(__fmul_rn(ff[3 * m + k], dinv), dt), rnd);
        float x = __fadd_rn(rr[3 * m + k], tot);
        raw[3 * m + k] = __fadd_rn(raw[3 * m + k], tot);
        rr[3 * m + k] = __fsub_rn(x, __fmul_rn(side, floorf(__fmul_rn(side_inv, x))));
    }
}

// ------------------------------------------------------------ g(r)
// get_gder_dev (get_gder.cu:69-127) as an exact integer histogram.  Each
// thread owns one particle of `ra`; the partner set is staged through shared
// memory in tiles; bins are added per warp with one shared atomic per
// distinct bin (__match_any_sync) into a block histogram that is flushed to
// 64-bit global counters.  SAME: unordered pairs j > i, each counted in both
// directions; the reverse distance is recomputed whenever the minimum-image
// rounding can differ between directions (some |d/L| >= 1/4).
constexpr int kGderTile = 1024;
__device__ __forceinline__ int gder_bin(float dx, float dy, float dz, float side, float side_inv, float range,
                                        float range2_hi, float bin_size, int nbins) {
    dx = min_image_gder(dx, side, side_inv);
    dy = min_image_gder(dy, side, side_inv);
    dz = min_image_gder(dz, side, side_inv);
    float d2 = dist2_rn(dx, dy, dz);
    if (!(d2 <= range2_hi)) return -1;
    float dist = __fsqrt_rn(d2);
    if (!(dist < range)) return -1;
    int bin = (int)__fdiv_rn(dist, bin_size);
    if (bin == nbins) bin--;
    return bin;
}
__device__ __forceinline__ void hist_add(unsigned *hist, int bin, unsigned lane_mask_all) {
    unsigned same = __match_any_sync(lane_mask_all, bin);
    int lane = threadIdx.x & 31;
    if (bin >= 0 && lane == __ffs(same) - 1) atomicAdd(&hist[bin], (unsigned)__popc(same));
}
template <bool SAME>
__global__ void __launch_bounds__(256) k_gder(const float *__restrict__ ra, int na, const float *__restrict__ rb,
                                              int nb, float side, float side_inv, float range, float range2_hi,
                                              float bin_size, int nbins, int jchunk,
                                              unsigned long long *counts) {
    extern __shared__ unsigned char smem[];
    float *tx = reinterpret_cast<float *>(smem);
    float *ty = tx + kGderTile, *tz = ty + kGderTile;
    unsigned *hist = reinterpret_cast<unsigned *>(tz + kGderTile);
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) hist[b] = 0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool vi = i < na;
    float xi = 0, yi = 0, zi = 0;
    if (vi) { xi = ra[3 * i]; yi = ra[3 * i + 1]; zi = ra[3 * i + 2]; }
    int j0 = blockIdx.y * jchunk, j1 = min(nb, j0 + jchunk);
    if (SAME) j0 = max(j0, (int)(blockIdx.x * blockDim.x) + 1);
    __syncthreads();
    for (int t0 = j0; t0 < j1; t0 += kGderTile) {
        int tn = min(kGderTile, j1 - t0);
        __syncthreads();
        for (int t = threadIdx.x; t < tn; t += blockDim.x) {
            tx[t] = rb[3 * (t0 + t)];
            ty[t] = rb[3 * (t0 + t) + 1];
            tz[t] = rb[3 * (t0 + t) + 2];
        }
        __syncthreads();
        for (int t = 0; t < tn; t++) {
            int j = t0 + t;
            bool ok = vi && (!SAME || j > i);
            int bf = -1, br = -1;
            if (ok) {
                float dx = __fsub_rn(xi, tx[t]), dy = __fsub_rn(yi, ty[t]), dz = __fsub_rn(zi, tz[t]);
                bf = gder_bin(dx, dy, dz, side, side_inv, range, range2_hi, bin_size, nbins);
                if (SAME) {
                    bool sym = fabsf(__fmul_rn(side_inv, dx)) < 0.25f && fabsf(__fmul_rn(side_inv, dy)) < 0.25f &&
                               fabsf(__fmul_rn(side_inv, dz)) < 0.25f;
                    br = sym ? bf : gder_bin(-dx, -dy, -dz, side, side_inv, range, range2_hi, bin_size, nbins);
                }
            }
            hist_add(hist, bf, 0xffffffffu);
            if (SAME) hist_add(hist, br, 0xffffffffu);
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        if (hist[b]) atomicAdd(&counts[b], (unsigned long long)hist[b]);
}

// ------------------------------------------------------------ F_s, MSD
// fself_isotropic (fself.cu:3-21) and the MSD loop (main.cu:776-792): per
// particle float terms as in the reference, summed in FP64.
// One FP64 partial per block, then one block adds the partials in index
// order, so the result does not depend on the order in which blocks finish.
constexpr int kDispThreads = 256, kDispMaxBlocks = 148 * 8;
static_assert(kDispMaxBlocks + 1 <= kWorkAccum, "partials fit the workspace");
template <int KIND>  // 0: F_s, 1: MSD
__global__ void __launch_bounds__(kDispThreads) k_disp_reduce(const float *__restrict__ raw,
                                                              const float *__restrict__ r0, int n, float q,
                                                              double *part) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float dx = raw[3 * i] - r0[3 * i], dy = raw[3 * i + 1] - r0[3 * i + 1], dz = raw[3 * i + 2] - r0[3 * i + 2];
        float d2 = dist2_rn(dx, dy, dz);
        if (KIND == 0) {
            float mag = __fsqrt_rn(d2);
            s += (double)(sinf(q * mag) / (q * mag));
        } else {
            s += (double)d2;
        }
    }
    for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ double red[kDispThreads / 32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kDispThreads / 32; w++) t += red[w];
        part[1 + blockIdx.x] = t;
    }
}
// part[0] = sum of part[1 .. nblocks] in a fixed order
__global__ void __launch_bounds__(kDispThreads) k_disp_finish(double *part, int nblocks) {
    __shared__ double red[kDispThreads];
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += part[1 + b];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kDispThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[0] = red[0];
}

static int disp_reduce(int kind, const float *raw, const float *r0, int n, float q, double *out, cudaStream_t s) {
    DeviceWork *w = device_work();
    if (!w) return BD_ERR_NOMEM;
    const int blocks = std::min(div_up(n, kDispThreads), kDispMaxBlocks);
    if (kind == 0) k_disp_reduce<0><<<blocks, kDispThreads, 0, s>>>(raw, r0, n, q, w->accum);
    else k_disp_reduce<1><<<blocks, kDispThreads, 0, s>>>(raw, r0, n, q, w->accum);
    BD_LAUNCH_CHECK();
    k_disp_finish<<<1, kDispThreads, 0, s>>>(w->accum, blocks);
    BD_LAUNCH_CHECK();
    BD_CUDA_TRY(cudaMemcpyAsync(out, w->accum, sizeof(double), cudaMemcpyDeviceToHost, s));
    BD_CUDA_TRY(cudaStreamSynchronize(s));
    return BD_OK;
}


// ------------------------------------------------------------ colours
// calculate_color / between (colors.cu:8-110) for every big particle, one
// thread each, in the reference's float operation order (rounding
// intrinsics: no contraction).  ids: 0 blue, 1 green, 2 red.
__device__ __forceinline__ bool between_dev(const float3 r1, const float3 r2, const float3 *__restrict__ rs, int ns,
                                            float side, float side_inv, float max_big, float max_line) {
    float ux = min_image_f(__fsub_rn(r1.x, r2.x), side, side_inv);
    float uy = min_image_f(__fsub_rn(r1.y, r2.y), side, side_inv);
    float uz = min_image_f(__fsub_rn(r1.z, r2.z), side, side_inv);
    const float ua = __fsqrt_rn(dist2_rn(ux, uy, uz));
    ux = __fdiv_rn(ux, ua);
    uy = __fdiv_rn(uy, ua);
    uz = __fdiv_rn(uz, ua);
    for (int i = 0; i < ns; i++) {
        const float3 r = rs[i];
        const float ax = min_image_f(__fsub_rn(r.x, r1.x), side, side_inv);
        const float ay = min_image_f(__fsub_rn(r.y, r1.y), side, side_inv);
        const float az = min_image_f(__fsub_rn(r.z, r1.z), side, side_inv);
        if (__fsqrt_rn(dist2_rn(ax, ay, az)) > max_big) continue;
        const float bx = min_image_f(__fsub_rn(r.x, r2.x), side, side_inv);
        const float by = min_image_f(__fsub_rn(r.y, r2.y), side, side_inv);
        const float bz = min_image_f(__fsub_rn(r.z, r2.z), side, side_inv);
        if (__fsqrt_rn(dist2_rn(bx, by, bz)) > max_big) continue;
        const float cx = __fsub_rn(__fmul_rn(ay, uz), __fmul_rn(az, uy));
        const float cy = __fadd_rn(__fmul_rn(-ax, uz), __fmul_rn(az, ux));
        const float cz = __fsub_rn(__fmul_rn(ax, uy), __fmul_rn(ay, ux));
        if (__fsqrt_rn(dist2_rn(cx, cy, cz)) > max_line) continue;
        return true;
    }
    return false;
}

__global__ void k_colors(const float3 *__restrict__ rb, int nb, const float3 *__restrict__ rs, int ns, float side,
                         float sigma_big, float sigma_sml, int *ids, unsigned *counts) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nb) return;
    const float side_inv_c = __double2float_rn(1.0 / (double)side);  // calculate_color: 1.0 / side
    const float side_inv_b = __fdiv_rn(1.0f, side);                  // between: 1 / side
    const float max_big = __double2float_rn(0.5 * (double)sigma_big + 2.0 * (double)sigma_sml);
    const float max_line = __double2float_rn(0.35 * (double)sigma_big);
    const double near2 = (double)sigma_big + 2.0 * (double)sigma_sml;
    const float3 rm = rb[m];
    int cid = 0;
    bool near = false;
    for (int n = 0; n < nb; n++) {
        if (n == m) continue;
        const float3 rn = rb[n];
        const float dx = min_image_f(__fsub_rn(rn.x, rm.x), side, side_inv_c);
        const float dy = min_image_f(__fsub_rn(rn.y, rm.y), side, side_inv_c);
        const float dz = min_image_f(__fsub_rn(rn.z, rm.z), side, side_inv_c);
        if ((double)dist2_rn(dx, dy, dz) > near2) continue;  // squared distance against a length, as written
        cid += between_dev(rm, rn, rs, ns, side, side_inv_b, max_big, max_line) ? 1 : -1;
        near = true;
    }
    const int id = near ? (cid > 0 ? 2 : 1) : 0;
    if (ids) ids[m] = id;
    atomicAdd(&counts[id], 1u);
}

}  // namespace bd

using namespace bd;

// ====================================================================== ABI
extern "C" {

const char *bd_status_string(int s) {
    switch (s) {
        case BD_OK: return "ok";
        case BD_ERR_ARG: return "invalid argument";
        case BD_ERR_CUDA: return "CUDA runtime error";
        case BD_ERR_CELL_OVERFLOW: return "ntags reached limit (cell capacity exceeded)";
        case BD_ERR_NOMEM: return "out of memory";
        case BD_ERR_STATE: return "call out of order";
        case BD_ERR_TIMEOUT: return "bounded device wait expired";
        case BD_ERR_FILE: return "file missing or unreadable";
        case BD_ERR_FORMAT: return "malformed input";
        case BD_ERR_NUMERIC: return "non-finite position";
        default: return "unknown status";
    }
}
int bd_abi_version(void) { return BD_ABI_VERSION; }

// main.cu:155-163, 244-298, 348-349
int bd_setup_params(bd_parametros *p, float side, int nb, int ns, float sigma_big, float sigma_sml, float mass_big,
                    float mass_sml, int ntags_big, int ntags_sml, int nbins_gder, float range_gder, double dt,
                    float temp0) {
    if (!p || nb < 0 || ns < 0 || !(side > 0) || !(sigma_big > 0) || !(sigma_sml > 0) || nbins_gder < 1)
        return BD_ERR_ARG;
    std::memset(p, 0, sizeof(*p));
    p->dt = (float)dt;
    p->temp_set = temp0;
    p->nbins_gder = nbins_gder;
    p->range_gder = range_gder;
    p->ntags_big = ntags_big;
    p->ntags_sml = ntags_sml;
    p->bin_size_gder = range_gder / ((float)nbins_gder);
    p->side = side;
    p->ngrain_big = nb;
    p->ngrain_sml = ns;
    p->ngrain_tot = nb + ns;
    p->sigma_big = sigma_big;
    p->sigma_sml = sigma_sml;
    p->mass_big = mass_big;
    p->mass_sml = mass_sml;
    float cutoff = sigma_big;
    int ncb = (int)(side / (1.05 * cutoff));
    p->ncell_big = ncb;
    p->cell_side_big = side / ((float)ncb);
    cutoff = sigma_sml;
    int ncs = (int)(side / (1.05 * cutoff));
    p->ncell_sml = ncs;
    p->cell_side_sml = side / ((float)ncs);
    p->nrange_bb = 1;
    float aux = (float)((sigma_big + sigma_sml) / 2.0);
    p->nrange_bs = 1 + (int)(aux / p->cell_side_sml);
    p->nrange_sb = 1;
    p->nrange_ss = 1;
    p->NH = 256;
    return (ncb < 1 || ncs < 1) ? BD_ERR_ARG : BD_OK;
}

int bd_cell_locate(char type, const float *rr, int *nocup, int *cell_vec, const bd_parametros *p, void *stream) {
    if (!p || (type != 'b' && type != 's') || !nocup || !cell_vec) return BD_ERR_ARG;
    const bool b = type == 'b';
    const int n = b ? p->ngrain_big : p->ngrain_sml, ncell = b ? p->ncell_big : p->ncell_sml;
    const int ntags = b ? p->ntags_big : p->ntags_sml;
    if (ncell < 1 || ntags < 1 || n < 0 || (n > 0 && !rr)) return BD_ERR_ARG;
    const float csi = (float)(1.0 / (b ? p->cell_side_big : p->cell_side_sml));
    const int nc3 = ncell * ncell * ncell;
    cudaStream_t s = as_stream(stream);
    DeviceWork *w = device_work();
    if (!w) return BD_ERR_NOMEM;
    BD_CUDA_TRY(cudaMemsetAsync(w->status, 0, sizeof(unsigned), s));
    BD_CUDA_TRY(cudaMemsetAsync(nocup, 0, sizeof(int) * (size_t)nc3, s));
    BD_CUDA_TRY(cudaMemsetAsync(cell_vec, 0xff, sizeof(int) * (size_t)nc3 * ntags, s));
    if (n > 0) {
        k_cell_bin<<<div_up(n, 256), 256, 0, s>>>(rr, n, csi, ncell, ntags, nocup, cell_vec, w->status);
        BD_LAUNCH_CHECK();
    }
    k_cell_sort<<<div_up(nc3, 256), 256, 0, s>>>(nocup, cell_vec, nc3, ntags);
    BD_LAUNCH_CHECK();
    return read_status(w, s);
}

int bd_get_forces_same(char type, const float *rr, float *ff, float *vir, float *pot, const int *nocup,
                       const int *cell_vec, const bd_parametros *p, void *stream) {
    if (!p || (type != 'b' && type != 's')) return BD_ERR_ARG;
    const bool b = type == 'b';
    const int n = b ? p->ngrain_big : p->ngrain_sml;
    if (n == 0) return BD_OK;
    if (!rr || !ff || !vir || !pot || !nocup || !cell_vec) return BD_ERR_ARG;
    const float sigma = b ? p->sigma_big : p->sigma_sml;
    const float csi = 1.0f / (b ? p->cell_side_big : p->cell_side_sml);
    const int ntags = b ? p->ntags_big : p->ntags_sml, ncell = b ? p->ncell_big : p->ncell_sml;
    const int nrange = b ? p->nrange_bb : p->nrange_ss;
    cudaStream_t s = as_stream(stream);
    DeviceWork *w = device_work();
    if (!w) return BD_ERR_NOMEM;
    BD_CUDA_TRY(cudaMemsetAsync(w->status, 0, sizeof(unsigned), s));
    k_forces<true><<<div_up(n, 128), 128, 0, s>>>(rr, ff, vir, pot, rr, nocup, cell_vec, n, ncell, ntags, nrange,
                                                   csi, sigma, p->side, w->status);
    BD_LAUNCH_CHECK();
    return read_status(w, s);
}

int bd_get_forces_diff(char type, char type_other, const float *rr, float *ff, const float *rr_other, float *vir,
                       float *pot, const int *nocup_o, const int *cell_o, const bd_parametros *p, void *stream) {
    if (!p || (type != 'b' && type != 's') || (type_other != 'b' && type_other != 's') || type == type_other)
        return BD_ERR_ARG;
    const bool b = type == 'b';
    const int n = b ? p->ngrain_big : p->ngrain_sml;
    if (n == 0) return BD_OK;
    if (!rr || !ff || !vir || !pot || !nocup_o || !cell_o || !rr_other) return BD_ERR_ARG;
    const float csi = 1.0f / (b ? p->cell_side_sml : p->cell_side_big);
    const float sigma = b ? 0.5f * (p->sigma_big + p->sigma_sml) : 0.5f * (p->sigma_sml + p->sigma_big);
    const int ntags = b ? p->ntags_sml : p->ntags_big, ncell = b ? p->ncell_sml : p->ncell_big;
    const int nrange = b ? p->nrange_bs : p->nrange_sb;
    cudaStream_t s = as_stream(stream);
    DeviceWork *w = device_work();
    if (!w) return BD_ERR_NOMEM;
    BD_CUDA_TRY(cudaMemsetAsync(w->status, 0, sizeof(unsigned), s));
    k_forces<false><<<div_up(n, 128), 128, 0, s>>>(rr, ff, vir, pot, rr_other, nocup_o, cell_o, n, ncell, ntags,
                                                    nrange, csi, sigma, p->side, w->status);
    BD_LAUNCH_CHECK();
    return read_status(w, s);
}

size_t bd_rng_state_size(void) { return sizeof(curandState); }

int bd_setup_rng(void *states, unsigned long long seed, int n, void *stream) {
    if (n < 0 || (n > 0 && !states)) return BD_ERR_ARG;
    if (n == 0) return BD_OK;
    k_setup_rng<<<div_up(n, 256), 256, 0, as_stream(stream)>>>((curandState *)states, seed, n);
    BD_LAUNCH_CHECK();
    return BD_OK;
}

static int update_common(char type, const bd_parametros *p, int &n, float &side_inv, float &dinv, float &amp) {
    if (!p || (type != 'b' && type != 's')) return BD_ERR_ARG;
    n = type == 'b' ? p->ngrain_big : p->ngrain_sml;
    float diameter = type == 'b' ? p->sigma_big : p->sigma_sml;
    side_inv = 1.0f / p->side;
    dinv = 1.0f / diameter;
    amp = (float)std::sqrt(2.0 * p->temp_set * dinv * p->dt);  // update_ermak.cu:114
    return BD_OK;
}

int bd_update_ermak(char type, float *rr, float *rr_raw, const float *ff, void *states, const bd_parametros *p,
                    void *stream) {
    int n;
    float side_inv, dinv, amp;
    int rc = update_common(type, p, n, side_inv, dinv, amp);
    if (rc) return rc;
    if (n == 0) return BD_OK;
    if (!rr || !rr_raw || !ff || !states) return BD_ERR_ARG;
    k_update_curand<<<div_up(n, 256), 256, 0, as_stream(stream)>>>(rr, rr_raw, ff, (curandState *)states, n, p->side,
                                                                   side_inv, dinv, p->dt, amp);
    BD_LAUNCH_CHECK();
    return BD_OK;
}

int bd_update_ermak_noise(char type, float *rr, float *rr_raw, const float *ff, const float *noise,
                          const bd_parametros *p, void *stream) {
    int n;
    float side_inv, dinv, amp;
    int rc = update_common(type, p, n, side_inv, dinv, amp);
    if (rc) return rc;
    if (n == 0) return BD_OK;
    if (!rr || !rr_raw || !ff || !noise) return BD_ERR_ARG;
    k_update_noise<<<div_up(n, 256), 256, 0, as_stream(stream)>>>(rr, rr_raw, ff, noise, n, p->side, side_inv, dinv,
                                                                  p->dt, amp);
    BD_LAUNCH_CHECK();
    return BD_OK;
}

float bd_calculate_temp_linear(float T0, float Tf, float t0, float tf, float t) {
    return temp_linear(T0, Tf, t0, tf, t);
}
// set_temp.cu:14-23
float bd_calculate_temp_sine(float T0, float Tf, float t0, float tf, float period, float t) {
    if (t < t0) return T0;
    if (t > tf) return Tf;
    float a = (float)(0.5 * (T0 + Tf));
    float b = (float)(0.5 * (Tf - T0));
    float argument = (float)(2 * kRefPi * (t / period - 0.25));
    volatile float sn = sinf(argument);
    volatile float bs = b * sn;
    return a + bs;
}

int bd_get_gder(char type, char type_other, const float *rr, const float *rr_other, unsigned long long *counts,
                const bd_parametros *p, void *stream) {
    if (!p || (type != 'b' && type != 's') || (type_other != 'b' && type_other != 's') || !counts) return BD_ERR_ARG;
    const int na = type == 'b' ? p->ngrain_big : p->ngrain_sml;
    const int nb = type_other == 'b' ? p->ngrain_big : p->ngrain_sml;
    const int nbins = p->nbins_gder;
    if (nbins < 1 || nbins > 8192 || !(p->range_gder > 0)) return BD_ERR_ARG;
    if (na == 0 || nb == 0) return BD_OK;
    if (!rr || !rr_other) return BD_ERR_ARG;
    const float side = p->side, side_inv = (float)(1.0 / side), range = p->range_gder;
    const float bin_size = range / ((float)nbins);
    const float range2_hi = range * range * 1.00001f;
    const bool same = type == type_other;
    const int jchunk = 8192;
    dim3 grid(div_up(na, 256), div_up(nb, jchunk));
    size_t sm = 3 * kGderTile * sizeof(float) + (size_t)nbins * sizeof(unsigned);
    cudaStream_t s = as_stream(stream);
    if (same) {
        BD_CUDA_TRY(cudaFuncSetAttribute(k_gder<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_gder<true><<<grid, 256, sm, s>>>(rr, na, rr_other, nb, side, side_inv, range, range2_hi, bin_size, nbins,
                                           jchunk, counts);
    } else {
        BD_CUDA_TRY(cudaFuncSetAttribute(k_gder<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_gder<false><<<grid, 256, sm, s>>>(rr, na, rr_other, nb, side, side_inv, range, range2_hi, bin_size, nbins,
                                            jchunk, counts);
    }
    BD_LAUNCH_CHECK();
    return BD_OK;
}

// main.cu:847-877 for one sample (host arithmetic as in the reference)
int bd_gder_normalize(const double *counts, int nbins, float bin_size, float side, int nb, int ns, float sigma_big,
                      float sigma_sml, int n_configs, float *gder) {
    if (!counts || !gder || nbins < 1 || n_configs < 1) return BD_ERR_ARG;
    const float volume = side * side * side, xb = (float)nb, xs = (float)ns;
    for (int k = 0; k < nbins; k++) {
        float xnb = (float)k;
        volatile float xnb2 = xnb * xnb;
        float shell_vol = (float)(4.0 * kRefPi * bin_size * bin_size * bin_size * ((1.0 / 3.0) + xnb2 + xnb));
        float g[4];
        for (int j = 0; j < 4; j++) g[j] = (float)counts[j * nbins + k];
        float sigma = sigma_big;
        float vol_free = (float)(volume - (4.0 / 3.0) * kRefPi * sigma * sigma * sigma);
        g[0] = g[0] / shell_vol;
        g[0] = (float)(g[0] / (xb * (xb - 1.0) / vol_free));
        sigma = (float)(0.5 * (sigma_big + sigma_sml));
        vol_free = (float)(volume - (4.0 / 3.0) * kRefPi * sigma * sigma * sigma);
        g[1] = g[1] / shell_vol;
        g[2] = g[2] / shell_vol;
        volatile float pbs = xb * xs, psb = xs * xb;
        g[1] /= (pbs / vol_free);
        g[2] /= (psb / vol_free);
        sigma = sigma_sml;
        vol_free = (float)(volume - (4.0 / 3.0) * kRefPi * sigma * sigma * sigma);
        g[3] = g[3] / shell_vol;
        g[3] = (float)(g[3] / (xs * (xs - 1.0) / vol_free));
        for (int j = 0; j < 4; j++) gder[j * nbins + k] = g[j] / n_configs;
    }
    return BD_OK;
}

int bd_fself_isotropic(const float *rr_raw, const float *rr0, int ngrain, float *fself_host, int sample_number,
                       float qmax, void *stream) {
    if (ngrain <= 0 || !rr_raw || !rr0 || !fself_host || sample_number < 0) return BD_ERR_ARG;
    double sum = 0.0;
    int rc = disp_reduce(0, rr_raw, rr0, ngrain, qmax, &sum, as_stream(stream));
    if (rc) return rc;
    fself_host[sample_number] += (float)(sum / ngrain);
    return BD_OK;
}

int bd_color_statistics(const float *rr_big, const float *rr_sml, int *color_ids, int *counts_host,
                        const bd_parametros *p, void *stream) {
    if (!p || !counts_host || p->ngrain_big < 0 || p->ngrain_sml < 0) return BD_ERR_ARG;
    counts_host[0] = counts_host[1] = counts_host[2] = 0;
    const int nb = p->ngrain_big, ns = p->ngrain_sml;
    if (nb == 0) return BD_OK;
    if (!rr_big || (ns > 0 && !rr_sml)) return BD_ERR_ARG;
    cudaStream_t s = as_stream(stream);
    unsigned *d_counts = nullptr;
    BD_CUDA_TRY(cudaMalloc(&d_counts, 3 * sizeof(unsigned)));
    cudaError_t ce = cudaMemsetAsync(d_counts, 0, 3 * sizeof(unsigned), s);
    if (ce == cudaSuccess) {
        k_colors<<<div_up(nb, 128), 128, 0, s>>>(reinterpret_cast<const float3 *>(rr_big), nb,
                                                 reinterpret_cast<const float3 *>(rr_sml), ns, p->side,
                                                 p->sigma_big, p->sigma_sml, color_ids, d_counts);
        ce = cudaGetLastError();
    }
    unsigned h[3] = {0, 0, 0};
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(h, d_counts, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    cudaFree(d_counts);
    if (ce != cudaSuccess) return BD_ERR_CUDA;
    for (int k = 0; k < 3; k++) counts_host[k] = (int)h[k];
    return BD_OK;
}

int bd_msd(const float *rr_raw, const float *rr0, int ngrain, float *msd_host, void *stream) {
    if (ngrain <= 0 || !rr_raw || !rr0 || !msd_host) return BD_ERR_ARG;
    double sum = 0.0;
    int rc = disp_reduce(1, rr_raw, rr0, ngrain, 0.0f, &sum, as_stream(stream));
    if (rc) return rc;
    *msd_host = (float)(sum / ngrain);
    return BD_OK;
}

}  // extern "C"
