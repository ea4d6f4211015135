// common.cuh -- device arithmetic shared by every kernel of libbd_aging_b200.
//
// Exactness rules.  Pair selection (cut-off test), cell indices and g(r) bins
// must be bit-identical to the reference's host functions given identical
// positions.  The reference host code rounds every product and sum separately
// (no fused multiply-add on x86-64), so these helpers use the explicitly
// rounded intrinsics __fmul_rn / __fadd_rn / __fsub_rn, which the compiler
// never contracts into FMA.  The force arithmetic itself only has to agree to
// a tolerance and is written in plain C so the compiler may fuse it.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bd {

// encabezados.h:25 and :30 (PI is 3.14159266f in the reference, sic)
constexpr float kRefPi = 3.14159266f;
constexpr float kEps = 1.0f;

// device status word bits (OR-ed by kernels, read by the host after a call)
enum : unsigned {
    kStatCellOverflow = 1u,   // a cell or staging buffer exceeded its capacity
    kStatNumeric = 2u,        // non-finite position
    kStatArg = 4u,            // inconsistent arguments detected on device
    kStatTimeout = 8u,        // a bounded wait expired
};

__device__ __forceinline__ void set_status(unsigned *st, unsigned bits) {
    if (st) atomicOr(st, bits);
}


// ------------------------------------------------------------ minimum image
// get_forces.cu:389-391: d -= side * floor(side_inv * d + 0.5f)  (float)
__device__ __forceinline__ float min_image_f(float d, float side, float side_inv) {
    return __fsub_rn(d, __fmul_rn(side, floorf(__fadd_rn(__fmul_rn(side_inv, d), 0.5f))));
}
// get_gder.cu:113-115: floorf(side_inv * d + 0.5) with the 0.5 added in
// double and the sum narrowed to float (same value as the float sum: the
// double sum is exact, so both are one correct rounding of it).
__device__ __forceinline__ float min_image_gder(float d, float side, float side_inv) {
    float t = __double2float_rn(__dadd_rn((double)__fmul_rn(side_inv, d), 0.5));
    return __fsub_rn(d, __fmul_rn(side, floorf(t)));
}
// min_image_gder with an exact shortcut: when |d / side| < 0.49 the floor
// term is 0 and the result is d itself
__device__ __forceinline__ float min_image_gder_fast(float d, float side, float side_inv) {
    return fabsf(__fmul_rn(side_inv, d)) < 0.49f ? d : min_image_gder(d, side, side_inv);
}
// ---------------------------------------------------------------- g(r) bins
// The reference bins a pair at (int)(dist / bin_size) with dist =
// sqrt(d2) (get_gder.cu:116-121), both correctly rounded, when dist < range;
// a bin equal to nbins (rounding at the range) goes to the last bin.  That
// bin is a non-decreasing function of d2, so it is fixed by thresholds:
// gr_thr[k] = the smallest float d2 whose bin is >= k (k = 1 .. nbins), and
// gr_thr[nbins + 1] = the smallest d2 with dist >= range.  Found once per
// call by bisection over the bit patterns of non-negative floats
// (k_gr_thresholds in engine.cu).
__device__ __forceinline__ int gr_bin_exact(float d2, float bin_size) {
    return (int)__fdiv_rn(__fsqrt_rn(d2), bin_size);
}
// bin of d2 (-1 outside the range) from the thresholds in shared memory: a
// fast estimate (off by at most one) corrected against them
__device__ __forceinline__ int gr_bin_thr(float d2, const float *thr, float inv_bin_size, int nbins) {
    if (!(d2 < thr[nbins + 1])) return -1;
    int b = (int)fmaxf(0.f, __fmul_rn(__fmul_rn(d2, rsqrtf(d2)), inv_bin_size));
    b = min(b, nbins);
    if (b < nbins && d2 >= thr[b + 1]) b++;
    else if (b > 0 && d2 < thr[b]) b--;
    return min(b, nbins - 1);
}

// (dx*dx + dy*dy) + dz*dz, every operation rounded (reference host order)
__device__ __forceinline__ float dist2_rn(float dx, float dy, float dz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// ------------------------------------------------------------------ other potentials
// Pair potentials of potentials.cu that the reference defines but never
// calls, for the engine's per-replica potential choice.  pair_extra returns
// the force factor g (force on the home particle = g (r_partner - r_home))
// and adds the pair energy to *u.  di = 1/r, sg = the pair's sigma.
enum PotKind { kPotWcaModified = 0, kPotWca = 1, kPotWca4950 = 2, kPotAO = 3, kPotHsay = 4 };

__device__ __forceinline__ float pair_extra(int pot, const float *pp, float sg, float di, float *u) {
    const float sor = di * sg;
    if (pot == kPotWca) {  // potential_wca (potentials.cu:124-135), the +1 outside epsilon as written
        float s6 = sor * sor * sor;
        s6 = s6 * s6;
        const float s12 = s6 * s6;
        *u += 4.0f * (s12 - s6) + 1.0f;
        return -4.0f * (12.0f * s12 - 6.0f * s6) * di * di;
    }
    const float ros_ao = __double2float_rn(1.0 / (double)sor);  // potentials.cu:102: ros = 1.0 / sor
    if (pot == kPotWca4950 || (pot == kPotAO && ros_ao <= 1.0f)) {
        // potential_wca49_50 (potentials.cu:83-95); the AO core (ros <= 1) is the same
        const float invT = pp[0], AA = pp[1];
        const float s6 = sor * sor * sor * sor * sor * sor;
        const float s12 = s6 * s6, s24 = s12 * s12, s48 = s24 * s24;
        const float s50 = s48 * sor * sor;
        *u += AA * invT * (s50 - s48 * sor) + invT;
        return -AA * invT * (50.0f * s50 - 49.0f * s48 * sor) * di * di;
    }
    if (pot == kPotAO) {  // depletion branch of potential_wca49_50_AO (potentials.cu:97-122)
        const float sigma_pol = pp[2], phi_pol = pp[3];
        const float size_ratio = sg / sigma_pol;
        const float ros = ros_ao;
        const float ros3 = ros * ros * ros;
        const float eta1 = size_ratio + 1.0f, eta2 = eta1 * eta1;
        *u += -phi_pol * (eta2 * eta1 - 1.5f * eta2 * ros + 0.5f * ros3);
        return phi_pol * (1.5f * eta2 * ros - 1.5f * ros3) * di * di;
    }
    // kPotHsay: hard-sphere core (40-20) plus attractive Yukawa tail,
    // U = [(s/r)^40 - 2 (s/r)^20 + 1]_{r<s} - (s/r) exp(-z (r/s - 1)), written
    // as potential_hsay (potentials.cu:149-176) intends: ros = r / s, energies
    // added, g = (dU/dr) / r
    const float z = pp[0];
    const float ros = 1.0f / sor;
    float dudr = 0.f;
    if (ros < 1.0f) {
        const float s2 = sor * sor, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8;
        const float s20 = s4 * s16, s40 = s20 * s20;
        *u += s40 - 2.0f * s20 + 1.0f;
        dudr += -40.0f * (s40 - s20) * di;
    }
    const float uatt = -sor * expf(-z * (ros - 1.0f));
    *u += uatt;
    dudr -= (1.0f + ros * z) * uatt * di;
    return dudr * di;
}
// cut distance of a pair in units of its sigma
__host__ __device__ inline float pot_cut_factor(int pot, const float *pp, float sg) {
    switch (pot) {
        case kPotWca: return 1.12246205f;        // 2^(1/6): the minimum of 4 (s^12 - s^6)
        case kPotWca4950: return 50.0f / 49.0f;  // the minimum of s^50 - s^49
        case kPotAO: return 1.0f + sg / pp[2];   // the depletion term vanishes at r = s (1 + s / sigma_pol)
        case kPotHsay: return pp[1];             // Yukawa tail truncated at pp[1] sigma
        default: return 1.0f;                    // get_forces.cu:331-334
    }
}

// ------------------------------------------------------------------ rannew64
// rannew64 (rannew64.cu:55-126): subtractive lagged Fibonacci x[np] -= x[nq]
// over a 250-word ring (taps 250 and 103, pointers walking down from 249 and
// 102) minus a 64-bit LCG, uniform = (x - y) / (2^64 - 1) in double.  The
// engine keeps one stream per particle; every particle draws 4 uniforms per
// step, so the ring pointers are the same for all particles and follow from
// the number of draws since seeding.
constexpr unsigned long long kRnSeedA = 6364136223846793005ULL, kRnSeedC = 1442695040888963407ULL;
constexpr unsigned long long kRnA = 2862933555777941757ULL, kRnC = 3037000493ULL;
constexpr int kRnWords = 250, kRnDrawsPerStep = 4;

__device__ __forceinline__ double rannew64_uniform(unsigned long long x, unsigned long long y) {
    return (1.0 / 18446744073709551615.0) * __ull2double_rn(x - y);
}
// three N(0,1) values from the 4 draws of step `steps_done` (Box-Muller on
// (u0, u1) and (u2, u3) in float, the sine of the second pair dropped)
__device__ __forceinline__ float3 rannew64_gauss3(unsigned long long *ring, unsigned long long *lcg, int sid,
                                                  size_t P, long long steps_done) {
    const int d = (int)((steps_done * kRnDrawsPerStep) % kRnWords);
    int np = 249 - d, nq = np - 147;
    if (nq < 0) nq += kRnWords;
    unsigned long long y = lcg[sid];
    float u[kRnDrawsPerStep];
#pragma unroll
    for (int k = 0; k < kRnDrawsPerStep; k++) {
        const unsigned long long x = ring[(size_t)np * P + sid] - ring[(size_t)nq * P + sid];
        ring[(size_t)np * P + sid] = x;
        np = np ? np - 1 : kRnWords - 1;
        nq = nq ? nq - 1 : kRnWords - 1;
        y = kRnA * y + kRnC;
        u[k] = __double2float_rn(rannew64_uniform(x, y));
    }
    lcg[sid] = y;
    const float r0 = sqrtf(-2.0f * logf(fmaxf(u[0], 1.17549435e-38f)));
    const float r1 = sqrtf(-2.0f * logf(fmaxf(u[2], 1.17549435e-38f)));
    const float t0 = __fmul_rn(6.2831853f, u[1]), t1 = __fmul_rn(6.2831853f, u[3]);
    return make_float3(__fmul_rn(r0, cosf(t0)), __fmul_rn(r0, sinf(t0)), __fmul_rn(r1, cosf(t1)));
}

// ------------------------------------------------------------------ WCA pair
// potential_wca_modified (potentials.cu:137-147) for a pair inside its cut
// distance sigma: eps[(s/r)^12 - 2 (s/r)^6 + 1] with dist_inv = sqrt(1/dist2)
// (get_forces.cu:397), pair force along d (get_forces.cu:403-405) and the
// virial increment -0.5 d.f (get_forces.cu:413).
struct PairOut {
    float fx, fy, fz, pot, vir;
};
__device__ __forceinline__ PairOut wca_modified_pair(float sigma, float dist2, float dx, float dy, float dz) {
    float dist_inv = __fsqrt_rn(__frcp_rn(dist2));
    float sor = dist_inv * sigma;
    float sor6 = sor * sor * sor;
    sor6 = sor6 * sor6;
    float sor12 = sor6 * sor6;
    PairOut o;
    o.pot = kEps * (sor12 - 2 * sor6 + 1);
    float nf = -kEps * 12 * (sor12 - sor6) * dist_inv;
    o.fx = nf * dist_inv * dx;
    o.fy = nf * dist_inv * dy;
    o.fz = nf * dist_inv * dz;
    o.vir = -0.5f * (dx * o.fx + dy * o.fy + dz * o.fz);
    return o;
}

// ------------------------------------------------------- counter-based RNG
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11, "Parallel random
// numbers: as easy as 1, 2, 3"): ten rounds of two 32x32->64 multiplies with
// a Weyl-sequence key schedule.  Stateless: the engine keys it on
// (replica seed) and counts on (particle id, step, stream).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}
// uniform in (0,1): (x >> 9) 2^-23 + 2^-24 = (2k+1) 2^-24 with 2k+1 < 2^24,
// exact in float
__device__ __forceinline__ float u01(uint32_t x) {
    return __fmaf_rn((float)(x >> 9), 1.1920928955078125e-07f, 5.9604644775390625e-08f);
}
// Three N(0,1) values by the Box-Muller transform of two uniform pairs.
__device__ __forceinline__ float3 gauss3(uint64_t seed, uint32_t id, uint64_t step, uint32_t stream) {
    uint4 b = philox4x32_10(make_uint4(id, (uint32_t)step, (uint32_t)(step >> 32), stream),
                            make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    float r0 = sqrtf(-2.0f * logf(u01(b.x)));
    float r1 = sqrtf(-2.0f * logf(u01(b.z)));
    float s0, c0;
    sincospif(2.0f * u01(b.y), &s0, &c0);
    float c1 = cospif(2.0f * u01(b.w));
    return make_float3(r0 * c0, r0 * s0, r1 * c1);
}

// --------------------------------------------------- compensated position
// Knuth's TwoSum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = __fadd_rn(a, b);
    float bp = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bp)), __fsub_rn(b, bp));
}
// Position carried as hi + lo (|lo| <= ulp(hi)/2).  Adds d exactly, then
// wraps into the periodic box by subtracting side*floor(hi/side) the same
// exact way.  hi stays in [0, side] (side itself only through rounding, as in
// the reference, update_ermak.cu:139-141), which cell indexing clamps.
// Returns the number of box lengths subtracted (0 unless the particle
// crossed a face).
__device__ __forceinline__ float advance_wrap(float &hi, float &lo, float d, float side, float side_inv) {
    float s, e;
    two_sum(hi, d, s, e);
    float c = __fadd_rn(lo, e);
    float h2 = __fadd_rn(s, c);
    c = __fsub_rn(c, __fsub_rn(h2, s));
    float kw = floorf(__fmul_rn(side_inv, h2));
    if (kw != 0.0f) {
        float s2, e2;
        two_sum(h2, -__fmul_rn(side, kw), s2, e2);
        c = __fadd_rn(c, e2);
        h2 = __fadd_rn(s2, c);
        c = __fsub_rn(c, __fsub_rn(h2, s2));
    }
    hi = h2;
    lo = c;
    return kw;
}

// Temperature protocols, set_temp.cu:7-23, same float arithmetic (the
// reference host code has no FMA; the intrinsics keep it that way).
__host__ __device__ inline float temp_linear(float T0, float Tf, float t0, float tf, float t) {
    if (t < t0) return T0;
    if (t > tf) return Tf;
#ifdef __CUDA_ARCH__
    float m = __fdiv_rn(__fsub_rn(Tf, T0), __fsub_rn(tf, t0));
    return __fadd_rn(T0, __fmul_rn(m, __fsub_rn(t, t0)));
#else
    volatile float m = (Tf - T0) / (tf - t0);
    volatile float p = m * (t - t0);
    return T0 + p;
#endif
}

}  // namespace bd
