// engine.cuh -- data layout of the batched replica engine.
//
// A batch holds R independent periodic systems ("replicas") of uneven size.
// Per replica the box is cut into ncell^3 cubic cells of side >= the largest
// pair cut distance (both species share one grid), so every pair inside its
// cut distance lies in the 27 cells around a particle.  Cells of all replicas
// are numbered consecutively (SysDev::cell_base).
//
// HBM layout (P particles, C cells in the whole batch):
//   cnt[3][C]        int    particles per cell, triple-buffered: step t reads
//                            buffer t%3, bins into (t+1)%3, clears (t+2)%3
//   pos[3][C*cap]    float4 cell-bucketed positions: x, y, z (wrapped, FP32
//                            high part) and w = storage id | species << 31
//   lo_{x,y,z}[P]    float  compensated remainder of the position
//   dsp_{x,y,z}[P]   double unwrapped displacement since the last origin
//   gid_of[P]        int    global particle index (replica base + reference
//                            particle index) of each storage id
// Storage ids are assigned once, in brick/cell order, so the private arrays
// are read almost contiguously by the bricks that own the particles.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace bd {

struct SysDev {
    float L, Linv, cinv;  // box side, 1/L (float division), ncell/L
    int ncell;
    int cell_base, n, n_big, part_base;
    float sig[3], cut2[3];  // bb, bs, ss cut distances and their squares
    float mob[2];           // mobility of big, small
    float dt, fcap;         // fcap > 0: cap on |F| (initial relaxation)
    double dt_d;
    int protocol;           // 0 linear, 1 sine, 2 constant
    float T0, Tf, t0, tf, period;
    float T_first;     // temperature of the first update (T0 unless the caller set another)
    unsigned long long seed;
    int nbx, nby, nbz, brick_base;
    int pot;           // PotKind
    float pp[4];       // potential parameters
    float lcut2[3];    // neighbour-list mode: (cut distance + skin)^2 per species pair
    float skin_half2;  //   (skin / 2)^2: a particle farther than this from its build position
    float interior;    //   a particle at least this far from every face has no list partner
                       //   across the boundary (largest list distance + skin, plus a margin)
};

// per-replica observation accumulators (FP64)
enum ObsField {
    kObsPotBig = 0,   // sum over big of pot_i  (energy = 0.5 sum / N_big)
    kObsPotSml = 1,
    kObsVir = 2,      // sum over all of vir_i
    kObsMsdBig = 3,   // sum |dsp|^2 over big
    kObsMsdSml = 4,
    kObsFsBig = 5,    // sum sin(q|dsp|)/(q|dsp|) over big
    kObsNbr = 6,      // number of interacting ordered pairs (census)
    kObsCount = 8
};

enum RngMode { kRngPhilox = 0, kRngCurand = 1, kRngNoise = 2, kRngRannew64 = 3 };

// candidates of one home cell held in registers per chunk (4 per lane)
constexpr int kMaxCand = 128;

struct StepArgs {
    const SysDev *sys;
    const int4 *bricks;  // (replica, ox, oy, oz)
    int nbricks;
    int bx, by, bz;      // brick dims in cells
    int cap;             // slots per cell
    int smax;            // staging capacity (particles) per CTA
    const int *cnt_in;
    const float4 *pos_in;
    int *cnt_out;
    float4 *pos_out;
    int *cnt_clr;
    float *lo_x, *lo_y, *lo_z;
    double *dsp_x, *dsp_y, *dsp_z;
    const int *gid_of;
    int np;              // particles in the batch (bound for storage ids)
    double *x0;          // [3P] origin of the unwrapped positions, by gid
    float4 *snap;        // [P] positions by gid, written by observation passes
    double *obs;         // [R][kObsCount]
    int *nbr_count;      // census: interacting partners per gid (or null)
    unsigned long long *nbr_hash;
    void *curand_states; // by gid
    const float *noise;  // [3P] by gid
    unsigned long long *rn_ring;  // rannew64 mode: [250][P] lagged-Fibonacci words by storage id
    unsigned long long *rn_lcg;   //   [P] LCG state by storage id
    long long rn_ni0;             //   step index at which the streams were seeded
    unsigned *status;
    int *cnt3[3];        // all three count / position buffers (persistent mode
    float4 *pos3[3];     //   rotates them itself, step s uses (cur0 + s) % 3)
    int cur0;
    const int *cl_start; // persistent mode: bricks of cluster c are
    const int *cl_bricks;//   cl_bricks[cl_start[c] .. cl_start[c+1])
    long long ni;        // reference step index of this update
    long long ni_first;  // first step of the run (the reference uses T0 there)
    float qmax;          // wave number of the built-in F_s accumulator
    int do_update;
    uint32_t rng_stream;
};

}  // namespace bd
