/*
 * bd_aging.h -- C ABI of the B200 Brownian-dynamics engine (libbd_aging_b200.so).
 *
 * Two layers:
 *
 *  1. Reference-mirror entry points.  One function per entry point of the
 *     reference (encabezados.h:86-158), same argument meaning, operating on
 *     device-accessible pointers (cudaMalloc'd or managed memory) with the
 *     reference's float3 array-of-structs layout (3 floats per particle).
 *     Differences: every call returns an int status (BD_OK or a BD_ERR_*
 *     code) instead of calling exit(), takes an explicit CUDA stream
 *     (NULL = legacy default stream), and never writes out of bounds.
 *
 *  2. The batched replica engine (bd_engine_*): many independent systems of
 *     uneven size stepped together by fused sm_100a kernels.  Positions enter
 *     and leave through host float3 arrays in the reference's particle order
 *     (big particles first, main.cu:377-394).
 *
 * All functions are thread-compatible (no hidden global state apart from
 * per-device kernel attributes); handles are not shared across threads.
 */
#ifndef BD_AGING_H
#define BD_AGING_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BD_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
#define BD_OK                 0
#define BD_ERR_ARG            1   /* invalid argument (NULL, size, species char) */
#define BD_ERR_CUDA           2   /* a CUDA runtime call failed                  */
#define BD_ERR_CELL_OVERFLOW  3   /* a cell held more particles than its capacity
                                     (reference: "ntags reached limit", exit 1,
                                     main.cu:655-659)                            */
#define BD_ERR_NOMEM          4
#define BD_ERR_STATE          5   /* call out of order (e.g. run before load)    */
#define BD_ERR_TIMEOUT        6   /* a bounded device wait expired               */
#define BD_ERR_FILE           7   /* file missing / unreadable (reference exit -2)*/
#define BD_ERR_FORMAT         8   /* malformed input (reference exit 1)          */
#define BD_ERR_NUMERIC        9   /* non-finite position detected                */

const char *bd_status_string(int status);
int bd_abi_version(void);

/* ---- parameter block: layout-identical to the reference `parametros`
 *      (encabezados.h:40-75) so a reference caller can pass its own struct. */
typedef struct bd_parametros {
    float side;
    float dt;
    float mass_big;
    float mass_sml;
    float sigma_big;
    float sigma_sml;
    float cell_side_big;
    float cell_side_sml;
    float temp_set;
    float bin_size_dplt;
    float bin_size_gder;
    float range_dplt;
    float range_gder;
    int ngrain_big;
    int ngrain_sml;
    int ngrain_tot;
    int ntags_big;
    int ntags_sml;
    int ncell_big;
    int ncell_med;
    int ncell_sml;
    int nrange_bb;
    int nrange_bs;
    int nrange_sb;
    int nrange_ss;
    int nbins_dplt;
    int nbins_gder;
    int nsearch_big;
    int not_finished;
    int NH;
    int WCA_flag;
    long idum;
} bd_parametros;

/* Parameter set-up of the reference driver (main.cu:155-163, 244-298,
 * 348-349): cell counts (int)(side/(1.05 sigma)), cell sides, neighbour
 * ranges nrange_bb/bs/sb/ss, gder bin size.  Host-only. */
int bd_setup_params(bd_parametros *pars, float side, int ngrain_big, int ngrain_sml, float sigma_big,
                    float sigma_sml, float mass_big, float mass_sml, int ntags_big, int ntags_sml,
                    int nbins_gder, float range_gder, double dt, float temp0);

/* ---- reference-mirror entry points (device pointers) -------------------- */

/* cell_locate_dev (cell_locate.cu:155-209) together with the clears that the
 * reference launches before it (set_vec_int_dev, main.cu:536-541).  type is
 * 'b' or 's'.  Output: nocup[ncell^3] occupancies and cell_vec[ncell^3 *
 * ntags] particle indices, occupied slots in ascending particle order (the
 * order of cell_locate_hst; the reference device order is arbitrary), unused
 * slots -1.  A cell above ntags particles returns BD_ERR_CELL_OVERFLOW and
 * writes only the first ntags slots. */
int bd_cell_locate(char type, const float *rr, int *nocup, int *cell_vec, const bd_parametros *pars,
                   void *stream);

/* get_forces_same_dev (get_forces.cu:297-424): WCA-modified forces, potential
 * and virial between particles of species `type`, ADDED to ff/vir/pot like
 * the reference (callers clear them first, main.cu:556-561).  nocup/cell_vec
 * come from bd_cell_locate for the same species. */
int bd_get_forces_same(char type, const float *rr, float *ff, float *vir, float *pot, const int *nocup,
                       const int *cell_vec, const bd_parametros *pars, void *stream);

/* get_forces_diff_dev (get_forces.cu:428-558): forces on `type` particles
 * from `type_other` particles, using the other species' cell list. */
int bd_get_forces_diff(char type, char type_other, const float *rr, float *ff, const float *rr_other,
                       float *vir, float *pot, const int *nocup_other, const int *cell_other,
                       const bd_parametros *pars, void *stream);

/* Size in bytes of the per-particle generator state used by bd_setup_rng /
 * bd_update_ermak (the reference's curandState, update_ermak.cu:83-89). */
size_t bd_rng_state_size(void);

/* setup_rng_kernel (update_ermak.cu:85-89): curand_init(seed, idx, 0) for
 * idx < n.  The reference seeds big with idum and small with idum+1
 * (main.cu:483-484). */
int bd_setup_rng(void *states, unsigned long long seed, int n, void *stream);

/* update_ermak_dev (update_ermak.cu:91-160): Ermak-McCammon step with the
 * reference's cuRAND XORWOW stream: r += F dt/sigma + sqrt(2 T dt/sigma) xi,
 * periodic wrap of rr, rr_raw advanced without wrap.  T = pars->temp_set. */
int bd_update_ermak(char type, float *rr, float *rr_raw, const float *ff, void *states,
                    const bd_parametros *pars, void *stream);

/* Same update with caller-supplied N(0,1) values noise[3*i+{0,1,2}]
 * (parity tests inject identical noise into the reference's host twin,
 * update_ermak.cu:8-77). */
int bd_update_ermak_noise(char type, float *rr, float *rr_raw, const float *ff, const float *noise,
                          const bd_parametros *pars, void *stream);

/* calculate_temp_linear / calculate_temp_sine (set_temp.cu:7-23), same
 * float arithmetic, including the reference's NaN at t == t0 == tf. */
float bd_calculate_temp_linear(float T0, float Tf, float t0, float tf, float t);
float bd_calculate_temp_sine(float T0, float Tf, float t0, float tf, float period, float t);

/* get_gder_dev (get_gder.cu:69-127) for one species pair: ordered pairs with
 * minimum-image distance < range_gder binned by (int)(dist/bin_size), with the
 * reference's float operation order.  Counts are ADDED to the caller's
 * device array counts[nbins_gder] as exact 64-bit integers (the reference
 * accumulates floats per block, exact below 2^24 per bin). */
int bd_get_gder(char type, char type_other, const float *rr, const float *rr_other,
                unsigned long long *counts, const bd_parametros *pars, void *stream);

/* g(r) normalisation of main.cu:849-877 for one sample, host arithmetic
 * identical to the reference: counts[4][nbins] (bb, bs, sb, ss) summed over
 * configs -> gder[4][nbins] averaged over n_configs.  Host pointers. */
int bd_gder_normalize(const double *counts, int nbins, float bin_size, float side, int ngrain_big,
                      int ngrain_sml, float sigma_big, float sigma_sml, int n_configs, float *gder);

/* fself_isotropic (fself.cu:3-21): adds (1/N) sum sin(q|dr|)/(q|dr|) over
 * dr = rr_raw - rr0 to fself_host[sample_number].  The FP64 sum runs in a
 * fixed order, so repeated calls give identical bits.  Device inputs, host
 * output, stream-synchronous. */
int bd_fself_isotropic(const float *rr_raw, const float *rr0, int ngrain, float *fself_host, int sample_number,
                       float qmax, void *stream);

/* No counterpart in the reference.  Same result as bd_fself_isotropic for
 * callers that cannot allocate device memory when they sample F_s: real-time
 * loops that forbid allocation after start-up, and programs whose device
 * memory is reserved up front by another allocator.  Its scratch is a fixed
 * 32 KB device array per GPU, held until process exit, so it calls no
 * cudaMalloc.  Limit: ngrain <= 1,048,576, larger calls return BD_ERR_ARG.
 * The first call on a device looks up the scratch address (a runtime call
 * that a global-mode stream capture elsewhere in the process would refuse),
 * so make it before such a capture starts.  The call synchronises its
 * stream, so it cannot itself be captured.  All calls on a GPU share the
 * scratch: calls that overlap on the GPU (two streams or threads) race, so
 * serialise them.  Device inputs, host output, stream-synchronous. */
int bd_fself_isotropic_noalloc(const float *rr_raw, const float *rr0, int ngrain, float *fself_host,
                               int sample_number, float qmax, void *stream);

/* calculate_color (colors.cu:64-110) for every big particle, as the snapshot
 * pass of main.cu:663-713 does (compiled in with GRO_FLAG): colour ids
 * (device, ngrain_big ints, or NULL) 0 blue (no big neighbour), 1 green,
 * 2 red (more neighbour pairs with a small particle between them than
 * without); counts_host[3] = blue, green, red (color_statistics.out). */
int bd_color_statistics(const float *rr_big, const float *rr_sml, int *color_ids, int *counts_host,
                        const bd_parametros *p, void *stream);

/* Mean squared displacement of main.cu:776-792 for one species: returns
 * (1/N) sum |rr_raw - rr0|^2 in *msd_host.  Stream-synchronous. */
int bd_msd(const float *rr_raw, const float *rr0, int ngrain, float *msd_host, void *stream);

/* ---- Contracting_Vector3D (Contracting_Vector3D.cuh:39-75) --------------- */
typedef struct bd_cv3d bd_cv3d;
/* constructor (Contracting_Vector3D.cu:11-55) */
int bd_cv3d_create(int bins, float range, bd_cv3d **out);
/* add_statistics (Contracting_Vector3D.cu:57-164): device rr/xx float3 arrays;
 * side <= 0 means no periodic images (std::nullopt in the reference).  The
 * normal equations are accumulated on the GPU in FP64. */
int bd_cv3d_add_statistics(bd_cv3d *cv, const float *rr, const float *xx, int nparticles, float side,
                           void *stream);
/* calculate_vector (Contracting_Vector3D.cu:166-297): SVD pseudo-inverse
 * solve per Cartesian component, averaged over the three.  Returns
 * BD_ERR_STATE when no statistics were added (the reference throws). */
int bd_cv3d_calculate_vector(bd_cv3d *cv);
/* get_vector (Contracting_Vector3D.cu:299-304); BD_ERR_STATE before
 * calculate_vector (the reference throws). Host output of `bins` floats. */
int bd_cv3d_get_vector(const bd_cv3d *cv, float *out);
int bd_cv3d_destroy(bd_cv3d *cv);

/* ---- batched replica engine ------------------------------------------------
 * Replaces the reference time loop (main.cu:494-588, one system per process,
 * 18 kernel launches and 3 device synchronisations per step, configurations
 * run one after another, main.cu:213) with one fused launch per step over
 * all replicas, or one persistent launch per chunk of steps. */
typedef struct bd_engine bd_engine;

#define BD_PROTOCOL_LINEAR 0   /* calculate_temp_linear, set_temp.cu:7-12 */
#define BD_PROTOCOL_SINE 1     /* calculate_temp_sine, set_temp.cu:14-23 */
#define BD_PROTOCOL_CONST 2    /* T = T0 throughout */

#define BD_RNG_PHILOX 0   /* counter-based Philox4x32-10 + Box-Muller (default) */
#define BD_RNG_CURAND 1   /* the reference's cuRAND XORWOW stream: big seeded with
                             seed, small with seed+1, subsequence = index within
                             the species (main.cu:478-484) */
#define BD_RNG_NOISE 2    /* caller-supplied N(0,1) values (bd_engine_set_noise) */
#define BD_RNG_RANNEW64 3 /* one rannew64 stream per particle (rannew64.cu:55-126),
                             idum = seed + particle index, 4 uniforms per step,
                             Box-Muller in float; 2008 bytes of state per particle */

#define BD_MODE_AUTO 0
#define BD_MODE_PLAIN 1       /* one launch per step, steps captured in CUDA graphs */
#define BD_MODE_PERSISTENT 2  /* one launch per chunk; thread-block clusters own
                                 replicas and synchronise between steps */

typedef struct bd_system_desc {
    int n_big, n_sml;          /* particles 0..n_big-1 are big (main.cu:387-393) */
    float side;                /* cubic periodic box side */
    float sigma_big, sigma_sml;/* reference `sigma`: the WCA cut distance s; the
                                  big-small pair uses (s_b + s_s)/2 */
    float mob_big, mob_sml;    /* mobilities; the reference uses 1/sigma
                                  (update_ermak.cu:106-114) */
    double dt;
    int temp_protocol;         /* BD_PROTOCOL_* */
    float T0, Tf, t0, tf, period;
    unsigned long long seed;   /* RNG key of this replica (idum for BD_RNG_CURAND) */
    float force_cap;           /* > 0: |F| capped (initial-configuration relaxation) */
    int potential;             /* BD_POT_* (0: the reference's modified WCA) */
    float pot_param[4];        /* parameters of the potential, see BD_POT_* */
    int first_temp_set;        /* != 0: the replica's first update runs at T_first instead of T0.
                                  The reference sets temp_set to T0 once, before its loop over
                                  configurations (main.cu:156), so every configuration after the
                                  first starts at the temperature the previous one ended on */
    float T_first;
} bd_system_desc;

/* Pair potentials (potentials.cu).  The reference's step uses the modified
 * WCA only (get_forces.cu); the others are defined there and never called.
 * Cut distances are per species pair, in units of the pair's sigma s. */
#define BD_POT_WCA_MODIFIED 0  /* (s/r)^12 - 2 (s/r)^6 + 1, cut s (potentials.cu:137-147) */
#define BD_POT_WCA 1           /* 4 ((s/r)^12 - (s/r)^6) + 1, cut 2^(1/6) s (potentials.cu:124-135) */
#define BD_POT_WCA49_50 2      /* A invT ((s/r)^50 - (s/r)^49) + invT, cut 50/49 s; pot_param = {invT, A}
                                  (potentials.cu:83-95) */
#define BD_POT_AO 3            /* 49-50 core for r <= s, Asakura-Oosawa depletion beyond, cut
                                  s (1 + s / sigma_pol); pot_param = {invT, A, sigma_pol, phi_pol}
                                  (potentials.cu:97-122) */
#define BD_POT_HSAY 4          /* 40-20 core for r < s plus -(s/r) exp(-z (r/s - 1)), cut c s;
                                  pot_param = {z, c}.  potentials.cu:149-176 writes ros = s r, assigns
                                  the energy and flips the core force; this is its evident intent */

typedef struct bd_engine_opts {
    int rng;                   /* BD_RNG_* */
    int cell_capacity;         /* slots per cell, at most 24 (0: 16, or 24 in list mode, or more
                                  when the cells hold more than 4 particles on average) */
    int brick[3];              /* cells per brick (0 = autotune / default) */
    int threads;               /* CTA size (0 = default) */
    int mode;                  /* BD_MODE_* */
    int cluster;               /* CTAs per cluster in persistent mode (0 = 8) */
    int autotune;              /* 1: time brick/CTA shapes at first run */
    int graph_steps;           /* steps per captured CUDA graph (0 = 96) */
    float qmax;                /* wave number of the built-in F_s observable */
    long long ni_start;        /* reference step index of the first update
                                  (-ntrans, main.cu:407 and 494) */
    unsigned rng_stream;       /* Philox stream number (0 dynamics, 1 relaxation) */
    float neighbor_skin;       /* > 0 (default 0.25): neighbour-list mode (plain mode,
                                  generated noise): lists of partners within cut + skin,
                                  rebuilt on the device when a particle of the replica
                                  has moved skin / 2; 0: the 27-cell sweep every step.
                                  At most 1, and at most 0.9 of each replica's largest
                                  cut distance (BD_ERR_ARG otherwise) */
    int list_variant;          /* list-step launch variant 0 .. BD_LIST_VARIANTS-1, same
                                  results in every variant: 0-2 launch each step (CTA size,
                                  registers, load placement) with separate rebuild kernels;
                                  3-5 run a whole batch of steps in one launch, one block
                                  of 256 / 512 / 1024 threads per replica that rebuilds its
                                  replica's lists itself (Philox noise; the other noise
                                  streams run variant 0).  -1 (default): variant 0, or with
                                  autotune chosen with the brick shape at the first run */
} bd_engine_opts;
#define BD_LIST_VARIANTS 6

typedef struct bd_observables {
    double energy_big, energy_sml; /* (1/N) sum 0.5 pot_i per species (main.cu:627-631) */
    double virial;                 /* sum of per-particle virials (main.cu:801-803) */
    double msd_big, msd_sml;       /* mean |r - r(step 0)|^2 (main.cu:776-792), FP64 */
    double fself_big;              /* F_s(qmax) of the big particles (fself.cu), FP64 */
    double nbr_pairs;              /* interacting ordered pairs (census only) */
    double temperature;            /* temp_set after the last completed step */
} bd_observables;

typedef struct bd_engine_info {
    int nsys;
    long long n_particles, n_cells;
    int brick[3], threads, cell_capacity, staging_capacity, mode, cluster;
    size_t smem_bytes;
    long long next_step;          /* reference ni of the next update */
    float neighbor_skin;          /* 0 when the engine sweeps every step */
    long long list_builds;        /* neighbour-list builds so far (per replica) */
    long long list_rebuild_steps; /* time steps that rebuilt some replica's lists */
    int list_variant;             /* list-step launch variant in use (-1: sweep mode) */
    float tuned_ms;               /* autotuner: time per step of the chosen layout (0 untuned) */
} bd_engine_info;

void bd_engine_opts_default(bd_engine_opts *opts);
/* Geometry + buffers for nsys replicas.  Box sides must hold >= 3 cells of
 * the largest cut distance. */
int bd_engine_create(const bd_system_desc *systems, int nsys, const bd_engine_opts *opts, bd_engine **out);
int bd_engine_destroy(bd_engine *e);
int bd_engine_get_info(const bd_engine *e, bd_engine_info *info);
/* The CUDA stream all engine work is issued on (for caller-side events). */
int bd_engine_get_stream(const bd_engine *e, void **stream);
/* Host positions of all replicas, float3 per particle, replica after replica,
 * each in the reference order (big first).  Resets displacements. */
int bd_engine_set_positions(bd_engine *e, const float *pos_host);
/* Advance every replica by nsteps reference steps. */
int bd_engine_run(bd_engine *e, long long nsteps);
/* Observables of the current state (the reference's sample step: forces of
 * the positions after the last update).  out: nsys entries. */
int bd_engine_observe(bd_engine *e, bd_observables *out);
/* Wrapped (rr) and unwrapped (rr_raw) positions, float3 per particle in the
 * set_positions order.  Either pointer may be NULL. */
int bd_engine_get_positions(bd_engine *e, float *pos_host, float *raw_host);
/* g(r) counts of the current state: counts_host[nsys][4][nbins] (bb, bs, sb,
 * ss ordered pairs, get_gder.cu arithmetic), exact integers. */
int bd_engine_gder(bd_engine *e, int nbins, float range, unsigned long long *counts_host);
#define BD_GDER_AUTO 0       /* per replica: cell-bounded whenever the box holds the stencil region
                                (4 + 2 ceil(range / cell side) cells per axis), else all pairs */
#define BD_GDER_ALL_PAIRS 1  /* every pair, as get_gder_dev (get_gder.cu:69-127) */
#define BD_GDER_CELLS 2      /* only cells within the range (BD_ERR_ARG if a replica's box
                                is under 4 + 2 ceil(range / cell side) cells) */
/* bd_engine_gder with an explicit candidate search; every method gives the
 * same exact counts. */
int bd_engine_gder_method(bd_engine *e, int nbins, float range, int method, unsigned long long *counts_host);
/* BD_RNG_NOISE: N(0,1) values for the next step, 3 per particle (set_positions order). */
int bd_engine_set_noise(bd_engine *e, const float *noise_host);
/* Interacting partners of every particle and a hash of their indices (the
 * neighbour set), from the engine's own pair selection.  Host outputs. */
int bd_engine_census(bd_engine *e, int *nbr_count, unsigned long long *nbr_hash);

/* ---- waiting-time correlations ---------------------------------------------
 * The reference measures F_s(q; t_w, t_w + tau) and the MSD at a waiting time
 * t_w by restarting from the configuration written at t_w (main.cu:809-835,
 * run-fself.sh:149-197) and evaluating fself_isotropic (fself.cu:3-21) and
 * the MSD loop (main.cu:776-797) against the restart origin (main.cu:497-506).
 * The engine keeps the FP64 displacement of every particle at each t_w in a
 * snapshot slot (24 bytes per particle per slot) and reduces all requested
 * (slot, replica) pairs in one pass. */
typedef struct bd_correlation {
    long long lag_steps;         /* steps since the snapshot */
    double fself_big, fself_sml; /* (1/N_s) sum sin(q|dr|) / (q|dr|), FP64 */
    double msd_big, msd_sml;     /* (1/N_s) sum |dr|^2 */
    double r4_big, r4_sml;       /* (1/N_s) sum |dr|^4 (non-Gaussian parameter) */
} bd_correlation;

/* Room for nslots snapshots (keeps those already taken). */
int bd_engine_reserve_snapshots(bd_engine *e, int nslots);
/* Record the current displacement of every particle in `slot`.  Taken just
 * before the reference's origin step (next step index 0) it is that origin. */
int bd_engine_snapshot(bd_engine *e, int slot);
/* Correlations of the current state with slots[0..nslots) (at most 64):
 * out[j * nsys + r] for slot j, replica r.  BD_ERR_STATE if a slot is empty,
 * predates bd_engine_set_positions, or predates the origin step. */
int bd_engine_correlate(bd_engine *e, const int *slots, int nslots, double q, bd_correlation *out);
/* FP64 displacement of every particle since the origin step (or since
 * bd_engine_set_positions before it), float3-like triples in the
 * set_positions order: the reference's rr_raw - rr_ini (main.cu:776-797). */
int bd_engine_get_displacements(bd_engine *e, double *dsp_host);

#ifdef __cplusplus
}
#endif
#endif /* BD_AGING_H */
