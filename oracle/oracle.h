/*
 * oracle.h -- CPU restatement of the reference hot path (Ramborquito/bd_aging),
 * used ONLY as the checker by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs.  Never linked into the product library.
 *
 * Two groups of functions:
 *   or_ref_*  restate the reference's own arithmetic (float/double operation
 *             order of the *_hst functions) so that results can be compared
 *             bit for bit with the reference built from its sources
 *             (oracle/_ref/libref.so, golden vectors in tests/golden/).
 *   or_eng_*  restate the B200 engine's arithmetic (counter-based Gaussian
 *             generator, compensated FP32 position + FP64 unwrapped
 *             displacement update, FP64 observables) for the engine's tests.
 * Arrays of positions/forces are float3 AoS (3 floats per particle) as in the
 * reference.
 */
#ifndef BD_ORACLE_H
#define BD_ORACLE_H
#include <stdint.h>
#include "../include/bd_aging.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference restatement ---- */
void or_ref_setup_params(bd_parametros *p, float side, int nb, int ns, float sigma_big, float sigma_sml,
                         float mass_big, float mass_sml, int ntags_big, int ntags_sml, int nbins_gder,
                         float range_gder, double dt, float temp0);
int or_ref_cell_locate(char type, const float *rr, int *nocup, int *cell_vec, const bd_parametros *p);
void or_ref_forces_same(char type, const float *rr, float *ff, float *vir, float *pot, const int *nocup,
                        const int *cell_vec, const bd_parametros *p);
void or_ref_forces_diff(char type, char type_other, const float *rr, float *ff, const float *rr_other,
                        float *vir, float *pot, const int *nocup_o, const int *cell_o, const bd_parametros *p);
void or_ref_update_ermak(char type, float *rr, float *rr_raw, const float *ff, const float *noise,
                         const bd_parametros *p);
void or_ref_gder_counts(char type, char type_other, const float *rr, const float *rr_other, uint64_t *counts,
                        const bd_parametros *p);
void or_ref_gder_normalize(const double *counts, int nbins, float bin_size, float side, int nb, int ns,
                           float sigma_big, float sigma_sml, int n_configs, float *gder);
void or_ref_fself(const float *rr_raw, const float *rr0, int n, float *fself, int sample_number, float qmax);
float or_ref_msd(const float *rr_raw, const float *rr0, int n);
float or_ref_energy(const float *pot, int n);
float or_ref_pressure_z(const float *vir_b, int nb, const float *vir_s, int ns, float temp);
float or_ref_temp_linear(float T0, float Tf, float t0, float tf, float t);
float or_ref_temp_sine(float T0, float Tf, float t0, float tf, float period, float t);
float or_ref_time_of_step(double dt, int ni);
int or_ref_sampling_indexes(float minimal_decade, float run_time, float dt, int per_decade, int *out, int cap);
/* reference rannew64 (rannew64.cu:55-126) with explicit state (one stream) */
typedef struct { uint64_t useed[250]; uint64_t uuy; int np, nq, init; } or_rannew64_state;
void or_rannew64_seed(or_rannew64_state *s, long idum);
void or_rannew64_particle_noise(long long seed, int n, int steps, float *noise);
int or_precision_run(int mode, int n, int n_big, const float *pos0, double side, double sig_big, double sig_sml,
                     double mob_big, double mob_sml, double dt, double temp, uint64_t seed, uint32_t stream,
                     long long ni0, int steps, double q, double *obs, double *dsp_out);
double or_rannew64_next(or_rannew64_state *s);
/* Contracting_Vector3D::add_statistics (Contracting_Vector3D.cu:57-164) in the
 * reference's float arithmetic; ata: 3 x bins x bins, atb: 3 x bins. side<=0:
 * no periodic images.  Returns 0, or 1 if a neighbour list hit NEIGHS_MAX. */
int or_ref_cv3d_add(int bins, float range, const float *rr, const float *xx, int n, float side, float *ata,
                    float *atb);

/* ---- engine restatement ---- */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11 "Parallel random numbers:
 * as easy as 1, 2, 3"). */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Engine Gaussian triple for (seed, particle id, step, stream); double values
 * of the same Box-Muller transform the device evaluates in float. */
void or_eng_gauss3(uint64_t seed, uint32_t id, uint64_t step, uint32_t stream, double out[3]);
void or_eng_uniform_bits(uint64_t seed, uint32_t id, uint64_t step, uint32_t stream, uint32_t out[4]);
/* Engine pair force on all particles of one periodic system (O(N^2), sums in
 * ascending partner index): type[i] 0=big 1=small; sigma[2] are the
 * reference cut distances s_b, s_s; ff float3; pot/vir per particle; nbr
 * (optional) = number of partners within the pair cutoff. */
void or_eng_forces(int n, const float *pos, const int *type, float side, const float sigma[2], float *ff,
                   float *pot, float *vir, int *nbr, uint64_t *nbr_hash);
/* One engine step with given N(0,1) noise (3 per particle, float values):
 * compensated position (hi, lo), FP64 displacement, reference drift/noise
 * formula with mobility mob[type] and amplitude amp[type]. */
void or_eng_cap_forces(int n, float *ff, float fcap);
void or_eng_update(int n, float *hi, float *lo, double *dsp, const float *ff, const int *type, float side,
                   double dt, const float mob[2], const float amp[2], const float *noise);
float or_eng_amplitude(float temp, float mob, float dt);
/* FP64 F_s and MSD of a displacement set (n x 3 doubles). */
void or_eng_fself_msd(int n, const double *d, double q, double *fs, double *msd);

#ifdef __cplusplus
}
#endif
#endif
