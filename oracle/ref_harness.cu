// extern "C" wrappers around the reference's own host functions, compiled
// from the reference sources by oracle/Makefile into oracle/_ref/libref.so.
// Test infrastructure: it lets the tests and the golden-vector script call
// the reference implementation itself (cell_locate_hst, get_forces_*_hst,
// update_ermak_hst, get_gder_hst, fself_isotropic, calculate_temp_*,
// sampling_indexes, Contracting_Vector3D, calculate_color) on chosen inputs.
#include "encabezados.h"
#include "Contracting_Vector3D.cuh"
#include <vector>
#include <optional>

std::vector<int> sampling_indexes(float minimal_decade, float run_time, float dt, int samplings_per_decade);

extern "C" {

int ref_sizeof_parametros(void) { return (int)sizeof(parametros); }

void ref_cell_locate_hst(char type, float *rr, int *nocup, int *cell, const parametros *p) {
    cell_locate_hst(type, (float3 *)rr, nocup, cell, *p);
}
void ref_get_forces_same_hst(char type, float *rr, float *ff, float *vir, float *pot, int *nocup,
                             int *cell, const parametros *p) {
    get_forces_same_hst(type, (float3 *)rr, (float3 *)ff, vir, pot, nocup, cell, *p);
}
void ref_get_forces_diff_hst(char type, char type_other, float *rr, float *ff, float *rr_other,
                             float *vir, float *pot, int *nocup_o, int *cell_o, const parametros *p) {
    get_forces_diff_hst(type, type_other, (float3 *)rr, (float3 *)ff, (float3 *)rr_other, vir, pot,
                        nocup_o, cell_o, *p);
}
void gsl_shim_rng_set_noise(gsl_rng *r, const double *noise, long n);
void ref_update_ermak_hst(char type, float *rr, float *rr_raw, float *ff, const double *noise, long nnoise,
                          const parametros *p) {
    gsl_rng *r = gsl_rng_alloc(gsl_rng_mt19937);
    gsl_shim_rng_set_noise(r, noise, nnoise);
    update_ermak_hst(type, (float3 *)rr, (float3 *)rr_raw, (float3 *)ff, r, *p);
    gsl_rng_free(r);
}
void ref_get_gder_hst(char type, char type_other, float *rr, float *rr_other, float *gder, const parametros *p) {
    get_gder_hst(type, type_other, (float3 *)rr, (float3 *)rr_other, gder, *p);
}
void ref_fself_isotropic(float *rr_raw, float *rr0, int ngrain, float *fself, int sample_number, float qmax) {
    fself_isotropic((float3 *)rr_raw, (float3 *)rr0, ngrain, fself, sample_number, qmax);
}
float ref_calculate_temp_linear(float T0, float Tf, float t0, float tf, float t) {
    return calculate_temp_linear(T0, Tf, t0, tf, t);
}
float ref_calculate_temp_sine(float T0, float Tf, float t0, float tf, float period, float t) {
    return calculate_temp_sine(T0, Tf, t0, tf, period, t);
}
void ref_potential_wca_modified_hst(float sigma, float dist_inv, float *potential, float *normal_force) {
    potential_wca_modified_hst(sigma, dist_inv, *potential, *normal_force);
}
int ref_sampling_indexes(double minimal_decade, double run_time, double dt, int per_decade, int *out, int cap) {
    std::vector<int> v = sampling_indexes(minimal_decade, run_time, dt, per_decade);
    int n = (int)v.size();
    for (int i = 0; i < n && i < cap; i++) out[i] = v[i];
    return n;
}

void *ref_cv3d_create(int bins, float range) { return new Contracting_Vector3D(bins, range); }
void ref_cv3d_add_statistics(void *h, float *rr, float *xx, int n, float side) {
    auto *cv = (Contracting_Vector3D *)h;
    if (side > 0.0f) cv->add_statistics((float3 *)rr, (float3 *)xx, n, side);
    else cv->add_statistics((float3 *)rr, (float3 *)xx, n);
}
void ref_cv3d_calculate_vector(void *h) { ((Contracting_Vector3D *)h)->calculate_vector(); }
void ref_cv3d_get_vector(void *h, float *out) { ((Contracting_Vector3D *)h)->get_vector(out); }
void ref_cv3d_destroy(void *h) { delete (Contracting_Vector3D *)h; }
// the host potentials of potentials.cu that the reference never calls
void ref_potential_wca_hst(float sigma, float dist_inv, float *pot, float *nf) {
    potential_wca_hst(sigma, dist_inv, *pot, *nf);
}
void ref_potential_wca49_50_hst(float sigma, float dist_inv, float invT, float AA, float *pot, float *nf) {
    potential_wca49_50_hst(sigma, dist_inv, invT, AA, *pot, *nf);
}
void ref_potential_wca49_50_AO_hst(float sigma, float dist_inv, float invT, float AA, float sigma_pol, float phi_pol,
                                   float *pot, float *nf) {
    potential_wca49_50_AO_hst(sigma, dist_inv, invT, AA, sigma_pol, phi_pol, *pot, *nf);
}
// calculate_color (colors.cu:64-110) of big particle mm: 0 blue, 1 green, 2 red;
// counts[0..2] = blue, green, red accumulate as in the reference
int ref_calculate_color(int mm, float *rr_big, float *rr_sml, int *counts, const parametros *p) {
    char color[20];
    calculate_color(mm, (float3 *)rr_big, (float3 *)rr_sml, color, counts[0], counts[1], counts[2], *p);
    return color[0] == 'R' ? 2 : (color[0] == 'G' ? 1 : 0);
}

}  // extern "C"

extern "C" {
/* The reference's host time loop, in the order of the HOST branches of
 * main.cu:509-574 (update_ermak_hst x2, temperature, set_vec_int_hst +
 * cell_locate_hst x2, set_vec_float*_hst, get_forces_same_hst x2,
 * get_forces_diff_hst x2).  The HOST driver itself does not compile
 * (main.cu:323); its functions do, and are called here unchanged.  Noise:
 * the GSL stand-in's own normals.  rb/rs are advanced in place; ff/vir/pot
 * are the caller's work arrays.  Returns 0. */
int ref_hst_run(const parametros *p_in, float *rb, float *rs, float *rawb, float *raws, float *ffb, float *ffs,
                float *vb, float *vs, float *pb, float *ps, int *nocup_b, int *cell_b, int *nocup_s, int *cell_s,
                long nsteps, long ni_start, float T0, float Tf, float t0, float tf, double dt, unsigned long seed) {
    parametros pars = *p_in;
    gsl_rng *r = gsl_rng_alloc(gsl_rng_mt19937);
    gsl_rng_set(r, seed);
    const int nb = pars.ngrain_big, ns = pars.ngrain_sml;
    const int ncb3 = pars.ncell_big * pars.ncell_big * pars.ncell_big;
    const int ncs3 = pars.ncell_sml * pars.ncell_sml * pars.ncell_sml;
    float3 zero; zero.x = zero.y = zero.z = 0.0f;
    for (long k = 0; k < nsteps; k++) {
        long ni = ni_start + k;
        update_ermak_hst('b', (float3 *)rb, (float3 *)rawb, (float3 *)ffb, r, pars);
        update_ermak_hst('s', (float3 *)rs, (float3 *)raws, (float3 *)ffs, r, pars);
        float time = dt * (1.0 + (float)ni);
        pars.temp_set = calculate_temp_linear(T0, Tf, t0, tf, time);
        set_vec_int_hst(nocup_b, ncb3, 0);
        set_vec_int_hst(cell_b, ncb3 * pars.ntags_big, -1);
        cell_locate_hst('b', (float3 *)rb, nocup_b, cell_b, pars);
        set_vec_int_hst(nocup_s, ncs3, 0);
        set_vec_int_hst(cell_s, ncs3 * pars.ntags_sml, -1);
        cell_locate_hst('s', (float3 *)rs, nocup_s, cell_s, pars);
        set_vec_float3_hst((float3 *)ffb, nb, zero);
        set_vec_float_hst(vb, nb, 0.0);
        set_vec_float_hst(pb, nb, 0.0);
        set_vec_float3_hst((float3 *)ffs, ns, zero);
        set_vec_float_hst(vs, ns, 0.0);
        set_vec_float_hst(ps, ns, 0.0);
        get_forces_same_hst('b', (float3 *)rb, (float3 *)ffb, vb, pb, nocup_b, cell_b, pars);
        get_forces_same_hst('s', (float3 *)rs, (float3 *)ffs, vs, ps, nocup_s, cell_s, pars);
        get_forces_diff_hst('b', 's', (float3 *)rb, (float3 *)ffb, (float3 *)rs, vb, pb, nocup_s, cell_s, pars);
        get_forces_diff_hst('s', 'b', (float3 *)rs, (float3 *)ffs, (float3 *)rb, vs, ps, nocup_b, cell_b, pars);
    }
    gsl_rng_free(r);
    return 0;
}
}  // extern "C"
