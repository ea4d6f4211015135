// extern "C" wrappers around the reference's own host functions, compiled
// from the reference sources by oracle/Makefile into oracle/_ref/libref.so.
// Test infrastructure: it lets the tests and the golden-vector script call
// the reference implementation itself (cell_locate_hst, get_forces_*_hst,
// update_ermak_hst, get_gder_hst, fself_isotropic, calculate_temp_*,
// sampling_indexes, Contracting_Vector3D) on chosen inputs.
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

}  // extern "C"
