/* Minimal stand-in for the parts of the GNU Scientific Library that the
 * reference sources name.  GSL is not installed in this image; the reference
 * reaches it only from host-only code (update_ermak_hst's gsl_rng and
 * Contracting_Vector3D::calculate_vector's SVD).  This shim lets those
 * translation units compile unmodified so that their host functions can be
 * run as the test oracle.  It is test infrastructure, never product code.
 *
 *  - gsl_rng / gsl_ran_gaussian: return sigma * (next value of an injected
 *    noise buffer), so that the reference update and the CUDA engine consume
 *    identical N(0,1) draws in parity tests.  Without a buffer the shim draws
 *    its own normals (xorshift64* + Marsaglia polar method) so that the
 *    reference's host time loop can be timed with its RNG cost included.
 *  - gsl_linalg_SV_decomp: one-sided Jacobi SVD in double (own code).  The
 *    reference only uses the pseudo-inverse V diag(1/w) U^T, which does not
 *    depend on the SVD algorithm beyond rounding.
 */
#ifndef BD_GSL_SHIM_CORE_H
#define BD_GSL_SHIM_CORE_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct { size_t size; double *data; } gsl_vector;
typedef struct { size_t size1, size2; double *data; } gsl_matrix;

typedef struct { const char *name; } gsl_rng_type;
typedef struct { const double *noise; long n, pos; unsigned long long s; int has_spare; double spare; } gsl_rng;

extern const gsl_rng_type *gsl_rng_mt19937;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *t);
void gsl_rng_set(gsl_rng *r, unsigned long seed);
void gsl_rng_free(gsl_rng *r);
double gsl_ran_gaussian(gsl_rng *r, double sigma);
/* shim-only: point a generator at a caller-owned buffer of N(0,1) values */
void gsl_shim_rng_set_noise(gsl_rng *r, const double *noise, long n);

gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x);

int gsl_linalg_SV_decomp(gsl_matrix *A, gsl_matrix *V, gsl_vector *S, gsl_vector *work);

#ifdef __cplusplus
}
#endif
#endif
