/* Implementation of the GSL stand-in declared in gsl_shim/gsl/gsl_shim_core.h.
 * Test infrastructure only (see the header).  Own code. */
#include "gsl_shim/gsl/gsl_shim_core.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static const gsl_rng_type shim_mt = {"mt19937 (shim: injected noise)"};
const gsl_rng_type *gsl_rng_mt19937 = &shim_mt;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *t) {
    (void)t;
    gsl_rng *r = (gsl_rng *)calloc(1, sizeof(gsl_rng));
    gsl_rng_set(r, 0);
    return r;
}
void gsl_rng_set(gsl_rng *r, unsigned long seed) {
    r->pos = 0;
    r->s = 0x9E3779B97F4A7C15ULL ^ (unsigned long long)seed;
    if (!r->s) r->s = 1;
    r->has_spare = 0;
}
/* xorshift64* (Vigna 2016) -> uniform in (-1, 1) */
static double shim_u11(gsl_rng *r) {
    r->s ^= r->s >> 12; r->s ^= r->s << 25; r->s ^= r->s >> 27;
    unsigned long long x = r->s * 2685821657736338717ULL;
    return ((double)(x >> 11) + 0.5) * (2.0 / 9007199254740992.0) - 1.0;
}
void gsl_rng_free(gsl_rng *r) { free(r); }
void gsl_shim_rng_set_noise(gsl_rng *r, const double *noise, long n) {
    r->noise = noise; r->n = n; r->pos = 0;
}
double gsl_ran_gaussian(gsl_rng *r, double sigma) {
    if (!r->noise) { /* Marsaglia polar method */
        if (r->has_spare) { r->has_spare = 0; return sigma * r->spare; }
        double u, v, q;
        do { u = shim_u11(r); v = shim_u11(r); q = u * u + v * v; } while (q >= 1.0 || q == 0.0);
        double f = sqrt(-2.0 * log(q) / q);
        r->spare = v * f; r->has_spare = 1;
        return sigma * u * f;
    }
    if (r->pos >= r->n) {
        fprintf(stderr, "gsl shim: injected noise buffer exhausted (%ld)\n", r->pos);
        abort();
    }
    return sigma * r->noise[r->pos++];
}

gsl_vector *gsl_vector_alloc(size_t n) {
    gsl_vector *v = (gsl_vector *)malloc(sizeof(gsl_vector));
    v->size = n; v->data = (double *)calloc(n ? n : 1, sizeof(double));
    return v;
}
void gsl_vector_free(gsl_vector *v) { if (v) { free(v->data); free(v); } }
double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i]; }
void gsl_vector_set(gsl_vector *v, size_t i, double x) { v->data[i] = x; }

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2) {
    gsl_matrix *m = (gsl_matrix *)malloc(sizeof(gsl_matrix));
    m->size1 = n1; m->size2 = n2;
    m->data = (double *)calloc(n1 * n2 ? n1 * n2 : 1, sizeof(double));
    return m;
}
void gsl_matrix_free(gsl_matrix *m) { if (m) { free(m->data); free(m); } }
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->size2 + j]; }
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x) { m->data[i * m->size2 + j] = x; }

/* One-sided (Hestenes) Jacobi SVD: A (M x N, M >= N) -> U (in A), S, V.
 * Columns are rotated pairwise until mutually orthogonal; singular values are
 * the final column norms, sorted in decreasing order like GSL's output. */
int gsl_linalg_SV_decomp(gsl_matrix *A, gsl_matrix *V, gsl_vector *S, gsl_vector *work) {
    (void)work;
    const size_t M = A->size1, N = A->size2;
    double *a = A->data, *v = V->data;
    for (size_t i = 0; i < N; i++)
        for (size_t j = 0; j < N; j++) v[i * N + j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (size_t p = 0; p + 1 < N; p++)
            for (size_t q = p + 1; q < N; q++) {
                double alpha = 0, beta = 0, gamma = 0;
                for (size_t i = 0; i < M; i++) {
                    double ap = a[i * N + p], aq = a[i * N + q];
                    alpha += ap * ap; beta += aq * aq; gamma += ap * aq;
                }
                if (gamma == 0.0) continue;
                double denom = sqrt(alpha * beta);
                if (denom == 0.0) continue;
                double c_off = fabs(gamma) / denom;
                if (c_off > off) off = c_off;
                if (c_off < 1e-15) continue;
                double zeta = (beta - alpha) / (2.0 * gamma);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
                for (size_t i = 0; i < M; i++) {
                    double ap = a[i * N + p], aq = a[i * N + q];
                    a[i * N + p] = c * ap - s * aq;
                    a[i * N + q] = s * ap + c * aq;
                }
                for (size_t i = 0; i < N; i++) {
                    double vp = v[i * N + p], vq = v[i * N + q];
                    v[i * N + p] = c * vp - s * vq;
                    v[i * N + q] = s * vp + c * vq;
                }
            }
        if (off < 1e-15) break;
    }
    double *sv = S->data;
    for (size_t j = 0; j < N; j++) {
        double nrm = 0;
        for (size_t i = 0; i < M; i++) nrm += a[i * N + j] * a[i * N + j];
        nrm = sqrt(nrm);
        sv[j] = nrm;
        if (nrm > 0)
            for (size_t i = 0; i < M; i++) a[i * N + j] /= nrm;
    }
    /* selection sort by decreasing singular value, permuting U and V columns */
    for (size_t j = 0; j < N; j++) {
        size_t best = j;
        for (size_t k = j + 1; k < N; k++) if (sv[k] > sv[best]) best = k;
        if (best != j) {
            double t = sv[j]; sv[j] = sv[best]; sv[best] = t;
            for (size_t i = 0; i < M; i++) { t = a[i * N + j]; a[i * N + j] = a[i * N + best]; a[i * N + best] = t; }
            for (size_t i = 0; i < N; i++) { t = v[i * N + j]; v[i * N + j] = v[i * N + best]; v[i * N + best] = t; }
        }
    }
    return 0;
}
