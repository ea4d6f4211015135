/*
 * oracle.c -- CPU restatement of the reference hot path.  TEST INFRASTRUCTURE:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline/reference
 * legs load it, always as the checker.  Compiled with -ffp-contract=off so
 * that every a*b+c rounds twice, as in the reference's host functions.
 *
 * Each or_ref_* function states which reference lines it follows and keeps
 * the reference's mix of float and double operations; the or_eng_* functions
 * restate the B200 engine's own arithmetic.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159266f   /* encabezados.h:25 (sic) */
#define OR_EPS 1.0f         /* encabezados.h:30 */

/* ------------------------------------------------------------------ params */
/* main.cu:155-163 (dt, temp, gder), 244-298 (cells, ranges), 348-349 (NH). */
void or_ref_setup_params(bd_parametros *p, float side, int nb, int ns, float sigma_big, float sigma_sml,
                         float mass_big, float mass_sml, int ntags_big, int ntags_sml, int nbins_gder,
                         float range_gder, double dt, float temp0) {
    memset(p, 0, sizeof(*p));
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
}

/* --------------------------------------------------------------- cell list */
/* cell_locate_hst, cell_locate.cu:46-104: inverse cell side computed as a
 * double division narrowed to float; (int) truncation; ==ncell clamp;
 * slots filled in ascending particle order.  Returns 1 when a cell reaches
 * ntags particles (the reference's overflow condition, cell_locate.cu:91-95
 * and main.cu:655), writing no slot beyond ntags. */
int or_ref_cell_locate(char type, const float *rr, int *nocup, int *cell_vec, const bd_parametros *p) {
    float csi;
    int n, ntags, ncell;
    if (type == 'b') { csi = (float)(1.0 / p->cell_side_big); n = p->ngrain_big; ntags = p->ntags_big; ncell = p->ncell_big; }
    else { csi = (float)(1.0 / p->cell_side_sml); n = p->ngrain_sml; ntags = p->ntags_sml; ncell = p->ncell_sml; }
    int nc3 = ncell * ncell * ncell, bad = 0;
    for (int c = 0; c < nc3; c++) nocup[c] = 0;
    for (long s = 0; s < (long)nc3 * ntags; s++) cell_vec[s] = -1;
    for (int m = 0; m < n; m++) {
        int ii = (int)(csi * rr[3 * m]), jj = (int)(csi * rr[3 * m + 1]), kk = (int)(csi * rr[3 * m + 2]);
        if (ii == ncell) ii--;
        if (jj == ncell) jj--;
        if (kk == ncell) kk--;
        int c = ii + ncell * (jj + ncell * kk);
        int shift = nocup[c]++;
        if (shift < ntags) cell_vec[c * ntags + shift] = m;
        if (shift + 1 >= ntags) bad = 1;
    }
    return bad;
}

/* ------------------------------------------------------------------ forces */
/* potential_wca_modified_hst, potentials.cu:66-76 */
static void wca_modified(float sigma, float dist_inv, float *potential, float *normal_force) {
    float sor = dist_inv * sigma;
    float sor6 = sor * sor * sor;
    sor6 = sor6 * sor6;
    float sor12 = sor6 * sor6;
    *potential += OR_EPS * (sor12 - 2 * sor6 + 1);
    *normal_force = -OR_EPS * 12 * (sor12 - sor6) * dist_inv;
}

/* Shared body of get_forces_same_hst (get_forces.cu:21-145) and
 * get_forces_diff_hst (get_forces.cu:149-277): one particle m against the
 * cells of the other set within +-nrange, float arithmetic. */
static void forces_sweep(const float *rrm_p, int m, int same, const float *rr_other, const int *nocup,
                         const int *cell_vec, int ncell, int ntags, int nrange, float csi, float sigma,
                         float side, float *ffm, float *virial, float *potential) {
    float cutoff = 1.0f * sigma, cutoff2 = cutoff * cutoff, side_inv = 1.0f / side;
    float rx = rrm_p[0], ry = rrm_p[1], rz = rrm_p[2];
    int ii = (int)(csi * rx), jj = (int)(csi * ry), kk = (int)(csi * rz);
    if (ii == ncell) ii--;
    if (jj == ncell) jj--;
    if (kk == ncell) kk--;
    for (int di = -nrange; di <= nrange; di++)
        for (int dj = -nrange; dj <= nrange; dj++)
            for (int dk = -nrange; dk <= nrange; dk++) {
                int iip = (ii + di + ncell) % ncell, jjp = (jj + dj + ncell) % ncell, kkp = (kk + dk + ncell) % ncell;
                int c = iip + ncell * (jjp + ncell * kkp);
                int occ = nocup[c];
                for (int t = 0; t < occ; t++) {
                    int nn = cell_vec[c * ntags + t];
                    if (same && nn == m) continue;
                    float dx = rr_other[3 * nn] - rx, dy = rr_other[3 * nn + 1] - ry, dz = rr_other[3 * nn + 2] - rz;
                    dx -= side * floorf(side_inv * dx + 0.5f);
                    dy -= side * floorf(side_inv * dy + 0.5f);
                    dz -= side * floorf(side_inv * dz + 0.5f);
                    float dist2 = dx * dx + dy * dy + dz * dz;
                    if (dist2 < cutoff2) {
                        float dist_inv = sqrtf(1.0f / dist2), nf;
                        wca_modified(sigma, dist_inv, potential, &nf);
                        float fx = nf * dist_inv * dx, fy = nf * dist_inv * dy, fz = nf * dist_inv * dz;
                        ffm[0] += fx; ffm[1] += fy; ffm[2] += fz;
                        *virial -= 0.5f * (dx * fx + dy * fy + dz * fz);
                    }
                }
            }
}

void or_ref_forces_same(char type, const float *rr, float *ff, float *vir, float *pot, const int *nocup,
                        const int *cell_vec, const bd_parametros *p) {
    int b = (type == 'b');
    float sigma = b ? p->sigma_big : p->sigma_sml;
    int n = b ? p->ngrain_big : p->ngrain_sml;
    float csi = 1.0f / (b ? p->cell_side_big : p->cell_side_sml);
    int ntags = b ? p->ntags_big : p->ntags_sml, ncell = b ? p->ncell_big : p->ncell_sml;
    int nrange = b ? p->nrange_bb : p->nrange_ss;
    for (int m = 0; m < n; m++)
        forces_sweep(rr + 3 * m, m, 1, rr, nocup, cell_vec, ncell, ntags, nrange, csi, sigma, p->side, ff + 3 * m,
                     vir + m, pot + m);
}

void or_ref_forces_diff(char type, char type_other, const float *rr, float *ff, const float *rr_other,
                        float *vir, float *pot, const int *nocup_o, const int *cell_o, const bd_parametros *p) {
    (void)type_other;
    int b = (type == 'b');
    int n = b ? p->ngrain_big : p->ngrain_sml;
    float csi = 1.0f / (b ? p->cell_side_sml : p->cell_side_big);
    float sigma = b ? 0.5f * (p->sigma_big + p->sigma_sml) : 0.5f * (p->sigma_sml + p->sigma_big);
    int ntags = b ? p->ntags_sml : p->ntags_big, ncell = b ? p->ncell_sml : p->ncell_big;
    int nrange = b ? p->nrange_bs : p->nrange_sb;
    for (int m = 0; m < n; m++)
        forces_sweep(rr + 3 * m, m, 0, rr_other, nocup_o, cell_o, ncell, ntags, nrange, csi, sigma, p->side,
                     ff + 3 * m, vir + m, pot + m);
}

/* ------------------------------------------------------------------ update */
/* update_ermak_hst, update_ermak.cu:8-77 with noise[3m+k] in place of the
 * three gsl_ran_gaussian draws.  amplitude in double, narrowed to float. */
void or_ref_update_ermak(char type, float *rr, float *rr_raw, const float *ff, const float *noise,
                         const bd_parametros *p) {
    float side = p->side, side_inv = 1.0f / side, temperature = p->temp_set, dt = p->dt;
    int n = (type == 'b') ? p->ngrain_big : p->ngrain_sml;
    float diameter = (type == 'b') ? p->sigma_big : p->sigma_sml;
    float dinv = 1.0f / diameter;
    float amplitude = (float)sqrt(2.0 * temperature * dinv * dt);
    for (int m = 0; m < n; m++) {
        for (int k = 0; k < 3; k++) {
            float rnd = (float)(amplitude * (double)noise[3 * m + k]);
            float tot = ff[3 * m + k] * dinv * dt + rnd;
            float r = rr[3 * m + k] + tot;
            rr_raw[3 * m + k] = rr_raw[3 * m + k] + tot;
            r -= side * floorf(side_inv * r);
            rr[3 * m + k] = r;
        }
    }
}

/* -------------------------------------------------------------------- g(r) */
/* get_gder_hst, get_gder.cu:7-63: ordered pairs (skipping m==n for the same
 * species), side_inv = (float)(1.0/side), floorf(side_inv*d + 0.5) with the
 * 0.5 added in double, float sqrt, bin = (int)(dist/bin_size), ==nbins clamp.
 * counts[nbins] are exact integers (the reference adds 1.0f per pair). */
void or_ref_gder_counts(char type, char type_other, const float *rr, const float *rr_other, uint64_t *counts,
                        const bd_parametros *p) {
    int n = (type == 'b') ? p->ngrain_big : p->ngrain_sml;
    int no = (type_other == 'b') ? p->ngrain_big : p->ngrain_sml;
    float side = p->side, range = p->range_gder;
    int nbins = p->nbins_gder;
    float side_inv = (float)(1.0 / side);
    float bin_size = range / ((float)nbins);
    for (int m = 0; m < n; m++)
        for (int j = 0; j < no; j++) {
            if (type == type_other && m == j) continue;
            float dx = rr[3 * m] - rr_other[3 * j], dy = rr[3 * m + 1] - rr_other[3 * j + 1],
                  dz = rr[3 * m + 2] - rr_other[3 * j + 2];
            dx -= side * floorf((float)((double)(side_inv * dx) + 0.5));
            dy -= side * floorf((float)((double)(side_inv * dy) + 0.5));
            dz -= side * floorf((float)((double)(side_inv * dz) + 0.5));
            float dist = sqrtf(dx * dx + dy * dy + dz * dz);
            if (dist < range) {
                int bin = (int)(dist / bin_size);
                if (bin == nbins) bin--;
                counts[bin]++;
            }
        }
}

/* main.cu:847-877: shell volume 4 PI dr^3 (1/3 + n^2 + n) in double narrowed
 * to float, free volume V - 4/3 PI sigma^3, pair densities, then / n_configs.
 * counts: [4][nbins] totals over configs; gder out [4][nbins]. */
void or_ref_gder_normalize(const double *counts, int nbins, float bin_size, float side, int nb, int ns,
                           float sigma_big, float sigma_sml, int n_configs, float *gder) {
    float volume = side * side * side;
    float xb = (float)nb, xs = (float)ns;
    for (int k = 0; k < nbins; k++) {
        float xnb = (float)k;
        float shell_vol = (float)(4.0 * OR_PI * bin_size * bin_size * bin_size * ((1.0 / 3.0) + xnb * xnb + xnb));
        float g[4];
        for (int j = 0; j < 4; j++) g[j] = (float)counts[j * nbins + k];
        float sigma = sigma_big;
        float vol_free = (float)(volume - (4.0 / 3.0) * OR_PI * sigma * sigma * sigma);
        g[0] = g[0] / shell_vol;
        g[0] = (float)(g[0] / (xb * (xb - 1.0) / vol_free));
        sigma = (float)(0.5 * (sigma_big + sigma_sml));
        vol_free = (float)(volume - (4.0 / 3.0) * OR_PI * sigma * sigma * sigma);
        g[1] = g[1] / shell_vol;
        g[2] = g[2] / shell_vol;
        g[1] /= (xb * xs / vol_free);
        g[2] /= (xs * xb / vol_free);
        sigma = sigma_sml;
        vol_free = (float)(volume - (4.0 / 3.0) * OR_PI * sigma * sigma * sigma);
        g[3] = g[3] / shell_vol;
        g[3] = (float)(g[3] / (xs * (xs - 1.0) / vol_free));
        for (int j = 0; j < 4; j++) gder[j * nbins + k] = g[j] / n_configs;
    }
}

/* ------------------------------------------------------------ observables */
/* fself_isotropic, fself.cu:3-21 (float sum, sinf). */
void or_ref_fself(const float *rr_raw, const float *rr0, int n, float *fself, int sample_number, float qmax) {
    float sum = 0.0f;
    for (int i = 0; i < n; i++) {
        float dx = rr_raw[3 * i] - rr0[3 * i], dy = rr_raw[3 * i + 1] - rr0[3 * i + 1], dz = rr_raw[3 * i + 2] - rr0[3 * i + 2];
        float mag = sqrtf(dx * dx + dy * dy + dz * dz);
        sum += sinf(qmax * mag) / (qmax * mag);
    }
    sum /= n;
    fself[sample_number] += sum;
}
/* main.cu:776-792 */
float or_ref_msd(const float *rr_raw, const float *rr0, int n) {
    float msd = 0.0f;
    for (int i = 0; i < n; i++) {
        float dx = rr_raw[3 * i] - rr0[3 * i], dy = rr_raw[3 * i + 1] - rr0[3 * i + 1], dz = rr_raw[3 * i + 2] - rr0[3 * i + 2];
        msd += dx * dx + dy * dy + dz * dz;
    }
    return msd / (float)n;
}
/* main.cu:627-631: float accumulator, 0.5*pot added in double each time. */
float or_ref_energy(const float *pot, int n) {
    float e = 0.0f;
    for (int i = 0; i < n; i++) e = (float)(e + 0.5 * pot[i]);
    return e / (float)n;
}
/* main.cu:801-804 */
float or_ref_pressure_z(const float *vir_b, int nb, const float *vir_s, int ns, float temp) {
    float virial = 0.0f;
    for (int i = 0; i < nb; i++) virial += vir_b[i];
    for (int i = 0; i < ns; i++) virial += vir_s[i];
    float xt = (float)(nb + ns);
    return (float)(1.0 + virial / (3.0 * xt * temp));
}

/* ------------------------------------------------------------- schedules */
/* set_temp.cu:7-12 */
float or_ref_temp_linear(float T0, float Tf, float t0, float tf, float t) {
    if (t < t0) return T0;
    if (t > tf) return Tf;
    float m = (Tf - T0) / (tf - t0);
    return T0 + m * (t - t0);
}
/* set_temp.cu:14-23 */
float or_ref_temp_sine(float T0, float Tf, float t0, float tf, float period, float t) {
    if (t < t0) return T0;
    if (t > tf) return Tf;
    float a = (float)(0.5 * (T0 + Tf));
    float b = (float)(0.5 * (Tf - T0));
    float argument = (float)(2 * OR_PI * (t / period - 0.25));
    return a + b * sinf(argument);
}
/* main.cu:520: time = dt * (1.0 + (float) ni), double product narrowed. */
float or_ref_time_of_step(double dt, int ni) { return (float)(dt * (1.0 + (float)ni)); }

/* log_sampling / sampling_indexes, main.cu:14-53 (float arguments). */
int or_ref_sampling_indexes(float minimal_decade, float run_time, float dt, int per_decade, int *out, int cap) {
    int last_power = (int)roundf(log10f(run_time));
    int initial_power = (int)roundf(log10f(minimal_decade));
    int decades = last_power - initial_power;
    float values[1024];
    float r = powf(10.0f, 1.0f / per_decade), x = 1.0f;
    for (int i = 0; i <= per_decade && i < 1024; i++) { values[i] = x; x *= r; }
    int total = decades * per_decade;
    int cnt = 0;
    if (cap > 0) out[0] = 0;
    for (int ipow = initial_power; ipow < last_power; ++ipow) {
        float power = (float)pow(10.0, (double)ipow);
        for (int j = 0; j < per_decade; ++j) {
            float scaled = values[j] * power;
            int index = (int)roundf(scaled / dt);
            cnt++;
            if (cnt < cap) out[cnt] = index;
        }
    }
    (void)total;
    return cnt + 1;
}

/* rannew64.cu:55-126: subtractive lagged Fibonacci (250, 103) minus a 64-bit
 * LCG, both mod 2^64, seeded by 1000+250 steps of a second LCG. */
void or_rannew64_seed(or_rannew64_state *s, long idum) {
    if (idum < 0) idum = -idum;
    uint64_t udum = (uint64_t)idum;
    const uint64_t uaa = 6364136223846793005ULL, ucc = 1442695040888963407ULL;
    for (int i = 0; i < 1000; i++) udum = udum * uaa + ucc;
    for (int i = 0; i < 250; i++) { udum = udum * uaa + ucc; s->useed[i] = udum; }
    s->uuy = udum;
    s->np = 249; s->nq = 102; s->init = 1;
}
double or_rannew64_next(or_rannew64_state *s) {
    const uint64_t ua = 2862933555777941757ULL, uc = 3037000493ULL;
    uint64_t uux = s->useed[s->np] - s->useed[s->nq];
    s->useed[s->np] = uux;
    s->np--; s->nq--;
    if (s->np < 0) s->np = 249;
    if (s->nq < 0) s->nq = 249;
    s->uuy = ua * s->uuy + uc;
    uint64_t uu = uux - s->uuy;
    double omm = 1. / 18446744073709551615.;
    return omm * ((double)uu);
}

/* Gaussians of the engine's per-particle rannew64 mode: particle p uses
 * rannew64 seeded with idum = seed + p; each step takes 4 uniforms (double,
 * narrowed to float) and applies Box-Muller on (u0, u1) -> x, y and
 * (u2, u3) -> z.  noise[(s * n + p) * 3 + k]. */
void or_rannew64_particle_noise(long long seed, int n, int steps, float *noise) {
    or_rannew64_state st;
    for (int p = 0; p < n; p++) {
        or_rannew64_seed(&st, (long)(seed + p));
        for (int s = 0; s < steps; s++) {
            float u[4];
            for (int k = 0; k < 4; k++) u[k] = (float)or_rannew64_next(&st);
            const float tiny = 1.17549435e-38f;
            float r0 = sqrtf(-2.0f * logf(u[0] > tiny ? u[0] : tiny));
            float r1 = sqrtf(-2.0f * logf(u[2] > tiny ? u[2] : tiny));
            float t0 = 6.2831853f * u[1], t1 = 6.2831853f * u[3];
            float *o = noise + ((size_t)s * n + p) * 3;
            o[0] = r0 * cosf(t0);
            o[1] = r0 * sinf(t0);
            o[2] = r1 * cosf(t1);
        }
    }
}

/* Contracting_Vector3D::add_statistics, Contracting_Vector3D.cu:57-164, float
 * arithmetic; the periodic image uses floor() of the double sum
 * side_inv*d + 0.5 (Contracting_Vector3D.cu:101-105). */
int or_ref_cv3d_add(int bins, float range, const float *rr, const float *xx, int n, float side, float *ata,
                    float *atb) {
    float bin_size = range / (float)bins;
    float bin_size_inv = 1.0f / ((float)bin_size);
    float range_square = range * range;
    float side_inv = side > 0 ? 1.0f / side : 0.0f;
    float *hit = (float *)calloc((size_t)bins * 3, sizeof(float));
    int bad = 0;
    for (int m = 0; m < n; m++) {
        int neighs = 0;
        for (int j = 0; j < n; j++) {
            if (j == m) continue;
            float dx = rr[3 * m] - rr[3 * j], dy = rr[3 * m + 1] - rr[3 * j + 1], dz = rr[3 * m + 2] - rr[3 * j + 2];
            if (side > 0) {
                dx -= side * (float)floor(side_inv * dx + 0.5);
                dy -= side * (float)floor(side_inv * dy + 0.5);
                dz -= side * (float)floor(side_inv * dz + 0.5);
            }
            float dist2 = dx * dx + dy * dy + dz * dz;
            if (dist2 < range_square) {
                float dist = sqrtf(dist2);
                int nb = (int)(bin_size_inv * dist);
                if (nb >= bins) nb = bins - 1; /* reference writes hit_vec[bins] here (out of bounds) */
                hit[3 * nb] += dx / dist;
                hit[3 * nb + 1] += dy / dist;
                hit[3 * nb + 2] += dz / dist;
                neighs++;
                if (neighs == 10000) bad = 1;
            }
        }
        if (neighs > 0) {
            for (int c = 0; c < 3; c++)
                for (int i = 0; i < bins; i++)
                    for (int j = 0; j <= i; j++) {
                        float aux = hit[3 * i + c] * hit[3 * j + c];
                        ata[(size_t)c * bins * bins + (size_t)i * bins + j] += aux;
                        if (i != j) ata[(size_t)c * bins * bins + (size_t)j * bins + i] += aux;
                    }
            for (int i = 0; i < bins; i++)
                for (int c = 0; c < 3; c++) atb[c * bins + i] += hit[3 * i + c] * xx[3 * m + c];
            memset(hit, 0, (size_t)bins * 3 * sizeof(float));
        }
    }
    free(hit);
    return bad;
}

/* ================================================================ engine */
void or_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
void or_eng_uniform_bits(uint64_t seed, uint32_t id, uint64_t step, uint32_t stream, uint32_t out[4]) {
    uint32_t ctr[4] = {id, (uint32_t)step, (uint32_t)(step >> 32), stream};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    or_philox4x32_10(ctr, key, out);
}
/* uniform in (0,1): (x >> 9) * 2^-23 + 2^-24 (exact in float) */
static double u01(uint32_t x) { return (double)(x >> 9) * (1.0 / 8388608.0) + (1.0 / 16777216.0); }
void or_eng_gauss3(uint64_t seed, uint32_t id, uint64_t step, uint32_t stream, double out[3]) {
    uint32_t b[4];
    or_eng_uniform_bits(seed, id, step, stream, b);
    double r0 = sqrt(-2.0 * log(u01(b[0]))), r1 = sqrt(-2.0 * log(u01(b[2])));
    double a0 = 2.0 * M_PI * u01(b[1]), a1 = 2.0 * M_PI * u01(b[3]);
    out[0] = r0 * cos(a0);
    out[1] = r0 * sin(a0);
    out[2] = r1 * cos(a1);
}

/* Engine pair force: same pair arithmetic as the reference (float, minimum
 * image d -= L floor(d/L + 1/2)), per-species-pair cut distance
 * s_ab = (s_a + s_b)/2 for a != b, sums in ascending partner index. */
void or_eng_forces(int n, const float *pos, const int *type, float side, const float sigma[2], float *ff,
                   float *pot, float *vir, int *nbr, uint64_t *nbr_hash) {
    float side_inv = 1.0f / side;
    float sig[2][2];
    sig[0][0] = sigma[0]; sig[1][1] = sigma[1];
    sig[0][1] = sig[1][0] = 0.5f * (sigma[0] + sigma[1]);
    for (int m = 0; m < n; m++) {
        float fx = 0, fy = 0, fz = 0, pm = 0, vm = 0;
        int cnt = 0;
        uint64_t h = 0;
        for (int j = 0; j < n; j++) {
            if (j == m) continue;
            float s = sig[type[m]][type[j]], c2 = s * s;
            float dx = pos[3 * j] - pos[3 * m], dy = pos[3 * j + 1] - pos[3 * m + 1], dz = pos[3 * j + 2] - pos[3 * m + 2];
            dx -= side * floorf(side_inv * dx + 0.5f);
            dy -= side * floorf(side_inv * dy + 0.5f);
            dz -= side * floorf(side_inv * dz + 0.5f);
            float d2 = dx * dx + dy * dy + dz * dz;
            if (d2 < c2) {
                float di = sqrtf(1.0f / d2), nf;
                wca_modified(s, di, &pm, &nf);
                float px = nf * di * dx, py = nf * di * dy, pz = nf * di * dz;
                fx += px; fy += py; fz += pz;
                vm -= 0.5f * (dx * px + dy * py + dz * pz);
                cnt++;
                h += ((uint64_t)(j + 1)) * 0x9E3779B97F4A7C15ULL;
            }
        }
        ff[3 * m] = fx; ff[3 * m + 1] = fy; ff[3 * m + 2] = fz;
        if (pot) pot[m] = pm;
        if (vir) vir[m] = vm;
        if (nbr) nbr[m] = cnt;
        if (nbr_hash) nbr_hash[m] = h;
    }
}

/* Force cap of the initial relaxation (the reference ships no generator,
 * run-fself.sh:84-86; the engine relaxes random placements with capped
 * forces): a force whose magnitude exceeds fcap is scaled to magnitude fcap
 * along its direction, computed as g = F / max|F_k|, |g|, F' = g * (fcap / |g|);
 * a force with a non-finite component (an overlap so deep that the pair
 * force overflows) becomes zero.  In place on ff[3n]. */
void or_eng_cap_forces(int n, float *ff, float fcap) {
    for (int m = 0; m < n; m++) {
        float *f = ff + 3 * m;
        float fmx = fmaxf(fabsf(f[0]), fmaxf(fabsf(f[1]), fabsf(f[2])));
        if (fmx > 0.0f && isfinite(fmx)) {
            float gx = f[0] / fmx, gy = f[1] / fmx, gz = f[2] / fmx;
            float ng = sqrtf(gx * gx + gy * gy + gz * gz);
            if (fmx * ng > fcap) {
                float sc = fcap / ng;
                f[0] = gx * sc;
                f[1] = gy * sc;
                f[2] = gz * sc;
            }
        } else if (!isfinite(fmx)) {
            f[0] = f[1] = f[2] = 0.0f;
        }
    }
}

/* amplitude of the random displacement, update_ermak.cu:114 with the
 * mobility mob in place of 1/sigma: (float) sqrt(2.0 * T * mob * dt). */
float or_eng_amplitude(float temp, float mob, float dt) { return (float)sqrt(2.0 * temp * mob * dt); }

/* Engine update.  Displacement d = (F*mob)*dt + amp*xi (float, two
 * roundings per product as in the reference), then the position pair
 * (hi, lo) absorbs d exactly (Knuth TwoSum + renormalisation), the periodic
 * wrap subtracts L*floor(hi/L) the same way, and dsp += (double)d. */
static void two_sum(float a, float b, float *s, float *e) {
    float ss = a + b, bp = ss - a;
    *e = (a - (ss - bp)) + (b - bp);
    *s = ss;
}
void or_eng_update(int n, float *hi, float *lo, double *dsp, const float *ff, const int *type, float side,
                   double dt_d, const float mob[2], const float amp[2], const float *noise) {
    float dt = (float)dt_d, side_inv = 1.0f / side;
    for (int m = 0; m < n; m++) {
        int t = type[m];
        for (int k = 0; k < 3; k++) {
            float d = ff[3 * m + k] * mob[t] * dt + amp[t] * noise[3 * m + k];
            float s, e;
            two_sum(hi[3 * m + k], d, &s, &e);
            float c = lo[3 * m + k] + e;
            float h2 = s + c;
            c = c - (h2 - s);
            float kw = floorf(side_inv * h2);
            if (kw != 0.0f) {
                float s2, e2;
                two_sum(h2, -(side * kw), &s2, &e2);
                c = c + e2;
                h2 = s2 + c;
                c = c - (h2 - s2);
            }
            hi[3 * m + k] = h2;
            lo[3 * m + k] = c;
            dsp[3 * m + k] += (double)d;
        }
    }
}

void or_eng_fself_msd(int n, const double *d, double q, double *fs, double *msd) {
    double sf = 0, sm = 0;
    for (int i = 0; i < n; i++) {
        double r2 = d[3 * i] * d[3 * i] + d[3 * i + 1] * d[3 * i + 1] + d[3 * i + 2] * d[3 * i + 2];
        double r = sqrt(r2);
        sm += r2;
        sf += (r > 0) ? sin(q * r) / (q * r) : 1.0;
    }
    *fs = sf / n;
    *msd = sm / n;
}

/* ------------------------------------------------------------------------
 * Precision study (FP32 + compensated positions and FP64 displacements vs
 * an FP64 run and a run at the reference's FP32 precision).  All three use
 * the engine's Philox noise (or_eng_gauss3 of seed, particle index, step,
 * stream), the same WCA pair (potentials.cu:137-147 with per-species-pair
 * cut distances) and the update d = F mob dt + amp xi (update_ermak.cu:
 * 122-141); they differ only in arithmetic.  Forces use a cell list (cell
 * side >= the largest cut distance) or all pairs when the box holds fewer
 * than 3 cells.  obs: msd_big, msd_sml, fself_big(q), energy_big,
 * energy_sml (0.5 sum pot / N), virial (sum vir_i).  dsp_out: [3n]
 * unwrapped displacement. */
typedef struct { int nc; int *head, *next, *cell; } or_cells;

static void cells_build_d(or_cells *c, int n, const double *pos, double side, double rcmax) {
    c->nc = (int)floor(side / rcmax);
    if (c->nc < 3) { c->nc = 0; return; }
    int nc3 = c->nc * c->nc * c->nc;
    for (int i = 0; i < nc3; i++) c->head[i] = -1;
    for (int m = 0; m < n; m++) {
        int ix[3];
        for (int k = 0; k < 3; k++) {
            ix[k] = (int)(pos[3 * m + k] / side * c->nc);
            if (ix[k] < 0) ix[k] = 0;
            if (ix[k] >= c->nc) ix[k] = c->nc - 1;
        }
        int ci = ix[0] + c->nc * (ix[1] + c->nc * ix[2]);
        c->cell[m] = ci;
        c->next[m] = c->head[ci];
        c->head[ci] = m;
    }
}

static void pair_d(double s, double dx, double dy, double dz, double *f, double *pot, double *vir) {
    double d2 = dx * dx + dy * dy + dz * dz;
    if (!(d2 < s * s)) return;
    double di = 1.0 / sqrt(d2), sor = s * di, s6 = sor * sor * sor;
    s6 *= s6;
    double s12 = s6 * s6, nf = -12.0 * (s12 - s6) * di;
    *pot += s12 - 2.0 * s6 + 1.0;
    double px = nf * di * dx, py = nf * di * dy, pz = nf * di * dz;
    f[0] += px; f[1] += py; f[2] += pz;
    *vir -= 0.5 * (dx * px + dy * py + dz * pz);
}

static void forces_d(int n, int n_big, const double *pos, double side, const double sig[3], or_cells *c, double *ff,
                     double *pot, double *vir) {
    double rcmax = sig[0] > sig[2] ? sig[0] : sig[2];
    if (sig[1] > rcmax) rcmax = sig[1];
    cells_build_d(c, n, pos, side, rcmax * (1.0 + 1e-9));
    const double half = 0.5 * side;  /* positions lie in [0, side): one image shift at most */
    for (int m = 0; m < n; m++) {
        double f[3] = {0, 0, 0}, pm = 0, vm = 0;
        int tm = m >= n_big;
        if (c->nc) {
            int nc = c->nc, ci = c->cell[m];
            int cx = ci % nc, cy = (ci / nc) % nc, cz = ci / (nc * nc);
            for (int oz = -1; oz <= 1; oz++)
                for (int oy = -1; oy <= 1; oy++)
                    for (int ox = -1; ox <= 1; ox++) {
                        int gx = (cx + ox + nc) % nc, gy = (cy + oy + nc) % nc, gz = (cz + oz + nc) % nc;
                        for (int j = c->head[gx + nc * (gy + nc * gz)]; j >= 0; j = c->next[j]) {
                            if (j == m) continue;
                            double d[3];
                            for (int k = 0; k < 3; k++) {
                                d[k] = pos[3 * j + k] - pos[3 * m + k];
                                if (d[k] > half) d[k] -= side;
                                else if (d[k] < -half) d[k] += side;
                            }
                            pair_d(sig[tm + (j >= n_big)], d[0], d[1], d[2], f, &pm, &vm);
                        }
                    }
        } else {
            for (int j = 0; j < n; j++) {
                if (j == m) continue;
                double d[3];
                for (int k = 0; k < 3; k++) {
                    d[k] = pos[3 * j + k] - pos[3 * m + k];
                    d[k] -= side * floor(d[k] / side + 0.5);
                }
                pair_d(sig[tm + (j >= n_big)], d[0], d[1], d[2], f, &pm, &vm);
            }
        }
        ff[3 * m] = f[0]; ff[3 * m + 1] = f[1]; ff[3 * m + 2] = f[2];
        pot[m] = pm;
        vir[m] = vm;
    }
}

static void observables_d(int n, int n_big, const double *dsp, const double *pot, const double *vir, double q,
                          double *obs) {
    double msd[2] = {0, 0}, fs = 0, e[2] = {0, 0}, w = 0;
    for (int m = 0; m < n; m++) {
        int t = m >= n_big;
        double r2 = dsp[3 * m] * dsp[3 * m] + dsp[3 * m + 1] * dsp[3 * m + 1] + dsp[3 * m + 2] * dsp[3 * m + 2];
        msd[t] += r2;
        if (!t) {
            double qr = q * sqrt(r2);
            fs += qr > 0 ? sin(qr) / qr : 1.0;
        }
        e[t] += 0.5 * pot[m];
        w += vir[m];
    }
    int ns = n - n_big;
    obs[0] = n_big ? msd[0] / n_big : 0;
    obs[1] = ns ? msd[1] / ns : 0;
    obs[2] = n_big ? fs / n_big : 0;
    obs[3] = n_big ? e[0] / n_big : 0;
    obs[4] = ns ? e[1] / ns : 0;
    obs[5] = w;
}

static int cells_alloc(or_cells *c, int n, double side, double rcmax) {
    int nc = (int)floor(side / rcmax);
    size_t nc3 = nc >= 3 ? (size_t)nc * nc * nc : 1;
    c->head = (int *)malloc(sizeof(int) * nc3);
    c->next = (int *)malloc(sizeof(int) * n);
    c->cell = (int *)malloc(sizeof(int) * n);
    return c->head && c->next && c->cell;
}
static void cells_free(or_cells *c) { free(c->head); free(c->next); free(c->cell); }

/* mode 0: FP64 everything.  mode 1: reference precision: float positions
 * (wrapped with side_inv = 1/side in float) and float unwrapped positions
 * rr_raw, float displacement d = (F mob) dt + amp xi with float forces from
 * the FP64 pair routine rounded to float, float amp (update_ermak.cu:114). */
int or_precision_run(int mode, int n, int n_big, const float *pos0, double side, double sig_big, double sig_sml,
                     double mob_big, double mob_sml, double dt, double temp, uint64_t seed, uint32_t stream,
                     long long ni0, int steps, double q, double *obs, double *dsp_out) {
    double sig[3] = {sig_big, 0.5 * (sig_big + sig_sml), sig_sml};
    double *pos = (double *)malloc(sizeof(double) * 3 * n), *ff = (double *)malloc(sizeof(double) * 3 * n);
    double *pot = (double *)malloc(sizeof(double) * n), *vir = (double *)malloc(sizeof(double) * n);
    double *dsp = (double *)calloc(3 * (size_t)n, sizeof(double));
    float *rr = (float *)malloc(sizeof(float) * 3 * n), *raw = (float *)malloc(sizeof(float) * 3 * n);
    or_cells c;
    double rcmax = sig_big > sig_sml ? sig_big : sig_sml;
    if (!pos || !ff || !pot || !vir || !dsp || !rr || !raw || !cells_alloc(&c, n, side, rcmax * (1.0 + 1e-9))) return 1;
    for (int i = 0; i < 3 * n; i++) { pos[i] = pos0[i]; rr[i] = pos0[i]; raw[i] = pos0[i]; }
    const float fside = (float)side, fside_inv = 1.0f / fside, fdt = (float)dt;
    for (int s = 0; s < steps; s++) {
        if (mode == 1)
            for (int i = 0; i < 3 * n; i++) pos[i] = rr[i];
        forces_d(n, n_big, pos, side, sig, &c, ff, pot, vir);
        long long ni = ni0 + s;
        for (int m = 0; m < n; m++) {
            int t = m >= n_big;
            double mob = t ? mob_sml : mob_big, xi[3];
            or_eng_gauss3(seed, (uint32_t)m, (uint64_t)ni, stream, xi);
            if (mode == 0) {
                double amp = sqrt(2.0 * temp * mob * dt);
                for (int k = 0; k < 3; k++) {
                    double d = ff[3 * m + k] * mob * dt + amp * xi[k];
                    pos[3 * m + k] += d;
                    pos[3 * m + k] -= side * floor(pos[3 * m + k] / side);
                    dsp[3 * m + k] += d;
                }
            } else {
                float amp = (float)sqrt(2.0 * temp * (double)(float)mob * dt), fm = (float)mob;
                for (int k = 0; k < 3; k++) {
                    float d = (float)ff[3 * m + k] * fm * fdt + amp * (float)xi[k];
                    rr[3 * m + k] += d;
                    raw[3 * m + k] += d;
                    rr[3 * m + k] -= fside * floorf(fside_inv * rr[3 * m + k]);
                }
            }
        }
    }
    if (mode == 1)
        for (int i = 0; i < 3 * n; i++) {
            pos[i] = rr[i];
            dsp[i] = (double)(raw[i] - pos0[i]);
        }
    forces_d(n, n_big, pos, side, sig, &c, ff, pot, vir);
    observables_d(n, n_big, dsp, pot, vir, q, obs);
    if (dsp_out) memcpy(dsp_out, dsp, sizeof(double) * 3 * n);
    cells_free(&c);
    free(pos); free(ff); free(pot); free(vir); free(dsp); free(rr); free(raw);
    return 0;
}

/* ------------------------------------------------------------------------
 * Colour statistics of the snapshot writer (colors.cu:8-110, main.cu:
 * 663-713): a big particle is Blue without big neighbours (squared distance
 * compared with sigma_b + 2 sigma_s, as written), else Red when more of its
 * neighbour pairs have a small particle "between" them than not, else Green.
 * Float arithmetic in the reference's order; ids: 0 blue, 1 green, 2 red. */
static float min_image_ref(float d, float side, float side_inv) { return d - side * floorf(side_inv * d + 0.5f); }

static int between_ref(const float *r1, const float *r2, const float *rs, int ns, float side, float sigma_big,
                       float sigma_sml) {
    float max_big = (float)(0.5 * sigma_big + 2.0 * sigma_sml);
    float max_line = (float)(0.35 * sigma_big);
    float side_inv = 1 / side;
    float u[3];
    for (int k = 0; k < 3; k++) u[k] = min_image_ref(r1[k] - r2[k], side, side_inv);
    float ua = sqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    for (int k = 0; k < 3; k++) u[k] /= ua;
    for (int i = 0; i < ns; i++) {
        const float *r = rs + 3 * i;
        float d1[3], d2[3];
        for (int k = 0; k < 3; k++) d1[k] = min_image_ref(r[k] - r1[k], side, side_inv);
        float n1 = sqrtf(d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
        if (n1 > max_big) continue;
        for (int k = 0; k < 3; k++) d2[k] = min_image_ref(r[k] - r2[k], side, side_inv);
        float n2 = sqrtf(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]);
        if (n2 > max_big) continue;
        float cx = d1[1] * u[2] - d1[2] * u[1], cy = -d1[0] * u[2] + d1[2] * u[0], cz = d1[0] * u[1] - d1[1] * u[0];
        float dl = sqrtf(cx * cx + cy * cy + cz * cz);
        if (dl > max_line) continue;
        return 1;
    }
    return 0;
}

void or_ref_colors(int nb, int ns, const float *rb, const float *rs, float side, float sigma_big, float sigma_sml,
                   int *ids, int counts[3]) {
    float side_inv = (float)(1.0 / side);
    counts[0] = counts[1] = counts[2] = 0;
    for (int m = 0; m < nb; m++) {
        int cid = 0, near = 0;
        for (int n = 0; n < nb; n++) {
            if (n == m) continue;
            float d[3];
            for (int k = 0; k < 3; k++) d[k] = min_image_ref(rb[3 * n + k] - rb[3 * m + k], side, side_inv);
            float dist = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (dist > sigma_big + 2.0 * sigma_sml) continue;
            between_ref(rb + 3 * m, rb + 3 * n, rs, ns, side, sigma_big, sigma_sml) ? cid++ : cid--;
            near = 1;
        }
        int id = near ? (cid > 0 ? 2 : 1) : 0;
        ids[m] = id;
        counts[id]++;
    }
}

/* ------------------------------------------------------------------------
 * Pair potentials of potentials.cu that the reference never calls (host
 * float formulas as written, EPS = 1): *pot accumulates, *nf = normal force
 * (dU/dr).  pot: 1 wca, 2 wca49_50, 3 AO, 4 HSAY (the intended form: ros = r/s,
 * energies added, dU/dr).  pp = {invT, AA, sigma_pol, phi_pol} or {z, cut}. */
void or_pair_extra(int pot, const float *pp, float sigma, float dist_inv, float *u, float *nf) {
    float sor = dist_inv * sigma;
    if (pot == 1) {
        float s6 = sor * sor * sor;
        s6 = s6 * s6;
        float s12 = s6 * s6;
        *u += 4 * (s12 - s6) + 1;
        *nf = -4 * (12 * s12 - 6 * s6) * dist_inv;
        return;
    }
    float ros_ao = (float)(1.0 / sor);
    if (pot == 2 || (pot == 3 && ros_ao <= 1.0)) {
        float invT = pp[0], AA = pp[1];
        float s6;
        if (pot == 2) {  /* potential_wca49_50_hst: (s^3)^2 */
            s6 = sor * sor * sor;
            s6 = s6 * s6;
        } else {         /* potential_wca49_50_AO_hst: s s s s s s */
            s6 = sor * sor * sor * sor * sor * sor;
        }
        float s12 = s6 * s6, s24 = s12 * s12, s48 = s24 * s24, s50 = s48 * sor * sor;
        *u += AA * invT * (s50 - s48 * sor) + invT;
        *nf = -AA * invT * (50 * s50 - 49 * s48 * sor) * dist_inv;
        return;
    }
    if (pot == 3) {
        float size_ratio = sigma / pp[2], phi_pol = pp[3];
        float ros = ros_ao, ros3 = ros * ros * ros;
        float eta1 = (float)(size_ratio + 1.0), eta2 = eta1 * eta1;
        /* double literals: the bracket, the product and the sum are double */
        double val = (double)(-1.0f * phi_pol) * (((double)(eta2 * eta1) - 1.5 * eta2 * ros) + 0.5 * ros3);
        *u = (float)((double)*u + val);
        *nf = (float)((double)(1.0f * phi_pol) * (1.5 * eta2 * ros - 1.5 * ros3) * dist_inv);
        return;
    }
    /* 4: HSAY as intended */
    float z = pp[0], ros = 1.0f / sor, dudr = 0.0f;
    if (ros < 1.0f) {
        float s2 = sor * sor, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8, s20 = s4 * s16, s40 = s20 * s20;
        *u += s40 - 2.0f * s20 + 1.0f;
        dudr += -40.0f * (s40 - s20) * dist_inv;
    }
    float uatt = -sor * expf(-z * (ros - 1.0f));
    *u += uatt;
    dudr -= (1.0f + ros * z) * uatt * dist_inv;
    *nf = dudr;
}

/* Engine forces with a potential of potentials.cu (all pairs, index order,
 * the engine's cut distances): as or_eng_forces, pair arithmetic from
 * or_pair_extra (pot 0: the modified WCA). */
void or_eng_forces_pot(int n, const float *pos, const int *type, float side, const float sigma[2], int pot,
                       const float *pp, float *ff, float *potv, float *vir) {
    float side_inv = 1.0f / side;
    float sg[2][2];
    sg[0][0] = sigma[0]; sg[1][1] = sigma[1];
    sg[0][1] = sg[1][0] = 0.5f * (sigma[0] + sigma[1]);
    for (int m = 0; m < n; m++) {
        float fx = 0, fy = 0, fz = 0, pm = 0, vm = 0;
        for (int j = 0; j < n; j++) {
            if (j == m) continue;
            float s = sg[type[m]][type[j]], c;
            switch (pot) {
                case 1: c = s * 1.12246205f; break;
                case 2: c = s * (50.0f / 49.0f); break;
                case 3: c = s * (1.0f + s / pp[2]); break;
                case 4: c = s * pp[1]; break;
                default: c = s;
            }
            float dx = pos[3 * j] - pos[3 * m], dy = pos[3 * j + 1] - pos[3 * m + 1], dz = pos[3 * j + 2] - pos[3 * m + 2];
            dx -= side * floorf(side_inv * dx + 0.5f);
            dy -= side * floorf(side_inv * dy + 0.5f);
            dz -= side * floorf(side_inv * dz + 0.5f);
            float d2 = dx * dx + dy * dy + dz * dz;
            if (d2 < c * c) {
                float di = sqrtf(1.0f / d2), nf;
                if (pot == 0) wca_modified(s, di, &pm, &nf);
                else or_pair_extra(pot, pp, s, di, &pm, &nf);
                float px = nf * di * dx, py = nf * di * dy, pz = nf * di * dz;
                fx += px; fy += py; fz += pz;
                vm -= 0.5f * (dx * px + dy * py + dz * pz);
            }
        }
        ff[3 * m] = fx; ff[3 * m + 1] = fy; ff[3 * m + 2] = fz;
        if (potv) potv[m] = pm;
        if (vir) vir[m] = vm;
    }
}
