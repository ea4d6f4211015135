// Driver for the reference's own CUDA kernels (cell_locate_dev,
// set_vec_*_dev, get_forces_same_dev / get_forces_diff_dev, setup_rng_kernel,
// update_ermak_dev, get_gder_dev), launched in the order of the reference
// time loop (main.cu:415-485 set-up, main.cu:494-588 per step) on managed
// memory, as the reference does (main.cu:303-321).  Built from the reference
// sources into oracle/_ref/libref.so.  Test infrastructure and the
// "reference CUDA build" baseline: nothing in the product calls it.
#include "encabezados.h"
#include <cstring>
#include <vector>

extern "C" {

/* Parameter set-up of main.cu:155-163, 244-298, 348-349 (cell geometry,
 * ranges, gder bins).  Fills a reference `parametros`. */
void ref_setup_params(parametros *pars, float side, int ngrain_big, int ngrain_sml, float sigma_big,
                      float sigma_sml, float mass_big, float mass_sml, int ntags_big, int ntags_sml,
                      int nbins_gder, float range_gder, double dt, float T0) {
    std::memset(pars, 0, sizeof(parametros));
    float cutoff, aux, cell_side_big, cell_side_sml;
    int ncell_big, ncell_sml;
    pars->dt = dt;
    pars->temp_set = T0;
    pars->nbins_gder = nbins_gder;
    pars->range_gder = range_gder;
    pars->ntags_big = ntags_big;
    pars->ntags_sml = ntags_sml;
    pars->bin_size_gder = range_gder / ((float)nbins_gder);
    pars->side = side;
    pars->ngrain_big = ngrain_big;
    pars->ngrain_sml = ngrain_sml;
    pars->ngrain_tot = ngrain_big + ngrain_sml;
    pars->sigma_big = sigma_big;
    pars->sigma_sml = sigma_sml;
    pars->mass_big = mass_big;
    pars->mass_sml = mass_sml;
    cutoff = sigma_big;
    ncell_big = (int)(side / (1.05 * cutoff));
    cell_side_big = side / ((float)ncell_big);
    pars->ncell_big = ncell_big;
    pars->cell_side_big = cell_side_big;
    cutoff = sigma_sml;
    ncell_sml = (int)(side / (1.05 * cutoff));
    cell_side_sml = side / ((float)ncell_sml);
    pars->ncell_sml = ncell_sml;
    pars->cell_side_sml = cell_side_sml;
    pars->nrange_bb = 1;
    aux = (sigma_big + sigma_sml) / 2.0;
    pars->nrange_bs = 1 + (int)(aux / cell_side_sml);
    pars->nrange_sb = 1;
    pars->nrange_ss = 1;
    pars->NH = 256;
}

struct RefState {
    parametros pars;
    float3 *rr_b, *raw_b, *ini_b, *ff_b, *rr_s, *raw_s, *ini_s, *ff_s;
    float *vir_b, *pot_b, *vir_s, *pot_s;
    int *nocup_b, *cell_b, *nocup_s, *cell_s;
    int nb, ns, ncb3, ncs3, ntb, nts, NH, NB_B, NB_S;
};

static void ref_alloc(RefState &S, const parametros *p) {
    S.pars = *p;
    S.nb = p->ngrain_big; S.ns = p->ngrain_sml;
    S.ncb3 = p->ncell_big * p->ncell_big * p->ncell_big;
    S.ncs3 = p->ncell_sml * p->ncell_sml * p->ncell_sml;
    S.ntb = S.ncb3 * p->ntags_big; S.nts = S.ncs3 * p->ntags_sml;
    S.NH = 256; S.NB_B = 1 + (S.nb - 1) / S.NH; S.NB_S = 1 + (S.ns - 1) / S.NH;
    cudaMallocManaged(&S.rr_b, S.nb * sizeof(float3)); cudaMallocManaged(&S.raw_b, S.nb * sizeof(float3));
    cudaMallocManaged(&S.ini_b, S.nb * sizeof(float3)); cudaMallocManaged(&S.ff_b, S.nb * sizeof(float3));
    cudaMallocManaged(&S.vir_b, S.nb * sizeof(float)); cudaMallocManaged(&S.pot_b, S.nb * sizeof(float));
    cudaMallocManaged(&S.nocup_b, S.ncb3 * sizeof(int)); cudaMallocManaged(&S.cell_b, S.ntb * sizeof(int));
    cudaMallocManaged(&S.rr_s, S.ns * sizeof(float3)); cudaMallocManaged(&S.raw_s, S.ns * sizeof(float3));
    cudaMallocManaged(&S.ini_s, S.ns * sizeof(float3)); cudaMallocManaged(&S.ff_s, S.ns * sizeof(float3));
    cudaMallocManaged(&S.vir_s, S.ns * sizeof(float)); cudaMallocManaged(&S.pot_s, S.ns * sizeof(float));
    cudaMallocManaged(&S.nocup_s, S.ncs3 * sizeof(int)); cudaMallocManaged(&S.cell_s, S.nts * sizeof(int));
}
static void ref_free(RefState &S) {
    cudaFree(S.rr_b); cudaFree(S.raw_b); cudaFree(S.ini_b); cudaFree(S.ff_b); cudaFree(S.vir_b); cudaFree(S.pot_b);
    cudaFree(S.nocup_b); cudaFree(S.cell_b);
    cudaFree(S.rr_s); cudaFree(S.raw_s); cudaFree(S.ini_s); cudaFree(S.ff_s); cudaFree(S.vir_s); cudaFree(S.pot_s);
    cudaFree(S.nocup_s); cudaFree(S.cell_s);
}
/* cell rebuild + force evaluation exactly as main.cu:536-585 */
static void ref_cells_forces(RefState &S) {
    const int NH = S.NH;
    const int NBC_B = 1 + (S.ncb3 - 1) / NH, NBC_S = 1 + (S.ncs3 - 1) / NH;
    const int NBT_B = 1 + (S.ntb - 1) / NH, NBT_S = 1 + (S.nts - 1) / NH;
    float3 zero; zero.x = zero.y = zero.z = 0.0f;
    parametros &pars = S.pars;
    set_vec_int_dev<<<NBC_B, NH>>>(S.nocup_b, S.ncb3, 0);
    set_vec_int_dev<<<NBT_B, NH>>>(S.cell_b, S.ntb, -1);
    cell_locate_dev<<<S.NB_B, NH>>>('b', S.rr_b, S.nocup_b, S.cell_b, pars);
    set_vec_int_dev<<<NBC_S, NH>>>(S.nocup_s, S.ncs3, 0);
    set_vec_int_dev<<<NBT_S, NH>>>(S.cell_s, S.nts, -1);
    cell_locate_dev<<<S.NB_S, NH>>>('s', S.rr_s, S.nocup_s, S.cell_s, pars);
    set_vec_float3_dev<<<S.NB_B, NH>>>(S.ff_b, S.nb, zero);
    set_vec_float_dev<<<S.NB_B, NH>>>(S.vir_b, S.nb, 0.0);
    set_vec_float_dev<<<S.NB_B, NH>>>(S.pot_b, S.nb, 0.0);
    set_vec_float3_dev<<<S.NB_S, NH>>>(S.ff_s, S.ns, zero);
    set_vec_float_dev<<<S.NB_S, NH>>>(S.vir_s, S.ns, 0.0);
    set_vec_float_dev<<<S.NB_S, NH>>>(S.pot_s, S.ns, 0.0);
    get_forces_same_dev<<<S.NB_B, NH>>>('b', S.rr_b, S.ff_b, S.vir_b, S.pot_b, S.nocup_b, S.cell_b, pars);
    get_forces_same_dev<<<S.NB_S, NH>>>('s', S.rr_s, S.ff_s, S.vir_s, S.pot_s, S.nocup_s, S.cell_s, pars);
    get_forces_diff_dev<<<S.NB_B, NH>>>('b', 's', S.rr_b, S.ff_b, S.rr_s, S.vir_b, S.pot_b, S.nocup_s, S.cell_s, pars);
    get_forces_diff_dev<<<S.NB_S, NH>>>('s', 'b', S.rr_s, S.ff_s, S.rr_b, S.vir_s, S.pot_s, S.nocup_b, S.cell_b, pars);
}
static int max_occ(const int *n, int m) { int x = 0; for (int i = 0; i < m; i++) if (n[i] > x) x = n[i]; return x; }

/* Forces, potential and virial of the given positions from the reference
 * device kernels.  Returns 0, or 1 if a cell overflowed ntags. */
int ref_cuda_forces(const parametros *p, const float *rr_big, const float *rr_sml, float *ff_big, float *ff_sml,
                    float *vir_big, float *vir_sml, float *pot_big, float *pot_sml) {
    RefState S; ref_alloc(S, p);
    std::memcpy(S.rr_b, rr_big, S.nb * sizeof(float3));
    std::memcpy(S.rr_s, rr_sml, S.ns * sizeof(float3));
    ref_cells_forces(S);
    cudaDeviceSynchronize();
    int bad = max_occ(S.nocup_b, S.ncb3) > p->ntags_big || max_occ(S.nocup_s, S.ncs3) > p->ntags_sml;
    std::memcpy(ff_big, S.ff_b, S.nb * sizeof(float3)); std::memcpy(ff_sml, S.ff_s, S.ns * sizeof(float3));
    std::memcpy(vir_big, S.vir_b, S.nb * sizeof(float)); std::memcpy(vir_sml, S.vir_s, S.ns * sizeof(float));
    std::memcpy(pot_big, S.pot_b, S.nb * sizeof(float)); std::memcpy(pot_sml, S.pot_s, S.ns * sizeof(float));
    ref_free(S);
    return bad;
}

/* The reference time loop main.cu:494-588 without the sample-step host work:
 * ni = -ntrans .. niter-1, linear temperature protocol, cuRAND states seeded
 * with idum / idum+1 (main.cu:478-484).  Positions in/out are float3 AoS.
 * When nsamp > 0, the unwrapped positions rr_raw (big then small) after
 * sample_after[j] steps from ni = 0 (that is, after the update of step
 * ni = sample_after[j] - 1, time dt * sample_after[j]) go to
 * raw_samples + j * 3 * ngrain_tot; sample_after ascending, in 1 .. niter.
 * elapsed_ms: CUDA-event time of the loop.  Returns 0, 1 on cell overflow,
 * 2 on a CUDA error, 3 on a bad sample list. */
static int ref_cuda_loop(const parametros *p, const float *rr_big, const float *rr_sml, int ntrans, int niter,
                         int idum, float T0, float Tf, float t0, float tf, double dt, float *rr_big_out,
                         float *rr_sml_out, float *raw_big_out, float *raw_sml_out, int nsamp,
                         const int *sample_after, float *raw_samples, float *elapsed_ms) {
    for (int j = 0; j < nsamp; j++)
        if (sample_after[j] < 1 || sample_after[j] > niter || (j && sample_after[j] <= sample_after[j - 1])) return 3;
    RefState S; ref_alloc(S, p);
    std::memcpy(S.rr_b, rr_big, S.nb * sizeof(float3)); std::memcpy(S.raw_b, rr_big, S.nb * sizeof(float3));
    std::memcpy(S.rr_s, rr_sml, S.ns * sizeof(float3)); std::memcpy(S.raw_s, rr_sml, S.ns * sizeof(float3));
    S.pars.temp_set = T0;
    ref_cells_forces(S);
    curandState *st_b, *st_s;
    cudaMalloc(&st_b, (size_t)S.nb * sizeof(curandState));
    cudaMalloc(&st_s, (size_t)S.ns * sizeof(curandState));
    setup_rng_kernel<<<S.NB_B, S.NH>>>(st_b, idum, S.nb);
    setup_rng_kernel<<<S.NB_S, S.NH>>>(st_s, idum + 1, S.ns);
    cudaDeviceSynchronize();
    cudaEvent_t e0, e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
    cudaEventRecord(e0);
    int js = 0;
    for (int ni = -ntrans; ni < niter; ni++) {
        cudaDeviceSynchronize();
        if (ni == 0) {
            cudaMemcpy(S.raw_b, S.rr_b, S.nb * sizeof(float3), cudaMemcpyHostToHost);
            cudaMemcpy(S.ini_b, S.rr_b, S.nb * sizeof(float3), cudaMemcpyHostToHost);
            cudaMemcpy(S.raw_s, S.rr_s, S.ns * sizeof(float3), cudaMemcpyHostToHost);
            cudaMemcpy(S.ini_s, S.rr_s, S.ns * sizeof(float3), cudaMemcpyHostToHost);
        }
        update_ermak_dev<<<S.NB_B, S.NH>>>('b', S.rr_b, S.raw_b, S.ff_b, st_b, S.pars);
        update_ermak_dev<<<S.NB_S, S.NH>>>('s', S.rr_s, S.raw_s, S.ff_s, st_s, S.pars);
        cudaDeviceSynchronize();
        if (js < nsamp && ni == sample_after[js] - 1) {
            float *dst = raw_samples + (size_t)js * 3 * (S.nb + S.ns);
            std::memcpy(dst, S.raw_b, S.nb * sizeof(float3));
            std::memcpy(dst + 3 * (size_t)S.nb, S.raw_s, S.ns * sizeof(float3));
            js++;
        }
        float time = dt * (1.0 + (float)ni);
        S.pars.temp_set = calculate_temp_linear(T0, Tf, t0, tf, time);
        ref_cells_forces(S);
        cudaDeviceSynchronize();
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(elapsed_ms, e0, e1);
    int rc = (cudaGetLastError() != cudaSuccess) ? 2 : 0;
    if (!rc && (max_occ(S.nocup_b, S.ncb3) > p->ntags_big || max_occ(S.nocup_s, S.ncs3) > p->ntags_sml)) rc = 1;
    std::memcpy(rr_big_out, S.rr_b, S.nb * sizeof(float3)); std::memcpy(rr_sml_out, S.rr_s, S.ns * sizeof(float3));
    if (raw_big_out) std::memcpy(raw_big_out, S.raw_b, S.nb * sizeof(float3));
    if (raw_sml_out) std::memcpy(raw_sml_out, S.raw_s, S.ns * sizeof(float3));
    cudaFree(st_b); cudaFree(st_s); cudaEventDestroy(e0); cudaEventDestroy(e1);
    ref_free(S);
    return rc;
}

int ref_cuda_run(const parametros *p, const float *rr_big, const float *rr_sml, int ntrans, int niter, int idum,
                 float T0, float Tf, float t0, float tf, double dt, float *rr_big_out, float *rr_sml_out,
                 float *raw_big_out, float *raw_sml_out, float *elapsed_ms) {
    return ref_cuda_loop(p, rr_big, rr_sml, ntrans, niter, idum, T0, Tf, t0, tf, dt, rr_big_out, rr_sml_out,
                         raw_big_out, raw_sml_out, 0, nullptr, nullptr, elapsed_ms);
}

int ref_cuda_run_sampled(const parametros *p, const float *rr_big, const float *rr_sml, int ntrans, int niter,
                         int idum, float T0, float Tf, float t0, float tf, double dt, int nsamp,
                         const int *sample_after, float *raw_samples, float *rr_big_out, float *rr_sml_out,
                         float *elapsed_ms) {
    return ref_cuda_loop(p, rr_big, rr_sml, ntrans, niter, idum, T0, Tf, t0, tf, dt, rr_big_out, rr_sml_out,
                         nullptr, nullptr, nsamp, sample_after, raw_samples, elapsed_ms);
}

/* g(r) histograms of the reference device kernel (main.cu:719-754): the four
 * per-block float histograms, summed over blocks on the host in the
 * reference's order.  gder_out: 4 x nbins (bb, bs, sb, ss). */
int ref_cuda_gder(const parametros *p, const float *rr_big, const float *rr_sml, float *gder_out) {
    RefState S; ref_alloc(S, p);
    std::memcpy(S.rr_b, rr_big, S.nb * sizeof(float3)); std::memcpy(S.rr_s, rr_sml, S.ns * sizeof(float3));
    int nbins = p->nbins_gder;
    float *bb, *bs, *sb, *ss;
    cudaMallocManaged(&bb, S.NB_B * nbins * sizeof(float)); cudaMallocManaged(&ss, S.NB_S * nbins * sizeof(float));
    cudaMallocManaged(&bs, S.NB_B * nbins * sizeof(float)); cudaMallocManaged(&sb, S.NB_S * nbins * sizeof(float));
    for (int i = 0; i < S.NB_B * nbins; i++) { bb[i] = 0.0f; bs[i] = 0.0f; }
    for (int i = 0; i < S.NB_S * nbins; i++) { ss[i] = 0.0f; sb[i] = 0.0f; }
    get_gder_dev<<<S.NB_B, S.NH>>>('b', 'b', S.rr_b, S.rr_b, bb, S.pars);
    get_gder_dev<<<S.NB_B, S.NH>>>('b', 's', S.rr_b, S.rr_s, bs, S.pars);
    get_gder_dev<<<S.NB_S, S.NH>>>('s', 'b', S.rr_s, S.rr_b, sb, S.pars);
    get_gder_dev<<<S.NB_S, S.NH>>>('s', 's', S.rr_s, S.rr_s, ss, S.pars);
    cudaDeviceSynchronize();
    for (int jj = 0; jj < nbins; jj++) {
        for (int nb = 1; nb < S.NB_B; nb++) bb[jj] += bb[jj + nb * nbins];
        for (int nb = 1; nb < S.NB_S; nb++) ss[jj] += ss[jj + nb * nbins];
        for (int nb = 1; nb < S.NB_S; nb++) sb[jj] += sb[jj + nb * nbins];
        for (int nb = 1; nb < S.NB_B; nb++) bs[jj] += bs[jj + nb * nbins];
    }
    for (int jj = 0; jj < nbins; jj++) {
        gder_out[jj] = bb[jj]; gder_out[nbins + jj] = bs[jj];
        gder_out[2 * nbins + jj] = sb[jj]; gder_out[3 * nbins + jj] = ss[jj];
    }
    cudaFree(bb); cudaFree(bs); cudaFree(sb); cudaFree(ss);
    ref_free(S);
    return cudaGetLastError() != cudaSuccess ? 2 : 0;
}

}  // extern "C"
