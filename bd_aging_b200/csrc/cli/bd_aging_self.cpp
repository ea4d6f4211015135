// bd_aging_self -- drop-in replacement of the reference executable
// bd_aging_self.bin (main.cu): same stdin protocol (or wca_aging_linear.data),
// same ../configs/[decadeN/]init_config_%d inputs, same bitacora and results/
// files written with %f, same exit codes.  All n_configs configurations run as
// one batch of replicas on the B200 engine instead of one after another.
//
// Reproduced reference behaviours (so that the files compare equal):
//  * every configuration uses the same cuRAND stream (the reference seeds each
//    configuration with the same idum, main.cu:483-484); BD_RNG=philox in the
//    environment switches to independent counter-based streams;
//  * fself.out row i holds the F_s of sample i (counter i+1 is 1-based,
//    main.cu:772, fself.cu:20), so row 0 is 0 and the last sample is dropped;
//  * msd_averaged.out holds the last configuration's MSD (main.cu:795-797
//    assigns instead of accumulating), the other files are averages;
//  * "log" sampling follows the LOG_SAMPLE build (main.cu:169-173, 612-616),
//    "linear" sampling the default build (main.cu:618-619);
//  * configurations after the first take their first step at the temperature
//    the previous configuration ended on (temp_set is set to T0 once,
//    main.cu:156, before the loop over configurations).
// Deviations: out-of-box input coordinates are wrapped into the box (the
// reference indexes cells out of bounds); bounds are checked where the
// reference reads past its arrays (main.cu:613).
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bd_aging.h"

namespace {

struct Config {
    float phi_big = 0, phi_sml = 0, side = 0, sigma_big = 0, sigma_sml = 0, mass_big = 0, mass_sml = 0;
    int n_big = 0, n_sml = 0, n_tot = 0;
    std::vector<float> pos;  // 3 * n_tot
};

bool read_line(FILE *f, char *buf, int n) { return fgets(buf, n, f) != nullptr; }

int read_config(const char *path, Config &c) {
    FILE *f = fopen(path, "r");
    if (!f) {
        printf("Verify file path: %s", path);
        fflush(stdout);
        exit(-2);
    }
    char ln[200];
    read_line(f, ln, sizeof ln); sscanf(ln, "%f %f", &c.phi_big, &c.phi_sml);
    read_line(f, ln, sizeof ln); sscanf(ln, "%f", &c.side);
    read_line(f, ln, sizeof ln); sscanf(ln, "%d %d %d", &c.n_big, &c.n_sml, &c.n_tot);
    read_line(f, ln, sizeof ln); sscanf(ln, "%f %f", &c.sigma_big, &c.sigma_sml);
    read_line(f, ln, sizeof ln); sscanf(ln, "%f %f", &c.mass_big, &c.mass_sml);
    read_line(f, ln, sizeof ln);
    c.pos.assign(3 * (size_t)c.n_tot, 0.f);
    for (int mm = 0; mm < c.n_tot; mm++) {
        int nn = -1;
        float x = 0, y = 0, z = 0;
        if (!read_line(f, ln, sizeof ln)) ln[0] = 0;
        sscanf(ln, "%d %f %f %f", &nn, &x, &y, &z);
        if (nn != mm) {  // main.cu:383-386
            printf("error: mm %d  nn %d no match\n", mm, nn);
            exit(1);
        }
        float *p = &c.pos[3 * (size_t)mm];
        p[0] = x; p[1] = y; p[2] = z;
        for (int k = 0; k < 3; k++) {
            p[k] -= c.side * std::floor(p[k] / c.side);
            if (!(p[k] >= 0.f) || p[k] > c.side) p[k] = 0.f;
        }
    }
    fclose(f);
    return 0;
}

// log_sampling / sampling_indexes, main.cu:14-53 (float arguments)
std::vector<int> sampling_indexes(float minimal_decade, float run_time, float dt, int per_decade) {
    int last_power = (int)roundf(log10f(run_time));
    int initial_power = (int)roundf(log10f(minimal_decade));
    std::vector<float> values;
    float r = powf(10.0f, 1.0f / per_decade), x = 1.0f;
    for (int i = 0; i <= per_decade; i++) { values.push_back(x); x *= r; }
    std::vector<int> idx(1, 0);
    for (int ipow = initial_power; ipow < last_power; ++ipow) {
        float power = (float)pow(10.0, (double)ipow);
        for (int j = 0; j < per_decade; j++) idx.push_back((int)roundf(values[j] * power / dt));
    }
    return idx;
}

void die_status(int rc, const char *where) {
    if (rc == BD_ERR_CELL_OVERFLOW) {
        printf("ntags reached limit\n");
        fflush(stdout);
        exit(1);
    }
    fprintf(stderr, "%s: %s\n", where, bd_status_string(rc));
    exit(rc == BD_ERR_FILE ? -2 : 1);
}

FILE *open_out(const char *path) {
    FILE *f = fopen(path, "w");
    if (!f) {
        printf("Verify file path: %s", path);
        fflush(stdout);
        exit(-2);
    }
    return f;
}

}  // namespace

int main() {
    FILE *fp_data = fopen("wca_aging_linear.data", "r");
    if (!fp_data) fp_data = stdin;
    char ln[200], protocol[40] = "", sample_type[40] = "";
    float T0 = 0, Tf = 0, t0 = 0, tf = 0, period = 1, range_gder = 0, qmax = 0;
    int ngap_rescaling = 0, nsamples = 0, ntags_big = 0, ntags_sml = 0, n_configs = 0, nbins_gder = 0, idum = 0;
    int print_decades = 0, number_of_tws = 0, current_decade = 0;
    double dt = 0, trans_time = 0, run_time = 0, minimal_decade = 0;
    printf("temp_protocol ?\n");
    read_line(fp_data, ln, sizeof ln); sscanf(ln, "%39s", protocol);
    printf("temp_settings ?\n");
    read_line(fp_data, ln, sizeof ln);
    if (!strcmp(protocol, "linear")) sscanf(ln, "%f %f %f %f %d", &T0, &Tf, &t0, &tf, &ngap_rescaling);
    if (!strcmp(protocol, "sine")) sscanf(ln, "%f %f %f %f %f %d", &T0, &Tf, &t0, &tf, &period, &ngap_rescaling);
    printf("dt ?\n");
    read_line(fp_data, ln, sizeof ln); sscanf(ln, "%lf", &dt);
    printf("sample type (linear, log) ?\n");
    read_line(fp_data, ln, sizeof ln); sscanf(ln, "%39s", sample_type);
    const bool logs = !strcmp(sample_type, "log");
    if (logs) {
        printf("log sampling selected. Must be added in compilation as -DLOG_SAMPLE\n");
        printf("trans_time, minimal_decade, run_time, nsamples (taken in run)\n");
        read_line(fp_data, ln, sizeof ln); sscanf(ln, "%lf %lf %lf", &trans_time, &minimal_decade, &run_time);
        printf("print decade configs?\n");
        read_line(fp_data, ln, sizeof ln); sscanf(ln, "%d %d %d", &print_decades, &number_of_tws, &current_decade);
    } else {
        printf("trans_time, run_time, nsamples (taken in run)\n");
        read_line(fp_data, ln, sizeof ln); sscanf(ln, "%lf %lf %d", &trans_time, &run_time, &nsamples);
    }
    printf("ntags: big, sml ?\n");
    read_line(fp_data, ln, sizeof ln); sscanf(ln, "%d %d", &ntags_big, &ntags_sml);
    printf("n_configs ?\n");
    read_line(fp_data, ln, sizeof ln); sscanf(ln, "%d", &n_configs);
    printf("nbins_gder, range_gder ?\n");
    read_line(fp_data, ln, sizeof ln); sscanf(ln, "%d %f", &nbins_gder, &range_gder);
    printf("qmax ?\n");
    read_line(fp_data, ln, sizeof ln); sscanf(ln, "%f", &qmax);
    printf("idum ?\n");
    read_line(fp_data, ln, sizeof ln); sscanf(ln, "%d", &idum);
    if (fp_data != stdin) fclose(fp_data);
    printf("Starts simulation_3D_2SP Device\n");
    if (n_configs < 1 || nbins_gder < 1) {
        fprintf(stderr, "bd_aging_self: n_configs and nbins_gder must be positive\n");
        return 1;
    }
    const float bin_size_gder = range_gder / ((float)nbins_gder);
    const int points_per_decade = 10;
    std::vector<int> sampling_idx;
    if (logs) {
        sampling_idx = sampling_indexes((float)minimal_decade, (float)run_time, (float)dt, points_per_decade);
        nsamples = (int)sampling_idx.size();
    }
    const int niter = (int)(run_time / dt);
    if (nsamples < 1) { printf("error: ngap %d\n", 0); return 1; }
    const int ngap = niter / nsamples;
    if (ngap < 1) { printf("error: ngap %d\n", ngap); return 1; }  // main.cu:403-406
    const int ntrans = (int)(trans_time / dt);

    // configurations
    std::vector<Config> cfg(n_configs);
    for (int i = 0; i < n_configs; i++) {
        char path[256];
        if (logs) snprintf(path, sizeof path, "../configs/decade%d/init_config_%d", current_decade, i + 1);
        else snprintf(path, sizeof path, "../configs/init_config_%d", i + 1);
        read_config(path, cfg[i]);
        if (i > 0 && (cfg[i].n_big != cfg[0].n_big || cfg[i].n_sml != cfg[0].n_sml)) {
            fprintf(stderr, "bd_aging_self: all configurations must have the particle counts of the first\n");
            return 1;
        }
    }
    const Config &c0 = cfg[0];
    const int nb = c0.n_big, ns = c0.n_sml, ntot = c0.n_tot;
    bd_parametros pars;
    if (bd_setup_params(&pars, c0.side, nb, ns, c0.sigma_big, c0.sigma_sml, c0.mass_big, c0.mass_sml, ntags_big,
                        ntags_sml, nbins_gder, range_gder, dt, T0) != BD_OK) {
        fprintf(stderr, "bd_aging_self: bad geometry\n");
        return 1;
    }
    FILE *fp_bitac = open_out("bitacora");
    fprintf(fp_bitac, "side  %f  ngr b s tot  %d  %d  %d\n", c0.side, nb, ns, ntot);
    fprintf(fp_bitac, "ncell b, s  %d  %d\n", pars.ncell_big, pars.ncell_sml);
    fprintf(fp_bitac, "cell_side b, s  %f  %f\n", pars.cell_side_big, pars.cell_side_sml);
    fprintf(fp_bitac, "ntags b, s  %d  %d\n", ntags_big, ntags_sml);
    fflush(fp_bitac);
    fprintf(fp_bitac, "ranges bb, bs  %d  %d\n", pars.nrange_bb, pars.nrange_bs);
    fprintf(fp_bitac, "ranges sb, ss  %d  %d\n", pars.nrange_sb, pars.nrange_ss);
    const int ncb3 = pars.ncell_big * pars.ncell_big * pars.ncell_big;
    const int ncs3 = pars.ncell_sml * pars.ncell_sml * pars.ncell_sml;
    fprintf(fp_bitac, "ncell_big3  %d  ntot_big  %d\n", ncb3, ncb3 * ntags_big);
    fprintf(fp_bitac, "ncell_sml3  %d  ntot_sml  %d\n", ncs3, ncs3 * ntags_sml);
    for (int i = 0; i < n_configs; i++)
        fprintf(fp_bitac, "niter, ntrans, nsamples, ngap %d %d %d %d\n", niter, ntrans, nsamples, ngap);

    // engine: one replica per configuration, all from the first file's geometry
    const char *rng_env = getenv("BD_RNG");
    const bool philox = rng_env && !strcmp(rng_env, "philox");
    // The reference sets temp_set to T0 once, before its loop over
    // configurations (main.cu:156), and updates it after every step
    // (main.cu:520-524): every configuration after the first starts at the
    // temperature the previous one ended on, after its last step niter - 1.
    float T_carry = T0;
    if (niter > -ntrans) {
        const float t_last = (float)(dt * (1.0 + (float)(niter - 1)));
        if (!strcmp(protocol, "linear")) T_carry = bd_calculate_temp_linear(T0, Tf, t0, tf, t_last);
        else if (!strcmp(protocol, "sine")) T_carry = bd_calculate_temp_sine(T0, Tf, t0, tf, period, t_last);
    }
    std::vector<bd_system_desc> desc(n_configs);
    for (int i = 0; i < n_configs; i++) {
        bd_system_desc &d = desc[i];
        memset(&d, 0, sizeof d);
        d.n_big = nb; d.n_sml = ns; d.side = c0.side;
        d.sigma_big = c0.sigma_big; d.sigma_sml = c0.sigma_sml;
        d.mob_big = 1.0f / c0.sigma_big; d.mob_sml = 1.0f / c0.sigma_sml;  // update_ermak.cu:106-114
        d.dt = dt;
        d.temp_protocol = !strcmp(protocol, "sine") ? BD_PROTOCOL_SINE : BD_PROTOCOL_LINEAR;
        d.T0 = T0; d.Tf = Tf; d.t0 = t0; d.tf = tf; d.period = period;
        d.seed = philox ? (unsigned long long)idum * 1000003ull + i : (unsigned long long)(long long)idum;
        if (i > 0) {
            d.first_temp_set = 1;
            d.T_first = T_carry;
        }
    }
    bd_engine_opts opts;
    bd_engine_opts_default(&opts);
    opts.rng = philox ? BD_RNG_PHILOX : BD_RNG_CURAND;
    opts.qmax = qmax;
    opts.ni_start = -ntrans;
    bd_engine *e = nullptr;
    int rc = bd_engine_create(desc.data(), n_configs, &opts, &e);
    if (rc) die_status(rc, "bd_engine_create");
    std::vector<float> all((size_t)3 * ntot * n_configs);
    for (int i = 0; i < n_configs; i++) memcpy(&all[(size_t)3 * ntot * i], cfg[i].pos.data(), sizeof(float) * 3 * ntot);
    rc = bd_engine_set_positions(e, all.data());
    if (rc) die_status(rc, "bd_engine_set_positions");

    // device buffers for the reference-geometry occupancy check (main.cu:642-659)
    std::vector<double> gacc((size_t)nsamples * 4 * nbins_gder, 0.0);
    std::vector<float> time_energy(nsamples, 0.f), energy_ub(nsamples, 0.f), energy_us(nsamples, 0.f),
        energy_temp(nsamples, 0.f), time_msd(nsamples, 0.f), msd_b(nsamples, 0.f), msd_s(nsamples, 0.f),
        time_pressure(nsamples, 0.f), pressure(nsamples, 0.f), fself(nsamples + 1, 0.f);
    std::vector<bd_observables> ob(n_configs);
    std::vector<unsigned long long> counts((size_t)n_configs * 4 * nbins_gder);
    std::vector<float> pos_out((size_t)3 * ntot * n_configs);
    std::vector<int> number_of_tw(n_configs, 1);
    int counter = 0, energy_counter = 0, sampling_counter = 0;
    auto occupancy = [&](int &ob_max, int &os_max) {
        // max cell occupancy of the reference's cell lists, over all configurations
        ob_max = os_max = 0;
        int r = bd_engine_get_positions(e, pos_out.data(), nullptr);
        if (r) die_status(r, "bd_engine_get_positions");
        for (int i = 0; i < n_configs; i++) {
            const float *p = &pos_out[(size_t)3 * ntot * i];
            std::vector<int> nbig(ncb3, 0), nsml(ncs3, 0);
            const float csb = (float)(1.0 / pars.cell_side_big), css = (float)(1.0 / pars.cell_side_sml);
            for (int m = 0; m < ntot; m++) {
                const bool big = m < nb;
                const float cs = big ? csb : css;
                const int nc = big ? pars.ncell_big : pars.ncell_sml;
                int ii = (int)(cs * p[3 * m]), jj = (int)(cs * p[3 * m + 1]), kk = (int)(cs * p[3 * m + 2]);
                if (ii == nc) ii--;
                if (jj == nc) jj--;
                if (kk == nc) kk--;
                ii = ii < 0 ? 0 : (ii >= nc ? nc - 1 : ii);
                jj = jj < 0 ? 0 : (jj >= nc ? nc - 1 : jj);
                kk = kk < 0 ? 0 : (kk >= nc ? nc - 1 : kk);
                int &o = big ? nbig[ii + nc * (jj + nc * kk)] : nsml[ii + nc * (jj + nc * kk)];
                o++;
                if (big && o > ob_max) ob_max = o;
                if (!big && o > os_max) os_max = o;
            }
        }
    };

    long long ni = -ntrans;
    while (ni < niter) {
        // next step at which the host has work: a sample or a transient report
        long long next = niter;
        if (logs) {
            if (sampling_counter < (int)sampling_idx.size() && sampling_idx[sampling_counter] >= ni)
                next = std::min<long long>(next, sampling_idx[sampling_counter]);
        } else {
            long long k = ni >= 0 ? ((ni + ngap - 1) / ngap) * ngap : 0;
            next = std::min<long long>(next, k);
        }
        if (ni < 0) {
            long long k = (ni / ngap) * ngap;  // ni <= k < 0 with k % ngap == 0 (C truncation)
            if (k < ni) k += ngap;
            if (k < 0) next = std::min<long long>(next, k);
        }
        if (next >= niter) {
            rc = bd_engine_run(e, niter - ni);
            if (rc) die_status(rc, "bd_engine_run");
            ni = niter;
            break;
        }
        rc = bd_engine_run(e, next - ni + 1);  // updates ni .. next
        if (rc) die_status(rc, "bd_engine_run");
        ni = next;
        const float time = (float)(dt * (1.0 + (float)ni));
        if (ni < 0 && ni % ngap == 0) {  // main.cu:591-609
            int obm, osm;
            occupancy(obm, osm);
            printf("run ni %lld/%d  %.2f%%  --  print %d/%d  --  ocup b s  %d %d\n", ni, niter,
                   100.0 * ((float)ni) / ((float)niter), counter, nsamples, obm, osm);
            fflush(stdout);
        }
        bool sample = false;
        if (logs) {
            if (sampling_counter < (int)sampling_idx.size() && ni == sampling_idx[sampling_counter]) {
                sample = true;
                sampling_counter++;
            }
        } else if (ni >= 0 && ni % ngap == 0) {
            sample = true;
        }
        if (!sample) { ni++; continue; }
        counter++;
        if (counter <= 0 || counter > nsamples) {  // main.cu:758-761
            fprintf(stderr, "ERROR: counter=%d fuera de rango\n", counter);
            exit(EXIT_FAILURE);
        }
        rc = bd_engine_observe(e, ob.data());
        if (rc) die_status(rc, "bd_engine_observe");
        const float temp_set = (float)ob[0].temperature;
        for (int i = 0; i < n_configs; i++) {
            energy_us[energy_counter] += (float)ob[i].energy_sml;
            energy_ub[energy_counter] += (float)ob[i].energy_big;
        }
        time_energy[energy_counter] = time;
        energy_temp[energy_counter] = temp_set;
        energy_counter++;
        int obm, osm;
        occupancy(obm, osm);
        printf("run ni %lld/%d  %.2f%%  --  print %d/%d  --  ocup b s  %d %d -- temp %.3f\n", ni, niter,
               100.0 * ((float)ni) / ((float)niter), counter, nsamples, obm, osm, temp_set);
        fflush(stdout);
        if (obm >= ntags_big || osm >= ntags_sml) {
            printf("ntags reached limit\n");
            fflush(stdout);
            exit(1);
        }
        rc = bd_engine_gder(e, nbins_gder, range_gder, counts.data());
        if (rc) die_status(rc, "bd_engine_gder");
        for (int i = 0; i < n_configs; i++)
            for (int k = 0; k < 4 * nbins_gder; k++)
                gacc[(size_t)(counter - 1) * 4 * nbins_gder + k] += (double)counts[(size_t)i * 4 * nbins_gder + k];
        for (int i = 0; i < n_configs; i++) fself[counter] += (float)ob[i].fself_big;  // fself.cu:20 index
        time_msd[counter - 1] = time;
        msd_b[counter - 1] = (float)ob[n_configs - 1].msd_big;
        msd_s[counter - 1] = (float)ob[n_configs - 1].msd_sml;
        for (int i = 0; i < n_configs; i++)
            pressure[counter - 1] += (float)(1.0 + ob[i].virial / (3.0 * (float)ntot * temp_set));
        time_pressure[counter - 1] = time;
        if (logs && (counter - 1) % points_per_decade == 1 && print_decades) {  // main.cu:809-835
            rc = bd_engine_get_positions(e, pos_out.data(), nullptr);
            if (rc) die_status(rc, "bd_engine_get_positions");
            for (int i = 0; i < n_configs; i++) {
                if (number_of_tw[i] > number_of_tws) continue;
                char path[256];
                snprintf(path, sizeof path, "../configs/decade%d/init_config_%d", number_of_tw[i], i + 1);
                FILE *fo = fopen(path, "w");
                if (fo) {
                    const Config &c = cfg[i];
                    fprintf(fo, "%f %f    phi b, s\n", c.phi_big, c.phi_sml);
                    fprintf(fo, "%f    side\n", c.side);
                    fprintf(fo, "%d %d %d    ngr b, s, tot\n", nb, ns, ntot);
                    fprintf(fo, "%f %f    sigma b, s\n", c.sigma_big, c.sigma_sml);
                    fprintf(fo, "%f %f    mass b, s\n", c.mass_big, c.mass_sml);
                    fprintf(fo, "\n");
                    const float *p = &pos_out[(size_t)3 * ntot * i];
                    for (int m = 0; m < ntot; m++) fprintf(fo, "%d %f %f %f\n", m, p[3 * m], p[3 * m + 1], p[3 * m + 2]);
                    fclose(fo);
                }
                number_of_tw[i]++;
            }
        }
        ni++;
    }
    for (int i = 1; i <= n_configs; i++) printf("Finished step %d of %d\n", i, n_configs);

    // normalisation (main.cu:847-882) and output (main.cu:886-980)
    std::vector<float> g((size_t)4 * nbins_gder);
    printf("printing files\n");
    for (int s = 0; s < nsamples; s++) {
        bd_gder_normalize(&gacc[(size_t)s * 4 * nbins_gder], nbins_gder, bin_size_gder, c0.side, nb, ns,
                          c0.sigma_big, c0.sigma_sml, n_configs, g.data());
        char path[256];
        if (logs) snprintf(path, sizeof path, "results/decade%d/gder_%d.out", current_decade, s);
        else snprintf(path, sizeof path, "results/gder_%d.out", s);
        FILE *f = open_out(path);
        for (int k = 0; k < nbins_gder; k++) {
            float dist = (0.5 + (float)k) * bin_size_gder;
            fprintf(f, "%f  %f  %f  %f  %f\n", dist, g[k], g[nbins_gder + k], g[2 * nbins_gder + k],
                    g[3 * nbins_gder + k]);
        }
        fclose(f);
    }
    auto path_of = [&](const char *name) {
        static char p[256];
        if (logs) snprintf(p, sizeof p, "results/decade%d/%s", current_decade, name);
        else snprintf(p, sizeof p, "results/%s", name);
        return std::string(p);
    };
    FILE *f = open_out(path_of("energies_averaged.out").c_str());
    for (int s = 0; s < nsamples; s++) {
        energy_ub[s] /= n_configs;
        energy_us[s] /= n_configs;
        fprintf(f, "%f  %f  %f  %f\n", time_energy[s], energy_ub[s], energy_us[s], energy_temp[s]);
    }
    fclose(f);
    f = open_out(path_of("fself.out").c_str());
    for (int s = 0; s < nsamples; s++) fprintf(f, "%f  %f\n", time_msd[s], fself[s] / n_configs);
    fclose(f);
    f = open_out(path_of("msd_averaged.out").c_str());
    for (int s = 0; s < nsamples; s++) fprintf(f, "%f  %f  %f\n", time_msd[s], msd_b[s], msd_s[s]);
    fclose(f);
    f = open_out(path_of("pressure.out").c_str());
    for (int s = 0; s < nsamples; s++) fprintf(f, "%f  %f\n", time_pressure[s], pressure[s] / n_configs);
    fclose(f);
    fclose(fp_bitac);
    bd_engine_destroy(e);
    printf("TERMINADO\n");
    return 0;
}
