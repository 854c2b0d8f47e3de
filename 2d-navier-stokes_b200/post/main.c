/*
 * main.c -- bin/ns2d_post: the spectral part of the reference's
 * post-processing program (PostProcessing/src/main.c, post_proc.c:24-60) on
 * the GPU.
 *
 *   ns2d_post -i <run dir>/ -o <out dir>/ -v 1e-4 -v 0 -v 2.0 -d 0.0 -d 0 -d -2.0 -k 0.5 -t TAG
 *
 * reads every /Iter_%05d/w_hat of <run dir>/Main_HDF_Data.h5 (or of the file
 * given by a second -i), and for each snapshot writes, under /Snap_%05d
 * (attribute TimeValue) of PostProcessing_HDF_Data_SECTORS[..]_KFRAC[..]_TAG[..].h5:
 *   w_hat                                  (hdf5_funcs.c:524-533)
 *   FullField{Phases,Amplitudes,EnergySpectrum,EnstrophySpectrum}
 *                                          (FullFieldData, full_field.c:29-110)
 *   EnstrophySpectrum, EnergySpectrum      (full_field.c:267-365)
 *   Enstrophy/Energy {Flux,TimeDerivative,Diss}Spectrum
 *                                          (FluxSpectra, full_field.c:367-557)
 * and at the end kx, ky, x, y, Time and the set-C sums EnstrophyFluxC,
 * EnstrophyDissC, EnergyFluxC, EnergyDissC (hdf5_funcs.c:1290-1370).
 *
 * The nonlinear term and the spectra come from the GPU: a handle with the
 * run's viscosity and drag, no forcing, the post-processing program's 2/3
 * edge (dealias_edge = 1: |k| > N/3 zeroed, full_field.c:128) and none of
 * the solver's quirks evaluates the RHS of each snapshot and bins it
 * (ns2d_system_measurables; FluxSpectra's sums are sys_msr.c's with the
 * forcing left out).  The full-field arrays are a re-indexing of w_hat done
 * on the host.  The reference's statistics (histograms, structure functions)
 * and sector phase-sync outputs are not produced.
 */
#include <complex.h>
#include <getopt.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include "ns2d.h"
#include "ns2d_h5.h"
#include "phase_sync.h"

#define NUM_K1_SECTORS 8 /* PostProcessing/src/data_types.h:97 */

typedef struct post_args {
    char input_dir[1024], output_dir[1024], tag[64], forcing[64];
    int input_file_only, output_file_only;
    int k3_sectors, k1_sectors, threads, force_k;
    double kmax_frac, nu, hyper_pow, alpha, drag_pow, force_scale;
    int hyper_flag, drag_flag, device;
    int reduced_k1, phase_sync;
} post_args;

static void die(const char* msg, double v) {
    fprintf(stderr, "\n[ERROR] Parsing of Command Line Arguments Failed: ");
    fprintf(stderr, msg, v);
    fprintf(stderr, "\n-->> Exiting!\n\n");
    exit(1);
}

static int flag01(const char* s, const char* what) {
    const int v = atoi(s);
    if (v != 0 && v != 1) {
        fprintf(stderr, "\n[ERROR] Parsing of Command Line Arguments Failed: Incorrect %s flag: [%d] Must be either 0 or 1\n-->> Exiting!\n\n",
                what, v);
        exit(1);
    }
    return v;
}

/* GetCMLArgs of the post-processing program (PostProcessing/src/utils.c:34-280). */
static void parse(int argc, char** argv, post_args* a) {
    memset(a, 0, sizeof(*a));
    strcpy(a->input_dir, "NONE");
    strcpy(a->output_dir, "NONE");
    strcpy(a->tag, "No-Tag");
    strcpy(a->forcing, "NONE");
    a->k3_sectors = 24;
    a->k1_sectors = NUM_K1_SECTORS;
    a->kmax_frac = 1.0;
    a->threads = 1;
    a->force_scale = 1.0;
    a->nu = 0.1;
    a->hyper_pow = 2.0;
    a->alpha = 0.1;
    a->drag_pow = -2.0;
    int seen_o = 0, seen_i = 0, seen_a = 0, seen_v = 0, seen_d = 0, seen_f = 0, c;
    static const struct option longs[] = {
        {"device", required_argument, 0, 1000}, {"phase-sync", no_argument, 0, 1001}, {0, 0, 0, 0}};
    optind = 1;
    while ((c = getopt_long(argc, argv, "a:o:h:n:s:e:t:v:i:c:p:f:z:k:t:d:", longs, NULL)) != -1) {
        switch (c) {
            case 'o':
                if (seen_o++ == 0) snprintf(a->output_dir, sizeof(a->output_dir), "%s", optarg);
                else a->output_file_only = 1;
                break;
            case 'i':
                if (seen_i++ == 0) snprintf(a->input_dir, sizeof(a->input_dir), "%s", optarg);
                else a->input_file_only = 1;
                break;
            case 'a':
                if (seen_a == 0) {
                    a->k3_sectors = a->k1_sectors = atoi(optarg);
                    if (a->k3_sectors <= 0) die("The number of sectors [%g] must be positive", a->k3_sectors);
                } else if (seen_a == 1) {
                    a->k1_sectors = atoi(optarg);
                    if (a->k1_sectors <= 0) die("The number of sectors [%g] must be positive", a->k1_sectors);
                } else if (seen_a == 2) {
                    /* reduced k1 search (utils.c:128-133) */
                    a->k1_sectors = NUM_K1_SECTORS;
                    a->reduced_k1 = 1;
                }
                seen_a++;
                break;
            case 'p':
                a->threads = atoi(optarg);
                if (a->threads <= 0) die("The number of threads [%g] must be positive", a->threads);
                break;
            case 'k':
                a->kmax_frac = atof(optarg);
                if (a->kmax_frac <= 0 || a->kmax_frac > 1.0) die("The fraction of kmax [%lf] must be in (0, 1]", a->kmax_frac);
                break;
            case 'v':
                if (seen_v == 0) {
                    a->nu = atof(optarg);
                    if (a->nu < 0) die("The provided viscosity: [%lf] must be positive", a->nu);
                } else if (seen_v == 1) {
                    a->hyper_flag = flag01(optarg, "Hyperviscosity");
                } else {
                    a->hyper_pow = atof(optarg);
                    if (a->hyper_pow <= 0.0) die("The provided hyperviscosity power: [%lf] must be strictly positive", a->hyper_pow);
                }
                if (seen_v < 2) seen_v++;
                break;
            case 'd':
                if (seen_d == 0) {
                    a->alpha = atof(optarg);
                    if (a->alpha < 0) die("The provided Ekman Drag: [%lf] must be positive", a->alpha);
                } else if (seen_d == 1) {
                    a->drag_flag = flag01(optarg, "Ekman Drag");
                } else {
                    a->drag_pow = atof(optarg);
                    if (a->drag_pow >= 0.0) die("The provided Hypodiffusivity power: [%lf] must be strictly negative", a->drag_pow);
                }
                if (seen_d < 2) seen_d++;
                break;
            case 'f':
                if (seen_f == 0 && (!strcmp(optarg, "ZERO") || !strcmp(optarg, "KOLM") || !strcmp(optarg, "NONE") ||
                                    !strcmp(optarg, "STOC"))) {
                    snprintf(a->forcing, sizeof(a->forcing), "%s", optarg);
                    seen_f = 1;
                } else if (seen_f == 1) {
                    a->force_k = atoi(optarg);
                    seen_f = 2;
                } else if (seen_f == 2) {
                    a->force_scale = atof(optarg);
                }
                break;
            case 't':
                snprintf(a->tag, sizeof(a->tag), "%s", optarg);
                break;
            case 1000:
                a->device = atoi(optarg);
                break;
            case 1001:
                /* the -D__SEC_PHASE_SYNC build (PostProcessing/src/data_types.h:62) */
                a->phase_sync = 1;
                break;
            default:
                fprintf(stderr, "\n[ERROR] Incorrect command line flag encountered\n\nExample usage:\n\tns2d_post -i "
                                "<run dir>/ -o <out dir>/ -v 1e-4 -v 0 -v 2.0 -d 0.0 -d 0 -d -2.0 -k 0.5 -t TAG\n\n-->> Now "
                                "Exiting!\n\n");
                exit(1);
        }
    }
}

static void h5die(int rc, ns2d_h5_file* f, const char* what) {
    if (rc == 0) return;
    fprintf(stderr, "\n[ERROR] --- %s: %s\n-->> Exiting...\n", what, ns2d_h5_error(f));
    exit(1);
}

static ns2d_handle* g_h;
static void check(ns2d_status s, const char* what) {
    if (s == NS2D_OK) return;
    fprintf(stderr, "\n[ERROR] ns2d: %s failed: %s (%s)\n-->> Exiting!\n", what, ns2d_status_string(s),
            g_h ? ns2d_last_error(g_h) : "no handle");
    exit(1);
}

/* FullFieldData (full_field.c:29-110): the modes with |kx|, |ky| <= kmax
   re-indexed onto a centred [2kmax+1]^2 grid, row kmax - kx, column kmax + ky,
   with the conjugate half filled in; modes outside |k| <= kmax hold -50. */
static void full_field(const double complex* w, long nx, long nyf, int kmax, double* phases, double* amps, double* enrg,
                       double* enst) {
    const int w2 = 2 * kmax + 1;
    const double kmax_sqr = (double)kmax * kmax;
    for (long i = 0; i < nx; ++i) {
        const int kx = (int)(i <= nx / 2 ? i : i - nx);
        if (abs(kx) > kmax) continue;
        const int r1 = (kmax - kx) * w2, r2 = (kmax + kx) * w2;
        for (long j = 0; j < nyf; ++j) {
            const int ky = (int)j;
            if (ky > kmax) continue;
            const double complex z = w[i * nyf + j];
            const double k_sqr = (double)(kx * kx + ky * ky);
            const double k_sqr_fac = (kx != 0 || ky != 0) ? 1.0 / k_sqr : 0.0;
            const double phase = fmod(carg(z) + 2.0 * M_PI, 2.0 * M_PI);
            const double amp = cabs(z * conj(z));
            const int in = k_sqr <= kmax_sqr;
            const int a = r1 + kmax + ky, b = r2 + kmax - ky;
            phases[a] = in ? phase : -50.0;
            amps[a] = in ? cabs(z) : -50.0;
            enrg[a] = in ? amp * k_sqr_fac : -50.0;
            enst[a] = in ? amp : -50.0;
            if (ky != 0) {
                phases[b] = in ? fmod(-phase + 2.0 * M_PI, 2.0 * M_PI) : -50.0;
                amps[b] = in ? cabs(z) : -50.0;
                enrg[b] = in ? amp * k_sqr_fac : -50.0;
                enst[b] = in ? amp : -50.0;
            }
        }
    }
}

int main(int argc, char** argv) {
    post_args a;
    parse(argc, argv, &a);
    const clock_t begin = clock();
    char in_file[1200], out_file[1400];
    if (!strcmp(a.input_dir, "NONE")) {
        fprintf(stderr, "\n[ERROR] --- No input directory or file given (-i)\n-->> Exiting...\n");
        return 1;
    }
    if (a.input_file_only)
        snprintf(in_file, sizeof(in_file), "%s", a.input_dir);
    else
        snprintf(in_file, sizeof(in_file), "%sMain_HDF_Data.h5", a.input_dir);
    if (access(in_file, F_OK) != 0) {
        fprintf(stderr, "\n[ERROR] --- Input file [%s] cannot be found\n-->> Exiting...\n", in_file);
        return 1;
    }
    char* out_dir = strcmp(a.output_dir, "NONE") ? a.output_dir : a.input_dir;
    if (a.input_file_only && out_dir == a.input_dir) {
        char* slash = strrchr(a.input_dir, '/');
        if (slash) slash[1] = '\0';
        else strcpy(a.input_dir, "./");
    }
    struct stat st;
    if (stat(out_dir, &st) != 0 && mkdir(out_dir, 0700) != 0) {
        fprintf(stderr, "\n[ERROR] --- Unable to create output directory [%s]\n-->> Exiting...\n", out_dir);
        return 1;
    }
    snprintf(out_file, sizeof(out_file), "%sPostProcessing_HDF_Data_SECTORS[%d,%d]_KFRAC[%1.2lf]_TAG[%s].h5", out_dir,
             a.k3_sectors, a.k1_sectors, a.kmax_frac, a.tag);

    /* snapshots: the /Iter_%05d groups (hdf5_funcs.c:101-127) */
    size_t cap = 1 << 20;
    char* names = (char*)malloc(cap);
    int nlinks;
    while ((nlinks = ns2d_h5_list(in_file, "/", names, cap)) < 0 && cap < ((size_t)1 << 30)) {
        cap *= 4;
        names = (char*)realloc(names, cap);
    }
    h5die(nlinks < 0 ? -1 : 0, NULL, in_file);
    int snaps = 0;
    for (char* s = names; *s;) {
        char* e = strchr(s, '\n');
        *e = '\0';
        int idx;
        char tail;
        if (sscanf(s, "Iter_%d%c", &idx, &tail) == 1 && strlen(s) >= 10 && idx >= 0 && idx < 1000000) snaps++;
        s = e + 1;
    }
    free(names);
    if (snaps == 0) {
        fprintf(stderr, "\n[ERROR] --- No /Iter_ snapshots in [%s]\n-->> Exiting...\n", in_file);
        return 1;
    }
    int type, rank;
    uint64_t dims[8];
    h5die(ns2d_h5_dataset_info(in_file, "/Iter_00000/w_hat", &type, &rank, dims), NULL, "/Iter_00000/w_hat");
    if (type != NS2D_H5_C128 || rank != 2) {
        fprintf(stderr, "\n[ERROR] --- /Iter_00000/w_hat is not a 2-D complex dataset\n-->> Exiting...\n");
        return 1;
    }
    const long nx = (long)dims[0], ny = ((long)dims[1] - 1) * 2, nyf = ny / 2 + 1;
    printf("\nInput File: %s\nOutput File: %s\nTotal Snapshots: [%d]  N = [%ld, %ld]\n", in_file, out_file, snaps, nx, ny);

    ns2d_params p;
    ns2d_params_default(&p);
    p.nx = (int32_t)nx;
    p.ny = (int32_t)ny;
    p.forcing = NS2D_FORCING_NONE;
    p.quirks = 0;
    p.dealias = NS2D_DEALIAS_23;
    p.dealias_edge = 1;
    p.flux_diagnostics = 1;
    p.nu = a.nu;
    p.hyper_visc_flag = a.hyper_flag;
    p.hyper_visc_pow = a.hyper_pow;
    p.ekmn_alpha = a.alpha;
    p.ekmn_drag_flag = a.drag_flag;
    p.ekmn_drag_pow = a.drag_pow;
    p.device = a.device;
    check(ns2d_create(&p, &g_h), "ns2d_create");
    int32_t n1, n2, n3, n_spec;
    check(ns2d_dims(g_h, &n1, &n2, &n3, &n_spec), "ns2d_dims");

    const int kmax = (int)(nx / 3.0);
    const int kmax_c = (int)ceil(a.kmax_frac * kmax);
    const int c_from = (int)round(sqrt((double)kmax_c * kmax_c));
    const size_t w2 = (size_t)(2 * kmax + 1) * (2 * kmax + 1);
    double complex* w = (double complex*)malloc(sizeof(double complex) * (size_t)(nx * nyf));
    double* spec = (double*)calloc((size_t)8 * n_spec, sizeof(double));
    double* ff = (double*)calloc(4 * w2, sizeof(double));
    double* tvals = (double*)calloc((size_t)snaps, sizeof(double));
    double* csum = (double*)calloc(4 * (size_t)snaps, sizeof(double));
    if (!w || !spec || !ff || !tvals || !csum) {
        fprintf(stderr, "out of memory\n");
        return 1;
    }
    ps_state* ps = NULL;
    double complex* rhs = NULL;
    if (a.phase_sync) {
        ps = ps_create((int)nx, kmax, a.kmax_frac, a.k3_sectors, a.k1_sectors, a.reduced_k1, a.nu, a.hyper_flag,
                       a.hyper_pow, a.alpha, a.drag_flag, a.drag_pow, a.device);
        rhs = (double complex*)malloc(sizeof(double complex) * (size_t)(nx * nyf));
        if (!ps || !rhs) {
            fprintf(stderr, "out of memory\n");
            return 1;
        }
    }
    ns2d_h5_file* f = ns2d_h5_create(out_file);
    h5die(f ? 0 : -1, NULL, out_file);
    /* dataset order of WriteDataToFile (hdf5_funcs.c:524-790); spectra index
       in the ns2d_system_measurables order */
    static const char* const ff_names[4] = {"FullFieldPhases", "FullFieldAmplitudes", "FullFieldEnergySpectrum",
                                            "FullFieldEnstrophySpectrum"};
    static const char* const sp_names[8] = {"EnstrophySpectrum",           "EnergySpectrum",
                                            "EnstrophyFluxSpectrum",       "EnstrophyTimeDerivativeSpectrum",
                                            "EnstrophyDissSpectrum",       "EnergyFluxSpectrum",
                                            "EnergyTimeDerivativeSpectrum", "EnergyDissSpectrum"};
    static const int sp_index[8] = {1, 0, 3, 2, 4, 6, 5, 7};
    for (int s = 0; s < snaps; ++s) {
        char g[64], path[160];
        snprintf(g, sizeof(g), "/Iter_%05d", s);
        snprintf(path, sizeof(path), "%s/w_hat", g);
        h5die(ns2d_h5_read(in_file, path, NS2D_H5_C128, w, (uint64_t)(nx * nyf)), NULL, path);
        if (ns2d_h5_read_attr_double(in_file, g, "TimeValue", &tvals[s])) tvals[s] = 0.0;
        check(ns2d_set_w_hat(g_h, (const double*)w), "ns2d_set_w_hat");
        ns2d_measures m;
        check(ns2d_system_measurables(g_h, &m, spec), "spectra");
        full_field(w, nx, nyf, kmax, ff, ff + w2, ff + 2 * w2, ff + 3 * w2);
        /* set-C sums (full_field.c:544-555): shells i >= round(kmax_C) */
        for (int i = 1; i < n_spec; ++i)
            if (i >= c_from) {
                csum[0 * snaps + s] += spec[3 * n_spec + i];
                csum[1 * snaps + s] += spec[4 * n_spec + i];
                csum[2 * snaps + s] += spec[6 * n_spec + i];
                csum[3 * snaps + s] += spec[7 * n_spec + i];
            }
        char sg[64];
        snprintf(sg, sizeof(sg), "/Snap_%05d", s);
        h5die(ns2d_h5_group(f, sg), f, sg);
        h5die(ns2d_h5_attr_double(f, sg, "TimeValue", tvals[s]), f, sg);
        const uint64_t dw[2] = {(uint64_t)nx, (uint64_t)nyf}, dff[2] = {(uint64_t)(2 * kmax + 1), (uint64_t)(2 * kmax + 1)};
        const uint64_t dsp[1] = {(uint64_t)n_spec};
        snprintf(path, sizeof(path), "%s/w_hat", sg);
        h5die(ns2d_h5_dataset(f, path, NS2D_H5_C128, 2, dw, w), f, path);
        for (int k = 0; k < 4; ++k) {
            snprintf(path, sizeof(path), "%s/%s", sg, ff_names[k]);
            h5die(ns2d_h5_dataset(f, path, NS2D_H5_F64, 2, dff, ff + (size_t)k * w2), f, path);
        }
        for (int k = 0; k < 8; ++k) {
            snprintf(path, sizeof(path), "%s/%s", sg, sp_names[k]);
            h5die(ns2d_h5_dataset(f, path, NS2D_H5_F64, 1, dsp, spec + (size_t)sp_index[k] * n_spec), f, path);
        }
        if (ps) {
            /* FluxSpectra's sector sums and PhaseSyncSector (post_proc.c:88-104) */
            check(ns2d_nonlinear_rhs(g_h, (const double*)w, (double*)rhs), "NonlinearRHS");
            check(ps_snapshot(ps, w, rhs, ff + w2, ff), "phase sync");
            h5die(ps_write_snapshot(ps, f, sg), f, sg);
        }
        printf("Snapshot: %d\n", s);
    }
    /* FinalWriteAndClose (hdf5_funcs.c:1290-1370) */
    int* kx = (int*)malloc(sizeof(int) * (size_t)nx);
    int* ky = (int*)malloc(sizeof(int) * (size_t)nyf);
    double* x = (double*)malloc(sizeof(double) * (size_t)nx);
    double* y = (double*)malloc(sizeof(double) * (size_t)ny);
    for (long i = 0; i < nx; ++i) {
        kx[i] = (int)(i <= nx / 2 ? i : i - nx);
        x[i] = (double)i * 2.0 * M_PI / (double)nx;
    }
    for (long j = 0; j < ny; ++j) {
        if (j < nyf) ky[j] = (int)j;
        y[j] = (double)j * 2.0 * M_PI / (double)ny;
    }
    const uint64_t dnx[1] = {(uint64_t)nx}, dnyf[1] = {(uint64_t)nyf}, dny[1] = {(uint64_t)ny}, ds[1] = {(uint64_t)snaps};
    h5die(ns2d_h5_dataset(f, "kx", NS2D_H5_I32, 1, dnx, kx), f, "kx");
    h5die(ns2d_h5_dataset(f, "ky", NS2D_H5_I32, 1, dnyf, ky), f, "ky");
    h5die(ns2d_h5_dataset(f, "x", NS2D_H5_F64, 1, dnx, x), f, "x");
    h5die(ns2d_h5_dataset(f, "y", NS2D_H5_F64, 1, dny, y), f, "y");
    h5die(ns2d_h5_dataset(f, "Time", NS2D_H5_F64, 1, ds, tvals), f, "Time");
    static const char* const c_names[4] = {"EnstrophyFluxC", "EnstrophyDissC", "EnergyFluxC", "EnergyDissC"};
    for (int k = 0; k < 4; ++k) h5die(ns2d_h5_dataset(f, c_names[k], NS2D_H5_F64, 1, ds, csum + (size_t)k * snaps), f, c_names[k]);
    if (ps) h5die(ps_write_final(ps, f), f, "phase sync");
    h5die(ns2d_h5_close(f), NULL, out_file);
    const double secs = (double)(clock() - begin) / CLOCKS_PER_SEC;
    printf("\n\nTotal Execution Time: [%5.10lf]\n\n", secs);
    ns2d_destroy(g_h);
    ps_free(ps);
    free(rhs);
    free(w);
    free(spec);
    free(ff);
    free(tvals);
    free(csum);
    free(kx);
    free(ky);
    free(x);
    free(y);
    return 0;
}
