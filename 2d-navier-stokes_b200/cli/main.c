/*
 * main.c -- bin/ns2d: the reference solver program (Solver/src/main.c) on the
 * GPU.
 *
 *   ns2d -o <dir> -n 256 -n 256 -s 0.0 -e 1.0 -h 1e-4 -h 0 -c 1 -c 0.9 \
 *        -v 1e-4 -v 0 -v 2.0 -d 0.0 -d 0 -d -2.0 -i DECAY_TURB_BB -t TAG \
 *        -f NONE -f 0 -f 1.0 -p 100
 *
 * accepts the reference's argv (args.c), builds its initial condition and
 * forcing (init.c), runs SpectralSolve's loop (solver.c:54-251) with the state
 * resident on the GPU (libns2d.so), and writes the reference's output files
 * with the stock dataset flags (Solver/Makefile DSET_FLAGS):
 *   Main_HDF_Data.h5            /Iter_%05d/{w [Nx][Ny], w_hat [Nx][Ny/2+1] {r,i}}
 *   Spectra_HDF_Data.h5         /Iter_%05d/{the eight energy/enstrophy spectra}
 *   SystemMeasures_HDF_Data.h5  time series, mean flows, kx, ky, x, y
 * every group with the TimeValue / TimeStep attributes, and
 * SimulationDetails.txt (hdf5_funcs.c:33-1870, utils.c:468-606).
 *
 * Launched by mpirun (run_solver.py does `mpirun -n P <executable>`) only
 * rank 0 runs; the other ranks exit at once.  Fixed-step runs without
 * host-drawn forcing advance between saves with ns2d_step_n (one replayed
 * CUDA graph per step, the SystemCheck test fused into the step).
 */
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include "ns2d_h5.h"
#include "run.h"

#define MIN_STEP_SIZE 1e-10 /* data_types.h:171 */
#define N_MEASURES 13

static ns2d_handle* g_h = NULL;

static void check(ns2d_status s, const char* what) {
    if (s == NS2D_OK) return;
    fprintf(stderr, "\n[ERROR] ns2d: %s failed: %s (%s)\n-->> Exiting!\n", what, ns2d_status_string(s),
            g_h ? ns2d_last_error(g_h) : "no handle");
    exit(1);
}

static const char* integrator_name(int i) {
    return i == NS2D_RK4 ? "RK4" : i == NS2D_AB4 ? "AB4" : i == NS2D_DP5 ? "DP5" : "RK4CN";
}

static int mpi_rank(void) {
    const char* vars[] = {"OMPI_COMM_WORLD_RANK", "PMI_RANK", "PMIX_RANK", "MV2_COMM_WORLD_RANK", NULL};
    for (int i = 0; vars[i]; ++i) {
        const char* v = getenv(vars[i]);
        if (v && *v) return atoi(v);
    }
    return 0;
}

static void print_json(const ns2d_run* r) {
    printf("{\"N\": [%ld, %ld], \"t0\": %.17g, \"T\": %.17g, \"dt\": %.17g, \"adapt_step\": %d, \"cfl_cond\": %d, "
           "\"cfl_const\": %.17g, \"u0\": \"%s\", \"forcing\": \"%s\", \"force_k\": %d, \"force_scale\": %.17g, "
           "\"trans_iters\": %d, \"trans_frac\": %.17g, \"nu\": %.17g, \"hyper_flag\": %d, \"hyper_pow\": %.17g, "
           "\"ekmn_alpha\": %.17g, \"ekmn_flag\": %d, \"ekmn_pow\": %.17g, \"save_every\": %d, \"output_dir\": \"%s\", "
           "\"output_tag\": \"%s\", \"input_file\": \"%s\", \"file_only\": %d, \"integrator\": \"%s\", "
           "\"dealias\": \"%s\", \"precision\": \"%s\", \"quirks\": %d, \"phase_only\": %d}\n",
           r->N[0], r->N[1], r->t0, r->T, r->dt, r->adapt_step, r->cfl_cond, r->cfl_const, r->u0, r->forcing,
           r->force_k, r->force_scale, r->trans_iters, r->trans_frac, r->nu, r->hyper_flag, r->hyper_pow,
           r->ekmn_alpha, r->ekmn_flag, r->ekmn_pow, r->save_every, r->output_dir, r->output_tag, r->input_file,
           r->file_only, integrator_name(r->integrator), r->dealias == NS2D_DEALIAS_HOU_LI ? "HOU_LI" : "23",
           r->precision == NS2D_FP32 ? "FP32" : "FP64", r->quirks, r->phase_only);
}

/* ---- run state ------------------------------------------------------------------ */
typedef struct state {
    ns2d_run* r;
    ns2d_grid g;
    long nx, ny, nyf;
    int n_spect;
    long num_t_steps, num_print_steps, trans_steps;
    int print_every;
    double min_dt, max_dt;
    long num_msr_counts;
    double* series[N_MEASURES];
    double* time;
    double* mean_x;  /* [nyf] */
    double* mean_y;  /* [nx]  */
    double* spectra; /* 8 * n_spect, of the last measurables call */
    double* w_real;
    double complex* w_hat;
    char main_file[1400], spect_file[1400], msr_file[1400];
    ns2d_h5_file* fmain;
    ns2d_h5_file* fspect;
} state;

static const char* const k_series[N_MEASURES] = {
    "TotalEnergy", "TotalEnstrophy", "TotalPalinstrophy", "TotalForcing", "TotalDivergence", "EnergyDissipation",
    "EnstrophyDissipation", "TimeDerivativeEnergySubset", "EnergyFluxSubset", "EnergyDissSubset",
    "TimeDerivativeEnstrophySubset", "EnstrophyFluxSubset", "EnstrophyDissSubset"};
/* ns2d_system_measurables spectra order -> dataset names */
static const char* const k_spectra[8] = {"EnergySpectrum",
                                         "EnstrophySpectrum",
                                         "TimeDerivativeEnstrophySpectrum",
                                         "EnstrophyFluxSpectrum",
                                         "EnstrophyDissipationSpectrum",
                                         "TimeDerivativeEnergySpectrum",
                                         "EnergyFluxSpectrum",
                                         "EnergyDissipationSpectrum"};
/* order the reference writes them in (hdf5_funcs.c:245-262) */
static const int k_spectra_order[8] = {1, 0, 2, 4, 3, 5, 7, 6};

static void h5check(int rc, ns2d_h5_file* f, const char* what) {
    if (rc == 0) return;
    fprintf(stderr, "\n[ERROR] --- HDF5 output: %s: %s\n-->> Exiting...\n", what, ns2d_h5_error(f));
    exit(1);
}

/* ComputeSystemMeasurables (sys_msr.c:32-373) at save index `iter`. */
static void measurables(state* s, double t, long iter) {
    s->num_msr_counts++;
    if (iter >= s->num_print_steps && iter % 100 == 0)
        printf("\n[WARNING] --- Unable to write system measures at Indx: [%ld] t: [%lf] ---- Number of integration "
               "steps is now greater then memory allocated\n",
               iter, t);
    ns2d_measures m;
    check(ns2d_system_measurables(g_h, &m, s->spectra), "ComputeSystemMeasurables");
    if (iter < s->num_print_steps) {
        const double v[N_MEASURES] = {m.energy,         m.enstrophy,      m.palinstrophy,   m.forcing_input,
                                      m.divergence,     m.energy_diss,    m.enstrophy_diss, m.d_enrg_dt_sbst,
                                      m.enrg_flux_sbst, m.enrg_diss_sbst, m.d_enst_dt_sbst, m.enst_flux_sbst,
                                      m.enst_diss_sbst};
        for (int k = 0; k < N_MEASURES; ++k) s->series[k][iter] = v[k];
        s->time[iter] = t;
    }
    double* mx = (double*)malloc(sizeof(double) * (size_t)s->nyf);
    double* my = (double*)malloc(sizeof(double) * (size_t)s->nx);
    if (!mx || !my) {
        fprintf(stderr, "out of memory\n");
        exit(1);
    }
    check(ns2d_mean_flow(g_h, mx, my), "mean flow");
    for (long j = 0; j < s->nyf; ++j) s->mean_x[j] += mx[j];
    for (long i = 0; i < s->nx; ++i) s->mean_y[i] += my[i];
    free(mx);
    free(my);
}

/* Group /Iter_%05d with its TimeValue / TimeStep attributes (CreateGroup,
   hdf5_funcs.c:1058-1125). */
static void group(ns2d_h5_file* f, const char* name, double t, double dt) {
    if (ns2d_h5_exists(f, name)) return;
    h5check(ns2d_h5_group(f, name), f, name);
    h5check(ns2d_h5_attr_double(f, name, "TimeValue", t), f, name);
    h5check(ns2d_h5_attr_double(f, name, "TimeStep", dt), f, name);
}

/* Fourier amplitudes and phases of the phase-only model, "a_k" = |w_hat| and
   "phi_k" = arg w_hat on [nx][nyf] (WriteDataToFile, hdf5_funcs.c:899-925).
   The initial save of the reference (hdf5_funcs.c:264-290) indexes both
   arrays by the row alone, so entry i holds mode (i, nyf-1) and the rest stay
   0; that form is kept with the reference's quirks on. */
static void write_amplitudes_phases(state* s, const char* gname, int initial) {
    const size_t n = (size_t)(s->nx * s->nyf);
    double* a = (double*)calloc(2 * n, sizeof(double));
    if (!a) {
        fprintf(stderr, "out of memory\n");
        exit(1);
    }
    double* phi = a + n;
    if (initial && s->r->quirks) {
        for (long i = 0; i < s->nx; ++i) {
            const double complex w = s->w_hat[(size_t)i * s->nyf + s->nyf - 1];
            a[i] = cabs(w);
            phi[i] = carg(w);
        }
    } else {
        for (size_t q = 0; q < n; ++q) {
            a[q] = cabs(s->w_hat[q]);
            phi[q] = carg(s->w_hat[q]);
        }
    }
    const uint64_t df[2] = {(uint64_t)s->nx, (uint64_t)s->nyf};
    char path[128];
    snprintf(path, sizeof(path), "%s/a_k", gname);
    h5check(ns2d_h5_dataset(s->fmain, path, NS2D_H5_F64, 2, df, a), s->fmain, path);
    snprintf(path, sizeof(path), "%s/phi_k", gname);
    h5check(ns2d_h5_dataset(s->fmain, path, NS2D_H5_F64, 2, df, phi), s->fmain, path);
    free(a);
}

/* The datasets of one save (WriteDataToFile, hdf5_funcs.c:650-1050; `initial`:
   the initial condition's, CreateOutputFilesWriteICs, hdf5_funcs.c:200-300). */
static void write_save(state* s, double t, double dt, long idx, int initial) {
    char gname[64], path[128];
    snprintf(gname, sizeof(gname), "/Iter_%05d", (int)idx);
    group(s->fmain, gname, t, dt);
    group(s->fspect, gname, t, dt);
    check(ns2d_get_w_real(g_h, s->w_real), "real-space vorticity");
    check(ns2d_get_w_hat(g_h, (double*)s->w_hat), "ns2d_get_w_hat");
    const uint64_t dr[2] = {(uint64_t)s->nx, (uint64_t)s->ny}, df[2] = {(uint64_t)s->nx, (uint64_t)s->nyf};
    snprintf(path, sizeof(path), "%s/w", gname);
    h5check(ns2d_h5_dataset(s->fmain, path, NS2D_H5_F64, 2, dr, s->w_real), s->fmain, path);
    snprintf(path, sizeof(path), "%s/w_hat", gname);
    h5check(ns2d_h5_dataset(s->fmain, path, NS2D_H5_C128, 2, df, s->w_hat), s->fmain, path);
    if (s->r->phase_only) write_amplitudes_phases(s, gname, initial);
    const uint64_t ds[1] = {(uint64_t)s->n_spect};
    for (int k = 0; k < 8; ++k) {
        const int q = k_spectra_order[k];
        snprintf(path, sizeof(path), "%s/%s", gname, k_spectra[q]);
        h5check(ns2d_h5_dataset(s->fspect, path, NS2D_H5_F64, 1, ds, s->spectra + (size_t)q * s->n_spect), s->fspect,
                path);
    }
}

static int make_dir(const char* d) {
    struct stat st;
    if (stat(d, &st) == 0) return 0;
    return mkdir(d, 0700);
}

/* GetOutputDirPath (hdf5_funcs.c:428-648). */
static void output_paths(state* s) {
    ns2d_run* r = s->r;
    if (make_dir(r->output_dir) != 0) {
        fprintf(stderr, "\n[ERROR] --- Unable to create provided output directory [%s]\n-->> Exiting...\n", r->output_dir);
        exit(1);
    }
    char data[1024];
    if (r->file_only) {
        if (!r->quiet) printf("\n[NOTE] --- File only output option selected...\n");
        snprintf(data, sizeof(data),
                 "_SIM[NAV-%s-%s]_N[%ld,%ld]_T[%1.1lf,%g,%1.3lf]_NU[%g,%d,%1.1lf]_DRAG[%g,%d,%1.1lf]_CFL[%1.2lf]_"
                 "FORC[%s,%d,%g]_u0[%s].h5",
                 integrator_name(r->integrator), r->phase_only ? "PO" : "FULL", r->N[0], r->N[1], r->t0, r->dt, r->T, r->nu, r->hyper_flag,
                 r->hyper_pow, r->ekmn_alpha, r->ekmn_flag, r->ekmn_pow, r->cfl_const, r->forcing, r->force_k,
                 r->force_scale, r->u0);
        snprintf(s->main_file, sizeof(s->main_file), "%sMain_HDF_Data%s", r->output_dir, data);
        snprintf(s->spect_file, sizeof(s->spect_file), "%sSpectra_HDF_Data%s", r->output_dir, data);
        /* the reference leaves the measures file unnamed in this mode */
        snprintf(s->msr_file, sizeof(s->msr_file), "%sSystemMeasures_HDF_Data%s", r->output_dir, data);
    } else {
        snprintf(data, sizeof(data),
                 "SIM_DATA_NAVIER_%s_%s_N[%ld,%ld]_T[%1.1lf,%g,%1.3lf]_NU[%g,%d,%1.1lf]_DRAG[%g,%d,%1.1lf]_"
                 "CFL[%1.2lf]_FORC[%s,%d,%g]_u0[%s]_TAG[%s]/",
                 integrator_name(r->integrator), r->phase_only ? "PHAEONLY" : "FULL", r->N[0], r->N[1], r->t0, r->dt, r->T, r->nu, r->hyper_flag,
                 r->hyper_pow, r->ekmn_alpha, r->ekmn_flag, r->ekmn_pow, r->cfl_const, r->forcing, r->force_k,
                 r->force_scale, r->u0, r->output_tag);
        if (strlen(r->output_dir) + strlen(data) >= sizeof(r->output_dir)) {
            fprintf(stderr, "\n[ERROR] --- output path too long\n");
            exit(1);
        }
        strcat(r->output_dir, data);
        if (make_dir(r->output_dir) != 0) {
            fprintf(stderr, "\n[ERROR] --- Unable to create folder for output files [%s]\n-->> Exiting...\n",
                    r->output_dir);
            exit(1);
        }
        snprintf(s->main_file, sizeof(s->main_file), "%sMain_HDF_Data.h5", r->output_dir);
        snprintf(s->msr_file, sizeof(s->msr_file), "%sSystemMeasures_HDF_Data.h5", r->output_dir);
        snprintf(s->spect_file, sizeof(s->spect_file), "%sSpectra_HDF_Data.h5", r->output_dir);
    }
    if (!r->quiet) {
        printf("\nMain Output File: %s\n\n", s->main_file);
        printf("\nSystem Measures File: %s\n\n", s->msr_file);
        printf("Spectra Output File: %s\n\n", s->spect_file);
    }
}

/* FinalWriteAndCloseOutputFiles (hdf5_funcs.c:1371-1800). */
static void final_write(state* s) {
    ns2d_h5_file* f = ns2d_h5_create(s->msr_file);
    if (!f) {
        fprintf(stderr, "\n[ERROR] --- Could not create HDF5 system measures file [%s]: %s\n-->> Exiting...\n",
                s->msr_file, ns2d_h5_error(NULL));
        exit(1);
    }
    const uint64_t dnx[1] = {(uint64_t)s->nx}, dnyf[1] = {(uint64_t)s->nyf}, dny[1] = {(uint64_t)s->ny};
    const uint64_t dsteps[1] = {(uint64_t)s->num_print_steps};
    h5check(ns2d_h5_dataset(f, "kx", NS2D_H5_I32, 1, dnx, s->g.kx), f, "kx");
    h5check(ns2d_h5_dataset(f, "ky", NS2D_H5_I32, 1, dnyf, s->g.ky), f, "ky");
    h5check(ns2d_h5_dataset(f, "x", NS2D_H5_F64, 1, dnx, s->g.x), f, "x");
    h5check(ns2d_h5_dataset(f, "y", NS2D_H5_F64, 1, dny, s->g.y), f, "y");
    h5check(ns2d_h5_dataset(f, "Time", NS2D_H5_F64, 1, dsteps, s->time), f, "Time");
    for (long i = 0; i < s->nx; ++i) s->mean_y[i] /= (double)s->num_msr_counts;
    for (long j = 0; j < s->nyf; ++j) s->mean_x[j] /= (double)s->num_msr_counts;
    h5check(ns2d_h5_dataset(f, "MeanFlow_y", NS2D_H5_F64, 1, dnx, s->mean_y), f, "MeanFlow_y");
    h5check(ns2d_h5_dataset(f, "MeanFlow_x", NS2D_H5_F64, 1, dnyf, s->mean_x), f, "MeanFlow_x");
    for (int k = 0; k < N_MEASURES; ++k)
        h5check(ns2d_h5_dataset(f, k_series[k], NS2D_H5_F64, 1, dsteps, s->series[k]), f, k_series[k]);
    h5check(ns2d_h5_close(f), NULL, s->msr_file);
}

static void close_outputs(state* s) {
    if (s->fmain) h5check(ns2d_h5_close(s->fmain), NULL, s->main_file);
    if (s->fspect) h5check(ns2d_h5_close(s->fspect), NULL, s->spect_file);
    s->fmain = s->fspect = NULL;
}

static void failure(state* s, ns2d_status st, long iters) {
    close_outputs(s);
    if (st == NS2D_ERR_BLOWUP)
        fprintf(stderr, "\n[SOLVER FAILURE] --- System has reached maximum Vorticity limit at Iter: [%ld]\n-->> Exiting!!!\n", iters);
    else if (st == NS2D_ERR_DT)
        fprintf(stderr, "\n[SOLVER FAILURE] --- Timestep has become too small to continue at Iter: [%ld]\n-->> Exiting!!!\n", iters);
    else if (st == NS2D_ERR_ITERS)
        fprintf(stderr, "\n[SOLVER FAILURE] --- The maximum number of iterations has been reached at Iter: [%ld]\n-->> Exiting!!!\n", iters);
    else
        check(st, "SystemCheck");
    exit(1);
}

/* SystemCheck (solver.c:2301-2326): blow-up, step size and iteration limits. */
static void system_check(state* s, double dt, long iters) {
    const ns2d_status st = ns2d_system_check(g_h, dt, iters);
    if (st != NS2D_OK) failure(s, st, iters);
}

/* Issue the fixed-dt steps queued since the last save; SystemCheck's
   vorticity test is fused into them on the GPU. */
static void advance(state* s, long* pending, double dt, long iters) {
    if (*pending <= 0) return;
    const ns2d_status st = ns2d_step_n(g_h, (int32_t)*pending, dt);
    *pending = 0;
    if (st == NS2D_ERR_BLOWUP || st == NS2D_ERR_DT || st == NS2D_ERR_ITERS) failure(s, st, iters);
    check(st, "RK4Step");
}

static void print_update(state* s, long iters, double t, double dt, long idx) {
    if (s->r->quiet) return;
    double max_vort = 0.0;
    check(ns2d_get_max_data(g_h, NS2D_MAX_VORT, &max_vort), "GetMaxData");
    if (idx < 0 || idx >= s->num_print_steps) idx = 0;
    printf("Iter: %ld/%ld\tt: %1.6lf/%1.3lf\tdt: %1.6g \tMax Vort: %1.5g \tKE: %1.5g\tENS: %1.5g\t PAL: %1.5g\t "
           "E_Diss: %1.5g\tEns_Diss: %1.5g\n",
           iters, s->num_t_steps, t, s->r->T, dt, max_vort, s->series[0][idx], s->series[1][idx], s->series[2][idx],
           s->series[5][idx], s->series[6][idx]);
}

/* PrintSimulationDetails (utils.c:468-606). */
static void simulation_details(state* s, int argc, char** argv, double sim_time, long tot_iters, long tot_saves) {
    const ns2d_run* r = s->r;
    char path[1200];
    snprintf(path, sizeof(path), "%sSimulationDetails.txt", r->output_dir);
    FILE* f = fopen(path, "w");
    if (!f) return;
    fprintf(f, "Executing Command:\n\n\t");
    for (int i = 0; i < argc; ++i) fprintf(f, "%s ", argv[i]);
    fprintf(f, "\n\n");
    fprintf(f, "Systen Type: NAVIER\nSolver Type: %s\nModel Type: %s\n", integrator_name(r->integrator),
            r->phase_only ? "PHAEONLY" : "FULL");
    fprintf(f, "Viscosity: %1.6lf\n", r->nu);
    fprintf(f, "Re: %5.1lf\n", 1.0 / r->nu);
    fprintf(f, "Ekman Drag: %s\n", r->ekmn_flag ? "YES" : "NO");
    if (r->ekmn_flag) fprintf(f, "Ekman Alpha: %1.4lf\nEkman Power: %1.1lf\n", r->ekmn_alpha, r->ekmn_pow);
    fprintf(f, "Hyperviscosity: %s\n", r->hyper_flag ? "YES" : "NO");
    if (r->hyper_flag) fprintf(f, "Hyperviscosity Power: %1.1lf\n", r->hyper_pow);
    fprintf(f, "\nCollocation Points: [%ld, %ld]\n", r->N[0], r->N[1]);
    fprintf(f, "Spatial Increment: [%1.4lf, %1.4lf]\n", 2.0 * M_PI / (double)r->N[0], 2.0 * M_PI / (double)r->N[1]);
    fprintf(f, "Fourier Modes: [%ld, %ld]\n\n", r->N[0], r->N[1] / 2 + 1);
    fprintf(f, "Initial Conditions: %s\n", r->u0);
    fprintf(f, "Dealiasing: %s\n", r->dealias == NS2D_DEALIAS_HOU_LI ? "HOU-LI" : "2/3 RDS");
    fprintf(f, "Forcing Type: %s\n\n", r->forcing);
    fprintf(f, "Time Range: [%1.1lf - %1.1lf]\n", r->t0, r->T);
    fprintf(f, "Finishing Timestep: %1.10lf\n", r->dt);
    fprintf(f, "CFL No.: %1.5lf\n", r->cfl_const);
    if (r->adapt_step) {
        fprintf(f, "Adaptive Stepping: YES\n");
        fprintf(f, "CFL Stepping Mode: %s\n", r->cfl_cond ? "YES" : "NO");
        fprintf(f, "Total Timesteps: %ld\n", s->num_t_steps);
        fprintf(f, "Total Timesteps Executed: %ld\n", tot_iters);
        fprintf(f, "Timestep Range [min - max]: [%1.10lf - %1.10lf]\n", s->min_dt, s->max_dt);
    } else {
        fprintf(f, "Adaptive Stepping: NO\n");
        fprintf(f, "Total Timesteps: %ld\n", s->num_t_steps);
    }
    fprintf(f, "Data Saved Every: %d\n", s->print_every);
    fprintf(f, "Total Saving Steps: %ld\n", tot_saves);
    const int hh = (int)sim_time / 3600;
    const int mm = ((int)sim_time - hh * 3600) / 60;
    const int ss = (int)(sim_time - hh * 3600 - mm * 60);
    fprintf(f, "\n\nTotal Execution Time: %5.10lf --> %d hrs : %d mins : %d secs\n\n", sim_time, hh, mm, ss);
    fclose(f);
}

static int pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

static void* xcalloc(size_t n, size_t sz) {
    void* p = calloc(n ? n : 1, sz);
    if (!p) {
        fprintf(stderr, "out of memory\n");
        exit(1);
    }
    return p;
}

int main(int argc, char** argv) {
    ns2d_run run;
    ns2d_cli_parse(argc, argv, &run);
    if (run.dry_run) {
        print_json(&run);
        return 0;
    }
    if (mpi_rank() > 0) return 0; /* one GPU process per job; other ranks have nothing to do */
    const clock_t begin = clock();
    if (run.N[0] != run.N[1] || !pow2(run.N[0]) || run.N[0] < 16 || run.N[0] > 2048) {
        fprintf(stderr, "\n[ERROR] ns2d runs square power-of-two grids of 16..2048 points per side; got [%ld, %ld]\n-->> Exiting!\n",
                run.N[0], run.N[1]);
        return 1;
    }
    state s;
    memset(&s, 0, sizeof(s));
    s.r = &run;
    s.nx = run.N[0];
    s.ny = run.N[1];
    s.nyf = run.N[1] / 2 + 1;
    if (ns2d_grid_init(&s.g, s.nx, s.ny)) {
        fprintf(stderr, "out of memory\n");
        return 1;
    }

    /* the handle: parameters of sys_vars and the compile-time switches */
    ns2d_params p;
    ns2d_params_default(&p);
    p.nx = (int32_t)s.nx;
    p.ny = (int32_t)s.ny;
    p.system = NS2D_NAVIER;
    p.integrator = run.integrator;
    p.dealias = run.dealias;
    p.forcing = !strcmp(run.forcing, "KOLM")   ? NS2D_FORCING_KOLM
                : !strcmp(run.forcing, "ZERO") ? NS2D_FORCING_ZERO
                                               : NS2D_FORCING_NONE;
    p.force_k = run.force_k;
    p.force_scale = run.force_scale;
    p.quirks = run.quirks;
    p.nu = run.nu;
    p.hyper_visc_flag = run.hyper_flag;
    p.hyper_visc_pow = run.hyper_pow;
    p.ekmn_alpha = run.ekmn_alpha;
    p.ekmn_drag_flag = run.ekmn_flag;
    p.ekmn_drag_pow = run.ekmn_pow;
    p.adapt_step_flag = run.adapt_step;
    p.cfl_cond_flag = run.cfl_cond;
    p.cfl_const = run.cfl_const;
    p.dt = run.dt;
    p.precision = run.precision;
    p.flux_diagnostics = 1;
    p.device = run.device;
    p.model = run.phase_only ? NS2D_MODEL_PHASE_ONLY : NS2D_MODEL_FULL;
    check(ns2d_create(&p, &g_h), "ns2d_create");

    /* InitialConditions + InitializeForcing (solver.c:1107, force.c:28) */
    s.w_hat = (double complex*)xcalloc((size_t)(s.nx * s.nyf), sizeof(double complex));
    s.w_real = (double*)xcalloc((size_t)(s.nx * s.ny), sizeof(double));
    if (ns2d_cli_initial(&run, &s.g, g_h, s.w_hat)) return 1;
    check(ns2d_set_w_hat(g_h, (const double*)s.w_hat), "ns2d_set_w_hat");
    double w_max_init = 0.0;
    check(ns2d_get_max_data(g_h, NS2D_MAX_VORT, &w_max_init), "GetMaxData");
    check(ns2d_set_w_max_init(g_h, w_max_init), "w_max_init");
    ns2d_forcing_modes fm;
    if (ns2d_cli_forcing_init(&run, &s.g, &fm)) {
        fprintf(stderr, "out of memory\n");
        return 1;
    }
    if (fm.kind == 3) check(ns2d_set_forcing_modes(g_h, fm.n, fm.indx, (const double*)fm.value), "forcing");

    /* InitializeIntegrationVariables (solver.c:2116-2163) */
    if (run.adapt_step) check(ns2d_get_timestep(g_h, &run.dt), "GetTimestep");
    const double T = run.T;
    double t = run.t0, dt = run.dt;
    s.min_dt = 10;
    s.max_dt = MIN_STEP_SIZE;
    s.num_t_steps = (long)((T - run.t0) / dt);
    if (run.trans_iters) {
        s.trans_steps = (long)(run.trans_frac * s.num_t_steps);
        s.num_print_steps = (s.num_t_steps >= run.save_every) ? (s.num_t_steps - s.trans_steps) / run.save_every
                                                              : s.num_t_steps - s.trans_steps;
        if (!run.quiet)
            printf("Total Iters: %ld\t Saving Iters: %ld\t Transient Steps: %ld\n", s.num_t_steps, s.num_print_steps,
                   s.trans_steps);
    } else {
        s.trans_steps = 0;
        s.num_print_steps = (s.num_t_steps >= run.save_every) ? s.num_t_steps / run.save_every + 1 : s.num_t_steps + 1;
        if (!run.quiet) printf("Total Iters: %ld\t Saving Iters: %ld\n", s.num_t_steps, s.num_print_steps);
    }
    s.print_every = (s.num_t_steps >= 10) ? run.save_every : 1;

    /* InitializeSystemMeasurables (sys_msr.c:378-615) */
    if (run.adapt_step) s.num_print_steps *= 2;
    if (s.num_print_steps < 1) s.num_print_steps = 1;
    int32_t dnx, dny, dnyf, nsp;
    check(ns2d_dims(g_h, &dnx, &dny, &dnyf, &nsp), "ns2d_dims");
    s.n_spect = nsp;
    for (int k = 0; k < N_MEASURES; ++k) s.series[k] = (double*)xcalloc((size_t)s.num_print_steps, sizeof(double));
    s.time = (double*)xcalloc((size_t)s.num_print_steps, sizeof(double));
    s.mean_x = (double*)xcalloc((size_t)s.nyf, sizeof(double));
    s.mean_y = (double*)xcalloc((size_t)s.nx, sizeof(double));
    s.spectra = (double*)xcalloc((size_t)(8 * s.n_spect), sizeof(double));
    measurables(&s, 0.0, 0);

    /* CreateOutputFilesWriteICs (hdf5_funcs.c:33-420) */
    output_paths(&s);
    s.fmain = ns2d_h5_create(s.main_file);
    if (!s.fmain) h5check(-1, NULL, s.main_file);
    s.fspect = ns2d_h5_create(s.spect_file);
    if (!s.fspect) h5check(-1, NULL, s.spect_file);
    if (!run.trans_iters) write_save(&s, 0.0, dt, 0, 1);

    /* SpectralSolve's loop (solver.c:127-236) */
    const int listed = fm.kind != 0;
    const int batched = !run.adapt_step && !listed && (run.integrator == NS2D_RK4 || run.integrator == NS2D_RK4CN);
    t += dt;
    long iters = 1;
    long save_idx = run.trans_iters ? 0 : 1;
    long pending = 0; /* fixed-dt steps not yet issued (batched mode) */
    int dp_fails = 0;
    double* dp_save = NULL;
    while (t <= T) {
        if (batched) {
            pending++;
        } else if (run.integrator == NS2D_DP5) {
            /* Dormand-Prince with the accept/retry test the right way round
               (the reference's solver.c:153-171 retries when err < 1) */
            if (!dp_save) dp_save = (double*)xcalloc(2 * (size_t)(s.nx * s.nyf), sizeof(double));
            check(ns2d_get_w_hat(g_h, dp_save), "ns2d_get_w_hat");
            for (;;) {
                double err = 0.0;
                if (listed) {
                    ns2d_cli_forcing_draw(&fm, dt);
                    check(ns2d_set_forcing_modes(g_h, fm.n, fm.indx, (const double*)fm.value), "forcing");
                }
                check(ns2d_dp5_step(g_h, dt, &err), "RK5DPStep");
                const double dt_new = dt * fmin(1.5, fmax(0.01, 0.8 * pow(1.0 / err, 0.2)));
                if (isfinite(err) && err <= 1.0) {
                    dt = dt_new;
                    break;
                }
                dp_fails++;
                check(ns2d_set_w_hat(g_h, dp_save), "ns2d_set_w_hat");
                check(ns2d_set_w_max_init(g_h, w_max_init), "w_max_init");
                dt = dt_new;
                if (dt <= MIN_STEP_SIZE) failure(&s, NS2D_ERR_DT, iters);
            }
        } else {
            if (listed) {
                ns2d_cli_forcing_draw(&fm, dt);
                check(ns2d_set_forcing_modes(g_h, fm.n, fm.indx, (const double*)fm.value), "forcing");
            }
            if (run.integrator == NS2D_AB4)
                check(ns2d_ab4_step(g_h, dt, (int32_t)iters), "AB4Step");
            else
                check(ns2d_rk4_step(g_h, dt), "RK4Step");
        }
        const int save_now = (iters % run.save_every == 0);
        if (save_now) {
            advance(&s, &pending, dt, iters);
            measurables(&s, t, save_idx);
            if (iters > s.trans_steps) {
                write_save(&s, t, dt, save_idx, 0);
                save_idx++;
            }
        }
        if (run.trans_iters && iters == s.trans_steps && !run.quiet) printf("\n\n...Transient Iterations Complete!\n\n");
        if (save_now) print_update(&s, iters, t, dt, iters <= s.trans_steps ? 0 : save_idx - 1);
        iters++;
        if (run.adapt_step) {
            check(ns2d_get_timestep(g_h, &dt), "GetTimestep");
            s.min_dt = fmin(dt, s.min_dt);
            s.max_dt = fmax(dt, s.max_dt);
            t += dt;
        } else if (run.integrator == NS2D_DP5) {
            t += dt;
        } else {
            t = iters * dt;
        }
        if (!batched) system_check(&s, dt, iters);
    }
    advance(&s, &pending, dt, iters);
    if (batched) system_check(&s, dt, iters);
    free(dp_save);
    run.dt = dt;

    /* FinalWriteAndCloseOutputFiles (hdf5_funcs.c:1371) */
    close_outputs(&s);
    final_write(&s);
    const long tot_iters = iters - 1, tot_saves = save_idx - 1;
    const double sim_time = (double)(clock() - begin) / CLOCKS_PER_SEC;
    if (!run.quiet) {
        const int hh = (int)sim_time / 3600, mm = ((int)sim_time - hh * 3600) / 60;
        const int ss = (int)(sim_time - hh * 3600 - mm * 60);
        printf("\n\nTotal Execution Time: [%5.10lf] --> %d hrs : %d mins : %d secs\n\n", sim_time, hh, mm, ss);
        if (run.integrator == NS2D_DP5) printf("DP5 rejected steps: %d\n", dp_fails);
    }
    if (!run.file_only) simulation_details(&s, argc, argv, sim_time, tot_iters, tot_saves);
    ns2d_cli_forcing_free(&fm);
    for (int k = 0; k < N_MEASURES; ++k) free(s.series[k]);
    free(s.time);
    free(s.mean_x);
    free(s.mean_y);
    free(s.spectra);
    free(s.w_hat);
    free(s.w_real);
    ns2d_grid_free(&s.g);
    ns2d_destroy(g_h);
    return 0;
}
