/*
 * oracle/ref_harness.c -- drives the reference solver's OWN compiled sources
 * (Solver/src/solver.c, force.c, sys_msr.c, built unmodified against the
 * single-rank stand-ins in oracle/shim/) through a small C API that the tests
 * load with ctypes.  Test infrastructure only: the product never links this.
 *
 * It plays the part of Solver/src/main.c:33-60 (global struct set-up) and of
 * SpectralSolve's set-up sequence (Solver/src/solver.c:54-115: AllocateMemory,
 * InitializeFFTWPlans, InitializeSpaceVariables, InitialConditions,
 * InitializeForcing, InitializeSystemMeasurables), then exposes the per-step
 * entry points (RK4Step, AB4Step, NonlinearRHSBatch, GetTimestep, GetMaxData,
 * ComputeSystemMeasurables) one call at a time.
 */
#include <complex.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "data_types.h"
#include "solver.h"
#include "sys_msr.h"
#include "force.h"
#include "../fft.h"

runtime_data_struct* run_data;
system_vars_struct* sys_vars;
HDF_file_info_struct* file_info;
stats_data_struct* stats_data;

static runtime_data_struct g_run;
static system_vars_struct g_sys;
static HDF_file_info_struct g_file;
static stats_data_struct g_stats;
static Int_data_struct g_int;
static long int g_N[2];
static int g_ready = 0;

/* Parameters a run takes from the command line (Solver/src/utils.c:51-90). */
typedef struct ref_params {
    int nx, ny;
    double nu;
    int hyper_visc_flag;
    double hyper_visc_pow;
    double ekmn_alpha;
    int ekmn_drag_flag;
    double ekmn_drag_pow;
    int force_k;
    double force_scale;
    double dt;
    double t0, T;
    int adapt_step_flag;
    int cfl_cond_flag;
    double cfl_const;
    int save_every;
    int num_print_steps;
    char forcing[64];
    char u0[64];
} ref_params;

int ref_variant(void) {
#if defined(__DPRK5)
    return 3;
#elif defined(__AB4)
    return 2;
#elif defined(__RK4)
    return 1;
#else
    return 0;
#endif
}

/* main.c:33-60 and GetCMLArgs: globals and parameters, no allocation. */
static void set_globals(const ref_params* p, int threads) {
    offt_set_threads(threads);
    memset(&g_run, 0, sizeof g_run);
    memset(&g_sys, 0, sizeof g_sys);
    memset(&g_file, 0, sizeof g_file);
    memset(&g_stats, 0, sizeof g_stats);
    memset(&g_int, 0, sizeof g_int);
    run_data = &g_run;
    sys_vars = &g_sys;
    file_info = &g_file;
    stats_data = &g_stats;
    sys_vars->num_procs = 1;
    sys_vars->rank = 0;
    sys_vars->N[0] = p->nx;
    sys_vars->N[1] = p->ny;
    sys_vars->NU = p->nu;
    sys_vars->HYPER_VISC_FLAG = p->hyper_visc_flag;
    sys_vars->HYPER_VISC_POW = p->hyper_visc_pow;
    sys_vars->EKMN_ALPHA = p->ekmn_alpha;
    sys_vars->EKMN_DRAG_FLAG = p->ekmn_drag_flag;
    sys_vars->EKMN_DRAG_POW = p->ekmn_drag_pow;
    sys_vars->force_k = p->force_k;
    sys_vars->force_scale_var = p->force_scale;
    sys_vars->dt = p->dt;
    sys_vars->t0 = p->t0;
    sys_vars->T = p->T;
    sys_vars->ADAPT_STEP_FLAG = p->adapt_step_flag;
    sys_vars->CFL_COND_FLAG = p->cfl_cond_flag;
    sys_vars->CFL_CONST = p->cfl_const;
    sys_vars->SAVE_EVERY = p->save_every;
    sys_vars->num_print_steps = p->num_print_steps > 0 ? p->num_print_steps : 4;
    strncpy(sys_vars->forcing, p->forcing, 63);
    strncpy(sys_vars->u0, p->u0, 63);
    g_N[0] = p->nx;
    g_N[1] = p->ny;
}

int ref_init(const ref_params* p, int run_initial_conditions, int threads) {
    if (g_ready) return -1;
    set_globals(p, threads);
    const long int NBatch[2] = {p->nx, p->ny / 2 + 1};
#if defined(__DPRK5)
    /* AllocateMemory's __DPRK5 branch zeroes the Adams-Bashforth arrays
       (Solver/src/solver.c:2850-2856), which only its __AB4 branch allocates
       (:2774-2791); the harness provides them so that the reference's own
       AllocateMemory runs unchanged.  They live for the process. */
    {
        const size_t batch = 2 * (size_t)p->nx * (size_t)(p->ny / 2 + 1);
        g_int.AB_tmp = (fftw_complex*)calloc(batch, sizeof(fftw_complex));
        for (int a = 0; a < 3; ++a) g_int.AB_tmp_nonlin[a] = (fftw_complex*)calloc(batch, sizeof(fftw_complex));
    }
#endif
    AllocateMemory(NBatch, &g_int);
    InitializeFFTWPlans(g_N);
    InitializeSpaceVariables(run_data->x, run_data->k, g_N);
    if (run_initial_conditions) InitialConditions(run_data->w_hat, run_data->u, run_data->u_hat, g_N);
    InitializeForcing();
    /* InitializeSystemMeasurables allocates the diagnostics arrays and evaluates
       them once at t = 0 (which also runs NonlinearRHSBatch on w_hat). */
    InitializeSystemMeasurables(&g_int);
    g_ready = 1;
    return 0;
}

static size_t nspec(void) { return (size_t)g_N[0] * (size_t)(g_N[1] / 2 + 1); }

void ref_set_w_hat(const double* in) { memcpy(run_data->w_hat, in, sizeof(fftw_complex) * nspec()); }
void ref_get_w_hat(double* out) { memcpy(out, run_data->w_hat, sizeof(fftw_complex) * nspec()); }
void ref_get_k(int* kx, int* ky) {
    memcpy(kx, run_data->k[0], sizeof(int) * (size_t)g_N[0]);
    memcpy(ky, run_data->k[1], sizeof(int) * (size_t)(g_N[1] / 2 + 1));
}
int ref_hyper_visc_flag(void) { return sys_vars->HYPER_VISC_FLAG; }
void ref_set_hyper_visc_flag(int f) { sys_vars->HYPER_VISC_FLAG = f; }
void ref_compute_forcing(double dt) { ComputeForcing(dt); }
/* Host threads of the stand-in FFT (FFTW-MPI's place); the reference's own
   loops stay single-threaded, as in one MPI rank. */
void ref_set_threads(int threads) { offt_set_threads(threads); }

#if defined(__RK4) || defined(__RK4CN) || defined(__AB4)
void ref_rk4_step(double dt) { RK4Step(dt, g_N, sys_vars->local_Nx, &g_int); }
#endif

#if defined(__DPRK5)
/* One RK5DPStep (Solver/src/solver.c:360-570) at SpectralSolve iteration
   `iters`, called directly (SpectralSolve's accept/retry loop, :150-171, is
   not run); returns Int_data->DP_err, which the step sets only when iters > 1. */
double ref_dp5_step(double dt, int iters) {
    RK5DPStep(dt, g_N, iters, sys_vars->local_Nx, &g_int);
    return g_int.DP_err;
}
#endif

#if defined(__AB4)
void ref_ab4_step(double dt, int iters) { AB4Step(dt, g_N, iters, sys_vars->local_Nx, &g_int); }
#endif

/* NonlinearRHSBatch on the state itself (stage-1 form) or on a copy of `in`
   placed in RK_tmp (stage 2-4 form).  Both keep the ForceConjugacy side effect
   on run_data->w_hat (Solver/src/solver.c:1031). */
void ref_nonlinear_rhs_state(double* out) {
    NonlinearRHSBatch(run_data->w_hat, g_int.RK1, g_int.nonlin, g_int.nabla_psi, g_int.nabla_w);
    memcpy(out, g_int.RK1, sizeof(fftw_complex) * nspec());
}
void ref_nonlinear_rhs_input(const double* in, double* out) {
    memcpy(g_int.RK_tmp, in, sizeof(fftw_complex) * nspec());
    NonlinearRHSBatch(g_int.RK_tmp, g_int.RK1, g_int.nonlin, g_int.nabla_psi, g_int.nabla_w);
    memcpy(out, g_int.RK1, sizeof(fftw_complex) * nspec());
}

void ref_apply_dealiasing(double* arr, int dim) { ApplyDealiasing((fftw_complex*)arr, dim, g_N); }
void ref_force_conjugacy(double* arr) { ForceConjugacy((fftw_complex*)arr, g_N); }
double ref_get_max_vort(void) { return GetMaxData("VORT"); }
double ref_get_max_vel(void) { return GetMaxData("VEL"); }
double ref_get_timestep(double dt) { GetTimestep(&dt); return dt; }
double ref_w_max_init(void) { return sys_vars->w_max_init; }
void ref_set_w_max_init(double w) { sys_vars->w_max_init = w; }
void ref_set_dt(double dt) { sys_vars->dt = dt; }

/* Real-space fields last written by GetMaxData (padded [Nx][Ny+2] rows). */
void ref_get_w_real(double* out) { memcpy(out, run_data->w, sizeof(double) * (size_t)g_N[0] * (size_t)(g_N[1] + 2)); }

int ref_n_spect(void) { return sys_vars->n_spect; }

/* ComputeSystemMeasurables at save index `iter`; scalars in the order
   E, Z, P, forcing, divergence, energy diss, enstrophy diss,
   d_enrg_dt_sbst, enrg_flux_sbst, enrg_diss_sbst, d_enst_dt_sbst,
   enst_flux_sbst, enst_diss_sbst; spectra (n_spect each) in the order
   enrg, enst, d_enst_dt, enst_flux, enst_diss, d_enrg_dt, enrg_flux, enrg_diss. */
void ref_system_measurables(double t, int iter, double* scalars, double* spectra) {
    ComputeSystemMeasurables(t, iter, &g_int);
    double s[13] = {run_data->tot_energy[iter], run_data->tot_enstr[iter], run_data->tot_palin[iter],
                    run_data->tot_forc[iter],   run_data->tot_div[iter],   run_data->enrg_diss[iter],
                    run_data->enst_diss[iter],  run_data->d_enrg_dt_sbst[iter], run_data->enrg_flux_sbst[iter],
                    run_data->enrg_diss_sbst[iter], run_data->d_enst_dt_sbst[iter],
                    run_data->enst_flux_sbst[iter], run_data->enst_diss_sbst[iter]};
    memcpy(scalars, s, sizeof s);
    int n = sys_vars->n_spect;
    double* src[8] = {run_data->enrg_spect, run_data->enst_spect, run_data->d_enst_dt_spect,
                      run_data->enst_flux_spect, run_data->enst_diss_spect, run_data->d_enrg_dt_spect,
                      run_data->enrg_flux_spect, run_data->enrg_diss_spect};
    for (int i = 0; i < 8; ++i) memcpy(spectra + (size_t)i * n, src[i], sizeof(double) * (size_t)n);
}

/* The reference's own time loop, SpectralSolve (Solver/src/solver.c:54-251),
   from the initial condition named by p->u0 over [t0, T] with SAVE_EVERY =
   p->save_every: it allocates, runs and frees everything itself, as under
   main.c.  The state at each save (WriteDataToFile) is kept for
   ref_saved_w_hat.  Once per process. */
extern void (*shim_write_hook)(double t, long int iters);
static double* g_saved = NULL;
static double g_saved_t = 0.0;
static long int g_saved_count = 0;

static void keep_saved_state(double t, long int iters) {
    (void)iters;
    memcpy(g_saved, run_data->w_hat, sizeof(fftw_complex) * nspec());
    g_saved_t = t;
    g_saved_count++;
}

int ref_solve(const ref_params* p, int threads) {
    if (g_ready) return -1;
    set_globals(p, threads);
    sys_vars->TRANS_ITERS_FLAG = 0;
    g_saved = (double*)calloc(2 * nspec(), sizeof(double));
    if (!g_saved) return -2;
    shim_write_hook = keep_saved_state;
    g_ready = 1;
    SpectralSolve();
    shim_write_hook = 0;
    return 0;
}

long int ref_saved_w_hat(double* out, double* t) {
    if (g_saved) memcpy(out, g_saved, sizeof(double) * 2 * nspec());
    *t = g_saved_t;
    return g_saved_count;
}
