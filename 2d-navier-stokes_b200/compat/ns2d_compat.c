/*
 * ns2d_compat.c -- the reference solver's own per-step entry points, under
 * their own names and signatures (Solver/src/solver.h:26, 39-41, 53, 55),
 * implemented over libns2d.so.  Linked into the reference program in place of
 * the FFTW-MPI definitions in Solver/src/solver.c, it moves RK4Step,
 * NonlinearRHSBatch, ApplyDealiasing, GetMaxData and GetTimestep onto the GPU
 * while SpectralSolve, InitialConditions, ComputeSystemMeasurables, the HDF5
 * output and everything else run unchanged.
 *
 * Build: compile this file against the reference's headers (data_types.h,
 * solver.h and the FFTW/MPI/HDF5 headers they include) with the same -D flags
 * as the reference build, and link it before solver.o, whose definitions of
 * the six symbols below must give way (objcopy --weaken-symbol, or removal).
 * 2d-navier-stokes_b200/Makefile target `compat` does the compile.
 *
 * State: the reference keeps w_hat in host memory (run_data->w_hat).  Every
 * call copies what it needs to the device and back, so the reference's code
 * between calls sees exactly the arrays it expects.  One handle per process,
 * created from sys_vars on the first call.  Failures print the ns2d message
 * and exit(1), the reference's own convention (solver.c:2314-2325).
 *
 * Differences from the replaced bodies: NonlinearRHSBatch and GetMaxData do
 * not fill the real-space scratch arrays they are passed (nonlinear, u, w, and
 * run_data->u / run_data->w for GetMaxData); the reference's callers use only
 * the spectral output and the returned maximum.
 */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "data_types.h"
#include "solver.h"
#include "force.h"
#include "ns2d.h"

static ns2d_handle* g_ns2d = NULL;

static void ns2d_compat_check(ns2d_status s, const char* what) {
    if (s == NS2D_OK) return;
    fprintf(stderr, "\n[ERROR] ns2d: %s failed: %s (%s)\n-->> Exiting!\n", what, ns2d_status_string(s),
            g_ns2d ? ns2d_last_error(g_ns2d) : "no handle");
    exit(1);
}

/* Forcings whose values the reference draws on the host each step (STOC,
   STOC_GAUSS, CONST_GAUSS: force.c:104-433, 540-577). */
static int ns2d_compat_listed_forcing(void) {
    return !strcmp(sys_vars->forcing, "STOC") || !strcmp(sys_vars->forcing, "STOC_GAUSS") ||
           !strcmp(sys_vars->forcing, "CONST_GAUSS");
}

/* Handle built from sys_vars (filled by GetCMLArgs, utils.c:51-460) and the
   compile-time switches of data_types.h. */
static ns2d_handle* ns2d_compat_handle(void) {
    if (g_ns2d) return g_ns2d;
    ns2d_params p;
    ns2d_params_default(&p);
    p.nx = (int32_t)sys_vars->N[0];
    p.ny = (int32_t)sys_vars->N[1];
#if defined(__EULER)
    p.system = NS2D_EULER;
#endif
#if defined(__RK4)
    p.integrator = NS2D_RK4;
#elif defined(__AB4)
    p.integrator = NS2D_AB4;
#else
    p.integrator = NS2D_RK4CN;
#endif
#if defined(__DEALIAS_HOU_LI)
    p.dealias = NS2D_DEALIAS_HOU_LI;
#else
    p.dealias = NS2D_DEALIAS_23;
#endif
    if (!strcmp(sys_vars->forcing, "KOLM")) {
        p.forcing = NS2D_FORCING_KOLM;
    } else if (!strcmp(sys_vars->forcing, "ZERO")) {
        p.forcing = NS2D_FORCING_ZERO;
    } else if (!strcmp(sys_vars->forcing, "NONE") || ns2d_compat_listed_forcing()) {
        p.forcing = NS2D_FORCING_NONE;  /* listed-mode forcing goes in by ns2d_set_forcing_modes */
    } else {
        fprintf(stderr, "\n[ERROR] ns2d: forcing \"%s\" is not on the GPU path\n-->> Exiting!\n", sys_vars->forcing);
        exit(1);
    }
    p.force_k = sys_vars->force_k;
    p.force_scale = sys_vars->force_scale_var;
    p.quirks = NS2D_QUIRKS_REFERENCE;
    p.nu = sys_vars->NU;
    p.hyper_visc_flag = sys_vars->HYPER_VISC_FLAG;
    p.hyper_visc_pow = sys_vars->HYPER_VISC_POW;
    p.ekmn_alpha = sys_vars->EKMN_ALPHA;
    p.ekmn_drag_flag = sys_vars->EKMN_DRAG_FLAG;
    p.ekmn_drag_pow = sys_vars->EKMN_DRAG_POW;
    p.adapt_step_flag = sys_vars->ADAPT_STEP_FLAG;
    p.cfl_cond_flag = sys_vars->CFL_COND_FLAG;
    p.cfl_const = sys_vars->CFL_CONST;
    p.dt = sys_vars->dt;
    p.precision = NS2D_FP64;
    ns2d_compat_check(ns2d_create(&p, &g_ns2d), "ns2d_create");
    return g_ns2d;
}

/* The current run_data->forcing values of a listed-mode forcing, to the GPU. */
static void ns2d_compat_sync_forcing(ns2d_handle* h) {
    if (!ns2d_compat_listed_forcing() || !sys_vars->local_forcing_proc) return;
    ns2d_compat_check(ns2d_set_forcing_modes(h, (int32_t)sys_vars->num_forced_modes, run_data->forcing_indx,
                                             (const double*)run_data->forcing),
                      "forcing");
}

/* RK4Step (solver.c:625): one step of run_data->w_hat, in place.  The host
   side effects of the replaced body are kept: the forcing values of this step
   (ComputeForcing, solver.c:650), which ComputeSystemMeasurables reads, and
   the `=` in the viscous-branch test that sets HYPER_VISC_FLAG whenever Ekman
   drag is off (solver.c:675, 843). */
void RK4Step(const double dt, const long int* N, const ptrdiff_t local_Nx, Int_data_struct* Int_data) {
    (void)N;
    (void)local_Nx;
    (void)Int_data;
    ns2d_handle* h = ns2d_compat_handle();
    ComputeForcing(dt);
    ns2d_compat_sync_forcing(h);
    ns2d_compat_check(ns2d_rk4_step_host(h, (double*)run_data->w_hat, dt), "RK4Step");
#if !defined(__EULER)
    if (sys_vars->EKMN_DRAG_FLAG != EKMN_DRAG) sys_vars->HYPER_VISC_FLAG = HYPER_VISC;
#endif
}

/* ForceConjugacy (solver.c:2074): the ky = 0 entries of run_data->w_hat with
   kx < 0 become the conjugates of the input's entries at |kx|.  O(Nx) host
   work, done where the array lives. */
void ForceConjugacy(fftw_complex* w_hat, const long int* N) {
    const long int nx = N[0];
    const long int nyf = N[1] / 2 + 1;
    double* dst = (double*)run_data->w_hat;
    const double* src = (const double*)w_hat;
    for (long int i = nx / 2 + 1; i < nx; ++i) {
        const long int from = nx - i;  /* |kx| for row i, kx = i - nx */
        const double re = src[2 * (from * nyf)];
        const double im = src[2 * (from * nyf) + 1];
        dst[2 * (i * nyf)] = re;
        dst[2 * (i * nyf) + 1] = -im;
    }
}

/* NonlinearRHSBatch (solver.c:884): dw_hat_dt = RHS(w_hat), then the
   ForceConjugacy side effect on run_data->w_hat that the reference applies
   (solver.c:1031). */
void NonlinearRHSBatch(fftw_complex* w_hat, fftw_complex* dw_hat_dt, double* nonlinear, double* u, double* w) {
    (void)nonlinear;
    (void)u;
    (void)w;
    ns2d_handle* h = ns2d_compat_handle();
    const long int N[2] = {sys_vars->N[0], sys_vars->N[1]};
    ns2d_compat_sync_forcing(h);
    ns2d_compat_check(ns2d_nonlinear_rhs(h, (const double*)w_hat, (double*)dw_hat_dt), "NonlinearRHSBatch");
    ForceConjugacy(w_hat, N);
}

/* ApplyDealiasing (solver.c:1039) on array_dim interleaved fields, in place. */
void ApplyDealiasing(fftw_complex* array, int array_dim, const long int* N) {
    (void)N;
    ns2d_compat_check(ns2d_apply_dealiasing(ns2d_compat_handle(), (double*)array, array_dim), "ApplyDealiasing");
}

/* GetMaxData (solver.c:2171) of run_data->w_hat: "VORT", "VEL" or "VORT_FOUR". */
double GetMaxData(char* dtype) {
    ns2d_handle* h = ns2d_compat_handle();
    int32_t kind;
    if (!strcmp(dtype, "VORT")) kind = NS2D_MAX_VORT;
    else if (!strcmp(dtype, "VEL")) kind = NS2D_MAX_VEL;
    else if (!strcmp(dtype, "VORT_FOUR")) kind = NS2D_MAX_VORT_FOUR;
    else return 0.0;  /* the reference finds nothing to reduce either */
    ns2d_compat_check(ns2d_set_w_hat(h, (const double*)run_data->w_hat), "GetMaxData");
    double v = 0.0;
    ns2d_compat_check(ns2d_get_max_data(h, kind, &v), "GetMaxData");
    return v;
}

/* GetTimestep (solver.c:2376): the adaptive step of run_data->w_hat; keeps
   sys_vars->min_dt / max_dt as the reference does (solver.c:2486-2488). */
void GetTimestep(double* dt) {
    ns2d_handle* h = ns2d_compat_handle();
    ns2d_compat_check(ns2d_set_w_hat(h, (const double*)run_data->w_hat), "GetTimestep");
    ns2d_compat_check(ns2d_set_w_max_init(h, sys_vars->w_max_init), "GetTimestep");
    ns2d_compat_check(ns2d_get_timestep(h, dt), "GetTimestep");
    sys_vars->min_dt = fmin(*dt, sys_vars->min_dt);
    sys_vars->max_dt = fmax(*dt, sys_vars->max_dt);
}
