/*
 * run.h -- shared declarations of the ns2d command-line solver (bin/ns2d).
 *
 * The program is a drop-in for the reference executable Solver/bin/main
 * (Solver/src/main.c): the same argv grammar (utils.c:34-460), the same
 * initial conditions (solver.c:1107-2014) and forcings (force.c:28-581), the
 * SpectralSolve time loop (solver.c:54-251) and the same HDF5 output files
 * (hdf5_funcs.c:33-1870), with the state and every step on the GPU through
 * libns2d.so and the files written by libns2d_h5.so.
 */
#ifndef NS2D_CLI_RUN_H
#define NS2D_CLI_RUN_H
#include <complex.h>
#include <stdint.h>

#include "ns2d.h"

/* Parameters of one run: the fields of system_vars_struct and
   HDF_file_info_struct that GetCMLArgs fills (data_types.h:190-350), plus the
   switches the reference fixes at compile time. */
typedef struct ns2d_run {
    long N[2];
    double t0, T, dt, cfl_const;
    int adapt_step, cfl_cond;
    char u0[64];
    char forcing[64];
    int force_k;
    double force_scale;
    int trans_iters;
    double trans_frac;
    double nu;
    int hyper_flag;
    double hyper_pow;
    double ekmn_alpha;
    int ekmn_flag;
    double ekmn_pow;
    int save_every;
    char output_dir[1024];
    char output_tag[64];
    char input_file[512];
    char input_dir[512];
    int file_only;
    /* compile-time switches of the reference (data_types.h:54-62, Makefile) */
    int integrator;  /* ns2d_integrator, default RK4CN */
    int dealias;     /* ns2d_dealias, default 2/3 */
    int precision;   /* ns2d_precision */
    int device;
    int quirks;      /* NS2D_QUIRK_* bits, default all */
    int phase_only;  /* -D__PHASE_ONLY model (ns2d_model)    */
    int dry_run;     /* print the parsed parameters and exit */
    int quiet;
} ns2d_run;

/* argv -> run (GetCMLArgs).  Prints the reference's diagnostics and exits(1)
   on an invalid argument, as the reference does. */
void ns2d_cli_parse(int argc, char** argv, ns2d_run* r);

/* Wavenumbers and collocation points (InitializeSpaceVariables,
   solver.c:2022-2068). */
typedef struct ns2d_grid {
    long nx, ny, nyf;
    int* kx;   /* [nx]  */
    int* ky;   /* [nyf] */
    double* x; /* [nx]  */
    double* y; /* [ny]  */
} ns2d_grid;
int ns2d_grid_init(ns2d_grid* g, long nx, long ny);
void ns2d_grid_free(ns2d_grid* g);

/* Initial vorticity spectrum of r->u0 into w_hat [nx][nyf] (host), with
   srand(123456789) first and glibc rand() draws in the reference's order,
   dealiased and made conjugate-symmetric on the ky = 0 column.  Real-space
   fields are transformed on the GPU (ns2d_fft_r2c / _c2r of h). */
int ns2d_cli_initial(const ns2d_run* r, const ns2d_grid* g, ns2d_handle* h, double complex* w_hat);

/* Listed-mode forcings drawn on the host (STOC, STOC_GAUSS, CONST_GAUSS). */
typedef struct ns2d_forcing_modes {
    int kind;       /* 0 none, 1 STOC, 2 STOC_GAUSS, 3 CONST_GAUSS */
    int n;
    int32_t* indx;  /* flat [nx][nyf] index of each forced mode */
    double* scaling;
    double complex* value;
} ns2d_forcing_modes;
int ns2d_cli_forcing_init(const ns2d_run* r, const ns2d_grid* g, ns2d_forcing_modes* f);  /* InitializeForcing */
void ns2d_cli_forcing_draw(ns2d_forcing_modes* f, double dt);                              /* ComputeForcing */
void ns2d_cli_forcing_free(ns2d_forcing_modes* f);

#endif
