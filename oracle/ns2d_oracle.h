/*
 * oracle/ns2d_oracle.h -- CPU FP64 restatement of the reference solver's
 * pseudospectral step (EndCar808/2D-Navier-Stokes, Solver/src/solver.c,
 * force.c, sys_msr.c).  TEST INFRASTRUCTURE ONLY: the checker that the CUDA
 * product is compared with.  Only tests/, __graft_entry__.smoke() and the CPU
 * legs of bench.py load it; the product never does.
 *
 * Pinned against the reference's own sources compiled with oracle/Makefile
 * (target `ref`), which stand in for FFTW with oracle/fft.c.
 * The functions mirror include/ns2d.h one for one, with the same layouts.
 */
#ifndef NS2D_ORACLE_H
#define NS2D_ORACLE_H
#include <stdint.h>
#include "../include/ns2d.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ns2d_oracle ns2d_oracle;

ns2d_oracle* oracle_create(const ns2d_params* p, int threads);
void oracle_destroy(ns2d_oracle* o);
int oracle_n_spect(const ns2d_oracle* o);
void oracle_set_w_hat(ns2d_oracle* o, const double* w_hat);
void oracle_get_w_hat(const ns2d_oracle* o, double* w_hat);
void oracle_compute_forcing(ns2d_oracle* o, double dt);
void oracle_nonlinear_rhs(ns2d_oracle* o, const double* in, double* out);
void oracle_rk4_step(ns2d_oracle* o, double dt);
int oracle_ab4_step(ns2d_oracle* o, double dt, int iters);
int oracle_dp5_step(ns2d_oracle* o, double dt, double* err);
double oracle_rk5dp_step(ns2d_oracle* o, double dt, int iters);
void oracle_apply_dealiasing(const ns2d_oracle* o, double* arr, int array_dim);
void oracle_force_conjugacy(ns2d_oracle* o, const double* arr);
double oracle_get_max_data(ns2d_oracle* o, int kind);
double oracle_get_timestep(ns2d_oracle* o, double dt);
void oracle_set_w_max_init(ns2d_oracle* o, double w);
int oracle_hyper_visc_flag(const ns2d_oracle* o);
void oracle_system_measurables(ns2d_oracle* o, double* scalars13, double* spectra);
void oracle_get_w_real(ns2d_oracle* o, double* w);

/* Taylor-Green and seeded random-phase initial vorticity (test inputs). */
void oracle_ic_taylor_green(int nx, int ny, double* w_hat);

#ifdef __cplusplus
}
#endif
#endif
