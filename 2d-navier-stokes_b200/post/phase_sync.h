/*
 * phase_sync.h -- sector phase synchronisation of bin/ns2d_post (phase_sync.c).
 */
#ifndef NS2D_POST_PHASE_SYNC_H
#define NS2D_POST_PHASE_SYNC_H
#include <complex.h>

#include "ns2d.h"
#include "ns2d_h5.h"

typedef struct ps_state ps_state;

/* Sector geometry and angle tables for an nx^2 run, kmax = (int)(nx / 3),
   n_k3 x n_k1 sectors (reduced: the 8-sector k1 search of -a -a -a); the
   viscous parameters give FluxSpectra's prefactor.  NULL when out of memory. */
ps_state* ps_create(int nx, int kmax, double kmax_frac, int n_k3, int n_k1, int reduced, double nu, int hyper_flag,
                    double hyper_pow, double alpha, int drag_flag, double drag_pow, int device);
/* One snapshot: w and its RHS ([nx][nx/2+1]), the full-field amplitudes and
   phases ([2kmax+1]^2). */
ns2d_status ps_snapshot(ps_state* s, const double complex* w, const double complex* rhs, const double* amps,
                        const double* phases);
/* The snapshot's datasets into `group`; the final datasets into the root. */
int ps_write_snapshot(const ps_state* s, ns2d_h5_file* f, const char* group);
int ps_write_final(const ps_state* s, ns2d_h5_file* f);
void ps_free(ps_state* s);
#endif
