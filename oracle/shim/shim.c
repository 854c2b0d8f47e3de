/*
 * oracle/shim/shim.c -- bodies for the single-rank FFTW3-MPI stand-in (test
 * infrastructure only); the no-op output hooks are in hooks.c.  Transforms are
 * oracle/fft.c.  fftw_malloc returns zeroed memory so
 * that reference arrays it never initialises (e.g. the mean-flow sums in
 * Solver/src/sys_msr.c:454-461) are deterministic.
 */
#include <stdlib.h>
#include <string.h>
#include "fftw3-mpi.h"
#include "../fft.h"

struct shim_fftw_plan_s {
    int kind; /* 0 = r2c, 1 = c2r */
    int nx, ny, howmany;
};

void* fftw_malloc(size_t n) { return calloc(1, n ? n : 1); }
void fftw_free(void* p) { free(p); }
void fftw_mpi_init(void) {}
void fftw_mpi_cleanup(void) {}
void fftw_cleanup(void) {}

ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm,
                                 ptrdiff_t* local_n0, ptrdiff_t* local_0_start) {
    (void)comm;
    *local_n0 = n0;
    *local_0_start = 0;
    return n0 * n1;
}

ptrdiff_t fftw_mpi_local_size_many(int rnk, const ptrdiff_t* n, ptrdiff_t howmany,
                                   ptrdiff_t block0, MPI_Comm comm,
                                   ptrdiff_t* local_n0, ptrdiff_t* local_0_start) {
    (void)block0; (void)comm;
    ptrdiff_t tot = howmany;
    for (int i = 0; i < rnk; ++i) tot *= n[i];
    *local_n0 = n[0];
    *local_0_start = 0;
    return tot;
}

static fftw_plan mk(int kind, int nx, int ny, int howmany) {
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->kind = kind; p->nx = nx; p->ny = ny; p->howmany = howmany;
    return p;
}

fftw_plan fftw_mpi_plan_dft_r2c_2d(ptrdiff_t n0, ptrdiff_t n1, double* in, fftw_complex* out,
                                   MPI_Comm comm, unsigned flags) {
    (void)in; (void)out; (void)comm; (void)flags;
    return mk(0, (int)n0, (int)n1, 1);
}
fftw_plan fftw_mpi_plan_dft_c2r_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in, double* out,
                                   MPI_Comm comm, unsigned flags) {
    (void)in; (void)out; (void)comm; (void)flags;
    return mk(1, (int)n0, (int)n1, 1);
}
fftw_plan fftw_mpi_plan_many_dft_r2c(int rnk, const ptrdiff_t* n, ptrdiff_t howmany,
                                     ptrdiff_t iblock, ptrdiff_t oblock, double* in,
                                     fftw_complex* out, MPI_Comm comm, unsigned flags) {
    (void)rnk; (void)iblock; (void)oblock; (void)in; (void)out; (void)comm; (void)flags;
    return mk(0, (int)n[0], (int)n[1], (int)howmany);
}
fftw_plan fftw_mpi_plan_many_dft_c2r(int rnk, const ptrdiff_t* n, ptrdiff_t howmany,
                                     ptrdiff_t iblock, ptrdiff_t oblock, fftw_complex* in,
                                     double* out, MPI_Comm comm, unsigned flags) {
    (void)rnk; (void)iblock; (void)oblock; (void)in; (void)out; (void)comm; (void)flags;
    return mk(1, (int)n[0], (int)n[1], (int)howmany);
}
void fftw_mpi_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) {
    offt_r2c_2d(p->nx, p->ny, p->howmany, in, out);
}
void fftw_mpi_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) {
    offt_c2r_2d(p->nx, p->ny, p->howmany, in, out);
}
void fftw_destroy_plan(fftw_plan p) { free(p); }
