/*
 * oracle/shim/fftw3-mpi.h -- single-rank stand-in for the FFTW3 / FFTW3-MPI
 * API subset used by the reference solver (plans at Solver/src/solver.c:
 * 2873-2901, local sizes at :2614-2615, executes at :932, :964, :994 ...).
 * Test infrastructure only.  The transforms are oracle/fft.c (written from the
 * DFT definition), not FFTW; the conventions (unnormalised, padded real rows,
 * interleaved howmany batches) follow FFTW's documentation.
 */
#ifndef NS2D_SHIM_FFTW3_MPI_H
#define NS2D_SHIM_FFTW3_MPI_H
#include <complex.h>
#include <stddef.h>
#include "mpi.h"

typedef double _Complex fftw_complex;
typedef struct shim_fftw_plan_s* fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_MPI_DEFAULT_BLOCK (0)
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

void* fftw_malloc(size_t n);
void fftw_free(void* p);
void fftw_mpi_init(void);
void fftw_mpi_cleanup(void);
void fftw_cleanup(void);
ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm,
                                 ptrdiff_t* local_n0, ptrdiff_t* local_0_start);
ptrdiff_t fftw_mpi_local_size_many(int rnk, const ptrdiff_t* n, ptrdiff_t howmany,
                                   ptrdiff_t block0, MPI_Comm comm,
                                   ptrdiff_t* local_n0, ptrdiff_t* local_0_start);
fftw_plan fftw_mpi_plan_dft_r2c_2d(ptrdiff_t n0, ptrdiff_t n1, double* in, fftw_complex* out,
                                   MPI_Comm comm, unsigned flags);
fftw_plan fftw_mpi_plan_dft_c2r_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in, double* out,
                                   MPI_Comm comm, unsigned flags);
fftw_plan fftw_mpi_plan_many_dft_r2c(int rnk, const ptrdiff_t* n, ptrdiff_t howmany,
                                     ptrdiff_t iblock, ptrdiff_t oblock, double* in,
                                     fftw_complex* out, MPI_Comm comm, unsigned flags);
fftw_plan fftw_mpi_plan_many_dft_c2r(int rnk, const ptrdiff_t* n, ptrdiff_t howmany,
                                     ptrdiff_t iblock, ptrdiff_t oblock, fftw_complex* in,
                                     double* out, MPI_Comm comm, unsigned flags);
void fftw_mpi_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_mpi_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
void fftw_destroy_plan(fftw_plan p);
#endif
