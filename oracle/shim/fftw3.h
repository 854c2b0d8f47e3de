/*
 * oracle/shim/fftw3.h -- the serial FFTW3 API subset of the reference's
 * post-processing program (plans at PostProcessing/src/post_proc.c:430-470,
 * executes at full_field.c:206, 226, 247), on top of the single-rank
 * stand-in of fftw3-mpi.h.  Test infrastructure only; the transforms are
 * oracle/fft.c.  Serial plans act on unpadded real arrays [Nx][Ny] (howmany
 * interleaved), as FFTW's out-of-place plans do.
 */
#ifndef NS2D_SHIM_FFTW3_H
#define NS2D_SHIM_FFTW3_H
#include "fftw3-mpi.h"
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int* inembed, int istride,
                                 int idist, fftw_complex* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed,
                                 int istride, int idist, double* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int n);
void fftw_cleanup_threads(void);
#endif
