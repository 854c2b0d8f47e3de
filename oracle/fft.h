/*
 * oracle/fft.h -- CPU FP64 FFT used only as test infrastructure (the oracle).
 *
 * This is NOT product code.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load anything built from
 * oracle/.  The GPU product path never calls into this file.
 *
 * Semantics follow FFTW 3.3's documented conventions for the transforms the
 * reference solver plans in Solver/src/solver.c:2873-2901:
 *   - forward = exp(-i...), backward = exp(+i...), both unnormalised;
 *   - 2-D r2c/c2r on an [Nx][Ny] real array stored with the in-place padding
 *     of FFTW (row stride Ny+2 doubles) and an [Nx][Ny/2+1] complex array;
 *   - "howmany" interleaved batches (fftw_mpi_plan_many_dft_*, howmany = 2),
 *     element (index, batch) at index*howmany + batch;
 *   - c2r does the complex x-transform first and then the row c2r, which
 *     reads only the real part of the ky = 0 and ky = Ny/2 entries.
 * Grid sizes must be powers of two (>= 2).
 */
#ifndef NS2D_ORACLE_FFT_H
#define NS2D_ORACLE_FFT_H

#include <complex.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* In-place complex transform of length n (power of two); sign = -1 forward, +1 backward. */
void offt_c2c(double _Complex* x, int n, int sign);

/* 2-D real-to-complex, FFTW layout (padded real rows of Ny+2 doubles), howmany interleaved. */
void offt_r2c_2d(int nx, int ny, int howmany, const double* in, double _Complex* out);

/* 2-D complex-to-real, FFTW layout; the input is preserved. */
void offt_c2r_2d(int nx, int ny, int howmany, const double _Complex* in, double* out);

/* Number of OpenMP threads the 2-D transforms use (0 = library default). */
void offt_set_threads(int nthreads);
int  offt_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
