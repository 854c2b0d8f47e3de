/*
 * oracle/fft.c -- CPU FP64 FFT for the oracle (test infrastructure only; the
 * GPU product never links this file).  Written from the DFT definition:
 *
 *     X[k] = sum_n x[n] exp(sign * 2 pi i n k / n_len)
 *
 * as an iterative radix-2 decimation-in-time transform with a bit-reversal
 * permutation and twiddles w^m = exp(sign 2 pi i m / n) from libm sin/cos.
 *
 * The 2-D wrappers restate FFTW 3.3's rdft2 conventions for the plans made in
 * the reference at Solver/src/solver.c:2883-2895 (fftw_mpi_plan_dft_r2c_2d,
 * fftw_mpi_plan_dft_c2r_2d and the howmany = 2 fftw_mpi_plan_many_* plans):
 * unnormalised, real rows padded to Ny+2 doubles, complex rows of Ny/2+1.
 * Two real rows are packed into one complex transform (z = a + i b).
 */
#include "fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;

static int g_threads = 0;

void offt_set_threads(int nthreads) { g_threads = nthreads; }

int offt_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* Twiddle tables: exp(-2 pi i m / n), m < n/2, cached per log2(n). */
#define OFFT_MAX_LOG 16
static cplx* g_tw[OFFT_MAX_LOG + 1];

static int ilog2(int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

static const cplx* twiddles(int n) {
    int l = ilog2(n);
    if (l > OFFT_MAX_LOG || (1 << l) != n) abort();
    cplx* t = g_tw[l];
    if (t) return t;
    int h = n / 2 > 0 ? n / 2 : 1;
    t = (cplx*)malloc(sizeof(cplx) * (size_t)h);
    for (int m = 0; m < h; ++m) {
        double a = 2.0 * M_PI * (double)m / (double)n;
        t[m] = cos(a) - I * sin(a);
    }
#pragma omp critical(offt_tw)
    {
        if (!g_tw[l]) g_tw[l] = t;
        else { free(t); }
    }
    return g_tw[l];
}

void offt_c2c(cplx* x, int n, int sign) {
    if (n <= 1) return;
    const cplx* tw = twiddles(n);
    /* bit reversal */
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { cplx t = x[i]; x[i] = x[j]; x[j] = t; }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1, step = n / len;
        for (int s = 0; s < n; s += len) {
            for (int k = 0; k < half; ++k) {
                cplx w = tw[k * step];
                if (sign > 0) w = conj(w);
                cplx a = x[s + k];
                cplx b = x[s + k + half] * w;
                x[s + k] = a + b;
                x[s + k + half] = a - b;
            }
        }
    }
}

/* Column transforms over an [nx][ld] complex array (columns 0..ncol-1), in place. */
static void column_pass(cplx* a, int nx, int ld, int ncol, int sign) {
    twiddles(nx);
    const int blk = 8;
#pragma omp parallel num_threads(offt_get_threads())
    {
        cplx* buf = (cplx*)malloc(sizeof(cplx) * (size_t)nx * blk);
#pragma omp for schedule(static)
        for (int c0 = 0; c0 < ncol; c0 += blk) {
            int nc = ncol - c0 < blk ? ncol - c0 : blk;
            for (int x = 0; x < nx; ++x)
                for (int c = 0; c < nc; ++c) buf[(size_t)c * nx + x] = a[(size_t)x * ld + c0 + c];
            for (int c = 0; c < nc; ++c) offt_c2c(buf + (size_t)c * nx, nx, sign);
            for (int x = 0; x < nx; ++x)
                for (int c = 0; c < nc; ++c) a[(size_t)x * ld + c0 + c] = buf[(size_t)c * nx + x];
        }
        free(buf);
    }
}

void offt_r2c_2d(int nx, int ny, int howmany, const double* in, cplx* out) {
    const int nyf = ny / 2 + 1;
    const int ldr = ny + 2;
    cplx* t = (cplx*)malloc(sizeof(cplx) * (size_t)nx * nyf);
    twiddles(ny);
    for (int b = 0; b < howmany; ++b) {
        /* rows: r2c along y, two rows per complex transform */
#pragma omp parallel num_threads(offt_get_threads())
        {
            cplx* z = (cplx*)malloc(sizeof(cplx) * (size_t)ny);
#pragma omp for schedule(static)
            for (int x = 0; x < nx; x += 2) {
                int pair = (x + 1 < nx);
                for (int y = 0; y < ny; ++y) {
                    double av = in[((size_t)x * ldr + y) * howmany + b];
                    double bv = pair ? in[((size_t)(x + 1) * ldr + y) * howmany + b] : 0.0;
                    z[y] = av + I * bv;
                }
                offt_c2c(z, ny, -1);
                for (int j = 0; j < nyf; ++j) {
                    cplx zk = z[j], zm = conj(z[(ny - j) % ny]);
                    t[(size_t)x * nyf + j] = 0.5 * (zk + zm);
                    if (pair) t[(size_t)(x + 1) * nyf + j] = -0.5 * I * (zk - zm);
                }
            }
            free(z);
        }
        column_pass(t, nx, nyf, nyf, -1);
        for (size_t i = 0; i < (size_t)nx * nyf; ++i) out[i * howmany + b] = t[i];
    }
    free(t);
}

void offt_c2r_2d(int nx, int ny, int howmany, const cplx* in, double* out) {
    const int nyf = ny / 2 + 1;
    const int ldr = ny + 2;
    cplx* t = (cplx*)malloc(sizeof(cplx) * (size_t)nx * nyf);
    twiddles(ny);
    for (int b = 0; b < howmany; ++b) {
        for (size_t i = 0; i < (size_t)nx * nyf; ++i) t[i] = in[i * howmany + b];
        column_pass(t, nx, nyf, nyf, +1);
#pragma omp parallel num_threads(offt_get_threads())
        {
            cplx* z = (cplx*)malloc(sizeof(cplx) * (size_t)ny);
#pragma omp for schedule(static)
            for (int x = 0; x < nx; x += 2) {
                int pair = (x + 1 < nx);
                const cplx* A = t + (size_t)x * nyf;
                const cplx* B = pair ? t + (size_t)(x + 1) * nyf : NULL;
                /* Hermitian extension; DC and Nyquist use the real part only. */
                z[0] = creal(A[0]) + I * (pair ? creal(B[0]) : 0.0);
                if (ny > 1) z[ny / 2] = creal(A[ny / 2]) + I * (pair ? creal(B[ny / 2]) : 0.0);
                for (int k = 1; k < ny / 2; ++k) {
                    cplx a = A[k], bb = pair ? B[k] : 0.0;
                    z[k] = a + I * bb;
                    z[ny - k] = conj(a) + I * conj(bb);
                }
                offt_c2c(z, ny, +1);
                for (int y = 0; y < ny; ++y) {
                    out[((size_t)x * ldr + y) * howmany + b] = creal(z[y]);
                    if (pair) out[((size_t)(x + 1) * ldr + y) * howmany + b] = cimag(z[y]);
                }
            }
            free(z);
        }
    }
    free(t);
}
