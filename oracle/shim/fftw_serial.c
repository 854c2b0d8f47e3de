/*
 * oracle/shim/fftw_serial.c -- bodies of the serial FFTW stand-in
 * (oracle/shim/fftw3.h).  Test infrastructure only.  Each execute copies the
 * unpadded real array into FFTW's padded in-place layout (rows of Ny+2
 * doubles) that oracle/fft.c works on, or back out of it.
 */
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"
#include "../fft.h"

struct shim_fftw_plan_s {
    int kind; /* 0 = r2c, 1 = c2r */
    int nx, ny, howmany;
};

static fftw_plan mk(int kind, int nx, int ny, int howmany) {
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->kind = kind;
    p->nx = nx;
    p->ny = ny;
    p->howmany = howmany;
    return p;
}
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags) {
    (void)in; (void)out; (void)flags;
    return mk(0, n0, n1, 1);
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags) {
    (void)in; (void)out; (void)flags;
    return mk(1, n0, n1, 1);
}
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int* inembed, int istride,
                                 int idist, fftw_complex* out, const int* onembed, int ostride, int odist,
                                 unsigned flags) {
    (void)rank; (void)in; (void)inembed; (void)istride; (void)idist; (void)out; (void)onembed; (void)ostride;
    (void)odist; (void)flags;
    return mk(0, n[0], n[1], howmany);
}
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed,
                                 int istride, int idist, double* out, const int* onembed, int ostride, int odist,
                                 unsigned flags) {
    (void)rank; (void)in; (void)inembed; (void)istride; (void)idist; (void)out; (void)onembed; (void)ostride;
    (void)odist; (void)flags;
    return mk(1, n[0], n[1], howmany);
}
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) {
    const size_t row = (size_t)p->ny * p->howmany, prow = (size_t)(p->ny + 2) * p->howmany;
    double* pad = (double*)calloc((size_t)p->nx * prow, sizeof(double));
    for (int i = 0; i < p->nx; ++i) memcpy(pad + i * prow, in + i * row, row * sizeof(double));
    offt_r2c_2d(p->nx, p->ny, p->howmany, pad, out);
    free(pad);
}
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) {
    const size_t row = (size_t)p->ny * p->howmany, prow = (size_t)(p->ny + 2) * p->howmany;
    double* pad = (double*)calloc((size_t)p->nx * prow, sizeof(double));
    offt_c2r_2d(p->nx, p->ny, p->howmany, in, pad);
    for (int i = 0; i < p->nx; ++i) memcpy(out + i * row, pad + i * prow, row * sizeof(double));
    free(pad);
}
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int n) { (void)n; }
void fftw_cleanup_threads(void) {}
