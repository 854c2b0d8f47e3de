/*
 * init.c -- grid, initial conditions and host-drawn forcings of bin/ns2d.
 *
 * Initial conditions follow InitialConditions (Solver/src/solver.c:1107-2014)
 * branch by branch: the same formulas evaluated in the same order, with C99
 * complex arithmetic and glibc's rand() after srand(123456789), so that a
 * spectrum built here equals the reference's.  Real-space fields go through
 * the GPU's r2c/c2r (ns2d_fft_r2c / ns2d_fft_c2r, unnormalised like FFTW).
 * Where the reference reads memory it never set, the value used here is
 * stated at the branch.
 *
 * Forcings whose values the reference draws on the host (force.c:104-433,
 * 540-577) are drawn here with the same rand() sequence; KOLM and ZERO are
 * parameters of the GPU handle.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ns2d_h5.h"
#include "run.h"

/* data_types.h:143-169 */
#define KAPPA 1.0
#define DELTA 0.005
#define BETA 1.0
#define BLOB_S 6.0
#define DT_K0 6.0
#define DT_E0 0.5
#define DT2_K0 30
#define DT2_E0 0.5
#define DTEXP_K0 8.0
#define DTEXP_E0 (343.0 / 96.0)
#define RING_MIN_K 3.0
#define RING_MAX_K 10.0
#define EXTRM_ENS_MIN_K 1.5
#define EXTRM_ENS_POW 1.5
#define UNIF_MIN_K 2.5
#define UNIF_MAX_K 9.5
#define RAND_ENST0 1.0
#define STOC_FORC_UNIF_DELTA_K 1.5
#define CONST_GAUSS_K_MIN 10
#define CONST_GAUSS_K_MAX 12

static double urand(void) { return (double)rand() / (double)RAND_MAX; }

int ns2d_grid_init(ns2d_grid* g, long nx, long ny) {
    memset(g, 0, sizeof(*g));
    g->nx = nx;
    g->ny = ny;
    g->nyf = ny / 2 + 1;
    g->kx = (int*)malloc(sizeof(int) * (size_t)nx);
    g->ky = (int*)malloc(sizeof(int) * (size_t)g->nyf);
    g->x = (double*)malloc(sizeof(double) * (size_t)nx);
    g->y = (double*)malloc(sizeof(double) * (size_t)ny);
    if (!g->kx || !g->ky || !g->x || !g->y) return -1;
    for (long i = 0; i < nx; ++i) {
        g->kx[i] = (int)(i <= nx / 2 ? i : i - nx);
        g->x[i] = (double)i * 2.0 * M_PI / (double)nx;
    }
    for (long j = 0; j < ny; ++j) {
        if (j < g->nyf) g->ky[j] = (int)j;
        g->y[j] = (double)j * 2.0 * M_PI / (double)ny;
    }
    return 0;
}

void ns2d_grid_free(ns2d_grid* g) {
    free(g->kx);
    free(g->ky);
    free(g->x);
    free(g->y);
    memset(g, 0, sizeof(*g));
}

static int gpu(ns2d_handle* h, ns2d_status s, const char* what) {
    if (s == NS2D_OK) return 0;
    fprintf(stderr, "\n[ERROR] %s failed: %s (%s)\n", what, ns2d_status_string(s), ns2d_last_error(h));
    return -1;
}

/* Random-phase spectra of the DECAY_TURB family (solver.c:1234-1364). */
static void decay_turb(const ns2d_run* r, const ns2d_grid* g, double complex* w) {
    const long Nx = g->nx, Ny = g->ny, nyf = g->nyf;
    const int bb = !strcmp(r->u0, "DECAY_TURB_BB"), nb = !strcmp(r->u0, "DECAY_TURB_NB");
    const int ex = !strcmp(r->u0, "DECAY_TURB_EXP");
    double spec_1d = 0.0;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            if (g->kx[i] == 0 && g->ky[j] == 0) {
                spec_1d = 0.0;
                w[q] = 0.0;
                continue;
            }
            const double sqrt_k = sqrt((double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]));
            if (bb)
                spec_1d = sqrt_k / (1.0 + pow(sqrt_k, 4.0) / DT_K0);
            else if (nb)
                spec_1d = pow(sqrt_k, 6.0) / pow((1.0 + sqrt_k / (2.0 * DT2_K0)), 18.0);
            else if (ex)
                spec_1d = pow(sqrt_k, 7.0) / pow(DTEXP_K0, 8.0) * cexp(-3.5 * pow(sqrt_k / DTEXP_K0, 2.0));
            const double u1 = urand();
            if (ex)
                w[q] = sqrt(sqrt_k * spec_1d / (M_PI)) * cexp(2.0 * M_PI * u1 * I);
            else
                w[q] = sqrt(spec_1d * (sqrt_k / (2.0 * M_PI))) * cexp(2.0 * M_PI * u1 * I);
        }
    double enrg = 0.0;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            if (g->kx[i] == 0 && g->ky[j] == 0) continue;
            const long q = i * nyf + j;
            const double inv_k_sqr = 1.0 / (double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]);
            if (j == 0 || j == nyf - 1)
                enrg += inv_k_sqr * cabs(w[q] * conj(w[q]));
            else
                enrg += 2.0 * inv_k_sqr * cabs(w[q] * conj(w[q]));
        }
    enrg *= (0.5 / pow(Nx * Ny, 2.0)) * 4.0 * pow(M_PI, 2.0);
    /* the normalisation pass keeps kx = 0 or ky != 0 and zeroes the rest of
       the ky = 0 column (solver.c:1336-1362) */
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            if (g->kx[i] == 0 || g->ky[j] != 0) {
                if (bb)
                    w[q] *= sqrt(DT_E0 / enrg);
                else if (nb)
                    w[q] *= sqrt(DT2_E0 / enrg);
                else if (ex)
                    w[q] *= sqrt(DTEXP_E0 / enrg);
            } else {
                w[q] = 0.0;
            }
        }
}

/* Energy-normalised stream function of DECAY_TURB_ALT (solver.c:1365-1521). */
static int decay_turb_alt(const ns2d_grid* g, ns2d_handle* h, double complex* w) {
    const long Nx = g->nx, Ny = g->ny, nyf = g->nyf;
    double complex* psi_hat = (double complex*)malloc(sizeof(double complex) * (size_t)(Nx * nyf));
    double* psi = (double*)malloc(sizeof(double) * (size_t)(Nx * Ny));
    int rc = -1;
    if (!psi_hat || !psi) goto out;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            const double u1 = urand();
            const double u2 = urand();
            const double z1 = sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
            const double z2 = sqrt(-2.0 * log(u1)) * sin(2.0 * M_PI * u2);
            if (g->kx[i] == 0 && g->ky[j] == 0) {
                psi_hat[q] = 0.0;
            } else {
                const double k_sqrt = sqrt((double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]));
                const double spec_1d = 1.0 / (k_sqrt * (1.0 + pow(k_sqrt / 6.0, 4.0)));
                psi_hat[q] = (z1 + z2 * I) * sqrt(spec_1d * pow(k_sqrt, 2.0) / (pow(k_sqrt, 3.0) * 2.0 * M_PI));
            }
        }
    if (gpu(h, ns2d_fft_c2r(h, (const double*)psi_hat, psi), "c2r")) goto out;
    double mean = 0.0;
    for (long q = 0; q < Nx * Ny; ++q) {
        psi[q] /= (Nx * Ny);
        mean += psi[q];
    }
    for (long q = 0; q < Nx * Ny; ++q) psi[q] -= (mean / (Nx * Ny));
    if (gpu(h, ns2d_fft_r2c(h, psi, (double*)psi_hat), "r2c")) goto out;
    double enrg = 0.0;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            const double k_sqrd = (double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]);
            if (j == 0 || j == nyf - 1)
                enrg += k_sqrd * cabs(psi_hat[q] * conj(psi_hat[q]));
            else
                enrg += 2.0 * k_sqrd * cabs(psi_hat[q] * conj(psi_hat[q]));
        }
    enrg *= 4.0 * pow(M_PI, 2.0) * (0.5 / pow(Nx * Ny, 2.0));
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            psi_hat[q] *= sqrt(0.5 / enrg);
            const double k_sqrd = (double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]);
            w[q] = (g->kx[i] != 0 || g->ky[j] != 0) ? -k_sqrd * psi_hat[q] : 0.0;
        }
    rc = 0;
out:
    free(psi_hat);
    free(psi);
    return rc;
}

static void gauss_decay_turb(const ns2d_grid* g, double complex* w) {
    const long Nx = g->nx, Ny = g->ny, nyf = g->nyf;
    double complex* psi_hat = (double complex*)malloc(sizeof(double complex) * (size_t)(Nx * nyf));
    if (!psi_hat) return;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            if (g->kx[i] == 0 && g->ky[j] == 0) {
                psi_hat[q] = 0.0;
            } else {
                const double k_sqrt = sqrt((double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]));
                const double spec_1d = pow(k_sqrt, 6.0) / pow((1.0 + k_sqrt / 60.0), 18.0);
                const double u1 = urand();
                psi_hat[q] = sqrt(spec_1d * (1.0 / k_sqrt)) * cexp(I * 2.0 * M_PI * u1);
            }
        }
    double enrg = 0.0;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            if (g->kx[i] == 0 && g->ky[j] == 0) continue;
            const long q = i * nyf + j;
            const double k_sqrd = (double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]);
            if (j == 0 || j == nyf - 1)
                enrg += k_sqrd * cabs(psi_hat[q] * conj(psi_hat[q]));
            else
                enrg += 2.0 * k_sqrd * cabs(psi_hat[q] * conj(psi_hat[q]));
        }
    enrg *= 4.0 * pow(M_PI, 2.0) * (0.5 / pow(Nx * Ny, 2.0));
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            psi_hat[q] /= sqrt(enrg);
            psi_hat[q] *= sqrt(0.5);
            const double k_sqrd = (double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]);
            w[q] = (g->kx[i] != 0 || g->ky[j] != 0) ? k_sqrd * psi_hat[q] : 0.0;
        }
    free(psi_hat);
}

static void extrm_ens(const ns2d_grid* g, double complex* w) {
    const long Nx = g->nx, nyf = g->nyf;
    double norm = 0.0;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const double k_sqr = (double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]);
            const int edge = (j == 0 || j == nyf - 1);
            if ((k_sqr > 0) && (sqrt(k_sqr) > EXTRM_ENS_MIN_K))
                norm += edge ? pow(sqrt(k_sqr), -EXTRM_ENS_POW) : 2.0 * pow(sqrt(k_sqr), -EXTRM_ENS_POW);
            else if (sqrt(k_sqr) <= EXTRM_ENS_MIN_K)
                norm += edge ? pow(EXTRM_ENS_MIN_K, -EXTRM_ENS_POW) * exp((sqrt(k_sqr) - EXTRM_ENS_MIN_K) / 3.5)
                             : 2.0 * pow(EXTRM_ENS_MIN_K, -EXTRM_ENS_POW) * exp((sqrt(k_sqr) - EXTRM_ENS_MIN_K) / 3.5);
        }
    norm = sqrt(EXTRM_ENS_MIN_K / norm);
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            const double k_sqr = (double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]);
            if ((k_sqr > 0) && (sqrt(k_sqr) > EXTRM_ENS_MIN_K)) {
                const double u1 = urand();
                w[q] = pow(sqrt(k_sqr), -EXTRM_ENS_POW / 2.0) * norm * cexp(I * 2.0 * M_PI * u1);
            } else if (sqrt(k_sqr) <= EXTRM_ENS_MIN_K) {
                const double u1 = urand();
                w[q] = pow(EXTRM_ENS_MIN_K, -EXTRM_ENS_POW / 2.0) * exp((sqrt(k_sqr) - EXTRM_ENS_MIN_K) / 3.5) * norm *
                       cexp(I * 2.0 * M_PI * u1);
            } else {
                w[q] = 0.0;
            }
        }
}

static void ring(const ns2d_grid* g, double complex* w) {
    const long Nx = g->nx, nyf = g->nyf;
    double norm = 0.0;
    /* the normalisation pass draws one (unused) number per mode (solver.c:1686-1700) */
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const double abs_k = sqrt((double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]));
            (void)urand();
            if ((abs_k >= RING_MIN_K && abs_k <= RING_MAX_K) && (g->ky[j] != 0 || g->kx[i] > 0))
                norm += exp(-pow(abs_k - ((RING_MIN_K + RING_MAX_K) / 2.0), 2.0));
        }
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            const double abs_k = sqrt((double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]));
            if ((abs_k >= RING_MIN_K && abs_k <= RING_MAX_K) && (g->ky[j] != 0 || g->kx[i] > 0)) {
                const double u1 = urand();
                w[q] = sqrt(72.0 * exp(-pow(abs_k - ((RING_MIN_K + RING_MAX_K) / 2.0), 2.0)) / (M_PI * abs_k * norm)) *
                       cexp(2.0 * M_PI * I * u1);
            } else {
                w[q] = 0.0;
            }
        }
}

static void unif(const ns2d_grid* g, double complex* w) {
    const long Nx = g->nx, nyf = g->nyf;
    double norm = 0.0;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const double k_abs = sqrt((double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]));
            if (k_abs > UNIF_MIN_K && k_abs < UNIF_MAX_K) norm += (j == 0 || j == nyf - 1) ? 1.0 : 2.0;
        }
    norm = sqrt(1.0 / norm);
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            const double k_abs = sqrt((double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]));
            if (k_abs > UNIF_MIN_K && k_abs < UNIF_MAX_K) {
                const double u1 = urand();
                w[q] = norm * cexp(2.0 * M_PI * I * u1);
            } else {
                w[q] = 0.0;
            }
        }
}

/* RANDOM (solver.c:1875-1940).  The reference never initialises its
   enstrophy sum (enst_norm); it starts at 0 here. */
static void random_ic(const ns2d_grid* g, double complex* w) {
    const long Nx = g->nx, nyf = g->nyf;
    double enst_norm = 0.0;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            const double sqrt_k = sqrt(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]);
            if (sqrt_k > UNIF_MIN_K && sqrt_k < UNIF_MAX_K) {
                const double enrg_k = 1.0 / sqrt_k;
                const double enst_k = pow(sqrt_k, 2.0) * enrg_k;
                const double r1 = urand();
                w[q] = sqrt(enst_k / enrg_k) * cexp(r1 * 2.0 * M_PI * I);
            } else {
                w[q] = 0.0;
            }
            enst_norm += pow(cabs(w[q]), 2.0);
        }
    enst_norm *= 2.0;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            if (g->kx[i] != 0 || g->ky[j] != 0)
                w[q] *= sqrt(RAND_ENST0 / enst_norm);
            else
                w[q] = 0.0;
        }
}

static void testing_ic(const ns2d_grid* g, double complex* w) {
    for (long i = 0; i < g->nx; ++i)
        for (long j = 0; j < g->nyf; ++j) {
            const long q = i * g->nyf + j;
            if (g->kx[i] == 0 && g->ky[j] == 0) {
                w[q] = 0.0;
            } else {
                const double inv_k_sqr = 1.0 / (double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]);
                w[q] = (j == 0 && g->kx[i] < 0) ? inv_k_sqr * cexp(-I * M_PI / 4.0) : inv_k_sqr * cexp(I * M_PI / 4.0);
            }
        }
}

static void zero_ic(const ns2d_run* r, const ns2d_grid* g, double complex* w) {
    const int kolm = !strcmp(r->u0, "ZERO_KOLM");
    for (long i = 0; i < g->nx; ++i)
        for (long j = 0; j < g->nyf; ++j) {
            const long q = i * g->nyf + j;
            const int kx = g->kx[i], ky = g->ky[j];
            w[q] = 0.0;
            if (!kolm) continue;
            if (ky == 1 && kx == 1)
                w[q] = -0.5 + 0.0 * I;
            else if (ky == 2 && (kx == 3 || kx == 4))
                w[q] = -4.0 + 1.0 * I;
            else if (ky == 3 && (kx == 4 || kx == 5))
                w[q] = -2.0 + 3.0 * I;
            else if (ky == 4 && (kx == 5 || kx == 6))
                w[q] = 8.0 - 6.0 * I;
        }
}

/* Real-space initial conditions transformed with the GPU r2c. */
static int real_space_ic(const ns2d_run* r, const ns2d_grid* g, ns2d_handle* h, double complex* w) {
    const long Nx = g->nx, Ny = g->ny, nyf = g->nyf;
    const int vel = !strcmp(r->u0, "TG_VEL");
    double* f = (double*)malloc(sizeof(double) * (size_t)(Nx * Ny) * (vel ? 2 : 1));
    double complex* uh = vel ? (double complex*)malloc(sizeof(double complex) * (size_t)(Nx * nyf) * 2) : NULL;
    int rc = -1;
    if (!f || (vel && !uh)) goto out;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < Ny; ++j) {
            const long q = i * Ny + j;
            const double x = g->x[i], y = g->y[j];
            if (vel) {
                f[q] = cos(KAPPA * x) * sin(KAPPA * y);
                f[Nx * Ny + q] = -sin(KAPPA * x) * cos(KAPPA * y);
            } else if (!strcmp(r->u0, "TG_VORT")) {
                f[q] = 2.0 * KAPPA * cos(KAPPA * x) * cos(KAPPA * y);
            } else if (!strcmp(r->u0, "DOUBLE_SHEAR_LAYER")) {
                /* SIGMA = 15.0 / M_PI, expanded as the reference's macro is */
                f[q] = DELTA * cos(y) - 15.0 / M_PI / pow(cosh(15.0 / M_PI * (x - 0.5 * M_PI)), 2.0);
                f[q] += DELTA * cos(y) + 15.0 / M_PI / pow(cosh(15.0 / M_PI * (1.5 * M_PI - x)), 2.0);
            } else {
                /* GAUSS_BLOB (solver.c:1854-1874) evaluates the blob at the
                   integer wavenumbers k[0][i], k[1][j], reading k[1] beyond its
                   ny/2+1 entries; it is centred on the collocation points here. */
                f[q] = -exp(-(pow(x - M_PI, 2.0) + BETA * pow(y - M_PI, 2.0)) / pow(2.0 * M_PI / BLOB_S, 2.0));
            }
        }
    if (!vel) {
        rc = gpu(h, ns2d_fft_r2c(h, f, (double*)w), "r2c");
        goto out;
    }
    {
        /* TG_VEL: batched r2c of (u, v), dealiased, then w = i (kx v - ky u)
           (solver.c:1123-1160) */
        double complex* ux = uh;
        double complex* uy = uh + Nx * nyf;
        if (gpu(h, ns2d_fft_r2c(h, f, (double*)ux), "r2c") || gpu(h, ns2d_fft_r2c(h, f + Nx * Ny, (double*)uy), "r2c") ||
            gpu(h, ns2d_apply_dealiasing(h, (double*)ux, 1), "dealias") ||
            gpu(h, ns2d_apply_dealiasing(h, (double*)uy, 1), "dealias"))
            goto out;
        for (long i = 0; i < Nx; ++i)
            for (long j = 0; j < nyf; ++j) {
                const long q = i * nyf + j;
                if (g->kx[i] == 0 || g->ky[j] != 0)
                    w[q] = I * (g->kx[i] * uy[q] - g->ky[j] * ux[q]);
                else
                    w[q] = 0.0;
            }
        rc = 0;
    }
out:
    free(f);
    free(uh);
    return rc;
}

/* MAX_PALIN (solver.c:1775-1853): stream function "/psi" [nx][ny] of
   <input_dir>MaxPalinstrophy/maxdpdt_P10000_N<nx>_IG0_psi_f.h5, w = -k^2 psi_hat. */
static int max_palin(const ns2d_run* r, const ns2d_grid* g, ns2d_handle* h, double complex* w) {
    char path[1200];
    snprintf(path, sizeof(path), "%sMaxPalinstrophy/maxdpdt_P10000_N%ld_IG0_psi_f.h5", r->input_dir, r->N[0]);
    const long Nx = g->nx, Ny = g->ny, nyf = g->nyf;
    double* psi = (double*)malloc(sizeof(double) * (size_t)(Nx * Ny));
    if (!psi) return -1;
    if (ns2d_h5_read_double(path, "/psi", psi, (uint64_t)(Nx * Ny)) != 0) {
        fprintf(stderr, "\n[ERROR] --- Unable to read /psi of input file [%s]: %s\n-->> Exiting...\n", path,
                ns2d_h5_error(NULL));
        free(psi);
        return -1;
    }
    const int rc = gpu(h, ns2d_fft_r2c(h, psi, (double*)w), "r2c");
    free(psi);
    if (rc) return rc;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const long q = i * nyf + j;
            w[q] = -(double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]) * w[q];
        }
    return 0;
}

int ns2d_cli_initial(const ns2d_run* r, const ns2d_grid* g, ns2d_handle* h, double complex* w) {
    const char* u0 = r->u0;
    int rc = 0;
    srand(123456789);
    if (!strcmp(u0, "TG_VEL") || !strcmp(u0, "TG_VORT") || !strcmp(u0, "DOUBLE_SHEAR_LAYER") ||
        !strcmp(u0, "GAUSS_BLOB")) {
        rc = real_space_ic(r, g, h, w);
    } else if (!strcmp(u0, "ZERO") || !strcmp(u0, "ZERO_KOLM")) {
        zero_ic(r, g, w);
    } else if (!strcmp(u0, "DECAY_TURB_BB") || !strcmp(u0, "DECAY_TURB_NB") || !strcmp(u0, "DECAY_TURB_EXP")) {
        decay_turb(r, g, w);
    } else if (!strcmp(u0, "DECAY_TURB_ALT")) {
        rc = decay_turb_alt(g, h, w);
    } else if (!strcmp(u0, "GAUSS_DECAY_TURB")) {
        gauss_decay_turb(g, w);
    } else if (!strcmp(u0, "EXTRM_ENS")) {
        extrm_ens(g, w);
    } else if (!strcmp(u0, "RING")) {
        ring(g, w);
    } else if (!strcmp(u0, "UNIF")) {
        unif(g, w);
    } else if (!strcmp(u0, "MAX_PALIN")) {
        rc = max_palin(r, g, h, w);
    } else if (!strcmp(u0, "RANDOM")) {
        random_ic(g, w);
    } else if (!strcmp(u0, "TESTING")) {
        testing_ic(g, w);
    } else {
        if (!r->quiet) printf("\n[WARNING] --- No initial conditions specified\n---> Using random initial conditions...\n");
        /* amplitude first, then phase: the order gcc evaluates the
           reference's single expression in (solver.c:1986) */
        for (long q = 0; q < g->nx * g->nyf; ++q) {
            const double a = urand();
            const double p = urand();
            w[q] = a * cexp(p * 2.0 * M_PI * I);
        }
    }
    if (rc) return rc;
    /* ApplyDealiasing(w_hat, 1) and ForceConjugacy(w_hat) (solver.c:1994-1997) */
    if (gpu(h, ns2d_apply_dealiasing(h, (double*)w, 1), "dealias")) return -1;
    for (long i = 0; i < g->nx; ++i)
        if (g->kx[i] < 0) w[i * g->nyf] = conj(w[(long)abs(g->kx[i]) * g->nyf]);
    return 0;
}

/* ---- forcing ----------------------------------------------------------------- */
int ns2d_cli_forcing_init(const ns2d_run* r, const ns2d_grid* g, ns2d_forcing_modes* f) {
    memset(f, 0, sizeof(*f));
    const long Nx = g->nx, nyf = g->nyf;
    if (!strcmp(r->forcing, "STOC"))
        f->kind = 1;
    else if (!strcmp(r->forcing, "STOC_GAUSS"))
        f->kind = 2;
    else if (!strcmp(r->forcing, "CONST_GAUSS"))
        f->kind = 3;
    else
        return 0;
    /* which modes, and the normalisation sums (force.c:104-433) */
    double sum = 0.0;
    int n = 0;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            const double k_abs = sqrt((double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]));
            if (f->kind == 3) {
                if (k_abs >= CONST_GAUSS_K_MIN && k_abs < CONST_GAUSS_K_MAX) n++;
                continue;
            }
            if (g->kx[i] == 0 && g->ky[j] == 0) continue;
            if (f->kind == 1) {
                const double e = exp(-pow(k_abs - r->force_k, 2.0) / (2.0 * STOC_FORC_UNIF_DELTA_K * STOC_FORC_UNIF_DELTA_K));
                sum += (j == 0 || j == nyf - 1) ? e / (2.0 * pow(k_abs, 2.0)) : 2.0 * e / (2.0 * pow(k_abs, 2.0));
                n++;
            } else if (k_abs > r->force_k - 0.5 && k_abs < r->force_k + 0.5) {
                sum += (j == 0 || j == nyf - 1) ? pow(k_abs, 2.0) : 2.0 * pow(k_abs, 2.0);
                n++;
            }
        }
    f->n = n;
    f->indx = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    f->scaling = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    f->value = (double complex*)calloc((size_t)(n > 0 ? n : 1), sizeof(double complex));
    if (!f->indx || !f->scaling || !f->value) return -1;
    if (f->kind == 3) {
        /* Gaussian values drawn once and normalised by their total power
           (force.c:305-433); the reference also writes the draws for ky = 0
           into a scratch array through a row-indexed ky lookup, which nothing
           reads, so that write is left out. */
        double scale_fac_f0 = 0.0;
        int c = 0;
        for (long i = 0; i < Nx; ++i)
            for (long j = 0; j < nyf; ++j) {
                const double k_abs = sqrt((double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]));
                if (!(k_abs >= CONST_GAUSS_K_MIN && k_abs < CONST_GAUSS_K_MAX)) continue;
                const double r1 = urand();
                const double r2 = urand();
                const double re_f = sqrt(-2.0 * log(r1)) * cos(r2 * 2.0 * M_PI);
                const double im_f = sqrt(-2.0 * log(r1)) * sin(r2 * 2.0 * M_PI);
                f->value[c] = re_f + im_f * I;
                f->indx[c] = (int32_t)(i * nyf + j);
                c++;
                scale_fac_f0 += cabs(re_f + im_f * I) * cabs(re_f + im_f * I);
            }
        for (int m = 0; m < n; ++m) {
            f->value[m] = (f->value[m] / sqrt(scale_fac_f0)) * sqrt(0.0025);
            f->scaling[m] = sqrt(0.0025);
        }
        return 0;
    }
    const double sum_n = sum * (1.0 / pow(r->N[0] * r->N[1], 2.0));
    const double scale_fac_f0 = (f->kind == 1) ? r->force_scale / sum_n : sqrt(r->force_scale / sum_n);
    int c = 0;
    for (long i = 0; i < Nx; ++i)
        for (long j = 0; j < nyf; ++j) {
            if (g->kx[i] == 0 && g->ky[j] == 0) continue;
            const double k_abs = sqrt((double)(g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j]));
            if (f->kind == 1) {
                f->scaling[c] = scale_fac_f0 * exp(-pow(k_abs - r->force_k, 2.0) /
                                                   (2.0 * STOC_FORC_UNIF_DELTA_K * STOC_FORC_UNIF_DELTA_K));
            } else if (k_abs > r->force_k - 0.5 && k_abs < r->force_k + 0.5) {
                f->scaling[c] = scale_fac_f0 * pow(k_abs, 1.0);
            } else {
                continue;
            }
            f->indx[c++] = (int32_t)(i * nyf + j);
        }
    return 0;
}

/* ComputeForcing (force.c:540-577) for the host-drawn kinds. */
void ns2d_cli_forcing_draw(ns2d_forcing_modes* f, double dt) {
    for (int i = 0; i < f->n; ++i) {
        if (f->kind == 2) {
            const double r1 = urand();
            const double r2 = urand();
            const double re_f = sqrt(-2.0 * log(r1)) * cos(r2 * 2.0 * M_PI);
            const double im_f = sqrt(-2.0 * log(r1)) * sin(r2 * 2.0 * M_PI);
            f->value[i] = f->scaling[i] * (re_f + im_f * I);
        } else if (f->kind == 1) {
            const double r1 = urand();
            f->value[i] = sqrt(f->scaling[i]) * cexp(2.0 * M_PI * I * r1) / sqrt(dt);
        } else if (f->kind == 3) {
            f->value[i] *= f->scaling[i];
        }
    }
}

void ns2d_cli_forcing_free(ns2d_forcing_modes* f) {
    free(f->indx);
    free(f->scaling);
    free(f->value);
    memset(f, 0, sizeof(*f));
}
