/*
 * phase_sync.c -- sector phase synchronisation of bin/ns2d_post (--phase-sync),
 * the outputs of the post-processing program built with -D__SEC_PHASE_SYNC:
 *
 *   sector geometry          AllocatePhaseSyncMemory (phase_sync.c:1396-1434,
 *                            1744-1776), k1 sector bounds of the search
 *   triad sums               ns2d_triad_sector_sums on the GPU (the search of
 *                            phase_sync.c:1778-1948 and the accumulation of
 *                            PhaseSyncSector, phase_sync.c:281-1058)
 *   combination, order       PhaseSyncSector's per-type arrays and their
 *   parameters               normalisation (phase_sync.c:1060-1084)
 *   C_theta sums             FluxSpectra's -D__SEC_PHASE_SYNC part
 *                            (full_field.c:399-530), on the host from the GPU RHS
 *   datasets                 WriteDataToFile / FinalWriteAndCloseOutputFile
 *                            (hdf5_funcs.c:796-1060, 1698-1780)
 *
 * Triad types (NUM_TRIAD_TYPES + 1 = 7 rows): 0 all, 1 / 2 the positive flux
 * term with flux_pre_fac < 0 / > 0, 3 / 4 the negative term likewise, 5
 * flux_pre_fac == 0, 6 never reached (flux_pre_fac is finite).
 */
#include "phase_sync.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NT 7              /* NUM_TRIAD_TYPES + 1 (PostProcessing/src/data_types.h:96) */
#define NUM_K1_SECTORS 8  /* data_types.h:97 */

struct ps_state {
    int nx, nyf, kmax, A, L, device;
    double kmax_sqr, kmax_c_sqr;
    int hyper_flag, drag_flag;
    double nu, hyper_pow, alpha, drag_pow;
    double dtheta_k3, dtheta_k1;
    double *theta_k3, *theta_k1;
    double *k3_lwr, *k3_upr, *k1_lwr, *k1_upr, *ang, *ang_neg;
    double* sums;
    /* per snapshot, [NT][A] and [NT][A][L] */
    int *num, *num1, *num2;
    double *flux, *flux1, *flux2;
    double complex *ord, *ord1, *ord2;
    double complex *cth, *cthu, *cth1, *cthu1, *cth2, *cthu2;
    double *r, *phi, *r1, *phi1, *r2, *phi2;
    double *flux_c, *diss_c;
    double complex *order_c, *diss_field;
};

/* MyMod (PostProcessing/src/utils.c:283-291): fmod shifted into [0, y) */
static double my_mod(double x, double y) {
    double rem = fmod(x, y);
    if (rem < 0) rem += y;
    return rem;
}

ps_state* ps_create(int nx, int kmax, double kmax_frac, int n_k3, int n_k1, int reduced, double nu, int hyper_flag,
                    double hyper_pow, double alpha, int drag_flag, double drag_pow, int device) {
    ps_state* s = (ps_state*)calloc(1, sizeof(ps_state));
    if (!s) return NULL;
    s->nx = nx;
    s->nyf = nx / 2 + 1;
    s->kmax = kmax;
    s->A = n_k3;
    s->L = n_k1;
    s->device = device;
    s->nu = nu;
    s->hyper_flag = hyper_flag;
    s->hyper_pow = hyper_pow;
    s->alpha = alpha;
    s->drag_flag = drag_flag;
    s->drag_pow = drag_pow;
    s->kmax_sqr = pow(kmax, 2.0);
    const int kmax_c = (int)ceil(kmax_frac * kmax);
    s->kmax_c_sqr = pow(kmax_c, 2.0);
    const int A = n_k3, L = n_k1, side = 2 * kmax + 1;
    const size_t m = (size_t)side * side, na = (size_t)NT * A, nal = na * L;
    s->theta_k3 = calloc((size_t)A, sizeof(double));
    s->theta_k1 = calloc((size_t)L, sizeof(double));
    s->k3_lwr = calloc((size_t)A, sizeof(double));
    s->k3_upr = calloc((size_t)A, sizeof(double));
    s->k1_lwr = calloc((size_t)A * L, sizeof(double));
    s->k1_upr = calloc((size_t)A * L, sizeof(double));
    s->ang = calloc(m, sizeof(double));
    s->ang_neg = calloc(m, sizeof(double));
    s->sums = calloc((size_t)A * L * 6 * 4 * 8, sizeof(double));
    s->num = calloc(na, sizeof(int));
    s->num1 = calloc(na, sizeof(int));
    s->num2 = calloc(nal, sizeof(int));
    s->flux = calloc(na, sizeof(double));
    s->flux1 = calloc(na, sizeof(double));
    s->flux2 = calloc(nal, sizeof(double));
    s->ord = calloc(na, sizeof(double complex));
    s->ord1 = calloc(na, sizeof(double complex));
    s->ord2 = calloc(nal, sizeof(double complex));
    s->cth = calloc(na, sizeof(double complex));
    s->cthu = calloc(na, sizeof(double complex));
    s->cth1 = calloc(na, sizeof(double complex));
    s->cthu1 = calloc(na, sizeof(double complex));
    s->cth2 = calloc(nal, sizeof(double complex));
    s->cthu2 = calloc(nal, sizeof(double complex));
    s->r = calloc(na, sizeof(double));
    s->phi = calloc(na, sizeof(double));
    s->r1 = calloc(na, sizeof(double));
    s->phi1 = calloc(na, sizeof(double));
    s->r2 = calloc(nal, sizeof(double));
    s->phi2 = calloc(nal, sizeof(double));
    s->flux_c = calloc((size_t)A, sizeof(double));
    s->diss_c = calloc((size_t)A, sizeof(double));
    s->order_c = calloc((size_t)A, sizeof(double complex));
    s->diss_field = calloc((size_t)nx * s->nyf, sizeof(double complex));
    if (!s->theta_k3 || !s->theta_k1 || !s->k3_lwr || !s->k3_upr || !s->k1_lwr || !s->k1_upr || !s->ang ||
        !s->ang_neg || !s->sums || !s->num || !s->num1 || !s->num2 || !s->flux || !s->flux1 || !s->flux2 || !s->ord ||
        !s->ord1 || !s->ord2 || !s->cth || !s->cthu || !s->cth1 || !s->cthu1 || !s->cth2 || !s->cthu2 || !s->r ||
        !s->phi || !s->r1 || !s->phi1 || !s->r2 || !s->phi2 || !s->flux_c || !s->diss_c || !s->order_c ||
        !s->diss_field) {
        ps_free(s);
        return NULL;
    }
    /* sector mid-point angles (phase_sync.c:1397-1434) */
    s->dtheta_k3 = M_PI / (double)A;
    for (int i = 0; i < A; ++i) s->theta_k3[i] = -M_PI / 2.0 + i * s->dtheta_k3 + s->dtheta_k3 / 2.0 + 1e-10;
    s->dtheta_k1 = M_PI / (double)L;
    for (int i = 0; i < L; ++i) s->theta_k1[i] = -M_PI / 2.0 + i * s->dtheta_k1 + s->dtheta_k1 / 2.0 + 1e-10;
    /* the search's sector bounds (phase_sync.c:1744-1776); the k1 sector of loop
       index l is stored at (l + a) mod n_k1 */
    const double k1_sector_angles[NUM_K1_SECTORS] = {-A / 2.0, -A / 3.0, -A / 4.0, -A / 6.0,
                                                     A / 6.0,  A / 4.0,  A / 3.0,  A / 2.0};
    for (int a = 0; a < A; ++a) {
        const double c3 = s->theta_k3[a];
        s->k3_lwr[a] = c3 - s->dtheta_k3 / 2.0;
        s->k3_upr[a] = c3 + s->dtheta_k3 / 2.0;
        for (int l = 0; l < L; ++l) {
            double c1, lo, hi;
            if (reduced) {
                c1 = my_mod(c3 + (k1_sector_angles[l % NUM_K1_SECTORS] * s->dtheta_k3 / 2.0) + M_PI, 2.0 * M_PI) - M_PI;
                lo = c1 - s->dtheta_k3 / 2.0;
                hi = c1 + s->dtheta_k3 / 2.0;
            } else if (L == 1) {
                c1 = 0.0;
                lo = c1 - M_PI / 2.0 + 1e-10;
                hi = c1 + M_PI / 2.0 + 1e-10;
            } else {
                c1 = s->theta_k1[(a + l) % L];
                lo = c1 - s->dtheta_k1 / 2.0;
                hi = c1 + s->dtheta_k1 / 2.0;
            }
            const int ls = (l + a) % L;
            s->k1_lwr[(size_t)a * L + ls] = lo;
            s->k1_upr[(size_t)a * L + ls] = hi;
        }
    }
    /* wavevector angles as the search takes them (phase_sync.c:1795-1797) */
    for (int i = 0; i < side; ++i)
        for (int j = 0; j < side; ++j) {
            const int kx = kmax - i, ky = j - kmax;
            s->ang[(size_t)i * side + j] = atan2((double)kx, (double)ky);
            s->ang_neg[(size_t)i * side + j] = atan2((double)-kx, (double)-ky);
        }
    return s;
}

void ps_free(ps_state* s) {
    if (!s) return;
    void* p[] = {s->theta_k3, s->theta_k1, s->k3_lwr, s->k3_upr, s->k1_lwr, s->k1_upr, s->ang,   s->ang_neg,
                 s->sums,     s->num,      s->num1,   s->num2,   s->flux,   s->flux1,  s->flux2, s->ord,
                 s->ord1,     s->ord2,     s->cth,    s->cthu,   s->cth1,   s->cthu1,  s->cth2,  s->cthu2,
                 s->r,        s->phi,      s->r1,     s->phi1,   s->r2,     s->phi2,   s->flux_c, s->diss_c,
                 s->order_c,  s->diss_field};
    for (size_t k = 0; k < sizeof(p) / sizeof(p[0]); ++k) free(p[k]);
    free(s);
}

/* viscous prefactor of FluxSpectra (full_field.c:425-445) */
static double pre_factor(const ps_state* s, double k_sqr) {
    if (s->hyper_flag == 1 && s->drag_flag == 1)
        return s->nu * pow(k_sqr, s->hyper_pow) + s->alpha * pow(k_sqr, s->drag_pow);
    if (s->hyper_flag != 1 && s->drag_flag == 1) return s->nu * k_sqr + s->alpha * pow(k_sqr, s->drag_pow);
    if (s->hyper_flag == 1 && s->drag_flag != 1) return s->nu * pow(k_sqr, s->hyper_pow);
    return s->nu * k_sqr;
}

ns2d_status ps_snapshot(ps_state* s, const double complex* w, const double complex* rhs, const double* amps,
                        const double* phases) {
    const int A = s->A, L = s->L;
    const size_t na = (size_t)NT * A, nal = na * L;
    /* ---- FluxSpectra's sector sums (full_field.c:399-530) */
    const double norm_fac = 0.5 / pow((double)s->nx * s->nx, 2.0);
    const double const_fac = 4.0 * pow(M_PI, 2.0);
    for (int a = 0; a < A; ++a) {
        s->flux_c[a] = 0.0;
        s->diss_c[a] = 0.0;
        s->order_c[a] = 0.0;
    }
    for (int i = 0; i < s->nx; ++i) {
        const int kx = i <= s->nx / 2 ? i : i - s->nx;
        for (int j = 0; j < s->nyf; ++j) {
            const size_t q = (size_t)i * s->nyf + j;
            if (kx == 0 && j == 0) continue;
            const double k_sqr = (double)(kx * kx + j * j);
            const double pre_fac = pre_factor(s, k_sqr);
            const double tmp_deriv = creal(w[q] * conj(rhs[q]) + conj(w[q]) * rhs[q]) * const_fac * norm_fac;
            const double tmp_diss = pre_fac * cabs(w[q] * conj(w[q])) * const_fac * norm_fac;
            s->diss_field[q] = pre_fac * w[q];
            if (!(k_sqr > s->kmax_c_sqr && k_sqr <= s->kmax_sqr)) continue;
            const double angle = atan2((double)kx, (double)j);
            const int edge = (j == 0 || j == s->nyf - 1);
            for (int a = 0; a < A; ++a) {
                if (angle >= s->theta_k3[a] - s->dtheta_k3 / 2.0 && angle < s->theta_k3[a] + s->dtheta_k3 / 2.0) {
                    s->diss_c[a] += tmp_diss;
                    s->flux_c[a] += tmp_deriv;
                    if ((!edge || kx > 0) && fabs(tmp_deriv) != 0.0)
                        s->order_c[a] += (tmp_deriv + tmp_diss) / fabs(tmp_deriv);
                }
            }
        }
    }
    /* ---- triad sums on the GPU */
    ns2d_triad_sectors g;
    memset(&g, 0, sizeof(g));
    g.kmax = s->kmax;
    g.n_k3 = A;
    g.n_k1 = L;
    g.kmax_sqr = s->kmax_sqr;
    g.kmax_c_sqr = s->kmax_c_sqr;
    g.k3_lwr = s->k3_lwr;
    g.k3_upr = s->k3_upr;
    g.k1_lwr = s->k1_lwr;
    g.k1_upr = s->k1_upr;
    g.angle = s->ang;
    g.angle_neg = s->ang_neg;
    ns2d_status st = ns2d_triad_sector_sums(s->device, &g, amps, phases, s->sums);
    if (st != NS2D_OK) return st;
    /* ---- PhaseSyncSector's arrays (phase_sync.c:298-1058): type 0 and the
       triad's own type, all / 1d / 2d */
    memset(s->num, 0, na * sizeof(int));
    memset(s->num1, 0, na * sizeof(int));
    memset(s->num2, 0, nal * sizeof(int));
    memset(s->flux, 0, na * sizeof(double));
    memset(s->flux1, 0, na * sizeof(double));
    memset(s->flux2, 0, nal * sizeof(double));
    double complex* zc[] = {s->ord, s->ord1, s->cth, s->cthu, s->cth1, s->cthu1};
    for (int k = 0; k < 6; ++k) memset(zc[k], 0, na * sizeof(double complex));
    memset(s->ord2, 0, nal * sizeof(double complex));
    memset(s->cth2, 0, nal * sizeof(double complex));
    memset(s->cthu2, 0, nal * sizeof(double complex));
    static const int type_of[2][3] = {{1, 2, 5}, {3, 4, 5}};
    for (int a = 0; a < A; ++a)
        for (int l = 0; l < L; ++l)
            for (int term = 0; term < 2; ++term)
                for (int cls = 0; cls < 3; ++cls)
                    for (int contrib = 0; contrib < 2; ++contrib)
                        for (int uni = 0; uni < 2; ++uni) {
                            const double* v =
                                s->sums + (((((size_t)a * L + l) * 2 + term) * 3 + cls) * 2 + contrib) * 2 * 8 + uni * 8;
                            const int cnt = (int)v[0];
                            if (cnt == 0) continue;
                            const int types[2] = {0, type_of[term][cls]};
                            const double complex ordv[2] = {v[2] + I * v[3], v[4] + I * v[5]};
                            const double complex cv = v[6] + I * v[7];
                            for (int t = 0; t < 2; ++t) {
                                const size_t ia = (size_t)types[t] * A + a;
                                const size_t ial = ia * L + l;
                                s->num[ia] += cnt;
                                s->flux[ia] += v[1];
                                s->ord[ia] += ordv[t];
                                s->cth[ia] += cv;
                                if (uni) s->cthu[ia] += cv;
                                if (contrib == 0) {
                                    s->num1[ia] += cnt;
                                    s->flux1[ia] += v[1];
                                    s->ord1[ia] += ordv[t];
                                    s->cth1[ia] += cv;
                                    if (uni) s->cthu1[ia] += cv;
                                } else {
                                    s->num2[ial] += cnt;
                                    s->flux2[ial] += v[1];
                                    s->ord2[ial] += ordv[t];
                                    s->cth2[ial] += cv;
                                    if (uni) s->cthu2[ial] += cv;
                                }
                            }
                        }
    /* normalisation (phase_sync.c:1060-1084) */
    for (size_t k = 0; k < na; ++k) {
        if (s->num[k] != 0) s->ord[k] /= s->num[k];
        if (s->num1[k] != 0) s->ord1[k] /= s->num1[k];
        s->r[k] = cabs(s->ord[k]);
        s->phi[k] = carg(s->ord[k]);
        s->r1[k] = cabs(s->ord1[k]);
        s->phi1[k] = carg(s->ord1[k]);
    }
    for (size_t k = 0; k < nal; ++k) {
        if (s->num2[k] != 0) s->ord2[k] /= s->num2[k];
        s->r2[k] = cabs(s->ord2[k]);
        s->phi2[k] = carg(s->ord2[k]);
    }
    return NS2D_OK;
}

static int put(ns2d_h5_file* f, const char* group, const char* name, int type, int rank, const uint64_t* dims,
               const void* data) {
    char path[256];
    snprintf(path, sizeof(path), "%s/%s", group, name);
    if (ns2d_h5_dataset(f, path, type, rank, dims, data) != 0) {
        fprintf(stderr, "\n[ERROR] --- Unable to write [%s]: %s\n-->> Exiting...\n", path, ns2d_h5_error(f));
        return -1;
    }
    return 0;
}

int ps_write_snapshot(const ps_state* s, ns2d_h5_file* f, const char* group) {
    const uint64_t d1[1] = {(uint64_t)s->A}, dt[1] = {NT}, d2[2] = {NT, (uint64_t)s->A},
                   d3[3] = {NT, (uint64_t)s->A, (uint64_t)s->L}, dw[2] = {(uint64_t)s->nx, (uint64_t)s->nyf};
    double* zeros = calloc((size_t)(s->A > NT ? s->A : NT), sizeof(double));
    if (!zeros) return -1;
    int rc = 0;
    /* individual-phase order parameters and the single-sector test arrays: the
       reference zeroes them at set-up and never fills them */
    rc |= put(f, group, "PhaseSync", NS2D_H5_F64, 1, d1, zeros);
    rc |= put(f, group, "AverageAngle", NS2D_H5_F64, 1, d1, zeros);
    rc |= put(f, group, "TriadPhaseSyncTest", NS2D_H5_F64, 1, dt, zeros);
    rc |= put(f, group, "TriadAverageAngleTest", NS2D_H5_F64, 1, dt, zeros);
    rc |= put(f, group, "TriadPhaseSync", NS2D_H5_F64, 2, d2, s->r);
    rc |= put(f, group, "TriadAverageAngle", NS2D_H5_F64, 2, d2, s->phi);
    rc |= put(f, group, "TriadPhaseSync_1D", NS2D_H5_F64, 2, d2, s->r1);
    rc |= put(f, group, "TriadAverageAngle_1D", NS2D_H5_F64, 2, d2, s->phi1);
    rc |= put(f, group, "TriadPhaseSync_2D", NS2D_H5_F64, 3, d3, s->r2);
    rc |= put(f, group, "TriadAverageAngle_2D", NS2D_H5_F64, 3, d3, s->phi2);
    rc |= put(f, group, "EnstrophyFlux_C_theta", NS2D_H5_F64, 1, d1, s->flux_c);
    rc |= put(f, group, "EnstrophyDiss_C_theta", NS2D_H5_F64, 1, d1, s->diss_c);
    rc |= put(f, group, "CollectivePhaseOrder_C_theta", NS2D_H5_C128, 1, d1, s->order_c);
    rc |= put(f, group, "CollectivePhaseOrder_C_theta_Triads", NS2D_H5_C128, 2, d2, s->cth);
    rc |= put(f, group, "CollectivePhaseOrder_C_theta_Triads_Unidirectional", NS2D_H5_C128, 2, d2, s->cthu);
    rc |= put(f, group, "CollectivePhaseOrder_C_theta_Triads_1D", NS2D_H5_C128, 2, d2, s->cth1);
    rc |= put(f, group, "CollectivePhaseOrder_C_theta_Triads_1D_Unidirectional", NS2D_H5_C128, 2, d2, s->cthu1);
    rc |= put(f, group, "CollectivePhaseOrder_C_theta_Triads_2D", NS2D_H5_C128, 3, d3, s->cth2);
    rc |= put(f, group, "CollectivePhaseOrder_C_theta_Triads_2D_Unidirectional", NS2D_H5_C128, 3, d3, s->cthu2);
    rc |= put(f, group, "EnstrophyFluxTest", NS2D_H5_F64, 1, dt, zeros);
    rc |= put(f, group, "EnstrophyFluxPerSector", NS2D_H5_F64, 2, d2, s->flux);
    rc |= put(f, group, "EnstrophyFluxPerSector_1D", NS2D_H5_F64, 2, d2, s->flux1);
    rc |= put(f, group, "EnstrophyFluxPerSector_2D", NS2D_H5_F64, 3, d3, s->flux2);
    rc |= put(f, group, "EnstrophyDissipationField", NS2D_H5_C128, 2, dw, s->diss_field);
    free(zeros);
    return rc ? -1 : 0;
}

int ps_write_final(const ps_state* s, ns2d_h5_file* f) {
    const uint64_t d3k[1] = {(uint64_t)s->A}, d1k[1] = {(uint64_t)s->L}, dt[1] = {NT}, d2[2] = {NT, (uint64_t)s->A},
                   d3[3] = {NT, (uint64_t)s->A, (uint64_t)s->L};
    const int zeros[NT] = {0};
    int rc = 0;
    rc |= put(f, "", "SectorAngles_k3", NS2D_H5_F64, 1, d3k, s->theta_k3);
    rc |= put(f, "", "SectorAngles_k1", NS2D_H5_F64, 1, d1k, s->theta_k1);
    rc |= put(f, "", "NumTriadsTest", NS2D_H5_I32, 1, dt, zeros);
    rc |= put(f, "", "NumTriadsPerSector", NS2D_H5_I32, 2, d2, s->num);
    rc |= put(f, "", "NumTriadsPerSector_1D", NS2D_H5_I32, 2, d2, s->num1);
    rc |= put(f, "", "NumTriadsPerSector_2D", NS2D_H5_I32, 3, d3, s->num2);
    return rc ? -1 : 0;
}
