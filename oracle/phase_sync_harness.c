/*
 * oracle/phase_sync_harness.c -- the reference post-processing program's sector
 * phase synchronisation (PostProcessing/src/phase_sync.c, and the
 * -D__SEC_PHASE_SYNC parts of full_field.c's FluxSpectra) on one snapshot
 * through ctypes: the checker of bin/ns2d_post --phase-sync.  Test
 * infrastructure only.
 *
 * ps_init plays PostProcessing()'s set-up for that build (post_proc.c:308-470):
 * wavenumbers, AllocateFullFieldMemory, AllocatePhaseSyncMemory (sector
 * angles, the triad search, and the write of the wavevector file to
 * ./Data/PostProcess/PhaseSync/, which the caller creates), the serial FFTW
 * plans.  AllocateFullFieldMemory sizes the C_theta arrays by the number of
 * snapshots (full_field.c:678-690) while FluxSpectra fills one entry per k3
 * sector, so the harness asks for as many snapshots as sectors.
 * ps_snapshot runs FluxSpectra, FullFieldData and PhaseSyncSector on one
 * w_hat (post_proc.c:88-104); the ps_get_* calls copy the results out in the
 * layouts WriteDataToFile gives them (hdf5_funcs.c:796-1060, 1698-1780).
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "data_types.h"
#include "full_field.h"
#include "phase_sync.h"

runtime_data_struct* run_data;
system_vars_struct* sys_vars;
HDF_file_info_struct* file_info;
postprocess_data_struct* proc_data;
stats_data_struct* stats_data;

#define NT (NUM_TRIAD_TYPES + 1)

int ps_init(int n, double nu, int hyper_flag, double hyper_pow, double alpha, int drag_flag, double drag_pow,
            double kmax_frac, int n_k3, int n_k1, int reduced) {
    sys_vars = (system_vars_struct*)calloc(1, sizeof(system_vars_struct));
    run_data = (runtime_data_struct*)calloc(1, sizeof(runtime_data_struct));
    file_info = (HDF_file_info_struct*)calloc(1, sizeof(HDF_file_info_struct));
    proc_data = (postprocess_data_struct*)calloc(1, sizeof(postprocess_data_struct));
    stats_data = (stats_data_struct*)calloc(1, sizeof(stats_data_struct));
    sys_vars->N[0] = n;
    sys_vars->N[1] = n;
    sys_vars->num_snaps = n_k3 > 1 ? n_k3 : 1;
    sys_vars->NU = nu;
    sys_vars->HYPER_VISC_FLAG = hyper_flag;
    sys_vars->HYPER_VISC_POW = hyper_pow;
    sys_vars->EKMN_ALPHA = alpha;
    sys_vars->EKMN_DRAG_FLAG = drag_flag;
    sys_vars->EKMN_DRAG_POW = drag_pow;
    sys_vars->kmax_frac = kmax_frac;
    sys_vars->num_k3_sectors = n_k3;
    sys_vars->num_k1_sectors = n_k1;
    sys_vars->REDUCED_K1_SEARCH_FLAG = reduced;
    const long nyf = n / 2 + 1;
    run_data->k[0] = (int*)calloc((size_t)n, sizeof(int));
    run_data->k[1] = (int*)calloc((size_t)nyf, sizeof(int));
    for (int i = 0; i < n; ++i) run_data->k[0][i] = i <= n / 2 ? i : i - n;
    for (int j = 0; j < nyf; ++j) run_data->k[1][j] = j;
    run_data->w_hat = (fftw_complex*)calloc((size_t)(n * nyf), sizeof(fftw_complex));
    run_data->u_hat = (fftw_complex*)calloc((size_t)(2 * n * nyf), sizeof(fftw_complex));
    run_data->w = (double*)calloc((size_t)(n * n), sizeof(double));
    run_data->u = (double*)calloc((size_t)(2 * n * n), sizeof(double));
    AllocateFullFieldMemory(sys_vars->N);
    proc_data->enst_flux_C = (double*)calloc((size_t)sys_vars->num_snaps, sizeof(double));
    proc_data->enst_diss_C = (double*)calloc((size_t)sys_vars->num_snaps, sizeof(double));
    proc_data->enrg_flux_C = (double*)calloc((size_t)sys_vars->num_snaps, sizeof(double));
    proc_data->enrg_diss_C = (double*)calloc((size_t)sys_vars->num_snaps, sizeof(double));
    AllocatePhaseSyncMemory(sys_vars->N);
    const int nb[2] = {n, n};
    sys_vars->fftw_2d_dft_r2c = fftw_plan_dft_r2c_2d(n, n, run_data->w, run_data->w_hat, FFTW_MEASURE);
    sys_vars->fftw_2d_dft_batch_c2r =
        fftw_plan_many_dft_c2r(2, nb, 2, run_data->u_hat, NULL, 2, 1, run_data->u, NULL, 2, 1, FFTW_MEASURE);
    return sys_vars->kmax;
}

void ps_snapshot(const double* w_hat) {
    const long n = sys_vars->N[0], nyf = n / 2 + 1;
    memcpy(run_data->w_hat, w_hat, sizeof(fftw_complex) * (size_t)(n * nyf));
    proc_data->enst_flux_C[0] = proc_data->enst_diss_C[0] = 0.0;
    proc_data->enrg_flux_C[0] = proc_data->enrg_diss_C[0] = 0.0;
    FluxSpectra(0);
    FullFieldData();
    PhaseSyncSector(0);
}

/* [NT][n_k3] and [NT][n_k3][n_k1] arrays, row-major as WriteDataToFile lays them out */
static void put2(double* out, double** src) {
    const int A = sys_vars->num_k3_sectors;
    for (int i = 0; i < NT; ++i)
        for (int a = 0; a < A; ++a) out[i * A + a] = src[i][a];
}
static void put3(double* out, double*** src) {
    const int A = sys_vars->num_k3_sectors, L = sys_vars->num_k1_sectors;
    for (int i = 0; i < NT; ++i)
        for (int a = 0; a < A; ++a)
            for (int l = 0; l < L; ++l) out[(i * A + a) * L + l] = src[i][a][l];
}
static void put2c(double* out, fftw_complex** src) {
    const int A = sys_vars->num_k3_sectors;
    for (int i = 0; i < NT; ++i)
        for (int a = 0; a < A; ++a) {
            out[2 * (i * A + a)] = creal(src[i][a]);
            out[2 * (i * A + a) + 1] = cimag(src[i][a]);
        }
}
static void put3c(double* out, fftw_complex*** src) {
    const int A = sys_vars->num_k3_sectors, L = sys_vars->num_k1_sectors;
    for (int i = 0; i < NT; ++i)
        for (int a = 0; a < A; ++a)
            for (int l = 0; l < L; ++l) {
                out[2 * ((i * A + a) * L + l)] = creal(src[i][a][l]);
                out[2 * ((i * A + a) * L + l) + 1] = cimag(src[i][a][l]);
            }
}

/* counts: num [NT][A], num_1d [NT][A], num_2d [NT][A][L] */
void ps_get_counts(int* num, int* num1d, int* num2d) {
    const int A = sys_vars->num_k3_sectors, L = sys_vars->num_k1_sectors;
    for (int i = 0; i < NT; ++i)
        for (int a = 0; a < A; ++a) {
            num[i * A + a] = proc_data->num_triads[i][a];
            num1d[i * A + a] = proc_data->num_triads_1d[i][a];
            for (int l = 0; l < L; ++l) num2d[(i * A + a) * L + l] = proc_data->num_triads_2d[i][a][l];
        }
}

/* R, Phi, R_1d, Phi_1d ([NT][A] each), R_2d, Phi_2d ([NT][A][L]) */
void ps_get_sync(double* r, double* phi, double* r1, double* phi1, double* r2, double* phi2) {
    put2(r, proc_data->triad_R);
    put2(phi, proc_data->triad_Phi);
    put2(r1, proc_data->triad_R_1d);
    put2(phi1, proc_data->triad_Phi_1d);
    put3(r2, proc_data->triad_R_2d);
    put3(phi2, proc_data->triad_Phi_2d);
}

/* enstrophy flux per sector: [NT][A], [NT][A], [NT][A][L] */
void ps_get_flux(double* f, double* f1, double* f2) {
    put2(f, proc_data->enst_flux);
    put2(f1, proc_data->enst_flux_1d);
    put3(f2, proc_data->enst_flux_2d);
}

/* collective phase order of the triads (complex as re, im): C, C_unidirec,
   C_1d, C_unidirec_1d ([NT][A]), C_2d, C_unidirec_2d ([NT][A][L]) */
void ps_get_collective(double* c, double* cu, double* c1, double* cu1, double* c2, double* cu2) {
    put2c(c, proc_data->phase_order_C_theta_triads);
    put2c(cu, proc_data->phase_order_C_theta_triads_unidirec);
    put2c(c1, proc_data->phase_order_C_theta_triads_1d);
    put2c(cu1, proc_data->phase_order_C_theta_triads_unidirec_1d);
    put3c(c2, proc_data->phase_order_C_theta_triads_2d);
    put3c(cu2, proc_data->phase_order_C_theta_triads_unidirec_2d);
}

/* FluxSpectra's sector sums: flux [A], diss [A], order [A] complex; the
   enstrophy dissipation field [nx][nyf] complex; the sector angles */
void ps_get_c_theta(double* flux, double* diss, double* order, double* diss_field, double* th3, double* th1) {
    const int A = sys_vars->num_k3_sectors, L = sys_vars->num_k1_sectors;
    const long n = sys_vars->N[0], nyf = n / 2 + 1;
    for (int a = 0; a < A; ++a) {
        flux[a] = proc_data->enst_flux_C_theta[a];
        diss[a] = proc_data->enst_diss_C_theta[a];
        order[2 * a] = creal(proc_data->phase_order_C_theta[a]);
        order[2 * a + 1] = cimag(proc_data->phase_order_C_theta[a]);
        th3[a] = proc_data->theta_k3[a];
    }
    for (int l = 0; l < L; ++l) th1[l] = proc_data->theta_k1[l];
    memcpy(diss_field, proc_data->enst_diss_field, sizeof(fftw_complex) * (size_t)(n * nyf));
}
