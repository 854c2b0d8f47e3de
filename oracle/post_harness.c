/*
 * oracle/post_harness.c -- the reference post-processing program's spectra,
 * flux spectra and full-field code (PostProcessing/src/full_field.c:29-557),
 * run on one snapshot through ctypes: the checker of bin/ns2d_post.  Test
 * infrastructure only.
 *
 * Sets up what PostProcessing()'s set-up would (post_proc.c:308-470):
 * wavenumbers, AllocateFullFieldMemory, the serial FFTW plans, and kmax_sqr /
 * kmax_C / kmax_C_sqr as AllocatePhaseSyncMemory computes them
 * (phase_sync.c:1139-1141) -- the stock build never sets those, so
 * FullFieldData and the set-C sums would read whatever the stack held.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "data_types.h"
#include "full_field.h"

runtime_data_struct* run_data;
system_vars_struct* sys_vars;
HDF_file_info_struct* file_info;
postprocess_data_struct* proc_data;
stats_data_struct* stats_data;

int post_init(int n, double nu, int hyper_flag, double hyper_pow, double alpha, int drag_flag, double drag_pow,
              double kmax_frac) {
    sys_vars = (system_vars_struct*)calloc(1, sizeof(system_vars_struct));
    run_data = (runtime_data_struct*)calloc(1, sizeof(runtime_data_struct));
    file_info = (HDF_file_info_struct*)calloc(1, sizeof(HDF_file_info_struct));
    proc_data = (postprocess_data_struct*)calloc(1, sizeof(postprocess_data_struct));
    stats_data = (stats_data_struct*)calloc(1, sizeof(stats_data_struct));
    sys_vars->N[0] = n;
    sys_vars->N[1] = n;
    sys_vars->num_snaps = 1;
    sys_vars->NU = nu;
    sys_vars->HYPER_VISC_FLAG = hyper_flag;
    sys_vars->HYPER_VISC_POW = hyper_pow;
    sys_vars->EKMN_ALPHA = alpha;
    sys_vars->EKMN_DRAG_FLAG = drag_flag;
    sys_vars->EKMN_DRAG_POW = drag_pow;
    sys_vars->kmax_frac = kmax_frac;
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
    proc_data->enst_flux_C = (double*)calloc(1, sizeof(double));
    proc_data->enst_diss_C = (double*)calloc(1, sizeof(double));
    proc_data->enrg_flux_C = (double*)calloc(1, sizeof(double));
    proc_data->enrg_diss_C = (double*)calloc(1, sizeof(double));
    proc_data->enst_diss_field = (fftw_complex*)calloc((size_t)(n * nyf), sizeof(fftw_complex));
    sys_vars->kmax_sqr = pow(sys_vars->kmax, 2.0);
    sys_vars->kmax_C = (int)ceil(sys_vars->kmax_frac * sys_vars->kmax);
    sys_vars->kmax_C_sqr = pow(sys_vars->kmax_C, 2.0);
    const int nb[2] = {n, n};
    sys_vars->fftw_2d_dft_r2c = fftw_plan_dft_r2c_2d(n, n, run_data->w, run_data->w_hat, FFTW_MEASURE);
    sys_vars->fftw_2d_dft_batch_c2r =
        fftw_plan_many_dft_c2r(2, nb, 2, run_data->u_hat, NULL, 2, 1, run_data->u, NULL, 2, 1, FFTW_MEASURE);
    return sys_vars->n_spec;
}

int post_kmax(void) { return sys_vars->kmax; }

/* One snapshot: spec[8][n_spec] = enrg, enst, d_enst_dt, enst_flux, enst_diss,
   d_enrg_dt, enrg_flux, enrg_diss (the order of ns2d_system_measurables);
   full[4][(2kmax+1)^2] = phases, amps, enrg, enst; c[4] = enst_flux_C,
   enst_diss_C, enrg_flux_C, enrg_diss_C. */
void post_snapshot(const double* w_hat, double* spec, double* full, double* c) {
    const long n = sys_vars->N[0], nyf = n / 2 + 1;
    memcpy(run_data->w_hat, w_hat, sizeof(fftw_complex) * (size_t)(n * nyf));
    proc_data->enst_flux_C[0] = proc_data->enst_diss_C[0] = 0.0;
    proc_data->enrg_flux_C[0] = proc_data->enrg_diss_C[0] = 0.0;
    EnstrophySpectrum();
    EnergySpectrum();
    FluxSpectra(0);
    FullFieldData();
    const int ns = sys_vars->n_spec;
    const double* src[8] = {proc_data->enrg_spec,      proc_data->enst_spec,      proc_data->d_enst_dt_spec,
                            proc_data->enst_flux_spec, proc_data->enst_diss_spec, proc_data->d_enrg_dt_spec,
                            proc_data->enrg_flux_spec, proc_data->enrg_diss_spec};
    for (int k = 0; k < 8; ++k) memcpy(spec + (size_t)k * ns, src[k], sizeof(double) * (size_t)ns);
    const size_t m = (size_t)(2 * sys_vars->kmax + 1) * (size_t)(2 * sys_vars->kmax + 1);
    memcpy(full, proc_data->phases, sizeof(double) * m);
    memcpy(full + m, proc_data->amps, sizeof(double) * m);
    memcpy(full + 2 * m, proc_data->enrg, sizeof(double) * m);
    memcpy(full + 3 * m, proc_data->enst, sizeof(double) * m);
    c[0] = proc_data->enst_flux_C[0];
    c[1] = proc_data->enst_diss_C[0];
    c[2] = proc_data->enrg_flux_C[0];
    c[3] = proc_data->enrg_diss_C[0];
}
