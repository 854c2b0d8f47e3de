/*
 * oracle/ns2d_oracle.c -- CPU FP64 restatement of the reference solver's
 * pseudospectral time step.  TEST INFRASTRUCTURE ONLY (the checker for the
 * CUDA product; never linked into it).
 *
 * Every routine cites the reference lines it restates (paths relative to the
 * reference project).  The floating-point operations are kept in the
 * reference's order so that, with the same FFT (oracle/fft.c), results agree
 * bit for bit with the reference's own sources built by oracle/Makefile.
 * Reference behaviours that look like bugs are reproduced when the matching
 * NS2D_QUIRK_* bit is set and corrected when it is clear.
 */
#include "ns2d_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fft.h"

typedef double _Complex cplx;

/* Butcher / AB4 coefficients: Solver/src/solver.c:29-47 (classical RK4, AB4). */
static const double kA21 = 0.5, kA32 = 0.5, kA43 = 1.0;
static const double kB1 = 1.0 / 6.0, kB2 = 1.0 / 3.0, kB3 = 1.0 / 3.0, kB4 = 1.0 / 6.0;
static const double kAB1 = 55.0 / 24.0, kAB2 = -59.0 / 24.0, kAB3 = 37.0 / 24.0, kAB4 = -3.0 / 8.0;
/* Dormand-Prince 5(4): Solver/src/solver.c:33-42. */
static const double kDP_A21 = 0.2;
static const double kDP_A31 = 3.0 / 40.0, kDP_A32 = 9.0 / 40.0;
static const double kDP_A41 = 44.0 / 45.0, kDP_A42 = -56.0 / 15.0, kDP_A43 = 32.0 / 9.0;
static const double kDP_A51 = 19372.0 / 6561.0, kDP_A52 = -25360.0 / 2187.0, kDP_A53 = 64448.0 / 6561.0,
                    kDP_A54 = -212.0 / 729.0;
static const double kDP_A61 = 9017.0 / 3168.0, kDP_A62 = -355.0 / 33.0, kDP_A63 = 46732.0 / 5247.0,
                    kDP_A64 = 49.0 / 176.0, kDP_A65 = -5103.0 / 18656.0;
static const double kDP_B1 = 35.0 / 384.0, kDP_B3 = 500.0 / 1113.0, kDP_B4 = 125.0 / 192.0,
                    kDP_B5 = -2187.0 / 6784.0, kDP_B6 = 11.0 / 84.0;
static const double kDP_E1 = 5179.0 / 57600.0, kDP_E3 = 7571.0 / 16695.0, kDP_E4 = 393.0 / 640.0,
                    kDP_E5 = -92097.0 / 339200.0, kDP_E6 = 187.0 / 2100.0, kDP_E7 = 1.0 / 40.0;

struct ns2d_oracle {
    ns2d_params p;
    int nx, ny, nyf;
    size_t ns;        /* nx * nyf                                      */
    int* kx;          /* run_data->k[0]                                */
    int* ky;          /* run_data->k[1]                                */
    cplx* w_hat;      /* state                                         */
    cplx* rk[7];
    cplx* rk_tmp;
    cplx* ab_hist[3];
    cplx* ab_tmp;
    cplx* u_hat2;     /* run_data->u_hat, [nx][nyf][2], persists       */
    cplx* pair;       /* RHS scratch [nx][nyf][2]                      */
    double* real2a;   /* [nx][ny+2][2]                                 */
    double* real2b;
    double* real1;    /* [nx][ny+2]                                    */
    int hyper_flag;   /* live sys_vars->HYPER_VISC_FLAG                */
    int n_forced;
    size_t forcing_indx;
    cplx forcing_val;
    double dx, dy;
    double w_max_init;
    double min_dt, max_dt;
    int n_spect;
    cplx* w_hat_last; /* Int_data->w_hat_last (RK5DPStep as written)   */
    double dp_err;    /* Int_data->DP_err                              */
};

static int quirk(const ns2d_oracle* o, int bit) { return (o->p.quirks & bit) != 0; }

/* InitializeSpaceVariables: Solver/src/solver.c:2022-2068. */
static void init_space(ns2d_oracle* o) {
    for (int i = 0; i < o->nx; ++i) o->kx[i] = (i <= o->nx / 2) ? i : i - o->nx;
    for (int j = 0; j < o->nyf; ++j) o->ky[j] = j;
    o->dx = 2.0 * M_PI / (double)o->nx;
    o->dy = 2.0 * M_PI / (double)o->ny;
}

ns2d_oracle* oracle_create(const ns2d_params* p, int threads) {
    ns2d_oracle* o = (ns2d_oracle*)calloc(1, sizeof(*o));
    o->p = *p;
    o->nx = p->nx;
    o->ny = p->ny;
    o->nyf = p->ny / 2 + 1;
    o->ns = (size_t)o->nx * o->nyf;
    offt_set_threads(threads);
    o->kx = (int*)calloc((size_t)o->nx, sizeof(int));
    o->ky = (int*)calloc((size_t)o->nyf, sizeof(int));
    o->w_hat = (cplx*)calloc(o->ns, sizeof(cplx));
    for (int s = 0; s < 7; ++s) o->rk[s] = (cplx*)calloc(o->ns, sizeof(cplx));
    o->rk_tmp = (cplx*)calloc(o->ns, sizeof(cplx));
    for (int s = 0; s < 3; ++s) o->ab_hist[s] = (cplx*)calloc(o->ns, sizeof(cplx));
    o->ab_tmp = (cplx*)calloc(o->ns, sizeof(cplx));
    o->w_hat_last = (cplx*)calloc(o->ns, sizeof(cplx));
    o->u_hat2 = (cplx*)calloc(2 * o->ns, sizeof(cplx));
    o->pair = (cplx*)calloc(2 * o->ns, sizeof(cplx));
    size_t nr = (size_t)o->nx * (o->ny + 2);
    o->real2a = (double*)calloc(2 * nr, sizeof(double));
    o->real2b = (double*)calloc(2 * nr, sizeof(double));
    o->real1 = (double*)calloc(nr, sizeof(double));
    o->hyper_flag = p->hyper_visc_flag;
    init_space(o);
    /* InitializeForcing KOLM branch: Solver/src/force.c:45-100. */
    if (p->forcing == NS2D_FORCING_KOLM) {
        o->n_forced = 1;
        o->forcing_indx = (size_t)p->force_k;
    }
    o->min_dt = 10.0;
    o->max_dt = 1e-10;
    /* n_spect: Solver/src/sys_msr.c:394. */
    o->n_spect = (int)round(sqrt((double)(o->nx / 2.0) * (o->nx / 2.0) + (double)(o->ny / 2.0) * (o->ny / 2.0)) + 1);
    return o;
}

void oracle_destroy(ns2d_oracle* o) {
    if (!o) return;
    free(o->kx); free(o->ky); free(o->w_hat);
    for (int s = 0; s < 7; ++s) free(o->rk[s]);
    free(o->rk_tmp);
    for (int s = 0; s < 3; ++s) free(o->ab_hist[s]);
    free(o->ab_tmp); free(o->w_hat_last); free(o->u_hat2); free(o->pair);
    free(o->real2a); free(o->real2b); free(o->real1);
    free(o);
}

int oracle_n_spect(const ns2d_oracle* o) { return o->n_spect; }
int oracle_hyper_visc_flag(const ns2d_oracle* o) { return o->hyper_flag; }
void oracle_set_w_max_init(ns2d_oracle* o, double w) { o->w_max_init = w; }
void oracle_set_w_hat(ns2d_oracle* o, const double* w) { memcpy(o->w_hat, w, o->ns * sizeof(cplx)); }
void oracle_get_w_hat(const ns2d_oracle* o, double* w) { memcpy(w, o->w_hat, o->ns * sizeof(cplx)); }

/* ComputeForcing: Solver/src/force.c:516-581 (KOLM, ZERO).  ZERO kills every
   mode with |kx| <= force_k or |ky| <= force_k in the state (the modes chosen
   at force.c:436-501, zeroed at :527-533); its forcing values stay 0. */
void oracle_compute_forcing(ns2d_oracle* o, double dt) {
    (void)dt;
    if (o->p.forcing == NS2D_FORCING_KOLM && o->n_forced)
        o->forcing_val = -0.5 * o->p.force_scale * (o->p.force_k + 0.0 * I);
    if (o->p.forcing == NS2D_FORCING_ZERO) {
        for (int i = 0; i < o->nx; ++i)
            for (int j = 0; j < o->nyf; ++j)
                if (abs(o->kx[i]) <= o->p.force_k || abs(o->ky[j]) <= o->p.force_k)
                    o->w_hat[(size_t)i * o->nyf + j] = 0.0;
    }
}

/* Bracket of the linear operator D/dt (Solver/src/solver.c:839-856, also
   :668-683 and sys_msr.c:166-181).  `latch` = the reference's `=` typo. */
static double lin_bracket(ns2d_oracle* o, double k_sqr, int latch) {
    const ns2d_params* p = &o->p;
    if (o->hyper_flag == 1 && p->ekmn_drag_flag == 1)
        return p->nu * pow(k_sqr, p->hyper_visc_pow) + p->ekmn_alpha * pow(k_sqr, p->ekmn_drag_pow);
    if (o->hyper_flag != 1 && p->ekmn_drag_flag == 1)
        return p->nu * k_sqr + p->ekmn_alpha * pow(k_sqr, p->ekmn_drag_pow);
    if (latch) o->hyper_flag = 1;
    if (o->hyper_flag == 1 && p->ekmn_drag_flag != 1) return p->nu * pow(k_sqr, p->hyper_visc_pow);
    return p->nu * k_sqr;
}

/* ApplyDealiasing: Solver/src/solver.c:1039-1099. */
static void dealias(const ns2d_oracle* o, cplx* a, int dim) {
    const double kmax_sqr = pow((int)(o->nx / 3.0), 2.0);
    const int kolm = (o->p.forcing == NS2D_FORCING_KOLM);
    for (int i = 0; i < o->nx; ++i) {
        for (int j = 0; j < o->nyf; ++j) {
            size_t idx = (size_t)dim * ((size_t)i * o->nyf + j);
            int kx = o->kx[i], ky = o->ky[j];
            if (o->p.dealias == NS2D_DEALIAS_23) {
                double k_sqr = (double)kx * kx + ky * ky;
                if (k_sqr >= kmax_sqr || (kolm && kx == 0))
                    for (int l = 0; l < dim; ++l) a[idx + l] = 0.0;
            } else {
                double fx, fy;
                if (quirk(o, NS2D_QUIRK_HOU_LI_INT)) {
                    fx = (double)(kx / (o->nx / 2));
                    fy = (double)(ky / (o->ny / 2));
                } else {
                    fx = (double)kx / (o->nx / 2);
                    fy = (double)ky / (o->ny / 2);
                }
                double f = exp(-36.0 * pow(sqrt(pow(fx, 2.0) + pow(fy, 2.0)), 36.0));
                for (int l = 0; l < dim; ++l) a[idx + l] *= f;
            }
        }
    }
}

void oracle_apply_dealiasing(const ns2d_oracle* o, double* arr, int dim) { dealias(o, (cplx*)arr, dim); }

/* ForceConjugacy: Solver/src/solver.c:2074-2107.  Column ky = 0 of `in` is
   gathered first, then the state's kx < 0 rows are overwritten (the reference
   always writes run_data->w_hat, whatever array it is given).  Without the
   quirk the fix applies to `in` itself. */
static void force_conjugacy(ns2d_oracle* o, cplx* in) {
    cplx* col = (cplx*)malloc(sizeof(cplx) * (size_t)o->nx);
    for (int i = 0; i < o->nx; ++i) col[i] = in[(size_t)i * o->nyf];
    cplx* dst = quirk(o, NS2D_QUIRK_CONJ_STATE) ? o->w_hat : in;
    for (int i = 0; i < o->nx; ++i)
        if (o->kx[i] < 0) dst[(size_t)i * o->nyf] = conj(col[abs(o->kx[i])]);
    free(col);
}

void oracle_force_conjugacy(ns2d_oracle* o, const double* arr) {
    if (!arr) { force_conjugacy(o, o->w_hat); return; }
    cplx* tmp = (cplx*)malloc(o->ns * sizeof(cplx));
    memcpy(tmp, arr, o->ns * sizeof(cplx));
    force_conjugacy(o, tmp);
    free(tmp);
}

/* NonlinearRHSBatch: Solver/src/solver.c:884-1032. */
static void nonlinear_rhs(ns2d_oracle* o, cplx* w_hat, cplx* out) {
    const int nx = o->nx, ny = o->ny, nyf = o->nyf;
    const double norm_fac = 1.0 / (nx * ny);
    cplx* pr = o->pair;
    /* velocities u_hat = i ky/|k|^2 w, v_hat = -i kx/|k|^2 w (:904-925) */
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nyf; ++j) {
            size_t idx = (size_t)i * nyf + j;
            if (o->kx[i] != 0 || o->ky[j] != 0) {
                double k_sqr = 1.0 / (double)(o->kx[i] * o->kx[i] + o->ky[j] * o->ky[j]);
                pr[2 * idx + 0] = I * ((double)o->ky[j]) * k_sqr * w_hat[idx];
                pr[2 * idx + 1] = -1.0 * I * ((double)o->kx[i]) * k_sqr * w_hat[idx];
            } else {
                pr[2 * idx + 0] = 0.0;
                pr[2 * idx + 1] = 0.0;
            }
        }
    offt_c2r_2d(nx, ny, 2, pr, o->real2a); /* :932 */
    /* vorticity gradient i kx w, i ky w (:939-957) */
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nyf; ++j) {
            size_t idx = (size_t)i * nyf + j;
            if (o->kx[i] != 0 || o->ky[j] != 0) {
                pr[2 * idx + 0] = I * ((double)o->kx[i]) * w_hat[idx];
                pr[2 * idx + 1] = I * ((double)o->ky[j]) * w_hat[idx];
            } else {
                pr[2 * idx + 0] = 0.0;
                pr[2 * idx + 1] = 0.0;
            }
        }
    offt_c2r_2d(nx, ny, 2, pr, o->real2b); /* :964 */
    /* product u.grad(w) with the reference's + sign (:972-987) */
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            size_t idx = (size_t)i * (ny + 2) + j;
            double v1 = o->real2a[2 * idx + 0], v2 = o->real2a[2 * idx + 1];
            o->real1[idx] = 1.0 * (v1 * o->real2b[2 * idx + 0] + v2 * o->real2b[2 * idx + 1]);
        }
    offt_r2c_2d(nx, ny, 1, o->real1, out); /* :994 */
    /* (1/(NxNy))^2 normalisation, zero mean (:998-1013) */
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nyf; ++j) {
            size_t idx = (size_t)i * nyf + j;
            if (o->kx[i] != 0 || o->ky[j] != 0) out[idx] *= pow(norm_fac, 2.0);
            else out[idx] = 0.0;
        }
    dealias(o, out, 1);                                   /* :1019 */
    if (o->n_forced) out[o->forcing_indx] += o->forcing_val; /* :1022-1027 */
    force_conjugacy(o, w_hat);                            /* :1031 */
}

void oracle_nonlinear_rhs(ns2d_oracle* o, const double* in, double* out) {
    if (!in) {
        nonlinear_rhs(o, o->w_hat, o->rk[0]);
    } else {
        memcpy(o->rk_tmp, in, o->ns * sizeof(cplx));
        nonlinear_rhs(o, o->rk_tmp, o->rk[0]);
    }
    memcpy(out, o->rk[0], o->ns * sizeof(cplx));
}

/* Stage combine of RK4Step (Solver/src/solver.c:657-809); with -D__RK4 the
   stage RHS also gets +D*X (quirk NS2D_QUIRK_RK4_LINEAR; corrected: -D*X/dt
   so that the stage derivative carries the linear term). */
static void rk4_linear_add(ns2d_oracle* o, cplx* rk, const cplx* x, double dt) {
    const int latch = quirk(o, NS2D_QUIRK_HYPER_LATCH);
    for (int i = 0; i < o->nx; ++i)
        for (int j = 0; j < o->nyf; ++j) {
            size_t idx = (size_t)i * o->nyf + j;
            double k_sqr = (double)(o->kx[i] * o->kx[i] + o->ky[j] * o->ky[j]);
            if (quirk(o, NS2D_QUIRK_RK4_LINEAR)) {
                double D = dt * lin_bracket(o, k_sqr, latch);
                rk[idx] += D * x[idx];
            } else {
                if (k_sqr == 0.0) continue;
                double D = lin_bracket(o, k_sqr, latch);
                rk[idx] -= D * x[idx];
            }
        }
}

static void stage_combine(ns2d_oracle* o, const cplx* rk, double a_dt_coef, double dt) {
    for (size_t idx = 0; idx < o->ns; ++idx) o->rk_tmp[idx] = o->w_hat[idx] + dt * a_dt_coef * rk[idx];
}

/* RK4Step: Solver/src/solver.c:625-873. */
void oracle_rk4_step(ns2d_oracle* o, double dt) {
    const int explicit_rk4 = (o->p.integrator == NS2D_RK4);
    const int euler = (o->p.system == NS2D_EULER);
    oracle_compute_forcing(o, dt);
    nonlinear_rhs(o, o->w_hat, o->rk[0]);
    if (explicit_rk4 && !euler) rk4_linear_add(o, o->rk[0], o->w_hat, dt);
    stage_combine(o, o->rk[0], kA21, dt);
    nonlinear_rhs(o, o->rk_tmp, o->rk[1]);
    if (explicit_rk4 && !euler) rk4_linear_add(o, o->rk[1], o->rk_tmp, dt);
    stage_combine(o, o->rk[1], kA32, dt);
    nonlinear_rhs(o, o->rk_tmp, o->rk[2]);
    if (explicit_rk4 && !euler) rk4_linear_add(o, o->rk[2], o->rk_tmp, dt);
    stage_combine(o, o->rk[2], kA43, dt);
    nonlinear_rhs(o, o->rk_tmp, o->rk[3]);
    if (explicit_rk4 && !euler) rk4_linear_add(o, o->rk[3], o->rk_tmp, dt);
    /* update (:816-863) */
    const int latch = quirk(o, NS2D_QUIRK_HYPER_LATCH);
    for (int i = 0; i < o->nx; ++i)
        for (int j = 0; j < o->nyf; ++j) {
            size_t idx = (size_t)i * o->nyf + j;
            if (o->kx[i] != 0 || o->ky[j] != 0) {
                const double a_before = cabs(o->w_hat[idx]);
                if (explicit_rk4 || euler) {
                    o->w_hat[idx] = o->w_hat[idx] + (dt / 6.0) * (o->rk[0][idx] + 2.0 * o->rk[1][idx] +
                                                                 2.0 * o->rk[2][idx] + o->rk[3][idx]);
                } else {
                    double k_sqr = (double)(o->kx[i] * o->kx[i] + o->ky[j] * o->ky[j]);
                    double D = dt * lin_bracket(o, k_sqr, latch);
                    o->w_hat[idx] = o->w_hat[idx] * ((2.0 - D) / (2.0 + D)) +
                                    (2.0 * dt / (2.0 + D)) * (kB1 * o->rk[0][idx] + kB2 * o->rk[1][idx] +
                                                              kB3 * o->rk[2][idx] + kB4 * o->rk[3][idx]);
                }
                /* phase-only amplitude reset (:822-824, 855-857): w *= |w before| / |w after|;
                   the reference's 0/0 (NaN) where the update gives exactly 0 is kept at 0 */
                if (o->p.model == NS2D_MODEL_PHASE_ONLY && cabs(o->w_hat[idx]) > 0.0)
                    o->w_hat[idx] *= (a_before / cabs(o->w_hat[idx]));
            } else {
                o->w_hat[idx] = 0.0;
            }
        }
}

/* AB4Step: Solver/src/solver.c:261-350 (three RK4 start-up steps storing RK1,
   then AB4 with the CN linear factor and a 3-deep history). */
int oracle_ab4_step(ns2d_oracle* o, double dt, int iters) {
    if (iters <= 3) {
        oracle_rk4_step(o, dt);
        memcpy(o->ab_hist[iters - 1], o->rk[0], o->ns * sizeof(cplx));
        return 0;
    }
    oracle_compute_forcing(o, dt);
    nonlinear_rhs(o, o->w_hat, o->ab_tmp);
    for (int i = 0; i < o->nx; ++i)
        for (int j = 0; j < o->nyf; ++j) {
            size_t idx = (size_t)i * o->nyf + j;
            if (o->kx[i] != 0 || o->ky[j] != 0) {
                if (o->p.system == NS2D_EULER) {
                    o->w_hat[idx] = o->w_hat[idx] + dt * (kAB1 * o->ab_tmp[idx]) + dt * (kAB2 * o->ab_hist[2][idx]) +
                                    dt * (kAB3 * o->ab_hist[1][idx]) + dt * (kAB4 * o->ab_hist[0][idx]);
                } else {
                    double k_sqr = (double)(o->kx[i] * o->kx[i] + o->ky[j] * o->ky[j]);
                    double D = dt * lin_bracket(o, k_sqr, 0);
                    o->w_hat[idx] = o->w_hat[idx] * ((2.0 - D) / (2.0 + D)) +
                                    (2.0 * dt / (2.0 + D)) * ((kAB1 * o->ab_tmp[idx]) + (kAB2 * o->ab_hist[2][idx]) +
                                                              (kAB3 * o->ab_hist[1][idx]) + (kAB4 * o->ab_hist[0][idx]));
                }
            } else {
                o->w_hat[idx] = 0.0;
            }
        }
    cplx* oldest = o->ab_hist[0];
    o->ab_hist[0] = o->ab_hist[1];
    o->ab_hist[1] = o->ab_hist[2];
    o->ab_hist[2] = oldest;
    memcpy(o->ab_hist[2], o->ab_tmp, o->ns * sizeof(cplx));
    return 0;
}

/* Dormand-Prince 5(4) step, a corrected restatement of RK5DPStep
   (Solver/src/solver.c:360-570), which does not compile as shipped (it names
   run_data->w_hat_last and reads an uninitialised err_sum).  Stages use the
   Butcher table at :33-42 on the nonlinear term, with the same integrating
   factor treatment as RK4CN folded out: this restatement applies the linear
   term explicitly inside the stages (y' = N(y) - D y).  Returns the RMS error
   norm with DP_ABS_TOL = DP_REL_TOL = 1e-7 (data_types.h:137-138).  The state
   is advanced; the caller decides acceptance. */
int oracle_dp5_step(ns2d_oracle* o, double dt, double* err) {
    const size_t ns = o->ns;
    cplx* k[7];
    for (int s = 0; s < 7; ++s) k[s] = o->rk[s];
    cplx* y0 = (cplx*)malloc(ns * sizeof(cplx));
    memcpy(y0, o->w_hat, ns * sizeof(cplx));
    static const double a[6][6] = {
        {0.2, 0, 0, 0, 0, 0},
        {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0},
        {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
        {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
        {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
        {35.0 / 384.0, 0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
    (void)kDP_A21; (void)kDP_A31; (void)kDP_A32; (void)kDP_A41; (void)kDP_A42; (void)kDP_A43;
    (void)kDP_A51; (void)kDP_A52; (void)kDP_A53; (void)kDP_A54; (void)kDP_A61; (void)kDP_A62;
    (void)kDP_A63; (void)kDP_A64; (void)kDP_A65;
    oracle_compute_forcing(o, dt);
    for (int s = 0; s < 7; ++s) {
        cplx* x = (s == 0) ? y0 : o->rk_tmp;
        if (s > 0) {
            for (size_t idx = 0; idx < ns; ++idx) {
                cplx acc = 0.0;
                for (int r = 0; r < s; ++r) acc += a[s - 1][r] * k[r][idx];
                o->rk_tmp[idx] = y0[idx] + dt * acc;
            }
        }
        memcpy(o->w_hat, y0, ns * sizeof(cplx));
        nonlinear_rhs(o, x, k[s]);
        if (o->p.system != NS2D_EULER) {
            for (int i = 0; i < o->nx; ++i)
                for (int j = 0; j < o->nyf; ++j) {
                    size_t idx = (size_t)i * o->nyf + j;
                    double k_sqr = (double)(o->kx[i] * o->kx[i] + o->ky[j] * o->ky[j]);
                    if (k_sqr == 0.0) continue;
                    k[s][idx] -= lin_bracket(o, k_sqr, 0) * x[idx];
                }
        }
    }
    double sum = 0.0;
    for (int i = 0; i < o->nx; ++i)
        for (int j = 0; j < o->nyf; ++j) {
            size_t idx = (size_t)i * o->nyf + j;
            if (o->kx[i] == 0 && o->ky[j] == 0) { o->w_hat[idx] = 0.0; continue; }
            cplx y5 = y0[idx] + dt * (kDP_B1 * k[0][idx] + kDP_B3 * k[2][idx] + kDP_B4 * k[3][idx] +
                                      kDP_B5 * k[4][idx] + kDP_B6 * k[5][idx]);
            cplx y4 = y0[idx] + dt * (kDP_E1 * k[0][idx] + kDP_E3 * k[2][idx] + kDP_E4 * k[3][idx] +
                                      kDP_E5 * k[4][idx] + kDP_E6 * k[5][idx] + kDP_E7 * k[6][idx]);
            double sc = 1e-7 + 1e-7 * fmax(cabs(y0[idx]), cabs(y5));
            double e = cabs(y5 - y4) / sc;
            sum += e * e;
            o->w_hat[idx] = y5;
        }
    *err = sqrt(sum / (double)(o->nx * o->nyf));
    free(y0);
    return 0;
}

/* RK5DPStep as the reference writes it (Solver/src/solver.c:360-570), with
   the three defects that stop it compiling fixed the way oracle/Makefile's
   dp5 build fixes them (err_sum starts at 0, one surplus parenthesis, the
   w_hat_last member read from Int_data).  Everything else is kept:
   * the table of :35-43, whose a32 is 0.5 (the published Dormand-Prince value
     is 9/40), on the nonlinear term alone; each stage input is the live state
     plus dt sum a k, and every NonlinearRHSBatch call rewrites the state's
     ky = 0, kx < 0 modes from its input (the ForceConjugacy side effect);
   * the update of :494-514: Crank-Nicolson factors on the fifth-order sum
     (explicit for the Euler system);
   * the error of :515-552, only when iters > 1: dp_ho_step is a double, so it
     keeps the real part of w_new + dt sum bs k, pow() keeps the real part of
     its complex argument, the scale uses the state of the previous error step
     (w_hat_last, 0 until the first one), and DP_err = sqrt(sum / (Nx Nyf)).
   Returns DP_err, which keeps its previous value when iters == 1. */
static const double kR5_A32 = 0.5;
double oracle_rk5dp_step(ns2d_oracle* o, double dt, int iters) {
    cplx** k = o->rk;
    cplx* w = o->w_hat;
    cplx* x = o->rk_tmp;
    const size_t ns = o->ns;
    oracle_compute_forcing(o, dt);
    nonlinear_rhs(o, w, k[0]);
    for (size_t idx = 0; idx < ns; ++idx) x[idx] = w[idx] + dt * kDP_A21 * k[0][idx];
    nonlinear_rhs(o, x, k[1]);
    for (size_t idx = 0; idx < ns; ++idx)
        x[idx] = w[idx] + dt * kDP_A31 * k[0][idx] + dt * kR5_A32 * k[1][idx];
    nonlinear_rhs(o, x, k[2]);
    for (size_t idx = 0; idx < ns; ++idx)
        x[idx] = w[idx] + dt * kDP_A41 * k[0][idx] + dt * kDP_A42 * k[1][idx] + dt * kDP_A43 * k[2][idx];
    nonlinear_rhs(o, x, k[3]);
    for (size_t idx = 0; idx < ns; ++idx)
        x[idx] = w[idx] + dt * kDP_A51 * k[0][idx] + dt * kDP_A52 * k[1][idx] + dt * kDP_A53 * k[2][idx] +
                 dt * kDP_A54 * k[3][idx];
    nonlinear_rhs(o, x, k[4]);
    for (size_t idx = 0; idx < ns; ++idx)
        x[idx] = w[idx] + dt * kDP_A61 * k[0][idx] + dt * kDP_A62 * k[1][idx] + dt * kDP_A63 * k[2][idx] +
                 dt * kDP_A64 * k[3][idx] + dt * kDP_A65 * k[4][idx];
    nonlinear_rhs(o, x, k[5]);
    /* stage 7 input: the a7 row equals the fifth-order weights b */
    for (size_t idx = 0; idx < ns; ++idx)
        x[idx] = w[idx] + dt * kDP_B1 * k[0][idx] + dt * kDP_B3 * k[2][idx] + dt * kDP_B4 * k[3][idx] +
                 dt * kDP_B5 * k[4][idx] + dt * kDP_B6 * k[5][idx];
    nonlinear_rhs(o, x, k[6]);
    double err_sum = 0.0;
    for (int i = 0; i < o->nx; ++i)
        for (int j = 0; j < o->nyf; ++j) {
            size_t idx = (size_t)i * o->nyf + j;
            if (o->kx[i] != 0 || o->ky[j] != 0) {
                if (o->p.system == NS2D_EULER) {
                    w[idx] = w[idx] + (dt * (kDP_B1 * k[0][idx]) + dt * (kDP_B3 * k[2][idx]) +
                                       dt * (kDP_B4 * k[3][idx]) + dt * (kDP_B5 * k[4][idx]) +
                                       dt * (kDP_B6 * k[5][idx]));
                } else {
                    double k_sqr = (double)(o->kx[i] * o->kx[i] + o->ky[j] * o->ky[j]);
                    double D = dt * lin_bracket(o, k_sqr, 0);
                    w[idx] = w[idx] * ((2.0 - D) / (2.0 + D)) +
                             (2.0 * dt / (2.0 + D)) * (kDP_B1 * k[0][idx] + kDP_B3 * k[2][idx] + kDP_B4 * k[3][idx] +
                                                       kDP_B5 * k[4][idx] + kDP_B6 * k[5][idx]);
                }
                if (iters > 1) {
                    double ho = creal(w[idx] + (dt * (kDP_E1 * k[0][idx]) + dt * (kDP_E3 * k[2][idx]) +
                                                dt * (kDP_E4 * k[3][idx]) + dt * (kDP_E5 * k[4][idx]) +
                                                dt * (kDP_E6 * k[5][idx])) +
                                      dt * (kDP_E7 * k[6][idx]));
                    double a = cabs(o->w_hat_last[idx]), b = cabs(w[idx]);
                    double denom = 1e-7 + (a > b ? a : b) * 1e-7;
                    err_sum += pow(creal((w[idx] - ho) / denom), 2.0);
                }
            } else {
                w[idx] = 0.0;
            }
        }
    if (iters > 1) {
        o->dp_err = sqrt(1.0 / (double)((long)o->nx * (long)o->nyf) * err_sum);
        for (size_t idx = 0; idx < ns; ++idx) o->w_hat_last[idx] = w[idx];
        o->w_hat_last[0] = 0.0;
    }
    return o->dp_err;
}

/* c2r of the state, normalised by 1/(NxNy) (Solver/src/solver.c:2218-2230). */
static void vort_real(ns2d_oracle* o) {
    offt_c2r_2d(o->nx, o->ny, 1, o->w_hat, o->real1);
    for (int i = 0; i < o->nx; ++i)
        for (int j = 0; j < o->ny; ++j) o->real1[(size_t)i * (o->ny + 2) + j] *= 1.0 / (double)(o->nx * o->ny);
}

void oracle_get_w_real(ns2d_oracle* o, double* w) {
    vort_real(o);
    for (int i = 0; i < o->nx; ++i)
        memcpy(w + (size_t)i * o->ny, o->real1 + (size_t)i * (o->ny + 2), sizeof(double) * (size_t)o->ny);
}

/* Velocity from the state into the persistent u_hat buffer.  `scrambled`
   restates the CFL path's row index tmp = (i*Ny)/2 + 1 (Solver/src/solver.c:
   2394); the VEL path of GetMaxData uses i*Nyf (:2184). */
static void velocity_hat(ns2d_oracle* o, int scrambled) {
    const int nyf = o->nyf;
    for (int i = 0; i < o->nx; ++i) {
        long tmp = scrambled ? (long)i * o->ny / 2 + 1 : (long)i * nyf;
        for (int j = 0; j < nyf; ++j) {
            long idx = tmp + j;
            if (o->kx[i] != 0 || o->ky[j] != 0) {
                cplx I_over_k_sqr = I / (double)(o->kx[i] * o->kx[i] + o->ky[j] * o->ky[j]);
                o->u_hat2[2 * idx + 0] = ((double)o->ky[j]) * I_over_k_sqr * o->w_hat[idx];
                o->u_hat2[2 * idx + 1] = -1.0 * ((double)o->kx[i]) * I_over_k_sqr * o->w_hat[idx];
            } else {
                o->u_hat2[2 * idx + 0] = 0.0;
                o->u_hat2[2 * idx + 1] = 0.0;
            }
        }
    }
    offt_c2r_2d(o->nx, o->ny, 2, o->u_hat2, o->real2a);
    for (int i = 0; i < o->nx; ++i)
        for (int j = 0; j < o->ny; ++j) {
            size_t idx = (size_t)i * (o->ny + 2) + j;
            o->real2a[2 * idx + 0] *= 1.0 / (double)(o->nx * o->ny);
            o->real2a[2 * idx + 1] *= 1.0 / (double)(o->nx * o->ny);
        }
}

/* GetMaxData: Solver/src/solver.c:2171-2295. */
double oracle_get_max_data(ns2d_oracle* o, int kind) {
    double wmax = 0.0;
    if (kind == NS2D_MAX_VORT) {
        vort_real(o);
        for (int i = 0; i < o->nx; ++i)
            for (int j = 0; j < o->ny; ++j) {
                double v = fabs(o->real1[(size_t)i * (o->ny + 2) + j]);
                if (v > wmax) wmax = v;
            }
    } else if (kind == NS2D_MAX_VEL) {
        velocity_hat(o, 0);
        for (int i = 0; i < o->nx; ++i)
            for (int j = 0; j < o->ny; ++j)
                for (int l = 0; l < 2; ++l) {
                    double v = fabs(o->real2a[2 * ((size_t)i * (o->ny + 2) + j) + l]);
                    if (v > wmax) wmax = v;
                }
    } else {
        for (size_t idx = 0; idx < o->ns; ++idx)
            if (cabs(o->w_hat[idx]) > wmax) wmax = cabs(o->w_hat[idx]);
    }
    return wmax;
}

/* GetTimestep: Solver/src/solver.c:2376-2490. */
double oracle_get_timestep(ns2d_oracle* o, double dt) {
    if (o->p.cfl_cond_flag == 1) {
        velocity_hat(o, quirk(o, NS2D_QUIRK_CFL_INDEX));
        double scales_convect = 0.0;
        for (int i = 0; i < o->nx; ++i)
            for (int j = 0; j < o->ny; ++j) {
                size_t idx = (size_t)i * (o->ny + 2) + j;
                scales_convect = fmax(M_PI * (fabs(o->real2a[2 * idx + 0]) / o->dx + fabs(o->real2a[2 * idx + 1]) / o->dy),
                                      scales_convect);
            }
        double scales_diff = pow(M_PI, 2.0) * (o->p.nu / pow(o->dx, 2.0) + o->p.nu / pow(o->dy, 2.0));
        dt = o->p.cfl_const / (scales_convect + scales_diff);
    } else {
        double w_max = oracle_get_max_data(o, NS2D_MAX_VORT);
        double dt_new = o->p.dt * (o->w_max_init / w_max);
        dt = (dt_new > 2.0 * dt) ? 2.0 * dt : dt_new;
    }
    o->min_dt = fmin(dt, o->min_dt);
    o->max_dt = fmax(dt, o->max_dt);
    return dt;
}

/* ComputeSystemMeasurables: Solver/src/sys_msr.c:32-373 with the stock dataset
   flags (__SYS_MEASURES, __ENST/ENRG_FLUX, __ENST/ENRG_SPECT, flux spectra). */
void oracle_system_measurables(ns2d_oracle* o, double* s13, double* spectra) {
    const int nx = o->nx, ny = o->ny, nyf = o->nyf, ns = o->n_spect;
    const double norm_fac = 0.5 / pow(nx * ny, 2.0);
    const double const_fac = 4.0 * pow(M_PI, 2.0);
    const double lwr = pow(0, 2.0), upr = pow(64, 2.0); /* data_types.h:175-176 */
    double tot_energy = 0, tot_enstr = 0, tot_palin = 0, tot_forc = 0, tot_div = 0, enrg_diss = 0, enst_diss = 0;
    double d_enrg = 0, enrg_flux = 0, enrg_dsb = 0, d_enst = 0, enst_flux = 0, enst_dsb = 0;
    double* sp = spectra;
    double* e_sp = sp;
    double* z_sp = sp + ns;
    double* dz_sp = sp + 2 * ns;
    double* zf_sp = sp + 3 * ns;
    double* zd_sp = sp + 4 * ns;
    double* de_sp = sp + 5 * ns;
    double* ef_sp = sp + 6 * ns;
    double* ed_sp = sp + 7 * ns;
    memset(sp, 0, sizeof(double) * 8 * (size_t)ns);
    cplx* rk1 = o->rk[0];
    if (o->p.flux_diagnostics) {
        nonlinear_rhs(o, o->w_hat, rk1); /* :127, with its conjugacy side effect */
        if (o->n_forced) rk1[o->forcing_indx] -= o->forcing_val;
    } else {
        memset(rk1, 0, o->ns * sizeof(cplx));
    }
    if (o->n_forced) tot_forc += cabs(o->forcing_val * o->w_hat[o->forcing_indx]);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nyf; ++j) {
            size_t idx = (size_t)i * nyf + j;
            int kx = o->kx[i], ky = o->ky[j];
            int spec_indx = (int)round(sqrt((double)(kx * kx + ky * ky)));
            double k_sqr = (double)(kx * kx + ky * ky);
            double pre_fac = lin_bracket(o, k_sqr, 0);
            if (kx == 0 && ky == 0) continue;
            cplx w = o->w_hat[idx];
            cplx u_z = I * ((double)ky) * w / k_sqr;
            cplx v_z = -I * ((double)kx) * w / k_sqr;
            cplx div_u_z = I * ((double)kx * u_z + (double)ky * v_z);
            double w2 = cabs(w * conj(w));
            double edge = (j == 0) || (j == nyf - 1);
            double tmp_deriv = creal(w * conj(rk1[idx]) + conj(w) * rk1[idx]);
            double tmp_diss = pre_fac * w2;
            if (edge) {
                tot_energy += w2 * (1.0 / k_sqr);
                tot_enstr += w2;
                tot_div += cabs(div_u_z * conj(div_u_z));
                tot_palin += k_sqr * w2;
                enrg_diss += pre_fac * cabs(u_z * conj(u_z) + v_z * conj(v_z));
                enst_diss += pre_fac * w2;
                if (k_sqr >= lwr && k_sqr < upr) {
                    d_enrg += (tmp_deriv + tmp_diss) * (1.0 / k_sqr);
                    enrg_dsb += tmp_diss * (1.0 / k_sqr);
                    enrg_flux += tmp_deriv * (1.0 / k_sqr);
                    d_enst += tmp_deriv + tmp_diss;
                    enst_dsb += tmp_diss;
                    enst_flux += tmp_deriv;
                }
            } else {
                tot_energy += 2.0 * w2 * (1.0 / k_sqr);
                tot_enstr += 2.0 * w2;
                tot_div += 2.0 * cabs(div_u_z * conj(div_u_z));
                tot_palin += 2.0 * k_sqr * w2;
                enrg_diss += 2.0 * pre_fac * cabs(u_z * conj(u_z) + v_z * conj(v_z));
                enst_diss += quirk(o, NS2D_QUIRK_ENST_DISS) ? 2.0 * w2 : 2.0 * pre_fac * w2;
                if (k_sqr >= lwr && k_sqr < upr) {
                    d_enrg += (tmp_deriv + tmp_diss) * (2.0 / k_sqr);
                    enrg_dsb += tmp_diss * (2.0 / k_sqr);
                    enrg_flux += tmp_deriv * (2.0 / k_sqr);
                    d_enst += 2.0 * (tmp_deriv + tmp_diss);
                    enst_dsb += 2.0 * tmp_diss;
                    enst_flux += 2.0 * tmp_deriv;
                }
            }
            /* spectra (:250-331) */
            double sd = tmp_deriv * const_fac * norm_fac;
            double ss = pre_fac * w2 * const_fac * norm_fac;
            if (edge) {
                e_sp[spec_indx] += const_fac * norm_fac * w2 * (1.0 / k_sqr);
                z_sp[spec_indx] += const_fac * norm_fac * w2;
                dz_sp[spec_indx] += sd + ss;
                zd_sp[spec_indx] += ss;
                zf_sp[spec_indx] += sd;
                de_sp[spec_indx] += (sd + ss) / k_sqr;
                ed_sp[spec_indx] += ss / k_sqr;
                ef_sp[spec_indx] += sd / k_sqr;
            } else {
                e_sp[spec_indx] += 2.0 * const_fac * norm_fac * w2 * (1.0 / k_sqr);
                z_sp[spec_indx] += 2.0 * const_fac * norm_fac * w2;
                dz_sp[spec_indx] += 2.0 * (sd + ss);
                zd_sp[spec_indx] += 2.0 * ss;
                zf_sp[spec_indx] += 2.0 * sd;
                de_sp[spec_indx] += 2.0 * (sd + ss) / k_sqr;
                ed_sp[spec_indx] += 2.0 * ss / k_sqr;
                ef_sp[spec_indx] += 2.0 * sd / k_sqr;
            }
        }
    /* normalisation (:350-372); the d_*_dt subset sums are left unscaled as in the reference */
    enrg_diss *= 2.0 * const_fac * norm_fac;
    enst_diss *= 2.0 * const_fac * norm_fac;
    tot_enstr *= const_fac * norm_fac;
    tot_palin *= const_fac * norm_fac;
    tot_forc *= const_fac * norm_fac;
    tot_div *= const_fac * norm_fac;
    tot_energy *= const_fac * norm_fac;
    enrg_flux *= const_fac * norm_fac;
    enrg_dsb *= 2.0 * const_fac * norm_fac;
    enst_flux *= const_fac * norm_fac;
    enst_dsb *= 2.0 * const_fac * norm_fac;
    double out[13] = {tot_energy, tot_enstr, tot_palin, tot_forc, tot_div, enrg_diss, enst_diss,
                      d_enrg, enrg_flux, enrg_dsb, d_enst, enst_flux, enst_dsb};
    memcpy(s13, out, sizeof out);
}

/* Taylor-Green test input w = 2 sin x sin y (the 64^2 Taylor-Green workload), transformed
   with the oracle FFT: w_hat(+-1, 1) = -Nx*Ny/2 * (+-1). */
void oracle_ic_taylor_green(int nx, int ny, double* w_hat) {
    const int nyf = ny / 2 + 1;
    double* r = (double*)calloc((size_t)nx * (ny + 2), sizeof(double));
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            r[(size_t)i * (ny + 2) + j] = 2.0 * sin(2.0 * M_PI * i / nx) * sin(2.0 * M_PI * j / ny);
    offt_r2c_2d(nx, ny, 1, r, (cplx*)w_hat);
    (void)nyf;
    free(r);
}
