/*
 * include/ns2d.h -- C ABI of libns2d.so, the B200 (sm_100a) pseudospectral
 * time step of the 2-D vorticity Navier-Stokes solver.
 *
 * The entry points replace the reference solver's FFTW-MPI path
 * (EndCar808/2D-Navier-Stokes, Solver/src).  Each declaration names the
 * reference function it stands in for.  The arrays that cross this boundary use
 * the reference's own layouts:
 *
 *   spectral field  : [nx][ny/2+1] complex128, interleaved (re, im) doubles,
 *                     row i <-> kx = i (i <= nx/2) or i - nx, column j <-> ky = j
 *                     (Solver/src/solver.c:2042-2066); the state "w_hat".
 *   real field      : [nx][ny] float64 (unpadded; the reference pads rows to
 *                     ny+2 for FFTW in place, which is a storage detail).
 *
 * All functions return an ns2d_status; NS2D_OK is 0.  The reference exits the
 * process on every failure (Solver/src/solver.c:2314-2325, :2643-2651); here
 * the error is returned and a message is kept per handle (ns2d_last_error).
 * A handle is not thread-safe; distinct handles are independent.  All state is
 * device resident; host pointers are copied in and out within the call.
 */
#ifndef NS2D_H
#define NS2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NS2D_ABI_VERSION 2

typedef enum ns2d_status {
    NS2D_OK = 0,
    NS2D_ERR_INVALID = 1,     /* bad argument or parameter combination            */
    NS2D_ERR_UNSUPPORTED = 2, /* valid in the reference, not built here (e.g. N)  */
    NS2D_ERR_CUDA = 3,        /* CUDA runtime error (message in ns2d_last_error)  */
    NS2D_ERR_NOMEM = 4,       /* device or host allocation failed                 */
    NS2D_ERR_BLOWUP = 5,      /* max|w| >= 1e100 or non-finite (SystemCheck)      */
    NS2D_ERR_DT = 6,          /* dt <= 1e-10 (SystemCheck)                        */
    NS2D_ERR_ITERS = 7,       /* iteration limit 1e12 reached (SystemCheck)       */
    NS2D_ERR_STATE = 8,       /* call out of order (e.g. AB4 history missing)     */
    NS2D_ERR_NO_DEVICE = 9    /* no CUDA device / extension not usable            */
} ns2d_status;

/* Compile-time switches of Solver/src/data_types.h:49-61 and Solver/Makefile:55-67,
   selectable per handle. */
typedef enum ns2d_system { NS2D_NAVIER = 0, NS2D_EULER = 1 } ns2d_system;
typedef enum ns2d_integrator {
    NS2D_RK4CN = 0, /* __RK4CN: RK4 with Crank-Nicolson linear term (stock)  */
    NS2D_RK4 = 1,   /* __RK4  : explicit RK4                                  */
    NS2D_AB4 = 2,   /* __AB4  : AB4 + CN after three RK4CN start-up steps     */
    NS2D_DP5 = 3    /* __DPRK5: Dormand-Prince 5(4) with step-size control    */
} ns2d_integrator;
typedef enum ns2d_dealias { NS2D_DEALIAS_23 = 0, NS2D_DEALIAS_HOU_LI = 1 } ns2d_dealias;
typedef enum ns2d_forcing {
    NS2D_FORCING_NONE = 0,
    NS2D_FORCING_KOLM = 1, /* "KOLM": one mode (kx=0, ky=force_k), value -F*n/2 */
    NS2D_FORCING_ZERO = 2  /* "ZERO": modes with |kx| or |ky| <= force_k set to 0
                              at the start of every step (force.c:436-533);
                              single handles only                               */
} ns2d_forcing;
typedef enum ns2d_precision { NS2D_FP64 = 0, NS2D_FP32 = 1 } ns2d_precision;
/* Model type (-D__PHASE_ONLY, data_types.h:75; "PHAEONLY" in the output names,
   utils.c:515-519).  Phase-only keeps every mode's amplitude through the
   update of RK4Step (solver.c:634-647, 822-857): after the step each mode
   k != 0 is rescaled to |w_hat| of the state before it.  RK4CN and RK4 only
   (AB4Step has no reset, solver.c:261-350; the DP5 path's reset does not
   compile, solver.c:518-521).  Where the updated mode is exactly 0 (every mode
   the 2/3 rule zeroes; where the Hou-Li filter underflows, with the
   reference's integer ratios the corner |kx| = ky = N/2) the reference divides
   0 by 0 and its step returns NaN there; here the mode stays 0. */
typedef enum ns2d_model { NS2D_MODEL_FULL = 0, NS2D_MODEL_PHASE_ONLY = 1 } ns2d_model;

/* Reference behaviours that differ from the textbook scheme.  Setting the bit
   reproduces the reference exactly; clearing it gives the corrected form. */
enum {
    NS2D_QUIRK_CONJ_STATE = 1 << 0,  /* ForceConjugacy writes the *state* from the RHS input (solver.c:1031,2096-2103) */
    NS2D_QUIRK_HYPER_LATCH = 1 << 1, /* `=` for `==` in the viscous branches latches hyperviscosity on (solver.c:675,843) */
    NS2D_QUIRK_RK4_LINEAR = 1 << 2,  /* explicit RK4 adds +dt*D*X to each stage (solver.c:664-684)                     */
    NS2D_QUIRK_HOU_LI_INT = 1 << 3,  /* Hou-Li filter with integer k/(N/2) (solver.c:1088)                            */
    NS2D_QUIRK_CFL_INDEX = 1 << 4,   /* CFL velocity with row index (i*Ny)/2+1 (solver.c:2394)                        */
    NS2D_QUIRK_ENST_DISS = 1 << 5,   /* enstrophy dissipation weight-2 branch without pre_fac (sys_msr.c:225)          */
    NS2D_QUIRKS_REFERENCE = 0x3f
};

typedef struct ns2d_params {
    int32_t nx, ny;           /* grid; powers of two, 16..2048 (reference: -n -n)       */
    int32_t system;           /* ns2d_system                                           */
    int32_t integrator;       /* ns2d_integrator                                       */
    int32_t dealias;          /* ns2d_dealias                                          */
    int32_t forcing;          /* ns2d_forcing                                          */
    int32_t force_k;          /* -f 2nd                                                */
    int32_t quirks;           /* NS2D_QUIRK_* bits                                     */
    double force_scale;       /* -f 3rd                                                */
    double nu;                /* -v 1st                                                */
    double hyper_visc_pow;    /* -v 3rd                                                */
    double ekmn_alpha;        /* -d 1st                                                */
    double ekmn_drag_pow;     /* -d 3rd                                                */
    int32_t hyper_visc_flag;  /* -v 2nd                                                */
    int32_t ekmn_drag_flag;   /* -d 2nd                                                */
    int32_t adapt_step_flag;  /* -h 2nd                                                */
    int32_t cfl_cond_flag;    /* -c 1st                                                */
    double cfl_const;         /* -c 2nd                                                */
    double dt;                /* -h 1st: initial / fixed step                          */
    int32_t precision;        /* ns2d_precision                                        */
    int32_t flux_diagnostics; /* 1 = the stock dataset flags (__ENST_FLUX...): the
                                 measurables call evaluates the RHS of the state     */
    int32_t device;           /* CUDA device ordinal                                  */
    int32_t dealias_edge;     /* 2/3 rule edge: 0 = zero |k| >= (int)(N/3), the
                                 solver's ApplyDealiasing (solver.c:1049-1068);
                                 1 = zero |k| > (int)(N/3), the post-processing
                                 program's (PostProcessing/src/full_field.c:128);
                                 single handles only                          */
    int32_t model;            /* ns2d_model; RK4CN / RK4 (handles and ensembles)  */
} ns2d_params;

/* Scalars of ComputeSystemMeasurables (Solver/src/sys_msr.c:32-373), in order. */
typedef struct ns2d_measures {
    double energy, enstrophy, palinstrophy, forcing_input, divergence;
    double energy_diss, enstrophy_diss;
    double d_enrg_dt_sbst, enrg_flux_sbst, enrg_diss_sbst;
    double d_enst_dt_sbst, enst_flux_sbst, enst_diss_sbst;
} ns2d_measures;

/* What GetMaxData (Solver/src/solver.c:2171) reduces. */
typedef enum ns2d_max_kind { NS2D_MAX_VORT = 0, NS2D_MAX_VEL = 1, NS2D_MAX_VORT_FOUR = 2 } ns2d_max_kind;

typedef struct ns2d_handle ns2d_handle;

/* Defaults of GetCMLArgs (Solver/src/utils.c:51-90) plus the stock compile
   switches: 64x64, nu = 1e-4, dt = 1e-4, RK4CN, 2/3 dealias, no forcing,
   flux diagnostics on, all reference quirks on, FP64. */
ns2d_status ns2d_params_default(ns2d_params* p);

/* Allocates the handle's device arrays on p->device and encodes the tensor
   maps its column passes use for TMA tile copies.  With the environment
   variable NS2D_DISABLE_TMA set (to anything but "0") when the handle is
   created, or when the driver offers no tensor-map encoder, those passes copy
   per thread instead: the same results to rounding, slower.  (No counterpart
   in the reference, which allocates in AllocateMemory, solver.c:2603.) */
ns2d_status ns2d_create(const ns2d_params* p, ns2d_handle** out);
ns2d_status ns2d_destroy(ns2d_handle* h);
const char* ns2d_last_error(const ns2d_handle* h);
const char* ns2d_status_string(ns2d_status s);
int ns2d_abi_version(void);

/* Sizes: ny/2+1 and the spectrum bin count n_spect (sys_msr.c:394). */
ns2d_status ns2d_dims(const ns2d_handle* h, int32_t* nx, int32_t* ny, int32_t* nyf, int32_t* n_spect);

/* State in/out (reference layout, host memory).  Stand-in for the reference's
   direct use of run_data->w_hat after InitialConditions (solver.c:89). */
ns2d_status ns2d_set_w_hat(ns2d_handle* h, const double* w_hat);
ns2d_status ns2d_get_w_hat(ns2d_handle* h, double* w_hat);
/* Same, with device pointers (no host copy). */
ns2d_status ns2d_set_w_hat_device(ns2d_handle* h, const double* d_w_hat);
ns2d_status ns2d_get_w_hat_device(ns2d_handle* h, double* d_w_hat);

/* ComputeForcing (Solver/src/force.c:516): forcing values for this step. */
ns2d_status ns2d_compute_forcing(ns2d_handle* h, double dt);
/* Forcing of listed modes, added to every RHS evaluation until changed (the
   reference's run_data->forcing / forcing_indx, added at solver.c:1022-1027):
   values[2m], values[2m+1] = re, im of the forcing at flat index idx[m] of the
   [nx][ny/2+1] half spectrum.  The stochastic and Gaussian forcings of
   force.c:104-433 draw their values with glibc rand() on the host each step
   (ComputeForcing); a caller passes them here.  n = 0 removes the forcing.
   Adds to the built-in KOLM forcing when both are set. */
ns2d_status ns2d_set_forcing_modes(ns2d_handle* h, int32_t n, const int32_t* idx, const double* values);

/* NonlinearRHSBatch (Solver/src/solver.c:884; solver.h:39).  in == NULL means
   the state itself (stage-1 form).  out receives the dealiased nonlinear term
   plus forcing.  With NS2D_QUIRK_CONJ_STATE the state's ky = 0, kx < 0 entries
   are overwritten with conj(in[|kx|, 0]) exactly as the reference does. */
ns2d_status ns2d_nonlinear_rhs(ns2d_handle* h, const double* in, double* out);

/* RK4Step (Solver/src/solver.c:625; solver.h:26), RK4CN or RK4 per params. */
ns2d_status ns2d_rk4_step(ns2d_handle* h, double dt);

/* AB4Step (Solver/src/solver.c:261; solver.h:30).  iters is the reference's
   1-based iteration counter: iters <= 3 take RK4CN start-up steps. */
ns2d_status ns2d_ab4_step(ns2d_handle* h, double dt, int32_t iters);

/* RK5DPStep (Solver/src/solver.c:360-570; solver.h:33): one Dormand-Prince
   5(4) trial step of dt, in place (the state becomes the fifth-order solution),
   *err = RMS over the half spectrum of |y5 - y4| / (1e-7 + 1e-7 max(|y0|, |y5|))
   (DP_ABS_TOL, DP_REL_TOL, data_types.h:137-141), accumulated in FP64.  The
   linear term is explicit in every stage.  The shipped routine does not compile
   (w_hat_last, an uninitialised err_sum) and its driver's accept/retry test is
   inverted (solver.c:153-171); this is the corrected step, and accepting or
   retrying is the caller's (dt_new = dt min(1.5, max(0.01, 0.8 err^-1/5))). */
ns2d_status ns2d_dp5_step(ns2d_handle* h, double dt, double* err);

/* RK5DPStep (Solver/src/solver.c:360-570; solver.h:33) as the reference writes
   it, for parity with the reference's own arithmetic; ns2d_dp5_step is the
   corrected integrator.  The reference's three compile defects are fixed
   (err_sum starts at 0, a surplus parenthesis at :517, w_hat_last read from
   Int_data at :564); everything else is kept: the Butcher table of :35-43
   (its a32 is 0.5, not 9/40) on the nonlinear term alone, stage inputs built
   from the live state (which every RHS rewrites through the ForceConjugacy
   side effect), the Crank-Nicolson update of the fifth-order sum, and, for
   iters > 1 only, the error norm of :515-552: RMS over the half spectrum of
   Re(w_new - ho) / (1e-7 + 1e-7 max(|w_last|, |w_new|)) with ho the real part
   of w_new + dt sum bs k (the reference stores it in a double) and w_last
   the state after the previous error step (0 before it).  iters is
   SpectralSolve's iteration counter; *err = DP_err, unchanged when iters == 1
   (0 on a fresh handle).  The state is advanced. */
ns2d_status ns2d_rk5dp_step(ns2d_handle* h, double dt, int32_t iters, double* err);

/* nsteps fixed-dt steps of the configured integrator without host round trips
   (the loop body of SpectralSolve, solver.c:142-236, minus saving). */
ns2d_status ns2d_step_n(ns2d_handle* h, int32_t nsteps, double dt);

/* RK4Step with the state in host memory, as the reference keeps it in
   run_data->w_hat (solver.c:625): copies w_hat in, steps, copies it back.
   The drop-in form for callers that own a host array. */
ns2d_status ns2d_rk4_step_host(ns2d_handle* h, double* w_hat, double dt);

/* Enqueue nsteps fixed-dt steps on the handle's stream and return without
   waiting.  Failures detected on the device (SystemCheck) are reported by the
   next ns2d_check. */
ns2d_status ns2d_step_async(ns2d_handle* h, int32_t nsteps, double dt);
/* Wait for queued work and apply SystemCheck (solver.c:2301) to it.  Also
   returns NS2D_ERR_CUDA when a column pass's bounded wait for its own TMA tile
   copies ran out (no counterpart in the reference). */
ns2d_status ns2d_check(ns2d_handle* h);

/* ApplyDealiasing (solver.c:1039) on a host array of array_dim interleaved
   spectral fields, in place. */
ns2d_status ns2d_apply_dealiasing(ns2d_handle* h, double* arr, int32_t array_dim);

/* ForceConjugacy (solver.c:2074): state[kx<0, 0] = conj(arr[|kx|, 0]).
   arr == NULL means the state itself. */
ns2d_status ns2d_force_conjugacy(ns2d_handle* h, const double* arr);

/* GetMaxData (solver.c:2171). */
ns2d_status ns2d_get_max_data(ns2d_handle* h, int32_t kind, double* out);

/* GetTimestep (solver.c:2376): CFL or vorticity-ratio adaptive step; updates
   the handle's min/max dt record. */
ns2d_status ns2d_get_timestep(ns2d_handle* h, double* dt);
ns2d_status ns2d_dt_range(const ns2d_handle* h, double* min_dt, double* max_dt);
/* w_max_init of InitialConditions (solver.c:2003): reference value of the
   vorticity-ratio step rule; captured on every ns2d_set_w_hat. */
ns2d_status ns2d_set_w_max_init(ns2d_handle* h, double w_max_init);

/* SystemCheck (solver.c:2301): NS2D_ERR_BLOWUP / _DT / _ITERS instead of exit(1). */
ns2d_status ns2d_system_check(ns2d_handle* h, double dt, int64_t iters);

/* ComputeSystemMeasurables (sys_msr.c:32).  spectra may be NULL; otherwise it
   receives 8 * n_spect doubles: enrg, enst, d_enst_dt, enst_flux, enst_diss,
   d_enrg_dt, enrg_flux, enrg_diss spectra.  With flux_diagnostics the RHS of
   the state is evaluated first (with its conjugacy side effect, sys_msr.c:127). */
ns2d_status ns2d_system_measurables(ns2d_handle* h, ns2d_measures* out, double* spectra);

/* Real-space vorticity [nx][ny] (c2r of the state, normalised). */
ns2d_status ns2d_get_w_real(ns2d_handle* h, double* w);

/* The reference's 2-D FFTW transforms on the handle's device and precision,
   host buffers, unnormalised (fftw_mpi_plan_dft_r2c_2d / _c2r_2d,
   Solver/src/solver.c:2603-2615): r2c maps a real [nx][ny] field to the half
   spectrum [nx][ny/2+1] complex128 (e^{-i..}); c2r maps back (e^{+i..}) and,
   like FFTW's c2r, reads only the real parts of the ky = 0 and ky = ny/2
   columns.  For initial conditions and file input (solver.c:1139-1873);
   they use the handle's scratch fields, not its state. */
ns2d_status ns2d_fft_r2c(ns2d_handle* h, const double* real, double* spec);
ns2d_status ns2d_fft_c2r(ns2d_handle* h, const double* spec, double* real);

/* Mean-flow sums of one ComputeSystemMeasurables call on the state:
   mean_y[kx row] = sum_ky c |v_hat| (Solver/src/sys_msr.c:199, 227) and
   mean_x[ky] = sum_kx c |u_hat|, c = 1 on ky = 0, ny/2 and 2 elsewhere.
   mean_x is the sum sys_msr.c:338-348 intends (that loop reads the ky array
   with the row counter).  Either pointer may be NULL; needs nx + ny/2 + 1 <= 4096. */
ns2d_status ns2d_mean_flow(ns2d_handle* h, double* mean_x, double* mean_y);

/* The nonlinear term of NonlinearRHSBatch for callers that cannot allocate
   device memory.  No counterpart in the reference; it exists for code that runs
   under somebody else's stream capture (cudaMalloc cannot be recorded into a
   graph), for time loops that cannot afford cudaMalloc's implicit device
   synchronisation, and for applications whose device memory comes from their
   own pool.  No handle: the caller passes the parameters and two device arrays
   in the reference layout, [nx][ny/2+1] complex128 (d_w_hat read, d_rhs
   written), both starting on a 16-byte boundary (else NS2D_ERR_INVALID, with
   nothing launched), and the work is queued on cuda_stream (NULL = legacy
   default) of the current device, which p->device must name.  The parameters
   pass ns2d_create's checks or the call returns NS2D_ERR_INVALID.  An error
   already pending from the caller's earlier launches is reported as
   NS2D_ERR_CUDA and left pending; nothing is launched then.
   The output equals ns2d_nonlinear_rhs(h, w_hat, rhs) after
   ns2d_compute_forcing on a handle with the same parameters; the conjugacy
   side effect on a state does not apply (there is none).  FP64 only.
   Limit: square grids of 16..NS2D_NOALLOC_MAX_N; larger sizes return
   NS2D_ERR_UNSUPPORTED before touching the device.  The intermediate fields
   live in one static device array of NS2D_NOALLOC_SCRATCH_BYTES that every GPU
   loading the library holds until exit.  All calls on a device share that
   array, so calls that overlap on the GPU (unordered streams) race.  The first
   call on each device (and for each grid size) does set-up -- it looks up the
   array's device address and sets kernel shared-memory limits -- and should
   come before any stream capture. */
#define NS2D_NOALLOC_MAX_N 256
#define NS2D_NOALLOC_SCRATCH_BYTES (16u * (5u * 256u * 129u + 256u))
ns2d_status ns2d_nonlinear_rhs_noalloc(const ns2d_params* p, const double* d_w_hat, double* d_rhs,
                                       void* cuda_stream);

/* ---- Sector triad sums (post-processing phase synchronisation) -------------
   One snapshot's sums of PhaseSyncSector (PostProcessing/src/phase_sync.c:
   281-1058) over the triads (k1, k2 = k3 - k1, k3) of its sector search
   (AllocatePhaseSyncMemory, phase_sync.c:1744-1948), without storing the
   triads: the caller passes the sector bounds and the wavevector angles it
   computed, and the snapshot's amplitudes and phases in the full-field layout
   of FullFieldData (index (kmax - kx)(2 kmax + 1) + kmax + ky, |kx|, |ky| <=
   kmax).  The sums come back per class

     sums[((((a n_k1 + l) 2 + term) 3 + cls) 2 + contrib) 2 + unidir][8]

   with a the k3 sector, l the k1 sector as stored (phase_sync.c:1776),
   term 0 the positive flux term and 1 the negative one, cls the sign of
   flux_pre_fac (0: < 0, 1: > 0, 2: == 0), contrib 0 / 1 for 1d / 2d
   contributions and unidir the unidirectional condition of C_theta (k3_y >= 0
   for the positive term, k1_y >= 0 and k2_y >= 0 for the negative); the eight
   values are the triad count, the enstrophy flux (sign of the term applied),
   sum exp(i phi) of the generalised phase of type 0, the same for the triad's
   own type (they differ for cls 2 of the negative term), and the collective
   term's sum (re, im).  Host arrays; one call allocates, runs and frees on
   `device`. */
#define NS2D_TRIAD_VALUES 8
typedef struct ns2d_triad_sectors {
    int32_t kmax;               /* tables cover |kx|, |ky| <= kmax                  */
    int32_t n_k3, n_k1;         /* sector counts                                   */
    int32_t reserved;
    double kmax_sqr, kmax_c_sqr;/* kmax^2 (<= kmax * kmax) and kmax_C^2             */
    const double* k3_lwr;       /* [n_k3] sector bounds theta_k3 -+ dtheta_k3 / 2   */
    const double* k3_upr;
    const double* k1_lwr;       /* [n_k3 * n_k1] bounds of the k1 sector stored at (a, l) */
    const double* k1_upr;
    const double* angle;        /* [(2kmax+1)^2] atan2(kx, ky)                      */
    const double* angle_neg;    /* [(2kmax+1)^2] atan2(-kx, -ky)                    */
} ns2d_triad_sectors;
ns2d_status ns2d_triad_sector_sums(int32_t device, const ns2d_triad_sectors* g, const double* amps,
                                   const double* phases, double* sums);

/* ---- Discrete adjoint ------------------------------------------------------
   Gradient of a final-time functional J(w(T)) with respect to the initial
   vorticity for n fixed-dt RK4CN steps (RK4Step, solver.c:625-873, over
   NonlinearRHSBatch, solver.c:884-1032).  No counterpart in the reference,
   whose extreme-enstrophy and max-palinstrophy searches (MAX_PALIN,
   solver.c:1775-1853) read their initial conditions from files.

   Gradients use the half-spectrum inner product
       <a, b>_W = sum_j c_j Re(conj(a_j) b_j),  c_j = 1 on ky = 0 and ky = ny/2, 2 else,
   so dJ = <g, dw0>_W for every Hermitian perturbation dw0.  Arrays are the
   reference layout [nx][ny/2+1] complex128.  The adjoint covers the
   Navier-Stokes RK4CN step with NS2D_QUIRK_CONJ_STATE clear (the corrected
   ForceConjugacy, the identity on Hermitian states); other integrators and that
   quirk return NS2D_ERR_UNSUPPORTED.  The handle's precision applies to the
   adjoint too; J and inner products are accumulated in FP64. */
typedef enum ns2d_objective_kind {
    NS2D_OBJ_ENSTROPHY = 0,    /* Z = 4 pi^2 0.5/(nx ny)^2 sum_j c_j |w_j|^2 (sys_msr.c:190-227, 356-363) */
    NS2D_OBJ_PALINSTROPHY = 1  /* P = same with |k|^2 |w_j|^2                                              */
} ns2d_objective_kind;

/* Advance nsteps RK4CN steps of dt from the state, keeping a copy of w_hat
   every checkpoint_every steps for ns2d_adjoint_backward (memory: one field per
   checkpoint plus checkpoint_every steps x 8 real fields for the recomputed
   stages). */
ns2d_status ns2d_adjoint_record(ns2d_handle* h, int32_t nsteps, double dt, int32_t checkpoint_every);
/* Reverse sweep over the recorded run: lam_0 = (dw(T)/dw(0))^T lam_T in the W
   inner product.  Segments are recomputed from their checkpoints; the state is
   left at w(T).  Host and device-pointer forms. */
ns2d_status ns2d_adjoint_backward(ns2d_handle* h, const double* lam_T, double* lam_0);
ns2d_status ns2d_adjoint_backward_device(ns2d_handle* h, const double* d_lam_T, double* d_lam_0);
/* J(state) (ns2d_objective_kind) and, when d_grad != NULL, its W-gradient
   (device array). */
ns2d_status ns2d_objective(ns2d_handle* h, int32_t kind, double* value, double* d_grad);
/* The whole gradient: record, J(w(T)), reverse sweep; grad (host) = dJ/dw(0). */
ns2d_status ns2d_adjoint_gradient(ns2d_handle* h, int32_t nsteps, double dt, int32_t checkpoint_every,
                                  int32_t kind, double* value, double* grad);
/* Device time (ms) of the last ns2d_adjoint_record and of the last reverse
   sweep (stage recomputation and adjoint steps, which overlap on two streams). */
ns2d_status ns2d_adjoint_times(const ns2d_handle* h, double* ms_record, double* ms_reverse);
/* <a, b>_W of two device arrays, accumulated in FP64. */
ns2d_status ns2d_wdot_device(ns2d_handle* h, const double* d_a, const double* d_b, double* value);

/* ---- Batched ensembles -----------------------------------------------------
   Independent trajectories of possibly different square grid sizes (64..512)
   advanced together: every pass of a step is one launch for all members, and
   the step is replayed from a captured CUDA graph.  The reference has no
   counterpart inside the solver; it runs parameter sweeps as separate
   processes (run_solver.py:270-292).  Members share all parameters except the
   grid size; RK4CN or RK4, FP64 or FP32.  The ensemble's non-finite check
   replaces SystemCheck's bound. */
typedef struct ns2d_ensemble ns2d_ensemble;
ns2d_status ns2d_ensemble_create(const ns2d_params* base, int32_t n_members, const int32_t* sizes,
                                 ns2d_ensemble** out);
ns2d_status ns2d_ensemble_destroy(ns2d_ensemble* e);
const char* ns2d_ensemble_last_error(const ns2d_ensemble* e);
int64_t ns2d_ensemble_launch_count(const ns2d_ensemble* e);
ns2d_status ns2d_ensemble_set_w_hat(ns2d_ensemble* e, int32_t member, const double* w_hat);
ns2d_status ns2d_ensemble_get_w_hat(ns2d_ensemble* e, int32_t member, double* w_hat);
ns2d_status ns2d_ensemble_step_n(ns2d_ensemble* e, int32_t nsteps, double dt);
ns2d_status ns2d_ensemble_step_async(ns2d_ensemble* e, int32_t nsteps, double dt);
ns2d_status ns2d_ensemble_check(ns2d_ensemble* e);
/* Totals of ComputeSystemMeasurables for one member, flux terms set to 0. */
ns2d_status ns2d_ensemble_measurables(ns2d_ensemble* e, int32_t member, ns2d_measures* out);
/* Autotuner: picks, for the column and for the row passes, the block size
   (the tile shape, ns2d_ensemble_shape below) and the persistent grid (1..8
   blocks per SM), and whether one persistent launch per RK stage beats them,
   by timing steps at dt; returns the grids of the nine-launch form.  It
   advances the members.  ns2d_ensemble_set_grids keeps the other choices. */
ns2d_status ns2d_ensemble_tune(ns2d_ensemble* e, double dt, int32_t* col_grid, int32_t* row_grid);
ns2d_status ns2d_ensemble_set_grids(ns2d_ensemble* e, int32_t col_grid, int32_t row_grid);
/* Launch shape of the ensemble's step.  stage_launch = 0: nine launches, a
   column and a row pass per stage, with the block size of the column and of
   the row launches (256 or 128 threads; it sets the tile shape -- ky columns
   per column tile and row pairs per row block of every member, threads / T
   and threads / 2T with T the threads of one transform of the member's size)
   and their persistent grids.  stage_launch = 1: one persistent launch per RK
   stage (four per step, 256-thread blocks, grid stage_grid) whose tasks wait
   only for the same member's earlier tasks, so members' passes overlap.  The
   item counts of the chosen shapes are reported.  ns2d_ensemble_tune picks
   all of these by timing steps (no reference counterpart: the reference runs
   sweeps as separate processes, Solver/run_solver.py:270-292). */
typedef struct ns2d_ensemble_shape {
    int32_t col_threads, col_grid;
    int32_t row_threads, row_grid;
    int32_t stage_launch, stage_grid;
    int32_t col_items, row_items;   /* out only */
} ns2d_ensemble_shape;
ns2d_status ns2d_ensemble_set_shape(ns2d_ensemble* e, const ns2d_ensemble_shape* shape);
ns2d_status ns2d_ensemble_get_shape(const ns2d_ensemble* e, ns2d_ensemble_shape* shape);
ns2d_status ns2d_ensemble_set_stream(ns2d_ensemble* e, void* cuda_stream);

/* Execution control. */
ns2d_status ns2d_set_stream(ns2d_handle* h, void* cuda_stream);
ns2d_status ns2d_get_stream(const ns2d_handle* h, void** cuda_stream);
/* Per-kernel timing with CUDA events on the handle's stream.  Kernel classes:
   0 column pass (inverse transforms only), 1 column pass with RK stage
   combine, 2 column pass with the final update, 3 row pass, 4 other. */
#define NS2D_KERNEL_CLASSES 5
ns2d_status ns2d_set_kernel_timing(ns2d_handle* h, int32_t enable);
/* Totals since timing was enabled (waits for the stream). */
ns2d_status ns2d_kernel_times(ns2d_handle* h, double* ms_total, int64_t* launches, int32_t nclasses);
ns2d_status ns2d_synchronize(ns2d_handle* h);
/* Number of kernel launches issued by this handle since creation. */
int64_t ns2d_launch_count(const ns2d_handle* h);

#ifdef __cplusplus
}
#endif
#endif
