// api.cu -- C ABI of libns2d.so (include/ns2d.h): handle, device buffers and
// the host-side sequencing of the step kernels.  Each entry point names the
// reference function it replaces (EndCar808/2D-Navier-Stokes, Solver/src).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ns2d.h"
#include "diag.cuh"
#include "engine.cuh"
#include "handle.h"
#include "host_common.h"

using namespace ns2d;

namespace {

const char* kStatusNames[] = {"NS2D_OK", "NS2D_ERR_INVALID", "NS2D_ERR_UNSUPPORTED", "NS2D_ERR_CUDA",
                              "NS2D_ERR_NOMEM", "NS2D_ERR_BLOWUP", "NS2D_ERR_DT", "NS2D_ERR_ITERS",
                              "NS2D_ERR_STATE", "NS2D_ERR_NO_DEVICE"};

ns2d_status fail(ns2d_handle* h, ns2d_status s, const std::string& msg) {
    if (h) h->err = msg;
    return s;
}

#define CK(h, call)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail((h), e_ == cudaErrorMemoryAllocation ? NS2D_ERR_NOMEM : NS2D_ERR_CUDA,        \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

#define CKL(h)                                                                                        \
    do {                                                                                              \
        cudaError_t e_ = cudaGetLastError();                                                          \
        if (e_ != cudaSuccess) return fail((h), NS2D_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
    } while (0)

// Branch of the linear operator for this evaluation (see host_common.h).
int resolve_branch(ns2d_handle* h, bool latch) { return ns2d::resolve_branch(h->hyper_flag, h->p.ekmn_drag_flag, latch); }

LinOp make_lin(const ns2d_handle* h, int branch) { return make_lin_params(h->p, branch); }

bool quirk(const ns2d_handle* h, int bit) { return (h->p.quirks & bit) != 0; }

int col_tc(int n) {
    int tc = 0;
    with_size<double>(n, [&](auto L) { tc = decltype(L)::S::TC; });
    return tc;
}

template <typename Real>
using Cplx = typename Cx<Real>::T;

template <typename Real>
void fill_common(ns2d_handle* h, ColArgs<Real>& a, int branch) {
    using C = Cplx<Real>;
    std::memset(&a, 0, sizeof(a));
    a.state = (C*)h->state;
    a.acc = (C*)h->acc;
    a.f0 = (C*)h->f[0];
    a.f1 = (C*)h->f[1];
    a.f2 = (C*)h->f[2];
    a.f3 = (C*)h->f[3];
    a.tw = (const C*)h->tw;
    a.ldc = h->ldc;
    a.nyf = h->nyf;
    const int m = (int)(h->nx / 3.0);
    a.kmax_sqr = m * m + h->p.dealias_edge;
    a.dealias = h->p.dealias;
    a.houli_int = quirk(h, NS2D_QUIRK_HOU_LI_INT) ? 1 : 0;
    a.kolm = (h->p.forcing == NS2D_FORCING_KOLM) ? 1 : 0;
    a.has_force = h->forced ? 1 : 0;
    a.force_i = h->force_i;
    a.force_j = h->force_j;
    a.force_val.x = (Real)h->fre;
    a.force_val.y = (Real)h->fim;
    const double norm_fac = 1.0 / (double)(h->nx * h->ny);
    a.norm2 = (Real)std::pow(norm_fac, 2.0);
    a.inv_nxny = norm_fac;
    a.status = h->dstatus;
    a.final_tail = 1;
    a.force_field = h->ffield_on ? (const C*)h->ffield : nullptr;
    a.ntiles = (h->nyf + col_tc(h->nx) - 1) / col_tc(h->nx);
    a.lin = make_lin(h, branch);
    a.phase_only = h->p.model == NS2D_MODEL_PHASE_ONLY ? 1 : 0;
}

template <typename Real>
RowArgs<Real> row_args(ns2d_handle* h) {
    using C = Cplx<Real>;
    RowArgs<Real> r{};
    r.f0 = (const C*)h->f[0];
    r.f1 = (const C*)h->f[1];
    r.f2 = (const C*)h->f[2];
    r.f3 = (const C*)h->f[3];
    r.nl = (C*)h->nl;
    r.tw = (const C*)h->tw;
    r.ldc = h->ldc;
    r.nrows = h->nx;
    r.status = h->dstatus;
    return r;
}

cudaEvent_t take_event(ns2d_handle* h) {
    if (!h->ev_pool.empty()) {
        cudaEvent_t e = h->ev_pool.back();
        h->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets one launch with events when timing is on.
struct TimedLaunch {
    ns2d_handle* h;
    int cls;
    cudaEvent_t a = nullptr, b = nullptr;
    bool graph_slot = false;
    TimedLaunch(ns2d_handle* h_, int cls_) : h(h_), cls(cls_) {
        if (!h->timing) return;
        if (h->capturing_timed && h->gev_n < 16) {
            // event pair owned by the timed step graph, read after every replay
            const int k = h->gev_n++;
            auto& ev = h->gev_g[h->gev_set][k];
            for (int j = 0; j < 2; ++j)
                if (!ev[j]) cudaEventCreate(&ev[j]);
            a = ev[0];
            b = ev[1];
            h->gev_cls_g[h->gev_set][k] = cls;
            graph_slot = true;
        } else {
            a = take_event(h);
            b = take_event(h);
        }
        record(a);
    }
    // inside a capture the records become event nodes of the graph
    void record(cudaEvent_t e) {
        if (graph_slot) cudaEventRecordWithFlags(e, h->stream, cudaEventRecordExternal);
        else cudaEventRecord(e, h->stream);
    }
    ~TimedLaunch() {
        if (h->timing) {
            record(b);
            if (!graph_slot) h->ev_open.push_back({cls, {a, b}});
        }
        h->launches++;
    }
};

// Tensor maps for the column passes' TMA tile copies of f[0..3], acc, state and
// nl (see ColMaps).  Leaves h->col_maps null when a map cannot be encoded; the
// column passes then copy per thread.
template <typename Real>
void build_col_maps(ns2d_handle* h) {
    if (!tma_copies_enabled()) return;
    const int tc = col_tc(h->nx);
    auto* m = new (std::nothrow) ColMaps;
    if (!m) return;
    void* const bases[7] = {h->f[0], h->f[1], h->f[2], h->f[3], h->acc, h->state, h->nl};
    if (!encode_col_maps<Real>(m, bases, h->nx, h->nyf, h->ldc, tc)) {
        delete m;
        return;
    }
    h->col_maps = m;
}

// The TMA maps when the pass reads and writes exactly the arrays they describe.
template <typename Real>
const ColMaps* col_maps_for(const ns2d_handle* h, int mode, const ColArgs<Real>& a) {
    if (!h->col_maps || mode == COL_RHS) return nullptr;
    if (mode == COL_P1)
        return a.src == h->state && a.f0 == h->f[0] && a.f1 == h->f[1] && a.f2 == h->f[2] && a.f3 == h->f[3]
                   ? static_cast<const ColMaps*>(h->col_maps)
                   : nullptr;
    if (a.src != h->nl || a.state != h->state || a.acc != h->acc) return nullptr;
    if (mode == COL_STAGE && (a.f0 != h->f[0] || a.f1 != h->f[1] || a.f2 != h->f[2] || a.f3 != h->f[3])) return nullptr;
    return static_cast<const ColMaps*>(h->col_maps);
}

template <typename Real>
void launch_col(ns2d_handle* h, int mode, const ColArgs<Real>& a) {
    TimedLaunch t(h, mode == COL_STAGE ? 1 : mode == COL_FINAL ? 2 : 0);
    const ColMaps* maps = col_maps_for<Real>(h, mode, a);
    with_size<Real>(h->nx, [&](auto L) { decltype(L)::col(mode, a, h->stream, maps); });
}
// Row pass of stage `stage` (1..4); with a capture target set, the stage's real
// fields go to planes 2(stage-1) and 2(stage-1)+1 of it.
template <typename Real>
void launch_row(ns2d_handle* h, int stage = 0) {
    TimedLaunch t(h, 3);
    RowArgs<Real> r = row_args<Real>(h);
    if (h->cap_step && stage >= 1) {
        const size_t plane = (size_t)h->nx * h->ny;
        r.cap_uv = (Cplx<Real>*)h->cap_step + (size_t)(2 * (stage - 1)) * plane;
        r.cap_w = r.cap_uv + plane;
    }
    with_size<Real>(h->nx, [&](auto L) { decltype(L)::row(r, h->stream); });
}

// Forcing values for this step (ComputeForcing, Solver/src/force.c:516-581);
// ZERO forcing kills its modes of the state instead.
void compute_forcing(ns2d_handle* h, double dt) {
    (void)dt;
    if (h->p.forcing == NS2D_FORCING_ZERO) {
        if (h->fp32)
            zero_modes_kernel<float><<<296, 256, 0, h->stream>>>((float2*)h->state, h->nx, h->nyf, h->ldc, h->p.force_k);
        else
            zero_modes_kernel<double><<<296, 256, 0, h->stream>>>((double2*)h->state, h->nx, h->nyf, h->ldc, h->p.force_k);
        h->launches++;
    }
    if (h->p.forcing == NS2D_FORCING_KOLM && h->forced) {
        // -0.5 * F * (k + 0 i)  (force.c:537)
        h->fre = -0.5 * h->p.force_scale * (double)h->p.force_k;
        h->fim = -0.5 * h->p.force_scale * 0.0;
    }
}

// Rebuild the Crank-Nicolson factor table when dt or the operator branch changed.
ns2d_status ensure_cn(ns2d_handle* h, double dt, int branch) {
    if (h->cn_dt == dt && h->cn_branch == branch) return NS2D_OK;
    cn_table_kernel<<<296, 256, 0, h->stream>>>(h->cn, h->nx, h->nyf, h->ldc, dt, make_lin(h, branch));
    h->launches++;
    CKL(h);
    h->cn_dt = dt;
    h->cn_branch = branch;
    return NS2D_OK;
}

// One RK4 / RK4CN step (RK4Step, Solver/src/solver.c:625-873).  If rk1_out is
// non-null the stage-1 RHS is stored there (AB4 start-up, solver.c:283).
template <typename Real>
ns2d_status rk4_step_impl(ns2d_handle* h, double dt, void* rk1_out) {
    using C = Cplx<Real>;
    compute_forcing(h, dt);
    const bool euler = h->p.system == NS2D_EULER;
    const bool explicit_rk4 = euler || h->p.integrator == NS2D_RK4;
    const bool rk4_lin = !euler && h->p.integrator == NS2D_RK4;
    const bool latch = quirk(h, NS2D_QUIRK_HYPER_LATCH);
    int branch = 4;
    if (!euler || rk4_lin) branch = resolve_branch(h, latch);
    const int lin_stage = rk4_lin ? (quirk(h, NS2D_QUIRK_RK4_LINEAR) ? 1 : 2) : 0;
    const double A[3] = {0.5, 0.5, 1.0};
    const double B_cn[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    const double B_ex[4] = {1.0, 2.0, 2.0, 1.0};
    const bool conj_quirk = quirk(h, NS2D_QUIRK_CONJ_STATE);

    ColArgs<Real> a;
    fill_common<Real>(h, a, branch);
    a.src = (const C*)h->state;
    launch_col<Real>(h, COL_P1, a);
    for (int s = 1; s <= 4; ++s) {
        launch_row<Real>(h, s);
        fill_common<Real>(h, a, branch);
        a.src = (const C*)h->nl;
        a.dt = dt;
        a.conj_mode = (conj_quirk || s == 1) ? 1 : 0;
        if (s == 1) {
            a.conj_src = (const C*)h->state;
            a.conj_stride = h->ldc;
        } else {
            a.conj_src = (const C*)h->col0[(s - 1) & 1];
            a.conj_stride = 1;
        }
        a.lin_stage = lin_stage;
        a.xin = (lin_stage && s > 1) ? (const C*)h->tmpfull : nullptr;
        a.b_cur = explicit_rk4 ? B_ex[s - 1] : B_cn[s - 1];
        if (s == 1 && rk1_out) a.rhs_store = (C*)rk1_out;
        if (s < 4) {
            a.a_next = A[s - 1];
            a.first = (s == 1);
            a.col0_out = (C*)h->col0[s & 1];
            a.out = lin_stage ? (C*)h->tmpfull : nullptr;
            launch_col<Real>(h, COL_STAGE, a);
        } else {
            a.scheme = explicit_rk4 ? 1 : 0;
            if (!explicit_rk4) {
                ns2d_status s2 = ensure_cn(h, dt, branch);
                if (s2) return s2;
                a.cn = h->cn;
            }
            launch_col<Real>(h, COL_FINAL, a);
        }
    }
    CKL(h);
    return NS2D_OK;
}

// AB4Step past the start-up (Solver/src/solver.c:286-349).
template <typename Real>
ns2d_status ab4_update_impl(ns2d_handle* h, double dt) {
    using C = Cplx<Real>;
    compute_forcing(h, dt);
    const bool euler = h->p.system == NS2D_EULER;
    const int branch = euler ? 4 : resolve_branch(h, false);
    ColArgs<Real> a;
    fill_common<Real>(h, a, branch);
    a.src = (const C*)h->state;
    a.col0_out = (C*)h->col0[0];  // the final pass rewrites the state's column 0
    launch_col<Real>(h, COL_P1, a);
    launch_row<Real>(h);
    fill_common<Real>(h, a, branch);
    a.src = (const C*)h->nl;
    a.dt = dt;
    a.conj_mode = 1;
    a.conj_src = (const C*)h->col0[0];
    a.conj_stride = 1;
    a.scheme = euler ? 3 : 2;
    if (!euler) {
        ns2d_status s2 = ensure_cn(h, dt, branch);
        if (s2) return s2;
        a.cn = h->cn;
    }
    a.h0 = (const C*)h->ab[0];
    a.h1 = (const C*)h->ab[1];
    a.h2 = (const C*)h->ab[2];
    a.rhs_store = (C*)h->ab[3];
    launch_col<Real>(h, COL_FINAL, a);
    CKL(h);
    void* oldest = h->ab[0];
    h->ab[0] = h->ab[1];
    h->ab[1] = h->ab[2];
    h->ab[2] = h->ab[3];
    h->ab[3] = oldest;
    return NS2D_OK;
}

// NonlinearRHSBatch on `src` (device, [nx][ldc]); result in h->rhsbuf.
template <typename Real>
ns2d_status rhs_impl(ns2d_handle* h, const void* src, bool src_is_state) {
    using C = Cplx<Real>;
    ColArgs<Real> a;
    fill_common<Real>(h, a, 4);
    a.src = (const C*)src;
    launch_col<Real>(h, COL_P1, a);
    launch_row<Real>(h);
    fill_common<Real>(h, a, 4);
    a.src = (const C*)h->nl;
    a.rhs_store = (C*)h->rhsbuf;
    a.conj_mode = (quirk(h, NS2D_QUIRK_CONJ_STATE) || src_is_state) ? 1 : 0;
    a.conj_src = (const C*)src;
    a.conj_stride = h->ldc;
    launch_col<Real>(h, COL_RHS, a);
    CKL(h);
    return NS2D_OK;
}

// RK5DPStep (Solver/src/solver.c:360-570) as the reference intends it: seven
// stages k_s = N(X_s) - D X_s with X_s = y0 + dt sum_r a_sr k_r (Butcher table
// of solver.c:33-42), y5 into the state, and the RMS of the embedded error
// scaled by DP_ABS_TOL + DP_REL_TOL max(|y0|, |y5|) (data_types.h:137-141).
// The shipped code does not compile (it names run_data->w_hat_last and reads an
// uninitialised err_sum); this is the corrected form.
template <typename Real>
ns2d_status dp5_step_impl(ns2d_handle* h, double dt, double* err) {
    using C = Cplx<Real>;
    static const double A[6][6] = {
        {0.2, 0, 0, 0, 0, 0},
        {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0},
        {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
        {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
        {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
        {35.0 / 384.0, 0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
    if (!h->dp[0]) {
        for (void*& p : h->dp) {
            CK(h, cudaMalloc(&p, h->field_bytes));
            CK(h, cudaMemsetAsync(p, 0, h->field_bytes, h->stream));
        }
        CK(h, cudaMalloc((void**)&h->dp_kptr, sizeof(void*) * 7));
        CK(h, cudaMemcpy((void*)h->dp_kptr, h->dp, sizeof(void*) * 7, cudaMemcpyHostToDevice));
    }
    compute_forcing(h, dt);
    const bool euler = h->p.system == NS2D_EULER;
    const int branch = euler ? 4 : resolve_branch(h, false);
    void* y0 = h->dp[7];
    void* x = h->dp[8];
    CK(h, cudaMemcpyAsync(y0, h->state, h->field_bytes, cudaMemcpyDeviceToDevice, h->stream));
    for (int s = 0; s < 7; ++s) {
        const void* xs = y0;
        if (s > 0) {
            DpCoef cf{};
            cf.n = s;
            for (int r = 0; r < s; ++r) cf.c[r] = A[s - 1][r];
            const C* k[6];
            for (int r = 0; r < 6; ++r) k[r] = (const C*)h->dp[r];
            dp_combine_kernel<Real><<<296, 256, 0, h->stream>>>((C*)x, (const C*)y0, k[0], k[1], k[2], k[3], k[4],
                                                               k[5], cf, dt, h->nx, h->nyf, h->ldc);
            h->launches++;
            xs = x;
        }
        ColArgs<Real> a;
        fill_common<Real>(h, a, branch);
        a.src = (const C*)xs;
        launch_col<Real>(h, COL_P1, a);
        launch_row<Real>(h);
        fill_common<Real>(h, a, branch);
        a.src = (const C*)h->nl;
        a.rhs_store = (C*)h->dp[s];
        a.conj_mode = 0;
        a.lin_stage = euler ? 0 : 2;
        a.xin = (const C*)xs;
        launch_col<Real>(h, COL_RHS, a);
    }
    DpCoef b5{}, b4{};
    const double B5[7] = {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0.0};
    const double B4[7] = {5179.0 / 57600.0, 0.0, 7571.0 / 16695.0, 393.0 / 640.0, -92097.0 / 339200.0,
                          187.0 / 2100.0, 1.0 / 40.0};
    for (int r = 0; r < 7; ++r) {
        b5.c[r] = B5[r];
        b4.c[r] = B4[r];
    }
    b5.n = b4.n = 7;
    dp_final_kernel<Real><<<296, 256, 0, h->stream>>>((C*)h->state, (const C*)y0, (const C* const*)h->dp_kptr, b5, b4,
                                                     dt, 1e-7, 1e-7, h->nx, h->nyf, h->ldc, h->dpart);
    h->launches++;
    CKL(h);
    double part[296];
    CK(h, cudaMemcpyAsync(part, h->dpart, sizeof(part), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    double sum = 0.0;
    for (int b = 0; b < 296; ++b) sum += part[b];
    *err = std::sqrt(sum / (double)(h->nx * h->nyf));
    return NS2D_OK;
}

// RK5DPStep (Solver/src/solver.c:360-570) as the reference writes it, with the
// three defects that stop it compiling fixed (err_sum starts at 0, one surplus
// parenthesis, w_hat_last read from Int_data): the stages use the table of
// :35-43 (a32 = 0.5) on the nonlinear term alone, each stage input is the live
// state plus dt sum a k, every RHS evaluation applies the ForceConjugacy side
// effect to the state, the update takes Crank-Nicolson factors on the
// fifth-order sum, and for iters > 1 the error norm is the RMS of the real
// parts scaled by the state of the previous error step.
template <typename Real>
ns2d_status rk5dp_step_impl(ns2d_handle* h, double dt, int iters, double* err) {
    using C = Cplx<Real>;
    static const double A[6][6] = {
        {0.2, 0, 0, 0, 0, 0},
        {3.0 / 40.0, 0.5, 0, 0, 0, 0},
        {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
        {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
        {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
        {35.0 / 384.0, 0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
    if (!h->dp[0]) {
        for (void*& p : h->dp) {
            CK(h, cudaMalloc(&p, h->field_bytes));
            CK(h, cudaMemsetAsync(p, 0, h->field_bytes, h->stream));
        }
        CK(h, cudaMalloc((void**)&h->dp_kptr, sizeof(void*) * 7));
        CK(h, cudaMemcpy((void*)h->dp_kptr, h->dp, sizeof(void*) * 7, cudaMemcpyHostToDevice));
    }
    if (!h->dp_last) {
        CK(h, cudaMalloc(&h->dp_last, h->field_bytes));
        CK(h, cudaMemsetAsync(h->dp_last, 0, h->field_bytes, h->stream));
    }
    compute_forcing(h, dt);
    const bool euler = h->p.system == NS2D_EULER;
    const int branch = euler ? 4 : resolve_branch(h, false);
    const bool conj_quirk = quirk(h, NS2D_QUIRK_CONJ_STATE);
    void* x = h->dp[8];
    for (int s = 0; s < 7; ++s) {
        const void* xs = h->state;
        if (s > 0) {
            DpCoef cf{};
            cf.n = s;
            for (int r = 0; r < s; ++r) cf.c[r] = dt * A[s - 1][r];
            const C* k[6];
            for (int r = 0; r < 6; ++r) k[r] = (const C*)h->dp[r];
            dpw_combine_kernel<Real><<<296, 256, 0, h->stream>>>((C*)x, (const C*)h->state, k[0], k[1], k[2], k[3],
                                                                k[4], k[5], cf, h->nx, h->nyf, h->ldc);
            h->launches++;
            xs = x;
        }
        ColArgs<Real> a;
        fill_common<Real>(h, a, branch);
        a.src = (const C*)xs;
        launch_col<Real>(h, COL_P1, a);
        launch_row<Real>(h);
        fill_common<Real>(h, a, branch);
        a.src = (const C*)h->nl;
        a.rhs_store = (C*)h->dp[s];
        // NonlinearRHSBatch ends with ForceConjugacy of its input (solver.c:1031)
        a.conj_mode = (conj_quirk || s == 0) ? 1 : 0;
        a.conj_src = (const C*)xs;
        a.conj_stride = h->ldc;
        a.lin_stage = 0;
        launch_col<Real>(h, COL_RHS, a);
    }
    DpCoef b5{}, bs{};
    const double B5[7] = {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0.0};
    const double BS[7] = {5179.0 / 57600.0, 0.0, 7571.0 / 16695.0, 393.0 / 640.0, -92097.0 / 339200.0,
                          187.0 / 2100.0, 1.0 / 40.0};
    for (int r = 0; r < 7; ++r) {
        b5.c[r] = B5[r];
        bs.c[r] = BS[r];
    }
    b5.n = bs.n = 7;
    dpw_final_kernel<Real><<<296, 256, 0, h->stream>>>((C*)h->state, (C*)h->dp_last, (const C* const*)h->dp_kptr, b5,
                                                      bs, dt, euler ? 1 : 0, make_lin(h, branch), iters, h->nx,
                                                      h->nyf, h->ldc, h->dpart);
    h->launches++;
    CKL(h);
    if (iters > 1) {
        double part[296];
        CK(h, cudaMemcpyAsync(part, h->dpart, sizeof(part), cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        double sum = 0.0;
        for (int b = 0; b < 296; ++b) sum += part[b];
        h->dp_err = std::sqrt(1.0 / (double)((long)h->nx * (long)h->nyf) * sum);
    }
    *err = h->dp_err;
    return NS2D_OK;
}

// c2r of up to two spectral fields to x-space (f[0], f[1]) followed by a row
// pass with a reduction or a store.
template <typename Real>
ns2d_status c2r_impl(ns2d_handle* h, const InvField<Real>* fields, int nf, int op, double* outA, double* outB,
                     double* result, double scale = 0.0) {
    using C = Cplx<Real>;
    InvArgs<Real> ia;
    std::memset(&ia, 0, sizeof(ia));
    for (int k = 0; k < nf; ++k) {
        ia.f[k] = fields[k];
        ia.f[k].dst = (C*)h->f[k];
    }
    ia.nf = nf;
    ia.nyf = h->nyf;
    ia.ldc = h->ldc;
    ia.tw = (const C*)h->tw;
    with_size<Real>(h->nx, [&](auto L) { decltype(L)::col_inv(ia, h->stream); });
    h->launches++;
    RowC2RArgs<Real> ra;
    std::memset(&ra, 0, sizeof(ra));
    ra.A = (const C*)h->f[0];
    ra.B = nf > 1 ? (const C*)h->f[1] : nullptr;
    ra.ldc = h->ldc;
    ra.tw = (const C*)h->tw;
    ra.scale = scale != 0.0 ? scale : 1.0 / (double)(h->nx * h->ny);
    ra.dx = 2.0 * M_PI / (double)h->nx;
    ra.dy = 2.0 * M_PI / (double)h->ny;
    ra.maxbits = h->dmax;
    ra.outA = outA;
    ra.outB = outB;
    if (op != R2_STORE) CK(h, cudaMemsetAsync(h->dmax, 0, sizeof(unsigned long long), h->stream));
    with_size<Real>(h->nx, [&](auto L) { decltype(L)::row_c2r(op, ra, h->stream); });
    h->launches++;
    CKL(h);
    if (result) {
        unsigned long long bits = 0;
        CK(h, cudaMemcpyAsync(&bits, h->dmax, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        double v;
        std::memcpy(&v, &bits, sizeof(v));
        *result = v;
    }
    return NS2D_OK;
}

// Velocity of the state into the persistent reference-layout u_hat buffer
// (regular or CFL-quirk row index), then c2r with a max reduction.
template <typename Real>
ns2d_status velocity_c2r(ns2d_handle* h, int scrambled, int op, double* result) {
    using C = Cplx<Real>;
    cfl_scramble_kernel<Real><<<296, 256, 0, h->stream>>>((const C*)h->state, h->ldc, (C*)h->uhat_ref, h->nx, h->ny,
                                                          scrambled);
    h->launches++;
    CKL(h);
    InvField<Real> f[2];
    std::memset(f, 0, sizeof(f));
    for (int k = 0; k < 2; ++k) {
        f[k].p = (const C*)h->uhat_ref + k;
        f[k].rs = 2LL * h->nyf;
        f[k].es = 2;
        f[k].op = 0;
    }
    return c2r_impl<Real>(h, f, 2, op, nullptr, nullptr, result);
}

template <typename Real>
ns2d_status max_data_impl(ns2d_handle* h, int kind, double* out) {
    using C = Cplx<Real>;
    InvField<Real> f[2];
    std::memset(f, 0, sizeof(f));
    if (kind == NS2D_MAX_VORT) {
        f[0].p = (const C*)h->state;
        f[0].rs = h->ldc;
        f[0].es = 1;
        f[0].op = 0;
        return c2r_impl<Real>(h, f, 1, R2_MAXABS, nullptr, nullptr, out);
    }
    if (kind == NS2D_MAX_VEL) {
        // run_data->u_hat is rewritten with the regular index (solver.c:2184-2196);
        // the CFL path later reads the entries its own index misses.
        return velocity_c2r<Real>(h, 0, R2_MAXABS, out);
    }
    return fail(h, NS2D_ERR_UNSUPPORTED, "NS2D_MAX_VORT_FOUR is evaluated by ns2d_get_max_data on the host copy");
}

template <typename Real>
ns2d_status cfl_impl(ns2d_handle* h, double* scales_convect) {
    return velocity_c2r<Real>(h, quirk(h, NS2D_QUIRK_CFL_INDEX) ? 1 : 0, R2_CFL, scales_convect);
}
template <typename Real>
void fill_twiddles(std::vector<Cplx<Real>>& tw, int n) {
    tw.resize(n);
    for (int m = 0; m < n; ++m) {
        long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
        tw[m].x = (Real)cosl(a);
        tw[m].y = (Real)(-sinl(a));
    }
}

void free_all(ns2d_handle* h) {
    void* ptrs[] = {h->state, h->acc, h->nl, h->f[0], h->f[1], h->f[2], h->f[3], h->tmpfull, h->col0[0], h->col0[1],
                    h->tw, h->rhsbuf, h->ab[0], h->ab[1], h->ab[2], h->ab[3], h->uhat_ref, h->dreal, h->dscal, h->dmax,
                    h->dstatus, h->dio, h->ddiag, h->dpart, h->cn, h->dp_last};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (void* p : h->dp)
        if (p) cudaFree(p);
    void* fp[] = {h->ffield, h->fidx, h->fval};
    for (void* p : fp)
        if (p) cudaFree(p);
    if (h->dp_kptr) cudaFree((void*)h->dp_kptr);
    delete static_cast<ColMaps*>(h->col_maps);
    h->col_maps = nullptr;
}

template <typename Real>
ns2d_status create_impl(ns2d_handle* h) {
    using C = Cplx<Real>;
    const size_t fb = h->field_bytes;
    void** fields[] = {&h->state, &h->acc,   &h->nl,    &h->f[0],  &h->f[1],  &h->f[2], &h->f[3],
                       &h->tmpfull, &h->rhsbuf, &h->ab[0], &h->ab[1], &h->ab[2], &h->ab[3]};
    for (void** p : fields) {
        CK(h, cudaMalloc(p, fb));
        CK(h, cudaMemsetAsync(*p, 0, fb, h->stream));
    }
    for (int k = 0; k < 2; ++k) {
        CK(h, cudaMalloc(&h->col0[k], sizeof(C) * h->nx));
        CK(h, cudaMemsetAsync(h->col0[k], 0, sizeof(C) * h->nx, h->stream));
    }
    const size_t uref = sizeof(C) * 2 * (size_t)h->nx * h->nyf;
    CK(h, cudaMalloc(&h->uhat_ref, uref));
    CK(h, cudaMemsetAsync(h->uhat_ref, 0, uref, h->stream));
    CK(h, cudaMalloc(&h->dreal, sizeof(double) * (size_t)h->nx * h->ny));
    CK(h, cudaMalloc(&h->dscal, sizeof(double) * 4));
    CK(h, cudaMemsetAsync(h->dscal, 0, sizeof(double) * 4, h->stream));
    CK(h, cudaMalloc(&h->dmax, sizeof(unsigned long long) * 2));
    CK(h, cudaMalloc(&h->dstatus, sizeof(int) * 4));
    CK(h, cudaMemsetAsync(h->dstatus, 0, sizeof(int) * 4, h->stream));
    CK(h, cudaMalloc(&h->dio, sizeof(double2) * (size_t)h->nx * h->nyf));
    CK(h, cudaMalloc(&h->ddiag, sizeof(double) * (DG_N + 8 * (size_t)h->n_spect)));
    CK(h, cudaMalloc(&h->dpart, sizeof(double) * 4096));
    CK(h, cudaMalloc(&h->cn, sizeof(double2) * (size_t)h->nx * h->ldc));
    build_col_maps<Real>(h);
    CK(h, cudaFuncSetAttribute((const void*)diag_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(sizeof(double) * (8 * (size_t)h->n_spect + DG_N * 8))));
    std::vector<C> tw;
    fill_twiddles<Real>(tw, h->nx);
    CK(h, cudaMalloc(&h->tw, sizeof(C) * h->nx));
    CK(h, cudaMemcpy(h->tw, tw.data(), sizeof(C) * h->nx, cudaMemcpyHostToDevice));
    cudaError_t e = cudaSuccess;
    with_size<Real>(h->nx, [&](auto L) { e = decltype(L)::setup(); });
    CK(h, e);
    CK(h, cudaStreamSynchronize(h->stream));
    return NS2D_OK;
}

template <typename Real>
ns2d_status pack_in(ns2d_handle* h, const double2* d_src, void* dst) {
    pack_kernel<Real><<<296, 256, 0, h->stream>>>(d_src, (Cplx<Real>*)dst, h->nx, h->nyf, h->ldc);
    h->launches++;
    CKL(h);
    return NS2D_OK;
}
template <typename Real>
ns2d_status unpack_out(ns2d_handle* h, const void* src, double2* d_dst) {
    unpack_kernel<Real><<<296, 256, 0, h->stream>>>((const Cplx<Real>*)src, d_dst, h->nx, h->nyf, h->ldc);
    h->launches++;
    CKL(h);
    return NS2D_OK;
}

#define DISPATCH(h, fn, ...) ((h)->fp32 ? fn<float>(__VA_ARGS__) : fn<double>(__VA_ARGS__))

void drop_graph(ns2d_handle* h) {
    if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
    h->step_graph = nullptr;
    h->graph_branch = -1;
    if (h->timed_graph) cudaGraphExecDestroy(h->timed_graph);
    h->timed_graph = nullptr;
    h->timed_branch = -1;

}

// Captures the launches of one RK4/RK4CN step (recorded, not executed).
ns2d_status capture_step(ns2d_handle* h, double dt, cudaGraphExec_t* out) {
    const int64_t l0 = h->launches;
    cudaGraph_t g = nullptr;
    CK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    ns2d_status s = DISPATCH(h, rk4_step_impl, h, dt, nullptr);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->graph_kernels = (int)(h->launches - l0);
    h->launches = l0;
    if (s) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return fail(h, NS2D_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *out = nullptr;
        return fail(h, NS2D_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    return NS2D_OK;
}

// One fixed-dt RK4/RK4CN step for the time loops (ns2d_step_n, ns2d_step_async,
// the adjoint's record).  The first step with a given dt runs eagerly (it
// settles the operator branch and the CN table); the step is then captured
// once as a CUDA graph of its nine launches and replayed for the following
// steps.  With kernel timing on, a second graph carries an event pair around
// every launch and is read back after each replay.  Stage capture for the
// adjoint uses the eager form.
ns2d_status rk4_step_loop(ns2d_handle* h, double dt) {
    if (h->cap_step) return DISPATCH(h, rk4_step_impl, h, dt, nullptr);
    int hf = h->hyper_flag;
    const int branch = (h->p.system == NS2D_EULER && h->p.integrator != NS2D_RK4)
                           ? 4
                           : ns2d::resolve_branch(hf, h->p.ekmn_drag_flag, quirk(h, NS2D_QUIRK_HYPER_LATCH));
    const bool settled = (hf == h->hyper_flag) && h->cn_dt == dt && h->cn_branch == branch;
    cudaGraphExec_t* gx = h->timing ? &h->timed_graph : &h->step_graph;
    double* gdt = h->timing ? &h->timed_dt : &h->graph_dt;
    int* gbr = h->timing ? &h->timed_branch : &h->graph_branch;
    const int set = h->timing ? 1 : 0;
    if (!(*gx && *gdt == dt && *gbr == branch && settled)) {
        if (*gx) cudaGraphExecDestroy(*gx);
        *gx = nullptr;
        ns2d_status s = DISPATCH(h, rk4_step_impl, h, dt, nullptr);  // this call's step
        if (s) return s;
        h->capturing_timed = h->timing;
        h->gev_n = 0;
        h->gev_set = set;
        s = capture_step(h, dt, gx);
        h->capturing_timed = false;
        if (s) return s;
        h->gev_n_of[set] = h->gev_n;
        *gdt = dt;
        *gbr = h->cn_branch;
        return NS2D_OK;
    }
    cudaError_t e = cudaGraphLaunch(*gx, h->stream);
    if (e != cudaSuccess) return fail(h, NS2D_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
    h->launches += h->graph_kernels;
    if (h->timing) {
        CK(h, cudaStreamSynchronize(h->stream));
        for (int k = 0; k < h->gev_n_of[set]; ++k) {
            float ms = 0.f;
            CK(h, cudaEventElapsedTime(&ms, h->gev_g[set][k][0], h->gev_g[set][k][1]));
            h->t_ms[h->gev_cls_g[set][k]] += ms;
            h->t_n[h->gev_cls_g[set][k]] += 1;
        }
    }
    return NS2D_OK;
}

// One step for the per-call entry points (ns2d_rk4_step, ns2d_rk4_step_host):
// eager when dt differs from the previous call's (adaptive stepping would
// recapture every step), the graph-replayed step of the time loops when the
// same dt comes again.  Both run the same kernels on the same arguments.
ns2d_status single_step(ns2d_handle* h, double dt) {
    const bool again = (h->last_call_dt == dt);
    h->last_call_dt = dt;
    if (again) return rk4_step_loop(h, dt);
    return DISPATCH(h, rk4_step_impl, h, dt, nullptr);
}

// Host arrays in the reference layout [nx][ny/2+1] complex128 to and from an
// internal [nx][ldc] field.  FP64: one strided copy into the padded rows;
// FP32: through the staging buffer and a converting kernel.
ns2d_status host_to_state(ns2d_handle* h, const double* host, void* dst) {
    if (!h->fp32) {
        CK(h, cudaMemcpy2DAsync(dst, sizeof(double2) * (size_t)h->ldc, host, sizeof(double2) * (size_t)h->nyf,
                                sizeof(double2) * (size_t)h->nyf, (size_t)h->nx, cudaMemcpyHostToDevice, h->stream));
        return NS2D_OK;
    }
    CK(h, cudaMemcpyAsync(h->dio, host, sizeof(double2) * (size_t)h->nx * h->nyf, cudaMemcpyHostToDevice, h->stream));
    return DISPATCH(h, pack_in, h, h->dio, dst);
}
ns2d_status state_to_host(ns2d_handle* h, const void* src, double* host) {
    if (!h->fp32) {
        CK(h, cudaMemcpy2DAsync(host, sizeof(double2) * (size_t)h->nyf, src, sizeof(double2) * (size_t)h->ldc,
                                sizeof(double2) * (size_t)h->nyf, (size_t)h->nx, cudaMemcpyDeviceToHost, h->stream));
    } else {
        ns2d_status s = DISPATCH(h, unpack_out, h, src, h->dio);
        if (s) return s;
        CK(h, cudaMemcpyAsync(host, h->dio, sizeof(double2) * (size_t)h->nx * h->nyf, cudaMemcpyDeviceToHost, h->stream));
    }
    CK(h, cudaStreamSynchronize(h->stream));
    return NS2D_OK;
}

// Unnormalised r2c of a host [nx][ny] real field to a host half spectrum.
template <typename Real>
ns2d_status r2c_host_impl(ns2d_handle* h, const double* real, double* spec) {
    using C = Cplx<Real>;
    CK(h, cudaMemcpyAsync(h->dreal, real, sizeof(double) * (size_t)h->nx * h->ny, cudaMemcpyHostToDevice, h->stream));
    with_size<Real>(h->nx, [&](auto L) {
        decltype(L)::fwd(FWD_ROWS, h->dreal, nullptr, (C*)h->f[0], h->nx, h->ldc, (const C*)h->tw, h->stream);
        decltype(L)::fwd(FWD_COLS, nullptr, (const C*)h->f[0], (C*)h->f[1], h->nyf, h->ldc, (const C*)h->tw,
                         h->stream);
    });
    h->launches += 2;
    CKL(h);
    return state_to_host(h, h->f[1], spec);
}

// Unnormalised c2r of a host half spectrum to a host [nx][ny] real field.
template <typename Real>
ns2d_status c2r_host_impl(ns2d_handle* h, const double* spec, double* real) {
    ns2d_status s = host_to_state(h, spec, h->f[2]);
    if (s) return s;
    InvField<Real> f[1];
    std::memset(f, 0, sizeof(f));
    f[0].p = (const Cplx<Real>*)h->f[2];
    f[0].rs = h->ldc;
    f[0].es = 1;
    if ((s = c2r_impl<Real>(h, f, 1, R2_STORE, h->dreal, nullptr, nullptr, 1.0))) return s;
    CK(h, cudaMemcpyAsync(real, h->dreal, sizeof(double) * (size_t)h->nx * h->ny, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return NS2D_OK;
}

template <typename Real>
ns2d_status mean_flow_impl(ns2d_handle* h, double* mean_x, double* mean_y) {
    mean_flow_kernel<Real><<<h->nx + h->nyf, 256, 0, h->stream>>>((const Cplx<Real>*)h->state, h->nx, h->nyf, h->ldc,
                                                                h->dpart);
    h->launches++;
    CKL(h);
    std::vector<double> buf((size_t)h->nx + h->nyf);
    CK(h, cudaMemcpyAsync(buf.data(), h->dpart, sizeof(double) * buf.size(), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (mean_y) std::memcpy(mean_y, buf.data(), sizeof(double) * h->nx);
    if (mean_x) std::memcpy(mean_x, buf.data() + h->nx, sizeof(double) * h->nyf);
    return NS2D_OK;
}

ns2d_status read_status(ns2d_handle* h, int* bits, int* steps) {
    int st[2];
    CK(h, cudaMemcpyAsync(st, h->dstatus, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    *bits = st[0];
    if (steps) *steps = st[1];
    return NS2D_OK;
}

ns2d_status clear_status(ns2d_handle* h) {
    CK(h, cudaMemsetAsync(h->dstatus, 0, sizeof(int) * 2, h->stream));
    CK(h, cudaMemsetAsync(h->dscal, 0, sizeof(double) * 2, h->stream));
    return NS2D_OK;
}

// After a batch of steps: turn status bits into SystemCheck results.
ns2d_status check_status(ns2d_handle* h) {
    int bits = 0;
    ns2d_status s = read_status(h, &bits, nullptr);
    if (s) return s;
    if (bits & 8) return fail(h, NS2D_ERR_CUDA, "a column pass waited past its bound for its tile loads");
    if (bits & 1) return fail(h, NS2D_ERR_BLOWUP, "non-finite vorticity (SystemCheck)");
    if (bits & 2) {
        // exact max|w| (GetMaxData("VORT"))
        if ((s = clear_status(h))) return s;
        double wmax = 0.0;
        if ((s = DISPATCH(h, max_data_impl, h, NS2D_MAX_VORT, &wmax))) return s;
        if (!(wmax < 1e100)) return fail(h, NS2D_ERR_BLOWUP, "max vorticity reached 1e100 (SystemCheck)");
    }
    return NS2D_OK;
}


// ComputeSystemMeasurables (Solver/src/sys_msr.c:32-373) with the stock dataset
// flags; the RHS of the state is evaluated first when flux_diagnostics is set,
// with its conjugacy side effect on the state, as in the reference (:127).
template <typename Real>
ns2d_status measurables_impl(ns2d_handle* h, ns2d_measures* out, double* spectra) {
    using C = Cplx<Real>;
    ns2d_status s;
    const C* rhs = nullptr;
    if (h->p.flux_diagnostics) {
        if ((s = rhs_impl<Real>(h, h->state, true))) return s;
        rhs = (const C*)h->rhsbuf;
    }
    const int ns = h->n_spect;
    const size_t nout = DG_N + 8 * (size_t)ns;
    CK(h, cudaMemsetAsync(h->ddiag, 0, sizeof(double) * nout, h->stream));
    DiagArgs<Real> d;
    std::memset(&d, 0, sizeof(d));
    d.state = (const C*)h->state;
    d.rhs = rhs;
    d.ldc = h->ldc;
    d.nx = h->nx;
    d.ny = h->ny;
    d.nyf = h->nyf;
    int hyper = h->hyper_flag;
    {
        const int drag = h->p.ekmn_drag_flag;
        int br = (hyper == 1 && drag == 1) ? 1 : (hyper != 1 && drag == 1) ? 2 : (hyper == 1) ? 3 : 4;
        d.lin = make_lin(h, br);
    }
    d.enst_quirk = quirk(h, NS2D_QUIRK_ENST_DISS) ? 1 : 0;
    d.force_i = h->force_i;
    d.force_j = h->force_j;
    d.fre = h->fre;
    d.fim = h->fim;
    d.has_force = h->forced ? 1 : 0;
    d.ffield = h->ffield_on ? (const C*)h->ffield : nullptr;
    d.n_spect = ns;
    d.out = h->ddiag;
    const size_t smem = sizeof(double) * (8 * (size_t)ns + DG_N * 8);
    diag_kernel<Real><<<148, 256, smem, h->stream>>>(d);
    h->launches++;
    CKL(h);
    std::vector<double> raw(nout);
    CK(h, cudaMemcpyAsync(raw.data(), h->ddiag, sizeof(double) * nout, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    const double norm_fac = 0.5 / std::pow((double)(h->nx * h->ny), 2.0);
    const double const_fac = 4.0 * std::pow(M_PI, 2.0);
    const double cn = const_fac * norm_fac;
    if (out) {
        out->energy = raw[DG_E] * cn;
        out->enstrophy = raw[DG_Z] * cn;
        out->palinstrophy = raw[DG_P] * cn;
        out->forcing_input = raw[DG_FORC] * cn;
        out->divergence = raw[DG_DIV] * cn;
        out->energy_diss = raw[DG_EDISS] * (2.0 * const_fac * norm_fac);
        out->enstrophy_diss = raw[DG_ZDISS] * (2.0 * const_fac * norm_fac);
        out->d_enrg_dt_sbst = raw[DG_DE];
        out->enrg_flux_sbst = raw[DG_EFLUX] * cn;
        out->enrg_diss_sbst = raw[DG_EDSB] * (2.0 * const_fac * norm_fac);
        out->d_enst_dt_sbst = raw[DG_DZ];
        out->enst_flux_sbst = raw[DG_ZFLUX] * cn;
        out->enst_diss_sbst = raw[DG_ZDSB] * (2.0 * const_fac * norm_fac);
    }
    if (spectra)
        for (size_t q = 0; q < 8 * (size_t)ns; ++q) spectra[q] = raw[DG_N + q] * cn;
    return NS2D_OK;
}

}  // namespace

namespace ns2d {
namespace internal {

ns2d_status fail(ns2d_handle* h, ns2d_status s, const std::string& msg) { return ::fail(h, s, msg); }
ns2d_status rk4_step(ns2d_handle* h, double dt) { return DISPATCH(h, rk4_step_impl, h, dt, nullptr); }
ns2d_status rk4_step_loop(ns2d_handle* h, double dt) { return ::rk4_step_loop(h, dt); }
ns2d_status ensure_cn(ns2d_handle* h, double dt, int branch) { return ::ensure_cn(h, dt, branch); }
ns2d_status check_status(ns2d_handle* h) { return ::check_status(h); }
ns2d_status pack_in(ns2d_handle* h, const double2* d_src, void* dst) { return DISPATCH(h, ::pack_in, h, d_src, dst); }
ns2d_status unpack_out(ns2d_handle* h, const void* src, double2* d_dst) {
    return DISPATCH(h, ::unpack_out, h, src, d_dst);
}

}  // namespace internal
}  // namespace ns2d

extern "C" {

int ns2d_abi_version(void) { return NS2D_ABI_VERSION; }

const char* ns2d_status_string(ns2d_status s) {
    if ((int)s < 0 || (int)s >= (int)(sizeof(kStatusNames) / sizeof(kStatusNames[0]))) return "NS2D_ERR_UNKNOWN";
    return kStatusNames[s];
}

const char* ns2d_last_error(const ns2d_handle* h) { return h ? h->err.c_str() : "null handle"; }

ns2d_status ns2d_params_default(ns2d_params* p) {
    if (!p) return NS2D_ERR_INVALID;
    std::memset(p, 0, sizeof(*p));
    p->nx = p->ny = 64;
    p->system = NS2D_NAVIER;
    p->integrator = NS2D_RK4CN;
    p->dealias = NS2D_DEALIAS_23;
    p->forcing = NS2D_FORCING_NONE;
    p->force_k = 0;
    p->quirks = NS2D_QUIRKS_REFERENCE;
    p->force_scale = 1.0;
    p->nu = 1e-4;
    p->hyper_visc_pow = 2.0;
    p->ekmn_alpha = 0.0;
    p->ekmn_drag_pow = -2.0;
    p->hyper_visc_flag = 0;
    p->ekmn_drag_flag = 0;
    p->adapt_step_flag = 0;
    p->cfl_cond_flag = 1;
    p->cfl_const = 0.9;
    p->dt = 1e-4;
    p->precision = NS2D_FP64;
    p->flux_diagnostics = 1;
    p->device = 0;
    return NS2D_OK;
}

ns2d_status ns2d_create(const ns2d_params* p, ns2d_handle** out) {
    if (!p || !out) return NS2D_ERR_INVALID;
    *out = nullptr;
    if (p->nx != p->ny) return NS2D_ERR_UNSUPPORTED;
    if (!is_pow2(p->nx) || p->nx < 16 || p->nx > 2048) return NS2D_ERR_UNSUPPORTED;
    if (p->integrator < 0 || p->integrator > 3 || p->dealias < 0 || p->dealias > 1 || p->forcing < 0 ||
        p->forcing > 2 || (p->precision != NS2D_FP64 && p->precision != NS2D_FP32) || p->dealias_edge < 0 ||
        p->dealias_edge > 1 || p->model < 0 || p->model > 1)
        return NS2D_ERR_INVALID;
    // phase-only: RK4Step's reset only (solver.c:822-857)
    if (p->model == NS2D_MODEL_PHASE_ONLY && p->integrator != NS2D_RK4CN && p->integrator != NS2D_RK4)
        return NS2D_ERR_UNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return NS2D_ERR_NO_DEVICE;
    if (p->device < 0 || p->device >= ndev) return NS2D_ERR_INVALID;
    ns2d_handle* h = new (std::nothrow) ns2d_handle();
    if (!h) return NS2D_ERR_NOMEM;
    h->p = *p;
    h->nx = p->nx;
    h->ny = p->ny;
    h->nyf = p->ny / 2 + 1;
    h->ldc = (h->nyf + 3) & ~3;
    h->fp32 = p->precision == NS2D_FP32;
    h->elem = h->fp32 ? sizeof(float2) : sizeof(double2);
    h->field_bytes = (size_t)h->nx * h->ldc * h->elem;
    h->hyper_flag = p->hyper_visc_flag;
    // KOLM forcing: one mode at flat index force_k of the [nx][nyf] array (force.c:93-100)
    if (p->forcing == NS2D_FORCING_KOLM) {
        h->forced = true;
        h->force_i = p->force_k / h->nyf;
        h->force_j = p->force_k % h->nyf;
        if (h->force_i >= h->nx) {
            delete h;
            return NS2D_ERR_INVALID;
        }
    }
    h->n_spect = (int)std::round(std::sqrt((double)(h->nx / 2.0) * (h->nx / 2.0) + (double)(h->ny / 2.0) * (h->ny / 2.0)) + 1);
    ns2d_status s;
    if (cudaSetDevice(p->device) != cudaSuccess || cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return NS2D_ERR_CUDA;
    }
    h->stream = h->own;
    s = DISPATCH(h, create_impl, h);
    if (s != NS2D_OK) {
        std::fprintf(stderr, "ns2d_create: %s\n", h->err.c_str());
        free_all(h);
        cudaStreamDestroy(h->own);
        delete h;
        return s;
    }
    *out = h;
    return NS2D_OK;
}

ns2d_status ns2d_destroy(ns2d_handle* h) {
    if (!h) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    cudaStreamSynchronize(h->stream);
    drop_graph(h);
    for (auto& set : h->gev_g)
        for (auto& pair : set)
            for (cudaEvent_t e : pair)
                if (e) cudaEventDestroy(e);
    internal::adjoint_free(h);
    free_all(h);
    for (auto e : h->ev_pool) cudaEventDestroy(e);
    for (auto& e : h->ev_open) {
        cudaEventDestroy(e.second.first);
        cudaEventDestroy(e.second.second);
    }
    cudaStreamDestroy(h->own);
    delete h;
    return NS2D_OK;
}

ns2d_status ns2d_dims(const ns2d_handle* h, int32_t* nx, int32_t* ny, int32_t* nyf, int32_t* n_spect) {
    if (!h) return NS2D_ERR_INVALID;
    if (nx) *nx = h->nx;
    if (ny) *ny = h->ny;
    if (nyf) *nyf = h->nyf;
    if (n_spect) *n_spect = h->n_spect;
    return NS2D_OK;
}

ns2d_status ns2d_set_w_hat(ns2d_handle* h, const double* w_hat) {
    if (!h || !w_hat) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s = host_to_state(h, w_hat, h->state);
    if (s) return s;
    s = clear_status(h);
    if (s) return s;
    h->ab_count = 0;
    // w_max_init (InitialConditions, solver.c:2003)
    return DISPATCH(h, max_data_impl, h, NS2D_MAX_VORT, &h->w_max_init);
}

ns2d_status ns2d_get_w_hat(ns2d_handle* h, double* w_hat) {
    if (!h || !w_hat) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    return state_to_host(h, h->state, w_hat);
}

ns2d_status ns2d_set_w_hat_device(ns2d_handle* h, const double* d_w_hat) {
    if (!h || !d_w_hat) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s = DISPATCH(h, pack_in, h, (const double2*)d_w_hat, h->state);
    if (s) return s;
    s = clear_status(h);
    if (s) return s;
    h->ab_count = 0;
    return DISPATCH(h, max_data_impl, h, NS2D_MAX_VORT, &h->w_max_init);
}

ns2d_status ns2d_get_w_hat_device(ns2d_handle* h, double* d_w_hat) {
    if (!h || !d_w_hat) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    return DISPATCH(h, unpack_out, h, h->state, (double2*)d_w_hat);
}

ns2d_status ns2d_compute_forcing(ns2d_handle* h, double dt) {
    if (!h) return NS2D_ERR_INVALID;
    compute_forcing(h, dt);
    return NS2D_OK;
}

ns2d_status ns2d_nonlinear_rhs(ns2d_handle* h, const double* in, double* out) {
    if (!h || !out) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s;
    const void* src = h->state;
    if (in) {
        if ((s = host_to_state(h, in, h->tmpfull))) return s;
        src = h->tmpfull;
    }
    if ((s = DISPATCH(h, rhs_impl, h, src, in == nullptr))) return s;
    return state_to_host(h, h->rhsbuf, out);
}

ns2d_status ns2d_rk4_step(ns2d_handle* h, double dt) {
    if (!h) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s = single_step(h, dt);
    if (s) return s;
    return check_status(h);
}

ns2d_status ns2d_ab4_step(ns2d_handle* h, double dt, int32_t iters) {
    if (!h || iters < 1) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    if (h->p.model != NS2D_MODEL_FULL) return fail(h, NS2D_ERR_UNSUPPORTED, "AB4Step has no phase-only form");
    ns2d_status s;
    if (iters <= 3) {
        // start-up: RK4CN step storing RK1 in AB_tmp_nonlin[iters-1] (solver.c:276-284)
        if (h->ab_count != iters - 1) return fail(h, NS2D_ERR_STATE, "AB4 start-up steps must be 1, 2, 3 in order");
        ns2d_params saved = h->p;
        h->p.integrator = NS2D_RK4CN;
        s = DISPATCH(h, rk4_step_impl, h, dt, h->ab[iters - 1]);
        h->p = saved;
        if (s) return s;
        h->ab_count = iters;
    } else {
        if (h->ab_count < 3) return fail(h, NS2D_ERR_STATE, "AB4 needs three start-up steps first");
        s = DISPATCH(h, ab4_update_impl, h, dt);
        if (s) return s;
    }
    return check_status(h);
}

ns2d_status ns2d_step_n(ns2d_handle* h, int32_t nsteps, double dt) {
    if (!h || nsteps < 0) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    if (h->p.integrator == NS2D_DP5) return fail(h, NS2D_ERR_UNSUPPORTED, "DP5 is advanced by its own entry point");
    int done = 0;
    while (done < nsteps) {
        int bits = 0, steps0 = 0, steps1 = 0;
        ns2d_status s = read_status(h, &bits, &steps0);
        if (s) return s;
        if (bits) {
            if ((s = check_status(h))) return s;
            continue;
        }
        for (int k = done; k < nsteps; ++k) {
            if (h->p.integrator == NS2D_AB4 && h->ab_count < 3) {
                const int it = h->ab_count + 1;
                ns2d_params saved = h->p;
                h->p.integrator = NS2D_RK4CN;
                s = DISPATCH(h, rk4_step_impl, h, dt, h->ab[it - 1]);
                h->p = saved;
                h->ab_count = it;
            } else if (h->p.integrator == NS2D_AB4) {
                s = DISPATCH(h, ab4_update_impl, h, dt);
            } else {
                s = rk4_step_loop(h, dt);
            }
            if (s) return s;
        }
        if ((s = read_status(h, &bits, &steps1))) return s;
        done += steps1 - steps0;
        if (bits && (s = check_status(h))) return s;  // a false alarm is cleared and the loop resumes
    }
    return NS2D_OK;
}

ns2d_status ns2d_apply_dealiasing(ns2d_handle* h, double* arr, int32_t dim) {
    if (!h || !arr || dim < 1 || dim > 2) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    const size_t n = (size_t)h->nx * h->nyf * dim;
    double2* d = nullptr;
    CK(h, cudaMalloc(&d, sizeof(double2) * n));
    CK(h, cudaMemcpy(d, arr, sizeof(double2) * n, cudaMemcpyHostToDevice));
    const int m = (int)(h->nx / 3.0);
    dealias_kernel<double><<<296, 256, 0, h->stream>>>(d, dim, h->nx, h->ny, m * m + h->p.dealias_edge, h->p.dealias,
                                                       quirk(h, NS2D_QUIRK_HOU_LI_INT) ? 1 : 0,
                                                       h->p.forcing == NS2D_FORCING_KOLM ? 1 : 0);
    h->launches++;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(arr, d, sizeof(double2) * n, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(h, NS2D_ERR_CUDA, cudaGetErrorString(e));
    return NS2D_OK;
}

ns2d_status ns2d_force_conjugacy(ns2d_handle* h, const double* arr) {
    if (!h) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s;
    const void* src = h->state;
    if (arr) {
        if ((s = host_to_state(h, arr, h->tmpfull))) return s;
        src = h->tmpfull;
        if (!quirk(h, NS2D_QUIRK_CONJ_STATE)) return NS2D_OK;  // corrected form fixes only its input
    }
    if (h->fp32)
        conj_kernel<float><<<(h->nx + 127) / 128, 128, 0, h->stream>>>((float2*)h->state, h->ldc, (const float2*)src, h->ldc, h->nx);
    else
        conj_kernel<double><<<(h->nx + 127) / 128, 128, 0, h->stream>>>((double2*)h->state, h->ldc, (const double2*)src, h->ldc, h->nx);
    h->launches++;
    CKL(h);
    CK(h, cudaStreamSynchronize(h->stream));
    return NS2D_OK;
}

ns2d_status ns2d_get_max_data(ns2d_handle* h, int32_t kind, double* out) {
    if (!h || !out) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    if (kind == NS2D_MAX_VORT_FOUR) {
        // max |w_hat| over the half spectrum (solver.c:2245-2258)
        double* host = new (std::nothrow) double[2 * (size_t)h->nx * h->nyf];
        if (!host) return NS2D_ERR_NOMEM;
        ns2d_status s = state_to_host(h, h->state, host);
        double m = 0.0;
        for (size_t q = 0; s == NS2D_OK && q < (size_t)h->nx * h->nyf; ++q) {
            double a = std::hypot(host[2 * q], host[2 * q + 1]);
            if (a > m) m = a;
        }
        delete[] host;
        *out = m;
        return s;
    }
    return DISPATCH(h, max_data_impl, h, kind, out);
}

ns2d_status ns2d_get_timestep(ns2d_handle* h, double* dt) {
    if (!h || !dt) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s;
    if (h->p.cfl_cond_flag == 1) {
        double convect = 0.0;
        if ((s = DISPATCH(h, cfl_impl, h, &convect))) return s;
        const double dx = 2.0 * M_PI / (double)h->nx, dy = 2.0 * M_PI / (double)h->ny;
        const double diff = std::pow(M_PI, 2.0) * (h->p.nu / std::pow(dx, 2.0) + h->p.nu / std::pow(dy, 2.0));
        *dt = h->p.cfl_const / (convect + diff);
    } else {
        double w_max = 0.0;
        if ((s = DISPATCH(h, max_data_impl, h, NS2D_MAX_VORT, &w_max))) return s;
        const double dt_new = h->p.dt * (h->w_max_init / w_max);
        *dt = (dt_new > 2.0 * (*dt)) ? 2.0 * (*dt) : dt_new;
    }
    h->min_dt = std::fmin(*dt, h->min_dt);
    h->max_dt = std::fmax(*dt, h->max_dt);
    return NS2D_OK;
}

ns2d_status ns2d_dt_range(const ns2d_handle* h, double* min_dt, double* max_dt) {
    if (!h) return NS2D_ERR_INVALID;
    if (min_dt) *min_dt = h->min_dt;
    if (max_dt) *max_dt = h->max_dt;
    return NS2D_OK;
}

ns2d_status ns2d_set_w_max_init(ns2d_handle* h, double w) {
    if (!h) return NS2D_ERR_INVALID;
    h->w_max_init = w;
    return NS2D_OK;
}

ns2d_status ns2d_system_check(ns2d_handle* h, double dt, int64_t iters) {
    if (!h) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    double w_max = 0.0;
    ns2d_status s = DISPATCH(h, max_data_impl, h, NS2D_MAX_VORT, &w_max);
    if (s) return s;
    if (!(w_max < 1e100)) return fail(h, NS2D_ERR_BLOWUP, "max vorticity reached 1e100");
    if (dt <= 1e-10) return fail(h, NS2D_ERR_DT, "time step below 1e-10");
    if ((double)iters >= 1e12) return fail(h, NS2D_ERR_ITERS, "iteration limit reached");
    return NS2D_OK;
}

ns2d_status ns2d_system_measurables(ns2d_handle* h, ns2d_measures* out, double* spectra) {
    if (!h) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    return DISPATCH(h, measurables_impl, h, out, spectra);
}

ns2d_status ns2d_get_w_real(ns2d_handle* h, double* w) {
    if (!h || !w) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s;
    if (h->fp32) {
        InvField<float> f[1];
        std::memset(f, 0, sizeof(f));
        f[0].p = (const float2*)h->state;
        f[0].rs = h->ldc;
        f[0].es = 1;
        s = c2r_impl<float>(h, f, 1, R2_STORE, h->dreal, nullptr, nullptr);
    } else {
        InvField<double> f[1];
        std::memset(f, 0, sizeof(f));
        f[0].p = (const double2*)h->state;
        f[0].rs = h->ldc;
        f[0].es = 1;
        s = c2r_impl<double>(h, f, 1, R2_STORE, h->dreal, nullptr, nullptr);
    }
    if (s) return s;
    CK(h, cudaMemcpyAsync(w, h->dreal, sizeof(double) * (size_t)h->nx * h->ny, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return NS2D_OK;
}

ns2d_status ns2d_fft_r2c(ns2d_handle* h, const double* real, double* spec) {
    if (!h || !real || !spec) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    return DISPATCH(h, r2c_host_impl, h, real, spec);
}

ns2d_status ns2d_fft_c2r(ns2d_handle* h, const double* spec, double* real) {
    if (!h || !spec || !real) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    return DISPATCH(h, c2r_host_impl, h, spec, real);
}

ns2d_status ns2d_mean_flow(ns2d_handle* h, double* mean_x, double* mean_y) {
    if (!h || (!mean_x && !mean_y)) return NS2D_ERR_INVALID;
    if ((size_t)h->nx + h->nyf > 4096) return fail(h, NS2D_ERR_UNSUPPORTED, "mean flow needs nx + ny/2 + 1 <= 4096");
    cudaSetDevice(h->p.device);
    return DISPATCH(h, mean_flow_impl, h, mean_x, mean_y);
}

ns2d_status ns2d_rk4_step_host(ns2d_handle* h, double* w_hat, double dt) {
    if (!h || !w_hat) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s = host_to_state(h, w_hat, h->state);
    if (s) return s;
    if ((s = single_step(h, dt))) return s;
    if ((s = state_to_host(h, h->state, w_hat))) return s;
    return check_status(h);
}

ns2d_status ns2d_step_async(ns2d_handle* h, int32_t nsteps, double dt) {
    if (!h || nsteps < 0) return NS2D_ERR_INVALID;
    if (h->p.integrator == NS2D_DP5) return fail(h, NS2D_ERR_UNSUPPORTED, "DP5 is advanced by its own entry point");
    cudaSetDevice(h->p.device);
    for (int k = 0; k < nsteps; ++k) {
        ns2d_status s;
        if (h->p.integrator == NS2D_AB4 && h->ab_count < 3) {
            const int it = h->ab_count + 1;
            ns2d_params saved = h->p;
            h->p.integrator = NS2D_RK4CN;
            s = DISPATCH(h, rk4_step_impl, h, dt, h->ab[it - 1]);
            h->p = saved;
            h->ab_count = it;
        } else if (h->p.integrator == NS2D_AB4) {
            s = DISPATCH(h, ab4_update_impl, h, dt);
        } else {
            s = rk4_step_loop(h, dt);
        }
        if (s) return s;
    }
    return NS2D_OK;
}

ns2d_status ns2d_set_forcing_modes(ns2d_handle* h, int32_t n, const int32_t* idx, const double* values) {
    if (!h || n < 0 || (n > 0 && (!idx || !values))) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    const bool was_on = h->ffield_on;
    if (n == 0) {
        h->ffield_on = false;
        if (was_on) drop_graph(h);
        return NS2D_OK;
    }
    const int64_t total = (int64_t)h->nx * h->nyf;
    for (int32_t m = 0; m < n; ++m)
        if (idx[m] < 0 || idx[m] >= total) return fail(h, NS2D_ERR_INVALID, "forcing index outside the half spectrum");
    if (!h->ffield) CK(h, cudaMalloc(&h->ffield, h->field_bytes));
    if (h->fcap < n) {
        if (h->fidx) cudaFree(h->fidx);
        if (h->fval) cudaFree(h->fval);
        h->fidx = nullptr;
        h->fval = nullptr;
        h->fcap = 0;
        CK(h, cudaMalloc((void**)&h->fidx, sizeof(int32_t) * n));
        CK(h, cudaMalloc((void**)&h->fval, sizeof(double2) * n));
        h->fcap = n;
    }
    CK(h, cudaMemsetAsync(h->ffield, 0, h->field_bytes, h->stream));
    CK(h, cudaMemcpyAsync(h->fidx, idx, sizeof(int32_t) * n, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(h->fval, values, sizeof(double2) * n, cudaMemcpyHostToDevice, h->stream));
    const int blocks = std::min(148, (n + 255) / 256);
    if (h->fp32)
        scatter_forcing_kernel<float><<<blocks, 256, 0, h->stream>>>((float2*)h->ffield, h->nyf, h->ldc, h->fidx, h->fval, n);
    else
        scatter_forcing_kernel<double><<<blocks, 256, 0, h->stream>>>((double2*)h->ffield, h->nyf, h->ldc, h->fidx, h->fval, n);
    h->launches++;
    CKL(h);
    CK(h, cudaStreamSynchronize(h->stream));  // the caller's arrays may go away on return
    h->ffield_on = true;
    if (!was_on) drop_graph(h);  // captured steps carry the field pointer only when it is on
    return NS2D_OK;
}

ns2d_status ns2d_dp5_step(ns2d_handle* h, double dt, double* err) {
    if (!h || !err || !(dt > 0.0)) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    if (h->p.model != NS2D_MODEL_FULL) return fail(h, NS2D_ERR_UNSUPPORTED, "the DP5 step has no phase-only form");
    ns2d_status s = DISPATCH(h, dp5_step_impl, h, dt, err);
    if (s) return s;
    return check_status(h);
}

ns2d_status ns2d_rk5dp_step(ns2d_handle* h, double dt, int32_t iters, double* err) {
    if (!h || !err || !(dt > 0.0) || iters < 1) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    if (h->p.model != NS2D_MODEL_FULL) return fail(h, NS2D_ERR_UNSUPPORTED, "RK5DPStep's phase-only reset does not compile");
    ns2d_status s = DISPATCH(h, rk5dp_step_impl, h, dt, (int)iters, err);
    if (s) return s;
    return check_status(h);
}

ns2d_status ns2d_check(ns2d_handle* h) {
    if (!h) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    return check_status(h);
}

ns2d_status ns2d_get_stream(const ns2d_handle* h, void** stream) {
    if (!h || !stream) return NS2D_ERR_INVALID;
    *stream = (void*)h->stream;
    return NS2D_OK;
}

ns2d_status ns2d_set_kernel_timing(ns2d_handle* h, int32_t enable) {
    if (!h) return NS2D_ERR_INVALID;
    h->timing = enable != 0;
    for (int k = 0; k < 5; ++k) {
        h->t_ms[k] = 0.0;
        h->t_n[k] = 0;
    }
    return NS2D_OK;
}

ns2d_status ns2d_kernel_times(ns2d_handle* h, double* ms_total, int64_t* launches, int32_t nclasses) {
    if (!h || nclasses < 0) return NS2D_ERR_INVALID;
    CK(h, cudaStreamSynchronize(h->stream));
    for (auto& e : h->ev_open) {
        float ms = 0.f;
        CK(h, cudaEventElapsedTime(&ms, e.second.first, e.second.second));
        h->t_ms[e.first] += ms;
        h->t_n[e.first] += 1;
        h->ev_pool.push_back(e.second.first);
        h->ev_pool.push_back(e.second.second);
    }
    h->ev_open.clear();
    for (int k = 0; k < nclasses && k < 5; ++k) {
        if (ms_total) ms_total[k] = h->t_ms[k];
        if (launches) launches[k] = h->t_n[k];
    }
    return NS2D_OK;
}

ns2d_status ns2d_set_stream(ns2d_handle* h, void* stream) {
    if (!h) return NS2D_ERR_INVALID;
    CK(h, cudaStreamSynchronize(h->stream));
    h->stream = stream ? (cudaStream_t)stream : h->own;
    return NS2D_OK;
}

ns2d_status ns2d_synchronize(ns2d_handle* h) {
    if (!h) return NS2D_ERR_INVALID;
    CK(h, cudaStreamSynchronize(h->stream));
    return NS2D_OK;
}

int64_t ns2d_launch_count(const ns2d_handle* h) { return h ? h->launches : -1; }

}  // extern "C"
