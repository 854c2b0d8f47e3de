// handle.h -- the single-trajectory handle behind include/ns2d.h and the
// internal entry points shared by api.cu and adjoint.cu.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/ns2d.h"

namespace ns2d {
struct AdjointState;
}

struct ns2d_handle {
    ns2d_params p{};
    int nx = 0, ny = 0, nyf = 0, ldc = 0;
    bool fp32 = false;
    cudaStream_t stream = nullptr;
    cudaStream_t own = nullptr;  // stream created by ns2d_create
    std::string err;
    int64_t launches = 0;
    size_t elem = 0;         // bytes per complex element
    size_t field_bytes = 0;  // nx * ldc * elem
    // device buffers
    void* state = nullptr;
    void* acc = nullptr;
    void* nl = nullptr;
    void* f[4] = {nullptr, nullptr, nullptr, nullptr};
    void* tmpfull = nullptr;  // explicit-RK4 stage input / standalone RHS input
    void* col0[2] = {nullptr, nullptr};
    void* tw = nullptr;
    void* rhsbuf = nullptr;
    void* ab[4] = {nullptr, nullptr, nullptr, nullptr};  // AB4 ring: [0..2] history, [3] next
    void* uhat_ref = nullptr;  // persistent u_hat in the reference layout (CFL / VEL paths)
    double* dreal = nullptr;   // [nx][ny] real-space output
    double* dscal = nullptr;   // [0] bound accumulator, [1] ticket
    unsigned long long* dmax = nullptr;
    int* dstatus = nullptr;    // [0] bits, [1] completed steps
    double2* dio = nullptr;    // staging [nx][nyf] complex128
    double* ddiag = nullptr;   // measurables: DG_N totals + 8 * n_spect spectra
    double* dpart = nullptr;   // per-block partial bounds of the final column pass
    double2* cn = nullptr;     // Crank-Nicolson factors per mode ([nx][ldc])
    double cn_dt = 0.0;        // dt and branch the table was built for
    int cn_branch = -1;
    // model state kept on the host
    int hyper_flag = 0;
    bool forced = false;
    int force_i = 0, force_j = 0;
    double fre = 0.0, fim = 0.0;
    double w_max_init = 0.0, min_dt = 10.0, max_dt = 1e-10;
    int n_spect = 0;
    int ab_count = 0;
    // optional per-launch event timing
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_open;
    double t_ms[5] = {0, 0, 0, 0, 0};
    int64_t t_n[5] = {0, 0, 0, 0, 0};
    // adjoint: per-step capture target of the row passes (null = off) and the
    // adjoint's own buffers (adjoint.cu)
    void* cap_step = nullptr;
    void* col_maps = nullptr;  // ColMaps of f[0..3], acc, state and nl (TMA copies), null if unavailable
    ns2d::AdjointState* adj = nullptr;
    // forcing of listed modes (ns2d_set_forcing_modes): dense field added to the RHS
    void* ffield = nullptr;
    bool ffield_on = false;
    int32_t* fidx = nullptr;
    double2* fval = nullptr;
    int fcap = 0;
    // Dormand-Prince stages k0..k6, y0 and the stage input (allocated on first use)
    void* dp[9] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    const void** dp_kptr = nullptr;  // device array of the seven stage pointers
    // RK5DPStep as written: the state of the last error step (Int_data->w_hat_last,
    // zero until then) and the last error (Int_data->DP_err)
    void* dp_last = nullptr;
    double dp_err = 0.0;
    // one RK4/RK4CN step captured as a CUDA graph for fixed-dt stepping
    cudaGraphExec_t step_graph = nullptr;
    int graph_kernels = 9;  // kernels in one captured step
    double graph_dt = 0.0;
    int graph_branch = -1;
    double last_call_dt = -1.0;  // dt of the previous ns2d_rk4_step / _host call
    // the same with an event pair around every launch (kernel timing mode)
    cudaGraphExec_t timed_graph = nullptr;
    double timed_dt = 0.0;
    int timed_branch = -1;
    bool capturing_timed = false;

    int gev_n = 0;
    int gev_set = 0;                 // event set being captured: [0] full step, [1] fused step
    int gev_n_of[2] = {0, 0};
    cudaEvent_t gev_g[2][16][2] = {};
    int gev_cls_g[2][16] = {};
};

namespace ns2d {
namespace internal {

ns2d_status fail(ns2d_handle* h, ns2d_status s, const std::string& msg);
// One RK4 / RK4CN step in the handle's precision (no status read-back).
ns2d_status rk4_step(ns2d_handle* h, double dt);
// The same through the fixed-dt graph replay of the time loops.
ns2d_status rk4_step_loop(ns2d_handle* h, double dt);
// Crank-Nicolson factor table for (dt, operator branch).
ns2d_status ensure_cn(ns2d_handle* h, double dt, int branch);
// Status read-back and SystemCheck after a batch of steps.
ns2d_status check_status(ns2d_handle* h);
// complex128 [nx][nyf] device array <-> internal [nx][ldc] field.
ns2d_status pack_in(ns2d_handle* h, const double2* d_src, void* dst);
ns2d_status unpack_out(ns2d_handle* h, const void* src, double2* d_dst);
// Frees the adjoint's buffers (adjoint.cu).
void adjoint_free(ns2d_handle* h);

}  // namespace internal
}  // namespace ns2d
