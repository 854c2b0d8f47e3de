// adjoint.cu -- discrete adjoint of the RK4CN step (checkpointed reverse sweep)
// behind the ns2d_adjoint_* entry points of include/ns2d.h.
//
// The reference has no adjoint; this differentiates its RK4Step with __RK4CN
// (Solver/src/solver.c:625-873) over NonlinearRHSBatch (solver.c:884-1032).
//
// Record: n steps forward from the state, copying w_hat every C steps into a
// checkpoint.  Reverse: per segment (last first), restore its checkpoint and
// recompute its steps with the row passes capturing the four real fields of
// every stage, then run the segment's adjoint steps backwards over them.  One
// adjoint step is nine launches, the mirror of a forward step:
//   col START: lambda_x = A lambda'; kappa_4 = b_4 B lambda'; mu_x = IFFT_x(s^2 D kappa_4)
//   row (stage s): mu = c2r_y(mu_x); products with the stage's fields; two packed r2c_y
//   col MID (s = 4, 3, 2): L_s from the products; lambda_x += L_s;
//                          kappa_{s-1} = b_{s-1} B lambda' + a_s dt L_s; mu_x
//   col END (s = 1): lambda_x += L_1
// The reverse sweep runs on two streams: while the adjoint steps of segment k
// run on the adjoint stream, the handle's stream recomputes segment k-1 into
// the other of two capture buffers (one column pass of a 512^2 field covers
// under half of the SMs, so the two overlap).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ns2d.h"
#include "adjoint.cuh"
#include "engine.cuh"
#include "handle.h"

using namespace ns2d;
using ns2d::internal::fail;

namespace ns2d {

struct AdjointState {
    // recorded run
    bool recorded = false;
    int nsteps = 0, every = 0;
    double dt = 0.0;
    int branch = -1;
    // buffers
    void* ckpt = nullptr;  // checkpoints, one field each
    size_t ckpt_n = 0;
    void* cap[2] = {nullptr, nullptr};  // captured stage fields: steps x 8 planes of nx*ny complex
    size_t cap_steps[2] = {0, 0};
    void* lam[2] = {nullptr, nullptr};
    void* P[4] = {nullptr, nullptr, nullptr, nullptr};  // adjoint row-pass outputs
    void* mu = nullptr;                                 // adjoint column-pass output
    void* w_final = nullptr;
    double* dpart = nullptr;  // per-block partial sums
    bool ready = false;       // kernel attributes set
    cudaStream_t stream = nullptr;  // adjoint stream
    cudaEvent_t rec_done[2] = {nullptr, nullptr}, adj_done[2] = {nullptr, nullptr}, join = nullptr;
    cudaEvent_t t[4] = {nullptr, nullptr, nullptr, nullptr};  // timing: record, reverse sweep
    // device time of the last record and reverse sweep (ms)
    double ms_record = 0.0, ms_reverse = 0.0;
    // full-length segments replay captured graphs: the recomputation into
    // capture buffer b, and the adjoint steps over buffer b starting from
    // lambda buffer p
    cudaGraphExec_t rec_graph[2] = {nullptr, nullptr};
    cudaGraphExec_t adj_graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int graph_every = 0, graph_branch = -1;
    double graph_dt = 0.0;
};

}  // namespace ns2d

namespace {

constexpr int kRedBlocks = 296;
const double kB[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
const double kA[3] = {0.5, 0.5, 1.0};

#define ACK(h, call)                                                                                  \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail((h), e_ == cudaErrorMemoryAllocation ? NS2D_ERR_NOMEM : NS2D_ERR_CUDA,        \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

template <typename Real, int N>
struct AdjLaunch {
    using S = Shape<N>;
    static constexpr size_t col_smem() { return ColSmem<Real, N, S::TC>::bytes(); }
    static constexpr size_t row_smem() { return RowSmem<Real, N, 2 * S::PAIRS>::bytes(); }
    static cudaError_t setup() {
        cudaError_t e = cudaSuccess;
        auto set = [&](const void* f, size_t bytes) {
            if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        };
        set((const void*)adj_col_kernel<Real, N, S::TC, ADJ_START>, col_smem());
        set((const void*)adj_col_kernel<Real, N, S::TC, ADJ_MID>, col_smem());
        set((const void*)adj_col_kernel<Real, N, S::TC, ADJ_END>, col_smem());
        set((const void*)adj_row_kernel<Real, N, S::PAIRS>, row_smem());
        return e;
    }
    static void col(int mode, const AdjColArgs<Real>& a, cudaStream_t s) {
        dim3 grid((a.nyf + S::TC - 1) / S::TC), block(S::T * S::TC);
        switch (mode) {
            case ADJ_START: adj_col_kernel<Real, N, S::TC, ADJ_START><<<grid, block, col_smem(), s>>>(a); break;
            case ADJ_MID: adj_col_kernel<Real, N, S::TC, ADJ_MID><<<grid, block, col_smem(), s>>>(a); break;
            default: adj_col_kernel<Real, N, S::TC, ADJ_END><<<grid, block, col_smem(), s>>>(a); break;
        }
    }
    static void row(const AdjRowArgs<Real>& a, cudaStream_t s) {
        dim3 grid(N / (2 * S::PAIRS)), block(S::T * 2 * S::PAIRS);
        adj_row_kernel<Real, N, S::PAIRS><<<grid, block, row_smem(), s>>>(a);
    }
};

template <typename Real, typename F>
bool with_adj_size(int n, F&& f) {
    return with_size<Real>(n, [&](auto L) { f(AdjLaunch<Real, decltype(L)::SIZE>{}); });
}

size_t plane_elems(const ns2d_handle* h) { return (size_t)h->nx * h->ny; }

void drop_graphs(AdjointState* a) {
    for (auto& g : a->rec_graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    for (auto& row : a->adj_graph)
        for (auto& g : row) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
    a->graph_every = 0;
    a->graph_branch = -1;
}

void free_state(AdjointState* a) {
    drop_graphs(a);
    void* ptrs[] = {a->ckpt, a->cap[0], a->cap[1], a->lam[0], a->lam[1], a->P[0], a->P[1],
                    a->P[2], a->P[3], a->mu, a->w_final, a->dpart};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    cudaEvent_t evs[] = {a->rec_done[0], a->rec_done[1], a->adj_done[0], a->adj_done[1], a->join,
                         a->t[0], a->t[1], a->t[2], a->t[3]};
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    if (a->stream) cudaStreamDestroy(a->stream);
}

AdjointState* state_of(ns2d_handle* h) {
    if (!h->adj) h->adj = new (std::nothrow) AdjointState();
    return h->adj;
}

// Buffers for a run of nsteps with checkpoints every `every` steps.
ns2d_status ensure_buffers(ns2d_handle* h, int nsteps, int every) {
    AdjointState* a = state_of(h);
    if (!a) return fail(h, NS2D_ERR_NOMEM, "adjoint state");
    const size_t nck = (size_t)((nsteps + every - 1) / every);
    const size_t seg = (size_t)std::min(every, nsteps);
    if (a->ckpt_n < nck) {
        if (a->ckpt) cudaFree(a->ckpt);
        a->ckpt = nullptr;
        a->ckpt_n = 0;
        ACK(h, cudaMalloc(&a->ckpt, h->field_bytes * nck));
        a->ckpt_n = nck;
    }
    // the second capture buffer only when there is more than one segment
    const int ncap = nck > 1 ? 2 : 1;
    for (int b = 0; b < ncap; ++b)
        if (a->cap_steps[b] < seg) {
            drop_graphs(a);
            if (a->cap[b]) cudaFree(a->cap[b]);
            a->cap[b] = nullptr;
            a->cap_steps[b] = 0;
            ACK(h, cudaMalloc(&a->cap[b], h->elem * 8 * plane_elems(h) * seg));
            a->cap_steps[b] = seg;
        }
    void** fields[] = {&a->lam[0], &a->lam[1], &a->P[0], &a->P[1], &a->P[2], &a->P[3], &a->mu, &a->w_final};
    for (void** f : fields)
        if (!*f) {
            ACK(h, cudaMalloc(f, h->field_bytes));
            ACK(h, cudaMemsetAsync(*f, 0, h->field_bytes, h->stream));
        }
    if (!a->dpart) ACK(h, cudaMalloc(&a->dpart, sizeof(double) * kRedBlocks));
    if (!a->stream) {
        ACK(h, cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking));
        for (int b = 0; b < 2; ++b) {
            ACK(h, cudaEventCreateWithFlags(&a->rec_done[b], cudaEventDisableTiming));
            ACK(h, cudaEventCreateWithFlags(&a->adj_done[b], cudaEventDisableTiming));
        }
        ACK(h, cudaEventCreateWithFlags(&a->join, cudaEventDisableTiming));
        for (auto& e : a->t) ACK(h, cudaEventCreate(&e));
    }
    if (!a->ready) {
        cudaError_t e = cudaSuccess;
        bool ok = h->fp32 ? with_adj_size<float>(h->nx, [&](auto L) { e = decltype(L)::setup(); })
                          : with_adj_size<double>(h->nx, [&](auto L) { e = decltype(L)::setup(); });
        if (!ok) return fail(h, NS2D_ERR_UNSUPPORTED, "grid size");
        ACK(h, e);
        a->ready = true;
    }
    return NS2D_OK;
}

ns2d_status validate(ns2d_handle* h) {
    if (h->p.system != NS2D_NAVIER || h->p.integrator != NS2D_RK4CN)
        return fail(h, NS2D_ERR_UNSUPPORTED, "the adjoint covers the Navier-Stokes RK4CN step");
    if (h->p.model != NS2D_MODEL_FULL)
        return fail(h, NS2D_ERR_UNSUPPORTED, "the adjoint linearises the full model's step, not the phase-only one");
    if (h->p.quirks & NS2D_QUIRK_CONJ_STATE)
        return fail(h, NS2D_ERR_UNSUPPORTED,
                    "the adjoint differentiates the corrected ForceConjugacy: clear NS2D_QUIRK_CONJ_STATE");
    return NS2D_OK;
}

template <typename Real>
AdjColArgs<Real> col_common(ns2d_handle* h) {
    using C = typename Cx<Real>::T;
    AdjColArgs<Real> a;
    std::memset(&a, 0, sizeof(a));
    a.P0 = (const C*)h->f[0];
    a.P1 = (const C*)h->f[1];
    a.P2 = (const C*)h->f[2];
    a.P3 = (const C*)h->f[3];
    a.cn = h->cn;
    a.mu = (C*)h->nl;
    a.tw = (const C*)h->tw;
    a.ldc = h->ldc;
    a.nyf = h->nyf;
    a.norm2 = (Real)std::pow(1.0 / (double)(h->nx * h->ny), 2.0);
    const int m = (int)(h->nx / 3.0);
    a.kmax_sqr = m * m + h->p.dealias_edge;
    a.dealias = h->p.dealias;
    a.houli_int = (h->p.quirks & NS2D_QUIRK_HOU_LI_INT) ? 1 : 0;
    a.kolm = (h->p.forcing == NS2D_FORCING_KOLM) ? 1 : 0;
    return a;
}

// One adjoint step over the captured stage fields `cap` (8 planes), on the
// adjoint stream: lam_x = (step Jacobian)^T lam_p.
template <typename Real>
void adjoint_step(ns2d_handle* h, const void* cap, const void* lam_p, void* lam_x, double dt) {
    using C = typename Cx<Real>::T;
    AdjointState* st = h->adj;
    AdjColArgs<Real> a = col_common<Real>(h);
    a.P0 = (const C*)st->P[0];
    a.P1 = (const C*)st->P[1];
    a.P2 = (const C*)st->P[2];
    a.P3 = (const C*)st->P[3];
    a.mu = (C*)st->mu;
    a.lam_p = (const C*)lam_p;
    a.lam_x = (C*)lam_x;
    AdjRowArgs<Real> r;
    std::memset(&r, 0, sizeof(r));
    r.mu = (const C*)st->mu;
    r.P0 = (C*)st->P[0];
    r.P1 = (C*)st->P[1];
    r.P2 = (C*)st->P[2];
    r.P3 = (C*)st->P[3];
    r.tw = (const C*)h->tw;
    r.ldc = h->ldc;
    const size_t plane = plane_elems(h);
    const C* capc = (const C*)cap;
    cudaStream_t s = st->stream;
    with_adj_size<Real>(h->nx, [&](auto L) {
        using LL = decltype(L);
        a.b_next = kB[3];
        LL::col(ADJ_START, a, s);
        for (int stage = 4; stage >= 1; --stage) {
            r.cap_uv = capc + (size_t)(2 * (stage - 1)) * plane;
            r.cap_w = r.cap_uv + plane;
            LL::row(r, s);
            if (stage > 1) {
                a.b_next = kB[stage - 2];
                a.adt = kA[stage - 2] * dt;
                LL::col(ADJ_MID, a, s);
            } else {
                LL::col(ADJ_END, a, s);
            }
        }
    });
    h->launches += 9;
}

// Ends a stream capture and instantiates it.
ns2d_status end_capture(ns2d_handle* h, cudaStream_t st, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (e != cudaSuccess) return fail(h, NS2D_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *out = nullptr;
        return fail(h, NS2D_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    return NS2D_OK;
}

// The steps k0..k1-1 of the recorded run from the state, the row passes
// capturing every stage into capture buffer `buf` (eager launches).
ns2d_status recompute_steps(ns2d_handle* h, int k0, int k1, int buf) {
    AdjointState* a = h->adj;
    const size_t step_bytes = h->elem * 8 * plane_elems(h);
    ns2d_status st = NS2D_OK;
    for (int k = k0; k < k1 && st == NS2D_OK; ++k) {
        h->cap_step = (char*)a->cap[buf] + (size_t)(k - k0) * step_bytes;
        st = internal::rk4_step(h, a->dt);
    }
    h->cap_step = nullptr;
    return st;
}

// Recompute segment `seg` from its checkpoint on the handle's stream into
// capture buffer `buf`; full-length segments replay a captured graph.
ns2d_status recompute_segment(ns2d_handle* h, int seg, int buf) {
    AdjointState* a = h->adj;
    const int k0 = seg * a->every;
    const int k1 = std::min(k0 + a->every, a->nsteps);
    ACK(h, cudaMemcpyAsync(h->state, (char*)a->ckpt + (size_t)seg * h->field_bytes, h->field_bytes,
                           cudaMemcpyDeviceToDevice, h->stream));
    ns2d_status st = NS2D_OK;
    if (k1 - k0 == a->every && a->every > 1) {
        if (!a->rec_graph[buf]) {
            const int64_t l0 = h->launches;
            const bool timing = h->timing;  // no per-launch events inside the graph
            h->timing = false;
            ACK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            st = recompute_steps(h, k0, k1, buf);
            cudaGraphExec_t g = nullptr;
            ns2d_status st2 = end_capture(h, h->stream, &g);
            h->timing = timing;
            h->launches = l0;
            if (st) {
                if (g) cudaGraphExecDestroy(g);
                return st;
            }
            if (st2) return st2;
            a->rec_graph[buf] = g;
        }
        ACK(h, cudaGraphLaunch(a->rec_graph[buf], h->stream));
        h->launches += 9 * (k1 - k0);
    } else {
        st = recompute_steps(h, k0, k1, buf);
    }
    if (st) return st;
    if (h->cn_dt != a->dt || h->cn_branch != a->branch)
        return fail(h, NS2D_ERR_STATE, "operator branch changed between record and reverse sweep");
    ACK(h, cudaEventRecord(a->rec_done[buf], h->stream));
    return NS2D_OK;
}

// The adjoint steps of a segment of n steps over capture buffer `buf`, on the
// adjoint stream, starting from lambda buffer `par`; returns the parity after.
template <typename Real>
void adjoint_steps(ns2d_handle* h, int n, int buf, int par) {
    AdjointState* a = h->adj;
    const size_t step_bytes = h->elem * 8 * plane_elems(h);
    for (int k = n - 1; k >= 0; --k) {
        adjoint_step<Real>(h, (const char*)a->cap[buf] + (size_t)k * step_bytes, a->lam[par], a->lam[par ^ 1], a->dt);
        par ^= 1;
    }
}

template <typename Real>
ns2d_status adjoint_segment(ns2d_handle* h, int n, int buf, int par) {
    AdjointState* a = h->adj;
    if (n == a->every && a->every > 1) {
        cudaGraphExec_t& g = a->adj_graph[buf][par];
        if (!g) {
            const int64_t l0 = h->launches;
            ACK(h, cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal));
            adjoint_steps<Real>(h, n, buf, par);
            ns2d_status st = end_capture(h, a->stream, &g);
            h->launches = l0;
            if (st) return st;
        }
        ACK(h, cudaGraphLaunch(g, a->stream));
        h->launches += 9 * n;
    } else {
        adjoint_steps<Real>(h, n, buf, par);
    }
    return NS2D_OK;
}

// Reverse sweep over the recorded run: adj->lam[0] holds lambda(T) on entry and
// lambda(0) on return.  The state is left at the recorded final state.
// Segment k's adjoint steps (adjoint stream, capture buffer k % 2) overlap the
// recomputation of segment k-1 (handle stream, buffer (k-1) % 2); each buffer
// is rewritten only after the adjoint steps that read it are done.
template <typename Real>
ns2d_status backward_impl(ns2d_handle* h) {
    AdjointState* a = h->adj;
    const int nck = (a->nsteps + a->every - 1) / a->every;
    if (a->graph_every != a->every || a->graph_dt != a->dt || a->graph_branch != a->branch) {
        drop_graphs(a);
        a->graph_every = a->every;
        a->graph_dt = a->dt;
        a->graph_branch = a->branch;
    }
    int par = 0;  // lambda' lives in lam[par]
    // the CN table of the recorded dt, before any launch reads it
    ns2d_status s0 = internal::ensure_cn(h, a->dt, a->branch);
    if (s0) return s0;
    ACK(h, cudaEventRecord(a->t[2], h->stream));
    ACK(h, cudaStreamWaitEvent(a->stream, a->t[2], 0));  // lambda(T) is written on the handle's stream
    ns2d_status st = recompute_segment(h, nck - 1, (nck - 1) & 1);
    for (int seg = nck - 1; seg >= 0 && st == NS2D_OK; --seg) {
        const int buf = seg & 1;
        const int k0 = seg * a->every;
        const int n = std::min(k0 + a->every, a->nsteps) - k0;
        ACK(h, cudaStreamWaitEvent(a->stream, a->rec_done[buf], 0));
        if ((st = adjoint_segment<Real>(h, n, buf, par))) break;
        par ^= (n & 1);
        ACK(h, cudaEventRecord(a->adj_done[buf], a->stream));
        if (seg > 0) {
            // buffer (seg-1) & 1 was last read by segment seg+1's adjoint steps
            if (seg + 1 < nck) ACK(h, cudaStreamWaitEvent(h->stream, a->adj_done[(seg + 1) & 1], 0));
            st = recompute_segment(h, seg - 1, (seg - 1) & 1);
        }
    }
    // join: the handle's stream continues after the last adjoint step
    ACK(h, cudaEventRecord(a->join, a->stream));
    ACK(h, cudaStreamWaitEvent(h->stream, a->join, 0));
    if (st) return st;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, NS2D_ERR_CUDA, std::string("adjoint launch: ") + cudaGetErrorString(e));
    if (par != 0) ACK(h, cudaMemcpyAsync(a->lam[0], a->lam[1], h->field_bytes, cudaMemcpyDeviceToDevice, h->stream));
    ACK(h, cudaMemcpyAsync(h->state, a->w_final, h->field_bytes, cudaMemcpyDeviceToDevice, h->stream));
    ACK(h, cudaEventRecord(a->t[3], h->stream));
    ns2d_status s2 = internal::check_status(h);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a->t[2], a->t[3]);
    a->ms_reverse = ms;
    return s2;
}

ns2d_status backward(ns2d_handle* h) {
    if (!h->adj || !h->adj->recorded) return fail(h, NS2D_ERR_STATE, "no recorded run: call ns2d_adjoint_record first");
    return h->fp32 ? backward_impl<float>(h) : backward_impl<double>(h);
}

// J(state) into *value, its W-gradient into `lam` (internal layout) when non-null.
template <typename Real>
ns2d_status objective_impl(ns2d_handle* h, int kind, double* value, void* lam) {
    using C = typename Cx<Real>::T;
    AdjointState* a = h->adj;
    const double cz = 4.0 * M_PI * M_PI * 0.5 / std::pow((double)h->nx * (double)h->ny, 2.0);
    adj_objective_kernel<Real><<<kRedBlocks, 256, 0, h->stream>>>((const C*)h->state, (C*)lam, h->nx, h->nyf, h->ldc,
                                                                   cz, kind == NS2D_OBJ_PALINSTROPHY ? 1 : 0, a->dpart);
    h->launches++;
    ACK(h, cudaGetLastError());
    double part[kRedBlocks];
    ACK(h, cudaMemcpyAsync(part, a->dpart, sizeof(part), cudaMemcpyDeviceToHost, h->stream));
    ACK(h, cudaStreamSynchronize(h->stream));
    double tot = 0.0;
    for (int b = 0; b < kRedBlocks; ++b) tot += part[b];
    *value = tot;
    return NS2D_OK;
}

ns2d_status record(ns2d_handle* h, int nsteps, double dt, int every) {
    ns2d_status s = validate(h);
    if (s) return s;
    if (nsteps < 1 || every < 1 || !(dt > 0.0)) return fail(h, NS2D_ERR_INVALID, "nsteps, checkpoint interval and dt must be positive");
    if ((s = ensure_buffers(h, nsteps, every))) return s;
    AdjointState* a = h->adj;
    a->recorded = false;
    ACK(h, cudaEventRecord(a->t[0], h->stream));
    for (int k = 0; k < nsteps; ++k) {
        if (k % every == 0)
            ACK(h, cudaMemcpyAsync((char*)a->ckpt + (size_t)(k / every) * h->field_bytes, h->state, h->field_bytes,
                                   cudaMemcpyDeviceToDevice, h->stream));
        if ((s = internal::rk4_step_loop(h, dt))) return s;
    }
    ACK(h, cudaEventRecord(a->t[1], h->stream));
    if ((s = internal::check_status(h))) return s;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a->t[0], a->t[1]);
    a->ms_record = ms;
    ACK(h, cudaMemcpyAsync(a->w_final, h->state, h->field_bytes, cudaMemcpyDeviceToDevice, h->stream));
    a->nsteps = nsteps;
    a->every = every;
    a->dt = dt;
    a->branch = h->cn_branch;
    a->recorded = true;
    return NS2D_OK;
}

}  // namespace

namespace ns2d {
namespace internal {

void adjoint_free(ns2d_handle* h) {
    if (!h->adj) return;
    free_state(h->adj);
    delete h->adj;
    h->adj = nullptr;
}

}  // namespace internal
}  // namespace ns2d

extern "C" {

ns2d_status ns2d_adjoint_record(ns2d_handle* h, int32_t nsteps, double dt, int32_t checkpoint_every) {
    if (!h) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    return record(h, nsteps, dt, checkpoint_every);
}

ns2d_status ns2d_objective(ns2d_handle* h, int32_t kind, double* value, double* d_grad) {
    if (!h || !value || (kind != NS2D_OBJ_ENSTROPHY && kind != NS2D_OBJ_PALINSTROPHY)) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s = ensure_buffers(h, 1, 1);
    if (s) return s;
    void* lam = d_grad ? h->adj->lam[1] : nullptr;
    s = h->fp32 ? objective_impl<float>(h, kind, value, lam) : objective_impl<double>(h, kind, value, lam);
    if (s || !d_grad) return s;
    return internal::unpack_out(h, lam, (double2*)d_grad);
}

ns2d_status ns2d_adjoint_backward_device(ns2d_handle* h, const double* d_lam_T, double* d_lam_0) {
    if (!h || !d_lam_T || !d_lam_0) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    if (!h->adj || !h->adj->recorded) return fail(h, NS2D_ERR_STATE, "no recorded run: call ns2d_adjoint_record first");
    ns2d_status s = internal::pack_in(h, (const double2*)d_lam_T, h->adj->lam[0]);
    if (s) return s;
    if ((s = backward(h))) return s;
    return internal::unpack_out(h, h->adj->lam[0], (double2*)d_lam_0);
}

ns2d_status ns2d_adjoint_backward(ns2d_handle* h, const double* lam_T, double* lam_0) {
    if (!h || !lam_T || !lam_0) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    if (!h->adj || !h->adj->recorded) return fail(h, NS2D_ERR_STATE, "no recorded run: call ns2d_adjoint_record first");
    const size_t bytes = sizeof(double2) * (size_t)h->nx * h->nyf;
    ACK(h, cudaMemcpyAsync(h->dio, lam_T, bytes, cudaMemcpyHostToDevice, h->stream));
    ns2d_status s = internal::pack_in(h, h->dio, h->adj->lam[0]);
    if (s) return s;
    if ((s = backward(h))) return s;
    if ((s = internal::unpack_out(h, h->adj->lam[0], h->dio))) return s;
    ACK(h, cudaMemcpyAsync(lam_0, h->dio, bytes, cudaMemcpyDeviceToHost, h->stream));
    ACK(h, cudaStreamSynchronize(h->stream));
    return NS2D_OK;
}

ns2d_status ns2d_adjoint_gradient(ns2d_handle* h, int32_t nsteps, double dt, int32_t checkpoint_every, int32_t kind,
                                  double* value, double* grad) {
    if (!h || !value || !grad || (kind != NS2D_OBJ_ENSTROPHY && kind != NS2D_OBJ_PALINSTROPHY)) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s = record(h, nsteps, dt, checkpoint_every);
    if (s) return s;
    s = h->fp32 ? objective_impl<float>(h, kind, value, h->adj->lam[0])
                : objective_impl<double>(h, kind, value, h->adj->lam[0]);
    if (s) return s;
    if ((s = backward(h))) return s;
    if ((s = internal::unpack_out(h, h->adj->lam[0], h->dio))) return s;
    ACK(h, cudaMemcpyAsync(grad, h->dio, sizeof(double2) * (size_t)h->nx * h->nyf, cudaMemcpyDeviceToHost, h->stream));
    ACK(h, cudaStreamSynchronize(h->stream));
    return NS2D_OK;
}

ns2d_status ns2d_adjoint_times(const ns2d_handle* h, double* ms_record, double* ms_reverse) {
    if (!h || !h->adj) return NS2D_ERR_INVALID;
    if (ms_record) *ms_record = h->adj->ms_record;
    if (ms_reverse) *ms_reverse = h->adj->ms_reverse;
    return NS2D_OK;
}

ns2d_status ns2d_wdot_device(ns2d_handle* h, const double* d_a, const double* d_b, double* value) {
    if (!h || !d_a || !d_b || !value) return NS2D_ERR_INVALID;
    cudaSetDevice(h->p.device);
    ns2d_status s = ensure_buffers(h, 1, 1);
    if (s) return s;
    // the packed complex128 arrays are read as-is: nyf = ldc for this reduction
    adj_wdot_kernel<double><<<kRedBlocks, 256, 0, h->stream>>>((const double2*)d_a, (const double2*)d_b, h->nx, h->nyf,
                                                               h->nyf, h->adj->dpart);
    h->launches++;
    ACK(h, cudaGetLastError());
    double part[kRedBlocks];
    ACK(h, cudaMemcpyAsync(part, h->adj->dpart, sizeof(part), cudaMemcpyDeviceToHost, h->stream));
    ACK(h, cudaStreamSynchronize(h->stream));
    double tot = 0.0;
    for (int b = 0; b < kRedBlocks; ++b) tot += part[b];
    *value = tot;
    return NS2D_OK;
}

}  // extern "C"
