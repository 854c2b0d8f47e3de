// ensemble.cu -- C ABI of the batched ensemble (ns2d_ensemble_* in
// include/ns2d.h): independent trajectories of uneven square grid sizes
// advanced together, one launch per pass for all members, the step captured in
// a CUDA graph, and an autotuner for the persistent grid sizes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ns2d.h"
#include "aux_kernels.cuh"
#include "diag.cuh"
#include "ensemble.cuh"
#include "host_common.h"

using namespace ns2d;

struct ns2d_ensemble {
    ns2d_params p{};
    bool fp32 = false;
    int n = 0;
    std::vector<int> sizes;
    cudaStream_t stream = nullptr;
    cudaStream_t own = nullptr;
    std::string err;
    int64_t launches = 0;
    int hyper_flag = 0;
    // device memory
    std::vector<void*> allocs;
    void* members = nullptr;      // EnsMember<Real>[n]
    // work items of each block-size choice (kEnsThreadChoices) and the choice
    // each pass uses
    EnsItem* col_items[2] = {nullptr, nullptr};
    EnsItem* row_items[2] = {nullptr, nullptr};
    int n_col_items[2] = {0, 0}, n_row_items[2] = {0, 0};
    int col_var = 0, row_var = 0;
    // one persistent launch per RK stage (ens_stage_kernel): its task list
    // (first-pass column tiles, then row blocks, then column tiles), the work
    // and completion counters, the tasks' input counts, smem and grid
    bool fused = false;
    EnsTask* tasks = nullptr;
    int n_tasks = 0, n_p1_tasks = 0;
    int* sync = nullptr;          // [4] heads, then [5][n] completion counters
    int* need = nullptr;          // [n][2]
    size_t stage_smem = 0;
    int stage_grid = 0, stage_per_sm = 1;
    int* status = nullptr;
    double* ddiag = nullptr;
    std::vector<void*> state, nl, acc, tw;
    std::vector<double2*> cn;
    std::vector<int> ldc;
    double2* io = nullptr;        // staging for host I/O, largest member
    int col_grid = 0, row_grid = 0;
    // CN tables and graph for the current dt
    double cn_dt = -1.0;
    int cn_branch = -1;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double graph_dt = -1.0;
    int graph_col_grid = 0, graph_row_grid = 0, graph_col_var = -1, graph_row_var = -1;
    int graph_fused = -1, graph_stage_grid = 0;
    size_t col_smem[2] = {0, 0}, row_smem[2] = {0, 0}, col_tma_smem[2] = {0, 0};
    // tensor maps of every member's arrays for the TMA column kernels,
    // [member][block-size choice]; null when they are not used
    ColMaps* maps = nullptr;
    int nsm = 148;
};

namespace {

ns2d_status efail(ns2d_ensemble* e, ns2d_status s, const std::string& m) {
    if (e) e->err = m;
    return s;
}

#define ECK(e, call)                                                                                   \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return efail((e), e_ == cudaErrorMemoryAllocation ? NS2D_ERR_NOMEM : NS2D_ERR_CUDA,        \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

bool ens_size_ok(int n) {
    switch (n) {
#define NS2D_ENS_OK(NN) case NN:
        NS2D_ENS_SIZES(NS2D_ENS_OK)
#undef NS2D_ENS_OK
        return true;
        default: return false;
    }
}

// Column tile width and rows per row block of a member of size n under block
// size kEnsThreadChoices[v].
int ens_col_tc(int n, int v) {
    switch (n) {
#define NS2D_ENS_TC(NN) \
    case NN: return v == 0 ? EnsShape<NN, kEnsThreadChoices[0]>::TC : EnsShape<NN, kEnsThreadChoices[1]>::TC;
        NS2D_ENS_SIZES(NS2D_ENS_TC)
#undef NS2D_ENS_TC
        default: return 1;
    }
}
int ens_row_tc(int n, int v) {
    switch (n) {
#define NS2D_ENS_RT(NN) \
    case NN: return 2 * (v == 0 ? EnsShape<NN, kEnsThreadChoices[0]>::PAIRS : EnsShape<NN, kEnsThreadChoices[1]>::PAIRS);
        NS2D_ENS_SIZES(NS2D_ENS_RT)
#undef NS2D_ENS_RT
        default: return 2;
    }
}

template <typename Real, int V>
cudaError_t ens_set_smem(ns2d_ensemble* e) {
    constexpr int TH = kEnsThreadChoices[V];
    e->col_smem[V] = EnsSmem<Real, TH>::col();
    e->row_smem[V] = EnsSmem<Real, TH>::row();
    e->col_tma_smem[V] = EnsSmem<Real, TH>::col_tma();
    cudaError_t r = cudaSuccess;
    auto set = [&](const void* f, size_t b) {
        if (r == cudaSuccess) r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
    };
    set((const void*)ens_col_kernel<Real, COL_P1, TH>, e->col_smem[V]);
    set((const void*)ens_col_kernel<Real, COL_STAGE, TH>, e->col_smem[V]);
    set((const void*)ens_col_kernel<Real, COL_FINAL, TH>, e->col_smem[V]);
    set((const void*)ens_col_kernel<Real, COL_STAGE, TH, true>, e->col_smem[V]);
    set((const void*)ens_col_kernel<Real, COL_FINAL, TH, true>, e->col_smem[V]);
    set((const void*)ens_col_kernel<Real, COL_P1, TH, true, true>, e->col_tma_smem[V]);
    set((const void*)ens_col_kernel<Real, COL_STAGE, TH, true, true>, e->col_tma_smem[V]);
    set((const void*)ens_col_kernel<Real, COL_FINAL, TH, true, true>, e->col_tma_smem[V]);
    set((const void*)ens_row_kernel<Real, TH>, e->row_smem[V]);
    return r;
}

// Whether the stage and final column passes of this ensemble can run the
// epilogue compiled for the common step (col_fast_ok of the single passes).
bool ens_fast(const ns2d_ensemble* e) {
    return e->p.dealias == 0 && e->p.system != NS2D_EULER && e->p.integrator == NS2D_RK4CN &&
           e->p.model == NS2D_MODEL_FULL;
}

// Blocks per SM of the choice's column and row kernels.
template <typename Real, int V>
void ens_occupancy(const ns2d_ensemble* e, int* col_per_sm, int* row_per_sm) {
    constexpr int TH = kEnsThreadChoices[V];
    if (e->maps && ens_fast(e))
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(col_per_sm, ens_col_kernel<Real, COL_STAGE, TH, true, true>, TH,
                                                      e->col_tma_smem[V]);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(col_per_sm, ens_col_kernel<Real, COL_STAGE, TH>, TH, e->col_smem[V]);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(row_per_sm, ens_row_kernel<Real, TH>, TH, e->row_smem[V]);
}


template <typename Real, int MODE, int V, bool FAST, bool TMA = false>
void ens_launch_col_v(ns2d_ensemble* e, const EnsMember<Real>* mb, const EnsStage& st) {
    constexpr int TH = kEnsThreadChoices[V];
    ens_col_kernel<Real, MODE, TH, FAST, TMA><<<e->col_grid, TH, TMA ? e->col_tma_smem[V] : e->col_smem[V], e->stream>>>(
        mb, e->col_items[V], e->n_col_items[V], st, e->maps);
}

// The TMA column kernels run the common step (ens_fast) when the members'
// tensor maps exist; otherwise per-thread copies.
template <typename Real, int MODE>
void ens_launch_col(ns2d_ensemble* e, const EnsMember<Real>* mb, const EnsStage& st) {
    const bool fast = ens_fast(e);
    if (fast && e->maps) {
        if (e->col_var == 0) ens_launch_col_v<Real, MODE, 0, true, true>(e, mb, st);
        else ens_launch_col_v<Real, MODE, 1, true, true>(e, mb, st);
    } else if constexpr (MODE == COL_P1) {
        if (e->col_var == 0) ens_launch_col_v<Real, MODE, 0, false>(e, mb, st);
        else ens_launch_col_v<Real, MODE, 1, false>(e, mb, st);
    } else {
        if (e->col_var == 0) {
            if (fast) ens_launch_col_v<Real, MODE, 0, true>(e, mb, st);
            else ens_launch_col_v<Real, MODE, 0, false>(e, mb, st);
        } else {
            if (fast) ens_launch_col_v<Real, MODE, 1, true>(e, mb, st);
            else ens_launch_col_v<Real, MODE, 1, false>(e, mb, st);
        }
    }
}

template <typename Real>
void ens_launch_row(ns2d_ensemble* e, const EnsMember<Real>* mb) {
    const int v = e->row_var;
    if (v == 0)
        ens_row_kernel<Real, kEnsThreadChoices[0]><<<e->row_grid, kEnsThreadChoices[0], e->row_smem[0], e->stream>>>(
            mb, e->row_items[0], e->n_row_items[0], e->status);
    else
        ens_row_kernel<Real, kEnsThreadChoices[1]><<<e->row_grid, kEnsThreadChoices[1], e->row_smem[1], e->stream>>>(
            mb, e->row_items[1], e->n_row_items[1], e->status);
}

template <typename Real>
ns2d_status create_t(ns2d_ensemble* e) {
    using C = typename Cx<Real>::T;
    std::vector<EnsMember<Real>> hm(e->n);
    auto alloc = [&](size_t bytes, void** p) -> cudaError_t {
        cudaError_t r = cudaMalloc(p, bytes);
        if (r == cudaSuccess) {
            e->allocs.push_back(*p);
            r = cudaMemsetAsync(*p, 0, bytes, e->stream);
        }
        return r;
    };
    size_t io_elems = 0;
    e->state.resize(e->n);
    e->nl.resize(e->n);
    e->acc.resize(e->n);
    e->tw.resize(e->n);
    e->cn.resize(e->n);
    e->ldc.resize(e->n);
    for (int m = 0; m < e->n; ++m) {
        const int n = e->sizes[m];
        const int nyf = n / 2 + 1;
        const int ldc = (nyf + 3) & ~3;
        e->ldc[m] = ldc;
        const size_t fb = sizeof(C) * (size_t)n * ldc;
        void *st, *nl, *ac, *f[4], *c0[2], *tw, *cn;
        ECK(e, alloc(fb, &st));
        ECK(e, alloc(fb, &nl));
        ECK(e, alloc(fb, &ac));
        for (int k = 0; k < 4; ++k) ECK(e, alloc(fb, &f[k]));
        for (int k = 0; k < 2; ++k) ECK(e, alloc(sizeof(C) * n, &c0[k]));
        ECK(e, alloc(sizeof(C) * n, &tw));
        ECK(e, alloc(sizeof(double2) * (size_t)n * ldc, &cn));
        std::vector<C> htw(n);
        for (int q = 0; q < n; ++q) {
            long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)q / (long double)n;
            htw[q].x = (Real)cosl(a);
            htw[q].y = (Real)(-sinl(a));
        }
        ECK(e, cudaMemcpyAsync(tw, htw.data(), sizeof(C) * n, cudaMemcpyHostToDevice, e->stream));
        ECK(e, cudaStreamSynchronize(e->stream));
        e->state[m] = st;
        e->nl[m] = nl;
        e->acc[m] = ac;
        e->tw[m] = tw;
        e->cn[m] = (double2*)cn;
        io_elems = std::max(io_elems, (size_t)n * nyf);
        EnsMember<Real>& mb = hm[m];
        std::memset(&mb, 0, sizeof(mb));
        ColArgs<Real>& a = mb.col;
        a.src = (const C*)nl;
        a.state = (C*)st;
        a.acc = (C*)ac;
        a.f0 = (C*)f[0];
        a.f1 = (C*)f[1];
        a.f2 = (C*)f[2];
        a.f3 = (C*)f[3];
        a.tw = (const C*)tw;
        a.ldc = ldc;
        a.nyf = nyf;
        const int km = (int)(n / 3.0);
        a.kmax_sqr = km * km;
        a.dealias = e->p.dealias;
        a.houli_int = (e->p.quirks & NS2D_QUIRK_HOU_LI_INT) ? 1 : 0;
        a.kolm = (e->p.forcing == NS2D_FORCING_KOLM) ? 1 : 0;
        if (e->p.forcing == NS2D_FORCING_KOLM) {
            a.has_force = 1;
            a.force_i = e->p.force_k / nyf;
            a.force_j = e->p.force_k % nyf;
            a.force_val.x = (Real)(-0.5 * e->p.force_scale * (double)e->p.force_k);
            a.force_val.y = (Real)0;
        }
        a.norm2 = (Real)std::pow(1.0 / (double)(n * n), 2.0);
        a.inv_nxny = 1.0 / (double)(n * n);
        a.cn = (const double2*)cn;
        a.phase_only = e->p.model == NS2D_MODEL_PHASE_ONLY ? 1 : 0;
        mb.row.f0 = (const C*)f[0];
        mb.row.f1 = (const C*)f[1];
        mb.row.f2 = (const C*)f[2];
        mb.row.f3 = (const C*)f[3];
        mb.row.nl = (C*)nl;
        mb.row.tw = (const C*)tw;
        mb.row.ldc = ldc;
        mb.row.nrows = n;
        mb.row.status = nullptr;
        mb.col0[0] = (C*)c0[0];
        mb.col0[1] = (C*)c0[1];
        mb.n = n;
    }
    ECK(e, alloc(sizeof(EnsMember<Real>) * e->n, &e->members));
    ECK(e, cudaMemcpyAsync(e->members, hm.data(), sizeof(EnsMember<Real>) * e->n, cudaMemcpyHostToDevice, e->stream));
    if (ens_fast(e) && tma_copies_enabled()) {
        // tensor maps of each member's arrays for both block-size choices
        std::vector<ColMaps> hmaps(2 * (size_t)e->n);
        bool ok = true;
        for (int m = 0; m < e->n && ok; ++m) {
            const ColArgs<Real>& a = hm[m].col;
            void* const bases[7] = {a.f0, a.f1, a.f2, a.f3, a.acc, a.state, (void*)a.src};
            for (int v = 0; v < 2 && ok; ++v)
                ok = encode_col_maps<Real>(&hmaps[2 * m + v], bases, e->sizes[m], a.nyf, a.ldc, ens_col_tc(e->sizes[m], v));
        }
        if (ok) {
            void* dm = nullptr;
            ECK(e, alloc(sizeof(ColMaps) * hmaps.size(), &dm));
            ECK(e, cudaMemcpyAsync(dm, hmaps.data(), sizeof(ColMaps) * hmaps.size(), cudaMemcpyHostToDevice, e->stream));
            ECK(e, cudaStreamSynchronize(e->stream));
            e->maps = (ColMaps*)dm;
        }
    }
    ECK(e, alloc(sizeof(double2) * io_elems, (void**)&e->io));
    ECK(e, alloc(sizeof(int) * 4, (void**)&e->status));
    int nspect_max = 0;
    for (int n : e->sizes) nspect_max = std::max(nspect_max, (int)std::round(std::sqrt(2.0 * (n / 2.0) * (n / 2.0)) + 1));
    ECK(e, alloc(sizeof(double) * (DG_N + 8 * (size_t)nspect_max), (void**)&e->ddiag));
    ECK(e, cudaFuncSetAttribute((const void*)diag_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(double) * (8 * (size_t)nspect_max + DG_N * 8))));
    // work items of each block-size choice, largest grids first
    // (longest-processing-time order)
    std::vector<int> order(e->n);
    for (int m = 0; m < e->n; ++m) order[m] = m;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return e->sizes[x] > e->sizes[y]; });
    for (int v = 0; v < 2; ++v) {
        std::vector<EnsItem> ci, ri;
        for (int m : order) {
            const int n = e->sizes[m];
            const int tiles = (n / 2 + 1 + ens_col_tc(n, v) - 1) / ens_col_tc(n, v);
            for (int t = 0; t < tiles; ++t) ci.push_back({m, t});
            for (int r = 0; r < n / ens_row_tc(n, v); ++r) ri.push_back({m, r});
        }
        e->n_col_items[v] = (int)ci.size();
        e->n_row_items[v] = (int)ri.size();
        ECK(e, alloc(sizeof(EnsItem) * ci.size(), (void**)&e->col_items[v]));
        ECK(e, alloc(sizeof(EnsItem) * ri.size(), (void**)&e->row_items[v]));
        ECK(e, cudaMemcpyAsync(e->col_items[v], ci.data(), sizeof(EnsItem) * ci.size(), cudaMemcpyHostToDevice, e->stream));
        ECK(e, cudaMemcpyAsync(e->row_items[v], ri.data(), sizeof(EnsItem) * ri.size(), cudaMemcpyHostToDevice, e->stream));
    }
    {
        // task list of the per-stage launches, 256-thread shapes
        std::vector<EnsTask> p1, rows, cols;
        std::vector<int> need(2 * e->n);
        for (int m : order) {
            const int n = e->sizes[m];
            const int tiles = (n / 2 + 1 + ens_col_tc(n, 0) - 1) / ens_col_tc(n, 0);
            const int blocks = n / ens_row_tc(n, 0);
            need[2 * m] = tiles;
            need[2 * m + 1] = blocks;
            for (int t = 0; t < tiles; ++t) {
                p1.push_back({0, m, t});
                cols.push_back({2, m, t});
            }
            for (int r = 0; r < blocks; ++r) rows.push_back({1, m, r});
        }
        std::vector<EnsTask> all(p1);
        all.insert(all.end(), rows.begin(), rows.end());
        all.insert(all.end(), cols.begin(), cols.end());
        e->n_tasks = (int)all.size();
        e->n_p1_tasks = (int)p1.size();
        ECK(e, alloc(sizeof(EnsTask) * all.size(), (void**)&e->tasks));
        ECK(e, cudaMemcpyAsync(e->tasks, all.data(), sizeof(EnsTask) * all.size(), cudaMemcpyHostToDevice, e->stream));
        ECK(e, alloc(sizeof(int) * (4 + 5 * (size_t)e->n), (void**)&e->sync));
        ECK(e, alloc(sizeof(int) * need.size(), (void**)&e->need));
        ECK(e, cudaMemcpyAsync(e->need, need.data(), sizeof(int) * need.size(), cudaMemcpyHostToDevice, e->stream));
        constexpr int TH = kEnsThreadChoices[0];
        e->stage_smem = EnsSmem<Real, TH>::stage();
        ECK(e, cudaFuncSetAttribute((const void*)ens_stage_kernel<Real, COL_STAGE, TH>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e->stage_smem));
        ECK(e, cudaFuncSetAttribute((const void*)ens_stage_kernel<Real, COL_FINAL, TH>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e->stage_smem));
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ens_stage_kernel<Real, COL_STAGE, TH>, TH, e->stage_smem);
        e->stage_per_sm = std::max(1, per_sm);
    }
    ECK(e, (ens_set_smem<Real, 0>(e)));
    ECK(e, (ens_set_smem<Real, 1>(e)));
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, dev);
    // default: 256-thread blocks, persistent grids with every item in one wave where it fits
    int col_per_sm = 0, row_per_sm = 0;
    ens_occupancy<Real, 0>(e, &col_per_sm, &row_per_sm);
    e->col_var = e->row_var = 0;
    e->col_grid = std::max(1, std::min(e->n_col_items[0], e->nsm * std::max(1, col_per_sm)));
    e->row_grid = std::max(1, std::min(e->n_row_items[0], e->nsm * std::max(1, row_per_sm)));
    e->stage_grid = e->nsm * e->stage_per_sm;
    ECK(e, cudaStreamSynchronize(e->stream));
    return NS2D_OK;
}

// One RK4CN / RK4 step of every member: 9 launches.
template <typename Real>
ns2d_status step_t(ns2d_ensemble* e, double dt) {
    const bool explicit_rk4 = e->p.system == NS2D_EULER || e->p.integrator == NS2D_RK4;
    const bool latch = (e->p.quirks & NS2D_QUIRK_HYPER_LATCH) != 0;
    int branch = 4;
    if (e->p.system != NS2D_EULER) branch = ns2d::resolve_branch(e->hyper_flag, e->p.ekmn_drag_flag, latch);
    if (!explicit_rk4 && (e->cn_dt != dt || e->cn_branch != branch)) {
        const LinOp L = make_lin_params(e->p, branch);
        for (int m = 0; m < e->n; ++m) {
            const int n = e->sizes[m];
            cn_table_kernel<<<148, 256, 0, e->stream>>>(e->cn[m], n, n / 2 + 1, e->ldc[m], dt, L);
            e->launches++;
        }
        e->cn_dt = dt;
        e->cn_branch = branch;
    }
    const double A[3] = {0.5, 0.5, 1.0};
    const double B_cn[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    const double B_ex[4] = {1.0, 2.0, 2.0, 1.0};
    const EnsMember<Real>* mb = (const EnsMember<Real>*)e->members;
    EnsStage st;
    std::memset(&st, 0, sizeof(st));
    st.dt = dt;
    st.lin = make_lin_params(e->p, branch);
    st.conj_quirk = (e->p.quirks & NS2D_QUIRK_CONJ_STATE) ? 1 : 0;
    st.status = e->status;
    if (e->fused) {
        // one persistent launch per RK stage; the counters restart every step
        cudaError_t rm = cudaMemsetAsync(e->sync, 0, sizeof(int) * (4 + 5 * (size_t)e->n), e->stream);
        if (rm != cudaSuccess) return efail(e, NS2D_ERR_CUDA, cudaGetErrorString(rm));
        EnsSync sy;
        sy.head = e->sync;
        sy.done = e->sync + 4;
        sy.need = e->need;
        sy.nmem = e->n;
        constexpr int TH = kEnsThreadChoices[0];
        for (int s = 1; s <= 4; ++s) {
            st.stage = s;
            st.b_cur = explicit_rk4 ? B_ex[s - 1] : B_cn[s - 1];
            const EnsTask* tl = e->tasks + (s == 1 ? 0 : e->n_p1_tasks);
            const int nt = e->n_tasks - (s == 1 ? 0 : e->n_p1_tasks);
            if (s < 4) {
                st.a_next = A[s - 1];
                st.first = (s == 1);
                ens_stage_kernel<Real, COL_STAGE, TH><<<e->stage_grid, TH, e->stage_smem, e->stream>>>(mb, tl, nt, st, sy);
            } else {
                st.scheme = explicit_rk4 ? 1 : 0;
                ens_stage_kernel<Real, COL_FINAL, TH><<<e->stage_grid, TH, e->stage_smem, e->stream>>>(mb, tl, nt, st, sy);
            }
            e->launches++;
        }
        cudaError_t rf = cudaGetLastError();
        if (rf != cudaSuccess) return efail(e, NS2D_ERR_CUDA, cudaGetErrorString(rf));
        return NS2D_OK;
    }
    st.stage = 0;
    ens_launch_col<Real, COL_P1>(e, mb, st);
    e->launches++;
    for (int s = 1; s <= 4; ++s) {
        ens_launch_row<Real>(e, mb);
        e->launches++;
        st.stage = s;
        st.b_cur = explicit_rk4 ? B_ex[s - 1] : B_cn[s - 1];
        if (s < 4) {
            st.a_next = A[s - 1];
            st.first = (s == 1);
            ens_launch_col<Real, COL_STAGE>(e, mb, st);
        } else {
            st.scheme = explicit_rk4 ? 1 : 0;
            ens_launch_col<Real, COL_FINAL>(e, mb, st);
        }
        e->launches++;
    }
    cudaError_t r = cudaGetLastError();
    if (r != cudaSuccess) return efail(e, NS2D_ERR_CUDA, cudaGetErrorString(r));
    return NS2D_OK;
}

#define EDISPATCH(e, fn, ...) ((e)->fp32 ? fn<float>(__VA_ARGS__) : fn<double>(__VA_ARGS__))

// (Re)capture one step into a graph when dt or the grids changed.  Called only
// after an eager step at this dt, so the CN tables exist and the operator
// branch is settled: capturing records exactly the 9 pass launches.
ns2d_status ensure_graph(ns2d_ensemble* e, double dt) {
    if (e->exec && e->graph_dt == dt && e->graph_col_grid == e->col_grid && e->graph_row_grid == e->row_grid &&
        e->graph_col_var == e->col_var && e->graph_row_var == e->row_var && e->graph_fused == (int)e->fused &&
        e->graph_stage_grid == e->stage_grid)
        return NS2D_OK;
    if (e->exec) {
        cudaGraphExecDestroy(e->exec);
        cudaGraphDestroy(e->graph);
        e->exec = nullptr;
        e->graph = nullptr;
    }
    const int64_t l0 = e->launches;
    ECK(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    ns2d_status s = EDISPATCH(e, step_t, e, dt);
    cudaGraph_t g = nullptr;
    cudaError_t r = cudaStreamEndCapture(e->stream, &g);
    e->launches = l0;
    if (s) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (r != cudaSuccess) return efail(e, NS2D_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(r));
    r = cudaGraphInstantiate(&e->exec, g, 0);
    if (r != cudaSuccess) {
        cudaGraphDestroy(g);
        return efail(e, NS2D_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(r));
    }
    e->graph = g;
    e->graph_dt = dt;
    e->graph_col_grid = e->col_grid;
    e->graph_row_grid = e->row_grid;
    e->graph_col_var = e->col_var;
    e->graph_row_var = e->row_var;
    e->graph_fused = (int)e->fused;
    e->graph_stage_grid = e->stage_grid;
    return NS2D_OK;
}

bool branch_settled(const ns2d_ensemble* e) {
    int h = e->hyper_flag;
    const bool latch = (e->p.quirks & NS2D_QUIRK_HYPER_LATCH) != 0;
    const int b = ns2d::resolve_branch(h, e->p.ekmn_drag_flag, latch);
    return h == e->hyper_flag && (e->p.system == NS2D_EULER || e->cn_branch == b || e->p.integrator == NS2D_RK4);
}

ns2d_status step_async_impl(ns2d_ensemble* e, int nsteps, double dt, bool use_graph) {
    for (int k = 0; k < nsteps; ++k) {
        const bool ready = use_graph && (e->cn_dt == dt || e->p.integrator == NS2D_RK4 || e->p.system == NS2D_EULER) &&
                           branch_settled(e);
        if (!ready) {
            // eager step: builds the CN tables and settles the operator branch
            ns2d_status s = EDISPATCH(e, step_t, e, dt);
            if (s) return s;
            if (e->p.integrator == NS2D_RK4 || e->p.system == NS2D_EULER) e->cn_dt = dt;
            continue;
        }
        ns2d_status s = ensure_graph(e, dt);
        if (s) return s;
        ECK(e, cudaGraphLaunch(e->exec, e->stream));
        e->launches += e->fused ? 4 : 9;
    }
    return NS2D_OK;
}

ns2d_status check_impl(ns2d_ensemble* e) {
    int st[2] = {0, 0};
    ECK(e, cudaMemcpyAsync(st, e->status, sizeof(st), cudaMemcpyDeviceToHost, e->stream));
    ECK(e, cudaStreamSynchronize(e->stream));
    if (st[0] & 1) return efail(e, NS2D_ERR_BLOWUP, "non-finite vorticity in an ensemble member");
    if (st[0] & 4) return efail(e, NS2D_ERR_CUDA, "a per-stage launch waited past its bound for a member's tasks");
    if (st[0] & 8) return efail(e, NS2D_ERR_CUDA, "a column pass waited past its bound for its tile loads");
    return NS2D_OK;
}

template <typename Real>
ns2d_status set_t(ns2d_ensemble* e, int m, const double* host) {
    const int n = e->sizes[m], nyf = n / 2 + 1;
    ECK(e, cudaMemcpyAsync(e->io, host, sizeof(double2) * (size_t)n * nyf, cudaMemcpyHostToDevice, e->stream));
    pack_kernel<Real><<<148, 256, 0, e->stream>>>(e->io, (typename Cx<Real>::T*)e->state[m], n, nyf, e->ldc[m]);
    e->launches++;
    ECK(e, cudaGetLastError());
    ECK(e, cudaStreamSynchronize(e->stream));
    return NS2D_OK;
}

template <typename Real>
ns2d_status get_t(ns2d_ensemble* e, int m, double* host) {
    const int n = e->sizes[m], nyf = n / 2 + 1;
    unpack_kernel<Real><<<148, 256, 0, e->stream>>>((const typename Cx<Real>::T*)e->state[m], e->io, n, nyf, e->ldc[m]);
    e->launches++;
    ECK(e, cudaGetLastError());
    ECK(e, cudaMemcpyAsync(host, e->io, sizeof(double2) * (size_t)n * nyf, cudaMemcpyDeviceToHost, e->stream));
    ECK(e, cudaStreamSynchronize(e->stream));
    return NS2D_OK;
}

// Totals of ComputeSystemMeasurables for one member without the flux terms
// (they need the member's RHS; a single-trajectory handle provides them).
template <typename Real>
ns2d_status meas_t(ns2d_ensemble* e, int m, ns2d_measures* out) {
    using C = typename Cx<Real>::T;
    const int n = e->sizes[m];
    const int ns = (int)std::round(std::sqrt((double)(n / 2.0) * (n / 2.0) + (double)(n / 2.0) * (n / 2.0)) + 1);
    const size_t nout = DG_N + 8 * (size_t)ns;
    ECK(e, cudaMemsetAsync(e->ddiag, 0, sizeof(double) * nout, e->stream));
    DiagArgs<Real> d;
    std::memset(&d, 0, sizeof(d));
    d.state = (const C*)e->state[m];
    d.ldc = e->ldc[m];
    d.nx = n;
    d.ny = n;
    d.nyf = n / 2 + 1;
    const int drag = e->p.ekmn_drag_flag, hyper = e->hyper_flag;
    const int br = (hyper == 1 && drag == 1) ? 1 : (hyper != 1 && drag == 1) ? 2 : (hyper == 1) ? 3 : 4;
    d.lin = make_lin_params(e->p, br);
    d.enst_quirk = (e->p.quirks & NS2D_QUIRK_ENST_DISS) ? 1 : 0;
    d.n_spect = ns;
    d.out = e->ddiag;
    diag_kernel<Real><<<148, 256, sizeof(double) * (8 * (size_t)ns + DG_N * 8), e->stream>>>(d);
    e->launches++;
    ECK(e, cudaGetLastError());
    std::vector<double> raw(DG_N);
    ECK(e, cudaMemcpyAsync(raw.data(), e->ddiag, sizeof(double) * DG_N, cudaMemcpyDeviceToHost, e->stream));
    ECK(e, cudaStreamSynchronize(e->stream));
    const double norm_fac = 0.5 / std::pow((double)(n * n), 2.0);
    const double const_fac = 4.0 * std::pow(M_PI, 2.0);
    const double cn = const_fac * norm_fac;
    std::memset(out, 0, sizeof(*out));
    out->energy = raw[DG_E] * cn;
    out->enstrophy = raw[DG_Z] * cn;
    out->palinstrophy = raw[DG_P] * cn;
    out->divergence = raw[DG_DIV] * cn;
    out->energy_diss = raw[DG_EDISS] * (2.0 * cn);
    out->enstrophy_diss = raw[DG_ZDISS] * (2.0 * cn);
    return NS2D_OK;
}

double time_steps(ns2d_ensemble* e, double dt, int steps) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, e->stream);
    for (int k = 0; k < steps; ++k) EDISPATCH(e, step_t, e, dt);
    cudaEventRecord(b, e->stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / steps;
}

}  // namespace

extern "C" {

ns2d_status ns2d_ensemble_create(const ns2d_params* base, int32_t n_members, const int32_t* sizes, ns2d_ensemble** out) {
    if (!base || !sizes || !out || n_members < 1) return NS2D_ERR_INVALID;
    *out = nullptr;
    if (base->integrator != NS2D_RK4CN && base->integrator != NS2D_RK4) return NS2D_ERR_UNSUPPORTED;
    if (base->forcing == NS2D_FORCING_ZERO) return NS2D_ERR_UNSUPPORTED;  // mode killing: single handles only
    if (base->dealias_edge != 0) return NS2D_ERR_UNSUPPORTED;            // the solver's 2/3 edge only
    if (base->model != NS2D_MODEL_FULL && base->model != NS2D_MODEL_PHASE_ONLY) return NS2D_ERR_INVALID;
    if (base->precision != NS2D_FP64 && base->precision != NS2D_FP32) return NS2D_ERR_INVALID;
    for (int m = 0; m < n_members; ++m)
        if (!ens_size_ok(sizes[m])) return NS2D_ERR_UNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return NS2D_ERR_NO_DEVICE;
    ns2d_ensemble* e = new (std::nothrow) ns2d_ensemble();
    if (!e) return NS2D_ERR_NOMEM;
    e->p = *base;
    e->fp32 = base->precision == NS2D_FP32;
    e->n = n_members;
    e->sizes.assign(sizes, sizes + n_members);
    e->hyper_flag = base->hyper_visc_flag;
    if (cudaSetDevice(base->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete e;
        return NS2D_ERR_CUDA;
    }
    e->stream = e->own;
    ns2d_status s = EDISPATCH(e, create_t, e);
    if (s) {
        for (void* p : e->allocs) cudaFree(p);
        cudaStreamDestroy(e->own);
        delete e;
        return s;
    }
    *out = e;
    return NS2D_OK;
}

ns2d_status ns2d_ensemble_destroy(ns2d_ensemble* e) {
    if (!e) return NS2D_ERR_INVALID;
    cudaSetDevice(e->p.device);
    cudaStreamSynchronize(e->stream);
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    for (void* p : e->allocs) cudaFree(p);
    cudaStreamDestroy(e->own);
    delete e;
    return NS2D_OK;
}

const char* ns2d_ensemble_last_error(const ns2d_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }
int64_t ns2d_ensemble_launch_count(const ns2d_ensemble* e) { return e ? e->launches : -1; }

ns2d_status ns2d_ensemble_set_w_hat(ns2d_ensemble* e, int32_t member, const double* w_hat) {
    if (!e || !w_hat || member < 0 || member >= e->n) return NS2D_ERR_INVALID;
    cudaSetDevice(e->p.device);
    ns2d_status s = EDISPATCH(e, set_t, e, member, w_hat);
    if (s) return s;
    ECK(e, cudaMemsetAsync(e->status, 0, sizeof(int) * 4, e->stream));
    return NS2D_OK;
}

ns2d_status ns2d_ensemble_get_w_hat(ns2d_ensemble* e, int32_t member, double* w_hat) {
    if (!e || !w_hat || member < 0 || member >= e->n) return NS2D_ERR_INVALID;
    cudaSetDevice(e->p.device);
    return EDISPATCH(e, get_t, e, member, w_hat);
}

ns2d_status ns2d_ensemble_step_async(ns2d_ensemble* e, int32_t nsteps, double dt) {
    if (!e || nsteps < 0) return NS2D_ERR_INVALID;
    cudaSetDevice(e->p.device);
    return step_async_impl(e, nsteps, dt, true);
}

ns2d_status ns2d_ensemble_check(ns2d_ensemble* e) {
    if (!e) return NS2D_ERR_INVALID;
    cudaSetDevice(e->p.device);
    return check_impl(e);
}

ns2d_status ns2d_ensemble_step_n(ns2d_ensemble* e, int32_t nsteps, double dt) {
    ns2d_status s = ns2d_ensemble_step_async(e, nsteps, dt);
    if (s) return s;
    return check_impl(e);
}

ns2d_status ns2d_ensemble_measurables(ns2d_ensemble* e, int32_t member, ns2d_measures* out) {
    if (!e || !out || member < 0 || member >= e->n) return NS2D_ERR_INVALID;
    cudaSetDevice(e->p.device);
    return EDISPATCH(e, meas_t, e, member, out);
}

ns2d_status ns2d_ensemble_set_grids(ns2d_ensemble* e, int32_t col_grid, int32_t row_grid) {
    if (!e || col_grid < 1 || row_grid < 1) return NS2D_ERR_INVALID;
    e->col_grid = std::min(col_grid, e->n_col_items[e->col_var]);
    e->row_grid = std::min(row_grid, e->n_row_items[e->row_var]);
    return NS2D_OK;
}

ns2d_status ns2d_ensemble_set_shape(ns2d_ensemble* e, const ns2d_ensemble_shape* sh) {
    if (!e || !sh || sh->col_grid < 1 || sh->row_grid < 1 || sh->stage_launch < 0 || sh->stage_launch > 1 ||
        (sh->stage_launch && sh->stage_grid < 1))
        return NS2D_ERR_INVALID;
    int cv = -1, rv = -1;
    for (int v = 0; v < 2; ++v) {
        if (sh->col_threads == kEnsThreadChoices[v]) cv = v;
        if (sh->row_threads == kEnsThreadChoices[v]) rv = v;
    }
    if (cv < 0 || rv < 0) return NS2D_ERR_INVALID;
    e->col_var = cv;
    e->row_var = rv;
    e->col_grid = std::min(sh->col_grid, e->n_col_items[cv]);
    e->row_grid = std::min(sh->row_grid, e->n_row_items[rv]);
    e->fused = sh->stage_launch != 0;
    if (e->fused) e->stage_grid = std::min(sh->stage_grid, e->n_tasks);
    return NS2D_OK;
}

ns2d_status ns2d_ensemble_get_shape(const ns2d_ensemble* e, ns2d_ensemble_shape* sh) {
    if (!e || !sh) return NS2D_ERR_INVALID;
    sh->col_threads = kEnsThreadChoices[e->col_var];
    sh->col_grid = e->col_grid;
    sh->row_threads = kEnsThreadChoices[e->row_var];
    sh->row_grid = e->row_grid;
    sh->stage_launch = e->fused ? 1 : 0;
    sh->stage_grid = e->stage_grid;
    sh->col_items = e->n_col_items[e->col_var];
    sh->row_items = e->n_row_items[e->row_var];
    return NS2D_OK;
}

ns2d_status ns2d_ensemble_tune(ns2d_ensemble* e, double dt, int32_t* col_grid, int32_t* row_grid) {
    if (!e) return NS2D_ERR_INVALID;
    cudaSetDevice(e->p.device);
    // Autotuner: for each pass (the four column launches, then the four row
    // launches of a step), the block size -- which sets the tile shape: ky
    // columns per column tile and row pairs per row block of every member --
    // and the persistent grid as a multiple of the SM count (1..8 blocks per
    // SM, capped by the item count), chosen by timing full steps.  Steps taken
    // here advance the members; callers re-set their states.
    const int saved_hyper = e->hyper_flag;
    e->fused = false;
    EDISPATCH(e, step_t, e, dt);  // settle tables and the operator branch
    cudaStreamSynchronize(e->stream);
    const int mults[] = {1, 2, 3, 4, 6, 8};
    int best_cv = e->col_var, best_rv = e->row_var, best_c = e->col_grid, best_r = e->row_grid;
    double best = time_steps(e, dt, 3);
    for (int pass = 0; pass < 2; ++pass) {
        for (int v = 0; v < 2; ++v) {
            for (int k : mults) {
                if (pass == 0) {
                    e->col_var = v;
                    e->col_grid = std::min(k * e->nsm, e->n_col_items[v]);
                } else {
                    e->row_var = v;
                    e->row_grid = std::min(k * e->nsm, e->n_row_items[v]);
                }
                const double ms = time_steps(e, dt, 3);
                if (ms < best) {
                    best = ms;
                    if (pass == 0) {
                        best_cv = v;
                        best_c = e->col_grid;
                    } else {
                        best_rv = v;
                        best_r = e->row_grid;
                    }
                }
            }
        }
        if (pass == 0) {
            e->col_var = best_cv;
            e->col_grid = best_c;
        } else {
            e->row_var = best_rv;
            e->row_grid = best_r;
        }
    }
    // one persistent launch per RK stage, 1..(resident blocks per SM) x SMs
    bool best_fused = false;
    int best_sg = e->stage_grid;
    e->fused = true;
    for (int k = 1; k <= e->stage_per_sm; ++k) {
        e->stage_grid = std::min(k * e->nsm, e->n_tasks);
        const double ms = time_steps(e, dt, 3);
        if (ms < best) {
            best = ms;
            best_fused = true;
            best_sg = e->stage_grid;
        }
    }
    e->fused = best_fused;
    e->stage_grid = best_sg;
    e->hyper_flag = saved_hyper;
    cudaError_t r = cudaGetLastError();
    if (r != cudaSuccess) return efail(e, NS2D_ERR_CUDA, cudaGetErrorString(r));
    if (col_grid) *col_grid = best_c;
    if (row_grid) *row_grid = best_r;
    return NS2D_OK;
}

ns2d_status ns2d_ensemble_set_stream(ns2d_ensemble* e, void* stream) {
    if (!e) return NS2D_ERR_INVALID;
    ECK(e, cudaStreamSynchronize(e->stream));
    e->stream = stream ? (cudaStream_t)stream : e->own;
    if (e->exec) {
        cudaGraphExecDestroy(e->exec);
        cudaGraphDestroy(e->graph);
        e->exec = nullptr;
        e->graph = nullptr;
    }
    return NS2D_OK;
}

}  // extern "C"
