// ensemble.cuh -- many independent trajectories of uneven grid sizes advanced
// together: one launch per pass covers every member.  A launch walks a list
// of work items (member, tile) with a persistent grid; each item runs the same
// column or row body as the single-trajectory kernels, instantiated for the
// member's grid size.  All bodies use blocks of kEnsThreads threads, so one
// launch can mix sizes.
#pragma once
#include "kernels.cuh"

namespace ns2d {

// Block sizes of the ensemble kernels (one per launch, every member size), and
// the tile shapes they give: a block of THREADS threads covers THREADS / T
// ky columns of a member in a column pass and THREADS / (2 T) row pairs in a
// row pass (T = the threads of one transform of that size).  The autotuner
// picks the block size of each pass; 256 threads measured 12 % faster than
// 128 on the 64-member FP32 benchmark ensemble (the 512^2 members' column
// tiles grow from 2 to 4 columns, the 128^2 / 256^2 ones from 8 to 16).
constexpr int kEnsThreadChoices[2] = {256, 128};
template <int N, int THREADS>
struct EnsShape {
    static constexpr int T = Plan<N>::T;
    static constexpr int TC = THREADS / T;          // columns per column tile
    static constexpr int PAIRS = THREADS / (2 * T);  // row pairs per row block
    static_assert(TC >= 1 && PAIRS >= 1, "ensemble sizes need T <= THREADS / 2");
};

#define NS2D_ENS_SIZES(X) X(64) X(128) X(256) X(512)

template <typename Real>
struct EnsMember {
    ColArgs<Real> col;                    // member pointers and per-size constants
    RowArgs<Real> row;
    typename Cx<Real>::T* col0[2];        // column 0 of successive stage inputs
    int n;
};

struct EnsItem {
    int member;
    int tile;
};

// Per-launch stage parameters shared by all members.
struct EnsStage {
    double dt, a_next, b_cur;
    int first, scheme, conj_quirk, stage;  // stage 1..4; 0 = P1 of the step
    LinOp lin;
    int* status;
};

template <typename Real>
__device__ __forceinline__ void ens_apply_stage(ColArgs<Real>& a, const EnsMember<Real>& mb, const EnsStage& st) {
    a.dt = st.dt;
    a.a_next = st.a_next;
    a.b_cur = st.b_cur;
    a.first = st.first;
    a.scheme = st.scheme;
    a.lin = st.lin;
    a.final_tail = 0;
    a.status = st.status;
    if (st.stage >= 1) {
        // a.src is the member's product spectrum (set at creation)
        a.conj_mode = (st.conj_quirk || st.stage == 1) ? 1 : 0;
        if (st.stage == 1) {
            a.conj_src = a.state;
            a.conj_stride = a.ldc;
        } else {
            a.conj_src = mb.col0[(st.stage - 1) & 1];
            a.conj_stride = 1;
        }
        a.col0_out = mb.col0[st.stage & 1];
    } else {
        a.src = a.state;
        a.col0_out = nullptr;
    }
}

// Resident blocks per SM the ensemble kernels are compiled for: at most 128
// registers a thread in FP32 (two 256-thread or four 128-thread blocks), the
// register need of one FP64 body otherwise.
template <typename Real, int THREADS>
struct EnsMinBlocks {
    static constexpr int value = sizeof(Real) == 4 ? 512 / THREADS : 256 / THREADS;
};

// TMA (with FAST): the tiles move by TMA copies through maps[2 m + v], the
// tensor maps of member m for this block size (v = 0 for kEnsThreadChoices[0],
// 1 for the other); shared memory EnsSmem::col_tma().  A tile whose loads do
// not land within their bound stops the block (status bit 8).
template <typename Real, int MODE, int THREADS, bool FAST = false, bool TMA = false>
__global__ void __launch_bounds__(THREADS, (EnsMinBlocks<Real, THREADS>::value)) ens_col_kernel(const EnsMember<Real>* __restrict__ members,
                                                      const EnsItem* __restrict__ items, int nitems, EnsStage st,
                                                      const ColMaps* __restrict__ maps) {
    extern __shared__ __align__(16) unsigned char smraw[];
    if (block_should_exit(st.status)) return;
    unsigned char* sm = smraw;
    if constexpr (TMA) sm = smraw + ((1024u - ((unsigned)__cvta_generic_to_shared(smraw) & 1023u)) & 1023u);
    constexpr int VI = THREADS == kEnsThreadChoices[0] ? 0 : 1;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const EnsItem item = items[it];
        const EnsMember<Real>& mb = members[item.member];
        ColArgs<Real> a = mb.col;
        ens_apply_stage(a, mb, st);
        const ColMaps* mp = TMA ? maps + 2 * item.member + VI : nullptr;
        bool go = true;
        switch (mb.n) {
#define NS2D_ENS_COL(NN)                                                                           \
    case NN:                                                                                       \
        go = col_body<Real, NN, EnsShape<NN, THREADS>::TC, MODE, FAST, TMA>(a, item.tile, sm, mp); \
        break;
            NS2D_ENS_SIZES(NS2D_ENS_COL)
#undef NS2D_ENS_COL
            default: break;
        }
        if (!go) return;
    }
}

template <typename Real, int THREADS>
__global__ void __launch_bounds__(THREADS, (EnsMinBlocks<Real, THREADS>::value)) ens_row_kernel(const EnsMember<Real>* __restrict__ members,
                                                      const EnsItem* __restrict__ items, int nitems, int* status) {
    extern __shared__ __align__(16) unsigned char smraw[];
    if (block_should_exit(status)) return;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const EnsItem item = items[it];
        const EnsMember<Real>& mb = members[item.member];
        switch (mb.n) {
#define NS2D_ENS_ROW(NN)                                                                  \
    case NN:                                                                              \
        row_body<Real, NN, EnsShape<NN, THREADS>::PAIRS, false>(mb.row, item.tile, smraw); \
        break;
            NS2D_ENS_SIZES(NS2D_ENS_ROW)
#undef NS2D_ENS_ROW
            default: break;
        }
    }
}

// ---------------------------------------------------------------------------
// One persistent launch per RK stage.  Launch s (s = 1..4) walks one task list
// -- the column tiles of the first column pass (s = 1 only), then the row
// blocks of stage s, then the column tiles of stage s, every member's tasks
// largest member first -- through a work counter, so tasks are handed out in
// list order to the blocks that run.  A task of member m waits only for the
// tasks of m earlier in the same list (its row blocks for the first pass's
// column tiles, its column tiles for its row blocks): those were handed out
// before it, to blocks that are running, so every wait ends; members do not
// wait for each other, and one member's rows overlap another's columns.
// Each wait is bounded (about 2 s); when a bound is reached the block sets
// status bit 4 and the launch stops.
struct EnsTask {
    int kind;    // 0: first column pass tile, 1: row block, 2: column tile of the stage
    int member;
    int tile;
};

struct EnsSync {
    int* head;          // [4] work counters of the stage launches
    int* done;          // [5][nmem]: [0] first-pass column tiles done, [s] row blocks of stage s done
    const int* need;    // [nmem][2]: column tiles, row blocks of each member
    int nmem;
};

__device__ __forceinline__ bool ens_wait_count(const int* cnt, int need, int* status) {
    long long spins = 0;
    while (*(volatile const int*)cnt < need) {
        if (++spins > (1LL << 24)) {
            atomicOr(status, 4);
            return false;
        }
        __nanosleep(128);
    }
    __threadfence();
    return true;
}

template <typename Real, int MODE, int THREADS>
__global__ void __launch_bounds__(THREADS, (EnsMinBlocks<Real, THREADS>::value))
    ens_stage_kernel(const EnsMember<Real>* __restrict__ members, const EnsTask* __restrict__ tasks, int ntasks,
                     EnsStage st, EnsSync sy) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ int s_task, s_ok;
    if (block_should_exit(st.status)) return;
    for (;;) {
        if (threadIdx.x == 0) s_task = atomicAdd(sy.head + (st.stage - 1), 1);
        __syncthreads();
        const int it = s_task;
        if (it >= ntasks) return;
        const EnsTask task = tasks[it];
        const EnsMember<Real>& mb = members[task.member];
        // inputs of this task produced earlier in this launch
        if (threadIdx.x == 0) {
            bool ok = true;
            if (task.kind == 1 && st.stage == 1)
                ok = ens_wait_count(sy.done + task.member, sy.need[2 * task.member], st.status);
            else if (task.kind == 2)
                ok = ens_wait_count(sy.done + (size_t)st.stage * sy.nmem + task.member, sy.need[2 * task.member + 1],
                                    st.status);
            s_ok = ok ? 1 : 0;
        }
        __syncthreads();
        if (!s_ok) return;
        if (task.kind == 1) {
            switch (mb.n) {
#define NS2D_ENS_SROW(NN)                                                                 \
    case NN:                                                                              \
        row_body<Real, NN, EnsShape<NN, THREADS>::PAIRS, false>(mb.row, task.tile, smraw); \
        break;
                NS2D_ENS_SIZES(NS2D_ENS_SROW)
#undef NS2D_ENS_SROW
                default: break;
            }
        } else {
            ColArgs<Real> a = mb.col;
            EnsStage sc = st;
            if (task.kind == 0) sc.stage = 0;
            ens_apply_stage(a, mb, sc);
            switch (mb.n) {
#define NS2D_ENS_SCOL(NN)                                                                          \
    case NN:                                                                                       \
        if (task.kind == 0) {                                                                      \
            col_body<Real, NN, EnsShape<NN, THREADS>::TC, COL_P1>(a, task.tile, smraw);            \
        } else {                                                                                   \
            col_body<Real, NN, EnsShape<NN, THREADS>::TC, MODE>(a, task.tile, smraw);              \
        }                                                                                          \
        break;
                NS2D_ENS_SIZES(NS2D_ENS_SCOL)
#undef NS2D_ENS_SCOL
                default: break;
            }
        }
        // this task's outputs are written: every thread fences its stores, then
        // the task is counted for the tasks that wait on it
        if (task.kind < 2) {
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) atomicAdd(sy.done + (size_t)(task.kind == 0 ? 0 : st.stage) * sy.nmem + task.member, 1);
        }
        __syncthreads();
    }
}

template <typename Real, int THREADS>
struct EnsSmem {
    static size_t col() {
        size_t m = 0;
#define NS2D_ENS_CS(NN)                                                                       \
    m = m > ColSmem<Real, NN, EnsShape<NN, THREADS>::TC>::bytes() ? m                         \
                                                                  : ColSmem<Real, NN, EnsShape<NN, THREADS>::TC>::bytes();
        NS2D_ENS_SIZES(NS2D_ENS_CS)
#undef NS2D_ENS_CS
        return m;
    }
    static size_t row() {
        size_t m = 0;
#define NS2D_ENS_RS(NN)                                                                              \
    m = m > RowSmem<Real, NN, 2 * EnsShape<NN, THREADS>::PAIRS>::bytes()                             \
            ? m                                                                                      \
            : RowSmem<Real, NN, 2 * EnsShape<NN, THREADS>::PAIRS>::bytes();
        NS2D_ENS_SIZES(NS2D_ENS_RS)
#undef NS2D_ENS_RS
        return m;
    }
    // the TMA column kernels: three exchange-sized regions and 1 KB of alignment
    static size_t col_tma() {
        size_t m = 0;
#define NS2D_ENS_CT(NN)                                                                           \
    m = m > ColSmem<Real, NN, EnsShape<NN, THREADS>::TC>::bytes_tma() ? m                          \
                                                                      : ColSmem<Real, NN, EnsShape<NN, THREADS>::TC>::bytes_tma();
        NS2D_ENS_SIZES(NS2D_ENS_CT)
#undef NS2D_ENS_CT
        return m + 1024;
    }
    static size_t stage() { return col() > row() ? col() : row(); }
};

}  // namespace ns2d
