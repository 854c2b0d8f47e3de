// kernels.cuh -- the two passes of one nonlinear-term evaluation (sm_100a).
//
// The reference evaluates the RHS (Solver/src/solver.c:884-1032) as
//   u_hat, v_hat -> batched c2r; w_x, w_y -> batched c2r; product; r2c;
//   normalise; dealias; force; ForceConjugacy
// with FFTW-MPI doing each 2-D transform as an x pass and a y pass.  Here the
// same arithmetic is split into two HBM passes per evaluation:
//
//   column pass (x direction, tiles of TC ky-columns, all kx rows):
//     [forward x-FFT of the previous product + normalise/dealias/force/
//      conjugacy + RK stage combine]  ->  derived spectra of the next stage
//     input (i ky/k^2 X, -i kx/k^2 X, i kx X, i ky X)  ->  four inverse x-FFTs
//   row pass (y direction, pairs of x rows):
//     Z1 = U + iV, Z2 = WX + iWY (Hermitian extension in y) -> two inverse
//     y-FFTs give u, v, w_x, w_y in real space; n = u w_x + v w_y; the two
//     rows' products are packed into one forward y-FFT and split into the two
//     half spectra.
//
// Spectral arrays are [nx][ldc] complex (row = kx index as in the reference,
// ldc >= ny/2+1); the intermediate "x-space" arrays use the same shape with
// the row index meaning x.
#pragma once
#include <cuda.h>  // CUtensorMap (type only)

#include "fft.cuh"

namespace ns2d {

enum ColMode : int { COL_P1 = 0, COL_RHS = 1, COL_STAGE = 2, COL_FINAL = 3 };

// Linear-operator bracket selection (Solver/src/solver.c:839-856):
// 1: nu k^2p + a k^2q, 2: nu k^2 + a k^2q, 3: nu k^2p, 4: nu k^2.
struct LinOp {
    double nu, alpha, hp, dp;
    int branch;
    int hp_int, dp_int;  // exponents when integral, else INT_MIN
};

// Out of line: the callers sit in fully unrolled per-element loops, and one
// shared copy of this code keeps the kernels inside the instruction cache.
static __device__ __noinline__ double pow_general(double x, double p) { return pow(x, p); }

__device__ __forceinline__ double powk(double k2, double p, int pint) {
    if (pint != -2147483647 - 1) {
        int e = pint < 0 ? -pint : pint;
        double r = 1.0, b = k2;
        while (e) {
            if (e & 1) r *= b;
            b *= b;
            e >>= 1;
        }
        return pint < 0 ? 1.0 / r : r;
    }
    return pow_general(k2, p);
}

__device__ __forceinline__ double lin_bracket(const LinOp& L, double k2) {
    switch (L.branch) {
        case 1: return L.nu * powk(k2, L.hp, L.hp_int) + L.alpha * powk(k2, L.dp, L.dp_int);
        case 2: return L.nu * k2 + L.alpha * powk(k2, L.dp, L.dp_int);
        case 3: return L.nu * powk(k2, L.hp, L.hp_int);
        default: return L.nu * k2;
    }
}

template <typename Real>
struct ColArgs {
    using C = typename Cx<Real>::T;
    const C* src;        // COL_P1: spectral input X; else: product spectrum n(x, ky)
    C* state;            // w_hat
    C* acc;              // RK accumulator
    C* out;              // COL_STAGE: full next-stage input (explicit RK4 only), may be null
    C* rhs_store;        // any non-P1 mode: this evaluation's RHS, may be null
    C* f0;               // COL_P1/STAGE outputs (x-space): U, V, WX, WY
    C* f1;
    C* f2;
    C* f3;
    const C* conj_src;   // column 0 of the RHS input (stride conj_stride)
    int conj_stride;
    C* col0_out;         // COL_STAGE: column 0 of the next stage input (stride 1)
    const C* tw;         // exp(-2 pi i m / N), m < N
    const C* xin;        // RK4 explicit: stage input for the +D X term (stride ldc), may be null
    int ldc, nyf;
    int kmax_sqr;        // (int)(N/3)^2 for the 2/3 rule
    int dealias;         // 0: 2/3, 1: Hou-Li
    int houli_int;       // integer k/(N/2) (reference quirk)
    int kolm;            // zero the kx = 0 row (2/3 + KOLM)
    int force_i, force_j;
    C force_val;
    int has_force;
    Real norm2;          // (1/(Nx Ny))^2
    int conj_mode;       // 0: none, 1: write the state's column 0 from conj_src
    // stage combine
    double dt;
    double a_next;       // next stage input = state + (dt a_next) rhs
    double b_cur;        // accumulator coefficient of this stage's RHS
    int first;           // acc = b rhs (instead of acc += b rhs)
    int scheme;          // 0: RK4CN, 1: explicit RK4 (Euler or __RK4), 2: AB4 + CN, 3: AB4 explicit
    const C* h0;         // AB4 history: RHS of steps n-3, n-2, n-1 (AB_tmp_nonlin[0..2])
    const C* h1;
    const C* h2;
    int lin_stage;       // 0 none, 1: rhs += dt D X (quirk), 2: rhs -= D X (corrected)
    LinOp lin;
    const double2* cn;   // COL_FINAL, CN schemes: per-mode ((2-D)/(2+D), 2dt/(2+D)), stride ldc
    const C* force_field;  // forcing added to every mode of the RHS ([nx][ldc]), may be null
    double inv_nxny;     // 1/(Nx Ny)
    int final_tail;      // COL_FINAL: 1 = SystemCheck bound over ntiles tiles, 0 = non-finite check only
    int phase_only;      // COL_FINAL: rescale each updated mode k != 0 to the amplitude it had before
    int ntiles;          // number of column tiles of this field
    int* status;         // [0] status bits (kernels return early when set), [1] completed steps
};

// Early exit once the device status word is set (a failed SystemCheck).  One
// thread reads the word and the block agrees on it through shared memory, so
// every thread of a block takes the same path past the barriers that follow.
__device__ __forceinline__ bool block_should_exit(const int* status) {
    __shared__ int flag;
    if (threadIdx.x == 0) flag = status ? *(volatile const int*)status : 0;
    __syncthreads();
    const bool out = flag != 0;
    __syncthreads();
    return out;
}

template <typename Real>
__device__ __noinline__ Real houli_filter(int kx, int ky, int nx, int ny, int quirk) {
    double fx, fy;
    if (quirk) {
        fx = (double)(kx / (nx / 2));
        fy = (double)(ky / (ny / 2));
    } else {
        fx = (double)kx / (double)(nx / 2);
        fy = (double)ky / (double)(ny / 2);
    }
    double r2 = fx * fx + fy * fy;
    double r36 = r2 * r2;          // r^4
    r36 = r36 * r36;               // r^8
    r36 = r36 * r36;               // r^16
    r36 = r36 * r36 * r2;          // r^34
    r36 = r36 * r2;                // r^36
    double e = 36.0 * r36;
    if (e < 1e-17) return (Real)1;
    return (Real)exp(-e);
}

// Hint that a global line will be read soon (PTX prefetch.global.L2).
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Asynchronous global -> shared copies (cp.async, sm_80+ PTX).
template <typename C>
__device__ __forceinline__ void cp_async_elem(C* smem, const C* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(C) == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Tensor maps of the arrays a column pass moves by TMA tile copies: the four
// x-space fields, the RK accumulator, the state and the product spectrum (the
// stage and final passes' input), each a 2-D array of nx rows by 2*nyf reals
// (row stride ldc complex) with boxes of (2*TC reals, min(nx, 256) rows), i.e.
// one column tile in the [row][TC] order of the staging buffers.  Columns at or
// past nyf lie outside the maps: loads read zeros there and stores clip them.
struct ColMaps {
    CUtensorMap f[4];
    CUtensorMap acc;
    CUtensorMap state;
    CUtensorMap nl;
};

// Bulk-async (TMA) tile stores, shared memory -> global.  The staging writes of
// every thread are made visible to the async proxy (fence) and joined by a
// barrier before one thread issues the copies.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// the shared-memory sources of all committed stores have been read
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
// all committed stores have completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// mbarrier helpers for the TMA tile loads (one barrier per group of loads,
// used once per block: phase 0).
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// Invalidate `bar` (every thread is past its last wait on it) so that the
// same shared memory can hold a fresh barrier for the next tile.
__device__ __forceinline__ void mbar_inval(unsigned long long* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}
// Bounded wait for phase 0 of `bar`: false if the loads have not landed after
// 2^22 polls (each poll may suspend the thread for a while in hardware).
__device__ __forceinline__ bool mbar_wait0(unsigned long long* bar) {
    const unsigned a = smem_addr(bar);
    for (int it = 0; it < (1 << 22); ++it) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Load column tile `tile` through `map` into dst ([N][TC] complex, dense),
// completing on `bar` (whose expected byte count covers it).
template <typename C, int N, int TC>
__device__ __forceinline__ void tma_load_tile(const CUtensorMap* map, int tile, C* dst, unsigned long long* bar) {
    constexpr int BR = N < 256 ? N : 256;
    static_assert(((TC * sizeof(C)) % 16) == 0, "TMA x extent must be a multiple of 16 bytes");
    const int x = tile * TC * 2;  // in reals: a multiple of 16 bytes
#pragma unroll
    for (int q = 0; q < N / BR; ++q) {
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
                smem_addr(dst + (size_t)q * BR * TC)),
            "l"(map), "r"(x), "r"(q * BR), "r"(smem_addr(bar))
            : "memory");
    }
}

// Store column tile `tile` ([N][TC] complex, dense, at stg) through `map`.
template <typename C, int N, int TC>
__device__ __forceinline__ void tma_store_tile(const CUtensorMap* map, int tile, const C* stg) {
    constexpr int BR = N < 256 ? N : 256;
    static_assert(((TC * sizeof(C)) % 16) == 0, "TMA x extent must be a multiple of 16 bytes");
    const int x = tile * TC * 2;  // in reals: a multiple of 16 bytes
#pragma unroll
    for (int q = 0; q < N / BR; ++q) {
        const unsigned src = (unsigned)__cvta_generic_to_shared(stg + (size_t)q * BR * TC);
        asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(map),
                     "r"(x), "r"(q * BR), "r"(src)
                     : "memory");
    }
}

// Shared memory of the column pass: two FFT exchange buffers (the second one
// first holds the prefetched RK accumulator), then the [N][TC] staging array
// of the state, which becomes the next stage input X.
template <typename Real, int N, int TC>
struct ColSmem {
    using C = typename Cx<Real>::T;
    static constexpr int FFT = SmemLayout<N, TC>::ELEMS;
    static constexpr int PRE = N * TC;
    static_assert(FFT >= PRE, "accumulator staging must fit the second exchange buffer");
    static constexpr size_t bytes() { return sizeof(C) * (size_t)(2 * FFT + PRE); }
    // the TMA form: the third region is a full exchange buffer too (the second
    // inverse pair transforms in it while the first pair's stores drain)
    static constexpr size_t bytes_tma() { return sizeof(C) * (size_t)(3 * FFT); }
};

// 1/k^2 for the velocity spectra, k2 = kx^2 + ky^2 >= 1 held exactly.  FP64:
// Newton-Raphson for the reciprocal, r <- r + r (1 - k2 r), twice from the
// hardware approximation (PTX rcp.approx.ftz.f64, relative error far below
// 2^-14, so two quadratic steps leave about one rounding of FP64); the FP32
// form is the correctly rounded single-precision reciprocal.
template <typename Real>
__device__ __forceinline__ Real inv_k2(Real k2);
template <>
__device__ __forceinline__ double inv_k2<double>(double k2) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(k2));
    r = fma(r, fma(-k2, r, 1.0), r);
    r = fma(r, fma(-k2, r, 1.0), r);
    return r;
}
template <>
__device__ __forceinline__ float inv_k2<float>(float k2) { return __frcp_rn(k2); }

// kx of transform element m (row i = t + T m of an N-row column) as a real:
// i for i <= N/2, i - N above; tr = (Real)t.  m is a compile-time index in the
// unrolled loops, so only the element that can hold i = N/2 needs a select.
template <typename Real, int N, int T>
__device__ __forceinline__ Real kx_of(int m, int t, Real tr) {
    constexpr int H = N / (2 * T);
    if (m < H) return tr + (Real)(T * m);
    if (m > H) return tr + (Real)(T * m - N);
    return t == 0 ? (Real)(N / 2) : tr + (Real)(T * m - N);
}

// Derived spectra of the stage input X at (kx, ky) (solver.c:904-957), two at a
// time: pair 0 gives u = i ky/k^2 X and v = -i kx/k^2 X (one reciprocal), pair 2
// gives w_x = i kx X and w_y = i ky X.  Zero at the mean mode.  kx and ky are
// integers held as reals.
template <typename C>
__device__ __forceinline__ void derived_pair(int fp, decltype(C::x) kx, decltype(C::x) ky, C X, C& a, C& b) {
    using Real = decltype(C::x);
    if (kx == (Real)0 && ky == (Real)0) {
        a = cmake<C>(0, 0);
        b = a;
        return;
    }
    Real sa, sb;
    if (fp == 0) {
        const Real inv = inv_k2<Real>(kx * kx + ky * ky);
        sa = ky * inv;
        sb = -kx * inv;
    } else {
        sa = kx;
        sb = ky;
    }
    // i s X = (-s X.y, s X.x)
    a = cmake<C>(-sa * X.y, sa * X.x);
    b = cmake<C>(-sb * X.y, sb * X.x);
}

// Derived spectra of the stage input X (pre0, [N][TC] in shared memory) and
// their four inverse x-FFTs into f0..f3, two at a time (one copy of the
// transform code serves both pairs).
template <typename Real, int N, int TC>
__device__ __forceinline__ void derived_ifft(const typename Cx<Real>::T* pre0, typename Cx<Real>::T* sm,
                                          typename Cx<Real>::T* f0, typename Cx<Real>::T* f1,
                                          typename Cx<Real>::T* f2, typename Cx<Real>::T* f3, int ldc, int ky,
                                          bool valid, int t, int c, TwSeed<typename Cx<Real>::T> seed) {
    using C = typename Cx<Real>::T;
    constexpr int T = Plan<N>::T;
    constexpr int E = N / T;
    C* outs[4] = {f0, f1, f2, f3};
    const Real tr = (Real)t, kyr = (Real)ky;
#pragma unroll 1
    for (int fp = 0; fp < 4; fp += 2) {
        C v[2][E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            derived_pair(fp, kx_of<Real, N, T>(m, t, tr), kyr, pre0[i * TC + c], v[0][m], v[1][m]);
        }
        fft_batched<N, +1, 2>(v, IlvPolicy<N, TC, C>{sm, c}, seed, t);
        if (valid) {
            C* __restrict__ o0 = outs[fp];
            C* __restrict__ o1 = outs[fp + 1];
#pragma unroll
            for (int m = 0; m < E; ++m) {
                o0[(size_t)(t + T * m) * ldc + ky] = v[0][m];
                o1[(size_t)(t + T * m) * ldc + ky] = v[1][m];
            }
        }
    }
}

// derived_ifft with TMA stores.  The three shared regions B0 = sm, B1 = sm +
// STRIDE and B2 = pre0 (sized as an exchange buffer in this form) rotate.  The
// first pair (U, V) transforms batched in (B0, B1) and is staged there, each
// field stored by its own bulk-async group.  The second pair (WX, WY) runs as
// two single transforms: WX in B2 (the stage input, free once both spectra are
// formed), WY in B0 as soon as the U store has read it; so the first pair's
// stores drain under the second pair's transforms and only WY's store is left
// to drain at the end.  Without SPLIT the second pair transforms batched in
// (B2, B0) instead (a persistent caller's next tile overlaps the drain, and the
// batched pair keeps the transforms' ILP).  pending: a store issued before
// this call still reads B1 (the accumulator).  Thread 0 returns once all
// stores have completed.
template <typename Real, int N, int TC, bool SPLIT>
__device__ __forceinline__ void derived_ifft_tma(typename Cx<Real>::T* pre0, typename Cx<Real>::T* sm,
                                                 const ColMaps* maps, int tile, int ky, int t, int c,
                                                 TwSeed<typename Cx<Real>::T> seed, bool pending) {
    using C = typename Cx<Real>::T;
    constexpr int T = Plan<N>::T;
    constexpr int E = N / T;
    constexpr int STRIDE = SmemLayout<N, TC>::ELEMS;
    const Real tr = (Real)t, kyr = (Real)ky;
    C* const B0 = sm;
    C* const B1 = sm + STRIDE;
    C* const B2 = pre0;
    if constexpr (!SPLIT) {
        // both pairs batched, one copy of the transform code: (B0, B1), then (B2, B0)
#pragma unroll 1
        for (int fp = 0; fp < 4; fp += 2) {
            C v[2][E];
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int i = t + T * m;
                derived_pair(fp, kx_of<Real, N, T>(m, t, tr), kyr, pre0[i * TC + c], v[0][m], v[1][m]);
            }
            // first pair: the accumulator store (if any) must have read B1;
            // second pair: the first pair's first field must have left B0 (at
            // most its second group still pending), and every thread has read B2
            if (fp == 0 ? pending : true) {
                if (threadIdx.x == 0) {
                    if (fp == 0) bulk_wait_read_all();
                    else asm volatile("cp.async.bulk.wait_group.read 1;\n" ::: "memory");
                }
                __syncthreads();
            }
            C* const Pa = fp == 0 ? B0 : B2;
            C* const Pb = fp == 0 ? B1 : B0;
            fft_batched<N, +1, 2>(v, IlvPairPolicy<N, TC, C>{Pa, Pb, c}, seed, t);
#pragma unroll
            for (int m = 0; m < E; ++m) {
                Pa[(t + T * m) * TC + c] = v[0][m];
                Pb[(t + T * m) * TC + c] = v[1][m];
            }
            fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                tma_store_tile<C, N, TC>(&maps->f[fp], tile, Pa);
                bulk_commit();
                tma_store_tile<C, N, TC>(&maps->f[fp + 1], tile, Pb);
                bulk_commit();
            }
        }
    } else {
        {
            C v[2][E];
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int i = t + T * m;
                derived_pair(0, kx_of<Real, N, T>(m, t, tr), kyr, pre0[i * TC + c], v[0][m], v[1][m]);
            }
            if (pending) {  // the accumulator store must have read B1
                if (threadIdx.x == 0) bulk_wait_read_all();
                __syncthreads();
            }
            fft_batched<N, +1, 2>(v, IlvPairPolicy<N, TC, C>{B0, B1, c}, seed, t);
#pragma unroll
            for (int m = 0; m < E; ++m) {
                B0[(t + T * m) * TC + c] = v[0][m];
                B1[(t + T * m) * TC + c] = v[1][m];
            }
            fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                tma_store_tile<C, N, TC>(&maps->f[0], tile, B0);
                bulk_commit();
                tma_store_tile<C, N, TC>(&maps->f[1], tile, B1);
                bulk_commit();
            }
        }
        C v[2][E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            derived_pair(2, kx_of<Real, N, T>(m, t, tr), kyr, pre0[i * TC + c], v[0][m], v[1][m]);
        }
        __syncthreads();  // every thread has read B2
#pragma unroll 1
        for (int b = 0; b < 2; ++b) {
            C* const P = b == 0 ? B2 : B0;
            if (b == 1) {  // the U store (the oldest group) must have read B0
                if (threadIdx.x == 0) asm volatile("cp.async.bulk.wait_group.read 2;\n" ::: "memory");
                __syncthreads();
            }
            C u[1][E];
#pragma unroll
            for (int m = 0; m < E; ++m) u[0][m] = b == 0 ? v[0][m] : v[1][m];
            fft_batched<N, +1, 1>(u, IlvPairPolicy<N, TC, C>{P, P, c}, seed, t);
#pragma unroll
            for (int m = 0; m < E; ++m) P[(t + T * m) * TC + c] = u[0][m];
            fence_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                tma_store_tile<C, N, TC>(&maps->f[2 + b], tile, P);
                bulk_commit();
            }
        }
    }
    if (threadIdx.x == 0) bulk_wait_all();
}

// Column pass on tile `tile` (ky columns tile*TC .. tile*TC+TC-1), by the T*TC
// threads of a block, thread (t, c) with c = threadIdx.x % TC.  Shared memory:
// ColSmem::bytes().  Ends with the block synchronised (the shared memory may be
// reused for another tile).
// TMA (with FAST, modes P1, STAGE and FINAL): the pass's inputs (a.src, a.state,
// a.acc) arrive by TMA tile loads and its outputs (the x-space fields, the
// accumulator, the final state) leave by bulk-async tile stores, through `maps`
// (which must describe those arrays), instead of per-thread copies; smraw
// 1024-byte aligned; SPLIT: the last inverse pair as two single transforms
// (derived_ifft_tma).  Its mbarriers are invalidated once used, so a persistent
// caller can run the body again on the same shared memory.  A load that does
// not land within its bound sets status bit 8 and the body returns false (the
// block must stop); otherwise it returns true.
template <typename Real, int N, int TC, int MODE, bool FAST = false, bool TMA = false, bool SPLIT = false>
__device__ __forceinline__ bool col_body(const ColArgs<Real>& a, int tile, unsigned char* smraw,
                                         const ColMaps* maps = nullptr) {
    static_assert(!TMA || (FAST && MODE != COL_RHS), "TMA copies: FAST P1, STAGE and FINAL only");
    using C = typename Cx<Real>::T;
    using P = Plan<N>;
    using SM = ColSmem<Real, N, TC>;
    constexpr int T = P::T;
    constexpr int E = N / T;
    C* sm = reinterpret_cast<C*>(smraw);
    C* pre1 = sm + SM::FFT;       // accumulator, later the second exchange buffer
    C* pre0 = sm + 2 * SM::FFT;   // state, then the next stage input X
    const int c = threadIdx.x % TC;
    const int t = threadIdx.x / TC;
    const int ky = tile * TC + c;
    const bool valid = ky < a.nyf;
    const int kyc = valid ? ky : 0;
    const int ldc = a.ldc;
    const TwSeed<C> seed = twiddle_seeds<N>(a.tw, t);

    if constexpr (MODE == COL_P1) {
        if constexpr (TMA) {
            __shared__ __align__(8) unsigned long long bar_in;
            if (threadIdx.x == 0) {
                mbar_init(&bar_in);
                mbar_expect_tx(&bar_in, (unsigned)(sizeof(C) * N * TC));
                tma_load_tile<C, N, TC>(&maps->state, tile, pre0, &bar_in);
            }
            __syncthreads();
            const bool late = !mbar_wait0(&bar_in);
            if (__syncthreads_or(late)) {
                if (threadIdx.x == 0) {
                    atomicOr(a.status, 8);
                    mbar_wait0(&bar_in);
                }
                return false;
            }
            if (threadIdx.x == 0) mbar_inval(&bar_in);
        } else {
            const C* __restrict__ src = a.src;
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int i = t + T * m;
                if (valid) cp_async_elem(pre0 + i * TC + c, src + (size_t)i * ldc + ky);
                else pre0[i * TC + c] = cmake<C>(0, 0);
            }
            cp_async_commit();
            cp_async_wait_all();
        }
        if (a.col0_out && ky == 0) {
            // snapshot of the input's column 0 for a later conjugacy step whose
            // kernel also rewrites the state (AB4 update)
#pragma unroll
            for (int m = 0; m < E; ++m) a.col0_out[t + T * m] = pre0[(t + T * m) * TC + c];
        }
    } else {
        const C* __restrict__ src = a.src;
        C v[1][E];
        constexpr bool need_state = (MODE == COL_STAGE || MODE == COL_FINAL);
        const bool need_acc = (MODE == COL_STAGE && !a.first) || (MODE == COL_FINAL && a.scheme < 2);
        __shared__ __align__(8) unsigned long long bar_tile[2];  // TMA: [0] the input, [1] state and accumulator
        if constexpr (TMA) {
            if (threadIdx.x == 0) {
                mbar_init(&bar_tile[0]);
                mbar_init(&bar_tile[1]);
                constexpr unsigned tile_bytes = (unsigned)(sizeof(C) * N * TC);
                mbar_expect_tx(&bar_tile[0], tile_bytes);
                tma_load_tile<C, N, TC>(&maps->nl, tile, sm, &bar_tile[0]);
                mbar_expect_tx(&bar_tile[1], need_acc ? 2 * tile_bytes : tile_bytes);
                tma_load_tile<C, N, TC>(&maps->state, tile, pre0, &bar_tile[1]);
                if (need_acc) tma_load_tile<C, N, TC>(&maps->acc, tile, pre1, &bar_tile[1]);
            }
            __syncthreads();
            const bool late = !mbar_wait0(&bar_tile[0]);
#pragma unroll
            for (int m = 0; m < E; ++m) v[0][m] = sm[(t + T * m) * TC + c];
            // every thread has its input before the transform reuses the buffer
            if (__syncthreads_or(late)) {
                if (threadIdx.x == 0) {
                    // once more, bounded, for the copies still in flight
                    atomicOr(a.status, 8);
                    mbar_wait0(&bar_tile[0]);
                    mbar_wait0(&bar_tile[1]);
                }
                return false;
            }
            if (threadIdx.x == 0) mbar_inval(&bar_tile[0]);
        } else {
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int i = t + T * m;
                v[0][m] = valid ? src[(size_t)i * ldc + kyc] : cmake<C>(0, 0);
            }
        }
        // prefetch the epilogue operands while the forward transform runs
        if constexpr (need_state && !TMA) {
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int i = t + T * m;
                if (valid) {
                    cp_async_elem(pre0 + i * TC + c, a.state + (size_t)i * ldc + ky);
                    if (need_acc) cp_async_elem(pre1 + i * TC + c, a.acc + (size_t)i * ldc + ky);
                } else {
                    pre0[i * TC + c] = cmake<C>(0, 0);
                    pre1[i * TC + c] = cmake<C>(0, 0);
                }
            }
            cp_async_commit();
        }
        if constexpr (MODE == COL_FINAL) {
            // the Crank-Nicolson factors are read in the epilogue: start bringing
            // this thread's entries into L2 now, under the forward transform
            if (a.cn && valid) {
#pragma unroll
                for (int m = 0; m < E; ++m) prefetch_l2(a.cn + (size_t)(t + T * m) * ldc + ky);
            }
        }
        fft_batched<N, -1, 1>(v, IlvPolicy<N, TC, C>{sm, c}, seed, t);
        // The epilogue runs as a rolled loop over this thread's elements (one
        // copy of its code): the transform output is parked in the exchange
        // buffer, in slots only this thread touches.
#pragma unroll
        for (int m = 0; m < E; ++m) sm[(t + T * m) * TC + c] = v[0][m];
        if constexpr (TMA) {
            const bool late = !mbar_wait0(&bar_tile[1]);
            if (__syncthreads_or(late)) {
                if (threadIdx.x == 0) {
                    atomicOr(a.status, 8);
                    mbar_wait0(&bar_tile[1]);  // once more, bounded, for the copies still in flight
                }
                return false;
            }
            if (threadIdx.x == 0) mbar_inval(&bar_tile[1]);
        } else if constexpr (need_state) {
            cp_async_wait_all();
        }
        double bsum = 0.0;
        bool bad = false;
        // FAST: fully unrolled (its epilogue is short enough); else four at a time
        constexpr int EU = FAST ? E : 4;
#pragma unroll EU
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            const int q = i * TC + c;
            const int kx = (i <= N / 2) ? i : i - N;
            const int k2 = kx * kx + ky * ky;
            // normalisation and zero mean (solver.c:998-1013)
            C r = (kx == 0 && ky == 0) ? cmake<C>(0, 0) : cscale(sm[q], a.norm2);
            // dealiasing (solver.c:1039-1099)
            if (FAST || a.dealias == 0) {
                if (k2 >= a.kmax_sqr || (a.kolm && kx == 0)) r = cmake<C>(0, 0);
            } else {
                r = cscale(r, houli_filter<Real>(kx, ky, N, N, a.houli_int));
            }
            // forcing (solver.c:1022-1027)
            if (a.has_force && i == a.force_i && ky == a.force_j) r = cadd(r, a.force_val);
            if constexpr (!FAST) {
                if (a.force_field) r = cadd(r, a.force_field[(size_t)i * ldc + kyc]);
            }
            if constexpr (MODE == COL_RHS) {
                // stage derivative with the explicit linear term (Dormand-Prince
                // stages): r -= bracket(|k|^2) X, X the RHS input
                if (a.lin_stage == 2 && a.xin && k2 != 0)
                    r = csub(r, cscale(a.xin[(size_t)i * ldc + kyc], (Real)lin_bracket(a.lin, (double)k2)));
            }
            if constexpr (!FAST) {
                if (a.rhs_store && valid) a.rhs_store[(size_t)i * ldc + ky] = r;
            }
            // ForceConjugacy side effect on the state (solver.c:1031, 2096-2103)
            C w = cmake<C>(0, 0);
            if constexpr (need_state) w = pre0[q];
            if (a.conj_mode && ky == 0 && kx < 0 && valid) {
                w = cconj(a.conj_src[(size_t)(-kx) * a.conj_stride]);
                // (the TMA final pass stores this element's update through the tile copy)
                if constexpr (!(TMA && MODE == COL_FINAL)) a.state[(size_t)i * ldc] = w;
            }
            if constexpr (need_state) {
                // linear term of explicit RK4 stages (solver.c:664-684)
                if (!FAST && a.lin_stage && k2 != 0) {
                    const C xs = a.xin ? a.xin[(size_t)i * ldc + kyc] : w;
                    const double br = lin_bracket(a.lin, (double)k2);
                    if (a.lin_stage == 1) r = cadd(r, cscale(xs, (Real)(a.dt * br)));
                    else r = csub(r, cscale(xs, (Real)br));
                }
                if constexpr (MODE == COL_STAGE) {
                    C acc;
                    if (a.first) acc = cscale(r, (Real)a.b_cur);
                    else acc = cadd(pre1[q], cscale(r, (Real)a.b_cur));
                    if constexpr (TMA) pre1[q] = acc;  // staged for the tile store
                    else if (valid) a.acc[(size_t)i * ldc + ky] = acc;
                    const Real adt = (Real)(a.dt * a.a_next);
                    const C nx = cadd(w, cscale(r, adt));
                    pre0[q] = nx;
                    if (valid) {
                        if (ky == 0) a.col0_out[i] = nx;
                        if constexpr (!FAST) {
                            if (a.out) a.out[(size_t)i * ldc + ky] = nx;
                        }
                    }
                } else {  // COL_FINAL
                    C tot;
                    if (!FAST && a.scheme >= 2) {
                        // AB4 (solver.c:303-331): 55/24 N_n - 59/24 N_n-1 + 37/24 N_n-2 - 3/8 N_n-3
                        const size_t g = (size_t)i * ldc + kyc;
                        const C p2 = a.h2[g], p1 = a.h1[g], p0 = a.h0[g];
                        if (a.scheme == 3) {
                            const Real dt = (Real)a.dt;
                            tot = cadd(cadd(cadd(cscale(r, dt * (Real)(55.0 / 24.0)), cscale(p2, dt * (Real)(-59.0 / 24.0))),
                                            cscale(p1, dt * (Real)(37.0 / 24.0))),
                                       cscale(p0, dt * (Real)(-3.0 / 8.0)));
                        } else {
                            tot = cadd(cadd(cadd(cscale(r, (Real)(55.0 / 24.0)), cscale(p2, (Real)(-59.0 / 24.0))),
                                            cscale(p1, (Real)(37.0 / 24.0))),
                                       cscale(p0, (Real)(-3.0 / 8.0)));
                        }
                    } else {
                        tot = cadd(pre1[q], cscale(r, (Real)a.b_cur));
                    }
                    C wn;
                    if (kx == 0 && ky == 0) {
                        wn = cmake<C>(0, 0);
                    } else if (!FAST && a.scheme == 1) {
                        wn = cadd(w, cscale(tot, (Real)(a.dt / 6.0)));
                    } else if (!FAST && a.scheme == 3) {
                        wn = cadd(w, tot);
                    } else {
                        // Crank-Nicolson factors (solver.c:853), from the table
                        const double2 f = a.cn[(size_t)i * ldc + kyc];
                        wn = cadd(cscale(w, (Real)f.x), cscale(tot, (Real)f.y));
                    }
                    if (!FAST && a.phase_only && (kx != 0 || ky != 0)) {
                        // amplitude reset of the phase-only model (solver.c:822-824, 855-857):
                        // w_new *= |w_old| / |w_new|; a mode updated to exactly 0 stays 0
                        const double an = hypot((double)wn.x, (double)wn.y);
                        if (an > 0.0) {
                            const double r = hypot((double)w.x, (double)w.y) / an;
                            wn = cmake<C>((Real)((double)wn.x * r), (Real)((double)wn.y * r));
                        }
                    }
                    if constexpr (TMA) pre0[q] = wn;  // staged for the tile store
                    if (valid) {
                        if constexpr (!TMA) a.state[(size_t)i * ldc + ky] = wn;
                        const double mag = fabs((double)wn.x) + fabs((double)wn.y);
                        bad |= !isfinite(mag);
                        bsum += (ky == 0 || 2 * ky == N) ? mag : 2.0 * mag;
                    }
                }
            }
        }
        // the next transform's first stage writes other threads' parked slots
        if constexpr (TMA) fence_async_smem();
        __syncthreads();
        if constexpr (TMA && MODE == COL_STAGE) {
            if (threadIdx.x == 0) {
                tma_store_tile<C, N, TC>(&maps->acc, tile, pre1);
                bulk_commit();
            }
        }
        if constexpr (TMA && MODE == COL_FINAL) {
            if (threadIdx.x == 0) {
                tma_store_tile<C, N, TC>(&maps->state, tile, pre0);
                bulk_commit();
            }
        }
        if constexpr (MODE == COL_FINAL) {
            if (!a.final_tail) {
                // ensemble form: only the non-finite check
                if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(a.status, 1);
                __syncthreads();
                if constexpr (TMA) {
                    if (threadIdx.x == 0) bulk_wait_all();
                }
                return true;
            }
            // SystemCheck (solver.c:2301-2326) without a transform: max|w(x)| is
            // bounded by sum|w_hat|/(Nx Ny) over the full spectrum.  Status bit 1:
            // non-finite state; bit 2: the bound may reach 1e100 (the host then
            // evaluates max|w| exactly).  A bound of 1e100 needs one tile whose
            // share is at least 1e100/ntiles, so each block tests its own share
            // and no cross-block reduction is needed.
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) bsum += __shfl_xor_sync(0xffffffffu, bsum, o);
            const unsigned anybad = __ballot_sync(0xffffffffu, bad);
            double* wsum = reinterpret_cast<double*>(smraw);  // parked slots are free again
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            const int nwarps = (int)(blockDim.x >> 5);
            if (lane == 0) {
                wsum[warp] = bsum;
                if (anybad) atomicOr(a.status, 1);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                double tot = 0.0;
                for (int w = 0; w < nwarps; ++w) tot += wsum[w];
                if (!(tot * a.inv_nxny < 1e100 / (double)a.ntiles)) atomicOr(a.status, 2);
                if (tile == 0) atomicAdd(a.status + 1, 1);  // completed steps
            }
            __syncthreads();
            if constexpr (TMA) {
                if (threadIdx.x == 0) bulk_wait_all();
            }
            return true;
        }
        if constexpr (MODE == COL_RHS) return true;
    }

    if constexpr (TMA) derived_ifft_tma<Real, N, TC, SPLIT>(pre0, sm, maps, tile, ky, t, c, seed, MODE == COL_STAGE);
    else derived_ifft<Real, N, TC>(pre0, sm, a.f0, a.f1, a.f2, a.f3, ldc, ky, valid, t, c, seed);
    return true;
}

// Column pass of one field.  Grid: ceil(nyf / TC) blocks; block: T * TC threads.
// FAST: the epilogue compiled for the common step only (2/3 dealiasing, no
// listed-mode forcing, no stored RHS, no explicit linear term, Crank-Nicolson
// update of the full model); the launcher picks it when the arguments allow.
template <typename Real, int N, int TC, int MODE, bool FAST = false>
__global__ void __launch_bounds__(Plan<N>::T * TC) col_kernel(ColArgs<Real> a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    if (block_should_exit(a.status)) return;
    col_body<Real, N, TC, MODE, FAST>(a, blockIdx.x, smraw);
}

// Column pass with TMA tile loads and stores (FAST P1, STAGE and FINAL).  Shared
// memory: ColSmem::bytes_tma() + 1024 (the body's base is rounded up to 1024 bytes).
template <typename Real, int N, int TC, int MODE>
__global__ void __launch_bounds__(Plan<N>::T * TC) col_tma_kernel(ColArgs<Real> a, const __grid_constant__ ColMaps maps) {
    extern __shared__ __align__(16) unsigned char smraw[];
    if (block_should_exit(a.status)) return;
    unsigned char* sm = smraw + ((1024u - ((unsigned)__cvta_generic_to_shared(smraw) & 1023u)) & 1023u);
    col_body<Real, N, TC, MODE, true, true, true>(a, blockIdx.x, sm, &maps);
}

// Whether a stage or final column pass can run the FAST epilogue.
template <typename Real>
inline bool col_fast_ok(const ColArgs<Real>& a) {
    return a.dealias == 0 && !a.force_field && !a.rhs_store && a.lin_stage == 0 && !a.xin && !a.out &&
           a.scheme == 0 && !a.phase_only;
}

template <typename Real>
struct RowArgs {
    using C = typename Cx<Real>::T;
    const C* f0;  // U(x, ky)
    const C* f1;  // V
    const C* f2;  // WX
    const C* f3;  // WY
    C* nl;        // product spectrum n(x, ky)
    const C* tw;
    int ldc;
    int nrows;
    int* status;
    C* cap_uv;    // optional capture of the real fields: (u, v) and (w_x, w_y) as
    C* cap_w;     // complex pairs, [x][y] (adjoint stage recomputation); null = off
};

// Shared memory of the row pass: per row (one team of T threads), two padded
// exchange regions; after the inverse transforms the second region holds the
// row's product n(x, y) for the packed forward transform.
template <typename Real, int N, int TC>
struct RowSmem {
    using C = typename Cx<Real>::T;
    static constexpr int TEAM = 2 * TeamLayout<N>::ROWS;
    static_assert(TeamLayout<N>::ROWS * sizeof(C) >= N * sizeof(Real), "product must fit a region");
    static constexpr size_t bytes() { return sizeof(C) * (size_t)TEAM * TC; }
};

// Team width of the N/2-point plan (0 below the smallest plan).
template <int N>
constexpr int half_plan_width() {
    if constexpr (N / 2 >= 16) return Plan<N / 2>::T;
    else return 0;
}

// Row pass.  Block: TC = 2*PAIRS rows, one team of T threads per row (whole
// warps when T >= 32); grid: nrows / TC.  Each team runs its row's two inverse
// transforms together; rows 2p and 2p+1 then share one packed forward
// transform, done by team 2p alone when teams are whole warps (team 2p+1
// leaves) and by both teams, each keeping its half, below a warp.
template <typename Real, int N, int PAIRS, bool CAP = true>
__device__ __forceinline__ void row_body(const RowArgs<Real>& a, int rblock, unsigned char* smraw) {
    using C = typename Cx<Real>::T;
    using P = Plan<N>;
    constexpr int T = P::T;
    constexpr int E = N / T;
    constexpr int TC = 2 * PAIRS;
    using TL = TeamLayout<N>;
    using RS = RowSmem<Real, N, TC>;
    const int g = threadIdx.x / T;  // row (team) within the block
    const int t = threadIdx.x % T;
    const int x = rblock * TC + g;
    C* region = reinterpret_cast<C*>(smraw) + (size_t)g * RS::TEAM;
    const TwSeed<C> seed = twiddle_seeds<N>(a.tw, t);
    const TeamPolicy<N, C> pol{region, 1 + g};

    // Z1 = U + i V and Z2 = WX + i WY over the full y range (Hermitian
    // extension; DC and Nyquist use the real parts only, as FFTW's c2r does)
    C v[2][E];
    {
        const C* __restrict__ U = a.f0 + (size_t)x * a.ldc;
        const C* __restrict__ V = a.f1 + (size_t)x * a.ldc;
        const C* __restrict__ WX = a.f2 + (size_t)x * a.ldc;
        const C* __restrict__ WY = a.f3 + (size_t)x * a.ldc;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int y = t + T * m;
            const int yy = (y <= N / 2) ? y : N - y;
            const C p0 = U[yy], q0 = V[yy], p1 = WX[yy], q1 = WY[yy];
            if (y == 0 || y == N / 2) {
                v[0][m] = cmake<C>(p0.x, q0.x);
                v[1][m] = cmake<C>(p1.x, q1.x);
            } else if (y < N / 2) {
                v[0][m] = cmake<C>(p0.x - q0.y, p0.y + q0.x);
                v[1][m] = cmake<C>(p1.x - q1.y, p1.y + q1.x);
            } else {
                v[0][m] = cmake<C>(p0.x + q0.y, q0.x - p0.y);
                v[1][m] = cmake<C>(p1.x + q1.y, q1.x - p1.y);
            }
        }
    }
    fft_batched<N, +1, 2>(v, pol, seed, t);
    if (CAP && a.cap_uv) {
        C* __restrict__ cu = a.cap_uv + (size_t)x * N;
        C* __restrict__ cw = a.cap_w + (size_t)x * N;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            cu[t + T * m] = v[0][m];
            cw[t + T * m] = v[1][m];
        }
    }
    // n = 1.0 * (u w_x + v w_y)  (solver.c:979-981), parked for the packing
    Real* nl_own = reinterpret_cast<Real*>(region + TL::ROWS);
#pragma unroll
    for (int m = 0; m < E; ++m) nl_own[t + T * m] = v[0][m].x * v[1][m].x + v[0][m].y * v[1][m].y;
    // HALF: each team transforms its own row's real product as an N/2-point
    // complex sequence z[j] = n[2j] + i n[2j+1] and splits the result,
    //   X[k] = (Z[k] + conj Z[N/2-k])/2 + W^k (Z[k] - conj Z[N/2-k])/(2i),
    // W = exp(-2 pi i / N), k = 0..N/2 (Z periodic in N/2): both teams work and
    // only team barriers are needed (below a warp, both teams of a pair would
    // otherwise each run the pair's whole packed transform).  Where the N/2 plan
    // has another team width the rows of a pair share one packed N-point
    // transform instead.
    constexpr int NH = N / 2;
    constexpr bool HALF = half_plan_width<N>() == T;
    if constexpr (HALF) {
        constexpr int EH = NH / T;
        using TLH = TeamLayout<NH>;
        static_assert(TLH::ROWS <= TL::ROWS, "the half-size exchange must not reach the parked product");
        pol.sync();
        const C* zin = reinterpret_cast<const C*>(nl_own);
        C z[1][EH];
#pragma unroll
        for (int m = 0; m < EH; ++m) z[0][m] = zin[t + T * m];
        const TeamPolicy<NH, C> polh{region, 1 + g};
        fft_batched<NH, -1, 1>(z, polh, twiddle_seeds_strided<NH>(a.tw, t, 2), t);
#pragma unroll
        for (int m = 0; m < EH; ++m) region[TLH::slot(t + T * m)] = z[0][m];
        polh.sync();
        C* dst = a.nl + (size_t)x * a.ldc;
#pragma unroll
        for (int m = 0; m < EH; ++m) {
            const int k = t + T * m;
            const C zk = z[0][m];
            const C zm = region[TLH::slot((NH - k) & (NH - 1))];
            const C ev = cmake<C>((Real)0.5 * (zk.x + zm.x), (Real)0.5 * (zk.y - zm.y));
            const C od = cmake<C>((Real)0.5 * (zk.y + zm.y), (Real)0.5 * (zm.x - zk.x));
            dst[k] = cadd(ev, cmul(__ldg(a.tw + k), od));
            if (k == 0) dst[NH] = cmake<C>(zk.x - zk.y, (Real)0);  // W^(N/2) = -1
        }
    } else {
    __syncthreads();
    const int ga = g & ~1;
    bool active = true;
    if constexpr (T >= 32) active = (g & 1) == 0;  // the pair's packed transform is done by the even team
    if (active) {
    const Real* na = reinterpret_cast<const Real*>(reinterpret_cast<C*>(smraw) + (size_t)ga * RS::TEAM + TL::ROWS);
    const Real* nb = reinterpret_cast<const Real*>(reinterpret_cast<C*>(smraw) + (size_t)(ga + 1) * RS::TEAM + TL::ROWS);
    C z[1][E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int y = t + T * m;
        z[0][m] = cmake<C>(na[y], nb[y]);
    }
    fft_batched<N, -1, 1>(z, pol, seed, t);
    // split: X_a = (Z_k + conj Z_{N-k})/2, X_b = (Z_k - conj Z_{N-k})/(2i)
#pragma unroll
    for (int m = 0; m < E; ++m) region[TL::slot(t + T * m)] = z[0][m];
    pol.sync();
    C* dst_a = a.nl + (size_t)(rblock * TC + ga) * a.ldc;
    C* dst_b = dst_a + a.ldc;
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int k = t + T * m;
        if (k <= N / 2) {
            const C zk = region[TL::slot(k)];
            const C zm = region[TL::slot((N - k) & (N - 1))];
            const C ra = cmake<C>((Real)0.5 * (zk.x + zm.x), (Real)0.5 * (zk.y - zm.y));
            const C rb = cmake<C>((Real)0.5 * (zk.y + zm.y), (Real)0.5 * (zm.x - zk.x));
            if constexpr (T >= 32) {
                dst_a[k] = ra;
                dst_b[k] = rb;
            } else {
                if (g & 1) dst_b[k] = rb;
                else dst_a[k] = ra;
            }
        }
    }
    }  // active
    }  // HALF
    __syncthreads();  // the shared memory may be reused for another row block
}

// CAP: the capture of the real fields (adjoint recomputation) compiled in;
// the launcher uses the form without it when no capture target is set.
template <typename Real, int N, int PAIRS, bool CAP = true>
__global__ void __launch_bounds__(Plan<N>::T * 2 * PAIRS) row_kernel(RowArgs<Real> a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    if (block_should_exit(a.status)) return;
    row_body<Real, N, PAIRS, CAP>(a, blockIdx.x, smraw);
}

// Crank-Nicolson factors per mode for the current dt and operator branch:
// cn = ((2 - D)/(2 + D), 2 dt/(2 + D)), D = dt * bracket(|k|^2) (solver.c:839-853).
static __global__ void cn_table_kernel(double2* cn, int nx, int nyf, int ldc, double dt, LinOp lin) {
    const long long n = (long long)nx * nyf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / nyf), ky = (int)(q % nyf);
        const int kx = (i <= nx / 2) ? i : i - nx;
        const double k2 = (double)(kx * kx + ky * ky);
        double2 f = make_double2(0.0, 0.0);
        if (kx != 0 || ky != 0) {
            const double D = dt * lin_bracket(lin, k2);
            f = make_double2((2.0 - D) / (2.0 + D), (2.0 * dt) / (2.0 + D));
        }
        cn[(size_t)i * ldc + ky] = f;
    }
}

}  // namespace ns2d
