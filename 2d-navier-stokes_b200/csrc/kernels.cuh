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
    double* blowup_sum;  // COL_FINAL: [0] bound accumulator, [1] ticket counter
    double inv_nxny;     // 1/(Nx Ny)
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

// Shared memory of the column pass: the FFT exchange buffer, then two
// [N][TC] staging arrays (state or stage input, and the RK accumulator).
template <typename Real, int N, int TC>
struct ColSmem {
    using C = typename Cx<Real>::T;
    static constexpr int FFT = SmemLayout<N, TC>::ELEMS;
    static constexpr int PRE = N * TC;
    static constexpr size_t bytes() { return sizeof(C) * (size_t)(FFT + 2 * PRE); }
};

// Derived spectrum f of the stage input X at (kx, ky) (solver.c:904-957):
// 0: i ky/k^2 X, 1: -i kx/k^2 X, 2: i kx X, 3: i ky X.
template <typename C>
__device__ __forceinline__ C derived(int f, int kx, int ky, C X) {
    using Real = decltype(C::x);
    if (kx == 0 && ky == 0) return cmake<C>(0, 0);
    Real s;
    if (f < 2) {
        const double inv = 1.0 / (double)(kx * kx + ky * ky);
        s = (Real)((double)(f == 0 ? ky : kx) * inv);
    } else {
        s = (Real)(f == 2 ? kx : ky);
    }
    return (f == 1) ? cmake<C>(s * X.y, -s * X.x) : cmake<C>(-s * X.y, s * X.x);
}

// Column pass.  Grid: ceil(nyf / TC) blocks; block: T * TC threads, thread
// (t, c) with c = threadIdx.x % TC.  Dynamic shared memory: ColSmem::bytes().
template <typename Real, int N, int TC, int MODE>
__global__ void __launch_bounds__(Plan<N>::T * TC) col_kernel(ColArgs<Real> a) {
    using C = typename Cx<Real>::T;
    using P = Plan<N>;
    using SM = ColSmem<Real, N, TC>;
    constexpr int T = P::T;
    constexpr int E = N / T;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    C* pre0 = sm + SM::FFT;     // state, then the next stage input X
    C* pre1 = pre0 + SM::PRE;   // accumulator
    if (block_should_exit(a.status)) return;
    const int c = threadIdx.x % TC;
    const int t = threadIdx.x / TC;
    const int ky = blockIdx.x * TC + c;
    const bool valid = ky < a.nyf;
    const int kyc = valid ? ky : 0;
    const int ldc = a.ldc;

    if constexpr (MODE == COL_P1) {
        const C* __restrict__ src = a.src;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            if (valid) cp_async_elem(pre0 + i * TC + c, src + (size_t)i * ldc + ky);
            else pre0[i * TC + c] = cmake<C>(0, 0);
        }
        cp_async_commit();
        cp_async_wait_all();
        if (a.col0_out && ky == 0) {
            // snapshot of the input's column 0 for a later conjugacy step whose
            // kernel also rewrites the state (AB4 update)
#pragma unroll
            for (int m = 0; m < E; ++m) a.col0_out[t + T * m] = pre0[(t + T * m) * TC + c];
        }
    } else {
        const C* __restrict__ src = a.src;
        C v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            v[m] = valid ? src[(size_t)i * ldc + kyc] : cmake<C>(0, 0);
        }
        // prefetch the epilogue operands while the forward transform runs
        constexpr bool need_state = (MODE == COL_STAGE || MODE == COL_FINAL);
        const bool need_acc = (MODE == COL_STAGE && !a.first) || (MODE == COL_FINAL && a.scheme < 2);
        if constexpr (need_state) {
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
        fft<N, -1, TC>(v, sm, a.tw, t, c);
        if constexpr (need_state) cp_async_wait_all();
        double bsum = 0.0;
        bool bad = false;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            const int kx = (i <= N / 2) ? i : i - N;
            const int k2 = kx * kx + ky * ky;
            // normalisation and zero mean (solver.c:998-1013)
            C r = (kx == 0 && ky == 0) ? cmake<C>(0, 0) : cscale(v[m], a.norm2);
            // dealiasing (solver.c:1039-1099)
            if (a.dealias == 0) {
                if ((double)k2 >= (double)a.kmax_sqr || (a.kolm && kx == 0)) r = cmake<C>(0, 0);
            } else {
                r = cscale(r, houli_filter<Real>(kx, ky, N, N, a.houli_int));
            }
            // forcing (solver.c:1022-1027)
            if (a.has_force && i == a.force_i && ky == a.force_j) r = cadd(r, a.force_val);
            if (a.rhs_store && valid) a.rhs_store[(size_t)i * ldc + ky] = r;
            // ForceConjugacy side effect on the state (solver.c:1031, 2096-2103)
            C w = cmake<C>(0, 0);
            if constexpr (need_state) w = pre0[i * TC + c];
            if (a.conj_mode && ky == 0 && kx < 0 && valid) {
                w = cconj(a.conj_src[(size_t)(-kx) * a.conj_stride]);
                a.state[(size_t)i * ldc] = w;
            }
            if constexpr (need_state) {
                // linear term of explicit RK4 stages (solver.c:664-684)
                if (a.lin_stage && k2 != 0) {
                    const C xs = a.xin ? a.xin[(size_t)i * ldc + kyc] : w;
                    const double br = lin_bracket(a.lin, (double)k2);
                    if (a.lin_stage == 1) r = cadd(r, cscale(xs, (Real)(a.dt * br)));
                    else r = csub(r, cscale(xs, (Real)br));
                }
                if constexpr (MODE == COL_STAGE) {
                    C acc;
                    if (a.first) acc = cscale(r, (Real)a.b_cur);
                    else acc = cadd(pre1[i * TC + c], cscale(r, (Real)a.b_cur));
                    if (valid) a.acc[(size_t)i * ldc + ky] = acc;
                    const Real adt = (Real)(a.dt * a.a_next);
                    const C nx = cadd(w, cscale(r, adt));
                    pre0[i * TC + c] = nx;
                    if (valid) {
                        if (ky == 0) a.col0_out[i] = nx;
                        if (a.out) a.out[(size_t)i * ldc + ky] = nx;
                    }
                } else {  // COL_FINAL
                    C tot;
                    if (a.scheme >= 2) {
                        // AB4 (solver.c:303-331): 55/24 N_n - 59/24 N_n-1 + 37/24 N_n-2 - 3/8 N_n-3
                        const size_t q = (size_t)i * ldc + kyc;
                        const C p2 = a.h2[q], p1 = a.h1[q], p0 = a.h0[q];
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
                        tot = cadd(pre1[i * TC + c], cscale(r, (Real)a.b_cur));
                    }
                    C wn;
                    if (kx == 0 && ky == 0) {
                        wn = cmake<C>(0, 0);
                    } else if (a.scheme == 1) {
                        wn = cadd(w, cscale(tot, (Real)(a.dt / 6.0)));
                    } else if (a.scheme == 3) {
                        wn = cadd(w, tot);
                    } else {
                        // Crank-Nicolson factors (solver.c:853)
                        const double D = a.dt * lin_bracket(a.lin, (double)k2);
                        const double rcp = 1.0 / (2.0 + D);
                        wn = cadd(cscale(w, (Real)((2.0 - D) * rcp)), cscale(tot, (Real)(2.0 * a.dt * rcp)));
                    }
                    if (valid) {
                        a.state[(size_t)i * ldc + ky] = wn;
                        const double mag = fabs((double)wn.x) + fabs((double)wn.y);
                        bad |= !isfinite(mag);
                        bsum += (ky == 0 || 2 * ky == N) ? mag : 2.0 * mag;
                    }
                }
            }
        }
        if constexpr (MODE == COL_FINAL) {
            // SystemCheck (solver.c:2301-2326) without a transform: max|w(x)| is
            // bounded by sum|w_hat|/(Nx Ny) over the full spectrum.  Status bit 1:
            // non-finite state; bit 2: bound >= 1e100 (the host then evaluates
            // max|w| exactly).  The last block to finish (atomic ticket, no
            // waiting) checks the total and resets the accumulator.
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) bsum += __shfl_xor_sync(0xffffffffu, bsum, o);
            const unsigned anybad = __ballot_sync(0xffffffffu, bad);
            if ((threadIdx.x & 31) == 0) {
                atomicAdd(a.blowup_sum, bsum);
                if (anybad) atomicOr(a.status, 1);
                __threadfence();
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                unsigned int* ticket = reinterpret_cast<unsigned int*>(a.blowup_sum + 1);
                const unsigned int done = atomicAdd(ticket, 1u);
                if (done == gridDim.x - 1) {
                    __threadfence();
                    const double total = atomicAdd(a.blowup_sum, 0.0);
                    if (!(total * a.inv_nxny < 1e100)) atomicOr(a.status, 2);
                    *a.blowup_sum = 0.0;
                    *ticket = 0u;
                    atomicAdd(a.status + 1, 1);  // completed steps
                    __threadfence();
                }
            }
            return;
        }
        if constexpr (MODE == COL_RHS) return;
    }

    // derived spectra of the stage input and four inverse x-FFTs; one copy of
    // the transform code serves all four fields
    C* outs[4] = {a.f0, a.f1, a.f2, a.f3};
#pragma unroll 1
    for (int f = 0; f < 4; ++f) {
        C v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            const int kx = (i <= N / 2) ? i : i - N;
            v[m] = derived(f, kx, ky, pre0[i * TC + c]);
        }
        fft<N, +1, TC>(v, sm, a.tw, t, c);
        if (valid) {
            C* __restrict__ o = outs[f];
#pragma unroll
            for (int m = 0; m < E; ++m) o[(size_t)(t + T * m) * ldc + ky] = v[m];
        }
    }
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
};

// Shared memory of the row pass: FFT exchange buffer, then the WX and WY
// half rows of the block's TC rows (prefetched with cp.async).
template <typename Real, int N, int TC>
struct RowSmem {
    using C = typename Cx<Real>::T;
    static constexpr int FFT = SmemLayout<N, TC>::ELEMS;
    // row pitch: N/2+1 rounded so that the TC rows start in different banks
    static constexpr int PITCH = ((N / 2 + 1 + 7) / 8) * 8 + (TC >= 8 ? 1 : 8 / TC);
    static constexpr int PRE = 2 * TC * PITCH;
    // u and v of pass 0, [2][N][TC] reals, after the prefetch area
    static constexpr size_t UV_OFFSET = sizeof(C) * (size_t)(FFT + PRE);
    static constexpr size_t bytes() {
        size_t a = UV_OFFSET + sizeof(Real) * 2 * (size_t)N * TC;
        size_t b = sizeof(Real) * (size_t)N * TC;
        return a > b ? a : b;
    }
};

// Row pass.  Block: 2*PAIRS*T threads = TC = 2*PAIRS transforms (one per x row);
// grid: nrows / (2*PAIRS).  Rows 2p and 2p+1 of the block share one packed
// forward transform, computed by both of their thread groups.
template <typename Real, int N, int PAIRS>
__global__ void __launch_bounds__(Plan<N>::T * 2 * PAIRS) row_kernel(RowArgs<Real> a) {
    using C = typename Cx<Real>::T;
    using P = Plan<N>;
    constexpr int T = P::T;
    constexpr int E = N / T;
    constexpr int TC = 2 * PAIRS;
    using L = SmemLayout<N, TC>;
    using RS = RowSmem<Real, N, TC>;
    constexpr int NYF = N / 2 + 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    C* pre = sm + RS::FFT;  // [field 0/1][row g][PITCH]
    if (block_should_exit(a.status)) return;
    const int g = threadIdx.x % TC;  // row within the block
    const int t = threadIdx.x / TC;
    const int x0 = blockIdx.x * TC;
    const int x = x0 + g;
    // prefetch WX, WY of all TC rows (pass 1) while pass 0 runs
    for (int q = threadIdx.x; q < 2 * TC * NYF; q += blockDim.x) {
        const int f = q / (TC * NYF);
        const int rem = q - f * TC * NYF;
        const int rg = rem / NYF, y = rem - rg * NYF;
        const C* base = (f == 0 ? a.f2 : a.f3) + (size_t)(x0 + rg) * a.ldc + y;
        cp_async_elem(pre + (f * TC + rg) * RS::PITCH + y, base);
    }
    cp_async_commit();

    Real* uv = reinterpret_cast<Real*>(smraw + RS::UV_OFFSET);  // own slots only
    Real nl[E];
    C z[E];
    // Z1 = U + i V over the full y range (Hermitian extension; DC and Nyquist
    // use the real parts only, as FFTW's c2r does)
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 0) {
            const C* __restrict__ A = a.f0 + (size_t)x * a.ldc;
            const C* __restrict__ B = a.f1 + (size_t)x * a.ldc;
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int y = t + T * m;
                const int yy = (y <= N / 2) ? y : N - y;
                const C p = A[yy], q = B[yy];
                if (y == 0 || y == N / 2) z[m] = cmake<C>(p.x, q.x);
                else if (y < N / 2) z[m] = cmake<C>(p.x - q.y, p.y + q.x);
                else z[m] = cmake<C>(p.x + q.y, q.x - p.y);
            }
        } else {
            cp_async_wait_all();
            __syncthreads();
            const C* A = pre + (0 * TC + g) * RS::PITCH;
            const C* B = pre + (1 * TC + g) * RS::PITCH;
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int y = t + T * m;
                const int yy = (y <= N / 2) ? y : N - y;
                const C p = A[yy], q = B[yy];
                if (y == 0 || y == N / 2) z[m] = cmake<C>(p.x, q.x);
                else if (y < N / 2) z[m] = cmake<C>(p.x - q.y, p.y + q.x);
                else z[m] = cmake<C>(p.x + q.y, q.x - p.y);
            }
        }
        fft<N, +1, TC>(z, sm, a.tw, t, g);
        if (pass == 0) {
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int q = (t + T * m) * TC + g;
                uv[q] = z[m].x;
                uv[N * TC + q] = z[m].y;
            }
        } else {
#pragma unroll
            for (int m = 0; m < E; ++m) {
                // n = 1.0 * (u w_x + v w_y)  (solver.c:979-981)
                const int q = (t + T * m) * TC + g;
                nl[m] = uv[q] * z[m].x + uv[N * TC + q] * z[m].y;
            }
        }
    }
    // pack rows (2p, 2p+1): zr = n_a + i n_b
    Real* rs = reinterpret_cast<Real*>(smraw);
#pragma unroll
    for (int m = 0; m < E; ++m) rs[(t + T * m) * TC + g] = nl[m];
    __syncthreads();
    const int ga = g & ~1;
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int y = t + T * m;
        z[m] = cmake<C>(rs[y * TC + ga], rs[y * TC + ga + 1]);
    }
    __syncthreads();
    fft<N, -1, TC>(z, sm, a.tw, t, g);
    // split: X_a = (Z_k + conj Z_{N-k})/2, X_b = (Z_k - conj Z_{N-k})/(2i)
    if ((g & 1) == 0) {
#pragma unroll
        for (int m = 0; m < E; ++m) sm[L::slot(t + T * m, g >> 1)] = z[m];
    }
    __syncthreads();
    const int p = g >> 1;
    C* dst = a.nl + (size_t)x * a.ldc;
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int k = t + T * m;
        if (k <= N / 2) {
            const C zk = sm[L::slot(k, p)];
            const C zm = sm[L::slot((N - k) & (N - 1), p)];
            C r;
            if ((g & 1) == 0) r = cmake<C>((Real)0.5 * (zk.x + zm.x), (Real)0.5 * (zk.y - zm.y));
            else r = cmake<C>((Real)0.5 * (zk.y + zm.y), (Real)0.5 * (zm.x - zk.x));
            dst[k] = r;
        }
    }
}

}  // namespace ns2d
