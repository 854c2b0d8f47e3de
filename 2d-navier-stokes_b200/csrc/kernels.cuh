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
};

// 1/k^2 for the velocity spectra.  FP64: Newton-Raphson for the reciprocal,
// r <- r + r (1 - k2 r), twice from the single-precision reciprocal (k2 < 2^24
// is exact in FP32, the seed's relative error is below 2^-23, so two steps
// leave about one rounding of FP64); single precision in the FP32 form.
template <typename Real>
__device__ __forceinline__ Real inv_k2(int k2);
template <>
__device__ __forceinline__ double inv_k2<double>(int k2) {
    const double d = (double)k2;
    double r = (double)__frcp_rn((float)k2);
    r = fma(r, fma(-d, r, 1.0), r);
    r = fma(r, fma(-d, r, 1.0), r);
    return r;
}
template <>
__device__ __forceinline__ float inv_k2<float>(int k2) { return __frcp_rn((float)k2); }

// Derived spectra of the stage input X at (kx, ky) (solver.c:904-957), two at a
// time: pair 0 gives u = i ky/k^2 X and v = -i kx/k^2 X (one reciprocal), pair 2
// gives w_x = i kx X and w_y = i ky X.  Zero at the mean mode.
template <typename C>
__device__ __forceinline__ void derived_pair(int fp, int kx, int ky, C X, C& a, C& b) {
    using Real = decltype(C::x);
    if (kx == 0 && ky == 0) {
        a = cmake<C>(0, 0);
        b = a;
        return;
    }
    Real sa, sb;
    if (fp == 0) {
        const Real inv = inv_k2<Real>(kx * kx + ky * ky);
        sa = (Real)ky * inv;
        sb = -(Real)kx * inv;
    } else {
        sa = (Real)kx;
        sb = (Real)ky;
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
#pragma unroll 1
    for (int fp = 0; fp < 4; fp += 2) {
        C v[2][E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            const int kx = (i <= N / 2) ? i : i - N;
            derived_pair(fp, kx, ky, pre0[i * TC + c], v[0][m], v[1][m]);
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

// Column pass on tile `tile` (ky columns tile*TC .. tile*TC+TC-1), by the T*TC
// threads of a block, thread (t, c) with c = threadIdx.x % TC.  Shared memory:
// ColSmem::bytes().  Ends with the block synchronised (the shared memory may be
// reused for another tile).
template <typename Real, int N, int TC, int MODE, bool FAST = false>
__device__ __forceinline__ void col_body(const ColArgs<Real>& a, int tile, unsigned char* smraw) {
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
        C v[1][E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            v[0][m] = valid ? src[(size_t)i * ldc + kyc] : cmake<C>(0, 0);
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
        if constexpr (need_state) cp_async_wait_all();
        double bsum = 0.0;
        bool bad = false;
#pragma unroll 4
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            const int q = i * TC + c;
            const int kx = (i <= N / 2) ? i : i - N;
            const int k2 = kx * kx + ky * ky;
            // normalisation and zero mean (solver.c:998-1013)
            C r = (kx == 0 && ky == 0) ? cmake<C>(0, 0) : cscale(sm[q], a.norm2);
            // dealiasing (solver.c:1039-1099)
            if (FAST || a.dealias == 0) {
                if ((double)k2 >= (double)a.kmax_sqr || (a.kolm && kx == 0)) r = cmake<C>(0, 0);
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
                a.state[(size_t)i * ldc] = w;
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
                    if (valid) a.acc[(size_t)i * ldc + ky] = acc;
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
                    if (valid) {
                        a.state[(size_t)i * ldc + ky] = wn;
                        const double mag = fabs((double)wn.x) + fabs((double)wn.y);
                        bad |= !isfinite(mag);
                        bsum += (ky == 0 || 2 * ky == N) ? mag : 2.0 * mag;
                    }
                }
            }
        }
        // the next transform's first stage writes other threads' parked slots
        __syncthreads();
        if constexpr (MODE == COL_FINAL) {
            if (!a.final_tail) {
                // ensemble form: only the non-finite check
                if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(a.status, 1);
                __syncthreads();
                return;
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
            return;
        }
        if constexpr (MODE == COL_RHS) return;
    }

    derived_ifft<Real, N, TC>(pre0, sm, a.f0, a.f1, a.f2, a.f3, ldc, ky, valid, t, c, seed);
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
