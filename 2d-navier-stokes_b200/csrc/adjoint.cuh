// adjoint.cuh -- discrete adjoint of the nonlinear term and of an RK4CN step.
//
// State x: the Hermitian half spectrum.  Inner product
//   <a, b>_W = sum_j c_j Re(conj(a_j) b_j),  c_j = 1 on ky = 0 and ky = N/2, 2 else,
// under which the unnormalised c2r (C) and r2c (R) are exact transposes.  With
// multipliers m_u = i ky/k^2, m_v = -i kx/k^2, m_x = i kx, m_y = i ky, dealias
// factor D and s = 1/(Nx Ny), the forward RHS is
//   F(X) = s^2 D R( C(m_u X) C(m_x X) + C(m_v X) C(m_y X) )
// and its adjoint at X applied to kappa is
//   F'(X)^T kappa = conj(m_u) R(wx mu) + conj(m_v) R(wy mu) + conj(m_x) R(u mu) + conj(m_y) R(v mu),
//   mu = C(s^2 D kappa),
// with u, v, wx, wy = C(m_u X), C(m_v X), C(m_x X), C(m_y X) the real fields of
// the forward stage, captured while the forward step is recomputed.
//
// Passes per adjoint stage (mirroring the forward step):
//   adj row pass  (y): mu = c2r(mu_x); products wx mu, wy mu, u mu, v mu; two
//                      packed r2c -> four x-space half spectra P0..P3.
//   adj col pass  (x): four forward x-FFTs of P0..P3, L = sum conj(m) P (the
//                      adjoint of this stage's input); lambda_x += L; the
//                      previous stage's kappa = b B lambda' + a dt L; then
//                      s^2 D kappa -> inverse x-FFT -> mu_x for the next row pass.
#pragma once
#include "kernels.cuh"

namespace ns2d {

enum AdjMode : int { ADJ_START = 0, ADJ_MID = 1, ADJ_END = 2 };

template <typename Real>
struct AdjColArgs {
    using C = typename Cx<Real>::T;
    const C* P0;          // x-space product spectra of the row pass (MID, END)
    const C* P1;
    const C* P2;
    const C* P3;
    C* lam_x;             // adjoint of the step input (accumulated), [kx][ldc]
    const C* lam_p;       // adjoint of the step output lambda'
    const double2* cn;    // ((2-D)/(2+D), 2dt/(2+D)) per mode
    C* mu;                // x-space mu_x for the next row pass (START, MID)
    const C* tw;
    int ldc, nyf;
    Real norm2;
    int kmax_sqr, dealias, houli_int, kolm;
    double b_next;        // weight of lambda' in the next kappa: b_{s-1} (MID) or b_4 (START)
    double adt;           // a_{s-1} dt (MID)
};

// Dealias factor of the forward RHS at (kx, ky) (solver.c:1039-1099).
template <typename Real>
__device__ __forceinline__ Real dealias_factor(int kx, int ky, int N, int kmax_sqr, int dealias, int houli_int,
                                               int kolm) {
    if (kx == 0 && ky == 0) return (Real)0;
    if (dealias == 0) {
        const double k2 = (double)kx * kx + (double)ky * ky;
        return (k2 >= (double)kmax_sqr || (kolm && kx == 0)) ? (Real)0 : (Real)1;
    }
    return houli_filter<Real>(kx, ky, N, N, houli_int);
}

// conj(m_f) * P for the four multipliers (f = 0..3: m_u, m_v, m_x, m_y).
template <typename C>
__device__ __forceinline__ C conj_mult(int f, int kx, int ky, C P) {
    using Real = decltype(C::x);
    if (kx == 0 && ky == 0) return cmake<C>(0, 0);
    Real s;
    if (f < 2) {
        const double inv = 1.0 / (double)(kx * kx + ky * ky);
        s = (Real)((double)(f == 0 ? ky : kx) * inv);
    } else {
        s = (Real)(f == 2 ? kx : ky);
    }
    // conj(i s) = -i s;  conj(-i s) = i s  (f == 1 has m_v = -i kx/k^2)
    return (f == 1) ? cmake<C>(-s * P.y, s * P.x) : cmake<C>(s * P.y, -s * P.x);
}

template <typename Real, int N, int TC, int MODE>
__global__ void __launch_bounds__(Plan<N>::T * TC) adj_col_kernel(AdjColArgs<Real> a) {
    using C = typename Cx<Real>::T;
    using P = Plan<N>;
    using SM = ColSmem<Real, N, TC>;
    constexpr int T = P::T;
    constexpr int E = N / T;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    C* Lbuf = sm + 2 * SM::FFT;  // [N][TC]: L, then s^2 D kappa
    const int c = threadIdx.x % TC;
    const int t = threadIdx.x / TC;
    const int ky = blockIdx.x * TC + c;
    const bool valid = ky < a.nyf;
    const int kyc = valid ? ky : 0;
    const int ldc = a.ldc;
    const TwSeed<C> seed = twiddle_seeds<N>(a.tw, t);

    if constexpr (MODE != ADJ_START) {
        // L = conj(m_u) P0 + conj(m_v) P1 + conj(m_x) P2 + conj(m_y) P3
        const C* Ps[4] = {a.P0, a.P1, a.P2, a.P3};
#pragma unroll 1
        for (int fp = 0; fp < 4; fp += 2) {
            C v[2][E];
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const size_t q = (size_t)(t + T * m) * ldc + kyc;
                v[0][m] = valid ? Ps[fp][q] : cmake<C>(0, 0);
                v[1][m] = valid ? Ps[fp + 1][q] : cmake<C>(0, 0);
            }
            fft_batched<N, -1, 2>(v, IlvPolicy<N, TC, C>{sm, c}, seed, t);
#pragma unroll
            for (int m = 0; m < E; ++m) {
                const int i = t + T * m;
                const int kx = (i <= N / 2) ? i : i - N;
                C L = cadd(conj_mult(fp, kx, ky, v[0][m]), conj_mult(fp + 1, kx, ky, v[1][m]));
                if (fp > 0) L = cadd(Lbuf[i * TC + c], L);
                Lbuf[i * TC + c] = L;
            }
        }
    }
    if constexpr (MODE == ADJ_END) {
#pragma unroll 4
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            if (valid) {
                const size_t q = (size_t)i * ldc + ky;
                a.lam_x[q] = cadd(a.lam_x[q], Lbuf[i * TC + c]);
            }
        }
        return;
    } else {
        // kappa of the next (earlier) stage and the source of mu
#pragma unroll 4
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            const int kx = (i <= N / 2) ? i : i - N;
            const size_t q = (size_t)i * ldc + kyc;
            const C lp = valid ? a.lam_p[q] : cmake<C>(0, 0);
            const double2 f = valid ? a.cn[q] : make_double2(0.0, 0.0);
            C kappa = cscale(lp, (Real)(a.b_next * f.y));
            if constexpr (MODE == ADJ_MID) {
                const C L = Lbuf[i * TC + c];
                if (valid) a.lam_x[(size_t)i * ldc + ky] = cadd(a.lam_x[(size_t)i * ldc + ky], L);
                kappa = cadd(kappa, cscale(L, (Real)a.adt));
            } else {
                // START: lambda_x = A lambda'
                if (valid) a.lam_x[(size_t)i * ldc + ky] = cscale(lp, (Real)f.x);
            }
            const Real d = dealias_factor<Real>(kx, ky, N, a.kmax_sqr, a.dealias, a.houli_int, a.kolm);
            Lbuf[i * TC + c] = cscale(kappa, a.norm2 * d);
        }
        __syncthreads();
        C v[1][E];
#pragma unroll
        for (int m = 0; m < E; ++m) v[0][m] = Lbuf[(t + T * m) * TC + c];
        fft_batched<N, +1, 1>(v, IlvPolicy<N, TC, C>{sm, c}, seed, t);
        if (valid) {
#pragma unroll
            for (int m = 0; m < E; ++m) a.mu[(size_t)(t + T * m) * ldc + ky] = v[0][m];
        }
    }
}

template <typename Real>
struct AdjRowArgs {
    using C = typename Cx<Real>::T;
    const C* mu;          // x-space mu_x [x][ldc]
    const C* cap_uv;      // captured real fields of the forward stage: (u, v) and
    const C* cap_w;       // (w_x, w_y) as complex pairs, [x][y]
    C* P0;                // outputs: x-space half spectra of w_x mu, w_y mu, u mu, v mu
    C* P1;
    C* P2;
    C* P3;
    const C* tw;
    int ldc;
};

// Adjoint row pass: one team of T threads per row x, TC = 2 PAIRS rows per block.
template <typename Real, int N, int PAIRS>
__global__ void __launch_bounds__(Plan<N>::T * 2 * PAIRS) adj_row_kernel(AdjRowArgs<Real> a) {
    using C = typename Cx<Real>::T;
    using P = Plan<N>;
    constexpr int T = P::T;
    constexpr int E = N / T;
    constexpr int TC = 2 * PAIRS;
    using TL = TeamLayout<N>;
    using RS = RowSmem<Real, N, TC>;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int g = threadIdx.x / T;
    const int t = threadIdx.x % T;
    const int x = blockIdx.x * TC + g;
    C* region = reinterpret_cast<C*>(smraw) + (size_t)g * RS::TEAM;
    const TwSeed<C> seed = twiddle_seeds<N>(a.tw, t);
    const TeamPolicy<N, C> pol{region, 1 + g};
    // mu = c2r(mu_x) along y: Hermitian extension, real parts at ky = 0 and N/2
    C z[1][E];
    {
        const C* __restrict__ M = a.mu + (size_t)x * a.ldc;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int y = t + T * m;
            const int yy = (y <= N / 2) ? y : N - y;
            const C p = M[yy];
            if (y == 0 || y == N / 2) z[0][m] = cmake<C>(p.x, 0);
            else if (y < N / 2) z[0][m] = p;
            else z[0][m] = cconj(p);
        }
    }
    fft_batched<N, +1, 1>(z, pol, seed, t);
    // products with the captured fields, packed two per complex transform
    C q[2][E];
    {
        const C* __restrict__ cu = a.cap_uv + (size_t)x * N;
        const C* __restrict__ cw = a.cap_w + (size_t)x * N;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int y = t + T * m;
            const Real mu = z[0][m].x;
            const C uv = cu[y], wxy = cw[y];
            q[0][m] = cmake<C>(wxy.x * mu, wxy.y * mu);
            q[1][m] = cmake<C>(uv.x * mu, uv.y * mu);
        }
    }
    fft_batched<N, -1, 2>(q, pol, seed, t);
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int m = 0; m < E; ++m) region[b * TL::ROWS + TL::slot(t + T * m)] = q[b][m];
    pol.sync();
    // split each packed transform: X_a = (Z_k + conj Z_{N-k})/2, X_b = (Z_k - conj Z_{N-k})/(2i)
    C* outs[4] = {a.P0, a.P1, a.P2, a.P3};
#pragma unroll
    for (int b = 0; b < 2; ++b) {
        C* __restrict__ oa = outs[2 * b] + (size_t)x * a.ldc;
        C* __restrict__ ob = outs[2 * b + 1] + (size_t)x * a.ldc;
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int k = t + T * m;
            if (k <= N / 2) {
                const C zk = region[b * TL::ROWS + TL::slot(k)];
                const C zm = region[b * TL::ROWS + TL::slot((N - k) & (N - 1))];
                oa[k] = cmake<C>((Real)0.5 * (zk.x + zm.x), (Real)0.5 * (zk.y - zm.y));
                ob[k] = cmake<C>((Real)0.5 * (zk.y + zm.y), (Real)0.5 * (zm.x - zk.x));
            }
        }
    }
}

// Objective and its W-gradient at the final state: enstrophy
// Z = cZ sum_j c_j |w_j|^2 -> 2 cZ w; palinstrophy P = cZ sum_j c_j k^2 |w_j|^2
// -> 2 cZ k^2 w (cZ = 4 pi^2 0.5/(Nx Ny)^2, mean mode excluded;
// sys_msr.c:190-227, 356-363).  One FP64 partial sum per block (fixed grid, so
// the host's ordered sum of the partials is deterministic).
template <typename Real>
__global__ void __launch_bounds__(256) adj_objective_kernel(const typename Cx<Real>::T* state,
                                                            typename Cx<Real>::T* lam, int nx, int nyf, int ldc,
                                                            double cz, int palin, double* partials) {
    const long long n = (long long)nx * nyf;
    double acc = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / nyf), ky = (int)(q % nyf);
        const int kx = (i <= nx / 2) ? i : i - nx;
        const size_t o = (size_t)i * ldc + ky;
        double f = palin ? (double)(kx * kx + ky * ky) : 1.0;
        if (kx == 0 && ky == 0) f = 0.0;
        const auto w = state[o];
        const double w2 = (double)w.x * (double)w.x + (double)w.y * (double)w.y;
        acc += ((ky == 0 || ky == nyf - 1) ? 1.0 : 2.0) * f * w2;
        if (lam) lam[o] = cscale(w, (Real)(2.0 * cz * f));
    }
    __shared__ double red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        partials[blockIdx.x] = cz * tot;
    }
}

// <a, b>_W = sum_j c_j Re(conj(a_j) b_j) over the half spectrum, FP64 partials per block.
template <typename Real>
__global__ void __launch_bounds__(256) adj_wdot_kernel(const typename Cx<Real>::T* a, const typename Cx<Real>::T* b,
                                                       int nx, int nyf, int ldc, double* partials) {
    const long long n = (long long)nx * nyf;
    double acc = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / nyf), ky = (int)(q % nyf);
        const size_t o = (size_t)i * ldc + ky;
        const auto x = a[o], y = b[o];
        acc += ((ky == 0 || ky == nyf - 1) ? 1.0 : 2.0) * ((double)x.x * (double)y.x + (double)x.y * (double)y.y);
    }
    __shared__ double red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        partials[blockIdx.x] = tot;
    }
}

}  // namespace ns2d
