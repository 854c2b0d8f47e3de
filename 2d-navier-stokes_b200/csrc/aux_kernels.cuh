// aux_kernels.cuh -- transforms to real space with reductions (GetMaxData,
// GetTimestep, real-space output) and small elementwise helpers.
#pragma once
#include "kernels.cuh"

namespace ns2d {

// Spectral source of one inverse x-FFT: element (i, j) at p[i*rs + j*es];
// op 0 = as is, 1 = u_hat = ky (i/k^2) w, 2 = v_hat = -kx (i/k^2) w
// (Solver/src/solver.c:2184-2196, 2393-2410).
template <typename Real>
struct InvField {
    using C = typename Cx<Real>::T;
    const C* p;
    long long rs, es;
    int op;
    C* dst;  // [nx][ldc] x-space output
};

template <typename Real>
struct InvArgs {
    InvField<Real> f[2];
    int nf;
    int nyf, ldc;
    const typename Cx<Real>::T* tw;
    // op 1/2 wavenumbers for a scrambled index: kx from row i of the loop, the
    // source element from the flat position (see cfl_scramble_kernel)
};

template <typename Real, int N, int TC>
__global__ void __launch_bounds__(Plan<N>::T * TC) col_inv_kernel(InvArgs<Real> a) {
    using C = typename Cx<Real>::T;
    constexpr int T = Plan<N>::T;
    constexpr int E = N / T;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int c = threadIdx.x % TC;
    const int t = threadIdx.x / TC;
    const int ky = blockIdx.x * TC + c;
    const bool valid = ky < a.nyf;
    const int kyc = valid ? ky : 0;
    const TwSeed<C> seed = twiddle_seeds<N>(a.tw, t);
    for (int f = 0; f < a.nf; ++f) {
        const InvField<Real> F = a.f[f];
        C v[E];
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int i = t + T * m;
            const int kx = (i <= N / 2) ? i : i - N;
            C w = valid ? F.p[(long long)i * F.rs + (long long)kyc * F.es] : cmake<C>(0, 0);
            if (F.op != 0) {
                if (kx == 0 && ky == 0) {
                    w = cmake<C>(0, 0);
                } else {
                    const double inv = 1.0 / (double)(kx * kx + ky * ky);
                    if (F.op == 1) {
                        const Real s = (Real)((double)ky * inv);
                        w = cmake<C>(-s * w.y, s * w.x);
                    } else {
                        const Real s = (Real)((double)kx * inv);
                        w = cmake<C>(s * w.y, -s * w.x);
                    }
                }
            }
            v[m] = w;
        }
        fft<N, +1, TC>(v, sm, seed, t, c);
        if (valid) {
#pragma unroll
            for (int m = 0; m < E; ++m) F.dst[(size_t)(t + T * m) * a.ldc + ky] = v[m];
        }
    }
}

enum RowC2ROp : int { R2_MAXABS = 0, R2_CFL = 1, R2_STORE = 2 };

template <typename Real>
struct RowC2RArgs {
    using C = typename Cx<Real>::T;
    const C* A;      // x-space field (real part of the output)
    const C* B;      // x-space field (imaginary part), may be null
    int ldc;
    const C* tw;
    double scale;    // 1/(Nx Ny)
    double dx, dy;   // CFL
    unsigned long long* maxbits;  // atomicMax target (bits of a non-negative double)
    double* outA;    // R2_STORE: [nx][ny] real outputs
    double* outB;
};

template <typename Real, int N, int PAIRS, int OP>
__global__ void __launch_bounds__(Plan<N>::T * 2 * PAIRS) row_c2r_kernel(RowC2RArgs<Real> a) {
    using C = typename Cx<Real>::T;
    constexpr int T = Plan<N>::T;
    constexpr int E = N / T;
    constexpr int TC = 2 * PAIRS;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int g = threadIdx.x % TC;
    const int t = threadIdx.x / TC;
    const int x = blockIdx.x * TC + g;
    const C* rA = a.A + (size_t)x * a.ldc;
    const C* rB = a.B ? a.B + (size_t)x * a.ldc : nullptr;
    const TwSeed<C> seed = twiddle_seeds<N>(a.tw, t);
    C z[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int y = t + T * m;
        const C zero = cmake<C>(0, 0);
        if (y == 0 || y == N / 2) {
            z[m] = cmake<C>(rA[y].x, rB ? rB[y].x : (Real)0);
        } else if (y < N / 2) {
            const C p = rA[y], q = rB ? rB[y] : zero;
            z[m] = cmake<C>(p.x - q.y, p.y + q.x);
        } else {
            const C p = rA[N - y], q = rB ? rB[N - y] : zero;
            z[m] = cmake<C>(p.x + q.y, q.x - p.y);
        }
    }
    fft<N, +1, TC>(z, sm, seed, t, g);
    double mx = 0.0;
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int y = t + T * m;
        const double u = (double)z[m].x * a.scale;
        const double v = (double)z[m].y * a.scale;
        if constexpr (OP == R2_MAXABS) {
            mx = fmax(mx, fmax(fabs(u), fabs(v)));
            if (!(u == u) || !(v == v)) mx = __longlong_as_double(0x7ff8000000000000ll);
        } else if constexpr (OP == R2_CFL) {
            // pi * (|u|/dx + |v|/dy)  (Solver/src/solver.c:2436-2438)
            mx = fmax(3.14159265358979323846 * (fabs(u) / a.dx + fabs(v) / a.dy), mx);
        } else {
            a.outA[(size_t)x * N + y] = u;
            if (a.outB) a.outB[(size_t)x * N + y] = v;
        }
    }
    if constexpr (OP != R2_STORE) {
        unsigned long long bits = (unsigned long long)__double_as_longlong(mx);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long other = __shfl_xor_sync(0xffffffffu, bits, o);
            bits = other > bits ? other : bits;
        }
        if ((threadIdx.x & 31) == 0) atomicMax(a.maxbits, bits);
    }
}

// CFL velocity spectrum with the reference's row index tmp = (i*Ny)/2 + 1
// (Solver/src/solver.c:2393-2410), written into a persistent buffer with the
// reference's interleaved [nx][nyf][2] layout; the state is read at the same
// scrambled flat position.  Entries the loop never reaches keep their previous
// contents, as in the reference.  Consecutive rows overlap by one element;
// the reference's sequential loop leaves row i+1's j = 0 value there, so the
// last element of every row but the last is not written here.
template <typename Real>
__global__ void cfl_scramble_kernel(const typename Cx<Real>::T* __restrict__ state, int ldc,
                                    typename Cx<Real>::T* __restrict__ uhat, int nx, int ny, int quirk) {
    using C = typename Cx<Real>::T;
    const int nyf = ny / 2 + 1;
    const long long n = (long long)nx * nyf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / nyf);
        const int j = (int)(q % nyf);
        if (quirk && j == nyf - 1 && i < nx - 1) continue;
        const long long idx = quirk ? ((long long)i * ny / 2 + 1 + j) : q;
        const int kx = (i <= nx / 2) ? i : i - nx;
        const int ky = j;
        C u = cmake<C>(0, 0), v = cmake<C>(0, 0);
        if (kx != 0 || ky != 0) {
            const C w = state[(size_t)(idx / nyf) * ldc + (size_t)(idx % nyf)];
            const double inv = 1.0 / (double)(kx * kx + ky * ky);
            const Real su = (Real)((double)ky * inv);
            const Real sv = (Real)((double)kx * inv);
            u = cmake<C>(-su * w.y, su * w.x);
            v = cmake<C>(sv * w.y, -sv * w.x);
        }
        uhat[2 * idx + 0] = u;
        uhat[2 * idx + 1] = v;
    }
}

// Pack/unpack between the reference layout [nx][nyf] (double) and the device
// layout [nx][ldc] (Real).
template <typename Real>
__global__ void pack_kernel(const double2* __restrict__ src, typename Cx<Real>::T* __restrict__ dst, int nx, int nyf,
                            int ldc) {
    using C = typename Cx<Real>::T;
    const long long n = (long long)nx * nyf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / nyf), j = (int)(q % nyf);
        const double2 s = src[q];
        dst[(size_t)i * ldc + j] = cmake<C>((Real)s.x, (Real)s.y);
    }
}
template <typename Real>
__global__ void unpack_kernel(const typename Cx<Real>::T* __restrict__ src, double2* __restrict__ dst, int nx, int nyf,
                              int ldc) {
    const long long n = (long long)nx * nyf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / nyf), j = (int)(q % nyf);
        const auto s = src[(size_t)i * ldc + j];
        dst[q] = make_double2((double)s.x, (double)s.y);
    }
}

// Forward (e^{-i...}) unnormalised transform passes of a real field, the r2c
// of FFTW's fftw_mpi_plan_dft_r2c_2d that the reference applies to real-space
// initial conditions (Solver/src/solver.c:1178, 1200, 1833, 1873).
//   ROWS: block = TC rows, one transform per row: real in[x][y] (double,
//         [nx][ny]) -> row spectrum out[x][ky] for ky <= ny/2 ([nx][ldc]).
//   COLS: block = TC columns: out[i][ky] = sum_x in[x][ky] e^{-2 pi i x kx / nx}.
// Used at set-up only (initial conditions, file input), so rows are read
// with the columns' interleaved smem layout instead of a packed real transform.
enum FwdPass : int { FWD_ROWS = 0, FWD_COLS = 1 };

template <typename Real, int N, int TC, int PASS>
__global__ void __launch_bounds__(Plan<N>::T * TC) fwd_kernel(const double* __restrict__ real_in,
                                                              const typename Cx<Real>::T* __restrict__ in,
                                                              typename Cx<Real>::T* __restrict__ out, int nlines,
                                                              int ldc, const typename Cx<Real>::T* __restrict__ tw) {
    using C = typename Cx<Real>::T;
    constexpr int T = Plan<N>::T;
    constexpr int E = N / T;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int c = threadIdx.x % TC;
    const int t = threadIdx.x / TC;
    const int line = blockIdx.x * TC + c;
    const bool valid = line < nlines;
    const int lc = valid ? line : 0;
    const TwSeed<C> seed = twiddle_seeds<N>(tw, t);
    C v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
        const int e = t + T * m;
        if constexpr (PASS == FWD_ROWS) {
            v[m] = cmake<C>(valid ? (Real)real_in[(size_t)lc * N + e] : (Real)0, (Real)0);
        } else {
            v[m] = valid ? in[(size_t)e * ldc + lc] : cmake<C>(0, 0);
        }
    }
    fft<N, -1, TC>(v, sm, seed, t, c);
    if (valid) {
#pragma unroll
        for (int m = 0; m < E; ++m) {
            const int e = t + T * m;
            if constexpr (PASS == FWD_ROWS) {
                if (e <= N / 2) out[(size_t)lc * ldc + e] = v[m];
            } else {
                out[(size_t)e * ldc + lc] = v[m];
            }
        }
    }
}

// Mean-flow sums of ComputeSystemMeasurables for one call: for every row
// kx, mean_y = sum_ky c_ky |v_hat| (Solver/src/sys_msr.c:199, 227), and for
// every column ky, mean_x = sum_kx c_ky |u_hat|, with u_hat = i ky w/k^2,
// v_hat = -i kx w/k^2, c = 1 on the ky = 0 and ky = ny/2 columns and 2
// elsewhere, the (0,0) mode skipped.  Blocks [0, nx) reduce rows, blocks
// [nx, nx + nyf) columns; out = [mean_y (nx) | mean_x (nyf)].  The column sum
// is what sys_msr.c:338-348 intends: that loop indexes the ky array with the
// row counter and reuses the last k^2 of the previous loop.
template <typename Real>
__global__ void __launch_bounds__(256) mean_flow_kernel(const typename Cx<Real>::T* __restrict__ w, int nx, int nyf,
                                                        int ldc, double* __restrict__ out) {
    __shared__ double red[8];
    const bool row = blockIdx.x < (unsigned)nx;
    const int line = row ? blockIdx.x : blockIdx.x - nx;
    const int count = row ? nyf : nx;
    double acc = 0.0;
    for (int q = threadIdx.x; q < count; q += blockDim.x) {
        const int i = row ? line : q;
        const int ky = row ? q : line;
        const int kx = (i <= nx / 2) ? i : i - nx;
        if (kx == 0 && ky == 0) continue;
        const double k2 = (double)kx * kx + (double)ky * ky;
        const auto z = w[(size_t)i * ldc + ky];
        const double wr = (double)z.x, wi = (double)z.y;
        const double kk = row ? (double)kx : (double)ky;
        const double a = hypot(kk * wi / k2, kk * wr / k2);
        acc += (ky == 0 || ky == nyf - 1) ? a : 2.0 * a;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
        out[blockIdx.x] = s;
    }
}

// ApplyDealiasing (Solver/src/solver.c:1039-1099) on `dim` interleaved fields
// in the reference layout.
template <typename Real>
__global__ void dealias_kernel(typename Cx<Real>::T* a, int dim, int nx, int ny, int kmax_sqr, int dealias, int houli_int,
                               int kolm) {
    using C = typename Cx<Real>::T;
    const int nyf = ny / 2 + 1;
    const long long n = (long long)nx * nyf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / nyf), ky = (int)(q % nyf);
        const int kx = (i <= nx / 2) ? i : i - nx;
        const double k2 = (double)kx * kx + ky * ky;
        for (int l = 0; l < dim; ++l) {
            C v = a[q * dim + l];
            if (dealias == 0) {
                if (k2 >= (double)kmax_sqr || (kolm && kx == 0)) v = cmake<C>(0, 0);
            } else {
                v = cscale(v, houli_filter<Real>(kx, ky, nx, ny, houli_int));
            }
            a[q * dim + l] = v;
        }
    }
}

// ForceConjugacy (Solver/src/solver.c:2074-2107): state[kx<0, 0] = conj(src[|kx|, 0]).
template <typename Real>
__global__ void conj_kernel(typename Cx<Real>::T* state, int ldc, const typename Cx<Real>::T* src, long long src_stride,
                            int nx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx || i <= nx / 2) return;
    const int kx = i - nx;
    state[(size_t)i * ldc] = cconj(src[(long long)(-kx) * src_stride]);
}

// ZERO forcing (ComputeForcing, Solver/src/force.c:527-533): every mode with
// |kx| <= k or |ky| <= k of the state is set to zero (modes of force.c:436-501).
template <typename Real>
__global__ void zero_modes_kernel(typename Cx<Real>::T* state, int nx, int nyf, int ldc, int k) {
    using C = typename Cx<Real>::T;
    const long long n = (long long)nx * nyf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / nyf), j = (int)(q % nyf);
        const int kx = (i <= nx / 2) ? i : i - nx;
        if ((kx < 0 ? -kx : kx) <= k || j <= k) state[(size_t)i * ldc + j] = cmake<C>(0, 0);
    }
}

// Forcing of listed modes: value m goes to flat index idx[m] of the
// reference layout [nx][nyf] (run_data->forcing_indx), other modes stay 0.
template <typename Real>
__global__ void scatter_forcing_kernel(typename Cx<Real>::T* field, int nyf, int ldc, const int32_t* idx,
                                       const double2* val, int n) {
    using C = typename Cx<Real>::T;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
        const int q = idx[m];
        field[(size_t)(q / nyf) * ldc + (q % nyf)] = cmake<C>((decltype(C::x))val[m].x, (decltype(C::x))val[m].y);
    }
}

// Dormand-Prince 5(4) (RK5DPStep, Solver/src/solver.c:360-570, corrected).
struct DpCoef {
    double c[7];
    int n;
};

// Stage input X = y0 + dt sum_{r < n} c_r k_r over the valid columns.
template <typename Real>
__global__ void dp_combine_kernel(typename Cx<Real>::T* __restrict__ x, const typename Cx<Real>::T* __restrict__ y0,
                                  const typename Cx<Real>::T* k0, const typename Cx<Real>::T* k1,
                                  const typename Cx<Real>::T* k2, const typename Cx<Real>::T* k3,
                                  const typename Cx<Real>::T* k4, const typename Cx<Real>::T* k5, DpCoef cf,
                                  double dt, int nx, int nyf, int ldc) {
    using C = typename Cx<Real>::T;
    const C* ks[6] = {k0, k1, k2, k3, k4, k5};
    const long long n = (long long)nx * nyf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const size_t o = (size_t)(q / nyf) * ldc + (size_t)(q % nyf);
        double ar = 0.0, ai = 0.0;
        for (int r = 0; r < cf.n; ++r) {
            const C v = ks[r][o];
            ar += cf.c[r] * (double)v.x;
            ai += cf.c[r] * (double)v.y;
        }
        const C y = y0[o];
        x[o] = cmake<C>((Real)((double)y.x + dt * ar), (Real)((double)y.y + dt * ai));
    }
}

// Fifth-order solution y5 into the state (zero mean) and the embedded error
// sum_j (|y5 - y4| / (atol + rtol max(|y0|, |y5|)))^2, one FP64 partial per block.
template <typename Real>
__global__ void __launch_bounds__(256) dp_final_kernel(typename Cx<Real>::T* __restrict__ state,
                                                       const typename Cx<Real>::T* __restrict__ y0,
                                                       const typename Cx<Real>::T* const* __restrict__ k,
                                                       DpCoef b5, DpCoef b4, double dt, double atol, double rtol,
                                                       int nx, int nyf, int ldc, double* partials) {
    using C = typename Cx<Real>::T;
    const long long n = (long long)nx * nyf;
    double acc = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / nyf), j = (int)(q % nyf);
        const size_t o = (size_t)i * ldc + j;
        if (i == 0 && j == 0) {
            state[o] = cmake<C>(0, 0);
            continue;
        }
        double s5r = 0.0, s5i = 0.0, s4r = 0.0, s4i = 0.0;
        for (int r = 0; r < 7; ++r) {
            const C v = k[r][o];
            s5r += b5.c[r] * (double)v.x;
            s5i += b5.c[r] * (double)v.y;
            s4r += b4.c[r] * (double)v.x;
            s4i += b4.c[r] * (double)v.y;
        }
        const C y = y0[o];
        const double y5r = (double)y.x + dt * s5r, y5i = (double)y.y + dt * s5i;
        const double y4r = (double)y.x + dt * s4r, y4i = (double)y.y + dt * s4i;
        const double sc = atol + rtol * fmax(hypot((double)y.x, (double)y.y), hypot(y5r, y5i));
        const double e = hypot(y5r - y4r, y5i - y4i) / sc;
        acc += e * e;
        state[o] = cmake<C>((Real)y5r, (Real)y5i);
    }
    __shared__ double red[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        partials[blockIdx.x] = tot;
    }
}

// RK5DPStep as the reference writes it (Solver/src/solver.c:404-466): stage
// input X = w + (dt a_1) k_1 + (dt a_2) k_2 + ..., summed left to right from
// the live state w, skipping the zero coefficients the reference leaves out
// (the a72 of the seventh stage).  cf.c[r] holds the products dt * a_r.
template <typename Real>
__global__ void dpw_combine_kernel(typename Cx<Real>::T* __restrict__ x, const typename Cx<Real>::T* __restrict__ w,
                                   const typename Cx<Real>::T* k0, const typename Cx<Real>::T* k1,
                                   const typename Cx<Real>::T* k2, const typename Cx<Real>::T* k3,
                                   const typename Cx<Real>::T* k4, const typename Cx<Real>::T* k5, DpCoef cf,
                                   int nx, int nyf, int ldc) {
    using C = typename Cx<Real>::T;
    const C* ks[6] = {k0, k1, k2, k3, k4, k5};
    const long long n = (long long)nx * nyf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const size_t o = (size_t)(q / nyf) * ldc + (size_t)(q % nyf);
        const C y = w[o];
        double xr = (double)y.x, xi = (double)y.y;
        for (int r = 0; r < cf.n; ++r) {
            if (cf.c[r] == 0.0) continue;
            const C v = ks[r][o];
            xr = xr + cf.c[r] * (double)v.x;
            xi = xi + cf.c[r] * (double)v.y;
        }
        x[o] = cmake<C>((Real)xr, (Real)xi);
    }
}

// Update and error of RK5DPStep as written (Solver/src/solver.c:470-566):
//   w <- w (2 - D)/(2 + D) + 2 dt/(2 + D) (b1 k1 + b3 k3 + b4 k4 + b5 k5 + b6 k6)
// (explicit w + sum dt (b k) for the Euler system), the mean mode 0; then, when
// iters > 1, the error sum of the real parts (dp_ho_step is a double and pow()
// takes the real part of its complex argument):
//   ho = Re(w_new + (sum_{s<=6} dt (bs_s k_s)) + dt (bs7 k7)),
//   e  = (Re w_new - ho) / (DP_ABS_TOL + max(|w_last|, |w_new|) DP_REL_TOL),
// one FP64 partial of sum e^2 per block, and w_last <- w_new.
template <typename Real>
__global__ void __launch_bounds__(256) dpw_final_kernel(typename Cx<Real>::T* __restrict__ state,
                                                        typename Cx<Real>::T* __restrict__ w_last,
                                                        const typename Cx<Real>::T* const* __restrict__ k, DpCoef b5,
                                                        DpCoef bs, double dt, int euler, LinOp lin, int iters, int nx,
                                                        int nyf, int ldc, double* partials) {
    using C = typename Cx<Real>::T;
    const long long n = (long long)nx * nyf;
    double acc = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / nyf), j = (int)(q % nyf);
        const size_t o = (size_t)i * ldc + j;
        if (i == 0 && j == 0) {
            state[o] = cmake<C>(0, 0);
            if (iters > 1) w_last[o] = cmake<C>(0, 0);
            continue;
        }
        const int kx = (i <= nx / 2) ? i : i - nx;
        const C w = state[o];
        double wr, wi;
        if (euler) {
            double sr = 0.0, si = 0.0;
            bool first = true;
            for (int r = 0; r < 7; ++r) {
                if (b5.c[r] == 0.0) continue;
                const C v = k[r][o];
                const double tr = dt * (b5.c[r] * (double)v.x), ti = dt * (b5.c[r] * (double)v.y);
                sr = first ? tr : sr + tr;
                si = first ? ti : si + ti;
                first = false;
            }
            wr = (double)w.x + sr;
            wi = (double)w.y + si;
        } else {
            double sr = 0.0, si = 0.0;
            bool first = true;
            for (int r = 0; r < 7; ++r) {
                if (b5.c[r] == 0.0) continue;
                const C v = k[r][o];
                const double tr = b5.c[r] * (double)v.x, ti = b5.c[r] * (double)v.y;
                sr = first ? tr : sr + tr;
                si = first ? ti : si + ti;
                first = false;
            }
            const double D = dt * lin_bracket(lin, (double)(kx * kx + j * j));
            const double f1 = (2.0 - D) / (2.0 + D), f2 = (2.0 * dt) / (2.0 + D);
            wr = (double)w.x * f1 + f2 * sr;
            wi = (double)w.y * f1 + f2 * si;
        }
        const C wn = cmake<C>((Real)wr, (Real)wi);
        if (iters > 1) {
            double hr = 0.0;
            bool first = true;
            for (int r = 0; r < 6; ++r) {
                if (bs.c[r] == 0.0) continue;
                const double t = dt * (bs.c[r] * (double)k[r][o].x);
                hr = first ? t : hr + t;
                first = false;
            }
            const double ho = ((double)wn.x + hr) + dt * (bs.c[6] * (double)k[6][o].x);
            const C wl = w_last[o];
            const double a = hypot((double)wl.x, (double)wl.y), b = hypot((double)wn.x, (double)wn.y);
            const double denom = 1e-7 + (a > b ? a : b) * 1e-7;
            const double e = ((double)wn.x - ho) / denom;
            acc += e * e;
            w_last[o] = wn;
        }
        state[o] = wn;
    }
    __shared__ double red[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        partials[blockIdx.x] = tot;
    }
}

}  // namespace ns2d
