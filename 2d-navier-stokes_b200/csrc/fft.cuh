// fft.cuh -- register/shared-memory Stockham FFT for one-dimensional passes of
// the pseudospectral step (sm_100a).  Written from the DFT definition
//     X[k] = sum_n x[n] exp(sign * 2 pi i n k / N)
// and the Stockham auto-sort formulation: stage (R, Ns) takes butterfly j,
// loads x[j + r N/R], twiddles by exp(sign 2 pi i (j mod Ns) r / (Ns R)),
// does an R-point DFT and stores to (j / Ns) Ns R + (j mod Ns) + r Ns.
//
// Every plan has the same radix in its first and last stage with one
// butterfly per thread there, so a thread t of the T threads that share one
// transform holds elements e = t + T m (m < E = N / T) both before the first
// stage and after the last one.  A forward transform can therefore feed an
// inverse transform (or an elementwise epilogue) without any data exchange.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ns2d {

template <typename Real>
struct Cx;
template <>
struct Cx<double> {
    using T = double2;
};
template <>
struct Cx<float> {
    using T = float2;
};

template <typename C>
__device__ __forceinline__ C cmake(decltype(C::x) a, decltype(C::x) b) {
    C r;
    r.x = a;
    r.y = b;
    return r;
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return cmake<C>(a.x + b.x, a.y + b.y); }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return cmake<C>(a.x - b.x, a.y - b.y); }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) { return cmake<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C>
__device__ __forceinline__ C cconj(C a) { return cmake<C>(a.x, -a.y); }
template <typename C>
__device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return cmake<C>(a.x * s, a.y * s); }
// a * (sign i)
template <int SIGN, typename C>
__device__ __forceinline__ C cmul_i(C a) {
    return SIGN > 0 ? cmake<C>(-a.y, a.x) : cmake<C>(a.y, -a.x);
}

// Constant twiddle exp(SIGN * 2 pi i K / R) applied to a, for the in-register
// small DFTs (R <= 16).  Exact cases (k R/4 multiples) avoid multiplications.
template <int R, int K, int SIGN, typename C>
__device__ __forceinline__ C ctw(C a) {
    using Real = decltype(C::x);
    constexpr int k = ((K % R) + R) % R;
    if constexpr (k == 0) {
        return a;
    } else if constexpr (4 * k == R) {
        return cmul_i<SIGN>(a);
    } else if constexpr (2 * k == R) {
        return cmake<C>(-a.x, -a.y);
    } else if constexpr (4 * k == 3 * R) {
        return cmul_i<-SIGN>(a);
    } else if constexpr (8 * k == R || 8 * k == 3 * R || 8 * k == 5 * R || 8 * k == 7 * R) {
        // 45-degree family: exp(s i pi/4) = (1 + s i)/sqrt2, rotated by multiples of i
        constexpr Real h = (Real)0.70710678118654752440;
        C b;
        if constexpr (SIGN > 0) b = cmake<C>((a.x - a.y) * h, (a.x + a.y) * h);
        else b = cmake<C>((a.x + a.y) * h, (a.y - a.x) * h);
        if constexpr (8 * k == R) return b;
        else if constexpr (8 * k == 3 * R) return cmul_i<SIGN>(b);
        else if constexpr (8 * k == 5 * R) return cmake<C>(-b.x, -b.y);
        else return cmul_i<-SIGN>(b);
    } else {
        // R == 16, odd k: cos/sin of multiples of pi/8
        constexpr Real c1 = (Real)0.92387953251128675613;  // cos(pi/8)
        constexpr Real s1 = (Real)0.38268343236508977173;  // sin(pi/8)
        constexpr int q = k % 4;                           // 1 or 3 within the quadrant
        constexpr Real cr = (q == 1) ? c1 : s1;
        constexpr Real si = (q == 1) ? s1 : c1;
        C b = cmake<C>(a.x * cr - a.y * (SIGN * si), a.x * (SIGN * si) + a.y * cr);
        constexpr int quad = k / 4;
        if constexpr (quad == 0) return b;
        else if constexpr (quad == 1) return cmul_i<SIGN>(b);
        else if constexpr (quad == 2) return cmake<C>(-b.x, -b.y);
        else return cmul_i<-SIGN>(b);
    }
}

// In-register DFT of size R (power of two <= 16) on v[0], v[S], ..., v[(R-1)S],
// result in natural order in the same slots.  Recursive radix-2 DIT.
template <int R, int SIGN, int S, typename C>
struct SmallDFT {
    __device__ __forceinline__ static void run(C* v) {
        SmallDFT<R / 2, SIGN, 2 * S, C>::run(v);      // even samples
        SmallDFT<R / 2, SIGN, 2 * S, C>::run(v + S);  // odd samples
        C tmp[R];
#pragma unroll
        for (int k = 0; k < R; ++k) tmp[k] = v[k * S];
        // tmp[2m] = E_m, tmp[2m+1] = O_m
        combine<0>(tmp, v);
    }
    template <int K>
    __device__ __forceinline__ static void combine(const C* tmp, C* v) {
        if constexpr (K < R / 2) {
            C e = tmp[2 * K];
            C o = ctw<R, K, SIGN>(tmp[2 * K + 1]);
            v[K * S] = cadd(e, o);
            v[(K + R / 2) * S] = csub(e, o);
            combine<K + 1>(tmp, v);
        }
    }
};
template <int SIGN, int S, typename C>
struct SmallDFT<1, SIGN, S, C> {
    __device__ __forceinline__ static void run(C*) {}
};

template <int R, int SIGN, typename C>
__device__ __forceinline__ void small_dft(C* v) { SmallDFT<R, SIGN, 1, C>::run(v); }

// Plans: first and last radix equal, one butterfly per thread at both ends.
template <int N>
struct Plan;
template <> struct Plan<16>   { static constexpr int T = 4,   S = 2, R0 = 4,  R1 = 4,  R2 = 1; };
template <> struct Plan<32>   { static constexpr int T = 8,   S = 3, R0 = 4,  R1 = 2,  R2 = 4; };
template <> struct Plan<64>   { static constexpr int T = 8,   S = 2, R0 = 8,  R1 = 8,  R2 = 1; };
template <> struct Plan<128>  { static constexpr int T = 16,  S = 3, R0 = 8,  R1 = 2,  R2 = 8; };
template <> struct Plan<256>  { static constexpr int T = 16,  S = 2, R0 = 16, R1 = 16, R2 = 1; };
template <> struct Plan<512>  { static constexpr int T = 64,  S = 3, R0 = 8,  R1 = 8,  R2 = 8; };
template <> struct Plan<1024> { static constexpr int T = 64,  S = 3, R0 = 16, R1 = 4,  R2 = 16; };
template <> struct Plan<2048> { static constexpr int T = 128, S = 3, R0 = 16, R1 = 8,  R2 = 16; };

// Shared-memory element slot for transform element e of lane-column c when
// TC transforms are interleaved (c fastest).  One padding row per PADR rows
// breaks the stride-R store pattern of the first stage across banks.
template <int N, int TC>
struct SmemLayout {
    static constexpr int PADR = Plan<N>::R0;
    static constexpr int ROWS = N + N / PADR;
    static constexpr int ELEMS = ROWS * TC;
    __device__ __forceinline__ static int slot(int e, int c) { return (e + e / PADR) * TC + c; }
};

// Twiddle exp(SIGN 2 pi i m / N) from the table tw[m] = exp(-2 pi i m / N).
template <int SIGN, typename C>
__device__ __forceinline__ C twiddle(const C* __restrict__ tw, int m) {
    C w = __ldg(tw + m);
    if constexpr (SIGN > 0) w.y = -w.y;
    return w;
}

// Middle stage: reads smem (pattern of the previous stage's writes), writes smem.
template <int N, int R, int NS, int SIGN, int TC, typename C>
__device__ __forceinline__ void middle_stage(C* sm, const C* __restrict__ tw, int t, int c) {
    using P = Plan<N>;
    using L = SmemLayout<N, TC>;
    constexpr int BPT = N / (R * P::T);
    static_assert(BPT * R * P::T == N, "plan");
    C v[BPT][R];
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
        const int j = t + P::T * b;
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = sm[L::slot(j + r * (N / R), c)];
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
        const int j = t + P::T * b;
        const int k = j % NS;
#pragma unroll
        for (int r = 1; r < R; ++r) v[b][r] = cmul(v[b][r], twiddle<SIGN>(tw, k * r * (N / (NS * R))));
        small_dft<R, SIGN>(v[b]);
        const int base = (j / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) sm[L::slot(base + r * NS, c)] = v[b][r];
    }
    __syncthreads();
}

// Full transform on v[m] = x[t + T m] (m < E), result in the same pattern.
// sm must hold SmemLayout<N,TC>::ELEMS elements shared by the TC transforms of
// the block; all threads of the block must call this together.
template <int N, int SIGN, int TC, typename C>
__device__ __forceinline__ void fft(C* v, C* sm, const C* __restrict__ tw, int t, int c) {
    using P = Plan<N>;
    using L = SmemLayout<N, TC>;
    constexpr int E = N / P::T;
    static_assert(E == P::R0, "first stage must be one butterfly per thread");
    // stage 0 (Ns = 1): no twiddles, outputs at t*R0 + r
    small_dft<P::R0, SIGN>(v);
#pragma unroll
    for (int r = 0; r < P::R0; ++r) sm[L::slot(t * P::R0 + r, c)] = v[r];
    __syncthreads();
    constexpr int NS1 = P::R0;
    if constexpr (P::S == 3) {
        middle_stage<N, P::R1, NS1, SIGN, TC>(sm, tw, t, c);
    }
    constexpr int RL = (P::S == 3) ? P::R2 : P::R1;
    constexpr int NSL = N / RL;
    static_assert(RL == P::R0, "last radix must equal the first");
    // last stage: j = t, Ns = N / RL = T, outputs at t + r T
#pragma unroll
    for (int r = 0; r < RL; ++r) v[r] = sm[L::slot(t + r * (N / RL), c)];
#pragma unroll
    for (int r = 1; r < RL; ++r) v[r] = cmul(v[r], twiddle<SIGN>(tw, (t % NSL) * r * (N / (NSL * RL))));
    small_dft<RL, SIGN>(v);
    __syncthreads();  // the shared buffer may be reused right after
}

}  // namespace ns2d
