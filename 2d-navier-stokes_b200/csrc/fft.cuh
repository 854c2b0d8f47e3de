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

// Per-thread twiddle seeds.  In every plan T is a multiple of the middle
// stage's Ns, so a thread's middle-stage butterflies all share k = t mod Ns and
// its twiddles are powers of one value; the last stage's twiddles are powers of
// exp(-2 pi i t / N).  The seeds are loaded once per kernel and the powers
// w^r (r < R) are formed by a multiplication tree of depth log2 R, so the
// transform issues no table loads of its own.
template <typename C>
struct TwSeed {
    C mid;   // exp(-2 pi i (t mod Ns1) (N / (Ns1 R1)) / N)
    C last;  // exp(-2 pi i t / N)
};

template <int N, typename C>
__device__ __forceinline__ TwSeed<C> twiddle_seeds(const C* __restrict__ tw, int t) {
    using P = Plan<N>;
    TwSeed<C> s;
    constexpr int NS1 = P::R0;
    s.mid = __ldg(tw + (t % NS1) * (N / (NS1 * P::R1)));
    s.last = __ldg(tw + t);
    return s;
}

// Seeds of the N-point plan read from the table of a multiple of N points:
// tw[stride * j] = exp(-2 pi i j / N).
template <int N, typename C>
__device__ __forceinline__ TwSeed<C> twiddle_seeds_strided(const C* __restrict__ tw, int t, int stride) {
    using P = Plan<N>;
    TwSeed<C> s;
    constexpr int NS1 = P::R0;
    s.mid = __ldg(tw + stride * ((t % NS1) * (N / (NS1 * P::R1))));
    s.last = __ldg(tw + stride * t);
    return s;
}

// out[r] = w^r for r < R (out[0] unused), with conj(w) for SIGN > 0.
template <int R, int SIGN, typename C>
__device__ __forceinline__ void tw_powers(C w, C* out) {
    if constexpr (SIGN > 0) w.y = -w.y;
    out[1] = w;
#pragma unroll
    for (int r = 2; r < R; ++r) out[r] = (r & 1) ? cmul(out[r - 1], w) : cmul(out[r / 2], out[r / 2]);
}

// Middle stage: reads smem (pattern of the previous stage's writes), writes smem.
template <int N, int R, int NS, int SIGN, int TC, typename C>
__device__ __forceinline__ void middle_stage(C* sm, C wseed, int t, int c) {
    using P = Plan<N>;
    using L = SmemLayout<N, TC>;
    constexpr int BPT = N / (R * P::T);
    static_assert(BPT * R * P::T == N, "plan");
    static_assert(P::T % NS == 0, "middle-stage twiddles must depend on t only");
    C v[BPT][R];
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
        const int j = t + P::T * b;
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = sm[L::slot(j + r * (N / R), c)];
    }
    __syncthreads();
    C w[R];
    tw_powers<R, SIGN>(wseed, w);
    const int k = t % NS;
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
        const int j = t + P::T * b;
#pragma unroll
        for (int r = 1; r < R; ++r) v[b][r] = cmul(v[b][r], w[r]);
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
__device__ __forceinline__ void fft(C* v, C* sm, const TwSeed<C>& seed, int t, int c) {
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
        middle_stage<N, P::R1, NS1, SIGN, TC>(sm, seed.mid, t, c);
    }
    constexpr int RL = (P::S == 3) ? P::R2 : P::R1;
    static_assert(RL == P::R0, "last radix must equal the first");
    // last stage: j = t, Ns = N / RL = T, outputs at t + r T, twiddles w^r with
    // w = exp(SIGN 2 pi i t / N)
#pragma unroll
    for (int r = 0; r < RL; ++r) v[r] = sm[L::slot(t + r * (N / RL), c)];
    C w[RL];
    tw_powers<RL, SIGN>(seed.last, w);
#pragma unroll
    for (int r = 1; r < RL; ++r) v[r] = cmul(v[r], w[r]);
    small_dft<RL, SIGN>(v);
    __syncthreads();  // the shared buffer may be reused right after
}

}  // namespace ns2d

namespace ns2d {

// ---------------------------------------------------------------------------
// Team transforms.  A team is the T threads of one transform (Plan<N>::T),
// laid out as whole warps when T >= 32, and it owns a private shared region of
// B * ROWS elements (one per transform in flight).  Teams synchronise with
// their own named barrier, so the teams of a block advance independently.
// ---------------------------------------------------------------------------
template <int N>
struct TeamLayout {
    static constexpr int PADR = Plan<N>::R0;
    static constexpr int ROWS = N + N / PADR;
    __device__ __forceinline__ static int slot(int e) { return e + e / PADR; }
};

template <int T>
__device__ __forceinline__ void team_sync(int bar) {
    if constexpr (T >= 32) {
        asm volatile("bar.sync %0, %1;\n" ::"r"(bar), "r"(T) : "memory");
    } else {
        __syncwarp();
    }
}

// Layout/sync policies for batched transforms.
// Interleaved: the TC transforms of a block share one padded buffer per batch
// entry (c fastest), synchronised with the block barrier.
template <int N, int TC, typename C>
struct IlvPolicy {
    C* sm;
    int c;
    static constexpr int STRIDE = SmemLayout<N, TC>::ELEMS;
    __device__ __forceinline__ C& at(int b, int e) const { return sm[b * STRIDE + SmemLayout<N, TC>::slot(e, c)]; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};
// Interleaved over two buffers at arbitrary places (p0 for batch entry 0, p1
// for entry 1), synchronised with the block barrier.
template <int N, int TC, typename C>
struct IlvPairPolicy {
    C* p0;
    C* p1;
    int c;
    __device__ __forceinline__ C& at(int b, int e) const { return (b ? p1 : p0)[SmemLayout<N, TC>::slot(e, c)]; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};
// Team: private padded regions, named barrier (or warp barrier below 32 threads).
template <int N, typename C>
struct TeamPolicy {
    C* sm;
    int bar;
    static constexpr int STRIDE = TeamLayout<N>::ROWS;
    __device__ __forceinline__ C& at(int b, int e) const { return sm[b * STRIDE + TeamLayout<N>::slot(e)]; }
    __device__ __forceinline__ void sync() const { team_sync<Plan<N>::T>(bar); }
};

// B transforms of length N in lockstep.  v[b][m] = x_b[t + T m] in and out.
// The twiddle powers are shared by the B transforms; one barrier phase serves
// all of them.
template <int N, int SIGN, int B, typename C, typename Pol>
__device__ __forceinline__ void fft_batched(C (&v)[B][N / Plan<N>::T], const Pol& pol, const TwSeed<C>& seed, int t) {
    using P = Plan<N>;
    constexpr int T = P::T;
    constexpr int E = N / T;
    static_assert(E == P::R0, "first stage must be one butterfly per thread");
#pragma unroll
    for (int b = 0; b < B; ++b) {
        small_dft<P::R0, SIGN>(v[b]);
#pragma unroll
        for (int r = 0; r < P::R0; ++r) pol.at(b, t * P::R0 + r) = v[b][r];
    }
    pol.sync();
    if constexpr (P::S == 3) {
        constexpr int R = P::R1;
        constexpr int NS = P::R0;
        constexpr int BPT = N / (R * T);
        static_assert(T % NS == 0, "middle-stage twiddles must depend on t only");
#pragma unroll
        for (int b = 0; b < B; ++b)
#pragma unroll
            for (int bb = 0; bb < BPT; ++bb)
#pragma unroll
                for (int r = 0; r < R; ++r) v[b][bb * R + r] = pol.at(b, t + T * bb + r * (N / R));
        pol.sync();
        C w[R];
        tw_powers<R, SIGN>(seed.mid, w);
        const int k = t % NS;
#pragma unroll
        for (int b = 0; b < B; ++b) {
#pragma unroll
            for (int bb = 0; bb < BPT; ++bb) {
                const int j = t + T * bb;
                C* u = &v[b][bb * R];
#pragma unroll
                for (int r = 1; r < R; ++r) u[r] = cmul(u[r], w[r]);
                small_dft<R, SIGN>(u);
                const int base = (j / NS) * NS * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) pol.at(b, base + r * NS) = u[r];
            }
        }
        pol.sync();
    }
    constexpr int RL = (P::S == 3) ? P::R2 : P::R1;
    static_assert(RL == P::R0, "last radix must equal the first");
    C w[RL];
    tw_powers<RL, SIGN>(seed.last, w);
#pragma unroll
    for (int b = 0; b < B; ++b) {
#pragma unroll
        for (int r = 0; r < RL; ++r) v[b][r] = pol.at(b, t + r * T);
#pragma unroll
        for (int r = 1; r < RL; ++r) v[b][r] = cmul(v[b][r], w[r]);
        small_dft<RL, SIGN>(v[b]);
    }
    pol.sync();  // the buffers may be reused right after
}

}  // namespace ns2d
