// wfft.cuh -- warp-synchronous 1024-point FFT: one warp per transform, two
// radix-32 stages in registers, one transpose through shared memory.
//
// Written from the DFT definition with the Cooley-Tukey split N = 32 * 32,
// n = t + 32 m (lane t holds x[t + 32 m], m < 32), k = k1 + 32 k2:
//
//   X[k1 + 32 k2] = sum_t W32^(t k2) [ W^(t k1) sum_m x[t + 32 m] W32^(m k1) ],
//
// with W = exp(SIGN 2 pi i / N).  Lane t first does the 32-point DFT over m
// (giving index k1), multiplies by the twiddles W^(t k1), and writes row k1 of
// a 32 x 33 shared-memory tile; after a warp barrier lane k1 reads its row and
// does the 32-point DFT over t (giving k2).  The output pattern equals the
// input pattern -- lane t holds X[t + 32 k2] -- so a transform can feed an
// elementwise epilogue or a transform of the other sign with no exchange.
//
// Against the block-wide three-stage transforms of fft.cuh this halves the
// shared-memory traffic (one transpose instead of two) and needs no barrier
// wider than the warp, so warps of a block proceed independently.
#pragma once
#include "fft.cuh"

namespace ns2d {

// exp(SIGN 2 pi i K / 32) applied to a, for the in-register 32-point DFT.
// K = 8 q + r: base angle r pi / 16 (r < 8), rotated by q quarter turns.
template <int K, int SIGN, typename C>
__device__ __forceinline__ C ctw32(C a) {
    using Real = decltype(C::x);
    constexpr int k = ((K % 32) + 32) % 32;
    if constexpr (k % 2 == 0) {
        return ctw<16, k / 2, SIGN>(a);
    } else {
        // cos / sin of r pi / 16 for odd r
        constexpr int r = k % 8;
        constexpr Real c1 = (Real)0.98078528040323044913;  // cos(pi/16)
        constexpr Real s1 = (Real)0.19509032201612826785;  // sin(pi/16)
        constexpr Real c3 = (Real)0.83146961230254523708;  // cos(3pi/16)
        constexpr Real s3 = (Real)0.55557023301960222474;  // sin(3pi/16)
        constexpr Real cr = (r == 1) ? c1 : (r == 3) ? c3 : (r == 5) ? s3 : s1;
        constexpr Real sr = (r == 1) ? s1 : (r == 3) ? s3 : (r == 5) ? c3 : c1;
        C b = cmake<C>(a.x * cr - a.y * (SIGN * sr), a.x * (SIGN * sr) + a.y * cr);
        constexpr int quad = k / 8;
        if constexpr (quad == 0) return b;
        else if constexpr (quad == 1) return cmul_i<SIGN>(b);
        else if constexpr (quad == 2) return cmake<C>(-b.x, -b.y);
        else return cmul_i<-SIGN>(b);
    }
}

// In-register 32-point DFT on v[0..31] (natural order in and out): radix-2
// decimation in time, the two 16-point halves by SmallDFT.
template <int SIGN, typename C>
__device__ __forceinline__ void dft32(C* v) {
    SmallDFT<16, SIGN, 2, C>::run(v);      // even samples -> v[0], v[2], ...
    SmallDFT<16, SIGN, 2, C>::run(v + 1);  // odd samples  -> v[1], v[3], ...
    C tmp[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) tmp[k] = v[k];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const C e = tmp[2 * k];
        C o = tmp[2 * k + 1];
        switch (k) {
#define NS2D_W32(KK) case KK: o = ctw32<KK, SIGN>(o); break;
            NS2D_W32(0) NS2D_W32(1) NS2D_W32(2) NS2D_W32(3) NS2D_W32(4) NS2D_W32(5) NS2D_W32(6) NS2D_W32(7)
            NS2D_W32(8) NS2D_W32(9) NS2D_W32(10) NS2D_W32(11) NS2D_W32(12) NS2D_W32(13) NS2D_W32(14) NS2D_W32(15)
#undef NS2D_W32
        }
        v[k] = cadd(e, o);
        v[k + 16] = csub(e, o);
    }
}

// Shared-memory tile of one warp's transpose: 32 rows of 33 complex.
template <typename C>
struct WfftTile {
    static constexpr int ROW = 33;
    static constexpr int ELEMS = 32 * ROW;
    static constexpr size_t bytes() { return sizeof(C) * (size_t)ELEMS; }
};

// One 1024-point transform by the calling warp: v[m] = x[lane + 32 m] in and
// X[lane + 32 m] out.  tile: this warp's WfftTile (ELEMS complex).  w1 =
// exp(-2 pi i lane / 1024) (conjugated here for SIGN > 0).  The warp must be
// converged; the tile may be reused as soon as this returns.
template <int SIGN, typename C>
__device__ __forceinline__ void wfft1024(C (&v)[32], C* tile, C w1, int lane) {
    dft32<SIGN>(v);
    // twiddles W^(lane k1): four chains k1 = j + 4 s (j < 4) stepped by W^(4 lane)
    if constexpr (SIGN > 0) w1.y = -w1.y;
    const C w2 = cmul(w1, w1);
    const C w3 = cmul(w2, w1);
    const C w4 = cmul(w2, w2);
    C p[4] = {cmake<C>(1, 0), w1, w2, w3};
#pragma unroll
    for (int s = 0; s < 8; ++s) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k1 = 4 * s + j;
            if (k1 > 0) v[k1] = cmul(v[k1], p[j]);
            if (s < 7) p[j] = (s == 0 && j == 0) ? w4 : cmul(p[j], w4);
        }
    }
    // transpose: row k1 of the tile holds Y[k1][t] for t < 32
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) tile[k1 * WfftTile<C>::ROW + lane] = v[k1];
    __syncwarp();
#pragma unroll
    for (int n2 = 0; n2 < 32; ++n2) v[n2] = tile[lane * WfftTile<C>::ROW + n2];
    __syncwarp();
    dft32<SIGN>(v);
}

}  // namespace ns2d
