// engine.cuh -- per-grid-size launch tables for the step kernels.
#pragma once
#include <cuda_runtime.h>

#include "aux_kernels.cuh"

namespace ns2d {

// Column-tile width (ky columns per block) and row pairs per block.  Column
// accesses fetch TC * 16 B per row, so wider tiles use each row's cache line
// better; at 512 and 1024 four columns per block measured faster than two
// (even with fewer blocks than SMs at 1024), so they get TC = 4.
template <int N>
struct Shape {
    static constexpr int T = Plan<N>::T;
    static constexpr int TC_RAW = 128 / T < 2 ? 2 : 128 / T;
    static constexpr int TC = (N == 16) ? 8 : (N == 512 || N == 1024) ? 4 : TC_RAW;
    static constexpr int PAIRS_RAW = (128 / T) / 2 < 1 ? 1 : (128 / T) / 2;
    static constexpr int PAIRS = PAIRS_RAW > N / 2 ? N / 2 : PAIRS_RAW;
};

template <typename Real, int N>
struct Launch {
    using C = typename Cx<Real>::T;
    using S = Shape<N>;
    static constexpr int SIZE = N;
    static constexpr size_t col_smem() { return ColSmem<Real, N, S::TC>::bytes(); }
    static constexpr size_t col_tma_smem() { return ColSmem<Real, N, S::TC>::bytes_tma() + 1024; }
    static constexpr size_t row_smem() { return RowSmem<Real, N, 2 * S::PAIRS>::bytes(); }
    static constexpr size_t inv_smem() { return sizeof(C) * SmemLayout<N, S::TC>::ELEMS; }
    static constexpr size_t c2r_smem() {
        size_t a = sizeof(C) * SmemLayout<N, 2 * S::PAIRS>::ELEMS;
        size_t b = sizeof(Real) * N * 2 * S::PAIRS;
        return a > b ? a : b;
    }

    static cudaError_t setup() {
        cudaError_t e = cudaSuccess;
        auto set = [&](const void* f, size_t bytes) {
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        };
        set((const void*)col_kernel<Real, N, S::TC, COL_P1>, col_smem());
        set((const void*)col_kernel<Real, N, S::TC, COL_RHS>, col_smem());
        set((const void*)col_kernel<Real, N, S::TC, COL_STAGE>, col_smem());
        set((const void*)col_kernel<Real, N, S::TC, COL_FINAL>, col_smem());
        set((const void*)col_kernel<Real, N, S::TC, COL_STAGE, true>, col_smem());
        set((const void*)col_kernel<Real, N, S::TC, COL_FINAL, true>, col_smem());
        set((const void*)col_tma_kernel<Real, N, S::TC, COL_P1>, col_tma_smem());
        set((const void*)col_tma_kernel<Real, N, S::TC, COL_STAGE>, col_tma_smem());
        set((const void*)col_tma_kernel<Real, N, S::TC, COL_FINAL>, col_tma_smem());
        set((const void*)row_kernel<Real, N, S::PAIRS>, row_smem());
        set((const void*)col_inv_kernel<Real, N, S::TC>, inv_smem());
        set((const void*)row_c2r_kernel<Real, N, S::PAIRS, R2_MAXABS>, c2r_smem());
        set((const void*)row_c2r_kernel<Real, N, S::PAIRS, R2_CFL>, c2r_smem());
        set((const void*)row_c2r_kernel<Real, N, S::PAIRS, R2_STORE>, c2r_smem());
        set((const void*)fwd_kernel<Real, N, S::TC, FWD_ROWS>, inv_smem());
        set((const void*)fwd_kernel<Real, N, S::TC, FWD_COLS>, inv_smem());
        return e;
    }

    // maps: tensor maps of the arrays the pass reads and writes (null: per-thread
    // copies); the first, stage and final passes then move their tiles by TMA.
    static void col(int mode, const ColArgs<Real>& a, cudaStream_t s, const ColMaps* maps = nullptr) {
        dim3 grid((a.nyf + S::TC - 1) / S::TC), block(S::T * S::TC);
        const bool fast = col_fast_ok(a);
        switch (mode) {
            case COL_P1:
                if (maps) col_tma_kernel<Real, N, S::TC, COL_P1><<<grid, block, col_tma_smem(), s>>>(a, *maps);
                else col_kernel<Real, N, S::TC, COL_P1><<<grid, block, col_smem(), s>>>(a);
                break;
            case COL_RHS: col_kernel<Real, N, S::TC, COL_RHS><<<grid, block, col_smem(), s>>>(a); break;
            case COL_STAGE:
                if (fast && maps) col_tma_kernel<Real, N, S::TC, COL_STAGE><<<grid, block, col_tma_smem(), s>>>(a, *maps);
                else if (fast) col_kernel<Real, N, S::TC, COL_STAGE, true><<<grid, block, col_smem(), s>>>(a);
                else col_kernel<Real, N, S::TC, COL_STAGE><<<grid, block, col_smem(), s>>>(a);
                break;
            default:
                if (fast && maps) col_tma_kernel<Real, N, S::TC, COL_FINAL><<<grid, block, col_tma_smem(), s>>>(a, *maps);
                else if (fast) col_kernel<Real, N, S::TC, COL_FINAL, true><<<grid, block, col_smem(), s>>>(a);
                else col_kernel<Real, N, S::TC, COL_FINAL><<<grid, block, col_smem(), s>>>(a);
                break;
        }
    }
    static void row(const RowArgs<Real>& a, cudaStream_t s) {
        dim3 grid(N / (2 * S::PAIRS)), block(S::T * 2 * S::PAIRS);
        row_kernel<Real, N, S::PAIRS><<<grid, block, row_smem(), s>>>(a);
    }
    static void col_inv(const InvArgs<Real>& a, cudaStream_t s) {
        dim3 grid((a.nyf + S::TC - 1) / S::TC), block(S::T * S::TC);
        col_inv_kernel<Real, N, S::TC><<<grid, block, inv_smem(), s>>>(a);
    }
    // Forward transform passes (set-up only): rows of a real [N][N] field, then columns.
    static void fwd(int pass, const double* real_in, const C* in, C* out, int nlines, int ldc, const C* tw,
                    cudaStream_t s) {
        dim3 grid((nlines + S::TC - 1) / S::TC), block(S::T * S::TC);
        if (pass == FWD_ROWS)
            fwd_kernel<Real, N, S::TC, FWD_ROWS><<<grid, block, inv_smem(), s>>>(real_in, in, out, nlines, ldc, tw);
        else
            fwd_kernel<Real, N, S::TC, FWD_COLS><<<grid, block, inv_smem(), s>>>(real_in, in, out, nlines, ldc, tw);
    }
    static void row_c2r(int op, const RowC2RArgs<Real>& a, cudaStream_t s) {
        dim3 grid(N / (2 * S::PAIRS)), block(S::T * 2 * S::PAIRS);
        switch (op) {
            case R2_MAXABS: row_c2r_kernel<Real, N, S::PAIRS, R2_MAXABS><<<grid, block, c2r_smem(), s>>>(a); break;
            case R2_CFL: row_c2r_kernel<Real, N, S::PAIRS, R2_CFL><<<grid, block, c2r_smem(), s>>>(a); break;
            default: row_c2r_kernel<Real, N, S::PAIRS, R2_STORE><<<grid, block, c2r_smem(), s>>>(a); break;
        }
    }
};

// Runtime dispatch over the supported sizes.
template <typename Real, typename F>
inline bool with_size(int n, F&& f) {
    switch (n) {
        case 16: f(Launch<Real, 16>{}); return true;
        case 32: f(Launch<Real, 32>{}); return true;
        case 64: f(Launch<Real, 64>{}); return true;
        case 128: f(Launch<Real, 128>{}); return true;
        case 256: f(Launch<Real, 256>{}); return true;
        case 512: f(Launch<Real, 512>{}); return true;
        case 1024: f(Launch<Real, 1024>{}); return true;
        case 2048: f(Launch<Real, 2048>{}); return true;
        default: return false;
    }
}

}  // namespace ns2d
