// host_common.h -- host-side rules shared by the single-trajectory handle and
// the ensemble: operator-branch selection, exponent handling and the tensor
// maps of the column passes' TMA tile copies.
#pragma once
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>

#include "../../include/ns2d.h"
#include "kernels.cuh"

namespace ns2d {

inline int int_exponent(double p) {
    double r = std::nearbyint(p);
    if (r == p && std::fabs(r) <= 64.0) return (int)r;
    return INT_MIN;
}

// Branch of the linear operator for one evaluation (Solver/src/solver.c:839-856).
// With the reference's `=` typo (latch) the third test assigns the flag first.
inline int resolve_branch(int& hyper_flag, int drag, bool latch) {
    if (hyper_flag == 1 && drag == 1) return 1;
    if (hyper_flag != 1 && drag == 1) return 2;
    if (latch) hyper_flag = 1;
    if (hyper_flag == 1 && drag != 1) return 3;
    return 4;
}

inline LinOp make_lin_params(const ns2d_params& p, int branch) {
    LinOp L;
    L.nu = p.nu;
    L.alpha = p.ekmn_alpha;
    L.hp = p.hyper_visc_pow;
    L.dp = p.ekmn_drag_pow;
    L.branch = branch;
    L.hp_int = int_exponent(L.hp);
    L.dp_int = int_exponent(L.dp);
    return L;
}

inline bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Whether the column passes may move their tiles by TMA copies: yes unless the
// environment variable NS2D_DISABLE_TMA is set to a value other than "0" when
// a handle or ensemble is created (the per-thread copies give the same
// results to rounding; the switch exists to compare the two and as a fallback).
inline bool tma_copies_enabled() {
    const char* v = std::getenv("NS2D_DISABLE_TMA");
    return !(v && v[0] && !(v[0] == '0' && v[1] == 0));
}

// The driver's tensor-map encoder, through the runtime (no libcuda link).
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The ColMaps of one field set, bases = {f0, f1, f2, f3, acc, state, nl}, each
// nx rows of ldc complex (nyf used) with column tiles of tc columns: boxes of
// (2 tc reals, min(nx, 256) rows).  False when the encoder is missing or
// rejects a map.
template <typename Real>
inline bool encode_col_maps(ColMaps* m, void* const bases[7], int nx, int nyf, int ldc, int tc) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || tc <= 0) return false;
    const cuuint64_t gdim[2] = {(cuuint64_t)2 * nyf, (cuuint64_t)nx};
    const cuuint64_t gstride[1] = {(cuuint64_t)ldc * 2 * sizeof(Real)};
    const cuuint32_t box[2] = {(cuuint32_t)(2 * tc), (cuuint32_t)std::min(nx, 256)};
    const cuuint32_t estride[2] = {1, 1};
    const CUtensorMapDataType dt = sizeof(Real) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUtensorMap* maps[7] = {&m->f[0], &m->f[1], &m->f[2], &m->f[3], &m->acc, &m->state, &m->nl};
    for (int k = 0; k < 7; ++k) {
        if (enc(maps[k], dt, 2, bases[k], gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

}  // namespace ns2d
