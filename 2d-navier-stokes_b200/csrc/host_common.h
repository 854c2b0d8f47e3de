// host_common.h -- host-side rules shared by the single-trajectory handle and
// the ensemble: operator-branch selection and exponent handling.
#pragma once
#include <climits>
#include <cmath>

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

}  // namespace ns2d
