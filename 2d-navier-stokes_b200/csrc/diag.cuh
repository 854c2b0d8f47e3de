// diag.cuh -- ComputeSystemMeasurables (Solver/src/sys_msr.c:32-373) as one
// pass over the half spectrum: 13 totals reduced in FP64 (per-thread sums,
// warp and block trees, one atomic per block and total) and 8 spectra binned
// by round(|k|) in shared memory.  Raw sums are scaled on the host by the
// reference's constants (4 pi^2 and 0.5/(Nx Ny)^2).
#pragma once
#include "kernels.cuh"

namespace ns2d {

enum { DG_E = 0, DG_Z, DG_P, DG_FORC, DG_DIV, DG_EDISS, DG_ZDISS, DG_DE, DG_EFLUX, DG_EDSB, DG_DZ, DG_ZFLUX, DG_ZDSB, DG_N };

template <typename Real>
struct DiagArgs {
    using C = typename Cx<Real>::T;
    const C* state;
    const C* rhs;    // RHS of the state minus forcing (flux terms), may be null
    int ldc, nx, ny, nyf;
    LinOp lin;       // pre_fac branch (sys_msr.c:166-181)
    int enst_quirk;  // weight-2 enstrophy dissipation without pre_fac (sys_msr.c:225)
    int force_i, force_j;
    double fre, fim;
    int has_force;
    const C* ffield;  // forcing of listed modes ([nx][ldc]), may be null
    int n_spect;
    double* out;     // [DG_N] raw totals, then 8 * n_spect raw spectra (zeroed by the host)
};

template <typename Real>
__global__ void __launch_bounds__(256) diag_kernel(DiagArgs<Real> a) {
    using C = typename Cx<Real>::T;
    extern __shared__ double dsm[];  // 8 * n_spect spectra + DG_N * 8 warp partials
    const int ns = a.n_spect;
    double* hist = dsm;
    double* wpart = dsm + 8 * ns;
    for (int q = threadIdx.x; q < 8 * ns; q += blockDim.x) hist[q] = 0.0;
    __syncthreads();
    double acc[DG_N];
#pragma unroll
    for (int k = 0; k < DG_N; ++k) acc[k] = 0.0;
    const long long n = (long long)a.nx * a.nyf;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / a.nyf), j = (int)(q % a.nyf);
        const int kx = (i <= a.nx / 2) ? i : i - a.nx;
        const int ky = j;
        if (kx == 0 && ky == 0) continue;
        const C wc = a.state[(size_t)i * a.ldc + j];
        const double wr = (double)wc.x, wi = (double)wc.y;
        const double k_sqr = (double)(kx * kx + ky * ky);
        const double pre_fac = lin_bracket(a.lin, k_sqr);
        const double w2 = wr * wr + wi * wi;
        // u_z = i ky w / k^2, v_z = -i kx w / k^2, div = i (kx u_z + ky v_z)
        const double ur = -((double)ky * wi) / k_sqr, ui = ((double)ky * wr) / k_sqr;
        const double vr = ((double)kx * wi) / k_sqr, vi = -((double)kx * wr) / k_sqr;
        const double dre = (double)kx * ur + (double)ky * vr, dim = (double)kx * ui + (double)ky * vi;
        const double div2 = dre * dre + dim * dim;
        const double uv2 = ur * ur + ui * ui + vr * vr + vi * vi;
        double deriv = 0.0;
        if (a.rhs) {
            C r = a.rhs[(size_t)i * a.ldc + j];
            // the flux terms ignore forcing (sys_msr.c:127-132)
            if (a.has_force && i == a.force_i && j == a.force_j) {
                r.x = (Real)((double)r.x - a.fre);
                r.y = (Real)((double)r.y - a.fim);
            }
            if (a.ffield) {
                const C f = a.ffield[(size_t)i * a.ldc + j];
                r.x = (Real)((double)r.x - (double)f.x);
                r.y = (Real)((double)r.y - (double)f.y);
            }
            // creal(w conj(r) + conj(w) r) = 2 Re(w conj r)
            deriv = (wr * (double)r.x + wi * (double)r.y) + ((double)r.x * wr + (double)r.y * wi);
        }
        const double diss = pre_fac * w2;
        const double wgt = (j == 0 || j == a.nyf - 1) ? 1.0 : 2.0;
        acc[DG_E] += wgt * w2 * (1.0 / k_sqr);
        acc[DG_Z] += wgt * w2;
        acc[DG_DIV] += wgt * div2;
        acc[DG_P] += wgt * k_sqr * w2;
        acc[DG_EDISS] += wgt * pre_fac * uv2;
        acc[DG_ZDISS] += (wgt == 2.0 && a.enst_quirk) ? 2.0 * w2 : wgt * diss;
        if (k_sqr >= 0.0 && k_sqr < 4096.0) {
            acc[DG_DE] += (deriv + diss) * (wgt / k_sqr);
            acc[DG_EDSB] += diss * (wgt / k_sqr);
            acc[DG_EFLUX] += deriv * (wgt / k_sqr);
            acc[DG_DZ] += wgt * (deriv + diss);
            acc[DG_ZDSB] += wgt * diss;
            acc[DG_ZFLUX] += wgt * deriv;
        }
        if (a.has_force && i == a.force_i && j == a.force_j) {
            // cabs(forcing * w_hat[forced])  (sys_msr.c:135-139)
            const double pr = a.fre * wr - a.fim * wi, pi = a.fre * wi + a.fim * wr;
            acc[DG_FORC] += sqrt(pr * pr + pi * pi);
        }
        if (a.ffield) {
            const C f = a.ffield[(size_t)i * a.ldc + j];
            const double fr = (double)f.x, fi = (double)f.y;
            const double pr = fr * wr - fi * wi, pi = fr * wi + fi * wr;
            acc[DG_FORC] += sqrt(pr * pr + pi * pi);
        }
        const int b = (int)round(sqrt(k_sqr));
        if (b < ns) {
            atomicAdd(&hist[0 * ns + b], wgt * w2 * (1.0 / k_sqr));  // enrg
            atomicAdd(&hist[1 * ns + b], wgt * w2);                  // enst
            atomicAdd(&hist[2 * ns + b], wgt * (deriv + diss));      // d_enst_dt
            atomicAdd(&hist[3 * ns + b], wgt * deriv);               // enst_flux
            atomicAdd(&hist[4 * ns + b], wgt * diss);                // enst_diss
            atomicAdd(&hist[5 * ns + b], wgt * (deriv + diss) / k_sqr);  // d_enrg_dt
            atomicAdd(&hist[6 * ns + b], wgt * deriv / k_sqr);       // enrg_flux
            atomicAdd(&hist[7 * ns + b], wgt * diss / k_sqr);        // enrg_diss
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < DG_N; ++k) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) wpart[k * 8 + warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < DG_N) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += wpart[threadIdx.x * 8 + w];
        atomicAdd(&a.out[threadIdx.x], v);
    }
    for (int q = threadIdx.x; q < 8 * ns; q += blockDim.x)
        if (hist[q] != 0.0) atomicAdd(&a.out[DG_N + q], hist[q]);
}

}  // namespace ns2d
