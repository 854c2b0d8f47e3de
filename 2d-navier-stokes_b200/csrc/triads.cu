// Sector triad sums of the post-processing program's phase synchronisation
// (PostProcessing/src/phase_sync.c): the triad search of AllocatePhaseSyncMemory
// (phase_sync.c:1744-1948) and the per-snapshot accumulation of PhaseSyncSector
// (phase_sync.c:281-1058), fused: each block takes one (k3 sector, k1 sector,
// flux term, flux_pre_fac sign) class, walks the k3 candidates in order, and
// its threads test and accumulate the k1 candidates of each selected k3.  No
// triad list is stored; the block's sums are reduced in a fixed order.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/ns2d.h"

namespace {

constexpr int kThreads = 256;
constexpr int kSub = 4;  // (contribution 1d/2d) x (unidirectional no/yes)
constexpr int kVals = NS2D_TRIAD_VALUES;

struct TriadArgs {
    int kmax, n_k1;
    double kmax_sqr, kmax_c_sqr;
    const double *k3_lwr, *k3_upr, *k1_lwr, *k1_upr;
    const double *ang, *ang_neg, *amps, *phases;
    double* sums;
    int use_list;  // compact the block's k1 candidates into shared memory first
};

// ((angle in [lo, hi)) or (angle of -k in [lo, hi))), as the search tests a sector
__device__ __forceinline__ bool in_sector(double ang, double ang_neg, double lo, double hi) {
    return (ang >= lo && ang < hi) || (ang_neg >= lo && ang_neg < hi);
}

// carg of a real number: atan2(+0, x)
__device__ __forceinline__ double carg_real(double x) { return signbit(x) ? M_PI : 0.0; }

// generalised triad phase fmod(phase + 2 pi + carg(w), 2 pi) - pi (phase_sync.c:375)
__device__ __forceinline__ double gen_phase(double tp, double w) {
    return fmod(tp + 2.0 * M_PI + carg_real(w), 2.0 * M_PI) - M_PI;
}

__global__ void __launch_bounds__(kThreads) triad_sector_kernel(TriadArgs g) {
    const int al = blockIdx.x;               // a * n_k1 + l (k1 sector as stored)
    const int a = al / g.n_k1;
    const int term = blockIdx.y / 3;         // 0: positive flux term, 1: negative
    const int cls = blockIdx.y % 3;          // flux_pre_fac < 0, > 0, == 0
    const double lo3 = g.k3_lwr[a], hi3 = g.k3_upr[a];
    const double lo1 = g.k1_lwr[al], hi1 = g.k1_upr[al];
    const double km = g.kmax_sqr, kc = g.kmax_c_sqr;
    const int side = 2 * g.kmax + 1;
    const int m = side * side;
    const double sgn = term == 0 ? 1.0 : -1.0;

    double acc[kSub][kVals];
#pragma unroll
    for (int s = 0; s < kSub; ++s)
#pragma unroll
        for (int v = 0; v < kVals; ++v) acc[s][v] = 0.0;

    // k1 candidates of this block's sectors and term, compacted in order into
    // shared memory (index | 1d flag << 30): the k1-only tests of the search
    // run once per block instead of once per selected k3
    extern __shared__ int k1_list[];
    __shared__ int warp_count[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int n1 = m;
    if (g.use_list) {
        n1 = 0;
        for (int base = 0; base < m; base += kThreads) {
            const int i1 = base + (int)threadIdx.x;
            int code = -1;
            if (i1 < m) {
                const int k1x = g.kmax - i1 / side, k1y = i1 % side - g.kmax;
                const double k1s = (double)(k1x * k1x + k1y * k1y);
                const double a1 = g.ang[i1], n1a = g.ang_neg[i1];
                const bool s13 = in_sector(a1, n1a, lo3, hi3), s11 = in_sector(a1, n1a, lo1, hi1);
                if (term == 0) {
                    const bool c1d = (k1s > 0.0 && k1s <= kc) && s13 && s11;
                    const bool c2d = (k1s > 0.0 && k1s <= km) && s11 && !s13;
                    if (c1d || c2d) code = i1 | (c1d ? (1 << 30) : 0);
                } else if ((k1s > kc && k1s <= km) && s13) {
                    code = i1;
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, code >= 0);
            if (lane == 0) warp_count[warp] = __popc(bal);
            __syncthreads();
            int off = n1, tot = 0;
            for (int w = 0; w < kThreads / 32; ++w) {
                if (w < warp) off += warp_count[w];
                tot += warp_count[w];
            }
            if (code >= 0) k1_list[off + __popc(bal & ((1u << lane) - 1u))] = code;
            __syncthreads();
            n1 += tot;
        }
    }

    for (int i3 = 0; i3 < m; ++i3) {
        // table index (kmax - kx) * side + kmax + ky (the full-field layout)
        const int k3x = g.kmax - i3 / side, k3y = i3 % side - g.kmax;
        const double k3s = (double)(k3x * k3x + k3y * k3y);
        const double a3 = g.ang[i3], n3 = g.ang_neg[i3];
        const bool s33 = in_sector(a3, n3, lo3, hi3), s31 = in_sector(a3, n3, lo1, hi1);
        // k3 branches of the search (phase_sync.c:1798-1800, 1863-1869)
        const bool pos = (k3s > kc && k3s <= km) && s33;
        const bool neg_1d = (k3s > 0.0 && k3s <= kc) && s33 && s31;
        const bool neg_2d = (k3s > 0.0 && k3s <= km) && s31 && !s33;
        const bool neg = !pos && (neg_2d || neg_1d);
        if (term == 0 ? !pos : !neg) continue;
        const double amp3 = g.amps[i3], ph3 = g.phases[i3];
        for (int j = threadIdx.x; j < n1; j += kThreads) {
            int i1, contrib;
            if (g.use_list) {
                const int code = k1_list[j];
                i1 = code & ((1 << 30) - 1);
                contrib = term == 0 ? ((code >> 30) ? 0 : 1) : (neg_1d ? 0 : 1);
            } else {
                i1 = j;
                const int kx = g.kmax - i1 / side, ky = i1 % side - g.kmax;
                const double ks = (double)(kx * kx + ky * ky);
                const double a1 = g.ang[i1], n1a = g.ang_neg[i1];
                const bool s13 = in_sector(a1, n1a, lo3, hi3), s11 = in_sector(a1, n1a, lo1, hi1);
                if (term == 0) {
                    const bool c1d = (ks > 0.0 && ks <= kc) && s13 && s11;
                    const bool c2d = (ks > 0.0 && ks <= km) && s11 && !s13;
                    if (!(c1d || c2d)) continue;
                    contrib = c1d ? 0 : 1;
                } else {
                    if (!((ks > kc && ks <= km) && s13)) continue;
                    contrib = neg_1d ? 0 : 1;
                }
            }
            const int k1x = g.kmax - i1 / side, k1y = i1 % side - g.kmax;
            const double k1s = (double)(k1x * k1x + k1y * k1y);
            const int k2x = k3x - k1x, k2y = k3y - k1y;
            const double k2s = (double)(k2x * k2x + k2y * k2y);
            if (term == 0) {
                if (!(k2s > 0.0 && k2s <= km)) continue;
            } else {
                if (!(k2s > kc && k2s <= km)) continue;
            }
            // |k2|^2 <= kmax^2 keeps k2 inside the tables
            const int i2 = (g.kmax - k2x) * side + g.kmax + k2y;
            const bool s23 = in_sector(g.ang[i2], g.ang_neg[i2], lo3, hi3);
            if (term == 0 ? ((k2s > kc && k2s <= km) && s23) : !s23) continue;
            // PhaseSyncSector (phase_sync.c:353-375)
            const double pre = (double)(k1x * k2y - k2x * k1y) * (1.0 / k1s - 1.0 / k2s);
            const int c = pre < 0.0 ? 0 : (pre > 0.0 ? 1 : 2);
            if (c != cls) continue;
            const double w = pre * (g.amps[i1] * g.amps[i2] * amp3);
            const double tp = g.phases[i1] + g.phases[i2] - ph3;
            double sn, cs;
            sincos(tp, &sn, &cs);
            const double ft = w * cs;
            const double cr = w * cs, ci = w * sn;
            const double g0 = gen_phase(tp, sgn * w);
            // the zero-prefactor type takes carg(flux_wght) in both terms (:917, :1261)
            const double gt = cls == 2 ? gen_phase(tp, w) : g0;
            double s0, c0, st, ct;
            sincos(g0, &s0, &c0);
            sincos(gt, &st, &ct);
            const bool coll = (cr != 0.0 || ci != 0.0);
            const bool unidir = term == 0 ? (k3y >= 0) : (k1y >= 0 && k2y >= 0);
            const int sub = contrib * 2 + (unidir ? 1 : 0);
#pragma unroll
            for (int s = 0; s < kSub; ++s) {
                if (s != sub) continue;
                acc[s][0] += 1.0;
                acc[s][1] += sgn * ft;
                acc[s][2] += c0;
                acc[s][3] += s0;
                acc[s][4] += ct;
                acc[s][5] += st;
                if (coll) {
                    acc[s][6] += sgn * cr;
                    acc[s][7] += sgn * ci;
                }
            }
        }
    }

    // block sums in a fixed order: warps by shuffle, then the warps in turn
    __shared__ double part[kThreads / 32][kSub * kVals];
#pragma unroll
    for (int s = 0; s < kSub; ++s)
#pragma unroll
        for (int v = 0; v < kVals; ++v) {
            double x = acc[s][v];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) part[warp][s * kVals + v] = x;
        }
    __syncthreads();
    if (threadIdx.x < kSub * kVals) {
        double x = 0.0;
        for (int wi = 0; wi < kThreads / 32; ++wi) x += part[wi][threadIdx.x];
        g.sums[((size_t)al * 6 + blockIdx.y) * kSub * kVals + threadIdx.x] = x;
    }
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

// Restores the calling thread's current device on return.
struct DeviceScope {
    int prev = -1;
    DeviceScope() { cudaGetDevice(&prev); }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" ns2d_status ns2d_triad_sector_sums(int32_t device, const ns2d_triad_sectors* g, const double* amps,
                                              const double* phases, double* sums) {
    if (!g || !amps || !phases || !sums || g->kmax < 1 || g->kmax > 1024 || g->n_k3 < 1 || g->n_k1 < 1 ||
        !g->k3_lwr || !g->k3_upr || !g->k1_lwr || !g->k1_upr || !g->angle || !g->angle_neg)
        return NS2D_ERR_INVALID;
    // the table lookups of k2 rely on |k|^2 <= kmax^2 keeping both components in range
    if (!(g->kmax_sqr <= (double)g->kmax * (double)g->kmax)) return NS2D_ERR_INVALID;
    if ((long long)g->n_k3 * g->n_k1 > 65535) return NS2D_ERR_UNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return NS2D_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return NS2D_ERR_INVALID;
    DeviceScope scope;
    if (cudaSetDevice(device) != cudaSuccess) return NS2D_ERR_INVALID;
    DevBuf buf;  // released before the device is restored
    const size_t side = 2 * (size_t)g->kmax + 1, m = side * side;
    const size_t nal = (size_t)g->n_k3 * g->n_k1;
    const size_t nsum = nal * 6 * kSub * kVals;
    // one buffer: tables (4 m), sector bounds (2 n_k3 + 2 nal), sums
    const size_t ndbl = 4 * m + 2 * (size_t)g->n_k3 + 2 * nal + nsum;
    if (cudaMalloc(&buf.p, sizeof(double) * ndbl) != cudaSuccess) return NS2D_ERR_NOMEM;
    double* d = (double*)buf.p;
    std::vector<double> host(ndbl - nsum);
    double* h = host.data();
    std::memcpy(h, g->angle, sizeof(double) * m);
    std::memcpy(h + m, g->angle_neg, sizeof(double) * m);
    std::memcpy(h + 2 * m, amps, sizeof(double) * m);
    std::memcpy(h + 3 * m, phases, sizeof(double) * m);
    double* hb = h + 4 * m;
    std::memcpy(hb, g->k3_lwr, sizeof(double) * g->n_k3);
    std::memcpy(hb + g->n_k3, g->k3_upr, sizeof(double) * g->n_k3);
    std::memcpy(hb + 2 * g->n_k3, g->k1_lwr, sizeof(double) * nal);
    std::memcpy(hb + 2 * g->n_k3 + nal, g->k1_upr, sizeof(double) * nal);
    if (cudaMemcpy(d, h, sizeof(double) * host.size(), cudaMemcpyHostToDevice) != cudaSuccess) return NS2D_ERR_CUDA;
    TriadArgs args;
    args.kmax = g->kmax;
    args.n_k1 = g->n_k1;
    args.kmax_sqr = g->kmax_sqr;
    args.kmax_c_sqr = g->kmax_c_sqr;
    args.ang = d;
    args.ang_neg = d + m;
    args.amps = d + 2 * m;
    args.phases = d + 3 * m;
    const double* db = d + 4 * m;
    args.k3_lwr = db;
    args.k3_upr = db + g->n_k3;
    args.k1_lwr = db + 2 * g->n_k3;
    args.k1_upr = db + 2 * g->n_k3 + nal;
    args.sums = d + (ndbl - nsum);
    // the compacted k1 list in shared memory (up to kmax = 112)
    const size_t list_bytes = sizeof(int) * m;
    args.use_list = list_bytes <= 200 * 1024 ? 1 : 0;
    const size_t smem = args.use_list ? list_bytes : 0;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(triad_sector_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return NS2D_ERR_CUDA;
    triad_sector_kernel<<<dim3((unsigned)nal, 6), kThreads, smem>>>(args);
    if (cudaGetLastError() != cudaSuccess) return NS2D_ERR_CUDA;
    if (cudaMemcpy(sums, args.sums, sizeof(double) * nsum, cudaMemcpyDeviceToHost) != cudaSuccess) return NS2D_ERR_CUDA;
    return NS2D_OK;
}
