// noalloc.cu -- ns2d_nonlinear_rhs_noalloc: the nonlinear-term evaluation of
// include/ns2d.h for callers that cannot allocate device memory.
//
// Who needs it: code that runs inside CUDA stream capture owned by another
// framework (cudaMalloc cannot be recorded into a graph), latency-critical time
// loops where cudaMalloc's implicit device synchronisation is not acceptable,
// and host applications whose device memory is handed out by their own pool
// allocator and must not grow behind its back.  They bring their own input and
// output buffers; the intermediate fields live in one file-scope device array.
//
// The scratch array below is part of the library image: every GPU that loads
// libns2d.so holds NS2D_NOALLOC_SCRATCH_BYTES of it until the process exits.
// All calls on a device share it and it keeps the previous call's contents;
// two calls that overlap on the GPU (different streams, no ordering) race.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/ns2d.h"
#include "engine.cuh"

using namespace ns2d;

namespace {

// Four x-space fields, the product spectrum and the twiddle table of the
// largest supported grid, in the [N][N/2+1] layout of the caller's arrays.
constexpr size_t kMaxN = NS2D_NOALLOC_MAX_N;
constexpr size_t kMaxNyf = kMaxN / 2 + 1;
constexpr size_t kFieldElems = kMaxN * kMaxNyf;
constexpr size_t kScratchBytes = sizeof(double2) * (5 * kFieldElems + kMaxN);
static_assert(kScratchBytes == NS2D_NOALLOC_SCRATCH_BYTES, "header and scratch size disagree");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};
bool g_size_ready[kMaxDevices][5] = {};  // N = 16, 32, 64, 128, 256

// Dispatch over the sizes this entry point supports (16..256).
template <typename F>
bool with_small_size(int n, F&& f) {
    switch (n) {
        case 16: f(Launch<double, 16>{}); return true;
        case 32: f(Launch<double, 32>{}); return true;
        case 64: f(Launch<double, 64>{}); return true;
        case 128: f(Launch<double, 128>{}); return true;
        case 256: f(Launch<double, 256>{}); return true;
        default: return false;
    }
}

int size_slot(int n) {
    switch (n) {
        case 16: return 0;
        case 32: return 1;
        case 64: return 2;
        case 128: return 3;
        case 256: return 4;
        default: return -1;
    }
}

// exp(-2 pi i m / N): the same table the handle path builds on the host, here
// written on the device so that the call needs no host buffer.
__global__ void noalloc_twiddles(double2* tw, int n) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double s, c;
    sincospi(2.0 * (double)m / (double)n, &s, &c);
    tw[m] = make_double2(c, -s);
}

// Set-up on the current device (first call per device, and per grid size):
// the device address of the scratch array and the kernels' shared-memory limits.
ns2d_status setup(int dev, int n, double2** base) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (dev < 0 || dev >= kMaxDevices) return NS2D_ERR_UNSUPPORTED;
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return NS2D_ERR_CUDA;
        g_scratch_ptr[dev] = p;
    }
    const int slot = size_slot(n);
    if (slot < 0) return NS2D_ERR_UNSUPPORTED;
    if (!g_size_ready[dev][slot]) {
        cudaError_t e = cudaSuccess;
        with_small_size(n, [&](auto L) { e = decltype(L)::setup(); });
        if (e != cudaSuccess) return NS2D_ERR_CUDA;
        g_size_ready[dev][slot] = true;
    }
    *base = (double2*)g_scratch_ptr[dev];
    return NS2D_OK;
}

}  // namespace

extern "C" ns2d_status ns2d_nonlinear_rhs_noalloc(const ns2d_params* p, const double* d_w_hat, double* d_rhs,
                                                  void* cuda_stream) {
    if (!p || !d_w_hat || !d_rhs) return NS2D_ERR_INVALID;
    // The kernels move the arrays in 16-byte units (cp.async and double2
    // stores): an array that starts off that boundary, a float64 view offset
    // by one element for instance, would raise a misaligned-address error,
    // which poisons the caller's whole CUDA context.  Refuse it instead.
    if (((uintptr_t)d_w_hat | (uintptr_t)d_rhs) & 15u) return NS2D_ERR_INVALID;
    const int n = p->nx;
    if (p->nx != p->ny || size_slot(n) < 0 || (size_t)n > kMaxN) return NS2D_ERR_UNSUPPORTED;
    // the parameter checks of ns2d_create that bear on the nonlinear term
    if (p->precision != NS2D_FP64 || p->dealias < 0 || p->dealias > 1 || p->dealias_edge < 0 ||
        p->dealias_edge > 1 || p->forcing < 0 || p->forcing > 2 || p->integrator < 0 || p->integrator > 3 ||
        p->model < 0 || p->model > 1)
        return NS2D_ERR_INVALID;
    const int nyf = n / 2 + 1;
    if (p->forcing == NS2D_FORCING_KOLM && (p->force_k < 0 || p->force_k / nyf >= n)) return NS2D_ERR_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NS2D_ERR_NO_DEVICE;
    // the work runs on the current device, which p->device must name
    if (p->device != dev) return NS2D_ERR_INVALID;
    // an error left by the caller's own earlier launches stays the caller's:
    // report it without clearing it, and launch nothing
    if (cudaPeekAtLastError() != cudaSuccess) return NS2D_ERR_CUDA;
    double2* base = nullptr;
    ns2d_status s = setup(dev, n, &base);
    if (s != NS2D_OK) return s;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const size_t fe = (size_t)n * nyf;
    double2* f[4] = {base, base + fe, base + 2 * fe, base + 3 * fe};
    double2* nl = base + 4 * fe;
    double2* tw = base + 5 * kFieldElems;

    noalloc_twiddles<<<(n + 127) / 128, 128, 0, st>>>(tw, n);

    ColArgs<double> a;
    std::memset(&a, 0, sizeof(a));
    a.src = (const double2*)d_w_hat;
    a.f0 = f[0];
    a.f1 = f[1];
    a.f2 = f[2];
    a.f3 = f[3];
    a.tw = tw;
    a.ldc = nyf;
    a.nyf = nyf;
    const int m = (int)(n / 3.0);
    a.kmax_sqr = m * m + (p->dealias_edge ? 1 : 0);
    a.dealias = p->dealias;
    a.houli_int = (p->quirks & NS2D_QUIRK_HOU_LI_INT) ? 1 : 0;
    a.kolm = (p->forcing == NS2D_FORCING_KOLM) ? 1 : 0;
    if (p->forcing == NS2D_FORCING_KOLM) {
        // the value ComputeForcing sets for KOLM (force.c:537), at flat index force_k
        a.has_force = 1;
        a.force_i = p->force_k / nyf;
        a.force_j = p->force_k % nyf;
        a.force_val = make_double2(-0.5 * p->force_scale * (double)p->force_k, 0.0);
    }
    a.norm2 = std::pow(1.0 / (double)(n * n), 2.0);
    with_small_size(n, [&](auto L) { decltype(L)::col(COL_P1, a, st); });

    RowArgs<double> r{};
    r.f0 = f[0];
    r.f1 = f[1];
    r.f2 = f[2];
    r.f3 = f[3];
    r.nl = nl;
    r.tw = tw;
    r.ldc = nyf;
    r.nrows = n;
    r.status = nullptr;
    with_small_size(n, [&](auto L) { decltype(L)::row(r, st); });

    a.src = nl;
    a.rhs_store = (double2*)d_rhs;  // no state here: the conjugacy side effect is not applied
    a.conj_mode = 0;
    with_small_size(n, [&](auto L) { decltype(L)::col(COL_RHS, a, st); });
    // no error was pending on entry, so one found now is a launch of this call
    if (cudaGetLastError() != cudaSuccess) return NS2D_ERR_CUDA;
    return NS2D_OK;
}
