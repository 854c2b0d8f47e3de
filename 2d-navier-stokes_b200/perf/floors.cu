// floors.cu -- measured lower bounds for the passes of the 1024^2 FP64 step.
//
// The roofline of a pass is usually quoted against the HBM bandwidth of a
// long copy.  A pass of the step moves only 40-70 MB in one launch of about
// 10-30 us, which no kernel streams at the long-copy rate.  This program
// measures, on the device it runs on:
//
//   1. a coalesced streaming kernel that moves exactly the bytes of each pass
//      class (reads R and writes W half spectra of 16 * 1024 * 513 B), with L2
//      warm (data left by the previous launch, as inside a step) and after a
//      256 MiB write that evicts it (as at the start of a step);
//   2. the compute throughput of the FFT engine (fft.cuh) on 1024-point FP64
//      transforms held in registers: eight transforms per load and store; and
//      the same for the warp-per-transform engine (wfft.cuh: two radix-32
//      stages, one shared-memory transpose), the alternative it was measured
//      against.
//
// Build and run:  make -C 2d-navier-stokes_b200 floors && 2d-navier-stokes_b200/bin/ns2d_floors
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../csrc/fft.cuh"
#include "../csrc/wfft.cuh"

using namespace ns2d;

#define FCK(x)                                                                      \
    do {                                                                            \
        cudaError_t e_ = (x);                                                       \
        if (e_ != cudaSuccess) {                                                    \
            std::fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            std::exit(1);                                                           \
        }                                                                           \
    } while (0)

namespace {

constexpr int kN = 1024;
constexpr int kNyf = kN / 2 + 1;
constexpr size_t kElems = (size_t)kN * kNyf;  // one half spectrum, complex

// Reads NR arrays and writes NW arrays of n double2, fully coalesced.
template <int NR, int NW>
__global__ void __launch_bounds__(256) stream_kernel(const double2* const* rd, double2* const* wr, size_t n) {
    for (size_t i = blockIdx.x * (size_t)256 + threadIdx.x; i < n; i += (size_t)gridDim.x * 256) {
        double2 s = make_double2(0.0, 0.0);
#pragma unroll
        for (int f = 0; f < NR; ++f) {
            const double2 v = rd[f][i];
            s.x += v.x;
            s.y += v.y;
        }
#pragma unroll
        for (int f = 0; f < NW; ++f) wr[f][i] = make_double2(s.x + f, s.y);
    }
}

// REPS in-register 1024-point transforms per row (64-thread teams, the
// engine's 16.4.16 plan), one load and one store per row.
template <int REPS>
__global__ void __launch_bounds__(128) fft_kernel(const double2* in, double2* out, const double2* tw, int rows) {
    extern __shared__ __align__(16) double2 smraw[];
    const int g = threadIdx.x / 64, t = threadIdx.x % 64;
    const int row = blockIdx.x * 2 + g;
    if (row >= rows) return;
    double2* region = smraw + g * TeamLayout<kN>::ROWS;
    const TeamPolicy<kN, double2> pol{region, 1 + g};
    const TwSeed<double2> seed = twiddle_seeds<kN>(tw, t);
    double2 v[1][16];
#pragma unroll
    for (int m = 0; m < 16; ++m) v[0][m] = in[(size_t)row * kN + t + 64 * m];
#pragma unroll 1
    for (int r = 0; r < REPS; ++r) fft_batched<kN, -1, 1>(v, pol, seed, t);
#pragma unroll
    for (int m = 0; m < 16; ++m) out[(size_t)row * kN + t + 64 * m] = v[0][m];
}

// REPS in-register 1024-point transforms per row by the warp engine: one warp
// per row (lane t holds x[t + 32 m]), four rows per 128-thread block, a private
// 32 x 33 transpose tile per warp.
template <int REPS>
__global__ void __launch_bounds__(128) wfft_kernel(const double2* in, double2* out, const double2* tw, int rows) {
    extern __shared__ __align__(16) double2 wsm[];
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int row = blockIdx.x * 4 + w;
    if (row >= rows) return;
    double2* tile = wsm + w * WfftTile<double2>::ELEMS;
    const double2 w1 = __ldg(tw + lane);
    double2 v[32];
#pragma unroll
    for (int m = 0; m < 32; ++m) v[m] = in[(size_t)row * kN + lane + 32 * m];
#pragma unroll 1
    for (int r = 0; r < REPS; ++r) wfft1024<-1>(v, tile, w1, lane);
#pragma unroll
    for (int m = 0; m < 32; ++m) out[(size_t)row * kN + lane + 32 * m] = v[m];
}

struct Timer {
    cudaEvent_t a, b;
    Timer() {
        FCK(cudaEventCreate(&a));
        FCK(cudaEventCreate(&b));
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

}  // namespace

int main() {
    int sms = 0;
    FCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    const size_t bytes = sizeof(double2) * kElems;
    std::vector<double2*> buf(9);
    for (auto& p : buf) {
        FCK(cudaMalloc(&p, bytes));
        FCK(cudaMemset(p, 0, bytes));
    }
    double2 **drd, **dwr;
    FCK(cudaMalloc(&drd, 4 * sizeof(double2*)));
    FCK(cudaMalloc(&dwr, 5 * sizeof(double2*)));
    FCK(cudaMemcpy(drd, buf.data(), 4 * sizeof(double2*), cudaMemcpyHostToDevice));
    FCK(cudaMemcpy(dwr, buf.data() + 4, 5 * sizeof(double2*), cudaMemcpyHostToDevice));
    void* flush;
    const size_t flush_bytes = (size_t)256 << 20;
    FCK(cudaMalloc(&flush, flush_bytes));
    Timer tm;

    std::printf("streaming floor per pass class (%d SMs; one half spectrum S = %zu B)\n", sms, bytes);
    std::printf("%-34s %10s %10s %12s %12s\n", "class", "warm us", "evicted us", "warm GB/s", "evicted GB/s");
    auto stream_case = [&](const char* name, int nr, int nw, auto launch) {
        const double mb = (double)(nr + nw) * bytes;
        float t[2] = {0, 0};
        for (int ev = 0; ev < 2; ++ev) {
            launch();
            FCK(cudaDeviceSynchronize());
            const int reps = 50;
            for (int it = 0; it < reps; ++it) {
                if (ev) FCK(cudaMemsetAsync(flush, it & 0xff, flush_bytes));
                FCK(cudaEventRecord(tm.a));
                launch();
                FCK(cudaEventRecord(tm.b));
                FCK(cudaEventSynchronize(tm.b));
                float ms;
                FCK(cudaEventElapsedTime(&ms, tm.a, tm.b));
                t[ev] += ms;
            }
            t[ev] *= 1000.0f / reps;
        }
        std::printf("%-34s %10.2f %10.2f %12.1f %12.1f\n", name, t[0], t[1], mb / (t[0] * 1e3), mb / (t[1] * 1e3));
    };
    const dim3 sg(sms * 8), sb(256);
    stream_case("8 S: read 3, write 5 (column stage)", 3, 5,
                [&] { stream_kernel<3, 5><<<sg, sb>>>(drd, dwr, kElems); });
    stream_case("5 S: read 4, write 1 (final, row)", 4, 1,
                [&] { stream_kernel<4, 1><<<sg, sb>>>(drd, dwr, kElems); });
    stream_case("5 S: read 1, write 4 (first column)", 1, 4,
                [&] { stream_kernel<1, 4><<<sg, sb>>>(drd, dwr, kElems); });
    FCK(cudaGetLastError());

    // FFT engine throughput
    const int rows = 8192;
    double2 *in, *out, *tw;
    FCK(cudaMalloc(&in, sizeof(double2) * (size_t)rows * kN));
    FCK(cudaMalloc(&out, sizeof(double2) * (size_t)rows * kN));
    FCK(cudaMalloc(&tw, sizeof(double2) * kN));
    std::vector<double2> h(kN);
    for (int m = 0; m < kN; ++m) h[m] = make_double2(std::cos(2.0 * M_PI * m / kN), -std::sin(2.0 * M_PI * m / kN));
    FCK(cudaMemcpy(tw, h.data(), sizeof(double2) * kN, cudaMemcpyHostToDevice));
    FCK(cudaMemset(in, 0, sizeof(double2) * (size_t)rows * kN));
    const size_t smem = 2 * TeamLayout<kN>::ROWS * sizeof(double2);
    FCK(cudaFuncSetAttribute((const void*)fft_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FCK(cudaFuncSetAttribute((const void*)fft_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    float ms8 = 0, ms1 = 0;
    for (int k = 0; k < 2; ++k) {
        fft_kernel<8><<<rows / 2, 128, smem>>>(in, out, tw, rows);
        fft_kernel<1><<<rows / 2, 128, smem>>>(in, out, tw, rows);
    }
    FCK(cudaDeviceSynchronize());
    for (int k = 0; k < 20; ++k) {
        float ms;
        FCK(cudaEventRecord(tm.a));
        fft_kernel<8><<<rows / 2, 128, smem>>>(in, out, tw, rows);
        FCK(cudaEventRecord(tm.b));
        FCK(cudaEventSynchronize(tm.b));
        FCK(cudaEventElapsedTime(&ms, tm.a, tm.b));
        ms8 += ms;
        FCK(cudaEventRecord(tm.a));
        fft_kernel<1><<<rows / 2, 128, smem>>>(in, out, tw, rows);
        FCK(cudaEventRecord(tm.b));
        FCK(cudaEventSynchronize(tm.b));
        FCK(cudaEventElapsedTime(&ms, tm.a, tm.b));
        ms1 += ms;
    }
    FCK(cudaGetLastError());
    // eight transforms minus one: the cost of seven in-register transforms
    const double ns_per = (ms8 - ms1) / 20.0 * 1e6 / (7.0 * rows);
    std::printf("\nFFT engine: 1024-point FP64 transform, in registers: %.2f ns per transform on the device\n", ns_per);
    std::printf("  (%d rows, 64-thread teams; the RK4 step needs about 20,500 such transforms: %.1f us)\n", rows,
                ns_per * 20500.0 * 1e-3);

    // the warp-per-transform engine, same method
    const size_t wsmem = 4 * WfftTile<double2>::bytes();
    FCK(cudaFuncSetAttribute((const void*)wfft_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsmem));
    FCK(cudaFuncSetAttribute((const void*)wfft_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsmem));
    float wms8 = 0, wms1 = 0;
    for (int k = 0; k < 2; ++k) {
        wfft_kernel<8><<<rows / 4, 128, wsmem>>>(in, out, tw, rows);
        wfft_kernel<1><<<rows / 4, 128, wsmem>>>(in, out, tw, rows);
    }
    FCK(cudaDeviceSynchronize());
    for (int k = 0; k < 20; ++k) {
        float ms;
        FCK(cudaEventRecord(tm.a));
        wfft_kernel<8><<<rows / 4, 128, wsmem>>>(in, out, tw, rows);
        FCK(cudaEventRecord(tm.b));
        FCK(cudaEventSynchronize(tm.b));
        FCK(cudaEventElapsedTime(&ms, tm.a, tm.b));
        wms8 += ms;
        FCK(cudaEventRecord(tm.a));
        wfft_kernel<1><<<rows / 4, 128, wsmem>>>(in, out, tw, rows);
        FCK(cudaEventRecord(tm.b));
        FCK(cudaEventSynchronize(tm.b));
        FCK(cudaEventElapsedTime(&ms, tm.a, tm.b));
        wms1 += ms;
    }
    FCK(cudaGetLastError());
    const double wns_per = (wms8 - wms1) / 20.0 * 1e6 / (7.0 * rows);
    std::printf("Warp engine (wfft.cuh): %.2f ns per transform on the device (one warp per row)\n", wns_per);
    return 0;
}
