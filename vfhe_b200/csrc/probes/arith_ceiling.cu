// Arithmetic ceilings of the butterfly kinds the transforms could use, on one GPU:
// register-only loops (no memory traffic in the timed region), 8 CTAs x 256 threads per
// SM, results stored at the end so nothing is dead code.  Prints operations per clock
// per SM at the device's maximum SM clock.  Not part of the engine library; build and
// run by hand:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 \
//        vfhe_b200/csrc/probes/arith_ceiling.cu -o arith_ceiling && ./arith_ceiling
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../fp64mod.cuh"

namespace {

constexpr int kIters = 4096;
constexpr int kThreads = 256;

// 64-bit Shoup butterflies on 16 residues (8 per stage): t = w y - floor(w' y / 2^64) q,
// in [0, 2q); sums and differences kept below 4q (Harvey's lazy bounds)
__global__ void __launch_bounds__(kThreads) k_shoup(uint64_t* out, uint64_t q, uint64_t w, uint64_t wp) {
    uint64_t x[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) x[m] = (threadIdx.x * 16 + m) % q;
    const uint64_t two_q = 2 * q;
    for (int it = 0; it < kIters; ++it) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            uint64_t u = x[m];
            u = u >= two_q ? u - two_q : u;
            const uint64_t y = x[m + 8];
            const uint64_t t = w * y - __umul64hi(wp, y) * q;
            x[m] = u + t;
            x[m + 8] = u - t + two_q;
        }
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] = x[m] >= two_q ? x[m] - two_q : x[m];
    }
    uint64_t s = 0;
#pragma unroll
    for (int m = 0; m < 16; ++m) s ^= x[m];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// the FP64 butterflies of the engine (fp64mod.cuh), reduced every fourth round
__global__ void __launch_bounds__(kThreads) k_fp64(double* out, double q, double qinv, double w, double wq) {
    double x[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) x[m] = (double)((threadIdx.x * 16 + m) & 1023);
    for (int it = 0; it < kIters; ++it) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const double v = vc::f_mulmod(x[m + 8], w, wq, q);
            const double u = x[m];
            x[m] = __dadd_rn(u, v);
            x[m + 8] = __dsub_rn(u, v);
        }
        if ((it & 3) == 3) {
#pragma unroll
            for (int m = 0; m < 16; ++m) x[m] = vc::f_reduce(x[m], q, qinv);
        }
    }
    double s = 0;
#pragma unroll
    for (int m = 0; m < 16; ++m) s += x[m];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// 8 independent chains of one instruction kind
__global__ void __launch_bounds__(kThreads) k_imad(uint32_t* out, uint32_t a, uint32_t b) {
    uint32_t x[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) x[m] = threadIdx.x + m;
    for (int it = 0; it < kIters; ++it)
#pragma unroll
        for (int m = 0; m < 8; ++m) x[m] = x[m] * a + b;
    out[blockIdx.x * blockDim.x + threadIdx.x] = x[0] ^ x[1] ^ x[2] ^ x[3] ^ x[4] ^ x[5] ^ x[6] ^ x[7];
}

__global__ void __launch_bounds__(kThreads) k_iadd(uint32_t* out, uint32_t a, uint32_t b) {
    uint32_t x[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) x[m] = threadIdx.x + m;
    for (int it = 0; it < kIters; ++it)
#pragma unroll
        for (int m = 0; m < 8; ++m) x[m] = (x[m] + a) ^ b;
    out[blockIdx.x * blockDim.x + threadIdx.x] = x[0] ^ x[1] ^ x[2] ^ x[3] ^ x[4] ^ x[5] ^ x[6] ^ x[7];
}

__global__ void __launch_bounds__(kThreads) k_dfma(double* out, double a, double b) {
    double x[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) x[m] = threadIdx.x + m;
    for (int it = 0; it < kIters; ++it)
#pragma unroll
        for (int m = 0; m < 8; ++m) x[m] = __fma_rn(x[m], a, b);
    out[blockIdx.x * blockDim.x + threadIdx.x] = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7];
}

template <typename F>
double time_ms(F launch) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch();
    cudaDeviceSynchronize();
    cudaEventRecord(e0);
    for (int r = 0; r < 5; ++r) launch();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / 5.0;
}

}  // namespace

int main() {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, 0) != cudaSuccess) {
        fprintf(stderr, "no CUDA device\n");
        return 1;
    }
    int clock_khz = 0;
    cudaDeviceGetAttribute(&clock_khz, cudaDevAttrClockRate, 0);
    const int sms = prop.multiProcessorCount;
    const int blocks = sms * 8;
    const double threads = (double)blocks * kThreads;
    void* buf = nullptr;
    if (cudaMalloc(&buf, (size_t)blocks * kThreads * 8) != cudaSuccess) return 1;
    const uint64_t q = (1ULL << 49) + 1ULL * 0x2A0001;  // any 50-bit odd modulus: timing only
    const uint64_t w = 123456789012345ULL % q;
    const uint64_t wp = (uint64_t)(((unsigned __int128)w << 64) / q);
    const double per_clk = 1e-3 * clock_khz * 1e3 * sms;  // clocks per ms over all SMs, / 1e3
    auto report = [&](const char* name, double ms, double ops_per_thread) {
        const double ops = threads * ops_per_thread;
        printf("%-34s %8.3f ms  %7.2f per clk per SM\n", name, ms, ops / (ms * per_clk));
    };
    const double qd = (double)q, qinv = 1.0 / qd, wd = (double)(w % (q / 2)), wq = wd / qd;
    report("64-bit Shoup butterfly", time_ms([&] { k_shoup<<<blocks, kThreads>>>((uint64_t*)buf, q, w, wp); }),
           8.0 * kIters);
    report("FP64 butterfly (exact, fp64mod)", time_ms([&] { k_fp64<<<blocks, kThreads>>>((double*)buf, qd, qinv, wd, wq); }),
           8.0 * kIters);
    report("32-bit IMAD", time_ms([&] { k_imad<<<blocks, kThreads>>>((uint32_t*)buf, 2654435761u, 12345u); }),
           8.0 * kIters);
    report("IADD + LOP pair", time_ms([&] { k_iadd<<<blocks, kThreads>>>((uint32_t*)buf, 2654435761u, 12345u); }),
           8.0 * 2 * kIters);
    report("DFMA", time_ms([&] { k_dfma<<<blocks, kThreads>>>((double*)buf, 0.999999, 1e-9); }), 8.0 * kIters);
    printf("SMs %d, max SM clock %d MHz\n", sms, clock_khz / 1000);
    cudaFree(buf);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
