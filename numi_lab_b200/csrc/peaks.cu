// Issue-rate and FP32 FMA peak of the current device, measured with CUDA
// events: the denominator of the issue roofline of the latency-bound
// control-step kernels (their HBM roofline does not bind).  Every thread
// runs kChains independent FMA chains, so each warp issues one FMA per
// cycle whenever a scheduler has an eligible warp; with 2048 resident
// threads per SM the schedulers never starve.
#include "numi_b200.h"
#include "runtime.h"

#include <cuda_runtime.h>

namespace {

using numi::rt::check;
using numi::rt::guarded;

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) fma_peak_kernel(float* out, int iterations, float a, float b) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = static_cast<float>(threadIdx.x + c);
    for (int i = 0; i < iterations; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 1.2345e-30f) out[threadIdx.x] = s;  // keeps the chains live; never true for these inputs
}

}  // namespace

extern "C" {

MR_API int mr_measure_issue_peak(double* fma_tflops, double* warp_instructions_per_second) {
    return guarded([&] {
        if (!fma_tflops || !warp_instructions_per_second) throw std::invalid_argument("outputs must be non-null");
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        cudaDeviceProp prop{};
        check(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
        const int threads = 256;
        const int blocks = prop.multiProcessorCount * (prop.maxThreadsPerMultiProcessor / threads);
        const int iterations = 1 << 16;
        float* out = nullptr;
        check(cudaMalloc(&out, threads * sizeof(float)), "cudaMalloc");
        cudaEvent_t a = nullptr, b = nullptr;
        check(cudaEventCreate(&a), "event");
        check(cudaEventCreate(&b), "event");
        float best = 1e30f;
        for (int r = 0; r < 4; ++r) {
            check(cudaEventRecord(a), "event");
            fma_peak_kernel<<<blocks, threads>>>(out, iterations, 0.999999f, 1e-7f);
            check(cudaGetLastError(), "fma peak launch");
            check(cudaEventRecord(b), "event");
            check(cudaEventSynchronize(b), "sync");
            float ms = 0.0f;
            check(cudaEventElapsedTime(&ms, a, b), "elapsed");
            if (r > 0) best = best < ms ? best : ms;  // the first run warms up
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaFree(out);
        const double fmas = static_cast<double>(blocks) * threads * iterations * kChains;
        *fma_tflops = 2.0 * fmas / (best * 1e-3) / 1e12;
        *warp_instructions_per_second = fmas / 32.0 / (best * 1e-3);
    });
}

}  // extern "C"
