// k_peak.cu -- FP64 FMA throughput microbenchmark (the roofline denominator
// of the FP64 kernels; the driver-measured peaks cover HBM and BF16 only).
#include <cstdio>

#include "dev_common.cuh"
#include "../../include/lmie_b200.h"

namespace {

constexpr int PEAK_CHAINS = 8;
constexpr int PEAK_ITERS = 4096;

__global__ void __launch_bounds__(256) k_fp64_fma(double seed, double *sink) {
    double v[PEAK_CHAINS];
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; ++c) v[c] = seed + threadIdx.x * 1e-9 + c;
    const double a = 0.999999999, b = 1e-9;
    for (int i = 0; i < PEAK_ITERS; ++i) {
#pragma unroll
        for (int c = 0; c < PEAK_CHAINS; ++c) v[c] = fma(v[c], a, b);
    }
    double s = 0.;
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; ++c) s += v[c];
    if (s == 1234.5) sink[threadIdx.x] = s;   // never true; keeps the chains live
}

}  // namespace

extern "C" int lmieb_stream(void **stream);

extern "C" int lmieb_fp64_peak(double *tflops) {
    void *sv = nullptr;
    if (lmieb_stream(&sv)) return -1;
    cudaStream_t s = (cudaStream_t) sv;
    int dev = 0, sms = 0;
    LMIEB_CUDA_TRY(cudaGetDevice(&dev));
    LMIEB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    double *sink = nullptr;
    LMIEB_CUDA_TRY(cudaMalloc((void **) &sink, 256 * sizeof(double)));
    cudaEvent_t e0, e1;
    LMIEB_CUDA_TRY(cudaEventCreate(&e0));
    LMIEB_CUDA_TRY(cudaEventCreate(&e1));
    const int blocks = sms * 8;
    k_fp64_fma<<<blocks, 256, 0, s>>>(1.0, sink);     // warm-up
    LMIEB_CUDA_TRY(cudaEventRecord(e0, s));
    const int reps = 5;
    for (int i = 0; i < reps; ++i) k_fp64_fma<<<blocks, 256, 0, s>>>(1.0 + i, sink);
    LMIEB_CUDA_TRY(cudaEventRecord(e1, s));
    LMIEB_CUDA_TRY(cudaEventSynchronize(e1));
    LMIEB_CUDA_TRY(cudaGetLastError());
    float ms = 0.f;
    LMIEB_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    const double flops = 2.0 * PEAK_CHAINS * PEAK_ITERS * 256.0 * blocks * reps;
    *tflops = flops / (ms * 1e-3) / 1e12;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return 0;
}
