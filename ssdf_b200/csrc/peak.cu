// peak.cu -- FP32 / FP64 fused multiply-add throughput of this GPU, for the roofline denominator.
//
// The measured copy bandwidth and GEMM peaks of the machine do not include the scalar FP32 pipe,
// which bounds the traversal kernels; this microbenchmark measures it: every thread runs 8
// independent FMA chains (enough ILP to saturate the pipe), on a grid of several waves.
#include <cuda_runtime.h>

#include "internal.h"

namespace ssdf_b200 {
namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma(int iters, T seed, T *sink) {
    T a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + T(threadIdx.x + k);
    const T m = T(0.999999), c = T(1e-7);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = fma(a[k], m, c);
    }
    T s = T(0);
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == T(-1)) sink[0] = s;  // never true; keeps the chains alive
}

}  // namespace
}  // namespace ssdf_b200

extern "C" int ssdf_b200_fma_peak(int f64, double *tflops) {
    using namespace ssdf_b200;
    if (!tflops) return fail(SSDF_ERR_INVALID_ARGUMENT, "null output");
    int dev = 0, sms = 0;
    SSDF_CUDA(cudaGetDevice(&dev));
    SSDF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, threads = 256, iters = f64 ? 4096 : 16384;
    void *sink = nullptr;
    SSDF_CUDA(cudaMalloc(&sink, 16));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        if (f64)
            k_fma<double><<<blocks, threads>>>(iters, 1.0, (double *)sink);
        else
            k_fma<float><<<blocks, threads>>>(iters, 1.0f, (float *)sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess) return cuda_fail(err, "k_fma", __FILE__, __LINE__);
    const double flops = 2.0 * 8.0 * double(iters) * double(blocks) * threads;
    *tflops = flops / (double(best) * 1e-3) / 1e12;
    return SSDF_OK;
}
