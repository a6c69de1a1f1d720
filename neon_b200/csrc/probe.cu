// probe.cu -- measured FP64 / FP32 CUDA-core FMA throughput, the denominator of the element
// kernel's compute roofline (the HBM and bf16 denominators are measured by the platform).
#include <cstdio>

#include "../../include/neon_b200_probe.h"

namespace {

template <typename T>
__global__ void k_fma_chain(T* out, int iters, T a, T b) {
    // 8 independent chains per thread keep the FMA pipe full
    T x0 = threadIdx.x * (T)1e-7, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
    T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fma(x0, a, b);
            x1 = fma(x1, a, b);
            x2 = fma(x2, a, b);
            x3 = fma(x3, a, b);
            x4 = fma(x4, a, b);
            x5 = fma(x5, a, b);
            x6 = fma(x6, a, b);
            x7 = fma(x7, a, b);
        }
    }
    T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-12345.0) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

template <typename T>
int run(double* flops_per_second) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    const int threads = 256, blocks = sms * 8, iters = 4096;
    T* out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * threads * blocks) != cudaSuccess) return 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_chain<T><<<blocks, threads>>>(out, 64, (T)0.999999, (T)1e-6);  // warm-up
    cudaEventRecord(e0);
    k_fma_chain<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-6);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return 8;
    const double flops = 2.0 * 8.0 * 16.0 * (double)iters * threads * blocks;
    *flops_per_second = flops / (ms * 1e-3);
    return 0;
}

}  // namespace

extern "C" int nb2_probe_fma_throughput(int32_t fp64, double* flops_per_second) {
    if (!flops_per_second) return 7;
    return fp64 ? run<double>(flops_per_second) : run<float>(flops_per_second);
}
