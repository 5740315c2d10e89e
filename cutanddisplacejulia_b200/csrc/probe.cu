// FP64 fused multiply-add throughput probe: the measured CUDA-core FP64 peak
// that the TD pair kernels' roofline divides by (the published B200 figure is
// a nominal clock number; this one is taken on the machine, at its clocks).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/cad_td.h"

namespace {

// 8 independent FMA chains per thread; a data-dependent result is stored so
// nothing is removed by the compiler.
__global__ void __launch_bounds__(256) fma_probe_kernel(int64_t iters, double seed, double* out)
{
    double a0 = seed + threadIdx.x, a1 = a0 + 1.0, a2 = a0 + 2.0, a3 = a0 + 3.0;
    double a4 = a0 + 4.0, a5 = a0 + 5.0, a6 = a0 + 6.0, a7 = a0 + 7.0;
    const double m = 0.999999999, c = 1e-9;
    for (int64_t k = 0; k < iters; ++k) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
            a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
        }
    }
    const double r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = r;   // practically never taken
    if (threadIdx.x == 0 && blockIdx.x == 0) out[0] = r;
}

}  // namespace

extern "C" int cad_fp64_fma_probe(cad_ctx* ctx, int64_t iters, double* tflops)
{
    (void)ctx;
    if (!tflops || iters <= 0) return CAD_ERR_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return CAD_ERR_CUDA;
    const int blocks = sms * 8, threads = 256;
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return CAD_ERR_OOM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_probe_kernel<<<blocks, threads>>>(iters / 4 + 1, 1.0, out);   // warm-up
    cudaEventRecord(e0);
    fma_probe_kernel<<<blocks, threads>>>(iters, 1.0, out);
    cudaEventRecord(e1);
    const cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return CAD_ERR_CUDA;
    const double flops = 2.0 * 8.0 * 16.0 * (double)iters * blocks * threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return CAD_OK;
}
