// FP64 FMA throughput probe: the roofline denominator for the depth-kernel
// stage, whose work runs on the FP64 CUDA-core pipe (MEASURED_PEAKS-style
// copy and GEMM figures do not cover it).  Each thread runs 8 independent
// FMA chains; the grid fills every SM several times over.
#include <cuda_runtime.h>
#include "../../include/dazi_dk.h"

namespace {

__global__ void fp64_fma_kernel(double* out, int iters, double s)
{
    double a0 = threadIdx.x * 1e-9, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
    double a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
    const double m = 0.999999999;
#pragma unroll 4
    for (int i = 0; i < iters; ++i) {
        a0 = fma(a0, m, s); a1 = fma(a1, m, s); a2 = fma(a2, m, s); a3 = fma(a3, m, s);
        a4 = fma(a4, m, s); a5 = fma(a5, m, s); a6 = fma(a6, m, s); a7 = fma(a7, m, s);
    }
    const double r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 12345.678) out[blockIdx.x] = r;   // keeps the chains live
}

}  // namespace

extern "C" int dazi_dk_fp64_peak(double* gflops)
{
    if (!gflops) return DAZI_ERR_BADARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DAZI_ERR_NODEVICE;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return DAZI_ERR_CUDA;
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * sms * 64) != cudaSuccess) return DAZI_ERR_NOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int threads = 256, blocks = sms * 8, iters = 1 << 14;
    fp64_fma_kernel<<<blocks, threads>>>(out, 256, 1e-3);   // warm-up
    double best = 0.0;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        fp64_fma_kernel<<<blocks, threads>>>(out, iters, 1e-3);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8.0 * (double)iters * threads * blocks;
        const double g = flops / (ms * 1e-3) / 1e9;
        if (g > best) best = g;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return DAZI_ERR_CUDA;
    *gflops = best;
    return 0;
}
