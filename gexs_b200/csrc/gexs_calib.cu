/*
 * gexs_calib.cu — FP32 FMA throughput probe.  The cross-section kernels are
 * bound by FP32/SFU issue, not by HBM or tensor cores, so their roofline
 * denominator is the device's measured FP32 FMA rate.
 */
#include <cuda_runtime.h>
#include "gexs_internal.h"

namespace gexs {

__global__ void __launch_bounds__(256) fma_probe(float* sink, int iters, float a, float b)
{
    float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
    float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 12345.678f) sink[blockIdx.x] = s;   /* keeps the chains live */
}

}  // namespace gexs

using namespace gexs;


/* measured FP32 FMA rate in TFLOP/s (2 FLOP per FMA) */
extern "C" int gexs_probe_fp32_tflops(int device, double* tflops)
{
    if (!tflops) return set_error(GEXS_ERR_INVALID, "tflops is NULL");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    float* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(float) * nsm * 8) != cudaSuccess) return set_error(GEXS_ERR_OOM, "sink");
    const int blocks = nsm * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        fma_probe<<<blocks, threads>>>(sink, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    e = cudaGetLastError();
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_error(e, "fma probe");
    double flops = 2.0 * 8.0 * 16.0 * (double)iters * threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return GEXS_OK;
}
