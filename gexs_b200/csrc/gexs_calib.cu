/*
 * gexs_calib.cu — FP32 FMA throughput probe.  The cross-section kernels are
 * bound by FP32/SFU issue, not by HBM or tensor cores, so their roofline
 * denominator is the device's measured FP32 FMA rate.
 */
#include <cuda_runtime.h>
#include "gexs_internal.h"
#include "gexs_device.cuh"

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

__global__ void __launch_bounds__(256) dfma_probe(double* sink, int iters, double a, double b)
{
    double x0 = threadIdx.x * 1e-7, x1 = x0 + 1.0, x2 = x0 + 2.0, x3 = x0 + 3.0;
    double x4 = x0 + 4.0, x5 = x0 + 5.0, x6 = x0 + 6.0, x7 = x0 + 7.0;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 12345.678) sink[blockIdx.x] = s;
}

/* reciprocal approximations (one MUFU op each) on independent chains.
 * Each step is r(1 + x/2): the FMA keeps the compiler from folding a
 * reciprocal of a reciprocal and costs an eighth of a MUFU op's issue
 * time on the FP32 pipe. */
__device__ __forceinline__ float rcp_step(float x)
{
    float r;
    asm volatile("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(fmaf(x, 0.5f, 1.0f)));
    return r;
}

__global__ void __launch_bounds__(256) rcp_probe(float* sink, int iters)
{
    float x0 = 1.f + threadIdx.x * 1e-7f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
    float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = rcp_step(x0); x1 = rcp_step(x1); x2 = rcp_step(x2); x3 = rcp_step(x3);
            x4 = rcp_step(x4); x5 = rcp_step(x5); x6 = rcp_step(x6); x7 = rcp_step(x7);
        }
    }
    float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 12345.678f) sink[blockIdx.x] = s;
}

}  // namespace gexs

using namespace gexs;

namespace {
/* ops / best launch time of three after a warm-up launch */
template <typename F>
int time_probe(int device, double ops, F launch, double* rate)
{
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        launch();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    e = cudaGetLastError();
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_error(e, "probe");
    *rate = ops / (best * 1e-3);
    return GEXS_OK;
}
}  // namespace

/* measured FP64 FMA rate in TFLOP/s (2 FLOP per FMA) */
extern "C" int gexs_probe_fp64_tflops(int device, double* tflops)
{
    if (!tflops) return set_error(GEXS_ERR_INVALID, "tflops is NULL");
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return set_error(GEXS_ERR_CUDA, "device attribute");
    double* sink = nullptr;
    if (cudaSetDevice(device) != cudaSuccess || cudaMalloc(&sink, sizeof(double) * nsm * 8) != cudaSuccess)
        return set_error(GEXS_ERR_OOM, "sink");
    const int blocks = nsm * 8, threads = 256, iters = 1024;
    double rate = 0.0;
    int st = time_probe(device, 2.0 * 8.0 * 16.0 * (double)iters * threads * blocks,
                        [&] { dfma_probe<<<blocks, threads>>>(sink, iters, 0.999999, 1e-7); }, &rate);
    cudaFree(sink);
    if (st) return st;
    *tflops = rate / 1e12;
    return GEXS_OK;
}

/* measured rcp.approx.f32 rate (the MUFU reciprocal that region I of the
 * FP32 Voigt form takes once per evaluation) in 1e9 operations/s */
extern "C" int gexs_probe_rcp_gops(int device, double* gops)
{
    if (!gops) return set_error(GEXS_ERR_INVALID, "gops is NULL");
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return set_error(GEXS_ERR_CUDA, "device attribute");
    float* sink = nullptr;
    if (cudaSetDevice(device) != cudaSuccess || cudaMalloc(&sink, sizeof(float) * nsm * 8) != cudaSuccess)
        return set_error(GEXS_ERR_OOM, "sink");
    const int blocks = nsm * 8, threads = 256, iters = 1024;
    double rate = 0.0;
    int st = time_probe(device, 8.0 * 16.0 * (double)iters * threads * blocks,
                        [&] { rcp_probe<<<blocks, threads>>>(sink, iters); }, &rate);
    cudaFree(sink);
    if (st) return st;
    *gops = rate / 1e9;
    return GEXS_OK;
}


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
