/*
 * ref_gpu_shim.h — force-included (nvcc -include) when the reference's CUDA
 * sources are compiled for sm_100a (TEST/BENCH INFRASTRUCTURE ONLY).  The
 * reference calls __shfl_xor (compute/CUDA/cross_kernal_v2.cu:97), which CUDA
 * no longer provides for sm_70 and later; it is mapped here to
 * __shfl_xor_sync over the full warp, its documented replacement.  Nothing
 * else of the reference is changed.
 */
#pragma once
#include <cuda_runtime.h>
#if defined(__CUDACC__)
/* the toolkit headers that declare the removed forms come first, so the
 * mapping below applies only to the reference's own calls */
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cuComplex.h>
#include <thrust/complex.h>
#include <cub/cub.cuh>
#define __shfl_xor(v, m) __shfl_xor_sync(0xffffffffu, (v), (m))
#endif
