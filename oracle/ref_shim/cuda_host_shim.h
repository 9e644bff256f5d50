/* Test-infrastructure shim: makes the reference's device pair functions in
 * src/gpu_kernel.impl.h compile as host C++ so the oracle can call them
 * (P2P_core_lite, P2P_core, P2P_core_1). The __global__ kernels in that file
 * only have to compile; they are never called on the host. rsqrt is written
 * as 1/sqrt, the meaning CUDA documents for it. */
#ifndef PHOTONS_ORACLE_CUDA_HOST_SHIM_H
#define PHOTONS_ORACLE_CUDA_HOST_SHIM_H
#include <math.h>
#define __device__
#define __global__ static inline
#define __shared__
#define __syncthreads() ((void)0)
#ifndef CUDART_VERSION
#define CUDART_VERSION 12000
#endif
#define WARP 32
typedef unsigned char uint_8b;
#ifdef GPU_DP
typedef double gpuT;
#else
typedef float gpuT;
#endif
struct float3 { float x, y, z; };
struct double3 { double x, y, z; };
struct shim_dim3 { unsigned x, y, z; };
static const shim_dim3 threadIdx = {0, 0, 0}, blockIdx = {0, 0, 0},
                       blockDim = {1, 1, 1}, gridDim = {1, 1, 1};
static inline float rsqrt(float v) { return 1.0f / sqrtf(v); }
static inline double rsqrt(double v) { return 1.0 / sqrt(v); }
template <typename T> static inline T __shfl_xor_sync(unsigned, T v, int) { return v; }
#endif
