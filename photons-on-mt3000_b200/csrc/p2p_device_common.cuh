// Device helpers shared by the pass kernels and the pair kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "p2p_internal.h"

namespace p2p {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

}  // namespace p2p
