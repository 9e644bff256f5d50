// Device helpers shared by the pass kernels and the pair kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "p2p_internal.h"

namespace p2p {

constexpr unsigned kFull = 0xffffffffu;

// Bounds on the scaled squared separation u of any pair of a list entry from
// the two leaves' frames: the FP32-rounded offset of the frame centres (ox,
// oy, oz) and the particles' half-extents (scaled, rounded up). The upper
// bound includes the softening; the lower bound omits it (valid for both
// softening rules).
__device__ __forceinline__ void entry_offset(const LeafMeta &s, const LeafMeta &t, const double cscale,
                                             float &ox, float &oy, float &oz) {
    ox = (float)((s.cx - t.cx) * cscale);
    oy = (float)((s.cy - t.cy) * cscale);
    oz = (float)((s.cz - t.cz) * cscale);
}
__device__ __forceinline__ float entry_u_max(const LeafMeta &s, const LeafMeta &t, const float ox,
                                             const float oy, const float oz, const float eps2) {
    const float bx = fabsf(ox) + s.hx + t.hx, by = fabsf(oy) + s.hy + t.hy, bz = fabsf(oz) + s.hz + t.hz;
    return fmaf(bx, bx, fmaf(by, by, fmaf(bz, bz, eps2)));
}
__device__ __forceinline__ float entry_u_min(const LeafMeta &s, const LeafMeta &t, const float ox,
                                             const float oy, const float oz) {
    const float bx = fmaxf(fabsf(ox) - s.hx - t.hx, 0.f), by = fmaxf(fabsf(oy) - s.hy - t.hy, 0.f),
                bz = fmaxf(fabsf(oz) - s.hz - t.hz, 0.f);
    return fmaf(bx, bx, fmaf(by, by, bz * bz));
}

__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

}  // namespace p2p
