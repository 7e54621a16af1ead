// cr_resolve.cuh — the per-pixel HQS resolve, shared by the resolve kernels
// and the exact re-run of the colour pass.
#pragma once

#include "cr_device.cuh"
#include "cr_internal.h"

namespace crd {

__device__ __forceinline__ uint32_t pack_rgba(float r, float g, float b, float a) {
    return unorm8(r) | (unorm8(g) << 8) | (unorm8(b) << 16) | (unorm8(a) << 24);
}

// resolveUpdate of one pixel, count path (Pipelines/Resolve/Shaders.metal:13-57).
__device__ __forceinline__ void resolve_pixel(const uint4 acc, uint32_t depth,
                                              const ResolveUniforms &u, uint32_t &rgba,
                                              float &depthf) {
    if (acc.w == 0u) {
        rgba = pack_rgba(u.background[0], u.background[1], u.background[2], 0.0f);
        depthf = 0.0f;
        return;
    }
    const float inv = 1.0f / (float)acc.w;
    rgba = pack_rgba(((float)acc.x * inv) / 255.0f, ((float)acc.y * inv) / 255.0f,
                     ((float)acc.z * inv) / 255.0f, 1.0f);
    depthf = uint_to_depth(depth);
}

}  // namespace crd
