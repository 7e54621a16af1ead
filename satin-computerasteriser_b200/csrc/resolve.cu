// resolve.cu — per-pixel passes: resolve, nearest resolve, hole fill.
//
//   resolve_hqs      resolveUpdate, count path (Pipelines/Resolve/Shaders.metal:13-57)
//   resolve_nearest  nearestResolveUpdate (Pipelines/NearestResolve/Shaders.metal:8-38)
//   hole_fill        holeFillUpdate (Pipelines/HoleFill/Shaders.metal:10-48), ping-pong
//                    as ComputeRasteriser.encodeHoleFill (ComputeRasteriser.swift:298-320)
//
// The reference writes an rgba8Unorm texture and an R32Float depth texture;
// here both are linear device buffers (row 0 = top row, as the passes flip
// y), one uint32 per pixel holding R | G<<8 | B<<16 | A<<24.
#include "cr_device.cuh"
#include "cr_internal.h"

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ uint32_t pack_rgba(float r, float g, float b, float a) {
    return crd::unorm8(r) | (crd::unorm8(g) << 8) | (crd::unorm8(b) << 16) | (crd::unorm8(a) << 24);
}

__global__ void __launch_bounds__(kThreads)
    resolve_hqs(const uint32_t *__restrict__ depth, const uint4 *__restrict__ accum,
                uint32_t *__restrict__ rgba, float *__restrict__ depthf, uint32_t npix,
                ResolveUniforms u, uint32_t *redo_flag, int check, const uint32_t *redo) {
    if (redo && *redo == 0u) return;
    for (uint32_t p = blockIdx.x * kThreads + threadIdx.x; p < npix; p += gridDim.x * kThreads) {
        const uint4 acc = accum[p];
        // Packed colour adds are exact while every count is at most
        // kPackedMaxCount: past it a channel sum may have carried into its
        // neighbour field, and the frame's colour pass is re-run exactly.
        if (check && acc.w > kPackedMaxCount) *redo_flag = 1u;
        if (acc.w == 0u) {
            rgba[p] = pack_rgba(u.background[0], u.background[1], u.background[2], 0.0f);
            depthf[p] = 0.0f;
            continue;
        }
        const float inv = 1.0f / (float)acc.w;
        rgba[p] = pack_rgba(((float)acc.x * inv) / 255.0f, ((float)acc.y * inv) / 255.0f,
                            ((float)acc.z * inv) / 255.0f, 1.0f);
        depthf[p] = crd::uint_to_depth(depth[p]);
    }
}

__global__ void __launch_bounds__(kThreads)
    resolve_nearest(const unsigned long long *__restrict__ keys,
                    const uint32_t *__restrict__ colors, uint32_t *__restrict__ rgba,
                    float *__restrict__ depthf, uint32_t npix, ResolveUniforms u) {
    const uint32_t p = blockIdx.x * kThreads + threadIdx.x;
    if (p >= npix) return;
    const unsigned long long k = keys[p];
    const uint32_t d = (uint32_t)(k >> 32);
    const uint32_t idx = ~(uint32_t)k;
    if (d == 0u || idx == 0xffffffffu) {
        rgba[p] = pack_rgba(u.background[0], u.background[1], u.background[2], 0.0f);
        depthf[p] = 0.0f;
        return;
    }
    const uint32_t c = colors[idx];
    rgba[p] = pack_rgba((float)(c & 0xffu) / 255.0f, (float)((c >> 8) & 0xffu) / 255.0f,
                        (float)((c >> 16) & 0xffu) / 255.0f, 1.0f);
    depthf[p] = crd::uint_to_depth(d);
}

__device__ __forceinline__ float unorm_ch(uint32_t v, int ch) {
    return (float)((v >> (8 * ch)) & 0xffu) / 255.0f;
}

__global__ void __launch_bounds__(kThreads)
    hole_fill(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, int w, int h) {
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * (kThreads / 32) + (threadIdx.x >> 5);
    if (x >= w || y >= h) return;
    const uint32_t center = src[(size_t)y * w + x];
    if (unorm_ch(center, 3) >= 0.5f) {
        dst[(size_t)y * w + x] = center;
        return;
    }
    float sr = 0.0f, sg = 0.0f, sb = 0.0f, cnt = 0.0f;
#pragma unroll
    for (int oy = -1; oy <= 1; ++oy) {
#pragma unroll
        for (int ox = -1; ox <= 1; ++ox) {
            if (ox == 0 && oy == 0) continue;
            const int sx = x + ox, sy = y + oy;
            if (sx < 0 || sx >= w || sy < 0 || sy >= h) continue;
            const uint32_t n = src[(size_t)sy * w + sx];
            if (unorm_ch(n, 3) >= 0.5f) {
                sr = sr + unorm_ch(n, 0);
                sg = sg + unorm_ch(n, 1);
                sb = sb + unorm_ch(n, 2);
                cnt = cnt + 1.0f;
            }
        }
    }
    dst[(size_t)y * w + x] = cnt > 0.0f ? pack_rgba(sr / cnt, sg / cnt, sb / cnt, 1.0f) : center;
}

__global__ void __launch_bounds__(kThreads)
    split_nearest(const unsigned long long *__restrict__ keys, uint32_t *__restrict__ depth,
                  uint32_t *__restrict__ index, size_t n) {
    const size_t p = (size_t)blockIdx.x * kThreads + threadIdx.x;
    if (p >= n) return;
    const unsigned long long k = keys[p];
    if (depth) depth[p] = (uint32_t)(k >> 32);
    if (index) index[p] = ~(uint32_t)k;
}

__global__ void __launch_bounds__(kThreads)
    accum_redo_clear(uint4 *__restrict__ accum, const uint32_t *redo, uint32_t npix) {
    if (*redo == 0u) return;
    for (uint32_t p = blockIdx.x * kThreads + threadIdx.x; p < npix; p += gridDim.x * kThreads)
        accum[p] = make_uint4(0u, 0u, 0u, 0u);
}

}  // namespace

cr_status launch_resolve_hqs(cr_frame *f, const ResolveUniforms &u, cudaStream_t s, bool check,
                             const uint32_t *redo) {
    const uint32_t npix = (uint32_t)f->width * (uint32_t)f->height;
    // One pixel per thread; the gated re-run (rarely needed) uses a small
    // grid-stride grid so that skipping it costs little.
    const uint32_t grid = redo ? (uint32_t)f->ctx->sm_count * 4 : (npix + kThreads - 1) / kThreads;
    resolve_hqs<<<grid, kThreads, 0, s>>>(
        f->d_depth, f->d_accum, f->d_rgba[0], f->d_depthf, npix, u, f->d_redo, check ? 1 : 0,
        redo);
    CR_CUDA(cudaGetLastError());
    f->final_rgba = 0;
    return CR_OK;
}

cr_status launch_accum_redo_clear(cr_frame *f, cudaStream_t s) {
    const uint32_t npix = (uint32_t)f->width * (uint32_t)f->height;
    accum_redo_clear<<<f->ctx->sm_count * 4, kThreads, 0, s>>>(f->d_accum, f->d_redo, npix);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

cr_status launch_resolve_nearest(cr_frame *f, const uint32_t *colors, const ResolveUniforms &u,
                                 cudaStream_t s) {
    const uint32_t npix = (uint32_t)f->width * (uint32_t)f->height;
    resolve_nearest<<<(npix + kThreads - 1) / kThreads, kThreads, 0, s>>>(
        f->d_nearest, colors, f->d_rgba[0], f->d_depthf, npix, u);
    CR_CUDA(cudaGetLastError());
    f->final_rgba = 0;
    return CR_OK;
}

cr_status launch_hole_fill(cr_frame *f, int iterations, cudaStream_t s) {
    // The resolve wrote d_rgba[final_rgba]; each iteration reads one buffer
    // and writes the other, and the last written buffer is the result.
    const dim3 grid((f->width + 31) / 32, (f->height + 7) / 8);
    for (int it = 0; it < iterations; ++it) {
        const int src = f->final_rgba, dst = 1 - f->final_rgba;
        hole_fill<<<grid, kThreads, 0, s>>>(f->d_rgba[src], f->d_rgba[dst], f->width, f->height);
        CR_CUDA(cudaGetLastError());
        f->final_rgba = dst;
    }
    return CR_OK;
}

cr_status launch_split_nearest(const unsigned long long *keys, uint32_t *depth_out,
                               uint32_t *index_out, size_t n, cudaStream_t s) {
    if (n == 0) return CR_OK;
    split_nearest<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(keys, depth_out,
                                                                               index_out, n);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}
