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
#include <algorithm>

#include "cr_device.cuh"
#include "cr_internal.h"
#include "cr_resolve.cuh"

namespace {

constexpr int kThreads = 256;

using crd::pack_rgba;
using crd::resolve_pixel;

__global__ void __launch_bounds__(kThreads)
    resolve_hqs(const uint32_t *__restrict__ depth, const uint4 *__restrict__ accum,
                uint32_t *__restrict__ rgba, float *__restrict__ depthf, uint32_t npix,
                ResolveUniforms u, uint32_t *redo_flag, int check, const uint32_t *redo) {
    crd::grid_wait();
    crd::launch_dependents();
    if (redo && *redo == 0u) return;
    // Four pixels per thread, a grid-stride apart (each load coalesced over
    // the warp), with all eight loads issued before any pixel is resolved.
    const uint32_t stride = gridDim.x * kThreads;
    for (uint32_t p0 = blockIdx.x * kThreads + threadIdx.x; p0 < npix; p0 += 4u * stride) {
        uint4 acc[4];
        uint32_t d[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t p = p0 + (uint32_t)j * stride;
            acc[j] = p < npix ? accum[p] : make_uint4(0u, 0u, 0u, 0u);
            d[j] = p < npix ? depth[p] : 0u;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t p = p0 + (uint32_t)j * stride;
            if (p >= npix) break;
            // Packed colour adds are exact while every count is at most
            // kPackedMaxCount: past it a channel sum may have carried into
            // its neighbour field, and the frame's colour pass is re-run
            // exactly.
            if (check && acc[j].w > kPackedMaxCount) *redo_flag = 1u;
            // An uncovered pixel's depth is not used.
            resolve_pixel(acc[j], d[j], u, rgba[p], depthf[p]);
        }
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

// holeFillUpdate of pixel (x, y) of a w x h image.
__device__ __forceinline__ uint32_t hole_fill_pixel(const uint32_t *__restrict__ src, int x, int y,
                                                    int w, int h) {
    const uint32_t center = src[(size_t)y * w + x];
    if (unorm_ch(center, 3) >= 0.5f) return center;
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
    return cnt > 0.0f ? pack_rgba(sr / cnt, sg / cnt, sb / cnt, 1.0f) : center;
}

__global__ void __launch_bounds__(kThreads)
    hole_fill(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, int w, int h) {
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * (kThreads / 32) + (threadIdx.x >> 5);
    if (x >= w || y >= h) return;
    dst[(size_t)y * w + x] = hole_fill_pixel(src, x, y, w, h);
}

// ---------------------------------------------------------------------------
// Batched views: every view's pixels form one range [0, total_pix), view
// after view (ViewDesc::pix_begin); a thread finds its pixel's view by
// binary search over the views' begins, staged in shared memory.
// ---------------------------------------------------------------------------
// Views [0, nviews) of `views` cover pixels [views[0].pix_begin, end).
__device__ __forceinline__ void stage_begins(const ViewDesc *views, uint32_t nviews, uint32_t end,
                                             uint32_t *begin) {
    for (uint32_t v = threadIdx.x; v <= nviews; v += kThreads)
        begin[v] = v < nviews ? views[v].pix_begin : end;
    __syncthreads();
}

__device__ __forceinline__ uint32_t view_of_pixel(const uint32_t *begin, uint32_t nviews,
                                                  uint32_t p) {
    uint32_t lo = 0, hi = nviews;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (begin[mid] <= p)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Zeroes every view's accumulators and (not only_if_flag) depth plane and
// the redo flag; only_if_flag: the accumulators alone, and only if the flag
// is set.
__global__ void __launch_bounds__(kThreads)
    clear_views(const ViewDesc *__restrict__ views, uint32_t nviews, uint32_t pix0,
                uint32_t npix, uint32_t *redo_flag, int only_if_flag, int zero_flag) {
    __shared__ uint32_t begin[kMaxViews + 1];
    if (only_if_flag && *redo_flag == 0u) return;
    stage_begins(views, nviews, pix0 + npix, begin);
    if (zero_flag && blockIdx.x == 0 && threadIdx.x == 0) *redo_flag = 0u;
    for (uint32_t p = pix0 + blockIdx.x * kThreads + threadIdx.x; p < pix0 + npix;
         p += gridDim.x * kThreads) {
        const uint32_t v = view_of_pixel(begin, nviews, p);
        const uint32_t q = p - begin[v];
        const ViewDesc &vd = views[v];
        vd.accum[q] = make_uint4(0u, 0u, 0u, 0u);
        if (!only_if_flag) vd.depth[q] = 0u;
    }
}

__global__ void __launch_bounds__(kThreads)
    resolve_views(const ViewDesc *__restrict__ views, uint32_t nviews, uint32_t pix0,
                  uint32_t npix, ResolveUniforms u, uint32_t *redo_flag, int check,
                  const uint32_t *redo) {
    __shared__ uint32_t begin[kMaxViews + 1];
    if (redo && *redo == 0u) return;
    stage_begins(views, nviews, pix0 + npix, begin);
    for (uint32_t p = pix0 + blockIdx.x * kThreads + threadIdx.x; p < pix0 + npix;
         p += gridDim.x * kThreads) {
        const uint32_t v = view_of_pixel(begin, nviews, p);
        const uint32_t q = p - begin[v];
        const ViewDesc &vd = views[v];
        const uint4 acc = vd.accum[q];
        if (check && acc.w > kPackedMaxCount) *redo_flag = 1u;
        resolve_pixel(acc, acc.w ? vd.depth[q] : 0u, u, vd.rgba[0][q], vd.depthf[q]);
    }
}

__global__ void __launch_bounds__(kThreads)
    hole_fill_views(const ViewDesc *__restrict__ views, uint32_t nviews, uint32_t total_pix,
                    int src) {
    __shared__ uint32_t begin[kMaxViews + 1];
    stage_begins(views, nviews, total_pix, begin);  // all views: pix_begin of view 0 is 0
    for (uint32_t p = blockIdx.x * kThreads + threadIdx.x; p < total_pix;
         p += gridDim.x * kThreads) {
        const uint32_t v = view_of_pixel(begin, nviews, p);
        const uint32_t q = p - begin[v];
        const ViewDesc &vd = views[v];
        const int x = (int)(q % (uint32_t)vd.width), y = (int)(q / (uint32_t)vd.width);
        vd.rgba[1 - src][q] = hole_fill_pixel(vd.rgba[src], x, y, vd.width, vd.height);
    }
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

// Differentiable colours: the pixel's mean FP32 colour (background where no
// sample), row 0 = top, 3 floats per pixel.
__global__ void __launch_bounds__(kThreads)
    resolve_f32(const float4 *__restrict__ fsum, const uint32_t *__restrict__ fcount,
                float *__restrict__ image, uint32_t npix, float bg0, float bg1, float bg2) {
    for (uint32_t p = blockIdx.x * kThreads + threadIdx.x; p < npix; p += gridDim.x * kThreads) {
        const uint32_t n = fcount[p];
        float *o = image + 3 * (size_t)p;
        if (n == 0u) {
            o[0] = bg0;
            o[1] = bg1;
            o[2] = bg2;
            continue;
        }
        const float4 s = fsum[p];
        const float fn = (float)n;
        o[0] = s.x / fn;
        o[1] = s.y / fn;
        o[2] = s.z / fn;
    }
}

// L2 loss: dldimg = 2 * scale * (image - target); the loss, accumulated in
// FP64 per block, is added to *loss.
__global__ void __launch_bounds__(kThreads)
    l2_loss(const float *__restrict__ image, const float *__restrict__ target, uint64_t n,
            float scale, float *__restrict__ dldimg, double *loss) {
    __shared__ double part[kThreads / 32];
    double acc = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * kThreads) {
        const float d = image[i] - target[i];
        dldimg[i] = 2.0f * scale * d;
        acc += (double)d * (double)d;
    }
    if (!loss) return;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += part[w];
        atomicAdd(loss, t * (double)scale);
    }
}

__global__ void __launch_bounds__(kThreads)
    accum_redo_clear(uint4 *__restrict__ accum, const uint32_t *redo, uint32_t npix) {
    if (*redo == 0u) return;
    for (uint32_t p = blockIdx.x * kThreads + threadIdx.x; p < npix; p += gridDim.x * kThreads)
        accum[p] = make_uint4(0u, 0u, 0u, 0u);
}

// resolveUpdate with coverageEnabled (Resolve/Shaders.metal:24-41): the
// weighted-blended average sum(c a S) / sum(a S) and alpha 1 - e^-(sum a).
__global__ void __launch_bounds__(kThreads)
    resolve_coverage(const uint32_t *__restrict__ depth, const uint4 *__restrict__ accum,
                     uint32_t *__restrict__ rgba, float *__restrict__ depthf, uint32_t npix,
                     ResolveUniforms u) {
    const uint32_t p = blockIdx.x * kThreads + threadIdx.x;
    if (p >= npix) return;
    const uint4 acc = accum[p];
    if (acc.w == 0u) {
        rgba[p] = pack_rgba(u.background[0], u.background[1], u.background[2], 0.0f);
        depthf[p] = 0.0f;
        return;
    }
    const float fa = (float)acc.w;
    const float sum_a = fa * (1.0f / 4096.0f);
    const float alpha = fminf(fmaxf(1.0f - crd::exp_neg(sum_a), 0.0f), 1.0f);
    rgba[p] = pack_rgba((float)acc.x / fa, (float)acc.y / fa, (float)acc.z / fa, alpha);
    depthf[p] = crd::uint_to_depth(depth[p]);
}

// Zeroes the depth plane and the accumulators (with the redo word behind
// them) of an HQS frame in one launch of 16-byte stores.
__global__ void __launch_bounds__(kThreads)
    frame_clear(uint4 *depth4, size_t ndepth4, uint32_t *depth_tail, uint32_t ntail,
                uint4 *accum, size_t naccum) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < naccum; i += stride)
        accum[i] = z;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < ndepth4; i += stride)
        depth4[i] = z;
    if (blockIdx.x == 0 && threadIdx.x < ntail) depth_tail[threadIdx.x] = 0u;
}

// Top bit of every depth word flipped: unsigned order <-> signed order.
__global__ void __launch_bounds__(kThreads)
    flip_depth_order(uint4 *d4, size_t n4, uint32_t *tail, uint32_t ntail) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        uint4 v = d4[i];
        v.x ^= 0x80000000u;
        v.y ^= 0x80000000u;
        v.z ^= 0x80000000u;
        v.w ^= 0x80000000u;
        d4[i] = v;
    }
    if (blockIdx.x == 0 && threadIdx.x < ntail) tail[threadIdx.x] ^= 0x80000000u;
}

}  // namespace

cr_status launch_resolve_hqs(cr_frame *f, const ResolveUniforms &u, cudaStream_t s, bool check,
                             const uint32_t *redo) {
    const uint32_t npix = (uint32_t)f->width * (uint32_t)f->height;
    // A grid-stride grid of sixteen CTAs per SM at most (four pixels per
    // thread per step: one step covers a 1080p frame); the gated re-run
    // (rarely needed) uses four per SM so that skipping it costs little.
    const uint32_t full = (npix + 4 * kThreads - 1) / (4 * kThreads);
    const uint32_t grid =
        redo ? (uint32_t)f->ctx->sm_count * 4 : std::min(full, (uint32_t)f->ctx->sm_count * 16);
    CR_CUDA(launch_programmatic(resolve_hqs, dim3(grid), dim3(kThreads), 0, s,
                                (const uint32_t *)f->d_depth, (const uint4 *)f->d_accum,
                                f->d_rgba[0], f->d_depthf, npix, u, f->d_redo, check ? 1 : 0,
                                redo));
    CR_CUDA(cudaGetLastError());
    f->final_rgba = 0;
    return CR_OK;
}

FrameClear frame_clear_of(cr_frame *f) {
    const size_t npix = (size_t)f->width * (size_t)f->height;
    const size_t n4 = npix / 4;  // depth words in whole 16-byte groups (the plane is 256-byte aligned)
    return FrameClear{reinterpret_cast<uint4 *>(f->d_depth), n4, f->d_depth + 4 * n4,
                      (uint32_t)(npix - 4 * n4), f->d_accum, npix + 1};
}

cr_status launch_frame_clear(cr_frame *f, cudaStream_t s) {
    const FrameClear c = frame_clear_of(f);
    frame_clear<<<f->ctx->sm_count * 8, kThreads, 0, s>>>(c.depth4, c.ndepth4, c.tail, c.ntail,
                                                           c.accum, c.naccum);
    CR_CUDA(cudaGetLastError());
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

static uint32_t views_grid(uint32_t total_pix, int sm_count) {
    const uint32_t need = (total_pix + kThreads - 1) / kThreads;
    const uint32_t cap = (uint32_t)sm_count * 8u;
    return std::max<uint32_t>(1u, std::min(need, cap));
}

cr_status launch_clear_views(const ViewDesc *views, uint32_t nviews, uint32_t pix0, uint32_t npix,
                             uint32_t *redo_flag, bool zero_flag, int sm_count, cudaStream_t s) {
    clear_views<<<views_grid(npix, sm_count), kThreads, 0, s>>>(views, nviews, pix0, npix,
                                                                redo_flag, 0, zero_flag ? 1 : 0);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

cr_status launch_accum_redo_clear_views(const ViewDesc *views, uint32_t nviews,
                                        uint32_t total_pix, const uint32_t *redo_flag,
                                        int sm_count, cudaStream_t s) {
    clear_views<<<sm_count * 4, kThreads, 0, s>>>(views, nviews, 0, total_pix,
                                                  const_cast<uint32_t *>(redo_flag), 1, 0);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

cr_status launch_resolve_views(const ViewDesc *views, uint32_t nviews, uint32_t pix0,
                               uint32_t npix, const ResolveUniforms &u, uint32_t *redo_flag,
                               bool check, const uint32_t *redo, int sm_count, cudaStream_t s) {
    const uint32_t grid = redo ? (uint32_t)sm_count * 4 : views_grid(npix, sm_count);
    resolve_views<<<grid, kThreads, 0, s>>>(views, nviews, pix0, npix, u, redo_flag,
                                           check ? 1 : 0, redo);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

cr_status launch_hole_fill_views(const ViewDesc *views, uint32_t nviews, uint32_t total_pix,
                                 int src, int sm_count, cudaStream_t s) {
    hole_fill_views<<<views_grid(total_pix, sm_count), kThreads, 0, s>>>(views, nviews, total_pix,
                                                                         src);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

cr_status launch_resolve_f32(cr_frame *f, const float background[3], float *image,
                             cudaStream_t s) {
    const uint32_t npix = (uint32_t)f->width * (uint32_t)f->height;
    resolve_f32<<<views_grid(npix, f->ctx->sm_count), kThreads, 0, s>>>(
        f->d_fsum, f->d_fcount, image, npix, background[0], background[1], background[2]);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

cr_status launch_l2_loss(const float *image, const float *target, uint64_t n, float scale,
                         float *dldimg, double *loss, int sm_count, cudaStream_t s) {
    if (n == 0) return CR_OK;
    const uint64_t need = (n + kThreads - 1) / kThreads;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(need, (uint64_t)sm_count * 8);
    l2_loss<<<grid, kThreads, 0, s>>>(image, target, n, scale, dldimg, loss);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

cr_status launch_flip_depth_order(cr_frame *f, cudaStream_t s) {
    // The plane comes from cudaMalloc (256-byte aligned): 16-byte words, then
    // the last npix % 4 words.
    const size_t npix = (size_t)f->width * f->height;
    const size_t n4 = npix / 4;
    const uint32_t ntail = (uint32_t)(npix - 4 * n4);
    const uint32_t grid = (uint32_t)std::max<size_t>(
        1, std::min<size_t>((n4 + kThreads - 1) / kThreads, (size_t)f->ctx->sm_count * 8));
    flip_depth_order<<<grid, kThreads, 0, s>>>(reinterpret_cast<uint4 *>(f->d_depth), n4,
                                               f->d_depth + 4 * n4, ntail);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

cr_status launch_resolve_coverage(cr_frame *f, const ResolveUniforms &u, cudaStream_t s) {
    const uint32_t npix = (uint32_t)f->width * (uint32_t)f->height;
    resolve_coverage<<<(npix + kThreads - 1) / kThreads, kThreads, 0, s>>>(
        f->d_depth, f->d_accum, f->d_rgba[0], f->d_depthf, npix, u);
    CR_CUDA(cudaGetLastError());
    f->final_rgba = 0;
    return CR_OK;
}
