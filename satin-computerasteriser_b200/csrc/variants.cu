// HQS depth and colour passes with the colour variants on: per-point
// displacement, tint, translucent-defocus coverage and motion blur
// (DepthPass/Shaders.metal:56-71, ColorPass/Shaders.metal:54-199).
//
// The variants read per-point float4 attributes that user kernels write into
// the cloud's buffers (cr_cloud_attribute) before the frame: displacement
// (xyz added to the decoded position; a NaN component drops the point), the
// previous frame's displacement (motion blur), and tint (rgba: mixed into the
// colour with weight a; a < 0 drops the point; with tintAlphaIsCoverage,
// coverage = 1 - a for the weighted-blended accumulation).  A cloud without a
// buffer reads zeros, as the reference's zeroed stand-in.
//
// These passes keep the reference's per-point order and fixed point (S =
// 4096) and use plain 32-bit adds; they run one thread per point over the
// cull's chunk records, without the fragment hand-off and screen tiles of the
// default passes (raster.cu), which stay free of the variant branches.
#include "cr_device.cuh"
#include "cr_internal.h"

namespace {

constexpr int kThreads = 256;

struct VariantArgs {
    const ChunkRec *chunks;
    const uint32_t *counters;
    const uint32_t *low, *med, *high, *colors;
    const uint8_t *levels;
    const cr_raster_file *files;
    const float4 *disp, *prev_disp, *tint;  // null: zeros (prev_disp null: disp)
    uint32_t *depth;
    uint32_t *accum;  // R, G, B, count per pixel
    RasterUniforms u;
    float keep_scale;  // 1 - depthTolerance
    int apply_disp, apply_tint, coverage_mode;
    float motion_blur;
    int mb_samples;
    float mb_max_spread;
};

__device__ __forceinline__ float4 attr(const float4 *a, uint32_t i) {
    return a ? a[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

__device__ __forceinline__ float sat(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }  // NaN -> 0

__device__ __forceinline__ void red_add(uint32_t *p, uint32_t v) {
    asm volatile("red.global.add.u32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(v)
                 : "memory");
}

template <bool COLOR>
__global__ void __launch_bounds__(kThreads) variant_pass(VariantArgs a) {
    const uint32_t nchunks = a.counters[CNT_CHUNKS];
    const int W = a.u.width, H = a.u.height;
    const crd::PointSize ps{a.u.pointSizeMode, a.u.minimumPointSize, a.u.maximumPointSize,
                            a.u.pointSizeScale};
    const bool mb_on = a.motion_blur > 0.0f;
    const bool oit = a.coverage_mode || mb_on;
    for (uint32_t k = blockIdx.x; k < nchunks; k += gridDim.x) {
        const ChunkRec c = a.chunks[k];
        const cr_raster_file &file = a.files[c.file];
        const uint32_t sl = c.level == 0 ? 20u : (c.level == 1 ? 10u : 0u);
        const uint32_t sm = c.level == 0 ? 10u : 0u;
        for (uint32_t local = threadIdx.x; local < c.count; local += kThreads) {
            const uint32_t pi = c.first + local;
            // Dither keep test (DepthPass/Shaders.metal:52-55).
            const float level = (float)(a.levels[pi] & 7u);
            const float dither = a.u.lodDither ? crd::hash_unit(pi) : 0.5f;
            if (dither >= (c.thr - level) + 0.5f) continue;
            if (!COLOR && a.coverage_mode && attr(a.tint, pi).w < 0.0f) continue;
            const uint32_t lo = a.low[pi];
            const uint32_t me = c.level <= 1 ? a.med[pi] : 0u;
            const uint32_t hi = c.level == 0 ? a.high[pi] : 0u;
            const uint32_t x = ((lo & 1023u) << sl) | ((me & 1023u) << sm) | (hi & 1023u);
            const uint32_t y = (((lo >> 10) & 1023u) << sl) | (((me >> 10) & 1023u) << sm) |
                               ((hi >> 10) & 1023u);
            const uint32_t z = (((lo >> 20) & 1023u) << sl) | (((me >> 20) & 1023u) << sm) |
                               ((hi >> 20) & 1023u);
            const float bx = (float)x * c.qx + c.minX, by = (float)y * c.qy + c.minY,
                        bz = (float)z * c.qz + c.minZ;
            float px = bx, py = by, pz = bz;
            if (a.apply_disp) {
                const float4 d = attr(a.disp, pi);
                px = px + d.x;
                py = py + d.y;
                pz = pz + d.z;
                if (px != px || py != py || pz != pz) continue;
            }
            const crd::f4 clip = crd::mulp(file.transform, px, py, pz);
            if (clip.w <= 0.0f) continue;
            const float nx = clip.x / clip.w, ny = clip.y / clip.w, nz = clip.z / clip.w;
            if (nx < -1.0f || ny < -1.0f || nx > 1.0f || ny > 1.0f || nz < 0.0f || nz > 1.0f)
                continue;
            const int ix = (int)((nx * 0.5f + 0.5f) * (float)W);
            int iy = (int)((ny * 0.5f + 0.5f) * (float)H);
            if (ix < 0 || ix >= W || iy < 0 || iy >= H) continue;
            iy = H - 1 - iy;
            if (!COLOR) {
                const uint32_t depth = crd::depth_to_uint(nz);
                const int rad =
                    crd::footprint_radius(px, py, pz, file.world, a.u.view, a.u.proj, H, ps);
                for (int oy = -rad; oy <= rad; ++oy)
                    for (int ox = -rad; ox <= rad; ++ox) {
                        if (!crd::inside_footprint(ox, oy, rad)) continue;
                        const int tx = ix + ox, ty = iy + oy;
                        if (tx < 0 || tx >= W || ty < 0 || ty >= H) continue;
                        atomicMax(a.depth + (uint32_t)(ty * W + tx), depth);
                    }
                continue;
            }
            // Colour (ColorPass/Shaders.metal:95-140).
            uint32_t color = a.colors[pi];
            if (a.u.colorizeChunks)
                color = c.batchIndex * 1234567u;
            else if (a.u.colorizeOverdraw)
                color = 0x00010101u;
            uint32_t r = color & 0xffu, g = (color >> 8) & 0xffu, b = (color >> 16) & 0xffu;
            float cov = 1.0f;
            if (a.apply_tint) {
                const float4 t = attr(a.tint, pi);
                if (t.w < 0.0f) continue;
                if (a.coverage_mode) {
                    cov = sat(1.0f - t.w);
                } else {
                    const float w = sat(t.w), k255 = 1.0f / 255.0f;
                    const float ox = (float)r * k255, oy = (float)g * k255, oz = (float)b * k255;
                    const float mx = ox + (sat(t.x) - ox) * w;  // mix(orig, tint, w)
                    const float my = oy + (sat(t.y) - oy) * w;
                    const float mz = oz + (sat(t.z) - oz) * w;
                    r = __float2uint_rz(sat(mx) * 255.0f + 0.5f);
                    g = __float2uint_rz(sat(my) * 255.0f + 0.5f);
                    b = __float2uint_rz(sat(mz) * 255.0f + 0.5f);
                }
            }
            if (oit && cov <= 0.0f) continue;
            const int rad = crd::footprint_radius(px, py, pz, file.world, a.u.view, a.u.proj, H, ps);
            // Motion blur: smear back toward the previous screen position
            // (ColorPass/Shaders.metal:149-171).
            int samples = 1;
            float stepx = 0.0f, stepy = 0.0f;
            if (mb_on) {
                float qx = bx, qy = by, qz = bz;
                if (a.apply_disp) {
                    const float4 d = attr(a.prev_disp ? a.prev_disp : a.disp, pi);
                    qx = qx + d.x;
                    qy = qy + d.y;
                    qz = qz + d.z;
                }
                const crd::f4 pc = crd::mulp(file.prevTransform, qx, qy, qz);
                if (pc.w > 0.0f) {
                    const float pnx = pc.x / pc.w, pny = pc.y / pc.w;
                    const int ppx = (int)((pnx * 0.5f + 0.5f) * (float)W);
                    const int ppy = H - 1 - (int)((pny * 0.5f + 0.5f) * (float)H);
                    float vx = (float)((long long)ix - (long long)ppx) * a.motion_blur;
                    float vy = (float)((long long)iy - (long long)ppy) * a.motion_blur;
                    float len = sqrtf(vx * vx + vy * vy);
                    if (len > a.mb_max_spread) {
                        const float kk = a.mb_max_spread / len;
                        vx = vx * kk;
                        vy = vy * kk;
                        len = a.mb_max_spread;
                    }
                    if (len > 0.75f) {
                        samples = min(max((int)ceilf(len), 1), a.mb_samples);
                        samples = max(samples, 1);
                        const float den = (float)max(samples - 1, 1);
                        stepx = vx / den;
                        stepy = vy / den;
                    }
                }
            }
            const float aN = cov / (float)samples;
            const float kS = 4096.0f, k255 = 1.0f / 255.0f;
            const uint32_t caR = __float2uint_rz((((float)r * k255) * aN) * kS + 0.5f);
            const uint32_t caG = __float2uint_rz((((float)g * k255) * aN) * kS + 0.5f);
            const uint32_t caB = __float2uint_rz((((float)b * k255) * aN) * kS + 0.5f);
            const uint32_t caA = __float2uint_rz(aN * kS + 0.5f);
            for (int s = 0; s < samples; ++s) {
                const int cx = ix - (int)roundf(stepx * (float)s);
                const int cy = iy - (int)roundf(stepy * (float)s);
                for (int oy = -rad; oy <= rad; ++oy)
                    for (int ox = -rad; ox <= rad; ++ox) {
                        if (!crd::inside_footprint(ox, oy, rad)) continue;
                        const int tx = cx + ox, ty = cy + oy;
                        if (tx < 0 || tx >= W || ty < 0 || ty >= H) continue;
                        const uint32_t pix = (uint32_t)(ty * W + tx);
                        uint32_t *acc = a.accum + 4 * (size_t)pix;
                        if (oit) {
                            red_add(acc + 0, caR);
                            red_add(acc + 1, caG);
                            red_add(acc + 2, caB);
                            red_add(acc + 3, caA);
                            continue;
                        }
                        const uint32_t closest = a.depth[pix];
                        if (closest == 0u) continue;
                        if (!(nz >= crd::uint_to_depth(closest) * a.keep_scale)) continue;
                        red_add(acc + 0, r);
                        red_add(acc + 1, g);
                        red_add(acc + 2, b);
                        red_add(acc + 3, 1u);
                    }
            }
        }
    }
}

}  // namespace

cr_status launch_variant_pass(cr_cloud *cloud, bool color, const RasterUniforms &u,
                              const cr_config &cfg, const RasterTargets &t, cudaStream_t s) {
    // The variant passes read the device file table.
    if (const cr_status st = ensure_device_files(cloud)) return st;
    VariantArgs a;
    a.chunks = cloud->d_chunks;
    a.counters = cloud->d_counters;
    a.low = cloud->d_low;
    a.med = cloud->d_med;
    a.high = cloud->d_high;
    a.colors = cloud->d_colors;
    a.levels = cloud->d_levels;
    a.files = cloud->d_files;
    a.disp = cloud->d_disp;
    a.prev_disp = cloud->d_prev_disp;
    a.tint = cloud->d_tint;
    a.depth = t.depth;
    a.accum = reinterpret_cast<uint32_t *>(t.accum);
    a.u = u;
    a.keep_scale = 1.0f - u.depthTolerance;
    a.apply_disp = cfg.applyDisplacement ? 1 : 0;
    a.apply_tint = cfg.applyTint ? 1 : 0;
    a.coverage_mode = (cfg.applyTint && cfg.tintAlphaIsCoverage) ? 1 : 0;
    a.motion_blur = cfg.motionBlur > 0.0f ? cfg.motionBlur : 0.0f;
    a.mb_samples = cfg.motionBlurSamples;
    a.mb_max_spread = cfg.motionBlurMaxSpread;
    const int grid = cloud->ctx->sm_count * 8;
    if (color)
        variant_pass<true><<<grid, kThreads, 0, s>>>(a);
    else
        variant_pass<false><<<grid, kThreads, 0, s>>>(a);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}
