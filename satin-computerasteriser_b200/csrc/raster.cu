// raster.cu — the per-point passes of the compute rasteriser.
//
//   PASS_DEPTH   depthPassUpdate   (Pipelines/DepthPass/Shaders.metal:21-116)
//   PASS_COLOR   colorPassUpdate   (Pipelines/ColorPass/Shaders.metal:30-219,
//                                   integer R,G,B,count path)
//   PASS_NEAREST nearestDepthUpdate + nearestIndexUpdate
//                (Pipelines/NearestDepth/Shaders.metal:14-91,
//                 Pipelines/NearestIndex/Shaders.metal:14-94) fused into one
//                traversal: the key (depth << 32) | ~pointIndex is combined
//                with a 64-bit max, so the winner is the largest depth and,
//                among equal depths, the lowest point index — the same pixel
//                result as the reference's max pass followed by its
//                min-index pass over the tied points.
//
// Launch shape.  The reference dispatches one 128-thread group per survivor
// of the cull (indirect dispatch).  Here the cull also cuts every survivor's
// point prefix into chunk records of at most `chunkPoints` points carrying
// the per-batch decode values and screen rectangle, and publishes their
// count (the CUDA counterpart of the indirect argument buffer).  A
// persistent grid sized to fill every SM claims the records from a work
// cursor, copying the next record into shared memory (cp.async) while the
// current chunk is processed, so batches of very different sizes spread
// evenly over the SMs.  Each CTA of 256 threads walks a chunk four points
// per thread with 16-byte loads of the level bytes and position / colour
// words; warps skip the projection and the atomics when none of their lanes
// survives the dither or clip tests, and a chunk whose LOD threshold keeps
// every level skips the dither hash.
//
// Screen tiles.  A batch is Morton-compact, so its points land in a small
// screen rectangle (the projection of its AABB's eight corners, widened by
// two pixels, computed by the cull).  When that rectangle has few pixels per
// point, the CTA
// accumulates in shared memory — depth max, or R | count << 20, G and B (a
// chunk of fewer than 4096 points keeps every field below its width), or
// the nearest key — and then flushes one global atomic per touched pixel.  The colour pass
// also stages the rectangle's settled depths in shared memory.  Points that
// round outside the rectangle use global atomics directly, so the tile is a
// cache and never changes a result.  Other batches, large on screen with
// few points per pixel, use one global atomic per point.  Atomics are
// predicated single instructions rather than branches around code.
// Integer max and sum are associative and commutative: the planes are
// bit-identical to a per-point atomic order either way.
#include "cr_bulk.cuh"
#include "cr_device.cuh"
#include "cr_internal.h"
#include "cr_resolve.cuh"

#ifndef CR_TILE_REJECT
#define CR_TILE_REJECT 0
#endif
#ifndef CR_DIV64
#define CR_DIV64 0
#endif
#ifndef CR_TILE_PX_PER_POINT
#define CR_TILE_PX_PER_POINT 1
#endif

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kFull = 0xffffffffu;

template <int PASS>
struct TileCfg;
template <>
struct TileCfg<PASS_DEPTH> {
    static constexpr int kPx = 8192;
    static constexpr int kBytes = kPx * 4;
};
template <>
struct TileCfg<PASS_COLOR> {
    static constexpr int kPx = 4096;
    static constexpr int kBytes = kPx * 16;  // R|count, G, B accumulators + settled depth
};
template <>
struct TileCfg<PASS_NEAREST> {
    static constexpr int kPx = 4096;
    static constexpr int kBytes = kPx * 8;
};

// The depth pass that writes fragments keeps two words per tile pixel: the
// running maximum (seeded with the frame's depth plane) and the plane value
// it was seeded with, so that the flush writes back only raised pixels.
#ifndef CR_BULK_STAGE
#define CR_BULK_STAGE 0
#endif
template <>
struct TileCfg<PASS_DEPTH_FRAG> {
    static constexpr int kPx = 4096;
    static constexpr int kTileBytes = kPx * (CR_TILE_REJECT ? 8 : 4);
    static constexpr int kBytes = kTileBytes + (CR_BULK_STAGE ? 2 * 2048 * 9 : 0);  // + stage buffers
};
template <>
struct TileCfg<PASS_COLOR_FRAG> : TileCfg<PASS_COLOR> {};
template <>
struct TileCfg<PASS_COLOR_F32> {  // no screen tiles
    static constexpr int kPx = 0;
    static constexpr int kBytes = 0;
};
template <>
struct TileCfg<PASS_GRAD> : TileCfg<PASS_COLOR_F32> {};

__host__ __device__ constexpr bool is_depth(int p) { return p == PASS_DEPTH || p == PASS_DEPTH_FRAG; }
__host__ __device__ constexpr bool is_color(int p) { return p == PASS_COLOR || p == PASS_COLOR_FRAG; }

struct RasterArgs {
    const ChunkRec *chunks;
    const cr_raster_file *files;
    InlineFiles ifiles;  // the one-view file table, when small (else ifiles.n = 0)
    uint32_t *counters;
    const uint32_t *low, *med, *high, *colors;
    const uint8_t *levels;
    RasterTargets t;
    RasterUniforms u;
    float keep_scale;  // 1 - depthTolerance
    int radius_zero;   // every footprint is a single pixel
    int use_tiles;
    uint32_t *frag_xy;  // pixel x | row << 16
    uint2 *frag_zc;     // NDC z bits, RGBA8: two stores per fragment
    uint32_t *frag_count;
    // Differentiable colours: learnable colours, dL/dpixel, gradient (3 floats each).
    const float *fcolors;
    const float *dldimg;
    float *fgrad;
    // Batched views (MV kernels): per-view frames, culls and file tables.
    const ViewDesc *views;
    uint32_t nviews;
    uint32_t nfiles;        // files per view; view v's table starts at files + v * nfiles
    uint32_t chunk_stride;  // view v's chunk records start at chunks + v * chunk_stride
    // Batched views with fragments: chunk record -> offset in its view's
    // fragment span; the arena's capacity; set by the depth pass when the
    // views' spans do not fit (the colour pass then decodes the points).
    const uint32_t *chunk_poff;
    unsigned long long frag_cap;
    uint32_t *frag_overflow;
    uint32_t *status;  // the context's device-side status word
};

// The frame and camera of the view whose chunk a CTA is drawing (MV kernels).
struct ViewState {
    int width, height;
    uint32_t *depth;
    uint4 *accum;
    unsigned long long *nearest;
    float view[16], proj[16];
};
__shared__ ViewState s_view;

// Frame and camera of the point being drawn: the kernel's own (one view) or
// the current chunk's view (batched views).
template <bool MV>
__device__ __forceinline__ int view_w(const RasterArgs &a) { return MV ? s_view.width : a.u.width; }
template <bool MV>
__device__ __forceinline__ int view_h(const RasterArgs &a) { return MV ? s_view.height : a.u.height; }
template <bool MV>
__device__ __forceinline__ uint32_t *view_depth(const RasterArgs &a) {
    return MV ? s_view.depth : a.t.depth;
}
template <bool MV>
__device__ __forceinline__ uint4 *view_accum(const RasterArgs &a) {
    return MV ? s_view.accum : a.t.accum;
}
template <bool MV>
__device__ __forceinline__ unsigned long long *view_nearest(const RasterArgs &a) {
    return MV ? s_view.nearest : a.t.nearest;
}
template <bool MV>
__device__ __forceinline__ const float *view_view(const RasterArgs &a) {
    return MV ? s_view.view : a.u.view;
}
template <bool MV>
__device__ __forceinline__ const float *view_proj(const RasterArgs &a) {
    return MV ? s_view.proj : a.u.proj;
}

// The current view's size and planes in registers: read once per chunk, not
// per point (loads from shared memory could not be hoisted past the
// shared-memory atomics); for one view, the kernel's own parameters.
template <bool MV>
struct ViewRegsT;
template <>
struct ViewRegsT<true> {
    int W, H;
    uint32_t *depth;
    uint4 *accum;
    unsigned long long *nearest;
};
template <>
struct ViewRegsT<false> {  // reads the kernel parameters where used
    const RasterArgs &a;
    __device__ __forceinline__ ViewRegsT(const RasterArgs &args) : a(args) {}
};
template <bool MV>
__device__ __forceinline__ int vw(const ViewRegsT<MV> &r);
template <>
__device__ __forceinline__ int vw<true>(const ViewRegsT<true> &r) { return r.W; }
template <>
__device__ __forceinline__ int vw<false>(const ViewRegsT<false> &r) { return r.a.u.width; }
template <bool MV>
__device__ __forceinline__ int vh(const ViewRegsT<MV> &r);
template <>
__device__ __forceinline__ int vh<true>(const ViewRegsT<true> &r) { return r.H; }
template <>
__device__ __forceinline__ int vh<false>(const ViewRegsT<false> &r) { return r.a.u.height; }
template <bool MV>
__device__ __forceinline__ uint32_t *vdepth(const ViewRegsT<MV> &r);
template <>
__device__ __forceinline__ uint32_t *vdepth<true>(const ViewRegsT<true> &r) { return r.depth; }
template <>
__device__ __forceinline__ uint32_t *vdepth<false>(const ViewRegsT<false> &r) { return r.a.t.depth; }
template <bool MV>
__device__ __forceinline__ uint4 *vaccum(const ViewRegsT<MV> &r);
template <>
__device__ __forceinline__ uint4 *vaccum<true>(const ViewRegsT<true> &r) { return r.accum; }
template <>
__device__ __forceinline__ uint4 *vaccum<false>(const ViewRegsT<false> &r) { return r.a.t.accum; }
template <bool MV>
__device__ __forceinline__ unsigned long long *vnearest(const ViewRegsT<MV> &r);
template <>
__device__ __forceinline__ unsigned long long *vnearest<true>(const ViewRegsT<true> &r) {
    return r.nearest;
}
template <>
__device__ __forceinline__ unsigned long long *vnearest<false>(const ViewRegsT<false> &r) {
    return r.a.t.nearest;
}
__device__ __forceinline__ ViewRegsT<true> view_regs_mv() {
    return ViewRegsT<true>{s_view.width, s_view.height, s_view.depth, s_view.accum,
                           s_view.nearest};
}

struct BatchShared {
    float T[16];      // file.transform
    float world[16];  // file.world (footprint only)
    uint32_t file;    // file cached in T / world
};

struct PointOut {
    bool ok;
    bool doomed;  // depth pass: the fragment cannot pass the colour pass's depth test
    int ix, iy;  // pixel after the y flip
    uint32_t depth;
    float nz;
    uint32_t color;
    uint32_t pointIndex;
    float px, py, pz;
};

// Dither keep-test of one point (DepthPass/Shaders.metal:174-179).
__device__ __forceinline__ bool keep_point(const RasterArgs &a, const ChunkRec &c,
                                           uint32_t pointIndex, uint32_t lvl) {
    const float pointLevel = (float)(lvl & 7u);
    const float dither = a.u.lodDither ? crd::hash_unit(pointIndex) : 0.5f;
    return !(dither >= (c.thr - pointLevel) + 0.5f);
}

// decodePoint + projection + clip + pixel (DepthPass/Shaders.metal:188-211,
// ColorPass/Shaders.metal:70-104, NearestDepth/Shaders.metal:68-85).
template <int PASS, bool MV>
__device__ __forceinline__ void project_point(const RasterArgs &a, const ViewRegsT<MV> &vr, const BatchShared &sb,
                                              const ChunkRec &c, uint32_t lo, uint32_t me,
                                              uint32_t hi, PointOut &o) {
    // Split-precision decode: the coarse (low), medium and fine (high) 10-bit
    // chunks for level >= 2 (10 bits), level 1 (20 bits) or level 0 (30
    // bits).  A word the chunk's level does not use was never loaded and is
    // zero; the level is the same for the whole chunk, so the branch is
    // uniform and each level does only its own shifts.
    uint32_t x, y, z;
    if (c.level >= 2) {
        x = lo & 1023u;
        y = (lo >> 10) & 1023u;
        z = (lo >> 20) & 1023u;
    } else if (c.level == 1) {
        x = ((lo & 1023u) << 10) | (me & 1023u);
        y = (((lo >> 10) & 1023u) << 10) | ((me >> 10) & 1023u);
        z = (((lo >> 20) & 1023u) << 10) | ((me >> 20) & 1023u);
    } else {
        const uint32_t sl = c.level == 0 ? 20u : 0u, sm = c.level == 0 ? 10u : 0u;
        x = ((lo & 1023u) << sl) | ((me & 1023u) << sm) | (hi & 1023u);
        y = (((lo >> 10) & 1023u) << sl) | (((me >> 10) & 1023u) << sm) | ((hi >> 10) & 1023u);
        z = (((lo >> 20) & 1023u) << sl) | (((me >> 20) & 1023u) << sm) | ((hi >> 20) & 1023u);
    }
    o.px = (float)x * c.qx + c.minX;
    o.py = (float)y * c.qy + c.minY;
    o.pz = (float)z * c.qz + c.minZ;
    const crd::f4 clip = crd::mulp(sb.T, o.px, o.py, o.pz);
    bool ok = o.ok;
    if (clip.w <= 0.0f) ok = false;
#if CR_DIV64
    float nx, ny, nz;
    crd::div3_shared(clip.x, clip.y, clip.z, clip.w, nx, ny, nz);
#else
    const float nx = clip.x / clip.w, ny = clip.y / clip.w, nz = clip.z / clip.w;
#endif
    // |x| > 1 is x < -1 || x > 1 for every float (false for NaN either way).
    if (fabsf(nx) > 1.0f || fabsf(ny) > 1.0f || nz > 1.0f) ok = false;
    if (PASS == PASS_NEAREST ? (nz <= 0.0f) : (nz < 0.0f)) ok = false;
    const int W = vw<MV>(vr), H = vh<MV>(vr);
    o.ix = (int)((nx * 0.5f + 0.5f) * (float)W);
    const int iy = (int)((ny * 0.5f + 0.5f) * (float)H);
    if (o.ix < 0 || o.ix >= W || iy < 0 || iy >= H) ok = false;
    o.iy = H - 1 - iy;
    // depth_to_uint without its clamps: the saturating conversion already
    // maps z * 2^32 to 0 for z <= 0 or NaN and to 0xFFFFFFFF for z >= 1.
    o.depth = __float2uint_rz(nz * 4294967296.0f);
    o.nz = nz;
    o.ok = ok;
    if (PASS == PASS_COLOR || PASS == PASS_DEPTH_FRAG) {  // ColorPass/Shaders.metal:95-100
        if (a.u.colorizeChunks)
            o.color = c.batchIndex * 1234567u;
        else if (a.u.colorizeOverdraw)
            o.color = 0x00010101u;
    }
}

__device__ __forceinline__ unsigned long long nearest_key(uint32_t depth, uint32_t index) {
    return ((unsigned long long)depth << 32) | (unsigned long long)(~index);
}


// Reductions into the frame planes (global memory).  Written as red.global
// on explicitly global addresses: the batched-view passes take the plane
// pointers from shared memory, where the compiler cannot tell their
// address space, and would otherwise emit generic atomics that wait for a
// returned value.
__device__ __forceinline__ void red_add_u32(uint32_t *p, uint32_t v) {
    asm volatile("red.global.add.u32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(v)
                 : "memory");
}
__device__ __forceinline__ void red_add_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v)
                 : "memory");
}
__device__ __forceinline__ void red_max_u32(uint32_t *p, uint32_t v) {
    asm volatile("red.global.max.u32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(v)
                 : "memory");
}
__device__ __forceinline__ uint32_t atom_max_u32(uint32_t *p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.global.max.u32 %0, [%1], %2;"
                 : "=r"(old)
                 : "l"(__cvta_generic_to_global(p)), "r"(v)
                 : "memory");
    return old;
}
__device__ __forceinline__ void red_max_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("red.global.max.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v)
                 : "memory");
}

__device__ __forceinline__ void red_add_f32x3(float4 *p, float r, float g, float b) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(
                     __cvta_generic_to_global(p)),
                 "f"(r), "f"(g), "f"(b), "f"(0.0f)
                 : "memory");
}

// Differentiable colours, one visible (point, pixel): the forward adds the
// point's FP32 colour and one sample; the adjoint adds dL/dpixel / count to
// the point's gradient (g, in registers, written once per point).
__device__ __forceinline__ void color_f32_sample(const RasterArgs &a, uint32_t pix,
                                                 uint32_t pointIndex) {
    const float *c = a.fcolors + 3 * (size_t)pointIndex;
    red_add_f32x3(a.t.fsum + pix, c[0], c[1], c[2]);
    red_add_u32(a.t.fcount + pix, 1u);
}
__device__ __forceinline__ void grad_sample(const RasterArgs &a, uint32_t pix, float g[3]) {
    const float n = (float)a.t.fcount[pix];
    const float *d = a.dldimg + 3 * (size_t)pix;
    g[0] = g[0] + d[0] / n;
    g[1] = g[1] + d[1] / n;
    g[2] = g[2] + d[2] / n;
}
__device__ __forceinline__ void grad_store(const RasterArgs &a, uint32_t pointIndex,
                                           const float g[3]) {
    float *o = a.fgrad + 3 * (size_t)pointIndex;
    o[0] = o[0] + g[0];
    o[1] = o[1] + g[1];
    o[2] = o[2] + g[2];
}

// Adds one sample group to a pixel's R, G, B and count.  Packed: the uint4
// as two 64-bit words, R | G << 32 and B | count << 32 — half the global
// atomics.  A lower field that passes 2^32 would carry into its neighbour;
// that needs more than kPackedMaxCount samples in the pixel, which the
// resolve detects (the frame is then re-run unpacked).  Unpacked: one
// 32-bit add per field.
template <bool MV>
__device__ __forceinline__ void color_global(const RasterArgs &a, const ViewRegsT<MV> &vr, uint32_t pix, uint32_t r,
                                             uint32_t g, uint32_t b, uint32_t n) {
    if (a.t.packed) {
        unsigned long long *w = reinterpret_cast<unsigned long long *>(&vaccum<MV>(vr)[pix]);
        red_add_u64(w, (unsigned long long)r | ((unsigned long long)g << 32));
        red_add_u64(w + 1, (unsigned long long)b | ((unsigned long long)n << 32));
    } else {
        unsigned int *acc = reinterpret_cast<unsigned int *>(&vaccum<MV>(vr)[pix]);
        red_add_u32(acc + 0, r);
        red_add_u32(acc + 1, g);
        red_add_u32(acc + 2, b);
        red_add_u32(acc + 3, n);
    }
}

// Direct path, radius 0: one global atomic per point (batches large on
// screen, where points rarely share a pixel).
#ifndef CR_DIRECT_EARLY_REJECT
#define CR_DIRECT_EARLY_REJECT 0
#endif
template <int PASS, bool MV>
__device__ __forceinline__ void emit_direct(const RasterArgs &a, const ViewRegsT<MV> &vr, PointOut &o) {
    const uint32_t pix = (uint32_t)(o.iy * vw<MV>(vr) + o.ix);
    if (PASS == PASS_DEPTH_FRAG && CR_DIRECT_EARLY_REJECT) {
        uint32_t seen = 0u;
        if (o.ok) seen = atom_max_u32(&vdepth<MV>(vr)[pix], o.depth);
        o.doomed = o.nz < crd::uint_to_depth(seen) * a.keep_scale;
    } else if (is_depth(PASS)) {
        if (o.ok) red_max_u32(&vdepth<MV>(vr)[pix], o.depth);
    } else if (is_color(PASS)) {
        const uint32_t closest = o.ok ? vdepth<MV>(vr)[pix] : 0u;
        const bool vis = closest != 0u && o.nz >= crd::uint_to_depth(closest) * a.keep_scale;
        if (vis)
            color_global<MV>(a, vr, pix, o.color & 0xffu, (o.color >> 8) & 0xffu, (o.color >> 16) & 0xffu,
                         1u);
    } else if (PASS == PASS_COLOR_F32 || PASS == PASS_GRAD) {
        const uint32_t closest = o.ok ? vdepth<MV>(vr)[pix] : 0u;
        const bool vis = closest != 0u && o.nz >= crd::uint_to_depth(closest) * a.keep_scale;
        if (PASS == PASS_COLOR_F32 && vis) color_f32_sample(a, pix, o.pointIndex);
        if (PASS == PASS_GRAD && vis) {
            float g[3] = {0.0f, 0.0f, 0.0f};
            grad_sample(a, pix, g);
            grad_store(a, o.pointIndex, g);
        }
    } else {
        if (o.ok) red_max_u64(&vnearest<MV>(vr)[pix], nearest_key(o.depth, o.pointIndex));
    }
}

// Tile path, radius 0: shared-memory accumulation, global atomics for points
// that round outside the rectangle.  Colour tiles hold R | count << 20, G and
// B per pixel in 32-bit words (exact while a chunk has at most 4095 points).
//
// Depth pass with fragments: the tile starts from the frame's depth plane, so
// the value a point's shared max returns is a lower bound of the pixel's
// final depth (depths only grow during the pass).  The colour pass keeps a
// fragment iff z >= uint_to_depth(final) * (1 - tolerance), which is
// monotone in the depth word for a positive factor (and true for every
// fragment when the factor is not positive), so a fragment with
// z < uint_to_depth(running maximum) * (1 - tolerance) fails it with the
// final depth too and is not written (o.doomed).
template <int PASS, bool MV>
__device__ __forceinline__ void emit_tile(const RasterArgs &a, const ViewRegsT<MV> &vr, const ChunkRec &c,
                                          unsigned char *smem, PointOut &o) {
    const int lx = o.ix - c.x0, ly = o.iy - c.y0;
    const bool inside = (unsigned)lx < (unsigned)c.tw && (unsigned)ly < (unsigned)c.th;
    const bool in_tile = o.ok && inside, outside = o.ok && !inside;
    const uint32_t pix = (uint32_t)(o.iy * vw<MV>(vr) + o.ix);
    const int l = inside ? ly * c.tw + lx : 0;
    if (PASS == PASS_DEPTH_FRAG && CR_TILE_REJECT) {
        uint32_t seen = 0u;
        if (in_tile) seen = atomicMax(reinterpret_cast<uint32_t *>(smem) + l, o.depth);
        if (outside) red_max_u32(&vdepth<MV>(vr)[pix], o.depth);
        o.doomed = o.nz < crd::uint_to_depth(seen) * a.keep_scale;
    } else if (is_depth(PASS)) {
        if (in_tile) atomicMax(reinterpret_cast<uint32_t *>(smem) + l, o.depth);
        if (outside) red_max_u32(&vdepth<MV>(vr)[pix], o.depth);
    } else if (is_color(PASS)) {
        constexpr int kPx = TileCfg<PASS_COLOR>::kPx;
        uint32_t *acc = reinterpret_cast<uint32_t *>(smem);
        const uint32_t *sdep = acc + 3 * kPx;
        uint32_t closest = sdep[l];
        if (outside) closest = vdepth<MV>(vr)[pix];
        const bool vis = o.ok && closest != 0u &&
                         o.nz >= crd::uint_to_depth(closest) * a.keep_scale;
        const uint32_t r = o.color & 0xffu, g = (o.color >> 8) & 0xffu,
                       b = (o.color >> 16) & 0xffu;
        if (vis && inside) {
            atomicAdd(acc + l, r | (1u << 20));
            atomicAdd(acc + kPx + l, g);
            atomicAdd(acc + 2 * kPx + l, b);
        }
        if (vis && !inside) color_global<MV>(a, vr, pix, r, g, b, 1u);
    } else {
        const unsigned long long k = nearest_key(o.depth, o.pointIndex);
        if (in_tile) atomicMax(reinterpret_cast<unsigned long long *>(smem) + l, k);
        if (outside) red_max_u64(&vnearest<MV>(vr)[pix], k);
    }
}

// General footprint (radius from pointFootprintRadius), global atomics.
template <int PASS, bool MV>
__device__ __forceinline__ void emit_footprint(const RasterArgs &a, const ViewRegsT<MV> &vr, const BatchShared &sb,
                                               const PointOut &o) {
    if (!o.ok) return;
    const crd::PointSize ps{a.u.pointSizeMode, a.u.minimumPointSize, a.u.maximumPointSize,
                            a.u.pointSizeScale};
    const int rad =
        crd::footprint_radius(o.px, o.py, o.pz, sb.world, view_view<MV>(a), view_proj<MV>(a), vh<MV>(vr), ps);
    const int W = vw<MV>(vr), H = vh<MV>(vr);
    float g[3] = {0.0f, 0.0f, 0.0f};  // PASS_GRAD
    for (int oy = -rad; oy <= rad; ++oy) {
        for (int ox = -rad; ox <= rad; ++ox) {
            if (!crd::inside_footprint(ox, oy, rad)) continue;
            const int tx = o.ix + ox, ty = o.iy + oy;
            if (tx < 0 || tx >= W || ty < 0 || ty >= H) continue;
            const uint32_t pix = (uint32_t)(ty * W + tx);
            if (is_depth(PASS)) {
                red_max_u32(&vdepth<MV>(vr)[pix], o.depth);
            } else if (is_color(PASS) || PASS == PASS_COLOR_F32 || PASS == PASS_GRAD) {
                const uint32_t closest = vdepth<MV>(vr)[pix];
                if (closest == 0u) continue;
                if (!(o.nz >= crd::uint_to_depth(closest) * a.keep_scale)) continue;
                if (PASS == PASS_COLOR_F32)
                    color_f32_sample(a, pix, o.pointIndex);
                else if (PASS == PASS_GRAD)
                    grad_sample(a, pix, g);
                else
                    color_global<MV>(a, vr, pix, o.color & 0xffu, (o.color >> 8) & 0xffu,
                                     (o.color >> 16) & 0xffu, 1u);
            } else {
                red_max_u64(&vnearest<MV>(vr)[pix], nearest_key(o.depth, o.pointIndex));
            }
        }
    }
    if (PASS == PASS_GRAD) grad_store(a, o.pointIndex, g);
}

// Shared count of the fragments the current chunk has kept.
__shared__ uint32_t s_frag_count;

// Appends the warp's kept points to the chunk's fragment range [fbase, fbase+n):
// one shared-memory atomic per warp, lanes placed by ballot rank.
__device__ __forceinline__ void emit_fragment(const RasterArgs &a, uint32_t fbase,
                                              const PointOut &o) {
    const bool keep = o.ok && !o.doomed;
    const uint32_t ballot = __ballot_sync(kFull, keep);
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&s_frag_count, __popc(ballot));
    base = __shfl_sync(kFull, base, 0);
    if (keep) {
        const uint32_t i = fbase + base + __popc(ballot & ((1u << lane) - 1u));
        a.frag_xy[i] = (uint32_t)o.ix | ((uint32_t)o.iy << 16);
        a.frag_zc[i] = make_uint2(__float_as_uint(o.nz), o.color);
    }
}

// A point's fragment, held back so that several points of a thread are
// appended with one shared-memory atomic per warp.  Two points per atomic:
// the one-view depth pass 212 -> 207 µs on the 100M-point 1080p frames;
// four spill registers and were slower, and so does the batched-view kernel
// with two.
struct Frag {
    bool keep;
    uint32_t xy;
    float z;
    uint32_t col;
};
#ifndef CR_FRAG_BATCH
#define CR_FRAG_BATCH 2
#endif

// Appends N fragments per lane: one ballot per fragment, one atomic per warp.
template <int N>
__device__ __forceinline__ void emit_fragments(const RasterArgs &a, uint32_t fbase,
                                               const Frag (&f)[N]) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t b[N], tot = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        b[k] = __ballot_sync(kFull, f[k].keep);
        tot += __popc(b[k]);
    }
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&s_frag_count, tot);
    base = __shfl_sync(kFull, base, 0);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        if (f[k].keep) {
            const uint32_t i = fbase + base + __popc(b[k] & lt);
            a.frag_xy[i] = f[k].xy;
            a.frag_zc[i] = make_uint2(__float_as_uint(f[k].z), f[k].col);
        }
        base += __popc(b[k]);
    }
}

// One point; every lane of the warp calls this (warp-uniform early outs).
// With fo, the depth pass's fragment is returned there instead of appended.
template <int PASS, bool MV>
__device__ __forceinline__ void do_point(const RasterArgs &a, const ViewRegsT<MV> &vr, const BatchShared &sb,
                                         unsigned char *smem, const ChunkRec &c, bool tiled,
                                         bool valid, uint32_t local, uint32_t lvl, uint32_t lo,
                                         uint32_t me, uint32_t hi, uint32_t color, uint32_t fbase,
                                         bool emit, bool all_keep, Frag *fo = nullptr) {
    PointOut o;
    o.pointIndex = c.first + local;
    o.color = color;
    o.ok = valid;
    o.doomed = false;
    if (!all_keep) o.ok = o.ok && keep_point(a, c, o.pointIndex, lvl);
    // The depth passes keep nearly every point, so a warp vote to skip the
    // projection or the emission would cost more than it saves (the
    // emission is correct for a warp with no kept point).
    if (!is_depth(PASS) && !__any_sync(kFull, o.ok)) return;
    project_point<PASS, MV>(a, vr, sb, c, lo, me, hi, o);
    if (!is_depth(PASS) && !__any_sync(kFull, o.ok)) return;
    if (!a.radius_zero)
        emit_footprint<PASS, MV>(a, vr, sb, o);
    else if (tiled)
        emit_tile<PASS, MV>(a, vr, c, smem, o);
    else
        emit_direct<PASS, MV>(a, vr, o);
    if (PASS == PASS_DEPTH_FRAG && emit) {
        if (fo) {
            fo->keep = o.ok && !o.doomed;
            fo->xy = (uint32_t)o.ix | ((uint32_t)o.iy << 16);
            fo->z = o.nz;
            fo->col = o.color;
        } else {
            emit_fragment(a, fbase, o);
        }
    }
}

// One fragment of the colour pass (PASS_COLOR_FRAG); every lane calls this.
template <bool MV>
__device__ __forceinline__ void do_fragment(const RasterArgs &a, const ViewRegsT<MV> &vr, unsigned char *smem,
                                            const ChunkRec &c, bool tiled, bool valid,
                                            uint32_t xy, float nz, uint32_t color) {
    PointOut o;
    o.ok = valid;
    o.doomed = false;
    o.ix = (int)(xy & 0xffffu);
    o.iy = (int)(xy >> 16);
    o.nz = nz;
    o.color = color;
    if (tiled)
        emit_tile<PASS_COLOR_FRAG, MV>(a, vr, c, smem, o);
    else
        emit_direct<PASS_COLOR_FRAG, MV>(a, vr, o);
}

// Four fragments of one thread in the colour pass, the first `nvalid` of
// them real.  The settled depths of all four pixels are read (read-only
// path, or the tile's staged copy) before any accumulation, so the thread
// waits for one L2 round trip per quad instead of one per fragment.
template <bool MV>
__device__ __forceinline__ void color_quad(const RasterArgs &a, const ViewRegsT<MV> &vr, unsigned char *smem,
                                           const ChunkRec &c, bool tiled, uint32_t nvalid,
                                           const uint4 &xy4, const float4 &z4, const uint4 &co4) {
    constexpr int kPx = TileCfg<PASS_COLOR>::kPx;
    uint32_t *acc = reinterpret_cast<uint32_t *>(smem);
    const uint32_t *sdep = acc + 3 * kPx;
    const uint32_t xy[4] = {xy4.x, xy4.y, xy4.z, xy4.w};
    const float nz[4] = {z4.x, z4.y, z4.z, z4.w};
    const uint32_t col[4] = {co4.x, co4.y, co4.z, co4.w};
    uint32_t pix[4], closest[4];
    int l[4];
    bool in[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int ix = (int)(xy[i] & 0xffffu), iy = (int)(xy[i] >> 16);
        pix[i] = (uint32_t)(iy * vw<MV>(vr) + ix);
        const int lx = ix - c.x0, ly = iy - c.y0;
        in[i] = tiled && (unsigned)lx < (unsigned)c.tw && (unsigned)ly < (unsigned)c.th;
        l[i] = in[i] ? ly * c.tw + lx : 0;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        closest[i] = 0u;
        if ((uint32_t)i < nvalid) closest[i] = in[i] ? sdep[l[i]] : __ldg(vdepth<MV>(vr) + pix[i]);
    }
    // Consecutive visible fragments of the quad on the same pixel (neighbour
    // points of a Morton-ordered batch often share one) are summed in
    // registers and added once: fewer adds to a contended address.
    uint32_t rr = 0, gg = 0, bb = 0, nn = 0, cur = 0xffffffffu;
    bool cin = false;
    int cl = 0;
    auto flush = [&]() {
        if (nn == 0u) return;
        if (cin) {
            atomicAdd(acc + cl, rr | (nn << 20));
            atomicAdd(acc + kPx + cl, gg);
            atomicAdd(acc + 2 * kPx + cl, bb);
        } else {
            color_global<MV>(a, vr, cur, rr, gg, bb, nn);
        }
    };
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const bool vis = closest[i] != 0u && nz[i] >= crd::uint_to_depth(closest[i]) * a.keep_scale;
        if (!vis) continue;
        if (pix[i] != cur) {
            flush();
            cur = pix[i];
            cin = in[i];
            cl = l[i];
            rr = gg = bb = nn = 0u;
        }
        rr += col[i] & 0xffu;
        gg += (col[i] >> 8) & 0xffu;
        bb += (col[i] >> 16) & 0xffu;
        nn += 1u;
    }
    flush();
}

template <int PASS, bool MV>
__device__ __forceinline__ void tile_init(const RasterArgs &a, const ChunkRec &c,
                                          unsigned char *smem) {
    const int n = c.tw * c.th;
    for (int l = threadIdx.x; l < n; l += kThreads) {
        if (PASS == PASS_DEPTH_FRAG && CR_TILE_REJECT) {
            // Running maximum and seed: the plane's current value (a lower
            // bound of the final depth; any earlier value of this frame is one).
            constexpr int kPx = TileCfg<PASS_DEPTH_FRAG>::kPx;
            const int gx = c.x0 + l % c.tw, gy = c.y0 + l / c.tw;
            const uint32_t d = view_depth<MV>(a)[gy * view_w<MV>(a) + gx];
            reinterpret_cast<uint32_t *>(smem)[l] = d;
            reinterpret_cast<uint32_t *>(smem)[kPx + l] = d;
        } else if (is_depth(PASS)) {
            reinterpret_cast<uint32_t *>(smem)[l] = 0u;
        } else if (is_color(PASS)) {
            constexpr int kPx = TileCfg<PASS_COLOR>::kPx;
            uint32_t *acc = reinterpret_cast<uint32_t *>(smem);
            acc[l] = 0u;
            acc[kPx + l] = 0u;
            acc[2 * kPx + l] = 0u;
            const int gx = c.x0 + l % c.tw, gy = c.y0 + l / c.tw;
            acc[3 * kPx + l] = view_depth<MV>(a)[gy * view_w<MV>(a) + gx];
        } else {
            reinterpret_cast<unsigned long long *>(smem)[l] = 0ull;
        }
    }
}

template <int PASS, bool MV>
__device__ __forceinline__ void tile_flush(const RasterArgs &a, const ViewRegsT<MV> &vr, const ChunkRec &c,
                                           const unsigned char *smem) {
    const int n = c.tw * c.th;
    for (int l = threadIdx.x; l < n; l += kThreads) {
        const uint32_t pix = (uint32_t)((c.y0 + l / c.tw) * vw<MV>(vr) + c.x0 + l % c.tw);
        if (PASS == PASS_DEPTH_FRAG && CR_TILE_REJECT) {
            constexpr int kPx = TileCfg<PASS_DEPTH_FRAG>::kPx;
            const uint32_t v = reinterpret_cast<const uint32_t *>(smem)[l];
            if (v > reinterpret_cast<const uint32_t *>(smem)[kPx + l])
                red_max_u32(&vdepth<MV>(vr)[pix], v);
        } else if (is_depth(PASS)) {
            const uint32_t v = reinterpret_cast<const uint32_t *>(smem)[l];
            if (v) red_max_u32(&vdepth<MV>(vr)[pix], v);
        } else if (is_color(PASS)) {
            constexpr int kPx = TileCfg<PASS_COLOR>::kPx;
            const uint32_t *acc = reinterpret_cast<const uint32_t *>(smem);
            const uint32_t rc = acc[l];
            const uint32_t cnt = rc >> 20;
            if (cnt) color_global<MV>(a, vr, pix, rc & 0xfffffu, acc[kPx + l], acc[2 * kPx + l], cnt);
        } else {
            const unsigned long long k = reinterpret_cast<const unsigned long long *>(smem)[l];
            if (k) red_max_u64(&vnearest<MV>(vr)[pix], k);
        }
    }
}

// 16-byte asynchronous global -> shared copy (cp.async), for the chunk record.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem_dst, const void *gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem_src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Bulk staging of a chunk's level bytes, coarse words and colours into shared
// memory (cp.async.bulk completing on an mbarrier; this GPU's memory only,
// no multicast).  A chunk is staged when its first point is 16-byte aligned
// in the level array and it has at most kStagePoints points.
constexpr uint32_t kStagePoints = 2048;
constexpr uint32_t kStageBytes = kStagePoints * (1 + 4 + 4);
constexpr uint32_t kStageWaitLimit = 1u << 16;  // polls of an mbarrier before giving up
__device__ __forceinline__ bool stage_ok(uint32_t first, uint32_t count) {
    return (first & 15u) == 0u && count <= kStagePoints && count > 0u;
}
using crb::bulk_g2s;
using crb::mbar_expect_tx;
using crb::mbar_init;
using crb::mbar_wait;
// Thread 0: the bulk copies of one chunk's level bytes, coarse words and
// colours into a stage buffer, completing on `bar`.
__device__ __forceinline__ void stage_issue(unsigned char *stage, uint64_t *bar,
                                            const uint8_t *levels, const uint32_t *low,
                                            const uint32_t *colors, uint32_t first,
                                            uint32_t count) {
    const uint32_t nl = (count + 15u) & ~15u, nw = ((count + 3u) & ~3u) * 4u;
    crb::fence_proxy_async_smem();
    mbar_expect_tx(bar, nl + 2u * nw);
    bulk_g2s(stage, levels + first, nl, bar);
    bulk_g2s(stage + kStagePoints, low + first, nw, bar);
    bulk_g2s(stage + 5 * kStagePoints, colors + first, nw, bar);
}

// Largest view v with begin[v] <= k (views without chunks share their
// begin with the next view, so the view found holds chunk k).
__device__ __forceinline__ uint32_t find_view(const uint32_t *begin, uint32_t nviews, uint32_t k) {
    uint32_t lo = 0, hi = nviews;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (begin[mid] <= k)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Persistent pass over the chunk records: the record of the CTA's next chunk
// is copied into shared memory with cp.async while the current chunk is
// processed.  One view: the CTAs claim chunks from the cloud's work cursor
// (dynamic schedule; a chunk's work varies with its batch's LOD prefix), and
// the last CTA to finish resets the cursor for the next launch.  Batched views (MV): the chunks of
// all views form one index space, view after view; each CTA scans the
// per-view chunk counts once, finds a chunk's view by binary search and
// switches frame, camera and file table when the view changes.
template <int PASS, bool MV>
__device__ __forceinline__ void raster_body(const RasterArgs &a) {
    constexpr bool kFrag = PASS == PASS_DEPTH_FRAG || PASS == PASS_COLOR_FRAG;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ BatchShared sb;
    __shared__ __align__(16) ChunkRec rec[2];
    __shared__ __align__(16) uint32_t rec_frags[2][4];  // frag count, span offset
    __shared__ uint32_t s_vbegin[MV ? kMaxViews + 1 : 1];
    __shared__ unsigned long long s_pbegin[MV && kFrag ? kMaxViews + 1 : 1];
    __shared__ uint32_t s_wsum[kThreads / 32];
    crd::grid_wait();
    crd::launch_dependents();
    if (a.t.redo && *a.t.redo == 0u) return;
    uint32_t nchunks;
    bool emit = true;  // fragments fit the arena (batched views)
    if (MV) {
        // Exclusive prefixes over the views (at most kMaxViews) of their chunk
        // counts and, with fragments, of their fragment spans.
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const uint32_t* vc = a.counters + threadIdx.x * CNT_COUNT;
        uint32_t x = threadIdx.x < a.nviews ? vc[CNT_CHUNKS] : 0u;
        unsigned long long y = (kFrag && threadIdx.x < a.nviews) ? vc[CNT_POINTS] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t xs = __shfl_up_sync(kFull, x, o);
            const unsigned long long ys = __shfl_up_sync(kFull, y, o);
            if (lane >= o) {
                x += xs;
                y += ys;
            }
        }
        if (lane == 31) s_wsum[warp] = x;
        if (kFrag && lane == 31) s_pbegin[warp] = y;
        __syncthreads();
        for (int w = 0; w < warp; ++w) {
            x += s_wsum[w];
            if (kFrag) y += s_pbegin[w];
        }
        __syncthreads();
        s_vbegin[threadIdx.x + 1] = x;
        if (kFrag) s_pbegin[threadIdx.x + 1] = y;
        if (threadIdx.x == 0) {
            s_vbegin[0] = 0u;
            if (kFrag) s_pbegin[0] = 0ull;
        }
        __syncthreads();
        nchunks = s_vbegin[a.nviews];
        if (kFrag) {
            emit = s_pbegin[a.nviews] <= a.frag_cap;
            if (PASS == PASS_DEPTH_FRAG && blockIdx.x == 0 && threadIdx.x == 0)
                *a.frag_overflow = emit ? 0u : 1u;
        }
    } else {
        nchunks = a.counters[CNT_CHUNKS];
    }
    // Chunks are claimed from a work cursor in the launch's counters (the
    // cull zeroes it; the last CTA to finish resets it for the next launch):
    // a dynamic schedule, since a chunk's work varies with its batch's LOD
    // prefix and its view.  Thread 0 claims the next chunk, finds its view
    // and record and prefetches the record while the CTA draws the current
    // one.
    __shared__ uint32_t s_k[2], s_kview[2], s_kslot[2];  // per record buffer
    constexpr bool kStage = CR_BULK_STAGE && PASS == PASS_DEPTH_FRAG && !MV;
    __shared__ __align__(8) uint64_t s_mbar[2];
    unsigned char *stage_base = smem + TileCfg<PASS_DEPTH_FRAG>::kTileBytes;
    uint32_t stage_phase = 0u;  // per buffer: the parity of its next completion
    auto finish = [&]() {
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(a.counters + CNT_DONE, 1u) == gridDim.x - 1u) {
                a.counters[CNT_WORK_DEPTH] = 0u;
                a.counters[CNT_DONE] = 0u;
            }
        }
    };
    // View of chunk kk and the index of its record (also its fragment-count slot).
    auto locate = [&](uint32_t kk, uint32_t &view) -> uint32_t {
        if (!MV) {
            view = 0u;
            return kk;
        }
        view = find_view(s_vbegin, a.nviews, kk);
        return view * a.chunk_stride + (kk - s_vbegin[view]);
    };
    // Thread 0: claim a chunk into record buffer b and start its copy.
    auto claim = [&](int b) {
        const uint32_t kk = atomicAdd(a.counters + CNT_WORK_DEPTH, 1u);
        s_k[b] = kk;
        if (kk >= nchunks) return;
        uint32_t view;
        const uint32_t slot = locate(kk, view);
        s_kview[b] = view;
        s_kslot[b] = slot;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            cp_async16(reinterpret_cast<uint4 *>(&rec[b]) + q,
                       reinterpret_cast<const uint4 *>(a.chunks + slot) + q);
        if (PASS == PASS_COLOR_FRAG) cp_async4(&rec_frags[b][0], a.frag_count + slot);
        if (MV && kFrag) cp_async4(&rec_frags[b][1], a.chunk_poff + slot);
        if (kStage) {
            const uint32_t f = __ldg(&a.chunks[slot].first), n = __ldg(&a.chunks[slot].count);
            if (stage_ok(f, n))
                stage_issue(stage_base + b * kStageBytes, &s_mbar[b], a.levels, a.low, a.colors,
                            f, n);
        }
    };
    if (kStage && threadIdx.x == 0) {
        mbar_init(&s_mbar[0], 1u);
        mbar_init(&s_mbar[1], 1u);
        crb::mbar_init_fence();
    }
    if (threadIdx.x == 0) {
        claim(0);
        sb.file = 0xffffffffu;
        s_frag_count = 0u;
    }
    cp_async_commit();
    uint32_t loaded_view = 0xffffffffu;
    for (int buf = 0;; buf ^= 1) {
        cp_async_wait_all();
        __syncthreads();  // rec[buf] complete; the previous chunk is fully done
        if (s_k[buf] >= nchunks) break;
        const uint32_t cur_view = s_kview[buf], cur_slot = s_kslot[buf];
        const ChunkRec c = rec[buf];
        const uint32_t nfrag = PASS == PASS_COLOR_FRAG ? rec_frags[buf][0] : 0u;
        const uint32_t fslot = cur_slot;
        // First fragment of the chunk: pool index space (one view), or the
        // view's fragment span in the arena (batched views).
        const uint32_t fbase =
            MV ? (kFrag ? (uint32_t)(s_pbegin[cur_view] + rec_frags[buf][1]) : 0u) : c.first;
        if (threadIdx.x == 0) claim(buf ^ 1);
        cp_async_commit();
        const uint32_t file_id = MV ? cur_view * a.nfiles + c.file : c.file;
        const bool new_file = file_id != sb.file;
        const uint32_t work = PASS == PASS_COLOR_FRAG ? nfrag : c.count;
        const bool tiled = a.use_tiles && a.radius_zero && c.tw > 0 &&
                           c.tw * c.th <= TileCfg<PASS>::kPx &&
                           c.tw * c.th <= CR_TILE_PX_PER_POINT * (int)work &&
                           (!is_color(PASS) || c.count < 4096u);
        if (new_file || tiled) {
            __syncthreads();  // everyone has read sb.file (and the view state)
            if (new_file) {
                // The kernels take RasterArgs as a __grid_constant__
                // parameter, so the inline table is read in place.
                const cr_raster_file *file = &(a.ifiles.n ? a.ifiles.f : a.files)[file_id];
                if (threadIdx.x < 16)
                    sb.T[threadIdx.x] = file->transform[threadIdx.x];
                else if (threadIdx.x < 32)
                    sb.world[threadIdx.x - 16] = file->world[threadIdx.x - 16];
                if (threadIdx.x == 0) sb.file = file_id;
            }
            if (MV && cur_view != loaded_view) {  // a new view always brings a new file id
                const ViewDesc &vd = a.views[cur_view];
                if (threadIdx.x >= 32 && threadIdx.x < 48)
                    s_view.view[threadIdx.x - 32] = vd.view[threadIdx.x - 32];
                else if (threadIdx.x >= 48 && threadIdx.x < 64)
                    s_view.proj[threadIdx.x - 48] = vd.proj[threadIdx.x - 48];
                else if (threadIdx.x == 64) {
                    s_view.width = vd.width;
                    s_view.height = vd.height;
                    s_view.depth = vd.depth;
                    s_view.accum = vd.accum;
                    s_view.nearest = vd.nearest;
                }
                loaded_view = cur_view;
                if (tiled) __syncthreads();  // the tile's set-up reads the view state
            }
            if (tiled) tile_init<PASS, MV>(a, c, smem);
            __syncthreads();
        }
        // The view's size and planes: registers (batched views, read once
        // per chunk) or the kernel's parameters (one view).
        const ViewRegsT<MV> vr = [&] {
            if constexpr (MV)
                return view_regs_mv();
            else
                return ViewRegsT<false>(a);
        }();
        const bool need_med = c.level <= 1, need_high = c.level == 0;
        constexpr bool kNeedColor = PASS == PASS_COLOR || PASS == PASS_DEPTH_FRAG;
        // Every point of the chunk passes the dither test when even its
        // highest level (7) does with the largest dither (hash_unit reaches
        // 1.0f; 0.5f without dither): (thr - L) + 0.5f only grows as L falls.
        const bool all_keep = (a.u.lodDither ? 1.0f : 0.5f) < (c.thr - 7.0f) + 0.5f;
        if (PASS == PASS_COLOR_FRAG) {
            // The chunk's fragments, four per thread when 16-byte aligned.
            if ((fbase & 3u) == 0u) {
                const uint32_t nquads = (nfrag + 3u) >> 2;
                for (uint32_t q0 = 0; q0 < nquads; q0 += kThreads) {
                    const uint32_t q = q0 + threadIdx.x;
                    const uint32_t base = fbase + 4u * q;
                    uint4 xy4 = make_uint4(0, 0, 0, 0), co4 = xy4;
                    float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (q < nquads) {
                        xy4 = __ldcs(reinterpret_cast<const uint4 *>(a.frag_xy + base));
                        const uint4 zc01 = __ldcs(reinterpret_cast<const uint4 *>(a.frag_zc + base));
                        const uint4 zc23 =
                            __ldcs(reinterpret_cast<const uint4 *>(a.frag_zc + base + 2));
                        z4 = make_float4(__uint_as_float(zc01.x), __uint_as_float(zc01.z),
                                         __uint_as_float(zc23.x), __uint_as_float(zc23.z));
                        co4 = make_uint4(zc01.y, zc01.w, zc23.y, zc23.w);
                    }
                    const uint32_t nv = q < nquads ? min(4u, nfrag - 4u * q) : 0u;
                    color_quad<MV>(a, vr, smem, c, tiled, nv, xy4, z4, co4);
                }
            } else {
                for (uint32_t l0 = 0; l0 < nfrag; l0 += kThreads) {
                    const uint32_t l = l0 + threadIdx.x;
                    const bool v = l < nfrag;
                    const uint32_t i = fbase + (v ? l : 0u);
                    const uint2 zc = v ? a.frag_zc[i] : make_uint2(0u, 0u);
                    do_fragment<MV>(a, vr, smem, c, tiled, v, v ? a.frag_xy[i] : 0u,
                                    __uint_as_float(zc.x), zc.y);
                }
            }
        } else if ((c.first & 3u) == 0u) {
            // Four points per thread, 16-byte loads (from the bulk-staged
            // copy in shared memory when the chunk was staged).
            bool staged = false;
            const unsigned char *stg = stage_base + buf * kStageBytes;
            if (kStage && stage_ok(c.first, c.count)) {
                staged = mbar_wait(&s_mbar[buf], (stage_phase >> buf) & 1u, kStageWaitLimit);
                if (!staged) {  // give up: record it, wait once more, read global memory
                    if (a.status) *(volatile uint32_t *)a.status = kErrStageWait;
                    mbar_wait(&s_mbar[buf], (stage_phase >> buf) & 1u, kStageWaitLimit);
                }
                stage_phase ^= 1u << buf;
            }
            const uint32_t nquads = (c.count + 3u) >> 2;
            for (uint32_t q0 = 0; q0 < nquads; q0 += kThreads) {
                const uint32_t q = q0 + threadIdx.x;
                const bool qv = q < nquads;
                const uint32_t base = c.first + 4u * q;
                uint32_t lv4 = 0;
                uint4 lo4 = make_uint4(0, 0, 0, 0), me4 = lo4, hi4 = lo4, co4 = lo4;
                if (qv && staged) {
                    lv4 = reinterpret_cast<const uint32_t *>(stg)[q];
                    lo4 = reinterpret_cast<const uint4 *>(stg + kStagePoints)[q];
                    co4 = reinterpret_cast<const uint4 *>(stg + 5 * kStagePoints)[q];
                    if (need_med) me4 = __ldg(reinterpret_cast<const uint4 *>(a.med + base));
                    if (need_high) hi4 = __ldg(reinterpret_cast<const uint4 *>(a.high + base));
                } else if (qv) {
                    lv4 = __ldg(reinterpret_cast<const uint32_t *>(a.levels + base));
                    lo4 = __ldg(reinterpret_cast<const uint4 *>(a.low + base));
                    if (need_med) me4 = __ldg(reinterpret_cast<const uint4 *>(a.med + base));
                    if (need_high) hi4 = __ldg(reinterpret_cast<const uint4 *>(a.high + base));
                    if (kNeedColor)
                        co4 = __ldg(reinterpret_cast<const uint4 *>(a.colors + base));
                }
                const uint32_t l0 = 4u * q;
                if (CR_FRAG_BATCH > 1 && PASS == PASS_DEPTH_FRAG && !MV && emit) {
                    // The fragments of CR_FRAG_BATCH points per atomic (one
                    // view: the batched-view kernel has no registers to
                    // spare for them).
                    constexpr int kB = CR_FRAG_BATCH > 1 ? CR_FRAG_BATCH : 1;
                    Frag f[kB];
                    const uint32_t lvs[4] = {lv4 & 0xffu, (lv4 >> 8) & 0xffu, (lv4 >> 16) & 0xffu,
                                             lv4 >> 24};
                    const uint32_t los[4] = {lo4.x, lo4.y, lo4.z, lo4.w};
                    const uint32_t mes[4] = {me4.x, me4.y, me4.z, me4.w};
                    const uint32_t his[4] = {hi4.x, hi4.y, hi4.z, hi4.w};
                    const uint32_t cos[4] = {co4.x, co4.y, co4.z, co4.w};
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        do_point<PASS, MV>(a, vr, sb, smem, c, tiled, qv && l0 + j < c.count,
                                           l0 + j, lvs[j], los[j], mes[j], his[j], cos[j], fbase,
                                           emit, all_keep, &f[j % kB]);
                        if (j % kB == kB - 1) emit_fragments<kB>(a, fbase, f);
                    }
                } else {
                    do_point<PASS, MV>(a, vr, sb, smem, c, tiled, qv && l0 + 0 < c.count, l0 + 0,
                                       lv4 & 0xffu, lo4.x, me4.x, hi4.x, co4.x, fbase, emit,
                                       all_keep);
                    do_point<PASS, MV>(a, vr, sb, smem, c, tiled, qv && l0 + 1 < c.count, l0 + 1,
                                       (lv4 >> 8) & 0xffu, lo4.y, me4.y, hi4.y, co4.y, fbase,
                                       emit, all_keep);
                    do_point<PASS, MV>(a, vr, sb, smem, c, tiled, qv && l0 + 2 < c.count, l0 + 2,
                                       (lv4 >> 16) & 0xffu, lo4.z, me4.z, hi4.z, co4.z, fbase,
                                       emit, all_keep);
                    do_point<PASS, MV>(a, vr, sb, smem, c, tiled, qv && l0 + 3 < c.count, l0 + 3,
                                       lv4 >> 24, lo4.w, me4.w, hi4.w, co4.w, fbase, emit,
                                       all_keep);
                }
            }
        } else {
            // Unaligned start (pointsPerBatch not a multiple of 4): one point per thread.
            for (uint32_t l0 = 0; l0 < c.count; l0 += kThreads) {
                const uint32_t local = l0 + threadIdx.x;
                const bool v = local < c.count;
                const uint32_t i = c.first + (v ? local : 0u);
                const uint32_t lv = v ? a.levels[i] : 0u;
                const uint32_t lo = v ? a.low[i] : 0u;
                const uint32_t me = (v && need_med) ? a.med[i] : 0u;
                const uint32_t hi = (v && need_high) ? a.high[i] : 0u;
                const uint32_t co = (v && kNeedColor) ? a.colors[i] : 0u;
                do_point<PASS, MV>(a, vr, sb, smem, c, tiled, v, local, lv, lo, me, hi, co, fbase, emit, all_keep);
            }
        }
        if (tiled || PASS == PASS_DEPTH_FRAG) {
            __syncthreads();
            if (tiled) tile_flush<PASS, MV>(a, vr, c, smem);
            if (PASS == PASS_DEPTH_FRAG && threadIdx.x == 0) {
                a.frag_count[fslot] = s_frag_count;
                s_frag_count = 0u;
            }
        }
    }
    cp_async_wait_all();
    finish();
}


// Colour pass over the depth pass's fragments for one view, one chunk per CTA
// (claimed from the work cursor).  A chunk's points are one compact region of
// a Morton-ordered batch: its fragments hit few distinct pixels, but rarely
// in a row (over a 1080p frame of 100M points, 10.7M visible fragments,
// 1.9M distinct pixels per chunk).  Each visible fragment is summed into a
// shared-memory hash table keyed by pixel (R, G, B, count as 32-bit sums: a
// chunk holds at most 65,536 points, so none overflows; 64-bit shared
// atomics were slower), and the table is flushed with one global add pair
// (or four 32-bit adds) per distinct pixel.  A fragment whose pixel finds no
// slot within kHashProbes probes is added to the frame directly.
constexpr int kHashBits = 10;
constexpr uint32_t kHashSlots = 1u << kHashBits;
constexpr int kHashProbes = 16;
constexpr uint32_t kHashEmpty = 0xffffffffu;

// Slot of pixel (x, y): x + 37 y over the table.  Distinct pixels of any
// 37 × 27 window take distinct slots, and the 32 lanes of a warp, whose
// fragments lie in one small patch of the screen, mostly fall in distinct
// shared-memory banks (x + 5 y mod 32).
__device__ __forceinline__ uint32_t hash_slot(uint32_t xy) {
    return ((xy & 0xffffu) + 37u * (xy >> 16)) & (kHashSlots - 1u);
}

#ifndef CR_HASH3
#define CR_HASH3 0
#endif
// Packed table rows: R | count << 20, G, B — exact while the chunk has fewer
// than 4096 fragments (a count below 2^12, a red sum below 255 * 4096 < 2^20).
__device__ __forceinline__ bool hash_packed(uint32_t nfrag) { return CR_HASH3 && nfrag < 4096u; }

template <bool MV>
__device__ __forceinline__ void hash_add_sums(uint32_t *hkey, uint32_t *hsum, const RasterArgs &a,
                                              const ViewRegsT<MV> &vr, uint32_t pix, uint32_t xy,
                                              uint32_t r, uint32_t g, uint32_t b, uint32_t n,
                                              bool p3 = false) {
    uint32_t h = hash_slot(xy);
    for (int probe = 0; probe < kHashProbes; ++probe) {
        uint32_t cur = hkey[h];
        if (cur == kHashEmpty) cur = atomicCAS(hkey + h, kHashEmpty, pix);
        if (cur == kHashEmpty || cur == pix) {
            if (p3) {
                atomicAdd(hsum + h, r | (n << 20));
                atomicAdd(hsum + kHashSlots + h, g);
                atomicAdd(hsum + 2 * kHashSlots + h, b);
            } else {
                atomicAdd(hsum + h, r);
                atomicAdd(hsum + kHashSlots + h, g);
                atomicAdd(hsum + 2 * kHashSlots + h, b);
                atomicAdd(hsum + 3 * kHashSlots + h, n);
            }
            return;
        }
        h = (h + 1u) & (kHashSlots - 1u);
    }
    color_global<MV>(a, vr, pix, r, g, b, n);
}

template <bool MV>
__device__ __forceinline__ void hash_add(uint32_t *hkey, uint32_t *hsum, const RasterArgs &a,
                                         const ViewRegsT<MV> &vr, uint32_t pix, uint32_t xy,
                                         uint32_t col, bool p3) {
    hash_add_sums<MV>(hkey, hsum, a, vr, pix, xy, col & 0xffu, (col >> 8) & 0xffu,
                      (col >> 16) & 0xffu, 1u, p3);
}

// Clears the table (at kernel start).
__device__ __forceinline__ void hash_clear(uint32_t *hkey, uint32_t *hsum) {
    for (uint32_t i = threadIdx.x; i < kHashSlots; i += kThreads) {
        hkey[i] = kHashEmpty;
        hsum[i] = hsum[kHashSlots + i] = hsum[2 * kHashSlots + i] = hsum[3 * kHashSlots + i] = 0u;
    }
}

// The colour pass over one chunk's n fragments starting at base, against
// the frame of W columns whose depth plane is `depth`: sums into the table.
template <bool MV>
__device__ __forceinline__ void hash_frags(const RasterArgs &a, const ViewRegsT<MV> &vr,
                                           uint32_t *hkey, uint32_t *hsum, uint32_t n,
                                           uint32_t base, int W, const uint32_t *depth) {
    const bool p3 = hash_packed(n);
    if ((base & 3u) == 0u) {
        for (uint32_t f = 4u * threadIdx.x; f < n; f += 4u * kThreads) {
            const uint4 xy = __ldcs(reinterpret_cast<const uint4 *>(a.frag_xy + base + f));
            const uint4 zc01 = __ldcs(reinterpret_cast<const uint4 *>(a.frag_zc + base + f));
            const uint4 zc23 = __ldcs(reinterpret_cast<const uint4 *>(a.frag_zc + base + f + 2));
            const uint32_t xs[4] = {xy.x, xy.y, xy.z, xy.w},
                           cs[4] = {zc01.y, zc01.w, zc23.y, zc23.w};
            const float zs[4] = {__uint_as_float(zc01.x), __uint_as_float(zc01.z),
                                 __uint_as_float(zc23.x), __uint_as_float(zc23.z)};
            uint32_t pix[4], cl[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                pix[q] = (xs[q] >> 16) * (uint32_t)W + (xs[q] & 0xffffu);
                cl[q] = f + q < n ? __ldg(depth + pix[q]) : 0u;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (cl[q] != 0u && zs[q] >= crd::uint_to_depth(cl[q]) * a.keep_scale)
                    hash_add<MV>(hkey, hsum, a, vr, pix[q], xs[q], cs[q], p3);
        }
    } else {
        for (uint32_t f = threadIdx.x; f < n; f += kThreads) {
            const uint32_t xy = a.frag_xy[base + f];
            const uint32_t pix = (xy >> 16) * (uint32_t)W + (xy & 0xffffu);
            const uint32_t cl = __ldg(depth + pix);
            const uint2 zc = a.frag_zc[base + f];
            if (cl != 0u && __uint_as_float(zc.x) >= crd::uint_to_depth(cl) * a.keep_scale)
                hash_add<MV>(hkey, hsum, a, vr, pix, xy, zc.y, p3);
        }
    }
}

// Flushes the table (one global add pair per distinct pixel) and clears it.
// With a cursor, thread 0 also claims the next chunk into *next, so the
// claim's round trip overlaps the flush.  Called after a barrier that
// completes the sums (and after every thread has read the current claim).
template <bool MV>
__device__ __forceinline__ void hash_flush(const RasterArgs &a, const ViewRegsT<MV> &vr,
                                           uint32_t *hkey, uint32_t *hsum, bool p3,
                                           uint32_t *cursor = nullptr, uint32_t *next = nullptr) {
    uint32_t claimed = 0u;
    if (cursor && threadIdx.x == 0) claimed = atomicAdd(cursor, 1u);
    for (uint32_t i = threadIdx.x; i < kHashSlots; i += kThreads) {
        const uint32_t pix = hkey[i];
        if (pix == kHashEmpty) continue;
        const uint32_t w0 = hsum[i];
        color_global<MV>(a, vr, pix, p3 ? (w0 & 0xfffffu) : w0, hsum[kHashSlots + i],
                         hsum[2 * kHashSlots + i], p3 ? (w0 >> 20) : hsum[3 * kHashSlots + i]);
        hkey[i] = kHashEmpty;
        hsum[i] = hsum[kHashSlots + i] = hsum[2 * kHashSlots + i] = hsum[3 * kHashSlots + i] = 0u;
    }
    if (cursor && threadIdx.x == 0) *next = claimed;
}

// The colour pass over chunk k of one view.  Every thread of the CTA calls
// this; the caller's barrier before the next chunk orders the clearing
// before its first add.
__device__ __forceinline__ void hash_chunk(const RasterArgs &a, const ViewRegsT<false> &vr,
                                           uint32_t *hkey, uint32_t *hsum, uint32_t k,
                                           uint32_t *cursor = nullptr, uint32_t *next = nullptr) {
    const uint32_t nfrag = __ldg(a.frag_count + k);
    hash_frags<false>(a, vr, hkey, hsum, nfrag, __ldg(&a.chunks[k].first), a.u.width, a.t.depth);
    __syncthreads();  // the chunk's sums are complete (and k has been read by all)
    hash_flush<false>(a, vr, hkey, hsum, hash_packed(nfrag), cursor, next);
}

// 1024 slots (about three times a chunk's typical distinct visible pixels)
// and at most 40 registers: six CTAs share an SM.
__global__ void __launch_bounds__(kThreads, 6) color_hash_kernel(const __grid_constant__ RasterArgs a) {
    crd::grid_wait();
    crd::launch_dependents();
    if (a.t.redo && *a.t.redo == 0u) return;
    __shared__ uint32_t hkey[kHashSlots];
    __shared__ uint32_t hsum[4 * kHashSlots];
    __shared__ uint32_t s_k;
    const uint32_t nchunks = a.counters[CNT_CHUNKS];
    const ViewRegsT<false> vr(a);
    hash_clear(hkey, hsum);
    uint32_t *cursor = a.counters + CNT_WORK_DEPTH;
    if (threadIdx.x == 0) s_k = atomicAdd(cursor, 1u);
    for (;;) {
        __syncthreads();  // s_k and the cleared table
        const uint32_t k = s_k;
        if (k >= nchunks) break;
        hash_chunk(a, vr, hkey, hsum, k, cursor, &s_k);  // claims the next chunk into s_k
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(a.counters + CNT_DONE, 1u) == gridDim.x - 1u) {
            a.counters[CNT_WORK_DEPTH] = 0u;
            a.counters[CNT_DONE] = 0u;
        }
    }
}

// The colour pass of a group of batched views over their fragments: the
// one-view hash kernel with each chunk's view found by binary search over
// the per-view chunk prefix (as the point passes do), accumulating into that
// view's planes.  It returns at once when the group's fragments overflowed
// the arena; color_views_kernel then decodes the points instead.
__global__ void __launch_bounds__(kThreads, 6)
    color_hash_views_kernel(const __grid_constant__ RasterArgs a) {
    crd::grid_wait();
    if (*a.frag_overflow) return;
    __shared__ uint32_t hkey[kHashSlots];
    __shared__ uint32_t hsum[4 * kHashSlots];
    __shared__ uint32_t s_vbegin[kMaxViews + 1];
    __shared__ unsigned long long s_pbegin[kMaxViews + 1];
    __shared__ uint32_t s_wsum[kThreads / 32];
    __shared__ unsigned long long s_psum[kThreads / 32];
    __shared__ uint32_t s_k;
    // Exclusive prefixes over the views (at most kMaxViews = kThreads) of
    // their chunk counts and fragment spans.
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const uint32_t *vc = a.counters + threadIdx.x * CNT_COUNT;
        uint32_t x = threadIdx.x < a.nviews ? vc[CNT_CHUNKS] : 0u;
        unsigned long long y = threadIdx.x < a.nviews ? vc[CNT_POINTS] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t xs = __shfl_up_sync(kFull, x, o);
            const unsigned long long ys = __shfl_up_sync(kFull, y, o);
            if (lane >= o) {
                x += xs;
                y += ys;
            }
        }
        if (lane == 31) {
            s_wsum[warp] = x;
            s_psum[warp] = y;
        }
        __syncthreads();
        for (int w = 0; w < warp; ++w) {
            x += s_wsum[w];
            y += s_psum[w];
        }
        s_vbegin[threadIdx.x + 1] = x;
        s_pbegin[threadIdx.x + 1] = y;
        if (threadIdx.x == 0) {
            s_vbegin[0] = 0u;
            s_pbegin[0] = 0ull;
        }
    }
    hash_clear(hkey, hsum);
    uint32_t *cursor = a.counters + CNT_WORK_DEPTH;
    if (threadIdx.x == 0) s_k = atomicAdd(cursor, 1u);
    __syncthreads();  // prefixes, table and first claim
    const uint32_t nchunks = s_vbegin[a.nviews];
    for (;;) {
        const uint32_t k = s_k;
        if (k >= nchunks) break;
        const uint32_t view = find_view(s_vbegin, a.nviews, k);
        const uint32_t slot = view * a.chunk_stride + (k - s_vbegin[view]);
        const ViewDesc &vd = a.views[view];
        const ViewRegsT<true> vr{vd.width, vd.height, vd.depth, vd.accum, vd.nearest};
        const uint32_t nfrag = __ldg(a.frag_count + slot);
        hash_frags<true>(a, vr, hkey, hsum, nfrag,
                         (uint32_t)(s_pbegin[view] + __ldg(a.chunk_poff + slot)), vd.width,
                         vd.depth);
        __syncthreads();  // the chunk's sums are complete (and k has been read by all)
        hash_flush<true>(a, vr, hkey, hsum, hash_packed(nfrag), cursor, &s_k);
        __syncthreads();  // the next claim and the cleared table
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(a.counters + CNT_DONE, 1u) == gridDim.x - 1u) {
            a.counters[CNT_WORK_DEPTH] = 0u;
            a.counters[CNT_DONE] = 0u;
        }
    }
}

// Exact re-run of a frame whose packed colour adds may have carried (the
// resolve set the redo word).  One CTA, launched every frame, that returns
// at once unless the word is set; then, in order, it zeroes the
// accumulators, runs the colour pass of every cloud over its fragments with
// one 32-bit add per field, and resolves every pixel.  A single CTA orders
// the three steps with block barriers, so they take one launch instead of
// three; the re-run is rare and its speed does not matter.
struct RedoCloud {
    const ChunkRec *chunks;
    const uint32_t *counters, *frag_count, *frag_xy;
    const uint2 *frag_zc;
};
constexpr uint32_t kRedoMaxClouds = 32;
struct RedoArgs {
    RasterArgs a;  // frame targets (unpacked adds) and uniforms; per-cloud fields from clouds[]
    RedoCloud clouds[kRedoMaxClouds];
    uint32_t nclouds;
    const uint32_t *redo;
    uint32_t *rgba;
    float *depthf;
    uint32_t npix;
    ResolveUniforms ru;
};

__global__ void __launch_bounds__(kThreads) hqs_redo_kernel(RedoArgs r) {
    crd::grid_wait();
    crd::launch_dependents();
    if (*r.redo == 0u) return;
    __shared__ uint32_t hkey[kHashSlots];
    __shared__ uint32_t hsum[4 * kHashSlots];
    for (uint32_t p = threadIdx.x; p < r.npix; p += kThreads) r.a.t.accum[p] = make_uint4(0, 0, 0, 0);
    hash_clear(hkey, hsum);
    __syncthreads();  // accumulators and table zeroed
    for (uint32_t ci = 0; ci < r.nclouds; ++ci) {
        RasterArgs a = r.a;
        a.chunks = r.clouds[ci].chunks;
        a.frag_count = const_cast<uint32_t *>(r.clouds[ci].frag_count);
        a.frag_xy = const_cast<uint32_t *>(r.clouds[ci].frag_xy);
        a.frag_zc = const_cast<uint2 *>(r.clouds[ci].frag_zc);
        const ViewRegsT<false> vr(a);
        const uint32_t nchunks = r.clouds[ci].counters[CNT_CHUNKS];
        for (uint32_t k = 0; k < nchunks; ++k) {
            hash_chunk(a, vr, hkey, hsum, k);
            __syncthreads();  // the table is clear again
        }
    }
    __threadfence();
    __syncthreads();  // every add of the block has reached L2
    for (uint32_t p = threadIdx.x; p < r.npix; p += kThreads) {
        const uint4 acc = __ldcg(r.a.t.accum + p);
        crd::resolve_pixel(acc, acc.w ? r.a.t.depth[p] : 0u, r.ru, r.rgba[p], r.depthf[p]);
    }
}

template <int PASS, bool MV>
__global__ void __launch_bounds__(kThreads) raster_kernel(const __grid_constant__ RasterArgs a) {
    raster_body<PASS, MV>(a);
}

// The one-view depth passes fit 64 registers without spilling, so four CTAs
// (and their 32 KB screen tiles) share an SM.
#ifndef CR_DEPTH_MIN_BLOCKS
#define CR_DEPTH_MIN_BLOCKS 4
#endif
template <int PASS>
__global__ void __launch_bounds__(kThreads, CR_DEPTH_MIN_BLOCKS) depth_kernel(const __grid_constant__ RasterArgs a) {
    raster_body<PASS, false>(a);
}

// The batched-view depth passes, also at four CTAs per SM (64 registers, a
// few spilled): 64 views of the 50M-point heightfield 8.23 -> 7.94 ms against
// the compiler's own choice of 80 registers (three CTAs per SM).
template <int PASS>
__global__ void __launch_bounds__(kThreads, 4)
    depth_views_kernel(const __grid_constant__ RasterArgs a) {
    raster_body<PASS, true>(a);
}

// The colour pass that decodes the points holds a 64 KB screen tile, so at
// most three CTAs share an SM whatever their registers; saying so lets the
// compiler use up to 85 registers per thread instead of spilling.
template <bool MV>
__global__ void __launch_bounds__(kThreads, 3) raster_kernel_color(const __grid_constant__ RasterArgs a) {
    raster_body<PASS_COLOR, MV>(a);
}

// Colour pass of batched views whose fragments overflowed the arena: the
// decode-and-project pass (color_hash_views_kernel draws the others).
__global__ void __launch_bounds__(kThreads, 3) color_views_kernel(const __grid_constant__ RasterArgs a) {
    if (*a.frag_overflow) raster_body<PASS_COLOR, true>(a);
}

// The kernel a pass launches.
template <int PASS, bool MV>
constexpr auto kernel_for() {
    if constexpr (PASS == PASS_COLOR)
        return raster_kernel_color<MV>;
    else if constexpr (!MV && is_depth(PASS))
        return depth_kernel<PASS>;
    else if constexpr (MV && is_depth(PASS))
        return depth_views_kernel<PASS>;
    else
        return raster_kernel<PASS, MV>;
}

template <int PASS, bool MV>
int blocks_per_sm_for() {
    int n = 0;
    constexpr auto k = kernel_for<PASS, MV>();
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, TileCfg<PASS>::kBytes);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kThreads, TileCfg<PASS>::kBytes) !=
        cudaSuccess)
        n = 1;
    return n < 1 ? 1 : n;
}

int color_views_blocks_per_sm() {
    int n = 0;
    constexpr int kBytes = TileCfg<PASS_COLOR>::kBytes;
    cudaFuncSetAttribute(color_views_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kBytes);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, color_views_kernel, kThreads, kBytes) !=
        cudaSuccess)
        n = 1;
    return n < 1 ? 1 : n;
}

template <bool MV>
int raster_blocks_per_sm(int pass) {
    switch (pass) {
    case PASS_DEPTH: return blocks_per_sm_for<PASS_DEPTH, MV>();
    case PASS_COLOR: return blocks_per_sm_for<PASS_COLOR, MV>();
    case PASS_DEPTH_FRAG: return blocks_per_sm_for<PASS_DEPTH_FRAG, MV>();
    case PASS_COLOR_FRAG:
        if (MV) return color_views_blocks_per_sm();
        {
            int n = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, color_hash_kernel, kThreads, 0) !=
                cudaSuccess)
                n = 1;
            return n < 1 ? 1 : n;
        }
    default:
        if constexpr (MV)
            return 1;  // batched views draw HQS only
        else
            return blocks_per_sm_for<PASS_NEAREST, false>();
    }
}

RasterArgs make_args(cr_cloud *cloud, const RasterUniforms &u, const RasterTargets &t) {
    RasterArgs a;
    a.chunks = cloud->d_chunks;
    a.files = cloud->d_files;
    a.ifiles = inline_files(cloud);
    a.counters = cloud->d_counters;
    a.low = cloud->d_low;
    a.med = cloud->d_med;
    a.high = cloud->d_high;
    a.colors = cloud->d_colors;
    a.levels = cloud->d_levels;
    a.t = t;
    a.u = u;
    a.keep_scale = 1.0f - u.depthTolerance;
    // pointFootprintRadius clamps the size to [lo, hi] with lo >= 1; when the
    // upper bound is 1 every radius is 0 whatever the distance.
    a.radius_zero = fmaxf(u.minimumPointSize, u.maximumPointSize) <= 1.0f ? 1 : 0;
    a.use_tiles = cloud->ctx->use_tiles ? 1 : 0;
    a.frag_xy = cloud->d_frag_xy;
    a.frag_zc = cloud->d_frag_zc;
    a.frag_count = cloud->d_frag_count;
    a.views = nullptr;
    a.nviews = 0;
    a.nfiles = 0;
    a.chunk_stride = 0;
    a.chunk_poff = nullptr;
    a.frag_cap = 0;
    a.frag_overflow = nullptr;
    a.fcolors = nullptr;
    a.dldimg = nullptr;
    a.fgrad = nullptr;
    a.status = cloud->ctx->d_status;
    return a;
}

// One-view passes start while the previous kernel drains (programmatic
// dependent launch); batched views, captured in a graph, launch plainly.
template <int PASS, bool MV>
void launch_pass(const RasterArgs &a, int grid, cudaStream_t s) {
    if constexpr (MV)
        kernel_for<PASS, MV>()<<<grid, kThreads, TileCfg<PASS>::kBytes, s>>>(a);
    else
        launch_programmatic(kernel_for<PASS, MV>(), dim3(grid), dim3(kThreads),
                            (size_t)TileCfg<PASS>::kBytes, s, a);
}

}  // namespace

cr_status launch_raster(cr_cloud *cloud, RasterPass pass, const RasterUniforms &u,
                        const RasterTargets &t, cudaStream_t s) {
    const RasterArgs a = make_args(cloud, u, t);
    cr_context *ctx = cloud->ctx;
    if (ctx->blocks_per_sm[pass] == 0) ctx->blocks_per_sm[pass] = raster_blocks_per_sm<false>(pass);
    const int grid = ctx->sm_count * ctx->blocks_per_sm[pass];
    switch (pass) {
    case PASS_DEPTH: launch_pass<PASS_DEPTH, false>(a, grid, s); break;
    case PASS_COLOR: launch_pass<PASS_COLOR, false>(a, grid, s); break;
    case PASS_DEPTH_FRAG: launch_pass<PASS_DEPTH_FRAG, false>(a, grid, s); break;
    case PASS_COLOR_FRAG:
        CR_CUDA(launch_programmatic(color_hash_kernel, dim3(grid), dim3(kThreads), 0, s, a));
        break;
    default: launch_pass<PASS_NEAREST, false>(a, grid, s); break;
    }
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

cr_status launch_hqs_redo(cr_frame *f, cr_cloud *const *clouds, uint32_t nclouds,
                          const RasterUniforms &u, const RasterTargets &t,
                          const ResolveUniforms &ru, cudaStream_t s) {
    if (nclouds > kRedoMaxClouds || t.packed || !t.redo)
        return cri::fail(CR_ERR_INTERNAL, "launch_hqs_redo: arguments");
    if (nclouds == 0) return CR_OK;  // no sample: the resolve cannot have asked for a re-run
    RedoArgs r;
    r.a = make_args(clouds[0], u, t);
    for (uint32_t i = 0; i < nclouds; ++i)
        r.clouds[i] = RedoCloud{clouds[i]->d_chunks,   clouds[i]->d_counters, clouds[i]->d_frag_count,
                                clouds[i]->d_frag_xy, clouds[i]->d_frag_zc};
    r.nclouds = nclouds;
    r.redo = t.redo;
    r.rgba = f->d_rgba[0];
    r.depthf = f->d_depthf;
    r.npix = (uint32_t)f->width * (uint32_t)f->height;
    r.ru = ru;
    CR_CUDA(launch_programmatic(hqs_redo_kernel, dim3(1), dim3(kThreads), 0, s, r));
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

uint32_t hqs_redo_max_clouds() { return kRedoMaxClouds; }

cr_status launch_raster_f32(cr_cloud *cloud, RasterPass pass, const RasterUniforms &u,
                            const RasterTargets &t, const float *colors, const float *dldimg,
                            float *grad, cudaStream_t s) {
    if (pass != PASS_COLOR_F32 && pass != PASS_GRAD)
        return cri::fail(CR_ERR_INTERNAL, "launch_raster_f32: pass");
    RasterArgs a = make_args(cloud, u, t);
    a.fcolors = colors;
    a.dldimg = dldimg;
    a.fgrad = grad;
    cr_context *ctx = cloud->ctx;
    if (ctx->blocks_per_sm[pass] == 0)
        ctx->blocks_per_sm[pass] = pass == PASS_COLOR_F32
                                       ? blocks_per_sm_for<PASS_COLOR_F32, false>()
                                       : blocks_per_sm_for<PASS_GRAD, false>();
    const int grid = ctx->sm_count * ctx->blocks_per_sm[pass];
    if (pass == PASS_COLOR_F32)
        launch_pass<PASS_COLOR_F32, false>(a, grid, s);
    else
        launch_pass<PASS_GRAD, false>(a, grid, s);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

void raster_prepare_views(cr_context *ctx) {
    for (int p : {PASS_DEPTH, PASS_COLOR, PASS_DEPTH_FRAG, PASS_COLOR_FRAG})
        if (ctx->blocks_per_sm_views[p] == 0) ctx->blocks_per_sm_views[p] = raster_blocks_per_sm<true>(p);
    if (ctx->blocks_per_sm_hash_views == 0) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, color_hash_views_kernel, kThreads, 0) !=
            cudaSuccess)
            n = 1;
        ctx->blocks_per_sm_hash_views = n < 1 ? 1 : n;
    }
}

cr_status launch_raster_views(cr_cloud *cloud, RasterPass pass, const RasterUniforms &u,
                              const RasterTargets &t, const ViewDesc *views, uint32_t nviews,
                              const cr_raster_file *files, uint32_t nfiles,
                              const ChunkRec *chunks, uint32_t chunk_stride,
                              uint32_t *counters, const ViewsFragments *frags, cudaStream_t s) {
    const bool frag_pass = pass == PASS_DEPTH_FRAG || pass == PASS_COLOR_FRAG;
    if (nviews == 0 || nviews > kMaxViews || (frag_pass && !frags) || pass == PASS_NEAREST)
        return cri::fail(CR_ERR_INTERNAL, "batched views: bad pass arguments");
    RasterArgs a = make_args(cloud, u, t);
    a.chunks = chunks;
    a.files = files;
    a.ifiles.n = 0;  // the views' own tables
    a.counters = counters;
    a.views = views;
    a.nviews = nviews;
    a.nfiles = nfiles;
    a.chunk_stride = chunk_stride;
    if (frags) {
        a.frag_xy = frags->xy;
        a.frag_zc = frags->zc;
        a.frag_count = frags->count;
        a.chunk_poff = frags->poff;
        a.frag_cap = frags->cap;
        a.frag_overflow = frags->overflow;
    }
    cr_context *ctx = cloud->ctx;
    if (ctx->blocks_per_sm_views[pass] == 0)
        ctx->blocks_per_sm_views[pass] = raster_blocks_per_sm<true>(pass);
    const int grid = ctx->sm_count * ctx->blocks_per_sm_views[pass];
    switch (pass) {
    case PASS_DEPTH: launch_pass<PASS_DEPTH, true>(a, grid, s); break;
    case PASS_COLOR: launch_pass<PASS_COLOR, true>(a, grid, s); break;
    case PASS_DEPTH_FRAG: launch_pass<PASS_DEPTH_FRAG, true>(a, grid, s); break;
    default: {  // PASS_COLOR_FRAG: fragments, or decode when they overflowed
        if (ctx->blocks_per_sm_hash_views == 0) raster_prepare_views(ctx);
        color_hash_views_kernel<<<ctx->sm_count * ctx->blocks_per_sm_hash_views, kThreads, 0, s>>>(
            a);
        color_views_kernel<<<grid, kThreads, TileCfg<PASS_COLOR>::kBytes, s>>>(a);
        break;
    }
    }
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}
