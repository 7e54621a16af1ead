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
// persistent grid sized to fill every SM walks the records with a static
// grid-stride schedule, copying the next record into shared memory
// (cp.async) while the current chunk is processed, so batches of very
// different sizes spread evenly over the SMs.  Each CTA of 256 threads walks
// a chunk four points per thread with 16-byte loads of the level bytes and
// position / colour words; warps skip the projection and the atomics when
// none of their lanes survives the dither or clip tests.
//
// Screen tiles.  A batch is Morton-compact, so its points land in a small
// screen rectangle (the projection of its AABB's eight corners, widened by
// two pixels, computed by the cull).  When that rectangle has few pixels per
// point, the CTA
// accumulates in shared memory — depth max, or R|G and B|count packed in two
// 64-bit adds (a batch's per-pixel sums stay below 2^32), or the nearest key
// — and then flushes one global atomic per touched pixel.  The colour pass
// also stages the rectangle's settled depths in shared memory.  Points that
// round outside the rectangle use global atomics directly, so the tile is a
// cache and never changes a result.  Other batches use global atomics with
// a warp-level pre-merge of same-pixel lanes (__match_any_sync + redux).
// Integer max and sum are associative and commutative: the planes are
// bit-identical to a per-point atomic order either way.
#include "cr_device.cuh"
#include "cr_internal.h"

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
    static constexpr int kPx = 2048;
    static constexpr int kBytes = kPx * 16 + kPx * 4;  // 2 x u64 accumulators + depth
};
template <>
struct TileCfg<PASS_NEAREST> {
    static constexpr int kPx = 4096;
    static constexpr int kBytes = kPx * 8;
};

struct RasterArgs {
    const ChunkRec *chunks;
    const cr_raster_file *files;
    uint32_t *counters;
    const uint32_t *low, *med, *high, *colors;
    const uint8_t *levels;
    RasterTargets t;
    RasterUniforms u;
    float keep_scale;  // 1 - depthTolerance
    int radius_zero;   // every footprint is a single pixel
    int use_tiles;
};

struct BatchShared {
    float T[16];      // file.transform
    float world[16];  // file.world (footprint only)
    uint32_t file;    // file cached in T / world
};

struct PointOut {
    bool ok;
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
template <int PASS>
__device__ __forceinline__ void project_point(const RasterArgs &a, const BatchShared &sb,
                                              const ChunkRec &c, uint32_t lo, uint32_t me,
                                              uint32_t hi, PointOut &o) {
    uint32_t x, y, z;
    if (c.level == 0) {
        x = ((lo & 1023u) << 20) | ((me & 1023u) << 10) | (hi & 1023u);
        y = (((lo >> 10) & 1023u) << 20) | (((me >> 10) & 1023u) << 10) | ((hi >> 10) & 1023u);
        z = (((lo >> 20) & 1023u) << 20) | (((me >> 20) & 1023u) << 10) | ((hi >> 20) & 1023u);
    } else if (c.level == 1) {
        x = ((lo & 1023u) << 10) | (me & 1023u);
        y = (((lo >> 10) & 1023u) << 10) | ((me >> 10) & 1023u);
        z = (((lo >> 20) & 1023u) << 10) | ((me >> 20) & 1023u);
    } else {
        x = lo & 1023u;
        y = (lo >> 10) & 1023u;
        z = (lo >> 20) & 1023u;
    }
    o.px = (float)x * c.qx + c.minX;
    o.py = (float)y * c.qy + c.minY;
    o.pz = (float)z * c.qz + c.minZ;
    const crd::f4 clip = crd::mulp(sb.T, o.px, o.py, o.pz);
    bool ok = o.ok;
    if (clip.w <= 0.0f) ok = false;
    const float nx = clip.x / clip.w, ny = clip.y / clip.w, nz = clip.z / clip.w;
    if (nx < -1.0f || ny < -1.0f || nx > 1.0f || ny > 1.0f || nz > 1.0f) ok = false;
    if (PASS == PASS_NEAREST ? (nz <= 0.0f) : (nz < 0.0f)) ok = false;
    const int W = a.u.width, H = a.u.height;
    o.ix = (int)((nx * 0.5f + 0.5f) * (float)W);
    const int iy = (int)((ny * 0.5f + 0.5f) * (float)H);
    if (o.ix < 0 || o.ix >= W || iy < 0 || iy >= H) ok = false;
    o.iy = H - 1 - iy;
    o.depth = crd::depth_to_uint(nz);
    o.nz = nz;
    o.ok = ok;
    if (PASS == PASS_COLOR) {  // ColorPass/Shaders.metal:95-100
        if (a.u.colorizeChunks)
            o.color = c.batchIndex * 1234567u;
        else if (a.u.colorizeOverdraw)
            o.color = 0x00010101u;
    }
}

__device__ __forceinline__ unsigned long long nearest_key(uint32_t depth, uint32_t index) {
    return ((unsigned long long)depth << 32) | (unsigned long long)(~index);
}

__device__ __forceinline__ void color_global(const RasterArgs &a, uint32_t pix, uint32_t r,
                                             uint32_t g, uint32_t b, uint32_t n) {
    unsigned int *acc = reinterpret_cast<unsigned int *>(&a.t.accum[pix]);
    atomicAdd(acc + 0, r);
    atomicAdd(acc + 1, g);
    atomicAdd(acc + 2, b);
    atomicAdd(acc + 3, n);
}

// Direct path, radius 0: warp pre-merge of same-pixel lanes, then one global
// atomic per distinct pixel.  Every lane of the warp calls this.
template <int PASS>
__device__ __forceinline__ void emit_direct(const RasterArgs &a, const PointOut &o) {
    const int lane = threadIdx.x & 31;
    const uint32_t pix = (uint32_t)(o.iy * a.u.width + o.ix);
    if (PASS == PASS_DEPTH) {
        const uint32_t peers = __match_any_sync(kFull, o.ok ? pix : kFull);
        if (o.ok) {
            const uint32_t m = __reduce_max_sync(peers, o.depth);
            if (lane == __ffs(peers) - 1) atomicMax(&a.t.depth[pix], m);
        }
    } else if (PASS == PASS_COLOR) {
        bool vis = false;
        if (o.ok) {
            const uint32_t closest = a.t.depth[pix];
            vis = closest != 0u && o.nz >= crd::uint_to_depth(closest) * a.keep_scale;
        }
        const uint32_t peers = __match_any_sync(kFull, vis ? pix : kFull);
        if (vis) {
            const uint32_t r = __reduce_add_sync(peers, o.color & 0xffu);
            const uint32_t g = __reduce_add_sync(peers, (o.color >> 8) & 0xffu);
            const uint32_t b = __reduce_add_sync(peers, (o.color >> 16) & 0xffu);
            if (lane == __ffs(peers) - 1) color_global(a, pix, r, g, b, (uint32_t)__popc(peers));
        }
    } else {
        const uint32_t peers = __match_any_sync(kFull, o.ok ? pix : kFull);
        if (o.ok) {
            const uint32_t m = __reduce_max_sync(peers, o.depth);
            const uint32_t tied = __ballot_sync(peers, o.depth == m);
            if (o.depth == m) {
                const uint32_t mi = __reduce_min_sync(tied, o.pointIndex);
                if (lane == __ffs(tied) - 1) atomicMax(&a.t.nearest[pix], nearest_key(m, mi));
            }
        }
    }
}

// Tile path, radius 0: shared-memory accumulation (global fallback outside).
template <int PASS>
__device__ __forceinline__ void emit_tile(const RasterArgs &a, const ChunkRec &c,
                                          unsigned char *smem, const PointOut &o) {
    if (!o.ok) return;
    const int lx = o.ix - c.x0, ly = o.iy - c.y0;
    const bool inside = (unsigned)lx < (unsigned)c.tw && (unsigned)ly < (unsigned)c.th;
    const uint32_t pix = (uint32_t)(o.iy * a.u.width + o.ix);
    const int l = ly * c.tw + lx;
    if (PASS == PASS_DEPTH) {
        if (inside)
            atomicMax(reinterpret_cast<uint32_t *>(smem) + l, o.depth);
        else
            atomicMax(&a.t.depth[pix], o.depth);
    } else if (PASS == PASS_COLOR) {
        const uint32_t *sdep =
            reinterpret_cast<const uint32_t *>(smem + TileCfg<PASS_COLOR>::kPx * 16);
        const uint32_t closest = inside ? sdep[l] : a.t.depth[pix];
        if (closest == 0u || !(o.nz >= crd::uint_to_depth(closest) * a.keep_scale)) return;
        const uint32_t r = o.color & 0xffu, g = (o.color >> 8) & 0xffu,
                       b = (o.color >> 16) & 0xffu;
        if (inside) {
            unsigned long long *acc = reinterpret_cast<unsigned long long *>(smem) + 2 * l;
            atomicAdd(acc, (unsigned long long)r | ((unsigned long long)g << 32));
            atomicAdd(acc + 1, (unsigned long long)b | (1ull << 32));
        } else {
            color_global(a, pix, r, g, b, 1u);
        }
    } else {
        const unsigned long long k = nearest_key(o.depth, o.pointIndex);
        if (inside)
            atomicMax(reinterpret_cast<unsigned long long *>(smem) + l, k);
        else
            atomicMax(&a.t.nearest[pix], k);
    }
}

// General footprint (radius from pointFootprintRadius), global atomics.
template <int PASS>
__device__ __forceinline__ void emit_footprint(const RasterArgs &a, const BatchShared &sb,
                                               const PointOut &o) {
    if (!o.ok) return;
    const crd::PointSize ps{a.u.pointSizeMode, a.u.minimumPointSize, a.u.maximumPointSize,
                            a.u.pointSizeScale};
    const int rad =
        crd::footprint_radius(o.px, o.py, o.pz, sb.world, a.u.view, a.u.proj, a.u.height, ps);
    const int W = a.u.width, H = a.u.height;
    for (int oy = -rad; oy <= rad; ++oy) {
        for (int ox = -rad; ox <= rad; ++ox) {
            if (!crd::inside_footprint(ox, oy, rad)) continue;
            const int tx = o.ix + ox, ty = o.iy + oy;
            if (tx < 0 || tx >= W || ty < 0 || ty >= H) continue;
            const uint32_t pix = (uint32_t)(ty * W + tx);
            if (PASS == PASS_DEPTH) {
                atomicMax(&a.t.depth[pix], o.depth);
            } else if (PASS == PASS_COLOR) {
                const uint32_t closest = a.t.depth[pix];
                if (closest == 0u) continue;
                if (!(o.nz >= crd::uint_to_depth(closest) * a.keep_scale)) continue;
                color_global(a, pix, o.color & 0xffu, (o.color >> 8) & 0xffu,
                             (o.color >> 16) & 0xffu, 1u);
            } else {
                atomicMax(&a.t.nearest[pix], nearest_key(o.depth, o.pointIndex));
            }
        }
    }
}

// One point; every lane of the warp calls this (warp-uniform early outs).
template <int PASS>
__device__ __forceinline__ void do_point(const RasterArgs &a, const BatchShared &sb,
                                         unsigned char *smem, const ChunkRec &c, bool tiled,
                                         bool valid, uint32_t local, uint32_t lvl, uint32_t lo,
                                         uint32_t me, uint32_t hi, uint32_t color) {
    PointOut o;
    o.pointIndex = c.first + local;
    o.color = color;
    o.ok = valid && keep_point(a, c, o.pointIndex, lvl);
    if (!__any_sync(kFull, o.ok)) return;
    project_point<PASS>(a, sb, c, lo, me, hi, o);
    if (!__any_sync(kFull, o.ok)) return;
    if (!a.radius_zero)
        emit_footprint<PASS>(a, sb, o);
    else if (tiled)
        emit_tile<PASS>(a, c, smem, o);
    else
        emit_direct<PASS>(a, o);
}

template <int PASS>
__device__ __forceinline__ void tile_init(const RasterArgs &a, const ChunkRec &c,
                                          unsigned char *smem) {
    const int n = c.tw * c.th;
    for (int l = threadIdx.x; l < n; l += kThreads) {
        if (PASS == PASS_DEPTH) {
            reinterpret_cast<uint32_t *>(smem)[l] = 0u;
        } else if (PASS == PASS_COLOR) {
            unsigned long long *acc = reinterpret_cast<unsigned long long *>(smem);
            acc[2 * l] = 0ull;
            acc[2 * l + 1] = 0ull;
            const int gx = c.x0 + l % c.tw, gy = c.y0 + l / c.tw;
            reinterpret_cast<uint32_t *>(smem + TileCfg<PASS_COLOR>::kPx * 16)[l] =
                a.t.depth[gy * a.u.width + gx];
        } else {
            reinterpret_cast<unsigned long long *>(smem)[l] = 0ull;
        }
    }
}

template <int PASS>
__device__ __forceinline__ void tile_flush(const RasterArgs &a, const ChunkRec &c,
                                           const unsigned char *smem) {
    const int n = c.tw * c.th;
    for (int l = threadIdx.x; l < n; l += kThreads) {
        const uint32_t pix = (uint32_t)((c.y0 + l / c.tw) * a.u.width + c.x0 + l % c.tw);
        if (PASS == PASS_DEPTH) {
            const uint32_t v = reinterpret_cast<const uint32_t *>(smem)[l];
            if (v) atomicMax(&a.t.depth[pix], v);
        } else if (PASS == PASS_COLOR) {
            const unsigned long long *acc = reinterpret_cast<const unsigned long long *>(smem);
            const unsigned long long rg = acc[2 * l], bc = acc[2 * l + 1];
            const uint32_t cnt = (uint32_t)(bc >> 32);
            if (cnt) color_global(a, pix, (uint32_t)rg, (uint32_t)(rg >> 32), (uint32_t)bc, cnt);
        } else {
            const unsigned long long k = reinterpret_cast<const unsigned long long *>(smem)[l];
            if (k) atomicMax(&a.t.nearest[pix], k);
        }
    }
}

// 16-byte asynchronous global -> shared copy (cp.async), for the chunk record.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Persistent pass over the chunk records (static grid-stride schedule): the
// record of the CTA's next chunk is copied into shared memory with cp.async
// while the current chunk is processed.
template <int PASS>
__global__ void __launch_bounds__(kThreads) raster_kernel(RasterArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ BatchShared sb;
    __shared__ __align__(16) ChunkRec rec[2];
    const uint32_t nchunks = a.counters[CNT_CHUNKS];
    uint32_t k = blockIdx.x;
    if (k >= nchunks) return;
    if (threadIdx.x < 4) cp_async16(reinterpret_cast<uint4 *>(&rec[0]) + threadIdx.x,
                                    reinterpret_cast<const uint4 *>(a.chunks + k) + threadIdx.x);
    cp_async_commit();
    if (threadIdx.x == 0) sb.file = 0xffffffffu;
    int buf = 0;
    for (; k < nchunks; k += gridDim.x, buf ^= 1) {
        cp_async_wait_all();
        __syncthreads();  // rec[buf] complete; the previous chunk is fully done
        const ChunkRec c = rec[buf];
        const uint32_t kn = k + gridDim.x;
        if (kn < nchunks && threadIdx.x < 4)
            cp_async16(reinterpret_cast<uint4 *>(&rec[buf ^ 1]) + threadIdx.x,
                       reinterpret_cast<const uint4 *>(a.chunks + kn) + threadIdx.x);
        cp_async_commit();
        const bool new_file = c.file != sb.file;
        const bool tiled = a.use_tiles && a.radius_zero && c.tw > 0 &&
                           c.tw * c.th <= TileCfg<PASS>::kPx && c.tw * c.th <= (int)(2 * c.count);
        if (new_file || tiled) {
            __syncthreads();  // everyone has read sb.file
            if (new_file) {
                const cr_raster_file *file = &a.files[c.file];
                if (threadIdx.x < 16)
                    sb.T[threadIdx.x] = file->transform[threadIdx.x];
                else if (threadIdx.x < 32)
                    sb.world[threadIdx.x - 16] = file->world[threadIdx.x - 16];
                if (threadIdx.x == 0) sb.file = c.file;
            }
            if (tiled) tile_init<PASS>(a, c, smem);
            __syncthreads();
        }
        const bool need_med = c.level <= 1, need_high = c.level == 0;
        if ((c.first & 3u) == 0u) {
            // Four points per thread, 16-byte loads.
            const uint32_t nquads = (c.count + 3u) >> 2;
            for (uint32_t q0 = 0; q0 < nquads; q0 += kThreads) {
                const uint32_t q = q0 + threadIdx.x;
                const bool qv = q < nquads;
                const uint32_t base = c.first + 4u * q;
                uint32_t lv4 = 0;
                uint4 lo4 = make_uint4(0, 0, 0, 0), me4 = lo4, hi4 = lo4, co4 = lo4;
                if (qv) {
                    lv4 = __ldg(reinterpret_cast<const uint32_t *>(a.levels + base));
                    lo4 = __ldg(reinterpret_cast<const uint4 *>(a.low + base));
                    if (need_med) me4 = __ldg(reinterpret_cast<const uint4 *>(a.med + base));
                    if (need_high) hi4 = __ldg(reinterpret_cast<const uint4 *>(a.high + base));
                    if (PASS == PASS_COLOR)
                        co4 = __ldg(reinterpret_cast<const uint4 *>(a.colors + base));
                }
                const uint32_t l0 = 4u * q;
                do_point<PASS>(a, sb, smem, c, tiled, qv && l0 + 0 < c.count, l0 + 0,
                               lv4 & 0xffu, lo4.x, me4.x, hi4.x, co4.x);
                do_point<PASS>(a, sb, smem, c, tiled, qv && l0 + 1 < c.count, l0 + 1,
                               (lv4 >> 8) & 0xffu, lo4.y, me4.y, hi4.y, co4.y);
                do_point<PASS>(a, sb, smem, c, tiled, qv && l0 + 2 < c.count, l0 + 2,
                               (lv4 >> 16) & 0xffu, lo4.z, me4.z, hi4.z, co4.z);
                do_point<PASS>(a, sb, smem, c, tiled, qv && l0 + 3 < c.count, l0 + 3,
                               lv4 >> 24, lo4.w, me4.w, hi4.w, co4.w);
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
                const uint32_t co = (v && PASS == PASS_COLOR) ? a.colors[i] : 0u;
                do_point<PASS>(a, sb, smem, c, tiled, v, local, lv, lo, me, hi, co);
            }
        }
        if (tiled) {
            __syncthreads();
            tile_flush<PASS>(a, c, smem);
        }
    }
    cp_async_wait_all();
}

template <int PASS>
int blocks_per_sm_for() {
    int n = 0;
    cudaFuncSetAttribute(raster_kernel<PASS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         TileCfg<PASS>::kBytes);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, raster_kernel<PASS>, kThreads,
                                                      TileCfg<PASS>::kBytes) != cudaSuccess)
        n = 1;
    return n < 1 ? 1 : n;
}

}  // namespace

int raster_blocks_per_sm(int pass) {
    switch (pass) {
    case PASS_DEPTH: return blocks_per_sm_for<PASS_DEPTH>();
    case PASS_COLOR: return blocks_per_sm_for<PASS_COLOR>();
    default: return blocks_per_sm_for<PASS_NEAREST>();
    }
}

cr_status launch_raster(cr_cloud *cloud, RasterPass pass, const RasterUniforms &u,
                        const RasterTargets &t, cudaStream_t s) {
    RasterArgs a;
    a.chunks = cloud->d_chunks;
    a.files = cloud->d_files;
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
    cr_context *ctx = cloud->ctx;
    if (ctx->blocks_per_sm[pass] == 0) ctx->blocks_per_sm[pass] = raster_blocks_per_sm(pass);
    const int grid = ctx->sm_count * ctx->blocks_per_sm[pass];
    switch (pass) {
    case PASS_DEPTH:
        raster_kernel<PASS_DEPTH><<<grid, kThreads, TileCfg<PASS_DEPTH>::kBytes, s>>>(a);
        break;
    case PASS_COLOR:
        raster_kernel<PASS_COLOR><<<grid, kThreads, TileCfg<PASS_COLOR>::kBytes, s>>>(a);
        break;
    default:
        raster_kernel<PASS_NEAREST><<<grid, kThreads, TileCfg<PASS_NEAREST>::kBytes, s>>>(a);
        break;
    }
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}
