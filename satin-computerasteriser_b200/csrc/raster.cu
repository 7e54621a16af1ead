// raster.cu — the per-point passes of the compute rasteriser.
//
//   PASS_DEPTH   depthPassUpdate   (Pipelines/DepthPass/Shaders.metal:21-116)
//   PASS_COLOR   colorPassUpdate   (Pipelines/ColorPass/Shaders.metal:30-219,
//                                   integer R,G,B,count path)
//   PASS_NEAREST nearestDepthUpdate + nearestIndexUpdate
//                (Pipelines/NearestDepth/Shaders.metal:14-91,
//                 Pipelines/NearestIndex/Shaders.metal:14-94) fused into one
//                traversal: the key (depth << 32) | ~pointIndex is combined
//                with a 64-bit atomicMax, so the winner is the largest depth
//                and, among equal depths, the lowest point index — the same
//                pixel result as the reference's max pass followed by its
//                min-index pass over the tied points.
//
// Launch shape.  The reference dispatches one 128-thread group per survivor
// of the cull (indirect dispatch).  Here a persistent grid sized to fill
// every SM pulls survivors from the ordered cull list with an atomic work
// cursor (the cull publishes the count the cursor runs to, the CUDA
// counterpart of the indirect argument buffer).  Each CTA of 256 threads
// walks a batch's survivor prefix four points per thread with 16-byte loads
// of the level bytes and position / colour words.
//
// Atomics.  Lanes of a warp whose points land on the same pixel merge first
// (__match_any_sync + redux), and one lane issues the atomic with the merged
// value: max for depth, sums for R,G,B and the count.  Integer max and sum
// are associative and commutative, so the planes are bit-identical to a
// per-point atomic order.
#include "cr_device.cuh"
#include "cr_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kFull = 0xffffffffu;

struct RasterArgs {
    const cr_raster_batch *batches;
    const cr_raster_file *files;
    const cr_visible_batch *visible;
    uint32_t *counters;
    const uint32_t *low, *med, *high, *colors;
    const uint8_t *levels;
    RasterTargets t;
    RasterUniforms u;
    float keep_scale;  // 1 - depthTolerance
    int radius_zero;   // every footprint is a single pixel
};

struct BatchShared {
    float T[16];      // file.transform
    float world[16];  // file.world (footprint only)
};

struct BatchRegs {
    float minX, minY, minZ, qx, qy, qz, thr;
    uint32_t first, active, batchIndex;
    int level;
};

template <int PASS>
__device__ __forceinline__ void emit_single(const RasterArgs &a, bool ok, uint32_t pix,
                                            uint32_t depth, float ndcz, uint32_t color,
                                            uint32_t pointIndex) {
    const int lane = threadIdx.x & 31;
    if (PASS == PASS_DEPTH) {
        const uint32_t key = ok ? pix : kFull;
        const uint32_t peers = __match_any_sync(kFull, key);
        if (ok) {
            const uint32_t m = __reduce_max_sync(peers, depth);
            if (lane == __ffs(peers) - 1) atomicMax(&a.t.depth[pix], m);
        }
    } else if (PASS == PASS_COLOR) {
        bool vis = false;
        if (ok) {
            const uint32_t closest = a.t.depth[pix];
            vis = closest != 0u && ndcz >= crd::uint_to_depth(closest) * a.keep_scale;
        }
        const uint32_t key = vis ? pix : kFull;
        const uint32_t peers = __match_any_sync(kFull, key);
        if (vis) {
            const uint32_t r = __reduce_add_sync(peers, color & 0xffu);
            const uint32_t g = __reduce_add_sync(peers, (color >> 8) & 0xffu);
            const uint32_t b = __reduce_add_sync(peers, (color >> 16) & 0xffu);
            if (lane == __ffs(peers) - 1) {
                unsigned int *acc = reinterpret_cast<unsigned int *>(&a.t.accum[pix]);
                atomicAdd(acc + 0, r);
                atomicAdd(acc + 1, g);
                atomicAdd(acc + 2, b);
                atomicAdd(acc + 3, (uint32_t)__popc(peers));
            }
        }
    } else {
        const uint32_t key = ok ? pix : kFull;
        const uint32_t peers = __match_any_sync(kFull, key);
        if (ok) {
            const uint32_t m = __reduce_max_sync(peers, depth);
            const uint32_t tied = __ballot_sync(peers, depth == m);
            if (depth == m) {
                const uint32_t mi = __reduce_min_sync(tied, pointIndex);
                if (lane == __ffs(tied) - 1)
                    atomicMax(&a.t.nearest[pix],
                              ((unsigned long long)m << 32) | (unsigned long long)(~mi));
            }
        }
    }
}

template <int PASS>
__device__ __forceinline__ void emit_footprint(const RasterArgs &a, const BatchShared &sb, int ix,
                                               int iy, float px, float py, float pz,
                                               uint32_t depth, float ndcz, uint32_t color,
                                               uint32_t pointIndex) {
    const crd::PointSize ps{a.u.pointSizeMode, a.u.minimumPointSize, a.u.maximumPointSize,
                            a.u.pointSizeScale};
    const int rad =
        crd::footprint_radius(px, py, pz, sb.world, a.u.view, a.u.proj, a.u.height, ps);
    const int W = a.u.width, H = a.u.height;
    for (int oy = -rad; oy <= rad; ++oy) {
        for (int ox = -rad; ox <= rad; ++ox) {
            if (!crd::inside_footprint(ox, oy, rad)) continue;
            const int tx = ix + ox, ty = iy + oy;
            if (tx < 0 || tx >= W || ty < 0 || ty >= H) continue;
            const uint32_t pix = (uint32_t)(ty * W + tx);
            if (PASS == PASS_DEPTH) {
                atomicMax(&a.t.depth[pix], depth);
            } else if (PASS == PASS_COLOR) {
                const uint32_t closest = a.t.depth[pix];
                if (closest == 0u) continue;
                if (!(ndcz >= crd::uint_to_depth(closest) * a.keep_scale)) continue;
                unsigned int *acc = reinterpret_cast<unsigned int *>(&a.t.accum[pix]);
                atomicAdd(acc + 0, color & 0xffu);
                atomicAdd(acc + 1, (color >> 8) & 0xffu);
                atomicAdd(acc + 2, (color >> 16) & 0xffu);
                atomicAdd(acc + 3, 1u);
            } else {
                atomicMax(&a.t.nearest[pix],
                          ((unsigned long long)depth << 32) | (unsigned long long)(~pointIndex));
            }
        }
    }
}

// One point of the traversal shared by the three passes
// (DepthPass/Shaders.metal:168-234).  Every lane of the warp calls this with
// its own `valid` so the warp-level merge sees all 32 lanes.
template <int PASS>
__device__ __forceinline__ void do_point(const RasterArgs &a, const BatchShared &sb,
                                         const BatchRegs &br, bool valid, uint32_t local,
                                         uint32_t lvl, uint32_t lo, uint32_t me, uint32_t hi,
                                         uint32_t color) {
    const uint32_t pointIndex = br.first + local;
    bool ok = valid;
    const float pointLevel = (float)(lvl & 7u);
    const float dither = a.u.lodDither ? crd::hash_unit(pointIndex) : 0.5f;
    if (dither >= (br.thr - pointLevel) + 0.5f) ok = false;
    // decodePoint (Common.metal:89-117).
    uint32_t x, y, z;
    if (br.level == 0) {
        x = ((lo & 1023u) << 20) | ((me & 1023u) << 10) | (hi & 1023u);
        y = (((lo >> 10) & 1023u) << 20) | (((me >> 10) & 1023u) << 10) | ((hi >> 10) & 1023u);
        z = (((lo >> 20) & 1023u) << 20) | (((me >> 20) & 1023u) << 10) | ((hi >> 20) & 1023u);
    } else if (br.level == 1) {
        x = ((lo & 1023u) << 10) | (me & 1023u);
        y = (((lo >> 10) & 1023u) << 10) | ((me >> 10) & 1023u);
        z = (((lo >> 20) & 1023u) << 10) | ((me >> 20) & 1023u);
    } else {
        x = lo & 1023u;
        y = (lo >> 10) & 1023u;
        z = (lo >> 20) & 1023u;
    }
    const float px = (float)x * br.qx + br.minX;
    const float py = (float)y * br.qy + br.minY;
    const float pz = (float)z * br.qz + br.minZ;
    const crd::f4 clip = crd::mulp(sb.T, px, py, pz);
    if (clip.w <= 0.0f) ok = false;
    const float nx = clip.x / clip.w, ny = clip.y / clip.w, nz = clip.z / clip.w;
    if (nx < -1.0f || ny < -1.0f || nx > 1.0f || ny > 1.0f || nz > 1.0f) ok = false;
    if (PASS == PASS_NEAREST ? (nz <= 0.0f) : (nz < 0.0f)) ok = false;
    const int W = a.u.width, H = a.u.height;
    const int ix = (int)((nx * 0.5f + 0.5f) * (float)W);
    int iy = (int)((ny * 0.5f + 0.5f) * (float)H);
    if (ix < 0 || ix >= W || iy < 0 || iy >= H) ok = false;
    iy = H - 1 - iy;
    const uint32_t depth = crd::depth_to_uint(nz);
    uint32_t c = color;
    if (PASS == PASS_COLOR) {  // ColorPass/Shaders.metal:95-100
        if (a.u.colorizeChunks)
            c = br.batchIndex * 1234567u;
        else if (a.u.colorizeOverdraw)
            c = 0x00010101u;
    }
    if (a.radius_zero) {
        emit_single<PASS>(a, ok, (uint32_t)(iy * W + ix), depth, nz, c, pointIndex);
    } else if (ok) {
        emit_footprint<PASS>(a, sb, ix, iy, px, py, pz, depth, nz, c, pointIndex);
    }
}

template <int PASS>
__global__ void __launch_bounds__(kThreads) raster_kernel(RasterArgs a) {
    __shared__ BatchShared sb;
    __shared__ uint32_t s_item;
    const uint32_t nvis = a.counters[CNT_VISIBLE];
    uint32_t *cursor = &a.counters[PASS == PASS_COLOR ? CNT_WORK_COLOR : CNT_WORK_DEPTH];
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(cursor, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= nvis) break;
        const cr_visible_batch vb = a.visible[item];
        const cr_raster_batch b = a.batches[vb.batchIndex];
        const cr_raster_file *file = &a.files[b.fileIndex];
        if (threadIdx.x < 16)
            sb.T[threadIdx.x] = file->transform[threadIdx.x];
        else if (threadIdx.x < 32)
            sb.world[threadIdx.x - 16] = file->world[threadIdx.x - 16];
        BatchRegs br;
        br.minX = b.minX;
        br.minY = b.minY;
        br.minZ = b.minZ;
        // batchSize (Common.metal:81-83) / steps of the precision level.
        const float steps = vb.level == 0 ? 1073741824.0f : vb.level == 1 ? 1048576.0f : 1024.0f;
        br.qx = fmaxf(b.maxX - b.minX, 0.000001f) / steps;
        br.qy = fmaxf(b.maxY - b.minY, 0.000001f) / steps;
        br.qz = fmaxf(b.maxZ - b.minZ, 0.000001f) / steps;
        br.thr = vb.lodThreshold;
        br.first = b.firstPoint;
        br.active = vb.activePoints;
        br.batchIndex = vb.batchIndex;
        br.level = vb.level;
        __syncthreads();

        const bool need_med = br.level <= 1, need_high = br.level == 0;
        if ((br.first & 3u) == 0u) {
            // Four points per thread, 16-byte loads.
            const uint32_t nquads = (br.active + 3u) >> 2;
            for (uint32_t q0 = 0; q0 < nquads; q0 += kThreads) {
                const uint32_t q = q0 + threadIdx.x;
                const bool qv = q < nquads;
                const uint32_t base = br.first + 4u * q;
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
                do_point<PASS>(a, sb, br, qv && l0 + 0 < br.active, l0 + 0, lv4 & 0xffu, lo4.x,
                               me4.x, hi4.x, co4.x);
                do_point<PASS>(a, sb, br, qv && l0 + 1 < br.active, l0 + 1, (lv4 >> 8) & 0xffu,
                               lo4.y, me4.y, hi4.y, co4.y);
                do_point<PASS>(a, sb, br, qv && l0 + 2 < br.active, l0 + 2, (lv4 >> 16) & 0xffu,
                               lo4.z, me4.z, hi4.z, co4.z);
                do_point<PASS>(a, sb, br, qv && l0 + 3 < br.active, l0 + 3, lv4 >> 24, lo4.w,
                               me4.w, hi4.w, co4.w);
            }
        } else {
            // Unaligned slot base (pointsPerBatch not a multiple of 4): one point per thread.
            for (uint32_t l0 = 0; l0 < br.active; l0 += kThreads) {
                const uint32_t local = l0 + threadIdx.x;
                const bool v = local < br.active;
                const uint32_t i = br.first + (v ? local : 0u);
                const uint32_t lv = v ? a.levels[i] : 0u;
                const uint32_t lo = v ? a.low[i] : 0u;
                const uint32_t me = (v && need_med) ? a.med[i] : 0u;
                const uint32_t hi = (v && need_high) ? a.high[i] : 0u;
                const uint32_t co = (v && PASS == PASS_COLOR) ? a.colors[i] : 0u;
                do_point<PASS>(a, sb, br, v, local, lv, lo, me, hi, co);
            }
        }
        __syncthreads();
    }
}

template <int PASS>
int blocks_per_sm_for() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, raster_kernel<PASS>, kThreads, 0) !=
        cudaSuccess)
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
    a.batches = cloud->d_batches;
    a.files = cloud->d_files;
    a.visible = cloud->d_visible;
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
    static int bps[3] = {0, 0, 0};
    if (bps[pass] == 0) bps[pass] = raster_blocks_per_sm(pass);
    const int grid = cloud->ctx->sm_count * bps[pass];
    switch (pass) {
    case PASS_DEPTH: raster_kernel<PASS_DEPTH><<<grid, kThreads, 0, s>>>(a); break;
    case PASS_COLOR: raster_kernel<PASS_COLOR><<<grid, kThreads, 0, s>>>(a); break;
    default: raster_kernel<PASS_NEAREST><<<grid, kThreads, 0, s>>>(a); break;
    }
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}
