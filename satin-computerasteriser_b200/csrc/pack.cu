// pack.cu — the GPU packer: raw points -> Morton-ordered, LOD-bucketed,
// split-precision batches written straight into a cloud's slot pool.
//
// Restates GPUPacker.encodePack (GPUPacker.swift:204-392) and its kernels
// (Pipelines/GPUPacker/Shaders.metal:41-414), which in turn mirror the CPU
// PackedPointCloudFixtures.pack (PackedPointCloudFixtures.swift:30-344):
//   1 bounds        global AABB (order-preserving flipped-bit min/max)
//   2 morton        10 bits/axis (30-bit key) or 21 bits/axis (63-bit key)
//   3 sort          stable LSD radix of (key, input index), one read of the
//                   keys for every digit's histogram, then one single-sweep
//                   pass per digit (decoupled look-back; the first pass
//                   makes the input indices)                     [radix.cu]
//   4 gather        positions in Morton order, levels = maxLevel
//   5 LOD           per level, coarsest first: dense voxel grid, atomicMin
//                   of the Morton position claims a voxel for the first
//                   eligible point in sorted order (the CPU's "first point
//                   to occupy an empty voxel"); the claims of a level ride
//                   in the kernel before (the gather, or the previous
//                   level's assignment)
//   6 batches       one CTA per batch, a contiguous segment per warp:
//                   AABB, level counts, stable level-ascending scatter (warp
//                   ballots, no block barrier), RasterBatch with the
//                   cumulative LOD counts
//   7 emit          gather in final order, 30-bit quantisation into three
//                   10-bit/axis words, colours, levels, source indices.
// Host-side float math (scale, voxel sizes, grid dims) is compiled without
// contraction and uses the same operation order as the CPU oracle.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cr_device.cuh"
#include "cr_internal.h"
#include "cr_pack.h"

namespace {

constexpr int kThreads = 256;
constexpr uint64_t kLodCellCap = 1ull << 28;  // 1 GiB of uint32 voxels

__host__ __device__ __forceinline__ uint32_t flip(float f) {
#ifdef __CUDA_ARCH__
    const uint32_t b = __float_as_uint(f);
#else
    uint32_t b;
    std::memcpy(&b, &f, 4);
#endif
    return b ^ ((b >> 31) ? 0xffffffffu : 0x80000000u);
}
__host__ __device__ __forceinline__ float unflip(uint32_t u) {
    const uint32_t b = u ^ ((u >> 31) ? 0x80000000u : 0xffffffffu);
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float f;
    std::memcpy(&f, &b, 4);
    return f;
#endif
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
    uint32_t x = v & 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__device__ __forceinline__ unsigned long long spread21(unsigned long long v) {
    unsigned long long x = v & 0x1fffffull;
    x = (x | (x << 32)) & 0x1f00000000ffffull;
    x = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

struct LoadArgs {
    const uint8_t *pos;
    uint32_t pos_stride;
    const uint8_t *col;
    uint32_t col_stride;
    int col_format;
};

// Stage 0: raw input -> float4 positions + packed RGBA8 (GPUPacker/Shaders.metal:219-235
// colour rule: uint(clamp(c, 0, 1) * 255), truncating).
// One 16-byte record per point: x, y, z and the packed RGBA8 colour's bits
// in w (moved, never computed on), so the Morton-order gather brings both
// with one access.
__global__ void __launch_bounds__(kThreads)
    pack_load(LoadArgs a, uint64_t n, float4 *__restrict__ pos) {
    const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const float *p = reinterpret_cast<const float *>(a.pos + i * a.pos_stride);
    uint32_t col;
    if (a.col_format == 1) {
        col = *reinterpret_cast<const uint32_t *>(a.col + i * a.col_stride);
    } else {
        const float *c = reinterpret_cast<const float *>(a.col + i * a.col_stride);
        const uint32_t r = (uint32_t)(fminf(fmaxf(c[0], 0.0f), 1.0f) * 255.0f);
        const uint32_t g = (uint32_t)(fminf(fmaxf(c[1], 0.0f), 1.0f) * 255.0f);
        const uint32_t b = (uint32_t)(fminf(fmaxf(c[2], 0.0f), 1.0f) * 255.0f);
        const uint32_t al = (uint32_t)(fminf(fmaxf(c[3], 0.0f), 1.0f) * 255.0f);
        col = r | (g << 8) | (b << 16) | (al << 24);
    }
    pos[i] = make_float4(p[0], p[1], p[2], __uint_as_float(col));
}

// Stage 1: global bounds (packBounds, GPUPacker/Shaders.metal:71-105).
__global__ void __launch_bounds__(kThreads)
    pack_bounds(const float4 *__restrict__ pos, uint64_t n, uint32_t *__restrict__ bounds) {
    uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * kThreads) {
        const float4 p = pos[i];
        const uint32_t f[3] = {flip(p.x), flip(p.y), flip(p.z)};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = min(mn[k], f[k]);
            mx[k] = max(mx[k], f[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const uint32_t a = __reduce_min_sync(0xffffffffu, mn[k]);
        const uint32_t b = __reduce_max_sync(0xffffffffu, mx[k]);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&bounds[k], a);
            atomicMax(&bounds[3 + k], b);
        }
    }
}

struct MortonArgs {
    float bmin[3];
    float scale[3];
    float top;
};

// Stage 2: Morton key (packMorton, GPUPacker/Shaders.metal:109-126); the
// identity index the reference writes beside it is made by the sort's first
// pass instead.
template <typename K>
__global__ void __launch_bounds__(kThreads)
    pack_morton(const float4 *__restrict__ pos, uint64_t n, MortonArgs m, K *__restrict__ keys) {
    const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    const uint32_t qx = (uint32_t)fminf(fmaxf((p.x - m.bmin[0]) * m.scale[0], 0.0f), m.top);
    const uint32_t qy = (uint32_t)fminf(fmaxf((p.y - m.bmin[1]) * m.scale[1], 0.0f), m.top);
    const uint32_t qz = (uint32_t)fminf(fmaxf((p.z - m.bmin[2]) * m.scale[2], 0.0f), m.top);
    if (sizeof(K) == 8)
        keys[i] = (K)((spread21(qx) << 2) | (spread21(qy) << 1) | spread21(qz));
    else
        keys[i] = (K)((spread10(qx) << 2) | (spread10(qy) << 1) | spread10(qz));
}

// Stage 4: gather into Morton order, all levels at maxLevel (packLODInit).
__global__ void __launch_bounds__(kThreads)
    pack_gather(const float4 *__restrict__ pos, const uint32_t *__restrict__ idx, uint64_t n,
                float4 *__restrict__ sorted, uint8_t *__restrict__ lv, uint8_t max_level) {
    const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    sorted[i] = pos[idx[i]];
    lv[i] = max_level;
}

struct LodArgs {
    float bmin[3];
    float inv;
    uint32_t dims[3];
    uint8_t max_level;
    uint8_t level;
};

__device__ __forceinline__ uint64_t lod_cell(const float4 &p, const LodArgs &a) {
    const float lx = (p.x - a.bmin[0]) * a.inv;
    const float ly = (p.y - a.bmin[1]) * a.inv;
    const float lz = (p.z - a.bmin[2]) * a.inv;
    const uint32_t cx = min((uint32_t)max(0, (int)floorf(lx)), a.dims[0] - 1u);
    const uint32_t cy = min((uint32_t)max(0, (int)floorf(ly)), a.dims[1] - 1u);
    const uint32_t cz = min((uint32_t)max(0, (int)floorf(lz)), a.dims[2] - 1u);
    return (uint64_t)cx + (uint64_t)a.dims[0] * ((uint64_t)cy + (uint64_t)a.dims[1] * cz);
}

// Stage 5 (packLODClaim / packLODAssign, GPUPacker/Shaders.metal:337-371).
// The points are in Morton order, so neighbouring lanes often share a cell;
// lanes carry increasing indices, so the lowest lane of each group of lanes
// with the same cell holds the group's minimum and alone does the atomicMin
// (the grid ends the same: min is order-independent).  The last level's
// assignment:
__global__ void __launch_bounds__(kThreads)
    pack_lod_assign(const float4 *__restrict__ sorted, uint8_t *__restrict__ lv, uint64_t n,
                    LodArgs a, const uint32_t *__restrict__ grid) {
    const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    if (i >= n || lv[i] != a.max_level) return;
    if (grid[lod_cell(sorted[i], a)] == (uint32_t)i) lv[i] = a.level;
}

// The claims are fused into the kernels that read the Morton-ordered points
// anyway: the gather also claims the coarsest level (every point is still
// unassigned there), and the assignment of level L also claims level L + 1
// for the points it leaves unassigned (each level has its own grid), so the
// points are read once per level instead of twice.
__device__ __forceinline__ void lod_claim_one(bool part, const float4 &p, uint32_t i,
                                              const LodArgs &a, uint32_t *grid) {
    const unsigned act = __ballot_sync(0xffffffffu, part);
    if (!part) return;
    const uint64_t cell = lod_cell(p, a);
    const unsigned same = __match_any_sync(act, (unsigned long long)cell);
    if ((int)(__ffs(same) - 1) == (int)(threadIdx.x & 31u)) atomicMin(&grid[cell], i);
}

__global__ void __launch_bounds__(kThreads)
    pack_gather_claim(const float4 *__restrict__ pos, const uint32_t *__restrict__ idx, uint64_t n,
                      float4 *__restrict__ sorted, uint8_t *__restrict__ lv, uint8_t max_level,
                      LodArgs a0, uint32_t *__restrict__ grid0) {
    const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    const bool v = i < n;
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
    if (v) {
        p = pos[idx[i]];
        sorted[i] = p;
        lv[i] = max_level;
    }
    lod_claim_one(v, p, (uint32_t)i, a0, grid0);
}

__global__ void __launch_bounds__(kThreads)
    pack_lod_assign_claim(const float4 *__restrict__ sorted, uint8_t *__restrict__ lv, uint64_t n,
                          LodArgs a, const uint32_t *__restrict__ grid, LodArgs next,
                          uint32_t *__restrict__ grid_next) {
    const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    const bool v = i < n && lv[i] == a.max_level;
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
    bool left = false;
    if (v) {
        p = sorted[i];
        if (grid[lod_cell(p, a)] == (uint32_t)i)
            lv[i] = a.level;
        else
            left = true;
    }
    lod_claim_one(left, p, (uint32_t)i, next, grid_next);
}

// Stage 6: per batch AABB + stable level bucketing + RasterBatch
// (packBatchAABB + packBucketLOD, GPUPacker/Shaders.metal:243-284, 383-414).
// One CTA per batch; each warp owns a contiguous segment of the batch's
// points.  Pass 1: the AABB and the warp's per-level counts (ballots).  The
// counts give every warp its first slot per level (the batch's exclusive
// level prefix plus the counts of the warps before it), so pass 2 needs no
// block barrier: each warp walks its segment in order, 32 points a round,
// placing each point after the earlier points of its level (ballot rank).
// Both passes load four rounds ahead.
constexpr int kBatchRounds = 4;
__global__ void __launch_bounds__(kThreads)
    pack_batches(const float4 *__restrict__ sorted, const uint8_t *__restrict__ lv, uint64_t n,
                 uint32_t ppb, uint32_t first_slot, cr_raster_batch *__restrict__ batches,
                 uint32_t *__restrict__ perm, uint8_t *__restrict__ lv_out) {
    constexpr int kWarps = kThreads / 32;
    constexpr unsigned kFull = 0xffffffffu;
    __shared__ uint32_t red[6][kWarps];
    __shared__ uint32_t wcnt[kWarps][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const uint64_t start = (uint64_t)blockIdx.x * ppb;
    const uint64_t end = (start + ppb < n) ? start + ppb : n;
    const uint32_t total = (uint32_t)(end - start);
    const uint32_t seg = (total + kWarps - 1u) / kWarps;
    const uint64_t s0 = start + min((uint64_t)total, (uint64_t)warp * seg);
    const uint64_t s1 = start + min((uint64_t)total, (uint64_t)(warp + 1) * seg);
    // 1. AABB and level counts of the warp's segment.
    uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    uint32_t c[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
    for (uint64_t r0 = s0; r0 < s1; r0 += 32u * kBatchRounds) {
        float4 p[kBatchRounds];
        uint32_t l[kBatchRounds];
#pragma unroll
        for (int k = 0; k < kBatchRounds; ++k) {
            const uint64_t i = r0 + 32u * k + lane;
            l[k] = i < s1 ? (lv[i] & 7u) : 8u;
            p[k] = i < s1 ? sorted[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < kBatchRounds; ++k) {
            if (l[k] < 8u) {
                const uint32_t f[3] = {flip(p[k].x), flip(p[k].y), flip(p[k].z)};
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    mn[a] = min(mn[a], f[a]);
                    mx[a] = max(mx[a], f[a]);
                }
            }
#pragma unroll
            for (int L = 0; L < 8; ++L) c[L] += __popc(__ballot_sync(kFull, l[k] == (uint32_t)L));
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const uint32_t x = __reduce_min_sync(kFull, mn[a]);
        const uint32_t y = __reduce_max_sync(kFull, mx[a]);
        if (lane == 0) {
            red[a][warp] = x;
            red[3 + a][warp] = y;
        }
    }
    if (lane < 8) {
        uint32_t mine = 0;
#pragma unroll
        for (int L = 0; L < 8; ++L)
            if (lane == L) mine = c[L];
        wcnt[warp][lane] = mine;
    }
    __syncthreads();
    // 2. This warp's first slot (from the batch start) per level.
    uint32_t run[8], cum[8];
    {
        uint32_t acc = 0;
#pragma unroll
        for (int L = 0; L < 8; ++L) {
            uint32_t tot = 0, before = 0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                const uint32_t x = wcnt[w][L];
                tot += x;
                if (w < warp) before += x;
            }
            run[L] = acc + before;
            acc += tot;
            cum[L] = acc;
        }
    }
    if (threadIdx.x == 0) {
        uint32_t m[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
        for (int w = 0; w < kWarps; ++w)
            for (int a = 0; a < 3; ++a) {
                m[a] = min(m[a], red[a][w]);
                m[3 + a] = max(m[3 + a], red[3 + a][w]);
            }
        cr_raster_batch rb;
        rb.state = 1;
        rb.minX = unflip(m[0]);
        rb.minY = unflip(m[1]);
        rb.minZ = unflip(m[2]);
        rb.maxX = unflip(m[3]);
        rb.maxY = unflip(m[4]);
        rb.maxZ = unflip(m[5]);
        rb.numPoints = total;
        rb.firstPoint = (first_slot + blockIdx.x) * ppb;
        rb.fileIndex = 0;
        rb.lodCum01 = cum[0] | (cum[1] << 16);
        rb.lodCum23 = cum[2] | (cum[3] << 16);
        rb.lodCum45 = cum[4] | (cum[5] << 16);
        rb.lodCum67 = cum[6] | (cum[7] << 16);
        rb.padding7 = 0;
        rb.padding8 = 0;
        batches[blockIdx.x] = rb;
    }
    // 3. Stable bucketing of the warp's segment.
    for (uint64_t r0 = s0; r0 < s1; r0 += 32u * kBatchRounds) {
        uint32_t raw[kBatchRounds];
#pragma unroll
        for (int k = 0; k < kBatchRounds; ++k) {
            const uint64_t i = r0 + 32u * k + lane;
            raw[k] = i < s1 ? (uint32_t)lv[i] : 0xffu;
        }
#pragma unroll
        for (int k = 0; k < kBatchRounds; ++k) {
            const uint64_t i = r0 + 32u * k + lane;
            const bool v = i < s1;
            const uint32_t l = v ? (raw[k] & 7u) : 8u;
            uint32_t dst = 0;
#pragma unroll
            for (int L = 0; L < 8; ++L) {
                const uint32_t b = __ballot_sync(kFull, l == (uint32_t)L);
                if (l == (uint32_t)L) dst = run[L] + __popc(b & lt);
                run[L] += __popc(b);
            }
            if (v && dst < total) {  // always true: the ranks come from the same levels
                perm[start + dst] = (uint32_t)i;
                lv_out[start + dst] = (uint8_t)raw[k];
            }
        }
    }
}

// Stage 7: final order, quantisation (packQuantize, GPUPacker/Shaders.metal:288-309).
__global__ void __launch_bounds__(kThreads)
    pack_emit(uint64_t n, uint32_t ppb, const uint32_t *__restrict__ perm,
              const uint32_t *__restrict__ idx_sorted, const float4 *__restrict__ sorted,
              const uint8_t *__restrict__ lv_out,
              const cr_raster_batch *__restrict__ batches, uint32_t *__restrict__ low,
              uint32_t *__restrict__ med, uint32_t *__restrict__ high,
              uint32_t *__restrict__ colors, uint8_t *__restrict__ levels,
              uint32_t *__restrict__ src_out) {
    const uint64_t j = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    if (j >= n) return;
    // perm only reorders points within their batch (level bucketing), so
    // the Morton-ordered arrays are read nearly in order.
    const uint32_t pj = perm[j];
    if (pj >= n) return;  // unreachable for a complete permutation
    const float4 p = sorted[pj];
    const cr_raster_batch &b = batches[j / ppb];
    const float sx = fmaxf(b.maxX - b.minX, 0.000001f);
    const float sy = fmaxf(b.maxY - b.minY, 0.000001f);
    const float sz = fmaxf(b.maxZ - b.minZ, 0.000001f);
    const float nx = fminf(fmaxf((p.x - b.minX) / sx, 0.0f), 0.99999994f);
    const float ny = fminf(fmaxf((p.y - b.minY) / sy, 0.0f), 0.99999994f);
    const float nz = fminf(fmaxf((p.z - b.minZ) / sz, 0.0f), 0.99999994f);
    // Float(2^30 - 1) rounds to 2^30 in f32.
    const uint32_t qx = (uint32_t)(nx * 1073741824.0f);
    const uint32_t qy = (uint32_t)(ny * 1073741824.0f);
    const uint32_t qz = (uint32_t)(nz * 1073741824.0f);
    low[j] = ((qx >> 20) & 1023u) | (((qy >> 20) & 1023u) << 10) | (((qz >> 20) & 1023u) << 20);
    med[j] = ((qx >> 10) & 1023u) | (((qy >> 10) & 1023u) << 10) | (((qz >> 10) & 1023u) << 20);
    high[j] = (qx & 1023u) | ((qy & 1023u) << 10) | ((qz & 1023u) << 20);
    colors[j] = __float_as_uint(p.w);
    levels[j] = lv_out[j];
    if (src_out) src_out[j] = idx_sorted[pj];
}

unsigned grid_for(uint64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

template <typename T>
cr_status grow(T **p, uint64_t &cap, uint64_t want_elems) {
    if (*p && cap >= want_elems) return CR_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    cudaError_t e = cudaMalloc((void **)p, std::max<uint64_t>(want_elems, 1) * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        cap = 0;
        return cri::cuda_fail(e, "cudaMalloc (pack scratch)");
    }
    cap = want_elems;
    return CR_OK;
}

// Keys are sized for 64-bit words so either key width fits.
cr_status ensure_points(PackScratch &s, uint64_t n) {
    if (s.cap_points >= n && s.keys[0]) return CR_OK;
    pack_scratch_free(s);
    const uint64_t m = std::max<uint64_t>(n, 1) + 64;
    cudaError_t e;
#define ALLOC(ptr, bytes)                                                   \
    do {                                                                    \
        e = cudaMalloc((void **)&(ptr), (bytes));                           \
        if (e != cudaSuccess) {                                             \
            pack_scratch_free(s);                                           \
            return cri::cuda_fail(e, "cudaMalloc (pack scratch)");          \
        }                                                                   \
    } while (0)
    ALLOC(s.pos, m * sizeof(float4));
    ALLOC(s.keys[0], m * 8);
    ALLOC(s.keys[1], m * 8);
    ALLOC(s.idx[0], m * 4);
    ALLOC(s.idx[1], m * 4);
    ALLOC(s.sorted, m * sizeof(float4));
    ALLOC(s.lv_morton, (m + 15) & ~15ull);
    ALLOC(s.lv_out, (m + 15) & ~15ull);
    ALLOC(s.perm, m * 4);
    ALLOC(s.src_idx, m * 4);
    ALLOC(s.bounds, 8 * 4);
#undef ALLOC
    s.cap_points = n;
    return CR_OK;
}

}  // namespace

void pack_scratch_free(PackScratch &s) {
    void *ptrs[] = {s.raw, s.pos, s.keys[0], s.keys[1], s.idx[0], s.idx[1], s.sorted,
                    s.lv_morton, s.lv_out, s.perm, s.grid, s.bounds, s.src_idx};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    radix_scratch_free(s.radix);
    s = PackScratch{};
}

// Packs `count` points into slots [first_slot, first_slot + ceil(count/ppb)) of
// the cloud's pool.  Enqueues on the context stream; one synchronisation reads
// the global bounds back to size the Morton scale and the LOD grid.
cr_status pack_run(cr_context *ctx, cr_cloud *cloud, const cr_pack_input *in, uint64_t count,
                   const cr_pack_params *prm, int on_device, uint32_t first_slot,
                   uint32_t *src_idx_host) {
    cudaStream_t s = ctx->stream;
    PackScratch &sc = *ctx->pack;
    const bool wide = prm->mortonBits == 21;
    cr_status st = ensure_points(sc, count);
    if (st) return st;
    const uint32_t ppb = cloud->cap.pointsPerBatch;
    const uint32_t nb = (uint32_t)((count + ppb - 1) / ppb);

    // Stage 0: stage host input (one copy when the colour sits inside the position record).
    LoadArgs la;
    la.pos_stride = in->positionStrideBytes;
    la.col_stride = in->colorStrideBytes;
    la.col_format = in->colorFormat;
    const uint64_t csize = in->colorFormat == CR_COLOR_RGBA8 ? 4 : 16;
    if (on_device) {
        la.pos = static_cast<const uint8_t *>(in->positions);
        la.col = static_cast<const uint8_t *>(in->colors);
    } else {
        const uint8_t *hp = static_cast<const uint8_t *>(in->positions);
        const uint8_t *hc = static_cast<const uint8_t *>(in->colors);
        const uint64_t pbytes = (count - 1) * in->positionStrideBytes + 12;
        const uint64_t cbytes = (count - 1) * in->colorStrideBytes + csize;
        const bool inside = hc >= hp && in->colorStrideBytes == in->positionStrideBytes &&
                            (uint64_t)(hc - hp) + csize <= in->positionStrideBytes;
        const uint64_t need = inside ? std::max(pbytes, (uint64_t)(hc - hp) + cbytes)
                                     : ((pbytes + 255) & ~255ull) + cbytes;
        if ((st = grow(reinterpret_cast<uint8_t **>(&sc.raw), sc.cap_raw_bytes, need))) return st;
        uint8_t *raw = static_cast<uint8_t *>(sc.raw);
        if (inside) {
            CR_CUDA(cudaMemcpyAsync(raw, hp, need, cudaMemcpyHostToDevice, s));
            la.pos = raw;
            la.col = raw + (hc - hp);
        } else {
            const uint64_t coff = (pbytes + 255) & ~255ull;
            CR_CUDA(cudaMemcpyAsync(raw, hp, pbytes, cudaMemcpyHostToDevice, s));
            CR_CUDA(cudaMemcpyAsync(raw + coff, hc, cbytes, cudaMemcpyHostToDevice, s));
            la.pos = raw;
            la.col = raw + coff;
        }
    }
    // Device-resident 16-byte records {x, y, z, rgba8} already have the
    // layout of the staged positions: read them in place.
    const bool in_place = on_device && in->positionStrideBytes == 16 &&
                          in->colorStrideBytes == 16 && in->colorFormat == CR_COLOR_RGBA8 &&
                          static_cast<const uint8_t *>(in->colors) ==
                              static_cast<const uint8_t *>(in->positions) + 12 &&
                          ((uintptr_t)in->positions & 15) == 0;
    const float4 *pos = in_place ? static_cast<const float4 *>(in->positions) : sc.pos;
    if (!in_place) {
        pack_load<<<grid_for(count), kThreads, 0, s>>>(la, count, sc.pos);
        CR_CUDA(cudaGetLastError());
    }

    // Stage 1: bounds, read back once.
    const uint32_t binit[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    CR_CUDA(cudaMemcpyAsync(sc.bounds, binit, sizeof(binit), cudaMemcpyHostToDevice, s));
    pack_bounds<<<std::min<unsigned>(grid_for(count), (unsigned)ctx->sm_count * 8), kThreads, 0,
                  s>>>(pos, count, sc.bounds);
    CR_CUDA(cudaGetLastError());
    uint32_t bflip[6];
    CR_CUDA(cudaMemcpyAsync(bflip, sc.bounds, sizeof(bflip), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    float bmin[3], bmax[3], ext[3];
    for (int k = 0; k < 3; ++k) {
        bmin[k] = unflip(bflip[k]);
        bmax[k] = unflip(bflip[3 + k]);
        ext[k] = std::fmax(bmax[k] - bmin[k], 0.000001f);
    }

    // Stage 2-3: Morton keys, stable sort.
    MortonArgs ma;
    ma.top = wide ? 2097151.0f : 1023.0f;
    for (int k = 0; k < 3; ++k) {
        ma.bmin[k] = bmin[k];
        ma.scale[k] = ma.top / ext[k];
    }
    bool in_alt = false;
    if (wide) {
        auto *k0 = static_cast<unsigned long long *>(sc.keys[0]);
        auto *k1 = static_cast<unsigned long long *>(sc.keys[1]);
        pack_morton<unsigned long long><<<grid_for(count), kThreads, 0, s>>>(pos, count, ma, k0);
        CR_CUDA(cudaGetLastError());
        st = radix_sort_pairs<unsigned long long>(k0, sc.idx[0], k1, sc.idx[1], count, 63, true,
                                                  sc.radix, ctx->d_status, ctx->sm_count, s,
                                                  &in_alt);
    } else {
        auto *k0 = static_cast<uint32_t *>(sc.keys[0]);
        auto *k1 = static_cast<uint32_t *>(sc.keys[1]);
        pack_morton<uint32_t><<<grid_for(count), kThreads, 0, s>>>(pos, count, ma, k0);
        CR_CUDA(cudaGetLastError());
        st = radix_sort_pairs<uint32_t>(k0, sc.idx[0], k1, sc.idx[1], count, 30, true, sc.radix,
                                        ctx->d_status, ctx->sm_count, s, &in_alt);
    }
    if (st) return st;
    const uint32_t *idx_sorted = sc.idx[in_alt ? 1 : 0];

    // Stage 4-5: gather, LOD levels (each level its own dense grid).
    const int L = std::max(1, std::min(prm->lodLevels, 8));
    const int divs = std::max(1, prm->coarseVoxelDivisions);
    const uint8_t max_level = (uint8_t)(L - 1);
    if (L == 1) {
        pack_gather<<<grid_for(count), kThreads, 0, s>>>(pos, idx_sorted, count, sc.sorted,
                                                         sc.lv_morton, max_level);
        CR_CUDA(cudaGetLastError());
    } else {
        const float longest = std::fmax(ext[0], std::fmax(ext[1], ext[2]));
        const float base_voxel = longest / (float)divs;
        std::vector<LodArgs> la_(L - 1);
        std::vector<uint64_t> goff(L);
        goff[0] = 0;
        for (int level = 0; level < L - 1; ++level) {
            LodArgs &a = la_[level];
            const float voxel = base_voxel * std::pow(0.5f, (float)level);
            a.inv = 1.0f / std::fmax(voxel, 0.000001f);
            uint64_t cells = 1;
            for (int k = 0; k < 3; ++k) {
                a.bmin[k] = bmin[k];
                const float d = std::floor(ext[k] * a.inv);
                if (!(d < 2097151.0f))
                    return cri::fail(CR_ERR_CAPACITY, "LOD grid exceeds 2^21 cells per axis");
                a.dims[k] = (uint32_t)d + 1u;
                cells *= a.dims[k];
            }
            if (cells > kLodCellCap)
                return cri::fail(CR_ERR_CAPACITY,
                                 "LOD grid of " + std::to_string(cells) + " cells exceeds the cap");
            a.max_level = max_level;
            a.level = (uint8_t)level;
            goff[level + 1] = goff[level] + cells;
        }
        if ((st = grow(&sc.grid, sc.cap_grid, goff[L - 1]))) return st;
        CR_CUDA(cudaMemsetAsync(sc.grid, 0xff, goff[L - 1] * 4, s));
        pack_gather_claim<<<grid_for(count), kThreads, 0, s>>>(
            pos, idx_sorted, count, sc.sorted, sc.lv_morton, max_level, la_[0], sc.grid);
        CR_CUDA(cudaGetLastError());
        for (int level = 0; level + 1 < L - 1; ++level) {
            pack_lod_assign_claim<<<grid_for(count), kThreads, 0, s>>>(
                sc.sorted, sc.lv_morton, count, la_[level], sc.grid + goff[level],
                la_[level + 1], sc.grid + goff[level + 1]);
            CR_CUDA(cudaGetLastError());
        }
        pack_lod_assign<<<grid_for(count), kThreads, 0, s>>>(sc.sorted, sc.lv_morton, count,
                                                             la_[L - 2], sc.grid + goff[L - 2]);
        CR_CUDA(cudaGetLastError());
    }

    // Stage 6-7: batches, final order, quantisation into the pool.
    cr_raster_batch *dst_batches = cloud->d_batches + first_slot;
    pack_batches<<<nb, kThreads, 0, s>>>(sc.sorted, sc.lv_morton, count, ppb, first_slot,
                                         dst_batches, sc.perm, sc.lv_out);
    CR_CUDA(cudaGetLastError());
    const uint64_t p0 = (uint64_t)first_slot * ppb;
    pack_emit<<<grid_for(count), kThreads, 0, s>>>(
        count, ppb, sc.perm, idx_sorted, sc.sorted, sc.lv_out, dst_batches,
        cloud->d_low + p0,
        cloud->d_med + p0, cloud->d_high + p0, cloud->d_colors + p0, cloud->d_levels + p0,
        src_idx_host ? sc.src_idx : nullptr);  // source indices only when asked for
    CR_CUDA(cudaGetLastError());
    if (src_idx_host)
        CR_CUDA(cudaMemcpyAsync(src_idx_host, sc.src_idx, count * 4, cudaMemcpyDeviceToHost, s));
    return CR_OK;
}
