// cull.cu — batch frustum cull + CLOD survivor prefix, compacted into an
// ordered work list.
//
// Restates cullUpdate (Pipelines/Cull/Shaders.metal:19-83) and
// cullFinalizeUpdate (Pipelines/CullFinalize/Shaders.metal:3-14).  The
// reference appends survivors with an atomic counter, so its list order is
// unspecified; here the list is in ascending slot order (deterministic and
// comparable to the CPU oracle):
//   1. cull_classify: one thread per slot; each 256-slot CTA compacts its
//      survivors in order with warp ballots and writes its count.
//   2. cull_compact: each CTA sums the counts of the CTAs before it, copies
//      its survivors to that offset; the last CTA publishes the total as the
//      "indirect argument" the persistent point passes read, and resets
//      their work cursors.
#include "cr_device.cuh"
#include "cr_internal.h"

namespace {

constexpr int kCullThreads = 256;

struct CullArgs {
    const cr_raster_batch *batches;
    uint32_t nbatches;
    const cr_raster_file *files;
    uint32_t nfiles;
    cr_visible_batch *tmp;
    uint32_t *cta_counts;
    CullUniforms u;
};

// One slot of cullUpdate (Cull/Shaders.metal:28-82).
__device__ __forceinline__ bool cull_slot(const CullArgs &a, uint32_t gid, cr_visible_batch &out) {
    const cr_raster_batch b = a.batches[gid];
    if (b.state == 0) return false;  // residency gate (:33-36)
    // A fileIndex past the file table is rejected here (the reference would
    // read past its buffer); the host also refuses such batches on upload.
    if (b.fileIndex >= a.nfiles) return false;
    const cr_raster_file *file = &a.files[b.fileIndex];
    if (a.u.enableFrustumCulling != 0) {
        if (!crd::intersects_frustum(file->transformFrustum, crd::f3{b.minX, b.minY, b.minZ},
                                     crd::f3{b.maxX, b.maxY, b.maxZ}))
            return false;
    }
    const float px =
        crd::pixel_size_on_screen(b, file->world, a.u.view, a.u.proj, a.u.width, a.u.height);
    const int level = crd::precision_level(px);
    // lodThresholdFromPixelSize (Common.metal:185-187); CLOD off -> 99 (:58-60).
    const float thr =
        (a.u.enableCLOD != 0)
            ? fmaxf(0.0f, (crd::log2_contract(fmaxf(px, 1.0f) / 25.0f) + 3.0f) + (float)a.u.lodBias)
            : 99.0f;
    uint32_t active = b.numPoints;
    if (b.lodCum67 != 0u) {  // survivor prefix (:62-74)
        const int lmax = min(max((int)floorf(thr + 0.5f), 0), 7);
        const uint32_t w = (lmax >> 1) == 0 ? b.lodCum01
                         : (lmax >> 1) == 1 ? b.lodCum23
                         : (lmax >> 1) == 2 ? b.lodCum45
                                            : b.lodCum67;
        active = (lmax & 1) ? (w >> 16) : (w & 0xffffu);
        // Malformed counts past numPoints would walk off the slot; well-formed
        // batches always satisfy cum[L] <= numPoints.
        active = min(active, b.numPoints);
    }
    if (active == 0u) return false;
    out.batchIndex = gid;
    out.level = level;
    out.lodThreshold = thr;
    out.activePoints = active;
    return true;
}

__global__ void __launch_bounds__(kCullThreads) cull_classify(CullArgs a) {
    __shared__ uint32_t warp_counts[kCullThreads / 32];
    const uint32_t gid = blockIdx.x * kCullThreads + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    cr_visible_batch rec;
    bool keep = false;
    if (gid < a.nbatches) keep = cull_slot(a, gid, rec);
    const uint32_t ballot = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_counts[warp] = __popc(ballot);
    __syncthreads();
    uint32_t before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kCullThreads / 32; ++w) {
        if (w < warp) before += warp_counts[w];
        total += warp_counts[w];
    }
    if (keep) {
        const uint32_t pos = before + __popc(ballot & ((1u << lane) - 1u));
        a.tmp[blockIdx.x * kCullThreads + pos] = rec;
    }
    if (threadIdx.x == 0) a.cta_counts[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kCullThreads)
    cull_compact(const cr_visible_batch *tmp, const uint32_t *cta_counts, cr_visible_batch *out,
                 uint32_t *counters) {
    __shared__ uint32_t partial[kCullThreads / 32];
    // Exclusive prefix of the CTA counts before this CTA.
    uint32_t s = 0;
    for (uint32_t i = threadIdx.x; i < blockIdx.x; i += kCullThreads) s += cta_counts[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = s;
    __syncthreads();
    uint32_t offset = 0;
#pragma unroll
    for (int w = 0; w < kCullThreads / 32; ++w) offset += partial[w];
    const uint32_t mine = cta_counts[blockIdx.x];
    for (uint32_t i = threadIdx.x; i < mine; i += kCullThreads)
        out[offset + i] = tmp[blockIdx.x * kCullThreads + i];
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        // cullFinalizeUpdate (CullFinalize/Shaders.metal:3-14): {count, 1, 1}.
        counters[CNT_VISIBLE] = offset + mine;
        counters[CNT_ARGS_X] = offset + mine;
        counters[CNT_ARGS_Y] = 1u;
        counters[CNT_ARGS_Z] = 1u;
        counters[CNT_WORK_DEPTH] = 0u;
        counters[CNT_WORK_COLOR] = 0u;
        counters[CNT_WORK_AUX] = 0u;
    }
}

__global__ void cull_empty(uint32_t *counters) {
    counters[CNT_VISIBLE] = 0u;
    counters[CNT_ARGS_X] = 0u;
    counters[CNT_ARGS_Y] = 1u;
    counters[CNT_ARGS_Z] = 1u;
    counters[CNT_WORK_DEPTH] = 0u;
    counters[CNT_WORK_COLOR] = 0u;
    counters[CNT_WORK_AUX] = 0u;
}

}  // namespace

cr_status launch_cull(cr_cloud *cloud, const CullUniforms &u, cudaStream_t s) {
    const uint32_t n = cloud->cap.maxResidentBatches;
    if (n == 0) {
        cull_empty<<<1, 1, 0, s>>>(cloud->d_counters);
        CR_CUDA(cudaGetLastError());
        return CR_OK;
    }
    const uint32_t ctas = (n + kCullThreads - 1) / kCullThreads;
    CullArgs a{cloud->d_batches, n, cloud->d_files, (uint32_t)cloud->files.size(), cloud->d_cull_tmp,
               cloud->d_cull_cta, u};
    cull_classify<<<ctas, kCullThreads, 0, s>>>(a);
    CR_CUDA(cudaGetLastError());
    cull_compact<<<ctas, kCullThreads, 0, s>>>(cloud->d_cull_tmp, cloud->d_cull_cta,
                                               cloud->d_visible, cloud->d_counters);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}
