// cull.cu — batch frustum cull + CLOD survivor prefix, compacted into an
// ordered work list, plus the chunk work records of the point passes.
//
// Restates cullUpdate (Pipelines/Cull/Shaders.metal:19-83) and
// cullFinalizeUpdate (Pipelines/CullFinalize/Shaders.metal:3-14).  The
// reference appends survivors with an atomic counter, so its list order is
// unspecified; here the list is in ascending slot order (deterministic and
// comparable to the CPU oracle):
//   1. cull_classify: one thread per slot; each 256-slot CTA compacts its
//      survivors in order with warp ballots, adds the per-batch values the
//      point passes need (decode steps, screen rectangle), and writes its
//      survivor and chunk counts.
//   2. cull_compact: each CTA sums the counts of the CTAs before it, copies
//      its survivors to that offset and writes one chunk record per
//      `chunkPoints` survivor points; the last CTA publishes the totals (the
//      CUDA counterpart of the indirect argument buffer).
// The one-view cull does both steps in one launch (cull_one_pass: each CTA
// publishes its counts and reads its predecessors'); batched views keep the
// two launches, one grid row per view.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cr_device.cuh"
#include "cr_internal.h"

namespace {

constexpr int kCullThreads = 256;


// Screen rectangle (buffer rows, widened by two pixels, clamped) covering the
// projection of the batch AABB's eight corners; tw = 0 when a corner lies
// behind the camera.  Every point of the box then projects inside the hull
// of the corners; the point passes treat the rectangle as a cache only.
__device__ __forceinline__ void screen_rect(const cr_raster_batch &b, const float *T, int W,
                                            int H, CullRec &r) {
    float xmin = 3.0e38f, xmax = -3.0e38f, ymin = 3.0e38f, ymax = -3.0e38f;
    bool front = true;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const crd::f4 clip = crd::mulp(T, (c & 1) ? b.maxX : b.minX, (c & 2) ? b.maxY : b.minY,
                                       (c & 4) ? b.maxZ : b.minZ);
        if (!(clip.w > 0.000001f) || !isfinite(clip.x) || !isfinite(clip.y)) front = false;
        // Approximate quotients: the rectangle only decides which points
        // take the shared-memory tile (the others take global atomics, with
        // the same result), and its 2-pixel margin covers their error.
        const float fx = (__fdividef(clip.x, clip.w) * 0.5f + 0.5f) * (float)W;
        const float fy = (__fdividef(clip.y, clip.w) * 0.5f + 0.5f) * (float)H;
        xmin = fminf(xmin, fx);
        xmax = fmaxf(xmax, fx);
        ymin = fminf(ymin, fy);
        ymax = fmaxf(ymax, fy);
    }
    r.x0 = r.y0 = r.tw = r.th = 0;
    if (!front || !(xmax - xmin < 1.0e6f) || !(ymax - ymin < 1.0e6f)) return;
    const int x0 = max((int)floorf(xmin) - 2, 0), x1 = min((int)ceilf(xmax) + 2, W - 1);
    const int yl = (int)floorf(ymin) - 2, yh = (int)ceilf(ymax) + 2;
    const int y0 = max(H - 1 - yh, 0), y1 = min(H - 1 - yl, H - 1);
    if (x1 < x0 || y1 < y0) return;
    r.x0 = x0;
    r.y0 = y0;
    r.tw = x1 - x0 + 1;
    r.th = y1 - y0 + 1;
}

// One slot of cullUpdate (Cull/Shaders.metal:28-82).
// files: the cull's file table (a.files, or the one-view launch's inline copy);
// pre: the per-file planes and view * world of the inline files (or null).
__device__ __forceinline__ bool cull_slot(const CullArgs &a, const cr_raster_file *files,
                                          uint32_t gid, CullRec &out,
                                          const crd::FilePre *pre = nullptr) {
    const cr_raster_batch b = a.batches[gid];
    if (b.state == 0) return false;  // residency gate (:33-36)
    // A fileIndex past the file table is rejected here (the reference would
    // read past its buffer); the host also refuses such batches on upload.
    if (b.fileIndex >= a.nfiles) return false;
    const cr_raster_file *file = &files[b.fileIndex];
    if (a.u.enableFrustumCulling != 0) {
        const crd::f3 mn{b.minX, b.minY, b.minZ}, mx{b.maxX, b.maxY, b.maxZ};
        if (pre ? !crd::intersects_frustum_pre(pre[b.fileIndex], mn, mx)
                : !crd::intersects_frustum(file->transformFrustum, mn, mx))
            return false;
    }
    const float px =
        pre ? crd::pixel_size_on_screen_vw(b, pre[b.fileIndex].vw, a.u.proj, a.u.width,
                                           a.u.height)
            : crd::pixel_size_on_screen(b, file->world, a.u.view, a.u.proj, a.u.width,
                                        a.u.height);
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
    out.vb.batchIndex = gid;
    out.vb.level = level;
    out.vb.lodThreshold = thr;
    out.vb.activePoints = active;
    // batchSize (Common.metal:81-83) over the steps of the precision level.
    const float steps = level == 0 ? 1073741824.0f : level == 1 ? 1048576.0f : 1024.0f;
    out.minX = b.minX;
    out.minY = b.minY;
    out.minZ = b.minZ;
    out.qx = fmaxf(b.maxX - b.minX, 0.000001f) / steps;
    out.qy = fmaxf(b.maxY - b.minY, 0.000001f) / steps;
    out.qz = fmaxf(b.maxZ - b.minZ, 0.000001f) / steps;
    out.first = b.firstPoint;
    out.file = b.fileIndex;
    screen_rect(b, file->transform, a.u.width, a.u.height, out);
    return true;
}

__device__ __forceinline__ uint32_t nchunks(uint32_t active, uint32_t c) {
    return (active + c - 1u) / c;
}

__device__ __forceinline__ uint32_t round4(uint32_t n) { return (n + 3u) & ~3u; }

// Fragment span of a survivor: its chunks' point counts, each rounded up to
// a multiple of four, so that every chunk's fragments start 16-byte aligned.
__device__ __forceinline__ uint32_t fragment_span(uint32_t active, uint32_t c) {
    const uint32_t nc = nchunks(active, c);
    return nc == 0u ? 0u : (nc - 1u) * round4(c) + round4(active - (nc - 1u) * c);
}

__device__ __forceinline__ void classify_body(const CullArgs &a) {
    __shared__ uint32_t warp_counts[kCullThreads / 32];
    __shared__ uint32_t warp_chunks[kCullThreads / 32];
    __shared__ uint32_t warp_points[kCullThreads / 32];
    const uint32_t gid = blockIdx.x * kCullThreads + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    CullRec rec;
    bool keep = false;
    if (gid < a.nbatches) keep = cull_slot(a, a.files, gid, rec);
    const uint32_t ballot = __ballot_sync(0xffffffffu, keep);
    const uint32_t ch = __reduce_add_sync(
        0xffffffffu, keep ? nchunks(rec.vb.activePoints, a.chunk_points) : 0u);
    const uint32_t pts = __reduce_add_sync(
        0xffffffffu, keep ? fragment_span(rec.vb.activePoints, a.chunk_points) : 0u);
    if (lane == 0) {
        warp_counts[warp] = __popc(ballot);
        warp_chunks[warp] = ch;
        warp_points[warp] = pts;
    }
    __syncthreads();
    uint32_t before = 0, total = 0, total_chunks = 0, total_points = 0;
#pragma unroll
    for (int w = 0; w < kCullThreads / 32; ++w) {
        if (w < warp) before += warp_counts[w];
        total += warp_counts[w];
        total_chunks += warp_chunks[w];
        total_points += warp_points[w];
    }
    if (keep) {
        const uint32_t pos = before + __popc(ballot & ((1u << lane) - 1u));
        a.tmp[blockIdx.x * kCullThreads + pos] = rec;
    }
    if (threadIdx.x == 0) {
        a.cta_counts[kCullCtaWords * blockIdx.x] = total;
        a.cta_counts[kCullCtaWords * blockIdx.x + 1] = total_chunks;
        a.cta_counts[kCullCtaWords * blockIdx.x + 2] = total_points;
    }
}

// Exclusive block-wide prefix of one value per thread (256 threads).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t c, uint32_t *scan_w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) scan_w[warp] = x;
    __syncthreads();
    uint32_t wbase = 0;
#pragma unroll
    for (int w = 0; w < kCullThreads / 32; ++w)
        if (w < warp) wbase += scan_w[w];
    return wbase + (x - c);
}

__device__ __forceinline__ void compact_body(const CullArgs &a) {
    const CullRec *tmp = a.tmp;
    const uint32_t *cta_counts = a.cta_counts;
    cr_visible_batch *out = a.visible;
    ChunkRec *chunks = a.chunks;
    const uint32_t chunk_points = a.chunk_points;
    uint32_t *counters = a.counters;
    __shared__ uint32_t part_v[kCullThreads / 32], part_c[kCullThreads / 32],
        part_p[kCullThreads / 32];
    __shared__ uint32_t scan_c[kCullThreads / 32], scan_p[kCullThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // Exclusive prefix of the survivor, chunk and point counts of the CTAs before this one.
    uint32_t sv = 0, sc = 0, sp = 0;
    for (uint32_t i = threadIdx.x; i < blockIdx.x; i += kCullThreads) {
        sv += cta_counts[kCullCtaWords * i];
        sc += cta_counts[kCullCtaWords * i + 1];
        sp += cta_counts[kCullCtaWords * i + 2];
    }
    sv = __reduce_add_sync(0xffffffffu, sv);
    sc = __reduce_add_sync(0xffffffffu, sc);
    sp = __reduce_add_sync(0xffffffffu, sp);
    if (lane == 0) {
        part_v[warp] = sv;
        part_c[warp] = sc;
        part_p[warp] = sp;
    }
    __syncthreads();
    uint32_t off_v = 0, off_c = 0, off_p = 0;
#pragma unroll
    for (int w = 0; w < kCullThreads / 32; ++w) {
        off_v += part_v[w];
        off_c += part_c[w];
        off_p += part_p[w];
    }
    const uint32_t mine = cta_counts[kCullCtaWords * blockIdx.x];
    const uint32_t mine_chunks = cta_counts[kCullCtaWords * blockIdx.x + 1];
    const uint32_t mine_points = cta_counts[kCullCtaWords * blockIdx.x + 2];
    // One survivor per thread (a CTA holds at most 256): ordered copy and
    // exclusive scans of the chunk and point counts for the chunk record
    // offsets and the chunks' point offsets.
    CullRec r;
    uint32_t c = 0, n = 0;
    if (threadIdx.x < mine) {
        r = tmp[blockIdx.x * kCullThreads + threadIdx.x];
        out[off_v + threadIdx.x] = r.vb;
        c = nchunks(r.vb.activePoints, chunk_points);
        n = fragment_span(r.vb.activePoints, chunk_points);
    }
    const uint32_t base = off_c + block_exclusive_scan(c, scan_c);
    const uint32_t pbase = off_p + block_exclusive_scan(n, scan_p);
    for (uint32_t j = 0; j < c; ++j) {
        ChunkRec k;
        k.first = r.first + j * chunk_points;
        k.count = min(chunk_points, r.vb.activePoints - j * chunk_points);
        k.level = r.vb.level;
        k.thr = r.vb.lodThreshold;
        k.batchIndex = r.vb.batchIndex;
        k.file = r.file;
        k.minX = r.minX;
        k.minY = r.minY;
        k.minZ = r.minZ;
        k.qx = r.qx;
        k.qy = r.qy;
        k.qz = r.qz;
        k.x0 = r.x0;
        k.y0 = r.y0;
        k.tw = r.tw;
        k.th = r.th;
        chunks[base + j] = k;
        if (a.chunk_poff) a.chunk_poff[base + j] = pbase + j * round4(chunk_points);
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        // cullFinalizeUpdate (CullFinalize/Shaders.metal:3-14): {count, 1, 1}.
        counters[CNT_VISIBLE] = off_v + mine;
        counters[CNT_ARGS_X] = off_v + mine;
        counters[CNT_ARGS_Y] = 1u;
        counters[CNT_ARGS_Z] = 1u;
        counters[CNT_WORK_DEPTH] = 0u;
        counters[CNT_WORK_COLOR] = 0u;
        counters[CNT_DONE] = 0u;
        counters[CNT_CHUNKS] = off_c + mine_chunks;
        counters[CNT_POINTS] = off_p + mine_points;
    }
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The one-view cull in one pass: every CTA classifies its 256 slots,
// publishes its survivor, chunk and point counts (flag = this launch's
// epoch + 1, after a release), sums the counts of the CTAs before it and
// writes its survivors and chunk records at those offsets.
//
// A CTA's slots are chosen by a ticket it claims on arrival (an atomic
// counter that wraps to zero after the launch's last CTA), not by its block
// index: the CTAs a CTA waits for hold smaller tickets, so they have already
// started, and each of them waits only for CTAs that started before it.  The
// waits therefore end whatever order or number of CTAs the GPU runs at once.
// A CTA that has polled a flag a.spin_limit times nevertheless gives up,
// counts that predecessor as empty (its writes stay inside the outputs; the
// frame is wrong) and stores kErrCullWait into the cloud's error counter and
// the context's status word, which the host reports as CR_ERR_TIMEOUT.  The
// last CTA to finish advances the epoch, so the flags never need clearing.
// ifl: the cloud's file table when small (read in place from the
// __grid_constant__ parameter; n = 0: a.files).
__global__ void __launch_bounds__(kCullThreads)
    cull_one_pass(const __grid_constant__ CullArgs a, FrameClear clear,
                  const __grid_constant__ InlineFiles ifl) {
    crd::grid_wait();          // the previous frame's passes have finished with the planes
    crd::launch_dependents();  // the depth pass waits for this grid itself
    __shared__ uint32_t s_ticket;
    // Tickets mostly follow block order: start bringing this block's likely
    // batch records towards L2 while the ticket is claimed.
    {
        const size_t g = (size_t)blockIdx.x * kCullThreads + threadIdx.x;
        if (g < a.nbatches)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(a.batches + g));
    }
    if (threadIdx.x == 0) s_ticket = atomicInc(a.counters + CNT_CULL_TICKET, gridDim.x - 1u);
    __syncthreads();
    const uint32_t ticket = s_ticket;
    // Tickets past the cull's zero the frame (none wait on them, and they
    // wait on nothing), overlapping the cull's latency-bound work.
    const uint32_t cull_ctas = (a.nbatches + kCullThreads - 1) / kCullThreads;
    if (ticket >= cull_ctas) {
        const size_t stride = (size_t)(gridDim.x - cull_ctas) * kCullThreads;
        const size_t t0 = (size_t)(ticket - cull_ctas) * kCullThreads + threadIdx.x;
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
        for (size_t i = t0; i < clear.naccum; i += stride) clear.accum[i] = z;
        for (size_t i = t0; i < clear.ndepth4; i += stride) clear.depth4[i] = z;
        if (t0 < clear.ntail) clear.tail[t0] = 0u;
        return;
    }
    __shared__ uint32_t warp_counts[kCullThreads / 32], warp_chunks[kCullThreads / 32],
        warp_points[kCullThreads / 32];
    __shared__ uint32_t part_v[kCullThreads / 32], part_c[kCullThreads / 32],
        part_p[kCullThreads / 32];
    __shared__ uint32_t scan_c[kCullThreads / 32], scan_p[kCullThreads / 32];
    __shared__ CullRec s_rec[kCullThreads];
    __shared__ uint32_t s_cbase[kCullThreads];
    __shared__ uint4 s_out[kCullThreads / 32][128];  // a warp's 32 chunk records
    __shared__ crd::FilePre s_pre[kInlineFiles];
    const uint32_t epoch = *(volatile const uint32_t *)(a.counters + CNT_CULL_EPOCH) + 1u;
    const uint32_t gid = ticket * kCullThreads + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // The inline files' frustum planes and view * world, once per CTA: a
    // thread per (file, plane) and per (file, view * world).
    if (ifl.n) {
        const uint32_t t = threadIdx.x;
        if (t < 6 * ifl.n) {
            crd::frustum_plane(ifl.f[t / 6].transformFrustum, (int)(t % 6), s_pre[t / 6].plane[t % 6]);
        } else if (t >= 32 && t < 32 + ifl.n) {
            crd::mat4mul(a.u.view, ifl.f[t - 32].world, s_pre[t - 32].vw);
        }
        __syncthreads();
    }
    CullRec rec;
    const bool keep = gid < a.nbatches &&
                      cull_slot(a, ifl.n ? ifl.f : a.files, gid, rec, ifl.n ? s_pre : nullptr);
    const uint32_t c = keep ? nchunks(rec.vb.activePoints, a.chunk_points) : 0u;
    const uint32_t n = keep ? fragment_span(rec.vb.activePoints, a.chunk_points) : 0u;
    const uint32_t ballot = __ballot_sync(0xffffffffu, keep);
    const uint32_t ch = __reduce_add_sync(0xffffffffu, c);
    const uint32_t pts = __reduce_add_sync(0xffffffffu, n);
    if (lane == 0) {
        warp_counts[warp] = __popc(ballot);
        warp_chunks[warp] = ch;
        warp_points[warp] = pts;
    }
    __syncthreads();
    uint32_t before = 0, total = 0, total_chunks = 0, total_points = 0;
#pragma unroll
    for (int w = 0; w < kCullThreads / 32; ++w) {
        if (w < warp) before += warp_counts[w];
        total += warp_counts[w];
        total_chunks += warp_chunks[w];
        total_points += warp_points[w];
    }
    if (threadIdx.x == 0) {
        uint32_t *mine = a.cta_counts + kCullCtaWords * ticket;
        mine[0] = total;
        mine[1] = total_chunks;
        mine[2] = total_points;
        st_release(mine + 3, epoch);
    }
    // Counts of the CTAs before this one, a thread per predecessor.
    uint32_t sv = 0, sc = 0, sp = 0;
    bool gave_up = false;
    for (uint32_t i = threadIdx.x; i < ticket; i += kCullThreads) {
        const uint32_t *w = a.cta_counts + kCullCtaWords * i;
        bool published = false;
        for (uint32_t polls = 0; polls < a.spin_limit; ++polls) {
            if (ld_acquire(w + 3) == epoch) {
                published = true;
                break;
            }
            __nanosleep(20);
        }
        if (!published) {
            gave_up = true;
            continue;
        }
        sv += __ldcg(w);
        sc += __ldcg(w + 1);
        sp += __ldcg(w + 2);
    }
    if (gave_up) {
        atomicCAS(a.counters + CNT_ERROR, 0u, kErrCullWait);
        if (a.status) *(volatile uint32_t *)a.status = kErrCullWait;
    }
    sv = __reduce_add_sync(0xffffffffu, sv);
    sc = __reduce_add_sync(0xffffffffu, sc);
    sp = __reduce_add_sync(0xffffffffu, sp);
    if (lane == 0) {
        part_v[warp] = sv;
        part_c[warp] = sc;
        part_p[warp] = sp;
    }
    __syncthreads();
    uint32_t off_v = 0, off_c = 0, off_p = 0;
#pragma unroll
    for (int w = 0; w < kCullThreads / 32; ++w) {
        off_v += part_v[w];
        off_c += part_c[w];
        off_p += part_p[w];
    }
    // Survivors in slot order, then their chunk records (exclusive scans of
    // the chunk and point counts in slot order, which is survivor order).
    const uint32_t lpos = before + __popc(ballot & ((1u << lane) - 1u));  // survivor in the CTA
    if (keep) a.visible[off_v + lpos] = rec.vb;
    // The CTA's chunk records, one record per thread in record order (the
    // records of a survivor are consecutive): each survivor's values and the
    // first of its records go to shared memory, and every thread finds the
    // survivor of its record by binary search.
    const uint32_t lbase = block_exclusive_scan(c, scan_c);
    const uint32_t pbase = off_p + block_exclusive_scan(n, scan_p);
    if (keep) {
        s_rec[lpos] = rec;
        s_cbase[lpos] = lbase;
        if (a.chunk_poff)
            for (uint32_t j = 0; j < c; ++j)
                a.chunk_poff[off_c + lbase + j] = pbase + j * round4(a.chunk_points);
    }
    __syncthreads();
    // A warp's 32 records go through shared memory so that they leave as
    // contiguous 16-byte words (one record per lane would store 64-byte
    // strided words).
    uint4 *stage = s_out[warp];
    uint4 *dst4 = reinterpret_cast<uint4 *>(a.chunks + off_c);
    for (uint32_t r0 = 0; r0 < total_chunks; r0 += kCullThreads) {
        const uint32_t r = r0 + threadIdx.x;
        if (r < total_chunks) {
            // The survivors' first records ascend (each has one at least).
            uint32_t lo = 0, hi = total;
            while (hi - lo > 1u) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s_cbase[mid] <= r)
                    lo = mid;
                else
                    hi = mid;
            }
            const CullRec &sr = s_rec[lo];
            const uint32_t j = r - s_cbase[lo];
            ChunkRec k;
            k.first = sr.first + j * a.chunk_points;
            k.count = min(a.chunk_points, sr.vb.activePoints - j * a.chunk_points);
            k.level = sr.vb.level;
            k.thr = sr.vb.lodThreshold;
            k.batchIndex = sr.vb.batchIndex;
            k.file = sr.file;
            k.minX = sr.minX;
            k.minY = sr.minY;
            k.minZ = sr.minZ;
            k.qx = sr.qx;
            k.qy = sr.qy;
            k.qz = sr.qz;
            k.x0 = sr.x0;
            k.y0 = sr.y0;
            k.tw = sr.tw;
            k.th = sr.th;
            const uint4 *kv = reinterpret_cast<const uint4 *>(&k);
#pragma unroll
            for (int q = 0; q < 4; ++q) stage[4 * lane + q] = kv[q];
        }
        __syncwarp();
        const uint32_t wrec = r0 + 32u * warp;  // the warp's first record
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const uint32_t w = 32u * m + lane;  // 16-byte word of the warp's records
            if (wrec + w / 4u < total_chunks) dst4[4u * wrec + w] = stage[w];
        }
        __syncwarp();
    }
    if (ticket == cull_ctas - 1 && threadIdx.x == 0) {
        // cullFinalizeUpdate (CullFinalize/Shaders.metal:3-14): {count, 1, 1}.
        uint32_t *counters = a.counters;
        counters[CNT_VISIBLE] = off_v + total;
        counters[CNT_ARGS_X] = off_v + total;
        counters[CNT_ARGS_Y] = 1u;
        counters[CNT_ARGS_Z] = 1u;
        counters[CNT_WORK_DEPTH] = 0u;
        counters[CNT_WORK_COLOR] = 0u;
        counters[CNT_DONE] = 0u;
        counters[CNT_CHUNKS] = off_c + total_chunks;
        counters[CNT_POINTS] = off_p + total_points;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(a.counters + CNT_CULL_DONE, 1u) == cull_ctas - 1u) {
            a.counters[CNT_CULL_DONE] = 0u;
            a.counters[CNT_CULL_EPOCH] = epoch;
        }
    }
}

__global__ void __launch_bounds__(kCullThreads) cull_classify(CullArgs a) { classify_body(a); }
__global__ void __launch_bounds__(kCullThreads) cull_compact(CullArgs a) { compact_body(a); }

// Batched views: blockIdx.y selects the view's arguments (its uniforms, file
// table and output ranges); the slots and the point pool are shared.
__global__ void __launch_bounds__(kCullThreads) cull_classify_views(const CullArgs *av) {
    classify_body(av[blockIdx.y]);
}
__global__ void __launch_bounds__(kCullThreads) cull_compact_views(const CullArgs *av) {
    compact_body(av[blockIdx.y]);
}

__global__ void cull_empty(uint32_t *counters) {
    counters[CNT_VISIBLE] = 0u;
    counters[CNT_ARGS_X] = 0u;
    counters[CNT_ARGS_Y] = 1u;
    counters[CNT_ARGS_Z] = 1u;
    counters[CNT_WORK_DEPTH] = 0u;
    counters[CNT_WORK_COLOR] = 0u;
    counters[CNT_DONE] = 0u;
    counters[CNT_CHUNKS] = 0u;
    counters[CNT_POINTS] = 0u;
}

}  // namespace

uint64_t chunk_capacity(const cr_capacity &cap, int chunk_points) {
    const uint64_t per = ((uint64_t)cap.pointsPerBatch + chunk_points - 1) / chunk_points;
    return std::max<uint64_t>(1, (uint64_t)cap.maxResidentBatches * per);
}

cr_status launch_cull(cr_cloud *cloud, const CullUniforms &u, cudaStream_t s,
                      const FrameClear *clear) {
    const uint32_t n = cloud->cap.maxResidentBatches;
    if (n == 0) {
        cull_empty<<<1, 1, 0, s>>>(cloud->d_counters);
        CR_CUDA(cudaGetLastError());
        if (clear) return cri::fail(CR_ERR_INTERNAL, "launch_cull: clear with an empty pool");
        return CR_OK;
    }
    const uint32_t cp = (uint32_t)std::max(cloud->ctx->chunk_points, kMinChunkPoints);
    const uint32_t ctas = (n + kCullThreads - 1) / kCullThreads;
    CullArgs a{cloud->d_batches,  n,
               cloud->d_files,    (uint32_t)cloud->files.size(),
               cloud->d_cull_tmp, cloud->d_cull_cta,
               cp,                u,
               cloud->d_visible,  cloud->d_chunks,
               cloud->d_counters, nullptr,
               (uint32_t)std::max(cloud->ctx->cull_spin_limit, 0), cloud->ctx->d_status};
    // Half as many clear CTAs as SMs: the cull's few latency-bound CTAs then
    // keep SMs of their own (with twice the SM count the cull took 33 µs
    // instead of 26.5 µs on the 100M-point 1080p frames; a quarter is as
    // fast, an eighth leaves the clear the longer part).
    const uint32_t clear_ctas = clear ? std::max(1u, (uint32_t)cloud->ctx->sm_count / 2u) : 0u;
    const InlineFiles ifl = inline_files(cloud);
    if (!ifl.n) {
        const cr_status st = ensure_device_files(cloud);
        if (st) return st;
    }
    CR_CUDA(launch_programmatic(cull_one_pass, dim3(ctas + clear_ctas), dim3(kCullThreads), 0, s, a,
                                clear ? *clear : FrameClear{}, ifl));
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

cr_status launch_cull_views(const CullArgs *d_args, uint32_t nslots, uint32_t nviews,
                            cudaStream_t s) {
    if (nslots == 0 || nviews == 0) return CR_OK;
    const dim3 grid((nslots + kCullThreads - 1) / kCullThreads, nviews);
    cull_classify_views<<<grid, kCullThreads, 0, s>>>(d_args);
    CR_CUDA(cudaGetLastError());
    cull_compact_views<<<grid, kCullThreads, 0, s>>>(d_args);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free cull (cr_cull_noalloc)
// ---------------------------------------------------------------------------
// Some callers cannot allocate device memory: plug-ins whose host application
// owns every device allocation (a fixed budget or its own allocator), and
// real-time loops that cannot afford cudaMalloc's implicit device-wide
// synchronisation in the middle of a frame.  For them this variant of the
// cull takes device inputs and outputs from the caller and keeps its only
// scratch — one survivor count per 256-slot CTA — in the file-scope array
// below, which every GPU that loads the library holds until the process
// exits.  Every slot of the scratch a call reads is written by the same call
// first, so nothing has to start at zero.  All calls share the one array:
// two calls that overlap on the GPU race on it.

namespace {

constexpr uint32_t kNoAllocMaxSlots = 1u << 20;  // 1,048,576 batch slots
constexpr uint32_t kNoAllocMaxCtas = kNoAllocMaxSlots / kCullThreads;

static __device__ __align__(256) uint32_t g_noalloc_cta_counts[kNoAllocMaxCtas];

__global__ void __launch_bounds__(kCullThreads)
    cull_noalloc_count(CullArgs a, uint32_t *cta_counts) {
    __shared__ uint32_t warp_counts[kCullThreads / 32];
    const uint32_t gid = blockIdx.x * kCullThreads + threadIdx.x;
    CullRec rec;
    const bool keep = gid < a.nbatches && cull_slot(a, a.files, gid, rec);
    const uint32_t ballot = __ballot_sync(0xffffffffu, keep);
    if ((threadIdx.x & 31) == 0) warp_counts[threadIdx.x >> 5] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t total = 0;
        for (int w = 0; w < kCullThreads / 32; ++w) total += warp_counts[w];
        cta_counts[blockIdx.x] = total;
    }
}

// The write kernel evaluates cull_slot again for its 256 slots instead of
// reading survivors that the count kernel kept (which would need scratch per
// slot); cull_slot is a pure function of the inputs, so both kernels agree.
// Each CTA sums the counts of all CTAs before it: at most kNoAllocMaxCtas
// (4,096) words, 16 loads per thread, which the slot limit keeps cheap.
__global__ void __launch_bounds__(kCullThreads)
    cull_noalloc_write(CullArgs a, const uint32_t *cta_counts, cr_visible_batch *out,
                       uint32_t *count_out) {
    __shared__ uint32_t part[kCullThreads / 32], warp_counts[kCullThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t s = 0;
    for (uint32_t i = threadIdx.x; i < blockIdx.x; i += kCullThreads) s += cta_counts[i];
    s = __reduce_add_sync(0xffffffffu, s);
    if (lane == 0) part[warp] = s;
    const uint32_t gid = blockIdx.x * kCullThreads + threadIdx.x;
    CullRec rec;
    const bool keep = gid < a.nbatches && cull_slot(a, a.files, gid, rec);
    const uint32_t ballot = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_counts[warp] = __popc(ballot);
    __syncthreads();
    uint32_t offset = 0, before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kCullThreads / 32; ++w) {
        offset += part[w];
        if (w < warp) before += warp_counts[w];
        total += warp_counts[w];
    }
    if (keep) out[offset + before + __popc(ballot & ((1u << lane) - 1u))] = rec.vb;
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *count_out = offset + total;
}

std::mutex g_noalloc_mutex;
std::vector<uint32_t *> g_noalloc_scratch;  // device address of the array, per device

// The array's device address on the current device; the first call on a
// device looks it up (cudaGetSymbolAddress), later calls reuse it.
cr_status noalloc_scratch(uint32_t **out) {
    int dev = 0;
    CR_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if ((size_t)dev >= g_noalloc_scratch.size()) g_noalloc_scratch.resize(dev + 1, nullptr);
    if (!g_noalloc_scratch[dev]) {
        void *p = nullptr;
        CR_CUDA(cudaGetSymbolAddress(&p, g_noalloc_cta_counts));
        g_noalloc_scratch[dev] = static_cast<uint32_t *>(p);
    }
    *out = g_noalloc_scratch[dev];
    return CR_OK;
}

}  // namespace

extern "C" CR_API cr_status cr_cull_noalloc(const cr_raster_batch *batches, uint32_t nbatches,
                                            const cr_raster_file *files, uint32_t nfiles,
                                            const cr_config *config, const cr_camera *camera,
                                            int width, int height, cr_visible_batch *visible,
                                            uint32_t *count, void *stream) {
    if (!config || !camera || !count || (nbatches && (!batches || !visible)) || !files ||
        nfiles == 0)
        return cri::fail(CR_ERR_INVALID_ARGUMENT, "null argument or empty file table");
    if (width <= 0 || height <= 0)
        return cri::fail(CR_ERR_INVALID_ARGUMENT, "width and height must be positive");
    if (nbatches > kNoAllocMaxSlots)
        return cri::fail(CR_ERR_CAPACITY,
                         "cr_cull_noalloc handles at most 1048576 batch slots (got " +
                             std::to_string(nbatches) + ")");
    uint32_t *scratch = nullptr;
    cr_status st = noalloc_scratch(&scratch);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (nbatches == 0) {
        CR_CUDA(cudaMemsetAsync(count, 0, sizeof(uint32_t), s));
        return CR_OK;
    }
    CullUniforms u;
    std::memcpy(u.view, camera->view, sizeof(u.view));
    std::memcpy(u.proj, camera->projection, sizeof(u.proj));
    u.width = width;
    u.height = height;
    u.enableFrustumCulling = config->enableFrustumCulling != 0;
    u.lodBias = config->lodBias;
    u.enableCLOD = config->enableCLOD != 0;
    CullArgs a{batches, nbatches, files, nfiles, nullptr, nullptr, (uint32_t)kMinChunkPoints, u};
    const uint32_t ctas = (nbatches + kCullThreads - 1) / kCullThreads;
    cull_noalloc_count<<<ctas, kCullThreads, 0, s>>>(a, scratch);
    CR_CUDA(cudaGetLastError());
    cull_noalloc_write<<<ctas, kCullThreads, 0, s>>>(a, scratch, visible, count);
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}
