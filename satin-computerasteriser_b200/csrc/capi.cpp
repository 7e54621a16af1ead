// capi.cpp — the C ABI (include/cr/cr.h): context, slot pool, frames, and
// the pass sequencing of ComputeRasteriser.encode.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cr_internal.h"
#include "cr_pack.h"

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
namespace cri {
static thread_local std::string g_detail;

void set_error(const std::string &detail) { g_detail = detail; }

cr_status fail(cr_status st, const std::string &detail) {
    g_detail = detail;
    return st;
}

cr_status cuda_fail(cudaError_t e, const char *what) {
    g_detail = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation) return CR_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ||
        e == cudaErrorInvalidDevice)
        return CR_ERR_NO_DEVICE;
    return CR_ERR_CUDA;
}
}  // namespace cri

using cri::fail;

namespace {

constexpr size_t kPointPad = 64;  // slack past the last slot for 16-byte vector loads

// Host 4x4 product with the library's operation order (no contraction:
// this file is compiled with -ffp-contract=off).
void mat4mul(const float *a, const float *b, float *out) {
    float r[16];
    for (int c = 0; c < 4; ++c)
        for (int row = 0; row < 4; ++row)
            r[c * 4 + row] = ((a[0 * 4 + row] * b[c * 4 + 0] + a[1 * 4 + row] * b[c * 4 + 1]) +
                              a[2 * 4 + row] * b[c * 4 + 2]) +
                             a[3 * 4 + row] * b[c * 4 + 3];
    std::memcpy(out, r, sizeof(r));
}

cr_raster_file identity_file() {
    cr_raster_file f;
    std::memset(&f, 0, sizeof(f));
    for (int i = 0; i < 4; ++i) {
        f.transform[i * 5] = 1.0f;
        f.transformFrustum[i * 5] = 1.0f;
        f.world[i * 5] = 1.0f;
        f.prevTransform[i * 5] = 1.0f;
    }
    return f;
}

template <typename T>
cr_status dalloc(T **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return cri::cuda_fail(e, "cudaMalloc");
    }
    return CR_OK;
}

template <typename T>
void dfree(T *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}


void free_cloud_buffers(cr_cloud *c) {
    dfree(c->d_low);
    dfree(c->d_med);
    dfree(c->d_high);
    dfree(c->d_colors);
    dfree(c->d_levels);
    dfree(c->d_batches);
    dfree(c->d_files);
    dfree(c->d_visible);
    dfree(c->d_cull_tmp);
    dfree(c->d_cull_cta);
    dfree(c->d_chunks);
    c->chunk_cap = 0;
    dfree(c->d_frag_xy);
    dfree(c->d_frag_zc);
    dfree(c->d_frag_count);
    dfree(c->d_counters);
    dfree(c->d_disp);
    dfree(c->d_prev_disp);
    dfree(c->d_tint);
}

}  // namespace

void mark_dirty(cr_cloud *c, int64_t lo, int64_t hi) {
    if (lo < c->dirty_lo) c->dirty_lo = lo;
    if (hi > c->dirty_hi) c->dirty_hi = hi;
}

// flushBatchMirror (ComputeRasteriserPointCloud.swift:629-644).
cr_status flush_mirror(cr_cloud *c) {
    if (c->dirty_lo > c->dirty_hi) return CR_OK;
    const int64_t lo = std::max<int64_t>(0, c->dirty_lo);
    const int64_t hi = std::min<int64_t>(c->dirty_hi, (int64_t)c->mirror.size() - 1);
    c->dirty_lo = INT64_MAX;
    c->dirty_hi = -1;
    if (lo > hi) return CR_OK;
    CR_CUDA(cudaMemcpyAsync(c->d_batches + lo, c->mirror.data() + lo,
                            (size_t)(hi - lo + 1) * sizeof(cr_raster_batch),
                            cudaMemcpyHostToDevice, c->ctx->stream));
    return CR_OK;
}

namespace {

static cr_status upload_files_now(cr_cloud *c, const std::vector<cr_raster_file> &files);

// A table the one-view kernels can carry inline is copied to the device only
// when a consumer of the device copy asks (ensure_device_files).
cr_status upload_files(cr_cloud *c, const std::vector<cr_raster_file> &files) {
    if (!files.empty() && files.size() <= kInlineFiles && c->h_files_ring) {
        c->files_dirty = true;
        return CR_OK;
    }
    c->files_dirty = false;
    return upload_files_now(c, files);
}

static cr_status upload_files_now(cr_cloud *c, const std::vector<cr_raster_file> &files) {
    if (files.empty()) return CR_OK;
    if (files.size() > c->d_files_cap) {
        dfree(c->d_files);
        cr_status st = dalloc(&c->d_files, files.size() * sizeof(cr_raster_file));
        if (st != CR_OK) return st;
        c->d_files_cap = (uint32_t)files.size();
    }
    // Stage through the pinned ring so the copy stays asynchronous and the
    // host may overwrite the next slot while earlier copies are in flight.
    const size_t nbytes = files.size() * sizeof(cr_raster_file);
    if (!c->h_files_ring || nbytes > sizeof(cr_raster_file) * c->d_files_cap) {
        CR_CUDA(cudaMemcpy(c->d_files, files.data(), nbytes, cudaMemcpyHostToDevice));
        return CR_OK;
    }
    c->ring_slot = (c->ring_slot + 1) % cr_cloud::kFileRing;
    const int s = c->ring_slot;
    if (c->ring_used[s]) CR_CUDA(cudaEventSynchronize(c->ring_events[s]));
    cr_raster_file *dst = c->h_files_ring + (size_t)s * c->d_files_cap;
    std::memcpy(dst, files.data(), nbytes);
    CR_CUDA(cudaMemcpyAsync(c->d_files, dst, nbytes, cudaMemcpyHostToDevice, c->ctx->stream));
    CR_CUDA(cudaEventRecord(c->ring_events[s], c->ctx->stream));
    c->ring_used[s] = true;
    return CR_OK;
}

cr_status alloc_ring(cr_cloud *c) {
    if (c->h_files_ring) {
        for (int i = 0; i < cr_cloud::kFileRing; ++i)
            if (c->ring_used[i]) cudaEventSynchronize(c->ring_events[i]);
        cudaFreeHost(c->h_files_ring);
        c->h_files_ring = nullptr;
    }
    CR_CUDA(cudaMallocHost((void **)&c->h_files_ring,
                           sizeof(cr_raster_file) * c->d_files_cap * cr_cloud::kFileRing));
    for (int i = 0; i < cr_cloud::kFileRing; ++i) {
        if (!c->ring_events[i])
            CR_CUDA(cudaEventCreateWithFlags(&c->ring_events[i], cudaEventDisableTiming));
        c->ring_used[i] = false;
    }
    c->ring_slot = -1;
    return CR_OK;
}

// Points of a cloud's per-point attribute buffers: one per pool point.
size_t attribute_points(const cr_cloud *c) {
    return (size_t)c->cap.maxResidentBatches * c->cap.pointsPerBatch;
}

// allocateBuffers + rebuildFilesBuffer + rebuildCullBuffers
// (ComputeRasteriserPointCloud.swift:532-589).
cr_status allocate_cloud(cr_cloud *c, cr_capacity cap, const cr_raster_file *files, uint32_t nf) {
    uploads_free(c);  // waits for copies in flight; the slot table is rebuilt
    free_cloud_buffers(c);
    c->cap = cap;
    c->files.clear();
    if (files && nf > 0)
        c->files.assign(files, files + nf);
    else
        c->files.push_back(identity_file());
    c->frame_files = c->files;
    c->mirror.assign(cap.maxResidentBatches, cr_raster_batch{});
    c->free_slots.clear();
    for (int64_t s = (int64_t)cap.maxResidentBatches - 1; s >= 0; --s)
        c->free_slots.push_back((int32_t)s);
    c->resident = 0;
    c->points = 0;
    c->dirty_lo = INT64_MAX;
    c->dirty_hi = -1;

    const size_t pts = (size_t)cap.maxResidentBatches * cap.pointsPerBatch + kPointPad;
    cr_status st;
    if ((st = dalloc(&c->d_low, pts * 4)) || (st = dalloc(&c->d_med, pts * 4)) ||
        (st = dalloc(&c->d_high, pts * 4)) || (st = dalloc(&c->d_colors, pts * 4)) ||
        (st = dalloc(&c->d_levels, (pts + 15) & ~size_t(15))))
        return st;
    const size_t nb = std::max<size_t>(cap.maxResidentBatches, 1);
    const size_t ctas = (nb + 255) / 256;
    if ((st = dalloc(&c->d_batches, nb * sizeof(cr_raster_batch))) ||
        (st = dalloc(&c->d_visible, nb * sizeof(cr_visible_batch))) ||
        (st = dalloc(&c->d_cull_tmp, ctas * 256 * sizeof(CullRec))) ||
        (st = dalloc(&c->d_cull_cta, ctas * kCullCtaWords * sizeof(uint32_t))) ||
        (st = dalloc(&c->d_counters, CNT_COUNT * sizeof(uint32_t))))
        return st;
    c->chunk_cap = chunk_capacity(cap, kMinChunkPoints);
    if ((st = dalloc(&c->d_chunks, c->chunk_cap * sizeof(ChunkRec))) ||
        (st = dalloc(&c->d_frag_count, c->chunk_cap * sizeof(uint32_t))) ||
        (st = dalloc(&c->d_frag_xy, pts * 4)) || (st = dalloc(&c->d_frag_zc, pts * 8)))
        return st;
    c->d_files_cap = (uint32_t)c->files.size();
    if ((st = dalloc(&c->d_files, c->d_files_cap * sizeof(cr_raster_file)))) return st;
    cudaStream_t s = c->ctx->stream;
    CR_CUDA(cudaMemsetAsync(c->d_low, 0, pts * 4, s));
    CR_CUDA(cudaMemsetAsync(c->d_med, 0, pts * 4, s));
    CR_CUDA(cudaMemsetAsync(c->d_high, 0, pts * 4, s));
    CR_CUDA(cudaMemsetAsync(c->d_colors, 0, pts * 4, s));
    CR_CUDA(cudaMemsetAsync(c->d_levels, 0, (pts + 15) & ~size_t(15), s));
    CR_CUDA(cudaMemsetAsync(c->d_batches, 0, nb * sizeof(cr_raster_batch), s));
    CR_CUDA(cudaMemsetAsync(c->d_visible, 0, nb * sizeof(cr_visible_batch), s));
    CR_CUDA(cudaMemsetAsync(c->d_counters, 0, CNT_COUNT * sizeof(uint32_t), s));
    CR_CUDA(cudaMemsetAsync(c->d_cull_cta, 0, ctas * kCullCtaWords * sizeof(uint32_t), s));
    if ((st = alloc_ring(c))) return st;
    if ((st = upload_files(c, c->files))) return st;
    CR_CUDA(cudaStreamSynchronize(s));
    return CR_OK;
}


CullUniforms make_cull_uniforms(const cr_config *cfg, const cr_camera *cam, int w, int h) {
    CullUniforms u;
    std::memcpy(u.view, cam->view, sizeof(u.view));
    std::memcpy(u.proj, cam->projection, sizeof(u.proj));
    u.width = w;
    u.height = h;
    u.enableFrustumCulling = cfg->enableFrustumCulling != 0;
    u.lodBias = cfg->lodBias;
    u.enableCLOD = cfg->enableCLOD != 0;
    return u;
}

RasterUniforms make_raster_uniforms(const cr_config *cfg, const cr_camera *cam, int w, int h) {
    RasterUniforms u;
    std::memcpy(u.view, cam->view, sizeof(u.view));
    std::memcpy(u.proj, cam->projection, sizeof(u.proj));
    u.width = w;
    u.height = h;
    u.lodDither = cfg->enableLODDither != 0;
    u.pointSizeMode = cfg->pointSizeMode;
    u.minimumPointSize = cfg->minimumPointSize;
    u.maximumPointSize = cfg->maximumPointSize;
    u.pointSizeScale = cfg->pointSizeScale;
    u.depthTolerance = cfg->depthTolerance;
    u.colorizeChunks = cfg->colorizeChunks != 0;
    u.colorizeOverdraw = cfg->colorizeOverdraw != 0;
    return u;
}

cr_status validate_render(cr_context *ctx, cr_frame *frame, const cr_config *cfg,
                          const cr_camera *cam) {
    if (!ctx || !frame || !cfg || !cam) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if (frame->ctx != ctx) return fail(CR_ERR_INVALID_ARGUMENT, "frame belongs to another context");
    return validate_config(cfg);
}

// encodeNearestIndexPass (ComputeRasteriser.swift:505-522) into the frame's key plane.
cr_status nearest_index_pass(cr_context *ctx, cr_frame *f, cr_cloud *cloud, const cr_config *cfg,
                             const cr_camera *cam) {
    cudaStream_t s = ctx->stream;
    const size_t npix = (size_t)f->width * f->height;
    CR_CUDA(cudaMemsetAsync(f->d_nearest, 0, npix * sizeof(unsigned long long), s));
    cr_status st = launch_cull(cloud, make_cull_uniforms(cfg, cam, f->width, f->height), s);
    if (st) return st;
    RasterTargets t{f->d_depth, f->d_accum, f->d_nearest};
    return launch_raster(cloud, PASS_NEAREST, make_raster_uniforms(cfg, cam, f->width, f->height),
                         t, s);
}

int trunc_i(float x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int)x;
}

}  // namespace

cr_status ensure_device_files(cr_cloud *c) {
    if (!c->files_dirty) return CR_OK;
    c->files_dirty = false;
    return upload_files_now(c, c->frame_files);
}

InlineFiles inline_files(const cr_cloud *c) {
    InlineFiles out;
    out.n = 0;
    if (!c->frame_files.empty() && c->frame_files.size() <= kInlineFiles) {
        out.n = (uint32_t)c->frame_files.size();
        std::memcpy(out.f, c->frame_files.data(), out.n * sizeof(cr_raster_file));
    }
    return out;
}


cr_status validate_config(const cr_config *cfg) {
    if (cfg->mode != CR_MODE_HIGH_QUALITY_AVERAGE && cfg->mode != CR_MODE_NEAREST_POINT)
        return fail(CR_ERR_INVALID_ARGUMENT, "config.mode must be 0 (HQS) or 1 (nearest)");
    if (cfg->pointSizeMode != 0 && cfg->pointSizeMode != 1)
        return fail(CR_ERR_INVALID_ARGUMENT, "config.pointSizeMode must be 0 or 1");
    if (cfg->motionBlur > 0.0f && cfg->motionBlurSamples < 1)
        return fail(CR_ERR_INVALID_ARGUMENT, "config.motionBlurSamples must be at least 1");
    return CR_OK;
}

bool variants_on(const cr_config *cfg) {
    return cfg->mode == CR_MODE_HIGH_QUALITY_AVERAGE &&
           (cfg->applyDisplacement || cfg->applyTint || cfg->motionBlur > 0.0f);
}

cr_status reject_variants(const cr_config *cfg, const char *where) {
    if (variants_on(cfg))
        return fail(CR_ERR_UNSUPPORTED, std::string(where) +
                                            ": the colour variants (displacement, tint, "
                                            "coverage, motion blur) need cr_render");
    return CR_OK;
}

// ===========================================================================
// Exported API
// ===========================================================================
cr_status device_status(cr_context *ctx) {
    volatile uint32_t *w = ctx->h_status;
    const uint32_t code = w ? *w : 0u;
    if (code == 0u) return CR_OK;
    *w = 0u;
    if (code == kErrCullWait)
        return fail(CR_ERR_TIMEOUT,
                    "a cull CTA gave up waiting for the survivor counts of the CTAs before it "
                    "(cr_tuning.cullSpinLimit = " + std::to_string(ctx->cull_spin_limit) +
                        " polls); the survivor lists and images of the frames enqueued before "
                        "this call may be incomplete");
    if (code == kErrSortWait)
        return fail(CR_ERR_TIMEOUT,
                    "a radix sort tile of the packer gave up waiting for the digit counts of "
                    "the tiles before it; the packed cloud may be wrong");
    if (code == kErrStageWait)
        return fail(CR_ERR_TIMEOUT,
                    "a point pass gave up waiting for a bulk copy into shared memory; the "
                    "frames enqueued before this call may be wrong");
    return fail(CR_ERR_TIMEOUT, "device-side status " + std::to_string(code));
}

cr_status frame_copy_fence(cr_frame *f, cudaStream_t s) {
    if (!f->copy_pending) return CR_OK;
    CR_CUDA(cudaStreamWaitEvent(s, f->ev_copied, 0));
    f->copy_pending = false;  // later work on `s` is ordered after the wait
    return CR_OK;
}

extern "C" {

CR_API const char *cr_status_string(cr_status s) {
    switch (s) {
    case CR_OK: return "CR_OK";
    case CR_ERR_INVALID_ARGUMENT: return "CR_ERR_INVALID_ARGUMENT";
    case CR_ERR_OUT_OF_MEMORY: return "CR_ERR_OUT_OF_MEMORY";
    case CR_ERR_CUDA: return "CR_ERR_CUDA";
    case CR_ERR_UNSUPPORTED: return "CR_ERR_UNSUPPORTED";
    case CR_ERR_CAPACITY: return "CR_ERR_CAPACITY";
    case CR_ERR_TIMEOUT: return "CR_ERR_TIMEOUT";
    case CR_ERR_NO_DEVICE: return "CR_ERR_NO_DEVICE";
    case CR_ERR_INTERNAL: return "CR_ERR_INTERNAL";
    }
    return "CR_ERR_UNKNOWN";
}

CR_API const char *cr_last_error_detail(void) { return cri::g_detail.c_str(); }

CR_API cr_status cr_layout_sizes(uint32_t sizes[5]) {
    if (!sizes) return fail(CR_ERR_INVALID_ARGUMENT, "sizes is null");
    sizes[0] = sizeof(cr_raster_batch);
    sizes[1] = sizeof(cr_raster_file);
    sizes[2] = sizeof(cr_raster_pixel);
    sizes[3] = sizeof(cr_visible_batch);
    sizes[4] = sizeof(cr_dispatch_args);
    return CR_OK;
}

CR_API cr_status cr_config_default(cr_config *out) {
    if (!out) return fail(CR_ERR_INVALID_ARGUMENT, "out is null");
    std::memset(out, 0, sizeof(*out));
    out->mode = CR_MODE_HIGH_QUALITY_AVERAGE;
    out->depthTolerance = 0.01f;
    out->enableFrustumCulling = 1;
    out->lodBias = 0;
    out->enableCLOD = 1;
    out->enableLODDither = 1;
    out->holeFillIterations = 0;
    out->pointSizeMode = CR_POINT_SIZE_SCREEN_SPACE;
    out->minimumPointSize = 1.0f;
    out->maximumPointSize = 1.0f;
    out->pointSizeScale = 1.0f;
    out->writesSceneDepth = 1;
    out->motionBlur = 0.0f;
    out->motionBlurSamples = 8;
    out->motionBlurMaxSpread = 64.0f;
    return CR_OK;
}

// ---------------------------------------------------------------- context
CR_API cr_status cr_context_create(int device, cr_context **out) {
    if (!out) return fail(CR_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(CR_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= n) return fail(CR_ERR_INVALID_ARGUMENT, "device out of range");
    DeviceGuard g(device);
    cudaDeviceProp prop;
    CR_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return fail(CR_ERR_NO_DEVICE, "this library is built for sm_100a (B200) devices");
    auto *ctx = new cr_context();
    ctx->pack = new PackScratch();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx->pack;
        delete ctx;
        return cri::cuda_fail(e, "cudaStreamCreateWithFlags");
    }
    // The device-side status word: page-locked host memory mapped into the
    // device's address space, so a kernel's store needs no copy to be seen.
    e = cudaHostAlloc(reinterpret_cast<void **>(&ctx->h_status), sizeof(uint32_t),
                      cudaHostAllocMapped);
    if (e == cudaSuccess)
        e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&ctx->d_status), ctx->h_status, 0);
    if (e != cudaSuccess) {
        if (ctx->h_status) cudaFreeHost(ctx->h_status);
        cudaStreamDestroy(ctx->stream);
        delete ctx->pack;
        delete ctx;
        return cri::cuda_fail(e, "cudaHostAlloc (status word)");
    }
    *ctx->h_status = 0u;
    *out = ctx;
    return CR_OK;
}

CR_API cr_status cr_context_destroy(cr_context *ctx) {
    if (!ctx) return CR_OK;
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto &fr : ctx->pass_ev)
        for (auto &pe : fr)
            for (auto &e : pe)
                if (e) cudaEventDestroy(e);
    if (ctx->pack) {
        pack_scratch_free(*ctx->pack);
        delete ctx->pack;
    }
    if (ctx->views) views_destroy(ctx->views);
    if (ctx->d_loss) cudaFree(ctx->d_loss);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    cudaStreamDestroy(ctx->stream);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    delete ctx;
    return CR_OK;
}

CR_API cr_status cr_context_synchronize(cr_context *ctx) {
    if (!ctx) return fail(CR_ERR_INVALID_ARGUMENT, "ctx is null");
    DeviceGuard g(ctx->device);
    CR_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->copy_stream) CR_CUDA(cudaStreamSynchronize(ctx->copy_stream));
    return device_status(ctx);
}

CR_API cr_status cr_context_stream(cr_context *ctx, void **stream_out) {
    if (!ctx || !stream_out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    *stream_out = (void *)ctx->stream;
    return CR_OK;
}

CR_API cr_status cr_context_trim(cr_context *ctx) {
    if (!ctx) return fail(CR_ERR_INVALID_ARGUMENT, "ctx is null");
    DeviceGuard g(ctx->device);
    CR_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->pack) pack_scratch_free(*ctx->pack);
    return CR_OK;
}

// ---------------------------------------------------------------- cloud
CR_API cr_status cr_cloud_create(cr_context *ctx, cr_capacity cap, const cr_raster_file *files,
                                 uint32_t nfiles, cr_cloud **out) {
    if (!ctx || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    // ComputeRasteriserCapacity preconditions (ComputeRasteriserPointCloud.swift:31-36).
    if (cap.maxResidentBatches == 0) return fail(CR_ERR_INVALID_ARGUMENT, "maxResidentBatches must be positive");
    if (cap.pointsPerBatch == 0) return fail(CR_ERR_INVALID_ARGUMENT, "pointsPerBatch must be positive");
    if ((uint64_t)cap.maxResidentBatches * cap.pointsPerBatch >= 0xffffffffull)
        return fail(CR_ERR_CAPACITY, "pool exceeds 2^32-1 points (point indices are 32-bit)");
    if (nfiles > 0 && !files) return fail(CR_ERR_INVALID_ARGUMENT, "files is null");
    DeviceGuard g(ctx->device);
    auto *c = new cr_cloud();
    c->ctx = ctx;
    cr_status st = allocate_cloud(c, cap, files, nfiles);
    if (st != CR_OK) {
        std::string d = cr_last_error_detail();
        free_cloud_buffers(c);
        delete c;
        return fail(st, d);
    }
    *out = c;
    return CR_OK;
}

CR_API cr_status cr_cloud_destroy(cr_cloud *c) {
    if (!c) return CR_OK;
    DeviceGuard g(c->ctx->device);
    uploads_free(c);  // waits for copies in flight
    cudaStreamSynchronize(c->ctx->stream);
    free_cloud_buffers(c);
    if (c->h_files_ring) cudaFreeHost(c->h_files_ring);
    for (auto &e : c->ring_events)
        if (e) cudaEventDestroy(e);
    delete c;
    return CR_OK;
}

CR_API cr_status cr_cloud_reallocate(cr_cloud *c, cr_capacity cap, const cr_raster_file *files,
                                     uint32_t nfiles) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    if (cap.maxResidentBatches == 0 || cap.pointsPerBatch == 0)
        return fail(CR_ERR_INVALID_ARGUMENT, "capacity must be positive");
    if ((uint64_t)cap.maxResidentBatches * cap.pointsPerBatch >= 0xffffffffull)
        return fail(CR_ERR_CAPACITY, "pool exceeds 2^32-1 points");
    DeviceGuard g(c->ctx->device);
    uploads_free(c);  // the slot table and pool change size
    CR_CUDA(cudaStreamSynchronize(c->ctx->stream));
    std::vector<cr_raster_file> keep;
    if (files && nfiles) keep.assign(files, files + nfiles);
    else keep = c->files;
    return allocate_cloud(c, cap, keep.data(), (uint32_t)keep.size());
}

CR_API cr_status cr_cloud_set_files(cr_cloud *c, const cr_raster_file *files, uint32_t nfiles) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    if (nfiles > 0 && !files) return fail(CR_ERR_INVALID_ARGUMENT, "files is null");
    DeviceGuard g(c->ctx->device);
    if (nfiles == 0) c->files.assign(1, identity_file());
    else c->files.assign(files, files + nfiles);
    c->frame_files = c->files;
    if (c->files.size() > c->d_files_cap) {
        CR_CUDA(cudaStreamSynchronize(c->ctx->stream));
        dfree(c->d_files);
        cr_status st = dalloc(&c->d_files, c->files.size() * sizeof(cr_raster_file));
        if (st) return st;
        c->d_files_cap = (uint32_t)c->files.size();
        if ((st = alloc_ring(c))) return st;
    }
    return upload_files(c, c->files);
}

CR_API cr_status cr_cloud_add_batches(cr_cloud *c, const uint32_t *low, const uint32_t *med,
                                      const uint32_t *high, const uint32_t *colors,
                                      const uint8_t *levels, uint64_t points_len,
                                      const cr_raster_batch *batches, uint32_t n, int commit,
                                      int32_t *slots_out) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    if (n > c->free_slots.size())
        return fail(CR_ERR_CAPACITY, "addBatches: not enough free slots (have " +
                                         std::to_string(c->free_slots.size()) + ", need " +
                                         std::to_string(n) + ")");
    if (n == 0) return CR_OK;
    if (!batches || !low || !med || !high || !colors || !levels)
        return fail(CR_ERR_INVALID_ARGUMENT, "null array");
    for (uint32_t i = 0; i < n; ++i) {
        const uint64_t src = batches[i].firstPoint, cnt = batches[i].numPoints;
        if (cnt > c->cap.pointsPerBatch)
            return fail(CR_ERR_CAPACITY, "batch numPoints (" + std::to_string(cnt) +
                                             ") exceeds slot capacity (" +
                                             std::to_string(c->cap.pointsPerBatch) + ")");
        if (src + cnt > points_len)
            return fail(CR_ERR_INVALID_ARGUMENT, "addBatches: source data too small for batch");
        if (batches[i].fileIndex >= c->files.size())
            return fail(CR_ERR_INVALID_ARGUMENT, "batch fileIndex outside the file table");
    }
    DeviceGuard g(c->ctx->device);
    cudaStream_t s = c->ctx->stream;
    // Copies of consecutive batches into consecutive slots merge into one run.
    uint64_t run_src = 0, run_dst = 0, run_n = 0;
    auto flush_run = [&]() -> cr_status {
        if (run_n == 0) return CR_OK;
        CR_CUDA(cudaMemcpyAsync(c->d_low + run_dst, low + run_src, run_n * 4, cudaMemcpyHostToDevice, s));
        CR_CUDA(cudaMemcpyAsync(c->d_med + run_dst, med + run_src, run_n * 4, cudaMemcpyHostToDevice, s));
        CR_CUDA(cudaMemcpyAsync(c->d_high + run_dst, high + run_src, run_n * 4, cudaMemcpyHostToDevice, s));
        CR_CUDA(cudaMemcpyAsync(c->d_colors + run_dst, colors + run_src, run_n * 4, cudaMemcpyHostToDevice, s));
        CR_CUDA(cudaMemcpyAsync(c->d_levels + run_dst, levels + run_src, run_n, cudaMemcpyHostToDevice, s));
        run_n = 0;
        return CR_OK;
    };
    for (uint32_t i = 0; i < n; ++i) {
        const int32_t slot = c->free_slots.back();
        c->free_slots.pop_back();
        if (slots_out) slots_out[i] = slot;
        const uint64_t dst = (uint64_t)slot * c->cap.pointsPerBatch;
        const uint64_t src = batches[i].firstPoint, cnt = batches[i].numPoints;
        if (cnt > 0) {
            if (run_n > 0 && run_src + run_n == src && run_dst + run_n == dst) {
                run_n += cnt;
            } else {
                cr_status st = flush_run();
                if (st) return st;
                run_src = src;
                run_dst = dst;
                run_n = cnt;
            }
        }
        cr_raster_batch b = batches[i];
        b.firstPoint = (uint32_t)dst;
        b.state = 1;
        c->mirror[slot] = b;
        mark_dirty(c, slot, slot);
        c->resident += 1;
        c->points += cnt;
    }
    cr_status st = flush_run();
    if (st) return st;
    if (commit) return flush_mirror(c);
    return CR_OK;
}

CR_API cr_status cr_cloud_remove_batches(cr_cloud *c, const int32_t *slots, uint32_t n, int commit) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    if (n == 0) return CR_OK;
    if (!slots) return fail(CR_ERR_INVALID_ARGUMENT, "slots is null");
    for (uint32_t i = 0; i < n; ++i)
        if (slots[i] < 0 || (uint32_t)slots[i] >= c->cap.maxResidentBatches)
            return fail(CR_ERR_INVALID_ARGUMENT,
                        "removeBatches: slot " + std::to_string(slots[i]) + " out of range");
    for (uint32_t i = 0; i < n; ++i) {
        if (uploads_cancel(c, slots[i])) continue;  // freed when its copy lands
        cr_raster_batch &b = c->mirror[slots[i]];
        if (b.state == 0) continue;
        c->points -= b.numPoints;
        c->resident -= 1;
        b.state = 0;
        b.numPoints = 0;
        mark_dirty(c, slots[i], slots[i]);
        c->free_slots.push_back(slots[i]);
    }
    if (commit) {
        DeviceGuard g(c->ctx->device);
        return flush_mirror(c);
    }
    return CR_OK;
}

CR_API cr_status cr_cloud_commit(cr_cloud *c) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    DeviceGuard g(c->ctx->device);
    return flush_mirror(c);
}

CR_API cr_status cr_cloud_clear(cr_cloud *c) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    cr_status st = uploads_drain(c);
    if (st) return st;
    for (auto &b : c->mirror) {
        b.state = 0;
        b.numPoints = 0;
    }
    c->free_slots.clear();
    for (int64_t s = (int64_t)c->cap.maxResidentBatches - 1; s >= 0; --s)
        c->free_slots.push_back((int32_t)s);
    c->resident = 0;
    c->points = 0;
    mark_dirty(c, 0, (int64_t)c->mirror.size() - 1);
    DeviceGuard g(c->ctx->device);
    return flush_mirror(c);
}

CR_API cr_status cr_cloud_update_files(cr_cloud *c, const float vp[16], const float model[16],
                                       const float *frustum, const float *prev_vp) {
    if (!c || !vp || !model) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    DeviceGuard g(c->ctx->device);
    std::vector<cr_raster_file> snap = c->files;
    for (size_t i = 0; i < snap.size(); ++i) {
        float world[16];
        mat4mul(model, c->files[i].world, world);
        mat4mul(vp, world, snap[i].transform);
        mat4mul(frustum ? frustum : vp, world, snap[i].transformFrustum);
        std::memcpy(snap[i].world, world, sizeof(world));
        mat4mul(prev_vp ? prev_vp : vp, world, snap[i].prevTransform);
    }
    c->frame_files = snap;
    return upload_files(c, snap);
}

CR_API cr_status cr_cloud_attribute(cr_cloud *c, int32_t which, void **device_ptr,
                                    uint64_t *count) {
    if (!c || !device_ptr) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    float4 **slot = which == CR_ATTR_DISPLACEMENT        ? &c->d_disp
                    : which == CR_ATTR_PREV_DISPLACEMENT ? &c->d_prev_disp
                    : which == CR_ATTR_TINT               ? &c->d_tint
                                                          : nullptr;
    if (!slot) return fail(CR_ERR_INVALID_ARGUMENT, "unknown attribute");
    DeviceGuard g(c->ctx->device);
    const size_t n = attribute_points(c);
    if (!*slot) {
        cr_status st = dalloc(slot, n * sizeof(float4));
        if (st) return st;
        CR_CUDA(cudaMemsetAsync(*slot, 0, n * sizeof(float4), c->ctx->stream));
    }
    *device_ptr = *slot;
    if (count) *count = n;
    return CR_OK;
}

CR_API cr_status cr_cloud_release_attribute(cr_cloud *c, int32_t which) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    float4 **slot = which == CR_ATTR_DISPLACEMENT        ? &c->d_disp
                    : which == CR_ATTR_PREV_DISPLACEMENT ? &c->d_prev_disp
                    : which == CR_ATTR_TINT               ? &c->d_tint
                                                          : nullptr;
    if (!slot) return fail(CR_ERR_INVALID_ARGUMENT, "unknown attribute");
    DeviceGuard g(c->ctx->device);
    CR_CUDA(cudaStreamSynchronize(c->ctx->stream));
    dfree(*slot);
    return CR_OK;
}

CR_API cr_status cr_cloud_device_arrays(cr_cloud *c, cr_cloud_arrays *out) {
    if (!c || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    out->batches = c->d_batches;
    out->xyzLow = c->d_low;
    out->xyzMed = c->d_med;
    out->xyzHigh = c->d_high;
    out->colors = c->d_colors;
    out->levels = c->d_levels;
    out->points = (uint64_t)c->cap.maxResidentBatches * c->cap.pointsPerBatch;
    out->slots = c->cap.maxResidentBatches;
    out->pointsPerBatch = c->cap.pointsPerBatch;
    return CR_OK;
}

CR_API cr_status cr_cloud_info_get(const cr_cloud *c, cr_cloud_info *out) {
    if (!c || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    out->capacity = c->cap;
    out->residentBatchCount = c->resident;
    out->pointCount = c->points;
    out->freeSlotCount = (uint32_t)c->free_slots.size();
    out->fileCount = (uint32_t)c->files.size();
    return CR_OK;
}

CR_API cr_status cr_cloud_read_files(const cr_cloud *c, cr_raster_file *out, uint32_t n) {
    if (!c || (!out && n)) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if (n > c->frame_files.size()) return fail(CR_ERR_INVALID_ARGUMENT, "n exceeds file count");
    std::memcpy(out, c->frame_files.data(), n * sizeof(cr_raster_file));
    return CR_OK;
}

CR_API cr_status cr_cloud_read_batches(cr_cloud *c, cr_raster_batch *out, uint32_t first, uint32_t n) {
    if (!c || (!out && n)) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if ((uint64_t)first + n > c->cap.maxResidentBatches)
        return fail(CR_ERR_INVALID_ARGUMENT, "slot range out of bounds");
    if (n == 0) return CR_OK;
    DeviceGuard g(c->ctx->device);
    CR_CUDA(cudaMemcpyAsync(out, c->d_batches + first, n * sizeof(cr_raster_batch),
                            cudaMemcpyDeviceToHost, c->ctx->stream));
    CR_CUDA(cudaStreamSynchronize(c->ctx->stream));
    return CR_OK;
}

CR_API cr_status cr_cloud_read_points(cr_cloud *c, uint64_t first, uint64_t n, uint32_t *low,
                                      uint32_t *med, uint32_t *high, uint32_t *colors,
                                      uint8_t *levels) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    const uint64_t total = (uint64_t)c->cap.maxResidentBatches * c->cap.pointsPerBatch;
    if (first + n > total) return fail(CR_ERR_INVALID_ARGUMENT, "point range out of bounds");
    if (n == 0) return CR_OK;
    DeviceGuard g(c->ctx->device);
    cudaStream_t s = c->ctx->stream;
    if (low) CR_CUDA(cudaMemcpyAsync(low, c->d_low + first, n * 4, cudaMemcpyDeviceToHost, s));
    if (med) CR_CUDA(cudaMemcpyAsync(med, c->d_med + first, n * 4, cudaMemcpyDeviceToHost, s));
    if (high) CR_CUDA(cudaMemcpyAsync(high, c->d_high + first, n * 4, cudaMemcpyDeviceToHost, s));
    if (colors) CR_CUDA(cudaMemcpyAsync(colors, c->d_colors + first, n * 4, cudaMemcpyDeviceToHost, s));
    if (levels) CR_CUDA(cudaMemcpyAsync(levels, c->d_levels + first, n, cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    return CR_OK;
}

CR_API cr_status cr_cloud_read_visible(cr_cloud *c, cr_visible_batch *out, uint32_t cap,
                                       uint32_t *count_out) {
    if (!c || !count_out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    DeviceGuard g(c->ctx->device);
    cudaStream_t s = c->ctx->stream;
    uint32_t count = 0;
    CR_CUDA(cudaMemcpyAsync(&count, c->d_counters + CNT_VISIBLE, 4, cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    *count_out = count;
    const uint32_t k = std::min(count, cap);
    if (k && out) {
        CR_CUDA(cudaMemcpyAsync(out, c->d_visible, k * sizeof(cr_visible_batch),
                                cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
    }
    return device_status(c->ctx);
}

// ---------------------------------------------------------------- frame
CR_API cr_status cr_frame_create(cr_context *ctx, int w, int h, cr_frame **out) {
    if (!ctx || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (w <= 0 || h <= 0) return fail(CR_ERR_INVALID_ARGUMENT, "frame size must be positive");
    if ((uint64_t)w * (uint64_t)h >= (1ull << 31))
        return fail(CR_ERR_CAPACITY, "frame exceeds 2^31 pixels");
    if (w > 65535 || h > 65535)
        return fail(CR_ERR_CAPACITY, "frame width and height must be at most 65535");
    DeviceGuard g(ctx->device);
    auto *f = new cr_frame();
    f->ctx = ctx;
    f->width = w;
    f->height = h;
    const size_t npix = (size_t)w * h;
    cr_status st;
    if ((st = dalloc(&f->d_depth, npix * 4)) || (st = dalloc(&f->d_accum, (npix + 1) * 16)) ||
        (st = dalloc(&f->d_nearest, npix * 8)) || (st = dalloc(&f->d_rgba[0], npix * 4)) ||
        (st = dalloc(&f->d_rgba[1], npix * 4)) || (st = dalloc(&f->d_depthf, npix * 4))) {
        std::string d = cr_last_error_detail();
        cr_frame_destroy(f);
        return fail(st, d);
    }
    f->d_redo = reinterpret_cast<uint32_t *>(f->d_accum + npix);
    cudaStream_t s = ctx->stream;
    cudaMemsetAsync(f->d_depth, 0, npix * 4, s);
    cudaMemsetAsync(f->d_accum, 0, (npix + 1) * 16, s);
    cudaMemsetAsync(f->d_nearest, 0, npix * 8, s);
    cudaMemsetAsync(f->d_rgba[0], 0, npix * 4, s);
    cudaMemsetAsync(f->d_rgba[1], 0, npix * 4, s);
    cudaMemsetAsync(f->d_depthf, 0, npix * 4, s);
    CR_CUDA(cudaStreamSynchronize(s));
    *out = f;
    return CR_OK;
}

CR_API cr_status cr_frame_destroy(cr_frame *f) {
    if (!f) return CR_OK;
    DeviceGuard g(f->ctx->device);
    cudaStreamSynchronize(f->ctx->stream);
    if (f->ev_copied) {
        cudaEventSynchronize(f->ev_copied);
        cudaEventDestroy(f->ev_copied);
    }
    for (cudaEvent_t e : f->ev_copy_ring)
        if (e) cudaEventDestroy(e);
    if (f->ev_rendered) cudaEventDestroy(f->ev_rendered);
    dfree(f->d_depth);
    dfree(f->d_accum);
    dfree(f->d_nearest);
    dfree(f->d_rgba[0]);
    dfree(f->d_rgba[1]);
    dfree(f->d_depthf);
    dfree(f->d_fsum);
    dfree(f->d_fcount);
    delete f;
    return CR_OK;
}

// cr_render and cr_render_stages: the HQS passes in three stages that a host
// may separate to combine frames' planes between them (a frame sharded by
// points over several GPUs).  Packed colour adds (with the exact re-run) only
// when the colour and resolve stages run in one call.
static cr_status render_impl(cr_context *ctx, cr_frame *f, cr_cloud *const *clouds,
                             uint32_t nclouds, const cr_config *cfg, const cr_camera *cam,
                             uint32_t stages) {
    cr_status st = validate_render(ctx, f, cfg, cam);
    if (st) return st;
    if (nclouds && !clouds) return fail(CR_ERR_INVALID_ARGUMENT, "clouds is null");
    for (uint32_t i = 0; i < nclouds; ++i)
        if (!clouds[i] || clouds[i]->ctx != ctx)
            return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null or from another context");
    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    const int W = f->width, H = f->height;
    const size_t npix = (size_t)W * H;
    ResolveUniforms ru{W, H, {cfg->backgroundColor[0], cfg->backgroundColor[1],
                              cfg->backgroundColor[2], cfg->backgroundColor[3]}};
    if (ctx->profiling && (stages & CR_STAGE_DEPTH)) {
        ctx->prof_frame = (ctx->prof_frame + 1) % cr_context::kProfRing;
        ctx->prof_count += 1;
        for (int p = 0; p < CR_PASS_COUNT; ++p) ctx->pass_recorded[ctx->prof_frame][p] = false;
    }
    if (cfg->mode == CR_MODE_HIGH_QUALITY_AVERAGE) {
        // encodeHighQualityAverage (ComputeRasteriser.swift:322-456).
        std::vector<cr_cloud *> resident;
        uint64_t max_samples = 0;  // upper bound on the frame's colour samples
        for (uint32_t i = 0; i < nclouds; ++i)
            if (clouds[i]->resident > 0) {
                resident.push_back(clouds[i]);
                max_samples += (uint64_t)clouds[i]->resident * clouds[i]->cap.pointsPerBatch;
            }
        const RasterUniforms rau = make_raster_uniforms(cfg, cam, W, H);
        // Colour variants (ComputeRasteriser.swift:229-253): their own depth
        // and colour passes with 32-bit adds, and the coverage resolve when
        // translucent defocus or motion blur is on.
        const bool variants = variants_on(cfg);
        const bool coverage =
            variants && ((cfg->applyTint && cfg->tintAlphaIsCoverage) || cfg->motionBlur > 0.0f);
        // With single-pixel footprints the depth pass keeps every point that
        // reaches the screen as a fragment and the colour pass reads those
        // instead of decoding and projecting the points again.
        const bool frags =
            !variants && std::fmax(cfg->minimumPointSize, cfg->maximumPointSize) <= 1.0f;
        // Packed colour adds while the frame holds fewer than 2^31 samples:
        // then a pixel's count field reads its true count plus at most 127
        // carries out of the blue sum, so a read count of at most
        // kPackedMaxCount proves that no field carried.
        const bool packed = !variants && (stages & CR_STAGE_COLOR) && (stages & CR_STAGE_RESOLVE) &&
                            max_samples < (1ull << 31);
        RasterTargets t{f->d_depth, f->d_accum, f->d_nearest};
        t.packed = packed ? 1 : 0;
        if (stages & CR_STAGE_DEPTH) {
            // The frame's depth plane, accumulators and redo word are zeroed
            // by extra CTAs of the first cull launch (its CTAs are few and
            // latency-bound), or by their own launch without a cloud to cull.
            const bool clear_in_cull = !resident.empty() && resident[0]->cap.maxResidentBatches > 0;
            if (!clear_in_cull) {
                PassTimer pt(ctx, CR_PASS_CLEAR);
                if ((st = launch_frame_clear(f, s))) return st;
            }
            const CullUniforms cu = make_cull_uniforms(cfg, cam, W, H);
            {
                PassTimer pt(ctx, CR_PASS_CULL);
                const FrameClear fc = frame_clear_of(f);
                for (size_t i = 0; i < resident.size(); ++i)
                    if ((st = launch_cull(resident[i], cu, s,
                                          i == 0 && clear_in_cull ? &fc : nullptr)))
                        return st;
            }
            {
                PassTimer pt(ctx, CR_PASS_DEPTH);
                for (cr_cloud *c : resident)
                    if ((st = variants ? launch_variant_pass(c, false, rau, *cfg, t, s)
                                       : launch_raster(c, frags ? PASS_DEPTH_FRAG : PASS_DEPTH,
                                                       rau, t, s)))
                        return st;
            }
        }
        if (stages & CR_STAGE_COLOR) {
            PassTimer pt(ctx, CR_PASS_COLOR);
            for (cr_cloud *c : resident)
                if ((st = variants ? launch_variant_pass(c, true, rau, *cfg, t, s)
                                   : launch_raster(c, frags ? PASS_COLOR_FRAG : PASS_COLOR, rau,
                                                   t, s)))
                    return st;
            // Motion blur: this frame's displacement is the next frame's
            // previous one (ComputeRasteriser.swift:453-480).
            if (variants && cfg->motionBlur > 0.0f)
                for (cr_cloud *c : resident) {
                    if (!c->d_disp) continue;
                    const size_t bytes = attribute_points(c) * sizeof(float4);
                    if (!c->d_prev_disp && (st = dalloc(&c->d_prev_disp, bytes))) return st;
                    CR_CUDA(cudaMemcpyAsync(c->d_prev_disp, c->d_disp, bytes,
                                            cudaMemcpyDeviceToDevice, s));
                }
        }
        if (stages & CR_STAGE_RESOLVE) {
            PassTimer pt(ctx, CR_PASS_RESOLVE);
            if ((st = frame_copy_fence(f, s))) return st;
            if (coverage) {
                if ((st = launch_resolve_coverage(f, ru, s))) return st;
            } else if ((st = launch_resolve_hqs(f, ru, s, packed, nullptr))) {
                return st;
            }
            if (packed) {
                // Exact re-run, which returns at once unless the resolve set
                // the redo flag: zero the accumulators, colour pass with one
                // 32-bit add per field, resolve.
                RasterTargets tx = t;
                tx.packed = 0;
                tx.redo = f->d_redo;
                if (frags && resident.size() <= hqs_redo_max_clouds()) {
                    // From the fragments: all three steps in one launch.
                    if ((st = launch_hqs_redo(f, resident.data(), (uint32_t)resident.size(), rau,
                                              tx, ru, s)))
                        return st;
                } else {
                    if ((st = launch_accum_redo_clear(f, s))) return st;
                    for (cr_cloud *c : resident)
                        if ((st = launch_raster(c, frags ? PASS_COLOR_FRAG : PASS_COLOR, rau, tx,
                                                s)))
                            return st;
                    if ((st = launch_resolve_hqs(f, ru, s, false, f->d_redo))) return st;
                }
            }
            f->last_mode = 0;
        }
    } else {
        // encodeNearestPoint (ComputeRasteriser.swift:483-497): first resident cloud only.
        cr_cloud *first = nullptr;
        for (uint32_t i = 0; i < nclouds && !first; ++i)
            if (clouds[i]->resident > 0) first = clouds[i];
        if (first) {
            {
                PassTimer pt(ctx, CR_PASS_CLEAR);
                CR_CUDA(cudaMemsetAsync(f->d_nearest, 0, npix * sizeof(unsigned long long), s));
            }
            {
                PassTimer pt(ctx, CR_PASS_CULL);
                if ((st = launch_cull(first, make_cull_uniforms(cfg, cam, W, H), s))) return st;
            }
            {
                PassTimer pt(ctx, CR_PASS_DEPTH);
                const RasterTargets t{f->d_depth, f->d_accum, f->d_nearest};
                if ((st = launch_raster(first, PASS_NEAREST, make_raster_uniforms(cfg, cam, W, H),
                                        t, s)))
                    return st;
            }
            {
                PassTimer pt(ctx, CR_PASS_RESOLVE);
                if ((st = frame_copy_fence(f, s))) return st;
                if ((st = launch_resolve_nearest(f, first->d_colors, ru, s))) return st;
            }
            f->last_mode = 1;
        }
    }
    if (!(stages & CR_STAGE_RESOLVE)) return CR_OK;
    // encodeHoleFill (ComputeRasteriser.swift:298-320) always starts from the
    // resolve target.
    f->final_rgba = 0;
    if (cfg->holeFillIterations > 0) {
        PassTimer pt(ctx, CR_PASS_HOLE_FILL);
        if ((st = frame_copy_fence(f, s))) return st;
        return launch_hole_fill(f, cfg->holeFillIterations, s);
    }
    return CR_OK;
}

CR_API cr_status cr_render(cr_context *ctx, cr_frame *f, cr_cloud *const *clouds,
                           uint32_t nclouds, const cr_config *cfg, const cr_camera *cam) {
    return render_impl(ctx, f, clouds, nclouds, cfg, cam, CR_STAGE_ALL);
}

CR_API cr_status cr_render_stages(cr_context *ctx, cr_frame *f, cr_cloud *const *clouds,
                                  uint32_t nclouds, const cr_config *cfg, const cr_camera *cam,
                                  uint32_t stages) {
    if (stages == 0 || (stages & ~(uint32_t)CR_STAGE_ALL))
        return fail(CR_ERR_INVALID_ARGUMENT, "stages must be a non-empty set of CR_STAGE_* bits");
    if (cfg && cfg->mode != CR_MODE_HIGH_QUALITY_AVERAGE && stages != CR_STAGE_ALL)
        return fail(CR_ERR_UNSUPPORTED, "separate stages need the HQS mode");
    return render_impl(ctx, f, clouds, nclouds, cfg, cam, stages);
}

CR_API cr_status cr_frame_device_planes(cr_frame *f, cr_frame_planes *out) {
    if (!f || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    out->depth = f->d_depth;
    out->accum = f->d_accum;
    out->pixels = (uint64_t)f->width * f->height;
    out->stream = (void *)f->ctx->stream;
    return CR_OK;
}

CR_API cr_status cr_frame_flip_depth_order(cr_frame *f) {
    if (!f) return fail(CR_ERR_INVALID_ARGUMENT, "frame is null");
    DeviceGuard g(f->ctx->device);
    return launch_flip_depth_order(f, f->ctx->stream);
}

static cr_status read_plane(cr_frame *f, void *out, const void *src, size_t bytes) {
    if (!f || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    DeviceGuard g(f->ctx->device);
    CR_CUDA(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, f->ctx->stream));
    CR_CUDA(cudaStreamSynchronize(f->ctx->stream));
    return device_status(f->ctx);
}

CR_API cr_status cr_frame_read_rgba8(cr_frame *f, uint8_t *out) {
    if (!f) return fail(CR_ERR_INVALID_ARGUMENT, "frame is null");
    return read_plane(f, out, f->d_rgba[f->final_rgba], (size_t)f->width * f->height * 4);
}

CR_API cr_status cr_frame_read_rgba8_async(cr_frame *f, uint8_t *out) {
    if (!f || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    cr_context *ctx = f->ctx;
    DeviceGuard g(ctx->device);
    if (!ctx->copy_stream)
        CR_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    if (!f->ev_rendered) CR_CUDA(cudaEventCreateWithFlags(&f->ev_rendered, cudaEventDisableTiming));
    if (!f->ev_copied) CR_CUDA(cudaEventCreateWithFlags(&f->ev_copied, cudaEventDisableTiming));
    CR_CUDA(cudaEventRecord(f->ev_rendered, ctx->stream));
    CR_CUDA(cudaStreamWaitEvent(ctx->copy_stream, f->ev_rendered, 0));
    CR_CUDA(cudaMemcpyAsync(out, f->d_rgba[f->final_rgba], (size_t)f->width * f->height * 4,
                            cudaMemcpyDeviceToHost, ctx->copy_stream));
    CR_CUDA(cudaEventRecord(f->ev_copied, ctx->copy_stream));
    cudaEvent_t &slot = f->ev_copy_ring[f->copies % cr_frame::kCopyRing];
    if (!slot) CR_CUDA(cudaEventCreateWithFlags(&slot, cudaEventDisableTiming));
    CR_CUDA(cudaEventRecord(slot, ctx->copy_stream));
    ++f->copies;
    f->copy_pending = true;
    return CR_OK;
}

CR_API cr_status cr_frame_read_wait(cr_frame *f) {
    if (!f) return fail(CR_ERR_INVALID_ARGUMENT, "frame is null");
    if (!f->ev_copied) return CR_OK;
    DeviceGuard g(f->ctx->device);
    CR_CUDA(cudaEventSynchronize(f->ev_copied));
    return device_status(f->ctx);
}

CR_API cr_status cr_frame_read_wait_keep(cr_frame *f, int keep) {
    if (!f) return fail(CR_ERR_INVALID_ARGUMENT, "frame is null");
    if (keep < 0 || keep >= cr_frame::kCopyRing)
        return fail(CR_ERR_INVALID_ARGUMENT,
                    "keep must be 0.." + std::to_string(cr_frame::kCopyRing - 1));
    if (keep == 0) return cr_frame_read_wait(f);
    if (f->copies <= (uint64_t)keep) return CR_OK;
    DeviceGuard g(f->ctx->device);
    // The copy stream runs the read-backs in order: once read-back
    // copies - 1 - keep has finished, every earlier one has too.
    const uint64_t n = f->copies - 1 - (uint64_t)keep;
    CR_CUDA(cudaEventSynchronize(f->ev_copy_ring[n % cr_frame::kCopyRing]));
    return device_status(f->ctx);
}

CR_API cr_status cr_frame_read_depth_f32(cr_frame *f, float *out) {
    if (!f) return fail(CR_ERR_INVALID_ARGUMENT, "frame is null");
    return read_plane(f, out, f->d_depthf, (size_t)f->width * f->height * 4);
}

CR_API cr_status cr_frame_read_pixels(cr_frame *f, cr_raster_pixel *out) {
    if (!f || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    const size_t npix = (size_t)f->width * f->height;
    std::vector<uint32_t> depth(npix);
    std::vector<uint4> acc(npix);
    cr_status st = read_plane(f, depth.data(), f->d_depth, npix * 4);
    if (st) return st;
    if ((st = read_plane(f, acc.data(), f->d_accum, npix * 16))) return st;
    for (size_t p = 0; p < npix; ++p) {
        out[p].depth = depth[p];
        out[p].red = acc[p].x;
        out[p].green = acc[p].y;
        out[p].blue = acc[p].z;
        out[p].count = acc[p].w;
        out[p].weight = 0;
        out[p].padding[0] = out[p].padding[1] = 0;
    }
    return CR_OK;
}

static cr_status read_nearest(cr_frame *f, uint32_t *depth, uint32_t *index, int row0, int nrows) {
    if (!f) return fail(CR_ERR_INVALID_ARGUMENT, "frame is null");
    if (row0 < 0 || nrows < 0 || row0 + nrows > f->height)
        return fail(CR_ERR_INVALID_ARGUMENT, "row range out of bounds");
    const size_t n = (size_t)nrows * f->width;
    if (n == 0) return CR_OK;
    std::vector<unsigned long long> keys(n);
    cr_status st = read_plane(f, keys.data(), f->d_nearest + (size_t)row0 * f->width, n * 8);
    if (st) return st;
    for (size_t p = 0; p < n; ++p) {
        if (depth) depth[p] = (uint32_t)(keys[p] >> 32);
        if (index) index[p] = ~(uint32_t)keys[p];
    }
    return CR_OK;
}

CR_API cr_status cr_frame_read_nearest_depth(cr_frame *f, uint32_t *out) {
    if (!out) return fail(CR_ERR_INVALID_ARGUMENT, "out is null");
    return read_nearest(f, out, nullptr, 0, f ? f->height : 0);
}

CR_API cr_status cr_frame_read_nearest_index(cr_frame *f, uint32_t *out) {
    if (!out) return fail(CR_ERR_INVALID_ARGUMENT, "out is null");
    return read_nearest(f, nullptr, out, 0, f ? f->height : 0);
}

CR_API cr_status cr_frame_read_nearest_index_rows(cr_frame *f, int row0, int nrows, uint32_t *out) {
    if (!out) return fail(CR_ERR_INVALID_ARGUMENT, "out is null");
    return read_nearest(f, nullptr, out, row0, nrows);
}

// pickPointIndex (ComputeRasteriser.swift:609-670).
// ---------------------------------------------------------------- differentiable colours
// The HQS colour pass with learnable FP32 colours (an FP32 variant beside the
// integer path; no counterpart in the reference) and its adjoint.

static cr_status validate_f32(cr_context *ctx, cr_frame *f, cr_cloud *cloud, const cr_config *cfg,
                              const cr_camera *cam, const void *in, const void *out) {
    cr_status st = validate_render(ctx, f, cfg, cam);
    if (st) return st;
    if (!cloud || cloud->ctx != ctx)
        return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null or from another context");
    if (!in || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null device pointer");
    if (cfg->mode != CR_MODE_HIGH_QUALITY_AVERAGE)
        return fail(CR_ERR_UNSUPPORTED, "differentiable colours need the HQS mode");
    if (cfg->colorizeChunks || cfg->colorizeOverdraw)
        return fail(CR_ERR_UNSUPPORTED, "colorize options replace the learnable colours");
    return reject_variants(cfg, "differentiable colours");
}

CR_API cr_status cr_hqs_forward_f32(cr_context *ctx, cr_frame *f, cr_cloud *cloud,
                                    const cr_config *cfg, const cr_camera *cam,
                                    const float *colors, float *image) {
    cr_status st = validate_f32(ctx, f, cloud, cfg, cam, colors, image);
    if (st) return st;
    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    const size_t npix = (size_t)f->width * f->height;
    if (!f->d_fsum) {
        if ((st = dalloc(&f->d_fsum, npix * sizeof(float4))) ||
            (st = dalloc(&f->d_fcount, npix * 4)))
            return st;
    }
    CR_CUDA(cudaMemsetAsync(f->d_depth, 0, npix * 4, s));
    CR_CUDA(cudaMemsetAsync(f->d_fsum, 0, npix * sizeof(float4), s));
    CR_CUDA(cudaMemsetAsync(f->d_fcount, 0, npix * 4, s));
    if (cloud->resident > 0) {
        const RasterUniforms rau = make_raster_uniforms(cfg, cam, f->width, f->height);
        RasterTargets t{f->d_depth, f->d_accum, f->d_nearest};
        t.fsum = f->d_fsum;
        t.fcount = f->d_fcount;
        if ((st = launch_cull(cloud, make_cull_uniforms(cfg, cam, f->width, f->height), s)) ||
            (st = launch_raster(cloud, PASS_DEPTH, rau, t, s)) ||
            (st = launch_raster_f32(cloud, PASS_COLOR_F32, rau, t, colors, nullptr, nullptr, s)))
            return st;
    }
    const float bg[3] = {cfg->backgroundColor[0], cfg->backgroundColor[1],
                         cfg->backgroundColor[2]};
    return launch_resolve_f32(f, bg, image, s);
}

CR_API cr_status cr_hqs_backward_colors(cr_context *ctx, cr_frame *f, cr_cloud *cloud,
                                        const cr_config *cfg, const cr_camera *cam,
                                        const float *dL_dimage, float *dL_dcolors) {
    cr_status st = validate_f32(ctx, f, cloud, cfg, cam, dL_dimage, dL_dcolors);
    if (st) return st;
    if (!f->d_fsum)
        return fail(CR_ERR_INVALID_ARGUMENT, "cr_hqs_forward_f32 has not run on this frame");
    if (cloud->resident == 0) return CR_OK;
    DeviceGuard g(ctx->device);
    const RasterUniforms rau = make_raster_uniforms(cfg, cam, f->width, f->height);
    RasterTargets t{f->d_depth, f->d_accum, f->d_nearest};
    t.fsum = f->d_fsum;
    t.fcount = f->d_fcount;
    return launch_raster_f32(cloud, PASS_GRAD, rau, t, nullptr, dL_dimage, dL_dcolors,
                             ctx->stream);
}

CR_API cr_status cr_l2_loss(cr_context *ctx, const float *image, const float *target, uint64_t n,
                            float scale, float *dL_dimage, double *loss) {
    if (!ctx || (n && (!image || !target || !dL_dimage)))
        return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    cr_status st;
    if (loss && !ctx->d_loss && (st = dalloc(&ctx->d_loss, sizeof(double)))) return st;
    if (loss) CR_CUDA(cudaMemsetAsync(ctx->d_loss, 0, sizeof(double), s));
    if ((st = launch_l2_loss(image, target, n, scale, dL_dimage, loss ? ctx->d_loss : nullptr,
                             ctx->sm_count, s)))
        return st;
    if (loss) {
        CR_CUDA(cudaMemcpyAsync(loss, ctx->d_loss, sizeof(double), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
    }
    return CR_OK;
}

CR_API cr_status cr_pick(cr_context *ctx, cr_frame *f, cr_cloud *cloud, const float ndc[2],
                         const cr_config *cfg, const cr_camera *cam, int search_radius,
                         uint32_t *index_out, int *found_out) {
    if (!ndc || !index_out || !found_out || !cloud)
        return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    *found_out = 0;
    cr_status st = validate_render(ctx, f, cfg, cam);
    if (st) return st;
    const int W = f->width, H = f->height;
    if (cloud->resident == 0) return CR_OK;
    DeviceGuard g(ctx->device);
    // NDC (y up) -> buffer pixel; the nearest pass stores row 0 at the top.
    const int px = std::min(std::max(trunc_i((ndc[0] * 0.5f + 0.5f) * (float)W), 0), W - 1);
    const int pyb = trunc_i((ndc[1] * 0.5f + 0.5f) * (float)H);
    const int py = std::min(std::max(H - 1 - pyb, 0), H - 1);
    if ((st = nearest_index_pass(ctx, f, cloud, cfg, cam))) return st;
    const int r = std::max(0, search_radius);
    const int row0 = std::max(0, py - r), row1 = std::min(H - 1, py + r);
    std::vector<uint32_t> band((size_t)(row1 - row0 + 1) * W);
    if ((st = read_nearest(f, nullptr, band.data(), row0, row1 - row0 + 1))) return st;
    long best_d = -1;
    uint32_t best = 0;
    const long r2 = (long)r * r;
    for (int y = row0; y <= row1; ++y) {
        const long dy = y - py;
        for (int x = std::max(0, px - r); x <= std::min(W - 1, px + r); ++x) {
            const long dx = x - px;
            const long d = dx * dx + dy * dy;
            if (d > r2 || (best_d >= 0 && d >= best_d)) continue;
            const uint32_t v = band[(size_t)(y - row0) * W + x];
            if (v != CR_INVALID_INDEX) {
                best_d = d;
                best = v;
            }
        }
    }
    if (best_d >= 0) {
        *index_out = best;
        *found_out = 1;
    }
    return CR_OK;
}

// ---------------------------------------------------------------- buffers
CR_API cr_status cr_buffer_create(cr_context *ctx, uint64_t bytes, void **out) {
    if (!ctx || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    DeviceGuard g(ctx->device);
    return dalloc(reinterpret_cast<uint8_t **>(out), bytes);
}

CR_API cr_status cr_buffer_destroy(cr_context *ctx, void *p) {
    if (!ctx) return fail(CR_ERR_INVALID_ARGUMENT, "ctx is null");
    if (!p) return CR_OK;
    DeviceGuard g(ctx->device);
    CR_CUDA(cudaStreamSynchronize(ctx->stream));
    CR_CUDA(cudaFree(p));
    return CR_OK;
}

CR_API cr_status cr_buffer_upload(cr_context *ctx, void *dst, const void *src, uint64_t bytes) {
    if (!ctx || (bytes && (!dst || !src))) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if (!bytes) return CR_OK;
    DeviceGuard g(ctx->device);
    CR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    CR_CUDA(cudaStreamSynchronize(ctx->stream));
    return CR_OK;
}

CR_API cr_status cr_buffer_download(cr_context *ctx, void *dst, const void *src, uint64_t bytes) {
    if (!ctx || (bytes && (!dst || !src))) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if (!bytes) return CR_OK;
    DeviceGuard g(ctx->device);
    CR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CR_CUDA(cudaStreamSynchronize(ctx->stream));
    return CR_OK;
}

CR_API cr_status cr_host_alloc(uint64_t bytes, void **out) {
    if (!out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    CR_CUDA(cudaMallocHost(out, bytes ? bytes : 16));
    return CR_OK;
}

CR_API cr_status cr_host_free(void *p) {
    if (p) CR_CUDA(cudaFreeHost(p));
    return CR_OK;
}

// ---------------------------------------------------------------- tuning
CR_API cr_status cr_context_get_tuning(cr_context *ctx, cr_tuning *out) {
    if (!ctx || !out) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    out->chunkPoints = ctx->chunk_points;
    out->useTiles = ctx->use_tiles ? 1 : 0;
    out->viewGroupPixels = ctx->view_group_pixels;
    out->cullSpinLimit = ctx->cull_spin_limit;
    return CR_OK;
}

CR_API cr_status cr_context_set_tuning(cr_context *ctx, const cr_tuning *t) {
    if (!ctx || !t) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if (t->chunkPoints < kMinChunkPoints || t->chunkPoints > 65536)
        return fail(CR_ERR_INVALID_ARGUMENT, "chunkPoints must be in [256, 65536]");
    if (t->viewGroupPixels < 0)
        return fail(CR_ERR_INVALID_ARGUMENT, "viewGroupPixels must be >= 0");
    if (t->cullSpinLimit < 0) return fail(CR_ERR_INVALID_ARGUMENT, "cullSpinLimit must be >= 0");
    ctx->chunk_points = t->chunkPoints;
    ctx->use_tiles = t->useTiles != 0;
    ctx->view_group_pixels = t->viewGroupPixels;
    ctx->cull_spin_limit = t->cullSpinLimit;
    return CR_OK;
}

// ---------------------------------------------------------------- profiling
CR_API cr_status cr_context_set_profiling(cr_context *ctx, int enable) {
    if (!ctx) return fail(CR_ERR_INVALID_ARGUMENT, "ctx is null");
    DeviceGuard g(ctx->device);
    if (enable && !ctx->pass_ev[0][0][0])
        for (auto &fr : ctx->pass_ev)
            for (auto &pe : fr)
                for (auto &e : pe) CR_CUDA(cudaEventCreate(&e));
    CR_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->profiling = enable != 0;
    ctx->prof_frame = -1;
    ctx->prof_count = 0;
    for (auto &fr : ctx->pass_recorded)
        for (bool &r : fr) r = false;
    return CR_OK;
}

CR_API cr_status cr_context_pass_times(cr_context *ctx, int32_t nframes, float *ms,
                                       int32_t *frames_out) {
    if (!ctx || !frames_out || (nframes > 0 && !ms))
        return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    DeviceGuard g(ctx->device);
    const int64_t avail = std::min<int64_t>(ctx->prof_count, cr_context::kProfRing);
    const int n = (int)std::min<int64_t>(std::max(nframes, 0), avail);
    *frames_out = n;
    for (int k = 0; k < n; ++k) {
        // k = 0 is the oldest of the last n frames.
        const int slot = (ctx->prof_frame - (n - 1 - k) + cr_context::kProfRing) % cr_context::kProfRing;
        for (int p = 0; p < CR_PASS_COUNT; ++p) {
            float &out = ms[(size_t)k * CR_PASS_COUNT + p];
            out = 0.0f;
            if (!ctx->pass_recorded[slot][p]) continue;
            CR_CUDA(cudaEventSynchronize(ctx->pass_ev[slot][p][1]));
            CR_CUDA(cudaEventElapsedTime(&out, ctx->pass_ev[slot][p][0], ctx->pass_ev[slot][p][1]));
        }
    }
    return CR_OK;
}

// ---------------------------------------------------------------- packer
CR_API cr_status cr_pack_params_default(cr_pack_params *out) {
    if (!out) return fail(CR_ERR_INVALID_ARGUMENT, "out is null");
    out->lodLevels = 4;             // PackedPointCloudFixtures.defaultLODLevels
    out->coarseVoxelDivisions = 64; // PackedPointCloudFixtures.defaultCoarseVoxelDivisions
    out->mortonBits = 10;
    return CR_OK;
}

static cr_status validate_pack(cr_context *ctx, cr_cloud *cloud, const cr_pack_params *prm) {
    if (!ctx || !cloud || !prm) return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if (cloud->ctx != ctx) return fail(CR_ERR_INVALID_ARGUMENT, "cloud belongs to another context");
    if (prm->mortonBits != 10 && prm->mortonBits != 21)
        return fail(CR_ERR_INVALID_ARGUMENT, "mortonBits must be 10 or 21");
    // GPUPacker.swift:215: uint16 cumulative LOD counts.
    if (cloud->cap.pointsPerBatch > 65535)
        return fail(CR_ERR_INVALID_ARGUMENT, "pointsPerBatch must fit the uint16 LOD prefix counts");
    return CR_OK;
}

static cr_status validate_input(const cr_pack_input *in) {
    if (!in || !in->positions || !in->colors) return fail(CR_ERR_INVALID_ARGUMENT, "null input");
    if (in->positionStrideBytes < 12 || (in->positionStrideBytes & 3))
        return fail(CR_ERR_INVALID_ARGUMENT, "positionStrideBytes must be >= 12 and a multiple of 4");
    if (in->colorFormat != CR_COLOR_F32X4 && in->colorFormat != CR_COLOR_RGBA8)
        return fail(CR_ERR_INVALID_ARGUMENT, "unknown colorFormat");
    const uint32_t cs = in->colorFormat == CR_COLOR_RGBA8 ? 4u : 16u;
    if (in->colorStrideBytes < cs || (in->colorStrideBytes & 3))
        return fail(CR_ERR_INVALID_ARGUMENT, "colorStrideBytes too small or unaligned");
    if (((uintptr_t)in->positions & 3) || ((uintptr_t)in->colors & 3))
        return fail(CR_ERR_INVALID_ARGUMENT, "input pointers must be 4-byte aligned");
    return CR_OK;
}

// Adopt GPU-written batches into the host mirror (adoptGPUBatchBounds /
// finalizeGPUChunk, ComputeRasteriserPointCloud.swift:313-363).
static cr_status adopt_batches(cr_cloud *c, uint32_t first, uint32_t n) {
    if (n == 0) return CR_OK;
    CR_CUDA(cudaMemcpyAsync(c->mirror.data() + first, c->d_batches + first,
                            (size_t)n * sizeof(cr_raster_batch), cudaMemcpyDeviceToHost,
                            c->ctx->stream));
    CR_CUDA(cudaStreamSynchronize(c->ctx->stream));
    return CR_OK;
}

CR_API cr_status cr_pack(cr_context *ctx, cr_cloud *c, const cr_pack_input *in, uint64_t count,
                         const cr_pack_params *prm, int on_device, uint32_t *src_idx) {
    cr_status st = validate_pack(ctx, c, prm);
    if (st) return st;
    DeviceGuard g(ctx->device);
    if ((st = uploads_drain(c))) return st;  // every slot is rewritten
    // GPUPacker.pack: an empty input clears the cloud (GPUPacker.swift:147-150).
    if (count == 0) return cr_cloud_clear(c);
    if ((st = validate_input(in))) return st;
    if (count >= 0xffffffffull) return fail(CR_ERR_CAPACITY, "count must be below 2^32-1");
    // prepareForGPUPack (ComputeRasteriserPointCloud.swift:278-307).
    const uint32_t ppb = c->cap.pointsPerBatch;
    const uint64_t nb64 = std::max<uint64_t>(1, (count + ppb - 1) / ppb);
    if (nb64 > c->cap.maxResidentBatches) {
        if ((uint64_t)nb64 * ppb >= 0xffffffffull)
            return fail(CR_ERR_CAPACITY, "pool would exceed 2^32-1 points");
        CR_CUDA(cudaStreamSynchronize(ctx->stream));
        std::vector<cr_raster_file> keep = c->files;
        if ((st = allocate_cloud(c, cr_capacity{(uint32_t)nb64, ppb}, keep.data(),
                                 (uint32_t)keep.size())))
            return st;
    }
    const uint32_t nb = (uint32_t)nb64;
    for (uint32_t slot = 0; slot < c->cap.maxResidentBatches; ++slot) {
        cr_raster_batch &b = c->mirror[slot];
        if (slot < nb) {
            b = cr_raster_batch{};
            b.state = 1;
            b.firstPoint = slot * ppb;
            b.numPoints = (uint32_t)std::min<uint64_t>(ppb, count - (uint64_t)slot * ppb);
        } else {
            b.state = 0;
            b.numPoints = 0;
        }
    }
    c->free_slots.clear();
    for (int64_t s2 = (int64_t)c->cap.maxResidentBatches - 1; s2 >= (int64_t)nb; --s2)
        c->free_slots.push_back((int32_t)s2);
    c->resident = nb;
    c->points = count;
    mark_dirty(c, 0, (int64_t)c->mirror.size() - 1);
    if ((st = flush_mirror(c))) return st;
    if ((st = pack_run(ctx, c, in, count, prm, on_device, 0, src_idx))) return st;
    return adopt_batches(c, 0, nb);
}

// reserveContiguousSlots (ComputeRasteriserPointCloud.swift:330-346): first-fit run of
// empty slots; the slots leave the free list and are marked resident provisionally.
static int64_t reserve_contiguous(cr_cloud *c, uint32_t n) {
    const uint32_t cap = c->cap.maxResidentBatches;
    if (n == 0 || n > cap) return -1;
    uint32_t s = 0;
    while ((uint64_t)s + n <= cap) {
        uint32_t k = 0;
        while (k < n && c->mirror[s + k].state == 0 && !upload_slot_busy(c, s + k)) ++k;
        if (k == n) {
            std::vector<int32_t> keep;
            keep.reserve(c->free_slots.size());
            for (int32_t f : c->free_slots)
                if (!((uint32_t)f >= s && (uint32_t)f < s + n)) keep.push_back(f);
            c->free_slots.swap(keep);
            for (uint32_t q = s; q < s + n; ++q) c->mirror[q].state = 1;
            mark_dirty(c, s, (int64_t)s + n - 1);
            return s;
        }
        s += k + 1;
    }
    return -1;
}

CR_API cr_status cr_pack_chunks(cr_context *ctx, cr_cloud *c, const cr_pack_input *chunks,
                                const uint64_t *counts, uint32_t nchunks,
                                const cr_pack_params *prm, int on_device, int32_t *first_slots,
                                uint32_t *placed_out) {
    cr_status st = validate_pack(ctx, c, prm);
    if (st) return st;
    if (!placed_out || (nchunks && (!chunks || !counts)))
        return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    *placed_out = 0;
    const uint32_t ppb = c->cap.pointsPerBatch;
    for (uint32_t i = 0; i < nchunks; ++i) {
        if (counts[i] == 0) continue;
        if ((st = validate_input(&chunks[i]))) return st;
        if (counts[i] >= 0xffffffffull) return fail(CR_ERR_CAPACITY, "chunk count too large");
    }
    DeviceGuard g(ctx->device);
    struct Placed {
        uint32_t first, nb, index;
    };
    std::vector<Placed> placed;
    for (uint32_t i = 0; i < nchunks; ++i) {
        if (counts[i] == 0) continue;
        const uint64_t nb = std::max<uint64_t>(1, (counts[i] + ppb - 1) / ppb);
        const int64_t first = reserve_contiguous(c, (uint32_t)std::min<uint64_t>(nb, UINT32_MAX));
        if (first < 0) continue;
        placed.push_back(Placed{(uint32_t)first, (uint32_t)nb, i});
    }
    for (const Placed &p : placed)
        if ((st = pack_run(ctx, c, &chunks[p.index], counts[p.index], prm, on_device, p.first,
                           nullptr)))
            return st;
    for (size_t k = 0; k < placed.size(); ++k) {
        const Placed &p = placed[k];
        if ((st = adopt_batches(c, p.first, p.nb))) return st;
        c->resident += p.nb;
        c->points += counts[p.index];
        if (first_slots) first_slots[k] = (int32_t)p.first;
    }
    *placed_out = (uint32_t)placed.size();
    return flush_mirror(c);
}

}  // extern "C"
