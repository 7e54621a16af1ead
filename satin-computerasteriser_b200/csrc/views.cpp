// views.cpp — batched rendering of many views of the same clouds, and the
// autotuner of its launch shape.
//
// The reference draws one viewport per ComputeRasteriser.encode
// (ComputeRasteriser.swift:277-296, 322-456).  cr_render_multiview draws
// up to kMaxViews views, each into its own cr_frame, with the same passes in
// a few launches shared by all views:
//   clear_views           every view's depth plane and accumulators
//   cull_*_views          per cloud: blockIdx.y = view, ordered survivor and
//                         chunk lists per view (fixed strides)
//   raster_kernel<*, MV>  per cloud and pass: one persistent grid over the
//                         chunks of all views, each chunk drawn into its view
//   resolve_views         every view's pixels (+ the exact re-run gate)
//   hole_fill_views       per iteration
// The sequence is captured once into a CUDA graph and replayed: the views'
// cameras, cull arguments and file tables travel in one pinned staging block
// copied by the graph's first node.  Two staging blocks and two graph
// executables alternate, so the host fills one while the other may still be
// copied.  Every view uses the per-view path's arithmetic (the same file
// table products, cull, passes and integer atomics), so its images are
// bit-identical to a cr_render of that view alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "cr_internal.h"

using cri::fail;

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

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

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Per-cloud cull scratch and outputs for all views.
struct ViewsCloud {
    CullRec *tmp = nullptr;               // nviews * nslots
    uint32_t *cta = nullptr;              // nviews * 2 * ctas
    cr_visible_batch *visible = nullptr;  // nviews * nslots
    ChunkRec *chunks = nullptr;           // nviews * chunk_stride
    uint32_t *counters = nullptr;         // nviews * CNT_COUNT
    uint32_t nslots = 0, ctas = 0, nfiles = 0;
    uint64_t chunk_stride = 0;
    size_t args_off = 0, files_off = 0;  // in the staging block
};

}  // namespace

// Cached state of the last batched render of a context.
struct ViewsState {
    std::vector<unsigned char> key;
    uint32_t nviews = 0, total_pix = 0;
    bool packed = false;
    int hole_fill = 0;
    std::vector<ViewsCloud> clouds;
    unsigned char *d_stage = nullptr;  // ViewDesc[nviews] | per cloud: CullArgs[nviews], files
    unsigned char *h_stage[2] = {nullptr, nullptr};
    size_t stage_bytes = 0;
    uint32_t *d_redo = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    bool launched[2] = {false, false};
    int next = 0;
};

namespace {

void views_free(ViewsState *s) {
    if (!s) return;
    for (int i = 0; i < 2; ++i) {
        if (s->done[i] && s->launched[i]) cudaEventSynchronize(s->done[i]);
        if (s->exec[i]) cudaGraphExecDestroy(s->exec[i]);
        if (s->done[i]) cudaEventDestroy(s->done[i]);
        if (s->h_stage[i]) cudaFreeHost(s->h_stage[i]);
        s->exec[i] = nullptr;
        s->done[i] = nullptr;
        s->h_stage[i] = nullptr;
        s->launched[i] = false;
    }
    for (ViewsCloud &c : s->clouds) {
        dfree(c.tmp);
        dfree(c.cta);
        dfree(c.visible);
        dfree(c.chunks);
        dfree(c.counters);
    }
    s->clouds.clear();
    dfree(s->d_stage);
    dfree(s->d_redo);
    s->key.clear();
}

// a * b for column-major 4x4 matrices in the library's fixed operation order
// (the same products cr_cloud_update_files forms).
void mat4mul(const float *a, const float *b, float *out) {
    float r[16];
    for (int c = 0; c < 4; ++c)
        for (int row = 0; row < 4; ++row)
            r[c * 4 + row] = ((a[0 * 4 + row] * b[c * 4 + 0] + a[1 * 4 + row] * b[c * 4 + 1]) +
                              a[2 * 4 + row] * b[c * 4 + 2]) +
                             a[3 * 4 + row] * b[c * 4 + 3];
    std::memcpy(out, r, sizeof(r));
}

template <typename T>
void put(std::vector<unsigned char> &k, const T &v) {
    const unsigned char *p = reinterpret_cast<const unsigned char *>(&v);
    k.insert(k.end(), p, p + sizeof(T));
}

// Everything a captured graph bakes in: frames, cloud pools, configuration,
// tuning and the packed-add choice.
std::vector<unsigned char> make_key(cr_context *ctx, cr_frame *const *frames, uint32_t nviews,
                                    cr_cloud *const *clouds, uint32_t nclouds,
                                    const cr_config *cfg, bool packed) {
    std::vector<unsigned char> k;
    put(k, nviews);
    for (uint32_t v = 0; v < nviews; ++v) {
        const cr_frame *f = frames[v];
        put(k, f->width);
        put(k, f->height);
        put(k, f->d_depth);
        put(k, f->d_accum);
        put(k, f->d_rgba[0]);
        put(k, f->d_rgba[1]);
        put(k, f->d_depthf);
    }
    put(k, nclouds);
    for (uint32_t i = 0; i < nclouds; ++i) {
        const cr_cloud *c = clouds[i];
        put(k, c->cap);
        put(k, c->d_low);
        put(k, c->d_med);
        put(k, c->d_high);
        put(k, c->d_colors);
        put(k, c->d_levels);
        put(k, c->d_batches);
        put(k, (uint32_t)c->files.size());
    }
    put(k, *cfg);  // every field is 4 bytes: no padding
    put(k, ctx->chunk_points);
    put(k, ctx->use_tiles);
    put(k, packed);
    return k;
}

CullUniforms cull_uniforms(const cr_config *cfg, const cr_camera *cam, int w, int h) {
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

// The configuration part of the point passes' uniforms (sizes and cameras
// come per view from the view descriptors).
RasterUniforms raster_uniforms(const cr_config *cfg) {
    RasterUniforms u;
    std::memset(&u, 0, sizeof(u));
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

// Allocates the per-view buffers for this frame set and cloud set.
cr_status views_alloc(cr_context *ctx, ViewsState *s, cr_frame *const *frames, uint32_t nviews,
                      cr_cloud *const *clouds, uint32_t nclouds) {
    s->nviews = nviews;
    uint64_t pix = 0;
    for (uint32_t v = 0; v < nviews; ++v) pix += (uint64_t)frames[v]->width * frames[v]->height;
    if (pix >= (1ull << 31)) return fail(CR_ERR_CAPACITY, "views exceed 2^31 pixels in all");
    s->total_pix = (uint32_t)pix;
    size_t off = align256(sizeof(ViewDesc) * nviews);
    s->clouds.resize(nclouds);
    const uint32_t cp = (uint32_t)std::max(ctx->chunk_points, kMinChunkPoints);
    cr_status st;
    for (uint32_t i = 0; i < nclouds; ++i) {
        ViewsCloud &vc = s->clouds[i];
        const cr_cloud *c = clouds[i];
        vc.nslots = c->cap.maxResidentBatches;
        vc.ctas = (vc.nslots + 255) / 256;
        vc.nfiles = (uint32_t)c->files.size();
        vc.chunk_stride = chunk_capacity(c->cap, (int)cp);
        const size_t n = (size_t)nviews * std::max(vc.nslots, 1u);
        if ((st = dalloc(&vc.tmp, n * sizeof(CullRec))) ||
            (st = dalloc(&vc.cta, (size_t)nviews * 2 * std::max(vc.ctas, 1u) * 4)) ||
            (st = dalloc(&vc.visible, n * sizeof(cr_visible_batch))) ||
            (st = dalloc(&vc.chunks, (size_t)nviews * vc.chunk_stride * sizeof(ChunkRec))) ||
            (st = dalloc(&vc.counters, (size_t)nviews * CNT_COUNT * 4)))
            return st;
        CR_CUDA(cudaMemsetAsync(vc.counters, 0, (size_t)nviews * CNT_COUNT * 4, ctx->stream));
        vc.args_off = off;
        off = align256(off + sizeof(CullArgs) * nviews);
        vc.files_off = off;
        off = align256(off + sizeof(cr_raster_file) * (size_t)nviews * std::max(vc.nfiles, 1u));
    }
    s->stage_bytes = off;
    if ((st = dalloc(&s->d_stage, off)) || (st = dalloc(&s->d_redo, 16))) return st;
    for (int b = 0; b < 2; ++b) {
        CR_CUDA(cudaMallocHost((void **)&s->h_stage[b], off));
        std::memset(s->h_stage[b], 0, off);
        CR_CUDA(cudaEventCreateWithFlags(&s->done[b], cudaEventDisableTiming));
    }
    return CR_OK;
}

// Enqueues one batched render reading staging block `b` (captured into a graph).
cr_status views_enqueue(cr_context *ctx, ViewsState *s, int b, cr_cloud *const *clouds,
                        uint32_t nclouds, const cr_config *cfg) {
    cudaStream_t st = ctx->stream;
    const ViewDesc *views = reinterpret_cast<const ViewDesc *>(s->d_stage);
    cr_status e;
    CR_CUDA(cudaMemcpyAsync(s->d_stage, s->h_stage[b], s->stage_bytes, cudaMemcpyHostToDevice, st));
    if ((e = launch_clear_views(views, s->nviews, s->total_pix, s->d_redo, ctx->sm_count, st)))
        return e;
    for (uint32_t i = 0; i < nclouds; ++i) {
        const ViewsCloud &vc = s->clouds[i];
        if (vc.nslots == 0) continue;
        const CullArgs *args = reinterpret_cast<const CullArgs *>(s->d_stage + vc.args_off);
        if ((e = launch_cull_views(args, vc.nslots, s->nviews, st))) return e;
    }
    const RasterUniforms u = raster_uniforms(cfg);
    RasterTargets t{nullptr, nullptr, nullptr};
    t.packed = s->packed ? 1 : 0;
    auto pass = [&](RasterPass p, const RasterTargets &tt) -> cr_status {
        for (uint32_t i = 0; i < nclouds; ++i) {
            const ViewsCloud &vc = s->clouds[i];
            if (vc.nslots == 0) continue;
            const cr_raster_file *files =
                reinterpret_cast<const cr_raster_file *>(s->d_stage + vc.files_off);
            cr_status r = launch_raster_views(clouds[i], p, u, tt, views, s->nviews, files,
                                              vc.nfiles, vc.chunks, (uint32_t)vc.chunk_stride,
                                              vc.counters, st);
            if (r) return r;
        }
        return CR_OK;
    };
    if ((e = pass(PASS_DEPTH, t)) || (e = pass(PASS_COLOR, t))) return e;
    ResolveUniforms ru{0, 0, {cfg->backgroundColor[0], cfg->backgroundColor[1],
                              cfg->backgroundColor[2], cfg->backgroundColor[3]}};
    if ((e = launch_resolve_views(views, s->nviews, s->total_pix, ru, s->d_redo, s->packed,
                                  nullptr, ctx->sm_count, st)))
        return e;
    if (s->packed) {
        // Exact re-run, gated on the resolve's flag (as cr_render).
        RasterTargets tx = t;
        tx.packed = 0;
        tx.redo = s->d_redo;
        if ((e = launch_accum_redo_clear_views(views, s->nviews, s->total_pix, s->d_redo,
                                               ctx->sm_count, st)) ||
            (e = pass(PASS_COLOR, tx)) ||
            (e = launch_resolve_views(views, s->nviews, s->total_pix, ru, s->d_redo, false,
                                      s->d_redo, ctx->sm_count, st)))
            return e;
    }
    for (int it = 0; it < s->hole_fill; ++it)
        if ((e = launch_hole_fill_views(views, s->nviews, s->total_pix, it & 1, ctx->sm_count,
                                        st)))
            return e;
    return CR_OK;
}

cr_status views_build_graphs(cr_context *ctx, ViewsState *s, cr_cloud *const *clouds,
                             uint32_t nclouds, const cr_config *cfg) {
    // Occupancy queries and kernel attributes first: only stream work while capturing.
    raster_prepare_views(ctx);
    for (int b = 0; b < 2; ++b) {
        cudaGraph_t g = nullptr;
        CR_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        cr_status e = views_enqueue(ctx, s, b, clouds, nclouds, cfg);
        cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
        if (e) {
            if (g) cudaGraphDestroy(g);
            return e;
        }
        if (ce != cudaSuccess) return cri::cuda_fail(ce, "cudaStreamEndCapture");
        ce = cudaGraphInstantiate(&s->exec[b], g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return cri::cuda_fail(ce, "cudaGraphInstantiate");
    }
    return CR_OK;
}

// Fills staging block b: view descriptors, per-cloud per-view cull arguments
// and file tables (the products cr_cloud_update_files forms for one view).
void views_fill(ViewsState *s, int b, cr_frame *const *frames, const cr_camera *cams,
                cr_cloud *const *clouds, const float *models, uint32_t nclouds,
                const cr_config *cfg, uint32_t chunk_points) {
    unsigned char *h = s->h_stage[b];
    ViewDesc *vd = reinterpret_cast<ViewDesc *>(h);
    uint32_t pix = 0;
    for (uint32_t v = 0; v < s->nviews; ++v) {
        const cr_frame *f = frames[v];
        ViewDesc &d = vd[v];
        d.depth = f->d_depth;
        d.accum = f->d_accum;
        d.nearest = f->d_nearest;
        d.rgba[0] = f->d_rgba[0];
        d.rgba[1] = f->d_rgba[1];
        d.depthf = f->d_depthf;
        d.width = f->width;
        d.height = f->height;
        d.pix_begin = pix;
        d.pad = 0;
        std::memcpy(d.view, cams[v].view, sizeof(d.view));
        std::memcpy(d.proj, cams[v].projection, sizeof(d.proj));
        pix += (uint32_t)(f->width * f->height);
    }
    for (uint32_t i = 0; i < nclouds; ++i) {
        const ViewsCloud &vc = s->clouds[i];
        const cr_cloud *c = clouds[i];
        const float *model = models + 16 * i;
        CullArgs *args = reinterpret_cast<CullArgs *>(h + vc.args_off);
        cr_raster_file *files = reinterpret_cast<cr_raster_file *>(h + vc.files_off);
        const cr_raster_file *d_files =
            reinterpret_cast<const cr_raster_file *>(s->d_stage + vc.files_off);
        for (uint32_t v = 0; v < s->nviews; ++v) {
            float vp[16];
            mat4mul(cams[v].projection, cams[v].view, vp);
            for (uint32_t fi = 0; fi < vc.nfiles; ++fi) {
                cr_raster_file &o = files[(size_t)v * vc.nfiles + fi];
                float world[16];
                mat4mul(model, c->files[fi].world, world);
                mat4mul(vp, world, o.transform);
                mat4mul(vp, world, o.transformFrustum);
                std::memcpy(o.world, world, sizeof(world));
                mat4mul(vp, world, o.prevTransform);
            }
            CullArgs &a = args[v];
            a.batches = c->d_batches;
            a.nbatches = vc.nslots;
            a.files = d_files + (size_t)v * vc.nfiles;
            a.nfiles = vc.nfiles;
            a.tmp = vc.tmp + (size_t)v * vc.nslots;
            a.cta_counts = vc.cta + (size_t)v * 2 * vc.ctas;
            a.chunk_points = chunk_points;
            a.u = cull_uniforms(cfg, &cams[v], frames[v]->width, frames[v]->height);
            a.visible = vc.visible + (size_t)v * vc.nslots;
            a.chunks = vc.chunks + (size_t)v * vc.chunk_stride;
            a.counters = vc.counters + (size_t)v * CNT_COUNT;
        }
    }
}

}  // namespace

void views_destroy(ViewsState *s) {
    views_free(s);
    delete s;
}

extern "C" {

CR_API cr_status cr_render_multiview(cr_context *ctx, cr_frame *const *frames,
                                     const cr_camera *cams, uint32_t nviews,
                                     cr_cloud *const *clouds, const float *models,
                                     uint32_t nclouds, const cr_config *cfg) {
    if (!ctx || !frames || !cams || !cfg || (nclouds && !clouds))
        return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if (nviews == 0 || nviews > kMaxViews)
        return fail(CR_ERR_INVALID_ARGUMENT, "nviews must be in [1, 256]");
    cr_status vst = validate_config(cfg);
    if (vst) return vst;
    if (cfg->mode != CR_MODE_HIGH_QUALITY_AVERAGE)
        return fail(CR_ERR_UNSUPPORTED, "batched views render the HQS mode only");
    if (cfg->holeFillIterations > 64)
        return fail(CR_ERR_INVALID_ARGUMENT, "batched views: holeFillIterations must be at most 64");
    for (uint32_t v = 0; v < nviews; ++v) {
        if (!frames[v] || frames[v]->ctx != ctx)
            return fail(CR_ERR_INVALID_ARGUMENT, "frame is null or from another context");
        for (uint32_t w = 0; w < v; ++w)
            if (frames[w] == frames[v])
                return fail(CR_ERR_INVALID_ARGUMENT, "a frame appears twice in the view list");
    }
    for (uint32_t i = 0; i < nclouds; ++i)
        if (!clouds[i] || clouds[i]->ctx != ctx)
            return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null or from another context");
    DeviceGuard g(ctx->device);
    // Non-resident clouds draw nothing; the rest are drawn in the given order.
    std::vector<cr_cloud *> resident;
    std::vector<float> rmodels;
    uint64_t max_samples = 0;
    for (uint32_t i = 0; i < nclouds; ++i) {
        if (clouds[i]->resident == 0) continue;
        resident.push_back(clouds[i]);
        max_samples += (uint64_t)clouds[i]->resident * clouds[i]->cap.pointsPerBatch;
        for (int j = 0; j < 16; ++j)
            rmodels.push_back(models ? models[16 * i + j] : (j % 5 == 0 ? 1.0f : 0.0f));
    }
    // Packed colour adds under the same bound as cr_render (per view).
    const bool packed = max_samples < (1ull << 31);
    const uint32_t nres = (uint32_t)resident.size();
    std::vector<unsigned char> key =
        make_key(ctx, frames, nviews, resident.data(), nres, cfg, packed);
    ViewsState *s = ctx->views;
    if (!s || s->key != key) {
        if (s) {
            CR_CUDA(cudaStreamSynchronize(ctx->stream));
            views_free(s);
        } else {
            s = ctx->views = new ViewsState();
        }
        cr_status st = views_alloc(ctx, s, frames, nviews, resident.data(), nres);
        if (!st) {
            s->packed = packed;
            s->hole_fill = std::max(cfg->holeFillIterations, 0);
            st = views_build_graphs(ctx, s, resident.data(), nres, cfg);
        }
        if (st) {
            views_free(s);
            return st;
        }
        s->key = key;
        s->next = 0;
    }
    const int b = s->next;
    if (s->launched[b]) CR_CUDA(cudaEventSynchronize(s->done[b]));
    views_fill(s, b, frames, cams, resident.data(), rmodels.data(), nres, cfg,
               (uint32_t)std::max(ctx->chunk_points, kMinChunkPoints));
    CR_CUDA(cudaGraphLaunch(s->exec[b], ctx->stream));
    CR_CUDA(cudaEventRecord(s->done[b], ctx->stream));
    s->launched[b] = true;
    s->next = b ^ 1;
    for (uint32_t v = 0; v < nviews; ++v) {
        frames[v]->final_rgba = s->hole_fill & 1;
        frames[v]->last_mode = 0;
    }
    return CR_OK;
}

CR_API cr_status cr_autotune_multiview(cr_context *ctx, cr_frame *const *frames,
                                       const cr_camera *cams, uint32_t nviews,
                                       cr_cloud *const *clouds, const float *models,
                                       uint32_t nclouds, const cr_config *cfg,
                                       const char *cache_path, int reps, cr_tuning *best_out,
                                       float *best_ms_out) {
    if (!ctx || !frames || !cams || !cfg || (nclouds && !clouds))
        return fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if (reps < 1 || reps > 1000) return fail(CR_ERR_INVALID_ARGUMENT, "reps must be in [1, 1000]");
    if (nviews == 0 || nviews > kMaxViews)
        return fail(CR_ERR_INVALID_ARGUMENT, "nviews must be in [1, 256]");
    for (uint32_t v = 0; v < nviews; ++v)
        if (!frames[v]) return fail(CR_ERR_INVALID_ARGUMENT, "frame is null");
    for (uint32_t i = 0; i < nclouds; ++i)
        if (!clouds[i]) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    DeviceGuard g(ctx->device);
    cudaDeviceProp prop;
    CR_CUDA(cudaGetDeviceProperties(&prop, ctx->device));
    uint64_t pix = 0, pts = 0;
    for (uint32_t v = 0; v < nviews; ++v) pix += (uint64_t)frames[v]->width * frames[v]->height;
    for (uint32_t i = 0; i < nclouds; ++i) pts += clouds[i]->points;
    // Workload signature: device, views, pixels, points and the options
    // that change the passes' work.
    std::ostringstream sig;
    sig << prop.name << "/sm" << prop.multiProcessorCount << "/views" << nviews << "/pix" << pix
        << "/pts" << pts << "/clouds" << nclouds << "/tol" << cfg->depthTolerance << "/clod"
        << cfg->enableCLOD << "/bias" << cfg->lodBias << "/dither" << cfg->enableLODDither
        << "/ps" << cfg->minimumPointSize << "-" << cfg->maximumPointSize << "/hf"
        << cfg->holeFillIterations;
    const std::string tag = "\"signature\": \"" + sig.str() + "\"";
    if (cache_path) {
        std::ifstream in(cache_path);
        std::string line;
        while (std::getline(in, line)) {
            if (line.find(tag) == std::string::npos) continue;
            const size_t a = line.find("\"chunkPoints\": "), t = line.find("\"useTiles\": "),
                         m = line.find("\"ms\": ");
            if (a == std::string::npos || t == std::string::npos) continue;
            const int cpn = std::atoi(line.c_str() + a + 15);
            const int tiles = std::atoi(line.c_str() + t + 12);
            if (cpn < kMinChunkPoints || cpn > 65536 || (tiles != 0 && tiles != 1)) continue;
            ctx->chunk_points = cpn;
            ctx->use_tiles = tiles != 0;
            if (best_out) *best_out = cr_tuning{cpn, tiles};
            if (best_ms_out)
                *best_ms_out = m == std::string::npos ? 0.0f : (float)std::atof(line.c_str() + m + 6);
            return CR_OK;
        }
    }
    const int candidates[][2] = {{512, 1}, {1024, 1}, {2048, 1}, {4096, 1},
                                 {512, 0}, {1024, 0}, {2048, 0}, {4096, 0}};
    cudaEvent_t e0, e1;
    CR_CUDA(cudaEventCreate(&e0));
    CR_CUDA(cudaEventCreate(&e1));
    std::ostringstream results;
    float best_ms = 0.0f;
    int best = -1;
    cr_status st = CR_OK;
    for (int ci = 0; ci < 8 && !st; ++ci) {
        ctx->chunk_points = candidates[ci][0];
        ctx->use_tiles = candidates[ci][1] != 0;
        for (int w = 0; w < 2 && !st; ++w)
            st = cr_render_multiview(ctx, frames, cams, nviews, clouds, models, nclouds, cfg);
        if (st) break;
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < reps && !st; ++r)
            st = cr_render_multiview(ctx, frames, cams, nviews, clouds, models, nclouds, cfg);
        cudaEventRecord(e1, ctx->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = fail(CR_ERR_CUDA, "autotune timing");
        if (st) break;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= (float)reps;
        results << (ci ? ", " : "") << "{\"chunkPoints\": " << candidates[ci][0]
                << ", \"useTiles\": " << candidates[ci][1] << ", \"ms\": " << ms << "}";
        if (best < 0 || ms < best_ms) {
            best = ci;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    ctx->chunk_points = candidates[best][0];
    ctx->use_tiles = candidates[best][1] != 0;
    if (best_out) *best_out = cr_tuning{candidates[best][0], candidates[best][1]};
    if (best_ms_out) *best_ms_out = best_ms;
    if (cache_path) {
        std::ofstream out(cache_path, std::ios::app);
        if (!out) return fail(CR_ERR_INVALID_ARGUMENT, "cannot write the autotune cache file");
        out << "{" << tag << ", \"chunkPoints\": " << candidates[best][0]
            << ", \"useTiles\": " << candidates[best][1] << ", \"ms\": " << best_ms
            << ", \"candidates\": [" << results.str() << "]}\n";
    }
    return CR_OK;
}

}  // extern "C"
