// views.cpp — batched rendering of many views of the same clouds, and the
// autotuner of its launch shape.
//
// The reference draws one viewport per ComputeRasteriser.encode
// (ComputeRasteriser.swift:277-296, 322-456).  cr_render_multiview draws
// up to kMaxViews views, each into its own cr_frame, with the same passes in
// launches shared by many views:
//   cull_*_views          per cloud, all views: blockIdx.y = view, ordered
//                         survivor and chunk lists per view (fixed strides)
//   then per group of consecutive views (ctx->view_group_pixels pixels):
//   clear_views           the group's depth planes and accumulators
//   raster_kernel<*, MV>  per cloud, depth then colour: one persistent grid
//                         over the chunks of the group's views
//   resolve_views         the group's pixels (+ the exact re-run's check)
//   hole_fill_views       all views, per iteration
// A group's planes and fragments stay in L2 from its clear to its resolve,
// as they do for one view at a time.  The sequence is captured once into a
// CUDA graph and replayed: the views' cameras, cull arguments and file
// tables travel in one pinned staging block copied by the graph's first
// node.  Two staging blocks and two graph executables alternate, so the
// host fills one while the other may still be copied.  Every view uses the
// per-view path's arithmetic (the same file table products, cull, passes
// and integer atomics), so its images are bit-identical to a cr_render of
// that view alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "cr_internal.h"

using cri::fail;

namespace {


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
    uint32_t *cta = nullptr;              // nviews * kCullCtaWords * ctas
    cr_visible_batch *visible = nullptr;  // nviews * nslots
    ChunkRec *chunks = nullptr;           // nviews * chunk_stride
    uint32_t *counters = nullptr;         // nviews * CNT_COUNT
    uint32_t *chunk_poff = nullptr;       // nviews * chunk_stride
    uint32_t *frag_count = nullptr;       // nviews * chunk_stride
    uint32_t *frag_xy = nullptr;  // frag_cap each
    uint2 *frag_zc = nullptr;
    uint32_t *frag_overflow = nullptr;
    unsigned long long frag_cap = 0;
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
    bool frags = false;  // fragment passes (single-pixel footprints)
    int hole_fill = 0;
    struct Group {
        uint32_t v0, nv;      // views [v0, v0 + nv)
        uint32_t pix0, npix;  // their pixels
    };
    std::vector<Group> groups;
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
        dfree(c.chunk_poff);
        dfree(c.frag_count);
        dfree(c.frag_xy);
        dfree(c.frag_zc);
        dfree(c.frag_overflow);
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
    put(k, ctx->view_group_pixels);
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

// Fragment span of a full batch (its chunks rounded up to multiples of 4).
uint64_t batch_fragment_span(uint32_t ppb, uint32_t cp) {
    const uint64_t nc = (ppb + cp - 1) / cp;
    return nc == 0 ? 0 : (nc - 1) * ((cp + 3) & ~3u) + ((ppb - (nc - 1) * cp + 3) & ~3ull);
}

// Allocates the per-view buffers for this frame set and cloud set.  The
// depth and colour passes run over groups of consecutive views of at most
// ctx->view_group_pixels pixels (0: one group), so that a group's fragments
// are still in L2 when its colour pass reads them.  With single-pixel
// footprints each cloud gets one fragment arena reused by every group: the
// largest group's worst case (every slot's full batch surviving in each of
// its views), within an eighth of the free device memory shared by the
// clouds; a group whose spans exceed it draws its colour pass from the
// points instead.
cr_status views_alloc(cr_context *ctx, ViewsState *s, cr_frame *const *frames, uint32_t nviews,
                      cr_cloud *const *clouds, uint32_t nclouds, bool frags) {
    s->nviews = nviews;
    uint64_t pix = 0;
    for (uint32_t v = 0; v < nviews; ++v) pix += (uint64_t)frames[v]->width * frames[v]->height;
    if (pix >= (1ull << 31)) return fail(CR_ERR_CAPACITY, "views exceed 2^31 pixels in all");
    s->total_pix = (uint32_t)pix;
    s->groups.clear();
    uint32_t largest = 0;
    {
        const uint64_t budget = ctx->view_group_pixels > 0 ? (uint64_t)ctx->view_group_pixels : pix;
        uint32_t first = 0, pix0 = 0;
        uint64_t acc = 0;
        for (uint32_t v = 0; v < nviews; ++v) {
            const uint64_t p = (uint64_t)frames[v]->width * frames[v]->height;
            if (v > first && acc + p > budget) {
                s->groups.push_back({first, v - first, pix0, (uint32_t)acc});
                largest = std::max(largest, v - first);
                first = v;
                pix0 += (uint32_t)acc;
                acc = 0;
            }
            acc += p;
        }
        s->groups.push_back({first, nviews - first, pix0, (uint32_t)acc});
        largest = std::max(largest, nviews - first);
    }
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
            (st = dalloc(&vc.cta, (size_t)nviews * kCullCtaWords * std::max(vc.ctas, 1u) * 4)) ||
            (st = dalloc(&vc.visible, n * sizeof(cr_visible_batch))) ||
            (st = dalloc(&vc.chunks, (size_t)nviews * vc.chunk_stride * sizeof(ChunkRec))) ||
            (st = dalloc(&vc.counters, (size_t)nviews * CNT_COUNT * 4)))
            return st;
        CR_CUDA(cudaMemsetAsync(vc.counters, 0, (size_t)nviews * CNT_COUNT * 4, ctx->stream));
        if (frags) {
            size_t free_b = 0, total_b = 0;
            CR_CUDA(cudaMemGetInfo(&free_b, &total_b));
            const unsigned long long need =
                (unsigned long long)largest * vc.nslots * batch_fragment_span(c->cap.pointsPerBatch, cp);
            const unsigned long long budget = free_b / 8 / std::max(nclouds, 1u) / 12;
            vc.frag_cap = std::min<unsigned long long>({need, budget, 0xfffffff0ull});
            const size_t slots = (size_t)nviews * vc.chunk_stride;
            if ((st = dalloc(&vc.chunk_poff, slots * 4)) || (st = dalloc(&vc.frag_count, slots * 4)) ||
                (st = dalloc(&vc.frag_xy, vc.frag_cap * 4)) ||
                (st = dalloc(&vc.frag_zc, vc.frag_cap * 8)) ||
                (st = dalloc(&vc.frag_overflow, 16)))
                return st;
            CR_CUDA(cudaMemsetAsync(vc.frag_overflow, 0, 16, ctx->stream));
        }
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
    for (uint32_t i = 0; i < nclouds; ++i) {
        const ViewsCloud &vc = s->clouds[i];
        if (vc.nslots == 0) continue;
        const CullArgs *args = reinterpret_cast<const CullArgs *>(s->d_stage + vc.args_off);
        if ((e = launch_cull_views(args, vc.nslots, s->nviews, st))) return e;
    }
    const RasterUniforms u = raster_uniforms(cfg);
    RasterTargets t{nullptr, nullptr, nullptr};
    t.packed = s->packed ? 1 : 0;
    // Pass p of every cloud over views [v0, v0 + nv).
    auto pass = [&](RasterPass p, const RasterTargets &tt, uint32_t v0, uint32_t nv) -> cr_status {
        for (uint32_t i = 0; i < nclouds; ++i) {
            const ViewsCloud &vc = s->clouds[i];
            if (vc.nslots == 0) continue;
            const cr_raster_file *files =
                reinterpret_cast<const cr_raster_file *>(s->d_stage + vc.files_off) +
                (size_t)v0 * vc.nfiles;
            const size_t slot0 = (size_t)v0 * vc.chunk_stride;
            const ViewsFragments fr{vc.frag_xy,
                                    vc.frag_zc,
                                    vc.frag_count ? vc.frag_count + slot0 : nullptr,
                                    vc.chunk_poff ? vc.chunk_poff + slot0 : nullptr,
                                    vc.frag_cap,
                                    vc.frag_overflow};
            const bool fp = p == PASS_DEPTH_FRAG || p == PASS_COLOR_FRAG;
            cr_status r = launch_raster_views(clouds[i], p, u, tt, views + v0, nv, files,
                                              vc.nfiles, vc.chunks + slot0,
                                              (uint32_t)vc.chunk_stride,
                                              vc.counters + (size_t)v0 * CNT_COUNT,
                                              fp ? &fr : nullptr, st);
            if (r) return r;
        }
        return CR_OK;
    };
    ResolveUniforms ru{0, 0, {cfg->backgroundColor[0], cfg->backgroundColor[1],
                              cfg->backgroundColor[2], cfg->backgroundColor[3]}};
    // Group after group: clear, depth, colour, resolve, so that the group's
    // planes (and, with single-pixel footprints, the fragments the depth
    // pass keeps for the colour pass, through one arena) stay in L2.
    const RasterPass depth_pass = s->frags ? PASS_DEPTH_FRAG : PASS_DEPTH;
    const RasterPass color_pass = s->frags ? PASS_COLOR_FRAG : PASS_COLOR;
    for (size_t gi = 0; gi < s->groups.size(); ++gi) {
        const ViewsState::Group &g = s->groups[gi];
        if ((e = launch_clear_views(views + g.v0, g.nv, g.pix0, g.npix, s->d_redo, gi == 0,
                                    ctx->sm_count, st)) ||
            (e = pass(depth_pass, t, g.v0, g.nv)) || (e = pass(color_pass, t, g.v0, g.nv)) ||
            (e = launch_resolve_views(views + g.v0, g.nv, g.pix0, g.npix, ru, s->d_redo,
                                      s->packed, nullptr, ctx->sm_count, st)))
            return e;
    }
    if (s->packed) {
        // Exact re-run, gated on the resolve's flag (as cr_render).
        RasterTargets tx = t;
        tx.packed = 0;
        tx.redo = s->d_redo;
        if ((e = launch_accum_redo_clear_views(views, s->nviews, s->total_pix, s->d_redo,
                                               ctx->sm_count, st)) ||
            // The arena holds the last group's fragments only: decode.
            (e = pass(PASS_COLOR, tx, 0, s->nviews)) ||
            (e = launch_resolve_views(views, s->nviews, 0, s->total_pix, ru, s->d_redo, false,
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
            a.cta_counts = vc.cta + (size_t)v * kCullCtaWords * vc.ctas;
            a.chunk_points = chunk_points;
            a.u = cull_uniforms(cfg, &cams[v], frames[v]->width, frames[v]->height);
            a.visible = vc.visible + (size_t)v * vc.nslots;
            a.chunks = vc.chunks + (size_t)v * vc.chunk_stride;
            a.counters = vc.counters + (size_t)v * CNT_COUNT;
            a.chunk_poff = vc.chunk_poff ? vc.chunk_poff + (size_t)v * vc.chunk_stride : nullptr;
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
    if ((vst = reject_variants(cfg, "batched views"))) return vst;
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
        const bool frags = std::fmax(cfg->minimumPointSize, cfg->maximumPointSize) <= 1.0f;
        cr_status st = views_alloc(ctx, s, frames, nviews, resident.data(), nres, frags);
        if (!st) {
            s->frags = frags;
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
    for (uint32_t v = 0; v < nviews; ++v) {
        cr_status fe = frame_copy_fence(frames[v], ctx->stream);
        if (fe) return fe;
    }
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
                         gp = line.find("\"viewGroupPixels\": "), m = line.find("\"ms\": ");
            if (a == std::string::npos || t == std::string::npos || gp == std::string::npos)
                continue;
            const int cpn = std::atoi(line.c_str() + a + 15);
            const int tiles = std::atoi(line.c_str() + t + 12);
            const int group = std::atoi(line.c_str() + gp + 19);
            if (cpn < kMinChunkPoints || cpn > 65536 || (tiles != 0 && tiles != 1) || group < 0)
                continue;
            ctx->chunk_points = cpn;
            ctx->use_tiles = tiles != 0;
            ctx->view_group_pixels = group;
            if (best_out) *best_out = cr_tuning{cpn, tiles, group, ctx->cull_spin_limit};
            if (best_ms_out)
                *best_ms_out = m == std::string::npos ? 0.0f : (float)std::atof(line.c_str() + m + 6);
            return CR_OK;
        }
    }
    // {chunkPoints, useTiles, viewGroupPixels}
    const int candidates[][3] = {
        {1024, 1, 1048576}, {2048, 1, 1048576}, {4096, 1, 1048576},
        {1024, 1, 2097152}, {2048, 1, 2097152}, {4096, 1, 2097152},
        {1024, 1, 4194304}, {2048, 1, 4194304}, {4096, 1, 4194304},
        {1024, 1, 8388608}, {2048, 1, 8388608}, {4096, 1, 8388608},
        {2048, 1, 0},       {2048, 0, 2097152}, {2048, 0, 4194304}};
    constexpr int kCandidates = (int)(sizeof(candidates) / sizeof(candidates[0]));
    cudaEvent_t e0, e1;
    CR_CUDA(cudaEventCreate(&e0));
    CR_CUDA(cudaEventCreate(&e1));
    std::ostringstream results;
    float best_ms = 0.0f;
    int best = -1;
    cr_status st = CR_OK;
    for (int ci = 0; ci < kCandidates && !st; ++ci) {
        ctx->chunk_points = candidates[ci][0];
        ctx->use_tiles = candidates[ci][1] != 0;
        ctx->view_group_pixels = candidates[ci][2];
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
                << ", \"useTiles\": " << candidates[ci][1] << ", \"viewGroupPixels\": "
                << candidates[ci][2] << ", \"ms\": " << ms << "}";
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
    ctx->view_group_pixels = candidates[best][2];
    if (best_out)
        *best_out = cr_tuning{candidates[best][0], candidates[best][1], candidates[best][2],
                              ctx->cull_spin_limit};
    if (best_ms_out) *best_ms_out = best_ms;
    if (cache_path) {
        std::ofstream out(cache_path, std::ios::app);
        if (!out) return fail(CR_ERR_INVALID_ARGUMENT, "cannot write the autotune cache file");
        out << "{" << tag << ", \"chunkPoints\": " << candidates[best][0]
            << ", \"useTiles\": " << candidates[best][1] << ", \"viewGroupPixels\": "
            << candidates[best][2] << ", \"ms\": " << best_ms
            << ", \"candidates\": [" << results.str() << "]}\n";
    }
    return CR_OK;
}

}  // extern "C"
