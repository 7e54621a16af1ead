// cr_internal.h — library-internal objects and kernel launch interfaces.
#pragma once

#include <cuda_runtime.h>
#include <utility>
#include <stdint.h>

#include <string>
#include <deque>
#include <vector>

#include "cr/cr.h"

// ---------------------------------------------------------------------------
// Error plumbing
// ---------------------------------------------------------------------------
namespace cri {
void set_error(const std::string &detail);
cr_status fail(cr_status st, const std::string &detail);
cr_status cuda_fail(cudaError_t e, const char *what);
}  // namespace cri

#define CR_CUDA(call)                                                        \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess) return cri::cuda_fail(e_, #call);             \
    } while (0)

// ---------------------------------------------------------------------------
// Per-cloud device counters (one cache line).
// ---------------------------------------------------------------------------
enum CounterSlot : int {
    CNT_VISIBLE = 0,     // survivors of the last cull (VisibleBatch count)
    CNT_WORK_DEPTH = 1,  // dynamic work cursor of the one-view point passes
    CNT_WORK_COLOR = 2,  // dynamic work cursor of the colour pass
    CNT_CHUNKS = 3,      // chunk work records written by the last cull
    CNT_ARGS_X = 4,      // CRDispatchArgs mirror: {count, 1, 1}
    CNT_ARGS_Y = 5,
    CNT_ARGS_Z = 6,
    CNT_ERROR = 7,       // first device-side error code (0 = none)
    CNT_POINTS = 8,      // fragment span of the last cull's survivors (chunks rounded to 4)
    CNT_DONE = 9,        // CTAs finished with the dynamic cursor (the last one resets both)
    CNT_CULL_EPOCH = 10,  // one-pass cull: launches completed (its CTAs' publish flags are epoch + 1)
    CNT_CULL_DONE = 11,   // one-pass cull: CTAs finished (the last one advances the epoch)
    CNT_CULL_TICKET = 12, // one-pass cull: next CTA ticket (wraps to 0 after the launch's last)
    CNT_COUNT = 32
};

struct PackScratch;
struct ViewsState;
void views_destroy(ViewsState *s);

// One survivor of the cull with the per-batch values the point passes need
// (cull_classify output, 64 bytes; 16-byte aligned so that it moves as four
// 16-byte words).
struct alignas(16) CullRec {
    cr_visible_batch vb;
    float minX, minY, minZ;  // batch min
    float qx, qy, qz;        // batchSize / steps of the survivor's precision level
    uint32_t first;          // batch firstPoint
    uint32_t file;           // batch fileIndex
    int32_t x0, y0, tw, th;  // screen rectangle (buffer rows), tw <= 0 when unknown
};

// One unit of point-pass work: up to `chunkPoints` consecutive survivor points
// of one batch (64 bytes, 16-byte aligned; written by the cull in survivor
// order).
struct alignas(16) ChunkRec {
    uint32_t first;  // absolute index of the chunk's first point
    uint32_t count;
    int32_t level;
    float thr;
    uint32_t batchIndex;
    uint32_t file;
    float minX, minY, minZ;
    float qx, qy, qz;
    int32_t x0, y0, tw, th;
};
static_assert(sizeof(CullRec) == 64, "CullRec is 64 bytes");
static_assert(sizeof(ChunkRec) == 64, "ChunkRec is 64 bytes");

constexpr int kMinChunkPoints = 256;

struct cr_context {
    PackScratch *pack = nullptr;  // grow-only packer scratch
    ViewsState *views = nullptr;  // buffers and graphs of the last batched render
    double *d_loss = nullptr;     // cr_l2_loss's device accumulator (lazy)
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;    // asynchronous RGBA8 read-backs (lazy)
    cudaStream_t upload_stream = nullptr;  // asynchronous slot-pool uploads (lazy)
    int sm_count = 0;
    int blocks_per_sm[7] = {};        // occupancy of the persistent point passes (per RasterPass)
    int blocks_per_sm_views[7] = {};  // the same, batched-view kernels
    int blocks_per_sm_hash_views = 0;  // the batched-view colour hash kernel
    int chunk_points = 2048;           // points per chunk work record
    int view_group_pixels = 4194304;   // batched views: pixels per depth/colour group
    bool use_tiles = true;             // shared-memory screen tiles
    int cull_spin_limit = 1 << 20;     // polls of a predecessor before a cull CTA gives up
    // Device-side status word (page-locked, mapped into the device's address
    // space): kernels store an error code into it, and the host reads it
    // after the calls that synchronise with the context's stream.
    uint32_t *h_status = nullptr;
    uint32_t *d_status = nullptr;
    // Profiling: a ring of frames, each with a start/stop event per pass.
    static constexpr int kProfRing = 256;
    bool profiling = false;
    int prof_frame = -1;      // ring index of the frame being recorded
    int64_t prof_count = 0;   // frames recorded since profiling was enabled
    cudaEvent_t pass_ev[kProfRing][CR_PASS_COUNT][2] = {};
    bool pass_recorded[kProfRing][CR_PASS_COUNT] = {};
};

// Brackets one pass with profiling events when profiling is on.
struct PassTimer {
    cr_context *ctx;
    int pass;
    PassTimer(cr_context *c, int p) : ctx(c), pass(p) {
        if (ctx->profiling)
            cudaEventRecord(ctx->pass_ev[ctx->prof_frame][pass][0], ctx->stream);
    }
    ~PassTimer() {
        if (ctx->profiling) {
            cudaEventRecord(ctx->pass_ev[ctx->prof_frame][pass][1], ctx->stream);
            ctx->pass_recorded[ctx->prof_frame][pass] = true;
        }
    }
};

// Makes `dev` current for a scope (the previous device is restored).
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

// Asynchronous slot-pool uploads of a cloud (csrc/upload.cpp).
constexpr uint8_t kSlotIdle = 0, kSlotPending = 1, kSlotCancelled = 2;
struct UploadBatch {
    int32_t slot;
    cr_raster_batch rec;  // the record published when the copy lands
};
struct PendingUpload {
    cudaEvent_t ev = nullptr;  // recorded on the upload stream after the copies
    uint64_t stage_off = 0;    // staging ring bytes held until the copy lands
    std::vector<UploadBatch> batches;
};
struct UploadState {
    unsigned char *h_stage = nullptr;  // page-locked staging ring
    uint64_t cap = 0, want_cap = 0;    // ring bytes; size asked for (0 = default)
    uint64_t head = 0, tail = 0;       // next free byte; start of the oldest region
    std::deque<PendingUpload> q;       // in flight, oldest first
    std::vector<uint8_t> slot;         // per slot: kSlotIdle / Pending / Cancelled
    std::vector<cudaEvent_t> spare;    // events of landed uploads, reused
    cudaEvent_t ready = nullptr;       // context-stream point the copies wait for
    uint32_t in_flight_batches = 0;
};

struct cr_cloud {
    cr_context *ctx = nullptr;
    UploadState *up = nullptr;  // asynchronous uploads (lazy)
    cr_capacity cap{0, 0};
    std::vector<cr_raster_file> files;        // file table (world matrices)
    std::vector<cr_raster_file> frame_files;  // last updateFiles snapshot (what the kernels read)
    // frame_files not yet copied to d_files: a table of at most kInlineFiles
    // files travels in the one-view kernels' parameters instead, and the
    // device copy is made only for the consumers that read it
    // (ensure_device_files).
    bool files_dirty = false;
    std::vector<cr_raster_batch> mirror;      // host mirror of every slot
    std::vector<int32_t> free_slots;          // LIFO, back() is handed out first
    int64_t dirty_lo = INT64_MAX, dirty_hi = -1;
    uint32_t resident = 0;
    uint64_t points = 0;

    // Device slot pool (structure of arrays, as the reference lays it out).
    uint32_t *d_low = nullptr, *d_med = nullptr, *d_high = nullptr, *d_colors = nullptr;
    uint8_t *d_levels = nullptr;
    cr_raster_batch *d_batches = nullptr;
    cr_raster_file *d_files = nullptr;
    uint32_t d_files_cap = 0;

    // Cull outputs and scratch.
    cr_visible_batch *d_visible = nullptr;   // ordered survivors
    CullRec *d_cull_tmp = nullptr;           // per-CTA compacted survivors
    uint32_t *d_cull_cta = nullptr;          // per-CTA survivor and chunk counts
    ChunkRec *d_chunks = nullptr;            // chunk work records
    uint64_t chunk_cap = 0;                  // capacity of d_chunks

    // Fragments of the last depth pass, in pool point index space: a chunk
    // starting at point p keeps its n kept points compacted at [p, p + n).
    uint32_t *d_frag_xy = nullptr;     // pixel x | row << 16
    uint2 *d_frag_zc = nullptr;        // NDC z bits, RGBA8 (after the colorize options)
    uint32_t *d_frag_count = nullptr;  // kept points per chunk record
    // Per-point float4 attributes of the colour variants, written by user
    // kernels (lazy, zeroed on allocation): displacement, the previous
    // frame's displacement (motion blur), tint.
    float4 *d_disp = nullptr, *d_prev_disp = nullptr, *d_tint = nullptr;
    uint32_t *d_counters = nullptr;          // CounterSlot words

    // Pinned staging ring for the per-frame file table upload.
    static constexpr int kFileRing = 8;
    cr_raster_file *h_files_ring = nullptr;
    cudaEvent_t ring_events[kFileRing] = {};
    bool ring_used[kFileRing] = {};
    int ring_slot = -1;
};

struct cr_frame {
    cr_context *ctx = nullptr;
    int width = 0, height = 0;
    uint32_t *d_depth = nullptr;            // HQS depth plane (RasterPixel.depth)
    uint4 *d_accum = nullptr;               // HQS red, green, blue, count (+1 entry: redo flag)
    uint32_t *d_redo = nullptr;             // word 0 of d_accum[width * height]
    unsigned long long *d_nearest = nullptr;  // (depth << 32) | ~pointIndex
    uint32_t *d_rgba[2] = {nullptr, nullptr}; // RGBA8 ping-pong (resolve, hole fill)
    float *d_depthf = nullptr;              // resolve R32F depth
    float4 *d_fsum = nullptr;               // differentiable colours: FP32 R, G, B sums (lazy)
    uint32_t *d_fcount = nullptr;           //   and their sample counts
    int final_rgba = 0;                     // which d_rgba holds the final image
    int last_mode = -1;                     // 0 HQS, 1 nearest, -1 none
    // Asynchronous read-back: `rendered` is recorded on the context stream
    // and waited on by the copy stream; `copied` is recorded after the copy
    // and waited on by the next write of the RGBA8 planes.
    cudaEvent_t ev_rendered = nullptr, ev_copied = nullptr;
    bool copy_pending = false;
    // The last kCopyRing read-backs' completion events (copy n in slot
    // n % kCopyRing) and the number of read-backs enqueued so far.
    static constexpr int kCopyRing = 4;
    cudaEvent_t ev_copy_ring[kCopyRing] = {};
    uint64_t copies = 0;
};

// Asynchronous uploads: wait for and publish every upload in flight; free
// the upload state; cancel a slot's upload in flight (true if it had one);
// whether a slot has an upload in flight.
cr_status uploads_drain(cr_cloud *c);
void uploads_free(cr_cloud *c);
bool uploads_cancel(cr_cloud *c, int32_t slot);
bool upload_slot_busy(const cr_cloud *c, uint32_t slot);
void mark_dirty(cr_cloud *c, int64_t lo, int64_t hi);
cr_status flush_mirror(cr_cloud *c);

// Makes later work on `s` wait (on the device) for the frame's enqueued
// asynchronous read-backs; call before the first write of the RGBA8 planes.
cr_status frame_copy_fence(cr_frame *f, cudaStream_t s);

// The device-side status word of the context, read after a call has
// synchronised with the context's stream: CR_ERR_TIMEOUT (and the word
// cleared) when a bounded device-side wait gave up, else CR_OK.
cr_status device_status(cr_context *ctx);

// ---------------------------------------------------------------------------
// Kernel launch interfaces
// ---------------------------------------------------------------------------
struct CullUniforms {
    float view[16];
    float proj[16];
    int width, height;
    int enableFrustumCulling, lodBias, enableCLOD;
};

// Words per 256-slot CTA in CullArgs::cta_counts: survivors, chunk records,
// fragment span.
// Per 256-slot CTA: survivor, chunk and point counts, and the one-pass
// cull's publish flag.
constexpr uint32_t kCullCtaWords = 4;
// CNT_ERROR code: a one-pass cull CTA gave up waiting for a predecessor.
constexpr uint32_t kErrCullWait = 1u;
// Status code: a radix sort tile of the packer gave up waiting for a
// predecessor's digit counts.
constexpr uint32_t kErrSortWait = 2u;
// Status code: a point pass gave up waiting for a bulk copy into shared memory.
constexpr uint32_t kErrStageWait = 3u;

// Arguments of the cull of one view of one cloud (inputs, scratch, outputs).
struct CullArgs {
    const cr_raster_batch *batches;
    uint32_t nbatches;
    const cr_raster_file *files;
    uint32_t nfiles;
    CullRec *tmp;           // nbatches records
    uint32_t *cta_counts;   // kCullCtaWords per 256-slot CTA
    uint32_t chunk_points;
    CullUniforms u;
    cr_visible_batch *visible;  // nbatches
    ChunkRec *chunks;           // chunk capacity of the cloud
    uint32_t *counters;         // CNT_COUNT words
    uint32_t *chunk_poff;       // per chunk record: offset of its fragments within the
                                // view's fragment span, a multiple of 4 (NULL: not written)
    uint32_t spin_limit;        // one-pass cull: polls of a predecessor before giving up
    uint32_t *status;           // one-pass cull: the context's device-side status word
};

// Launches a kernel that may begin while the previous kernel on the stream
// finishes (programmatic stream serialisation); the kernel orders itself
// after that kernel with crd::grid_wait().
template <typename... Params, typename... Args>
cudaError_t launch_programmatic(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem,
                                cudaStream_t s, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// File tables of at most this many files ride in the kernel parameters of
// the one-view passes (read through a __grid_constant__ parameter), so a
// camera move enqueues no copy between frames.
constexpr uint32_t kInlineFiles = 4;
struct InlineFiles {
    cr_raster_file f[kInlineFiles];
    uint32_t n;  // 0: read the device table
};
// The inline table of a cloud (n = 0 when its table is larger).
InlineFiles inline_files(const cr_cloud *c);
// Copies frame_files to d_files if a camera update left it only on the host.
cr_status ensure_device_files(cr_cloud *c);

// Zeroing of an HQS frame's depth plane (whole 16-byte groups, then a tail
// of up to three words) and accumulators with the redo word behind them.
struct FrameClear {
    uint4 *depth4;
    size_t ndepth4;
    uint32_t *tail;
    uint32_t ntail;
    uint4 *accum;
    size_t naccum;
};
FrameClear frame_clear_of(cr_frame *f);

// clear: also zero that frame in the same launch (CTAs after the cull's).
cr_status launch_cull(cr_cloud *cloud, const CullUniforms &u, cudaStream_t s,
                      const FrameClear *clear = nullptr);
// Culls of several views in one pair of launches; d_args holds one CullArgs
// per view (device memory).
cr_status launch_cull_views(const CullArgs *d_args, uint32_t nslots, uint32_t nviews,
                            cudaStream_t s);
// Chunk records a cloud may need at the given chunk size.
uint64_t chunk_capacity(const cr_capacity &cap, int chunk_points);

// PASS_DEPTH_FRAG is the depth pass that also writes each kept point as a
// fragment; PASS_COLOR_FRAG is the colour pass over those fragments.
enum RasterPass : int {
    PASS_DEPTH = 0,
    PASS_COLOR = 1,
    PASS_NEAREST = 2,
    PASS_DEPTH_FRAG = 3,
    PASS_COLOR_FRAG = 4,
    PASS_COLOR_F32 = 5,  // differentiable colours: FP32 sums of learnable colours + count
    PASS_GRAD = 6        // their adjoint: per point, dL/dpixel / count over its visible pixels
};
constexpr int kRasterPassCount = 7;
static_assert(kRasterPassCount == sizeof(cr_context::blocks_per_sm) / sizeof(int),
              "one occupancy entry per raster pass");

struct RasterUniforms {
    float view[16];
    float proj[16];
    int width, height;
    int lodDither;
    int pointSizeMode;
    float minimumPointSize, maximumPointSize, pointSizeScale;
    float depthTolerance;
    int colorizeChunks, colorizeOverdraw;
};

struct RasterTargets {
    uint32_t *depth;              // HQS depth plane
    uint4 *accum;                 // HQS accumulators
    unsigned long long *nearest;  // nearest key plane
    float4 *fsum = nullptr;       // differentiable colours: FP32 sums per pixel
    uint32_t *fcount = nullptr;   //   and sample counts
    // Colour adds as two 64-bit words per pixel (R | G << 32, B | count << 32)
    // instead of four 32-bit ones; exact while a pixel holds at most
    // kPackedMaxCount samples, which the resolve checks.
    int packed = 0;
    // Non-null: the pass runs only if *redo != 0 (the exact re-run of a
    // frame whose resolve found a pixel past kPackedMaxCount).
    const uint32_t *redo = nullptr;
};

// Largest per-pixel sample count whose 8-bit channel sums cannot wrap a
// 32-bit field: 255 * 16843009 = 2^32 - 1.
constexpr uint32_t kPackedMaxCount = 16843009u;

cr_status launch_raster(cr_cloud *cloud, RasterPass pass, const RasterUniforms &u,
                        const RasterTargets &t, cudaStream_t s);
// PASS_COLOR_F32 (colors: 3 floats per pool point) or PASS_GRAD (dldimg: 3
// floats per pixel, grad: 3 floats per pool point, added to) of one cloud.
cr_status launch_raster_f32(cr_cloud *cloud, RasterPass pass, const RasterUniforms &u,
                            const RasterTargets &t, const float *colors, const float *dldimg,
                            float *grad, cudaStream_t s);

// Mode, point-size mode and the unsupported colour effects of a configuration.
cr_status validate_config(const cr_config *cfg);
// The colour variants (displacement, tint, coverage, motion blur) of an HQS
// configuration; CR_ERR_UNSUPPORTED naming `where` when they are on.
bool variants_on(const cr_config *cfg);
cr_status reject_variants(const cr_config *cfg, const char *where);
// HQS depth (color = false) or colour pass with the colour variants on.
cr_status launch_variant_pass(cr_cloud *cloud, bool color, const RasterUniforms &u,
                              const cr_config &cfg, const RasterTargets &t, cudaStream_t s);
// Occupancy of the batched-view point passes (call before capturing them).
void raster_prepare_views(cr_context *ctx);

// Batched views: at most kMaxViews views per call.
constexpr uint32_t kMaxViews = 256;

// One view of a batched render (device memory): its frame's planes and
// camera.  pix_begin is the exclusive prefix of width * height over the
// views (the per-pixel kernels walk all views' pixels as one range).
struct ViewDesc {
    uint32_t *depth;
    uint4 *accum;
    unsigned long long *nearest;
    uint32_t *rgba[2];  // resolve target and hole-fill ping-pong
    float *depthf;
    int width, height;
    uint32_t pix_begin, pad;
    float view[16], proj[16];
};
static_assert(sizeof(ViewDesc) == 192, "ViewDesc is 192 bytes");

// Fragment arena of one cloud's batched views: view v's fragments occupy
// [prefix of the views' fragment spans, + its span); chunk record j of view
// v has its count at count[v * chunk_stride + j] and its offset within the
// view's span at poff[same].  cap entries; *overflow is set by the depth
// pass when the spans exceed cap (the colour pass then decodes the points).
struct ViewsFragments {
    uint32_t *xy;
    uint2 *zc;
    uint32_t *count;
    const uint32_t *poff;
    unsigned long long cap;
    uint32_t *overflow;
};

// The point pass `pass` of one cloud over all views in one launch.  Chunk
// records of view v start at chunks + v * chunk_stride and its counters at
// counters + v * CNT_COUNT; its file table at files + v * nfiles.  u carries
// the configuration (the per-view sizes and cameras come from views).
// PASS_DEPTH_FRAG / PASS_COLOR_FRAG need frags.
cr_status launch_raster_views(cr_cloud *cloud, RasterPass pass, const RasterUniforms &u,
                              const RasterTargets &t, const ViewDesc *views, uint32_t nviews,
                              const cr_raster_file *files, uint32_t nfiles,
                              const ChunkRec *chunks, uint32_t chunk_stride,
                              uint32_t *counters, const ViewsFragments *frags, cudaStream_t s);

struct ResolveUniforms {
    int width, height;
    float background[4];
};

// check: set *f->d_redo when a pixel's count exceeds kPackedMaxCount (the
// colour pass used packed adds).  redo: run only if *redo != 0.
cr_status launch_resolve_hqs(cr_frame *f, const ResolveUniforms &u, cudaStream_t s, bool check,
                             const uint32_t *redo);
// Zeroes the accumulators if *f->d_redo != 0.
cr_status launch_accum_redo_clear(cr_frame *f, cudaStream_t s);
// The exact re-run of a frame drawn from fragments, in one single-CTA launch
// that returns at once unless *t.redo != 0: zero the accumulators, colour pass
// of every cloud with 32-bit adds (t.packed = 0), resolve into d_rgba[0].
// At most hqs_redo_max_clouds() clouds.
cr_status launch_hqs_redo(cr_frame *f, cr_cloud *const *clouds, uint32_t nclouds,
                          const RasterUniforms &u, const RasterTargets &t,
                          const ResolveUniforms &ru, cudaStream_t s);
uint32_t hqs_redo_max_clouds();
// Zeroes the depth plane, the accumulators and the redo word of an HQS frame.
cr_status launch_frame_clear(cr_frame *f, cudaStream_t s);
// Coverage resolve (weighted-blended accumulation) into d_rgba[0].
cr_status launch_resolve_coverage(cr_frame *f, const ResolveUniforms &u, cudaStream_t s);

// Batched views: every view's pixels form one range, view after view
// (ViewDesc::pix_begin); views [0, nviews) of `views` cover [pix0, pix0+npix).
// Zero those views' depth planes and accumulators (and *redo_flag if
// zero_flag).
cr_status launch_clear_views(const ViewDesc *views, uint32_t nviews, uint32_t pix0, uint32_t npix,
                             uint32_t *redo_flag, bool zero_flag, int sm_count, cudaStream_t s);
// Zero every view's accumulators if *redo_flag != 0 (views from view 0).
cr_status launch_accum_redo_clear_views(const ViewDesc *views, uint32_t nviews,
                                        uint32_t total_pix, const uint32_t *redo_flag,
                                        int sm_count, cudaStream_t s);
// Resolve of those views (check / redo as launch_resolve_hqs).
cr_status launch_resolve_views(const ViewDesc *views, uint32_t nviews, uint32_t pix0,
                               uint32_t npix, const ResolveUniforms &u, uint32_t *redo_flag,
                               bool check, const uint32_t *redo, int sm_count, cudaStream_t s);
// Differentiable colours: image[3p + c] = fsum[p].c / fcount[p], or the
// background where the count is 0.
cr_status launch_resolve_f32(cr_frame *f, const float background[3], float *image,
                             cudaStream_t s);
// dldimg = 2 * scale * (image - target) over n floats; the loss
// scale * sum (image - target)^2 is added to *loss (device double) if loss.
cr_status launch_l2_loss(const float *image, const float *target, uint64_t n, float scale,
                         float *dldimg, double *loss, int sm_count, cudaStream_t s);
// One hole-fill iteration of every view: rgba[src] -> rgba[1 - src].
cr_status launch_hole_fill_views(const ViewDesc *views, uint32_t nviews, uint32_t total_pix,
                                 int src, int sm_count, cudaStream_t s);
cr_status launch_resolve_nearest(cr_frame *f, const uint32_t *colors, const ResolveUniforms &u,
                                 cudaStream_t s);
cr_status launch_hole_fill(cr_frame *f, int iterations, cudaStream_t s);
// XOR 0x80000000 into every word of the frame's depth plane.
cr_status launch_flip_depth_order(cr_frame *f, cudaStream_t s);
cr_status launch_split_nearest(const unsigned long long *keys, uint32_t *depth_out,
                               uint32_t *index_out, size_t n, cudaStream_t s);


cr_status pack_run(cr_context *ctx, cr_cloud *cloud, const cr_pack_input *in, uint64_t count,
                   const cr_pack_params *prm, int on_device, uint32_t first_slot,
                   uint32_t *src_idx_host);
