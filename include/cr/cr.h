/*
 * cr.h — C ABI of the B200 point-cloud compute rasteriser.
 *
 * This header is the drop-in boundary for the batch-oriented point-cloud
 * rasteriser of Satin-ComputeRasteriser.  It replaces the Swift/Metal plugin
 * surface of that package:
 *
 *   reference (Swift / Metal)                          C ABI here
 *   -----------------------------------------------    ---------------------------
 *   ComputeRasteriserTypes.h:11-63 (shared structs)    cr_raster_batch, cr_raster_file,
 *                                                      cr_raster_pixel, cr_visible_batch,
 *                                                      cr_dispatch_args
 *   ComputeRasteriserTypes.swift:26-142 (config)        cr_config
 *   ComputeRasteriserPointCloud.swift:23-40 (capacity)  cr_capacity
 *   ComputeRasteriserPointCloud.swift:202-547 (pool)    cr_cloud_*
 *   ComputeRasteriser.swift:201-296 (update/encode)     cr_cloud_update_files, cr_render
 *   ComputeRasteriser.swift:766-838 (per-size buffers)  cr_frame_*
 *   ComputeRasteriser.swift:609-670 (pickPointIndex)    cr_pick
 *   GPUPacker.swift:140-392 (pack / packChunk)          cr_pack
 *
 * Conventions
 *   - Every entry point returns a cr_status; CR_OK is 0.  The thread-local
 *     detail of the last failure is available from cr_last_error_detail().
 *   - Sizes are element counts unless a name says bytes.
 *   - Host pointers are borrowed for the duration of the call only.
 *   - Device memory is owned by the library (context, cloud, frame objects).
 *   - Each context owns one CUDA stream; every call that launches work
 *     enqueues it on that stream.  Read-back calls synchronise the stream.
 *   - Calls on one context (and the objects created from it) are not
 *     re-entrant: serialise them on the host, as the reference serialises
 *     its render loop on one thread.
 *   - Matrices are column-major float[16] (m[col*4 + row]), the simd_float4x4
 *     layout the reference passes to its shaders.
 */
#ifndef CR_CR_H
#define CR_CR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define CR_API __declspec(dllexport)
#else
#define CR_API __attribute__((visibility("default")))
#endif

/* ------------------------------------------------------------------------ */
/* Constants (ComputeRasteriserTypes.h:4-9, ComputeRasteriserTypes.swift:4-6) */
/* ------------------------------------------------------------------------ */
#define CR_THREADS_PER_GROUP 128
#define CR_DEFAULT_POINTS_PER_BATCH (CR_THREADS_PER_GROUP * 80) /* 10240 */
#define CR_MASK_10BIT 1023u
#define CR_MAX_DEPTH 0xffffffffu
#define CR_INVALID_INDEX 0xffffffffu

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum cr_status {
    CR_OK = 0,
    CR_ERR_INVALID_ARGUMENT = 1, /* null handle, bad size, bad enum          */
    CR_ERR_OUT_OF_MEMORY = 2,    /* device or pinned allocation failed      */
    CR_ERR_CUDA = 3,             /* a CUDA runtime call failed               */
    CR_ERR_UNSUPPORTED = 4,      /* feature flag outside the hot path is set */
    CR_ERR_CAPACITY = 5,         /* slot pool or fixed buffer too small      */
    CR_ERR_TIMEOUT = 6,          /* a bounded device-side wait gave up       */
    CR_ERR_NO_DEVICE = 7,        /* no CUDA device / library not usable      */
    CR_ERR_INTERNAL = 8,
    CR_ERR_FORMAT = 9            /* malformed input file (detail: the case)  */
} cr_status;

/* ------------------------------------------------------------------------ */
/* Shared GPU structs, byte-identical to ComputeRasteriserTypes.h:11-63.     */
/* ------------------------------------------------------------------------ */

/* RasterBatch (ComputeRasteriserTypes.h:11-33): one slot of the pool.
 * lodCum01..67 hold eight cumulative uint16 LOD counts, two per word (low
 * level in the low half).  lodCum67 == 0 marks a legacy (unbucketed) batch. */
typedef struct cr_raster_batch {
    int32_t state; /* 0 = slot not resident */
    float minX, minY, minZ;
    float maxX, maxY, maxZ;
    uint32_t numPoints;
    uint32_t firstPoint;
    uint32_t fileIndex;
    uint32_t lodCum01, lodCum23, lodCum45, lodCum67;
    uint32_t padding7, padding8;
} cr_raster_batch;

/* RasterFile (ComputeRasteriserTypes.h:35-40): per-file transforms. */
typedef struct cr_raster_file {
    float transform[16];        /* viewProjection * world              */
    float transformFrustum[16]; /* frustum matrix * world              */
    float world[16];            /* model * file world                  */
    float prevTransform[16];    /* previous frame's viewProjection*world */
} cr_raster_file;

/* RasterPixel (ComputeRasteriserTypes.h:42-50): the HQS accumulator of one
 * pixel as the reference lays it out.  Frames store the same quantities as
 * structure-of-arrays planes; cr_frame_read_pixels re-interleaves them. */
typedef struct cr_raster_pixel {
    uint32_t depth;
    uint32_t red, green, blue, count;
    uint32_t weight;
    uint32_t padding[2];
} cr_raster_pixel;

/* VisibleBatch (ComputeRasteriserTypes.h:52-57): one cull survivor. */
typedef struct cr_visible_batch {
    uint32_t batchIndex;
    int32_t level;
    float lodThreshold;
    uint32_t activePoints;
} cr_visible_batch;

/* CRDispatchArgs (ComputeRasteriserTypes.h:59-63). */
typedef struct cr_dispatch_args {
    uint32_t threadgroupsX, threadgroupsY, threadgroupsZ;
} cr_dispatch_args;

/* ------------------------------------------------------------------------ */
/* Configuration (ComputeRasteriserConfiguration, ComputeRasteriserTypes.swift:26-142) */
/* ------------------------------------------------------------------------ */
typedef enum cr_mode {
    CR_MODE_HIGH_QUALITY_AVERAGE = 0, /* .highQualityAverage */
    CR_MODE_NEAREST_POINT = 1         /* .nearestPoint        */
} cr_mode;

typedef enum cr_point_size_mode {
    CR_POINT_SIZE_SCREEN_SPACE = 0,
    CR_POINT_SIZE_WORLD_SPACE = 1
} cr_point_size_mode;

/* Field names and defaults follow ComputeRasteriserConfiguration.init
 * (ComputeRasteriserTypes.swift:97-119); booleans are int32 0/1.
 * applyDisplacement, applyTint, tintAlphaIsCoverage and motionBlur > 0 are
 * user-programmable effects outside this library; cr_render returns
 * CR_ERR_UNSUPPORTED when any of them is set. */
typedef struct cr_config {
    int32_t mode;              /* cr_mode,             default HQS  */
    float depthTolerance;      /* default 0.01                      */
    float backgroundColor[4];  /* default (0,0,0,0)                 */
    int32_t enableFrustumCulling; /* default 1                      */
    int32_t lodBias;           /* default 0                         */
    int32_t enableCLOD;        /* default 1                         */
    int32_t enableLODDither;   /* default 1                         */
    int32_t holeFillIterations; /* default 0                        */
    int32_t colorizeChunks;    /* default 0                         */
    int32_t colorizeOverdraw;  /* default 0                         */
    int32_t pointSizeMode;     /* cr_point_size_mode, default screen */
    float minimumPointSize;    /* default 1                         */
    float maximumPointSize;    /* default 1                         */
    float pointSizeScale;      /* default 1                         */
    int32_t applyDisplacement; /* default 0 (cr_cloud_attribute)    */
    int32_t applyTint;         /* default 0 (cr_cloud_attribute)    */
    int32_t tintAlphaIsCoverage; /* default 0: tint a = coverage    */
    int32_t writesSceneDepth;  /* default 1 (composite only)        */
    float motionBlur;          /* default 0 (velocity scale)        */
    int32_t motionBlurSamples; /* default 8                         */
    float motionBlurMaxSpread; /* default 64                        */
} cr_config;

/* Camera as the reference's processors receive it: Satin
 * camera.viewMatrix and camera.projectionMatrix (ComputeRasteriser.swift:208-213). */
typedef struct cr_camera {
    float view[16];
    float projection[16];
} cr_camera;

/* ComputeRasteriserCapacity (ComputeRasteriserPointCloud.swift:23-40). */
typedef struct cr_capacity {
    uint32_t maxResidentBatches;
    uint32_t pointsPerBatch;
} cr_capacity;

typedef struct cr_cloud_info {
    cr_capacity capacity;
    uint32_t residentBatchCount; /* slots with state != 0          */
    uint64_t pointCount;         /* sum of resident numPoints      */
    uint32_t freeSlotCount;
    uint32_t fileCount;
} cr_cloud_info;

typedef struct cr_context cr_context;
typedef struct cr_cloud cr_cloud;
typedef struct cr_frame cr_frame;

/* ------------------------------------------------------------------------ */
/* Errors and versions                                                       */
/* ------------------------------------------------------------------------ */
CR_API const char *cr_status_string(cr_status status);
/* Detail of the last failure on the calling thread ("" if none). */
CR_API const char *cr_last_error_detail(void);
/* Layout self-description, for bindings that mirror the structs:
 * sizes[0..4] = sizeof batch, file, pixel, visible, dispatch args. */
CR_API cr_status cr_layout_sizes(uint32_t sizes[5]);
/* ComputeRasteriserConfiguration() defaults. */
CR_API cr_status cr_config_default(cr_config *out);

/* ------------------------------------------------------------------------ */
/* Context                                                                   */
/* ------------------------------------------------------------------------ */
CR_API cr_status cr_context_create(int device, cr_context **out);
CR_API cr_status cr_context_destroy(cr_context *ctx);
/* Wait for all work queued on the context's stream.
 *
 * Device-side status.  The one-view cull waits, with a bounded number of
 * polls (cr_tuning.cullSpinLimit), for the survivor counts of the cull CTAs
 * before it.  A CTA whose wait runs out counts that predecessor as empty, so
 * the frame's survivor list and image are incomplete, and records the event
 * in a word of the context.  The next call that synchronises with the
 * context's work (cr_context_synchronize, the cr_frame_read_* calls,
 * cr_frame_read_wait, cr_cloud_read_visible, cr_pick) returns
 * CR_ERR_TIMEOUT, with the detail in cr_last_error_detail, and clears the
 * word.  The reference's passes report nothing from the GPU (their guards
 * are silent no-ops, ComputeRasteriser.swift:278-283). */
CR_API cr_status cr_context_synchronize(cr_context *ctx);
/* The context's cudaStream_t, as an opaque pointer. */
CR_API cr_status cr_context_stream(cr_context *ctx, void **stream_out);
/* Release the packer's grow-only scratch (it is re-allocated by the next pack). */
CR_API cr_status cr_context_trim(cr_context *ctx);

/* ------------------------------------------------------------------------ */
/* Point cloud slot pool (ComputeRasteriserPointCloud)                       */
/* ------------------------------------------------------------------------ */
/* init(context:capacity:files:originShift:label:)  — ComputeRasteriserPointCloud.swift:202-218.
 * files may be NULL with nfiles == 0, which installs one identity RasterFile. */
CR_API cr_status cr_cloud_create(cr_context *ctx, cr_capacity capacity,
                                 const cr_raster_file *files, uint32_t nfiles,
                                 cr_cloud **out);
CR_API cr_status cr_cloud_destroy(cr_cloud *cloud);
/* reallocate(to:files:) — ComputeRasteriserPointCloud.swift:519-530: new
 * capacity, all slots empty. */
CR_API cr_status cr_cloud_reallocate(cr_cloud *cloud, cr_capacity capacity,
                                     const cr_raster_file *files, uint32_t nfiles);
/* Replace the file table without touching slots (replacePackedPointCloud's
 * fitting branch, ComputeRasteriserPointCloud.swift:256-259). */
CR_API cr_status cr_cloud_set_files(cr_cloud *cloud, const cr_raster_file *files,
                                    uint32_t nfiles);
/* addBatches(...) — ComputeRasteriserPointCloud.swift:410-452.  Each input
 * batch names a run [firstPoint, firstPoint+numPoints) of the host arrays;
 * it is copied into a free slot (LIFO free list), its firstPoint rebased to
 * slot*pointsPerBatch and its state set to 1.  slots_out (n entries) receives
 * the chosen slot of each batch.  points_len is the element count of every
 * host array (bounds check).  CR_ERR_CAPACITY if fewer than n slots are free
 * or a batch exceeds pointsPerBatch. */
CR_API cr_status cr_cloud_add_batches(cr_cloud *cloud,
                                      const uint32_t *xyz_low, const uint32_t *xyz_med,
                                      const uint32_t *xyz_high, const uint32_t *colors,
                                      const uint8_t *levels, uint64_t points_len,
                                      const cr_raster_batch *batches, uint32_t n,
                                      int commit, int32_t *slots_out);
/* removeBatches(slots:commit:) — ComputeRasteriserPointCloud.swift:460-473. */
CR_API cr_status cr_cloud_remove_batches(cr_cloud *cloud, const int32_t *slots, uint32_t n,
                                         int commit);

/* Per-point float4 attributes of the colour variants (ColorPass/Shaders.metal
 * :38-42, DepthPass/Shaders.metal:30-34): the buffers a user kernel writes
 * before cr_render, as the reference's DisplacementPass / TintPass sketches
 * write the cloud's displacement and tint buffers.  One float4 per pool
 * point (index = the point's pool index, RasterBatch.firstPoint + i), *count
 * of them; allocated zeroed on first request and valid until the cloud is
 * reallocated, released or destroyed; write them on the context's stream
 * (cr_context_stream) or synchronise first.
 *   CR_ATTR_DISPLACEMENT       xyz added to the decoded position when
 *                              config.applyDisplacement; a NaN component
 *                              drops the point from both passes
 *   CR_ATTR_PREV_DISPLACEMENT  the previous frame's displacement (motion
 *                              blur); cr_render copies the displacement here
 *                              after each frame's colour pass while
 *                              config.motionBlur > 0
 *   CR_ATTR_TINT               rgba with config.applyTint: colour = mix(colour,
 *                              saturate(rgb), saturate(a)); a < 0 drops the
 *                              point's colour; with tintAlphaIsCoverage,
 *                              coverage = saturate(1 - a) for the
 *                              weighted-blended accumulation
 * A cloud without a buffer reads zeros.  The variants run in cr_render
 * (and cr_render_stages) only; batched views and the differentiable colours
 * return CR_ERR_UNSUPPORTED while they are on. */
typedef enum cr_attribute {
    CR_ATTR_DISPLACEMENT = 0,
    CR_ATTR_PREV_DISPLACEMENT = 1,
    CR_ATTR_TINT = 2
} cr_attribute;
CR_API cr_status cr_cloud_attribute(cr_cloud *cloud, int32_t which, void **device_ptr,
                                    uint64_t *count);
CR_API cr_status cr_cloud_release_attribute(cr_cloud *cloud, int32_t which);

/* The cloud's device arrays, for user kernels that compute the attributes
 * (the buffers the reference's DisplacementPass / TintPass bind for their
 * sketches: batches, split-precision words, levels, colours).  Read-only for
 * the caller; valid until the cloud is reallocated or destroyed. */
typedef struct cr_cloud_arrays {
    const cr_raster_batch *batches; /* maxResidentBatches slots */
    const uint32_t *xyzLow, *xyzMed, *xyzHigh, *colors;
    const uint8_t *levels;
    uint64_t points; /* pool points (maxResidentBatches * pointsPerBatch) */
    uint32_t slots;
    uint32_t pointsPerBatch;
} cr_cloud_arrays;
CR_API cr_status cr_cloud_device_arrays(cr_cloud *cloud, cr_cloud_arrays *out);

/* Asynchronous addBatches for streaming residency: takes the slots at once
 * (slots_out) and copies the points into them while frames render.  The
 * arrays are copied into the cloud's page-locked staging ring before the
 * call returns (host pointers borrowed for the call only); the device copies
 * run on the context's upload stream after the render work enqueued before
 * the call.  The slots stay non-resident (state 0, skipped by the cull) until
 * cr_cloud_poll_uploads or cr_cloud_wait_uploads sees their copy landed and
 * publishes them (state 1; `commit` then uploads the batch table, as
 * cr_cloud_commit).  flags = CR_UPLOAD_BORROW skips the staging copy (below).  Removing a slot whose copy is in flight cancels it: the
 * slot returns to the free list when the copy lands.  When the ring has no
 * room the call waits for the oldest copy; a call larger than the ring grows
 * it.  No counterpart in the reference, whose addBatches
 * (ComputeRasteriserPointCloud.swift:410-452) copies synchronously. */
enum {
    /* The arrays are page-locked (cr_host_alloc or registered memory) and stay
     * valid and unchanged until the upload is published: they are the source
     * of the device copies, with no staging copy. */
    CR_UPLOAD_BORROW = 1
};
CR_API cr_status cr_cloud_add_batches_async(cr_cloud *cloud, const uint32_t *xyz_low,
                                            const uint32_t *xyz_med, const uint32_t *xyz_high,
                                            const uint32_t *colors, const uint8_t *levels,
                                            uint64_t points_len, const cr_raster_batch *batches,
                                            uint32_t n, uint32_t flags, int32_t *slots_out);
/* Publishes the uploads whose copies have landed (non-blocking): batches
 * published by this call and batches still in flight (either may be NULL). */
CR_API cr_status cr_cloud_poll_uploads(cr_cloud *cloud, int commit, uint32_t *landed_batches,
                                       uint32_t *in_flight_batches);
/* Waits for every upload in flight and publishes it. */
CR_API cr_status cr_cloud_wait_uploads(cr_cloud *cloud, int commit);
/* Staging ring size in bytes (default 64 MiB; waits for copies in flight). */
CR_API cr_status cr_cloud_set_upload_staging(cr_cloud *cloud, uint64_t bytes);
/* commitBatchUpdates() — ComputeRasteriserPointCloud.swift:481-483 (uploads
 * the dirty slot range of the host batch mirror). */
CR_API cr_status cr_cloud_commit(cr_cloud *cloud);
/* clearAllBatches() — ComputeRasteriserPointCloud.swift:367-377. */
CR_API cr_status cr_cloud_clear(cr_cloud *cloud);
/* updateFiles(viewProjection:modelMatrix:frustumTransform:prevViewProjection:)
 * — ComputeRasteriserPointCloud.swift:487-515.  frustum and prev_vp may be NULL. */
CR_API cr_status cr_cloud_update_files(cr_cloud *cloud, const float vp[16],
                                       const float model[16], const float *frustum,
                                       const float *prev_vp);
CR_API cr_status cr_cloud_info_get(const cr_cloud *cloud, cr_cloud_info *out);
/* Host mirror of the file table as last written by cr_cloud_update_files. */
CR_API cr_status cr_cloud_read_files(const cr_cloud *cloud, cr_raster_file *out, uint32_t n);
/* Device batch table, slots [first, first+n). */
CR_API cr_status cr_cloud_read_batches(cr_cloud *cloud, cr_raster_batch *out, uint32_t first,
                                       uint32_t n);
/* Device point arrays, points [first, first+n); any output may be NULL. */
CR_API cr_status cr_cloud_read_points(cr_cloud *cloud, uint64_t first, uint64_t n,
                                      uint32_t *xyz_low, uint32_t *xyz_med, uint32_t *xyz_high,
                                      uint32_t *colors, uint8_t *levels);
/* Cull output of the last frame that rendered this cloud (cloud.visibleBatchesBuffer):
 * count_out receives the survivor count; up to cap records are copied. */
CR_API cr_status cr_cloud_read_visible(cr_cloud *cloud, cr_visible_batch *out, uint32_t cap,
                                       uint32_t *count_out);

/* ------------------------------------------------------------------------ */
/* Frames: per-viewport device resources (ComputeRasteriser.swift:766-838)   */
/* ------------------------------------------------------------------------ */
CR_API cr_status cr_frame_create(cr_context *ctx, int width, int height, cr_frame **out);
CR_API cr_status cr_frame_destroy(cr_frame *frame);

/* One frame: ComputeRasteriser.update + encode (ComputeRasteriser.swift:201-296).
 * Uses each cloud's file table as last set by cr_cloud_update_files.
 *   HQS:     clear -> [cull] -> [depth] -> [colour] over all clouds, phase-major
 *            -> resolve -> hole fill (ComputeRasteriser.swift:322-456, 298-320)
 *   nearest: first cloud with resident batches only: clear winner -> cull ->
 *            nearest depth/index -> nearest resolve -> hole fill
 *            (ComputeRasteriser.swift:483-522) */
CR_API cr_status cr_render(cr_context *ctx, cr_frame *frame, cr_cloud *const *clouds,
                           uint32_t nclouds, const cr_config *config, const cr_camera *camera);

/* The HQS passes as stages, for a frame whose points are split over several
 * frames (one per GPU, each holding a part of the batches): every part runs
 * CR_STAGE_DEPTH; the depth planes are combined by an element-wise maximum
 * (an all-reduce); every part runs CR_STAGE_COLOR against the combined
 * depth; the R, G, B, count planes are summed; CR_STAGE_RESOLVE produces the
 * image.  Integer max and sum are order-independent, so the image is
 * bit-identical to one cr_render of all the batches.
 *   CR_STAGE_DEPTH    clear depth and accumulators, cull, depth pass
 *   CR_STAGE_COLOR    colour pass against the frame's depth plane
 *   CR_STAGE_RESOLVE  resolve and hole fill
 * The clouds, their file tables and the configuration must not change
 * between the stage calls of one frame (the depth stage leaves the cull
 * results and fragments in the clouds).  A colour stage whose resolve runs in
 * another call adds each field with a 32-bit add (exact up to 2^32 - 1 per
 * field), so that accumulators of several frames can be summed; one call
 * with both stages uses the packed adds of cr_render.  HQS only: separate
 * stages of the nearest mode return CR_ERR_UNSUPPORTED.  cr_render is
 * cr_render_stages(..., CR_STAGE_ALL).  No counterpart in the reference. */
typedef enum cr_stage {
    CR_STAGE_DEPTH = 1,
    CR_STAGE_COLOR = 2,
    CR_STAGE_RESOLVE = 4,
    CR_STAGE_ALL = 7
} cr_stage;
CR_API cr_status cr_render_stages(cr_context *ctx, cr_frame *frame, cr_cloud *const *clouds,
                                  uint32_t nclouds, const cr_config *config,
                                  const cr_camera *camera, uint32_t stages);

/* Device planes of a frame, for combining frames between stages with a
 * collective library: depth is `pixels` uint32 (reverse-Z, larger is
 * nearer), accum is `pixels` x {R, G, B, count} uint32.  `stream` is the
 * context's cudaStream_t; work on the planes must be ordered with it. */
typedef struct cr_frame_planes {
    void *depth;
    void *accum;
    uint64_t pixels;
    void *stream;
} cr_frame_planes;
CR_API cr_status cr_frame_device_planes(cr_frame *frame, cr_frame_planes *out);

/* XORs the top bit of every depth word (enqueued on the context stream):
 * maps the unsigned order of the depth plane onto the signed order of int32
 * and back, for collectives that reduce signed 32-bit integers only. */
CR_API cr_status cr_frame_flip_depth_order(cr_frame *frame);

/* Read-backs (synchronise the context stream). */
CR_API cr_status cr_frame_read_rgba8(cr_frame *frame, uint8_t *out /* w*h*4 */);
CR_API cr_status cr_frame_read_depth_f32(cr_frame *frame, float *out /* w*h */);
CR_API cr_status cr_frame_read_pixels(cr_frame *frame, cr_raster_pixel *out /* w*h */);
CR_API cr_status cr_frame_read_nearest_depth(cr_frame *frame, uint32_t *out /* w*h */);
CR_API cr_status cr_frame_read_nearest_index(cr_frame *frame, uint32_t *out /* w*h */);
/* Asynchronous read-back of the final RGBA8 image: enqueues its copy into
 * `out` (w*h*4 bytes; page-locked host memory keeps the copy asynchronous) on
 * the context's copy stream, after the work enqueued so far, and returns at
 * once.  The next render into the frame waits on the device for the copy
 * before it rewrites the image (at its resolve), so the copy overlaps that
 * render's cull, depth and colour passes.  `out` holds the image once
 * cr_frame_read_wait (or cr_context_synchronize) returns.  No counterpart in
 * the reference, whose output is a Metal texture the caller blits itself. */
CR_API cr_status cr_frame_read_rgba8_async(cr_frame *frame, uint8_t *out /* w*h*4 */);
/* Waits for the frame's enqueued asynchronous read-backs. */
CR_API cr_status cr_frame_read_wait(cr_frame *frame);
/* Waits until at most the `keep` most recent asynchronous read-backs of the
 * frame may still be in flight (keep 0..3; 0 is cr_frame_read_wait), so that
 * a render loop can use frame k's image while frame k+1's copy travels and
 * frame k+2 renders.  No counterpart in the reference. */
CR_API cr_status cr_frame_read_wait_keep(cr_frame *frame, int keep);
/* Rows [row0, row0+nrows) of the nearest index plane (pick band read-back). */
CR_API cr_status cr_frame_read_nearest_index_rows(cr_frame *frame, int row0, int nrows,
                                                  uint32_t *out);

/* pickPointIndex(atNDC:in:camera:searchRadius:) — ComputeRasteriser.swift:609-670.
 * Runs cull + nearest depth/index for one cloud into the frame's nearest
 * planes, reads back the band of rows within search_radius of the pixel
 * under ndc (y up) and returns the nearest non-sentinel pixel's point index.
 * found_out = 0 when nothing lies within the radius. */
CR_API cr_status cr_pick(cr_context *ctx, cr_frame *frame, cr_cloud *cloud, const float ndc[2],
                         const cr_config *config, const cr_camera *camera, int search_radius,
                         uint32_t *index_out, int *found_out);

/* ------------------------------------------------------------------------ */
/* GPU packer (GPUPacker, GPUPacker.swift:27-392)                            */
/* ------------------------------------------------------------------------ */
typedef enum cr_color_format {
    CR_COLOR_F32X4 = 0, /* RGBA float32 in [0,1] (the reference's float4 colour buffer) */
    CR_COLOR_RGBA8 = 1  /* packed uint32 r | g<<8 | b<<16 | a<<24                        */
} cr_color_format;

/* One run of raw points.  positions: x, y, z float32 at each stride (12 for
 * packed float3, 16 for the reference's 16-byte float3 or a 16-byte record);
 * colors: one colour per stride in colorFormat.  A 16-byte record
 * {float x, y, z; uint32 rgba8} is positions = rec, positionStrideBytes = 16,
 * colors = (char*)rec + 12, colorStrideBytes = 16, colorFormat = CR_COLOR_RGBA8. */
typedef struct cr_pack_input {
    const void *positions;
    uint32_t positionStrideBytes;
    const void *colors;
    uint32_t colorStrideBytes;
    int32_t colorFormat; /* cr_color_format */
} cr_pack_input;

/* GPUPacker.init(context:lodLevels:coarseVoxelDivisions:) (GPUPacker.swift:75-99). */
typedef struct cr_pack_params {
    int32_t lodLevels;            /* default 4, clamped to 1..8              */
    int32_t coarseVoxelDivisions; /* default 64, at least 1                  */
    int32_t mortonBits;           /* 10 = 30-bit keys (default), 21 = 63-bit */
} cr_pack_params;

CR_API cr_status cr_pack_params_default(cr_pack_params *out);

/* GPUPacker.pack(positions:colors:count:into:commandBuffer:) followed by the
 * completion-handler bounds adoption (GPUPacker.swift:140-160, replacePackedPointCloud
 * :507-519): the pool grows to ceil(count/pointsPerBatch) slots if needed,
 * slots [0, nb) are filled in Morton order with per-batch AABBs, LOD levels
 * and split-precision words, and every other slot is emptied.  inputs_on_device
 * = 1 when the pointers are device memory.  source_indices (optional, host,
 * count entries) receives the input index of every packed point (the
 * PackedPointCloud.sourceIndices permutation).  Synchronous. */
CR_API cr_status cr_pack(cr_context *ctx, cr_cloud *cloud, const cr_pack_input *input,
                         uint64_t count, const cr_pack_params *params, int inputs_on_device,
                         uint32_t *source_indices);

/* addRawChunksGPU(packer:queue:chunks:maxConcurrent:) (GPUPacker.swift:545-577):
 * each chunk with count > 0 takes the first run of ceil(count/pointsPerBatch)
 * contiguous free slots and is packed there, leaving every other slot
 * untouched; chunks without a free run are skipped.  first_slots (nchunks
 * entries) receives the first slot of each placed chunk in input order and
 * placed_out their number.  Synchronous. */
CR_API cr_status cr_pack_chunks(cr_context *ctx, cr_cloud *cloud, const cr_pack_input *chunks,
                                const uint64_t *counts, uint32_t nchunks,
                                const cr_pack_params *params, int inputs_on_device,
                                int32_t *first_slots, uint32_t *placed_out);

/* ------------------------------------------------------------------------ */
/* Device buffers and pinned host memory (for callers without a CUDA runtime) */
/* ------------------------------------------------------------------------ */
CR_API cr_status cr_buffer_create(cr_context *ctx, uint64_t bytes, void **device_ptr);
CR_API cr_status cr_buffer_destroy(cr_context *ctx, void *device_ptr);
/* Stream-ordered copies on the context stream, synchronised before return. */
CR_API cr_status cr_buffer_upload(cr_context *ctx, void *dst_device, const void *src_host,
                                  uint64_t bytes);
CR_API cr_status cr_buffer_download(cr_context *ctx, void *dst_host, const void *src_device,
                                    uint64_t bytes);
CR_API cr_status cr_host_alloc(uint64_t bytes, void **host_ptr);
CR_API cr_status cr_host_free(void *host_ptr);

/* ------------------------------------------------------------------------ */
/* Per-pass timing (the reference's labelled encoders, ComputeRasteriser.swift:379-428) */
/* ------------------------------------------------------------------------ */
typedef enum cr_pass_id {
    CR_PASS_CLEAR = 0,
    CR_PASS_CULL = 1,
    CR_PASS_DEPTH = 2,   /* HQS depth, or the fused nearest depth/index pass */
    CR_PASS_COLOR = 3,
    CR_PASS_RESOLVE = 4,
    CR_PASS_HOLE_FILL = 5,
    CR_PASS_COUNT = 6
} cr_pass_id;

/* When enabled, every cr_render brackets each pass (over all clouds) with
 * CUDA events on the context stream, in a ring of the last 256 frames.
 * Enabling or disabling synchronises the stream and empties the ring. */
CR_API cr_status cr_context_set_profiling(cr_context *ctx, int enable);
/* Device milliseconds per pass of the last min(nframes, recorded, 256)
 * profiled frames, oldest first: ms[k*CR_PASS_COUNT + pass] (0 for passes
 * that did not run).  frames_out receives the number of frames written.
 * Synchronises on the events it reads. */
CR_API cr_status cr_context_pass_times(cr_context *ctx, int32_t nframes, float *ms,
                                       int32_t *frames_out);

/* ------------------------------------------------------------------------ */
/* Launch tuning of the point passes                                         */
/* ------------------------------------------------------------------------ */
/* chunkPoints: survivor points per work record of the depth / colour /
 * nearest passes (>= 256); useTiles: accumulate compact batches in
 * shared-memory screen tiles.  Results do not depend on either value. */
typedef struct cr_tuning {
    int32_t chunkPoints;     /* default 2048 */
    int32_t useTiles;        /* default 1    */
    /* Batched views: the depth and colour passes run over groups of
     * consecutive views of at most this many pixels in all (a view larger
     * than the budget forms its own group), so that a group's fragments
     * stay in L2 between the two passes; 0 = all views in one group.
     * Default 4194304. */
    int32_t viewGroupPixels;
    /* Polls of a predecessor's published counts before a cull CTA gives up
     * (about 0.1 us each; default 1048576).  0 gives up at once: every cull
     * CTA after the first reports CR_ERR_TIMEOUT (a test of the error path;
     * nothing waits). */
    int32_t cullSpinLimit;
} cr_tuning;

CR_API cr_status cr_context_get_tuning(cr_context *ctx, cr_tuning *out);
CR_API cr_status cr_context_set_tuning(cr_context *ctx, const cr_tuning *tuning);

/* ------------------------------------------------------------------------ */
/* Synthetic workloads (seeded; a pure function of seed and point index)     */
/* ------------------------------------------------------------------------ */
/* Fractal heightfield: 2-D gradient noise summed over `octaves` with
 * `lacunarity` and `gain`, times `amplitude`; x, y uniform in [0, extent];
 * `outlierFraction` of the points uniform in z over the height range widened
 * by `outlierMargin`; colour = height ramp + N(0, colorNoiseSigma) per channel. */
typedef struct cr_synth_terrain {
    uint64_t seed;
    float extent;          /* 4000 m  */
    float amplitude;       /* 200 m   */
    float baseWavelength;  /* 1500 m  */
    int32_t octaves;       /* 6       */
    float lacunarity;      /* 2       */
    float gain;            /* 0.5     */
    float outlierFraction; /* 0.05    */
    float outlierMargin;   /* 50 m    */
    float colorNoiseSigma; /* 10      */
} cr_synth_terrain;

CR_API cr_status cr_synth_terrain_default(cr_synth_terrain *t);
/* Height of the noise surface at (x, y), evaluated on the host. */
CR_API float cr_synth_terrain_height(const cr_synth_terrain *t, float x, float y);
/* Points [first, first+count) as 16-byte records {x, y, z, rgba8} in device memory. */
CR_API cr_status cr_synth_terrain_points(cr_context *ctx, const cr_synth_terrain *t, uint64_t first,
                                         uint64_t count, void *device_records);
/* n_axis^3 lattice over [lo, hi]^3 with uniform jitter, uniform RGB8, alpha 255. */
CR_API cr_status cr_synth_lattice_points(cr_context *ctx, uint64_t seed, uint32_t n_axis, float lo,
                                         float hi, float jitter, void *device_records);

/* ------------------------------------------------------------------------ */
/* Differentiable colours                                                    */
/* ------------------------------------------------------------------------ */
/* An FP32 variant of the HQS colour pass with learnable per-point colours,
 * beside the unchanged integer path, and its adjoint (no counterpart in the
 * reference).  All arrays are device memory: colors and dL_dcolors hold 3
 * floats (R, G, B) per pool point of the cloud (cr_cloud_info.capacity
 * maxResidentBatches * pointsPerBatch), image and dL_dimage 3 floats per
 * pixel, row 0 at the top.  The cloud's file table must hold the camera's
 * transforms (cr_cloud_update_files), as for cr_render.
 *
 * cr_hqs_forward_f32: depth pass, then for every sample that passes the
 * colour pass's depth test (the integer path's visible set) the point's
 * colour is added to the pixel's FP32 R, G, B sums (reductions flush
 * subnormals) and one to its 32-bit count; image = sums / count, or the
 * background where the count is 0.  No hole fill.  One cloud.
 *
 * cr_hqs_backward_colors: for every point, recomputes its visible pixels
 * from the depth plane and counts the forward left in the frame and adds
 * sum over them of dL_dimage[pixel] / count[pixel] to dL_dcolors[point]
 * (per channel).  Call it after cr_hqs_forward_f32 with the same frame,
 * cloud, configuration and camera, before any other render of that cloud
 * or frame; gradients of several views accumulate.  One thread per point,
 * no atomics.
 *
 * cr_l2_loss: dL_dimage[i] = 2 * scale * (image[i] - target[i]) for n
 * floats; with loss non-NULL (host), *loss = scale * sum (image - target)^2,
 * accumulated in FP64, and the call synchronises.
 *
 * Asynchronous on the context's stream unless stated. */
CR_API cr_status cr_hqs_forward_f32(cr_context *ctx, cr_frame *frame, cr_cloud *cloud,
                                    const cr_config *config, const cr_camera *camera,
                                    const float *colors, float *image);
CR_API cr_status cr_hqs_backward_colors(cr_context *ctx, cr_frame *frame, cr_cloud *cloud,
                                        const cr_config *config, const cr_camera *camera,
                                        const float *dL_dimage, float *dL_dcolors);
CR_API cr_status cr_l2_loss(cr_context *ctx, const float *image, const float *target, uint64_t n,
                            float scale, float *dL_dimage, double *loss);

/* ------------------------------------------------------------------------ */
/* Batched views                                                             */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference, whose renderer draws one viewport per
 * ComputeRasteriser.encode (ComputeRasteriser.swift:277-296).  Renders
 * `nviews` (1..256) HQS views of the same clouds, view v with camera cams[v]
 * into frames[v] (distinct frames, any sizes), in one CUDA-graph launch: the
 * per-view cull, depth, colour, resolve and hole-fill work of all views runs
 * in shared launches.  models: nclouds column-major model matrices (the
 * ComputeRasteriserPointCloud.worldMatrix each cloud's file table is
 * multiplied by, as cr_cloud_update_files does), or NULL for identity.  Each
 * view's planes are bit-identical to cr_render of that view after
 * cr_cloud_update_files(cloud, projection * view, model, NULL, NULL).  The
 * graph is captured on the first call and whenever the frames, clouds,
 * configuration or tuning change; do not call it while capturing.
 * Asynchronous; the frames' read functions synchronise.  HQS only
 * (CR_ERR_UNSUPPORTED for the nearest mode); holeFillIterations <= 64. */
CR_API cr_status cr_render_multiview(cr_context *ctx, cr_frame *const *frames,
                                     const cr_camera *cams, uint32_t nviews,
                                     cr_cloud *const *clouds, const float *models,
                                     uint32_t nclouds, const cr_config *cfg);

/* Autotuner of cr_render_multiview's launch shape (no counterpart in the
 * reference): times 15 candidates of chunkPoints {1024, 2048, 4096} (points
 * per thread = chunkPoints / 256), screen tiles on / off and the view-group
 * budget viewGroupPixels {1, 2, 4, 8 Mpx, all}, `reps` renders each after
 * two warm-up renders, sets the fastest on the context and
 * returns it (and its ms per render).  With cache_path, a result is appended
 * to that file as one JSON object per line keyed by a workload signature
 * (device, SM count, views, pixels, points, configuration), and a later call
 * with the same signature reads it instead of timing.  Synchronises. */
CR_API cr_status cr_autotune_multiview(cr_context *ctx, cr_frame *const *frames,
                                       const cr_camera *cams, uint32_t nviews,
                                       cr_cloud *const *clouds, const float *models,
                                       uint32_t nclouds, const cr_config *cfg,
                                       const char *cache_path, int reps, cr_tuning *best,
                                       float *best_ms);

/* ------------------------------------------------------------------------ */
/* Allocation-free cull                                                      */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory — plug-ins whose host application owns every device allocation,
 * real-time loops that cannot take cudaMalloc's device-wide synchronisation
 * mid-frame — this runs the same ordered cull as cr_render on arrays the
 * caller owns: `batches` (nbatches slots), `files` (nfiles) and the outputs
 * `visible` (room for nbatches records) and `count` (one uint32) are device
 * pointers; config and camera are host structs; `stream` is a cudaStream_t
 * (NULL = the legacy default stream) the work is queued on.  It allocates
 * nothing: its scratch (one count per 256 slots) is a fixed array in the
 * library's device image, held by every GPU that loads the library until the
 * process exits, so at most 1,048,576 slots are accepted (CR_ERR_CAPACITY
 * above that).  The first call on a device looks up that array's address on
 * the current device; make it before any stream capture.  The pointers must
 * belong to the device that is current when the call is made, and the
 * address is kept for the life of the process, so after a reset of that
 * device (cudaDeviceReset) this entry point must not be called again.  All
 * calls share the array: calls whose work overlaps on the GPU race.
 * Asynchronous: the results are valid once the stream has reached them. */
CR_API cr_status cr_cull_noalloc(const cr_raster_batch *batches, uint32_t nbatches,
                                 const cr_raster_file *files, uint32_t nfiles,
                                 const cr_config *config, const cr_camera *camera, int width,
                                 int height, cr_visible_batch *visible, uint32_t *count,
                                 void *stream);

/* ------------------------------------------------------------------------ */
/* PLY input (PLYPointCloudLoader, PLYPointCloudLoader.swift:33-369)          */
/* ------------------------------------------------------------------------ */
/* Header of a PLY file: vertexCount vertices from bodyOffset, format 0 =
 * ascii, 1 = binary_little_endian, propertyCount vertex properties (stride
 * bytes per binary vertex), colorProperties of them red / green / blue. */
typedef struct cr_ply_header {
    uint64_t vertexCount;
    uint64_t bodyOffset;
    uint32_t format;
    uint32_t propertyCount;
    uint32_t stride;
    uint32_t colorProperties;
} cr_ply_header;

/* PLYPointCloudLoader.parse's header step (parseHeader, :171-240, and
 * PLYVertexLayout, :140-158).  Errors are CR_ERR_FORMAT with the reference's
 * PLYPointCloudLoaderError case as the detail (cr_last_error_detail):
 * invalidHeader, unsupportedFormat(f), missingVertexElement,
 * missingProperty(x, y, z), unsupportedProperty(p), truncatedBody (also when
 * the body cannot hold vertexCount vertices). */
CR_API cr_status cr_ply_read_header(const uint8_t *data, uint64_t size, cr_ply_header *out);

/* The vertices of a PLY file in memory as float4 positions (x, y, z, 1) and
 * float4 colours (r, g, b, 1 in [0, 1]; white without colour properties),
 * vertexCount of each: the inputs of cr_pack (16-byte position stride,
 * CR_COLOR_F32X4), as the reference's parseASCII / parseBinaryLittleEndian
 * (:242-305) hand them to PackedPointCloudFixtures.pack.  threads <= 0 uses
 * every host core; the result does not depend on it.  ASCII errors:
 * truncatedBody, invalidASCIIValue(line: n, property: p) for the first
 * failing vertex line. */
CR_API cr_status cr_ply_parse(const uint8_t *data, uint64_t size, int threads, float *positions,
                              float *colors);

/* A file mapped read-only into memory (the reference's Data(contentsOf:
 * options: .mappedIfSafe)); an empty file maps to (NULL, 0). */
CR_API cr_status cr_file_map(const char *path, const uint8_t **data, uint64_t *size);
CR_API cr_status cr_file_unmap(const uint8_t *data, uint64_t size);

#ifdef __cplusplus
} /* extern "C" */
#endif

/* Layout checks mirroring LayoutTests.swift:5-26. */
#ifdef __cplusplus
static_assert(sizeof(cr_raster_batch) == 64, "RasterBatch stride");
static_assert(offsetof(cr_raster_batch, state) == 0, "RasterBatch.state");
static_assert(offsetof(cr_raster_batch, minX) == 4, "RasterBatch.minX");
static_assert(offsetof(cr_raster_batch, maxZ) == 24, "RasterBatch.maxZ");
static_assert(offsetof(cr_raster_batch, numPoints) == 28, "RasterBatch.numPoints");
static_assert(offsetof(cr_raster_batch, firstPoint) == 32, "RasterBatch.firstPoint");
static_assert(offsetof(cr_raster_batch, fileIndex) == 36, "RasterBatch.fileIndex");
static_assert(sizeof(cr_raster_file) == 256, "RasterFile stride");
static_assert(sizeof(cr_raster_pixel) == 32, "RasterPixel stride");
static_assert(sizeof(cr_visible_batch) == 16, "VisibleBatch stride");
static_assert(sizeof(cr_dispatch_args) == 12, "CRDispatchArgs stride");
#else
_Static_assert(sizeof(cr_raster_batch) == 64, "RasterBatch stride");
_Static_assert(offsetof(cr_raster_batch, state) == 0, "RasterBatch.state");
_Static_assert(offsetof(cr_raster_batch, minX) == 4, "RasterBatch.minX");
_Static_assert(offsetof(cr_raster_batch, maxZ) == 24, "RasterBatch.maxZ");
_Static_assert(offsetof(cr_raster_batch, numPoints) == 28, "RasterBatch.numPoints");
_Static_assert(offsetof(cr_raster_batch, firstPoint) == 32, "RasterBatch.firstPoint");
_Static_assert(offsetof(cr_raster_batch, fileIndex) == 36, "RasterBatch.fileIndex");
_Static_assert(sizeof(cr_raster_file) == 256, "RasterFile stride");
_Static_assert(sizeof(cr_raster_pixel) == 32, "RasterPixel stride");
_Static_assert(sizeof(cr_visible_batch) == 16, "VisibleBatch stride");
_Static_assert(sizeof(cr_dispatch_args) == 12, "CRDispatchArgs stride");
#endif

#endif /* CR_CR_H */
