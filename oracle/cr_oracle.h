/*
 * cr_oracle.h — CPU oracle for the point-cloud compute rasteriser.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a single-threaded C++ restatement of
 * the reference's pass semantics (Swift CPU code and Metal shaders of
 * Satin-ComputeRasteriser), used by the tests, by the smoke check and as the
 * timed CPU baseline of the bench.  The product library never links it.
 *
 * Numeric contract (both the oracle and the CUDA kernels obey it):
 *   N1 no FMA contraction: every +,-,* is rounded on its own; a matrix times
 *      a vector is ((c0*x + c1*y) + c2*z) + c3*w per row; a 4x4 product sums
 *      k = 0..3 left to right.
 *   N2 IEEE-rounded division and square root.
 *   N3 float->int conversions truncate toward zero, saturate at the type's
 *      range and map NaN to 0 (the GPU's cvt.rzi behaviour).
 *   N4 depthToUintReverseZ(1.0) saturates to 0xFFFFFFFF.
 *   N5 log2 is the project-written cr_log2f below on both sides.
 *   N6 unorm8 writes are rint(clamp(f*255, 0, 255)) (round half to even).
 *   N7 min/max follow fmaxf/fminf (a NaN operand yields the other operand).
 * Compiled with -O2 -ffp-contract=off -fno-fast-math.
 */
#ifndef CR_ORACLE_H
#define CR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Restatement of ComputeRasteriserTypes.h:11-57 (layouts are checked by the tests). */
typedef struct orc_batch {
    int32_t state;
    float minX, minY, minZ, maxX, maxY, maxZ;
    uint32_t numPoints, firstPoint, fileIndex;
    uint32_t lodCum01, lodCum23, lodCum45, lodCum67, padding7, padding8;
} orc_batch;

typedef struct orc_file {
    float transform[16], transformFrustum[16], world[16], prevTransform[16];
} orc_file;

typedef struct orc_visible {
    uint32_t batchIndex;
    int32_t level;
    float lodThreshold;
    uint32_t activePoints;
} orc_visible;

/* The fields of ComputeRasteriserConfiguration that reach the passes. */
typedef struct orc_config {
    int32_t mode; /* 0 HQS, 1 nearest */
    float depthTolerance;
    float backgroundColor[4];
    int32_t enableFrustumCulling, lodBias, enableCLOD, enableLODDither;
    int32_t holeFillIterations, colorizeChunks, colorizeOverdraw, pointSizeMode;
    float minimumPointSize, maximumPointSize, pointSizeScale;
    /* Colour variants (ColorPass/Shaders.metal:54-199, DepthPass/Shaders.metal:56-71,
     * Resolve/Shaders.metal:19-41); all off by default. */
    int32_t applyDisplacement, applyTint, tintAlphaIsCoverage;
    float motionBlur;
    int32_t motionBlurSamples;
    float motionBlurMaxSpread;
} orc_config;

/* One cloud's slot pool as the device holds it. */
typedef struct orc_cloud {
    const orc_batch *batches;
    uint32_t batchCount; /* = maxResidentBatches (slots scanned by cull) */
    const orc_file *files;
    uint32_t fileCount;
    const uint32_t *xyzLow, *xyzMed, *xyzHigh, *colors;
    const uint8_t *levels;
    /* Per-point float4 attributes of the colour variants (NULL reads zeros):
     * displacement (xyz), the previous frame's displacement (motion blur;
     * NULL uses the current one), tint (rgba). */
    const float *displacements, *prevDisplacements, *tints;
} orc_cloud;

/* ---- scalar helpers exposed for tests ---- */
float orc_log2f(float x);
float orc_exp_neg(float x);
float orc_hash_unit(uint32_t x);
uint32_t orc_depth_to_uint(float ndcz);
void orc_mat4_mul(const float a[16], const float b[16], float out[16]);

/* updateFiles (ComputeRasteriserPointCloud.swift:487-515). base: the cloud's
 * file table (world matrices); out receives the per-frame snapshot. */
void orc_update_files(const orc_file *base, uint32_t n, const float vp[16], const float model[16],
                      const float *frustum, const float *prev_vp, orc_file *out);

/* cullUpdate (Cull/Shaders.metal:19-83) with the survivors in ascending slot
 * order.  Returns the survivor count; writes at most cap records. */
uint32_t orc_cull(const orc_cloud *cloud, const orc_config *cfg, const float view[16],
                  const float proj[16], int width, int height, orc_visible *out, uint32_t cap);

/* Full frame, ComputeRasteriser.encode (ComputeRasteriser.swift:277-553).
 * Outputs (any may be NULL):
 *   depth[w*h]        HQS depth plane (RasterPixel.depth)
 *   accum[w*h*4]      HQS red, green, blue, count per pixel
 *   ndepth[w*h]       nearest depth plane; nindex[w*h] nearest index plane
 *   rgba[w*h*4]       final RGBA8 image after hole fill
 *   depthf[w*h]       resolve R32F depth
 *   visible / visible_count: per-cloud cull lists, cloud c at visible + c*visible_stride
 * threads: 1 = single-threaded oracle; >1 splits the point passes over threads
 * (integer atomics, identical results). Returns 0 on success. */
int orc_render(const orc_cloud *clouds, uint32_t nclouds, const orc_config *cfg,
               const float view[16], const float proj[16], int width, int height,
               uint32_t *depth, uint32_t *accum, uint32_t *ndepth, uint32_t *nindex,
               uint8_t *rgba, float *depthf, orc_visible *visible, uint32_t visible_stride,
               uint32_t *visible_count, int threads);

/* One HQS stage of a frame whose points are split over several frames:
 * stage 1 = clear depth[w*h] and accum[w*h*4], cull, depth pass; 2 = cull and
 * colour pass against depth[], added into accum[]; 4 = resolve depth[] and
 * accum[] and hole fill into rgba / depthf (either may be NULL).  The
 * clouds' resident batches are the part drawn.  Returns 0 on success. */
int orc_hqs_stage(const orc_cloud *clouds, uint32_t nclouds, const orc_config *cfg,
                  const float view[16], const float proj[16], int width, int height,
                  uint32_t stage, uint32_t *depth, uint32_t *accum, uint8_t *rgba,
                  float *depthf, int threads);

/* Differentiable HQS colours in FP64 for one view of one cloud (reference of
 * the FP32 forward / adjoint): colors and grad hold 3 doubles per pool point,
 * target and image 3 per pixel (row 0 = top).  loss, grad and fd are added
 * to; fd[k*3+c] = central difference (step fd_h) of the loss in channel c
 * of point fd_points[k].  Any output may be NULL. */
int orc_hqs_grad_f64(const orc_cloud *cloud, const orc_config *cfg, const float view[16],
                     const float proj[16], int width, int height, const double *colors,
                     const double *target, double scale, double *image, double *loss,
                     double *grad, const uint32_t *fd_points, uint32_t n_fd, double fd_h,
                     double *fd, int threads);

/* holeFillUpdate ping-pong (HoleFill/Shaders.metal:10-48, ComputeRasteriser.swift:298-320). */
void orc_hole_fill(uint8_t *rgba, int width, int height, int iterations);

/* NearestPointCPUReference.render (NearestPointCPUReference.swift:16-81), literally:
 * every batch, optional frustum test, precision level, every point, radius 0. */
void orc_nearest_cpu_reference(const orc_cloud *cloud, int width, int height, const float view[16],
                               const float proj[16], int enable_frustum, uint32_t *depths,
                               uint32_t *indices);

/* pickPointIndex band scan (ComputeRasteriser.swift:615-669) over a full index plane. */
int orc_pick_scan(const uint32_t *nindex, int width, int height, const float ndc[2], int radius,
                  uint32_t *out);

/* PackedPointCloudFixtures.pack (PackedPointCloudFixtures.swift:30-167).
 * Input: positions xyz (stride 3 floats) and either colors_f32 (RGBA, stride 4)
 * or colors_rgba8 (already packed).  morton_bits: 10 (the reference's 30-bit
 * key) or 21 (63-bit key).  Outputs sized by the caller: nb = ceil(n/ppb)
 * batches; n entries for every per-point array; bounds[6] = min xyz, max xyz. */
int orc_pack(const float *positions, const float *colors_f32, const uint32_t *colors_rgba8,
             uint64_t n, uint32_t points_per_batch, int lod_levels, int coarse_voxel_divisions,
             int morton_bits, orc_batch *batches, uint32_t *xyz_low, uint32_t *xyz_med,
             uint32_t *xyz_high, uint32_t *colors, uint8_t *levels, uint32_t *source_indices,
             float *ordered_positions, float *bounds);

/* The same pack on `threads` host threads, bit-identical to orc_pack: a
 * stable LSD radix sort (contiguous per-thread ranges, digit-major then
 * thread-major offsets), the LOD claims as a minimum point index per voxel
 * in a concurrent table (the first unassigned point of a voxel in sorted
 * order is its minimum index), and the per-batch steps split by batch.
 * source_indices, ordered_positions and bounds may be NULL. */
int orc_pack_threads(const float *positions, const float *colors_f32,
                     const uint32_t *colors_rgba8, uint64_t n, uint32_t points_per_batch,
                     int lod_levels, int coarse_voxel_divisions, int morton_bits,
                     orc_batch *batches, uint32_t *xyz_low, uint32_t *xyz_med, uint32_t *xyz_high,
                     uint32_t *colors, uint8_t *levels, uint32_t *source_indices,
                     float *ordered_positions, float *bounds, int threads);

/* Seeded synthetic clouds (host restatement of the library's generators,
 * bit-identical records {float x, y, z; uint32 rgba8}). */
typedef struct orc_terrain {
    uint64_t seed;
    float extent, amplitude, baseWavelength;
    int32_t octaves;
    float lacunarity, gain, outlierFraction, outlierMargin, colorNoiseSigma;
} orc_terrain;
float orc_terrain_height(const orc_terrain *t, float x, float y);
int orc_synth_terrain(const orc_terrain *t, uint64_t first, uint64_t count, float *records,
                      int threads);
int orc_synth_lattice(uint64_t seed, uint32_t n_axis, float lo, float hi, float jitter,
                      float *records, int threads);
float orc_ln_unit(float u);
float orc_cos_2pi(float u);

#ifdef __cplusplus
}
#endif
#endif
