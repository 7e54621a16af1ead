// cr_oracle.cpp — CPU oracle (test infrastructure; see cr_oracle.h).
//
// Each function cites the reference file:line it restates.  Paths are
// relative to the Satin-ComputeRasteriser package root; shader files live in
// Sources/SatinComputeRasteriser/Pipelines/, Swift files in
// Sources/SatinComputeRasteriser/.
#include "cr_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// Scalar numeric contract
// ---------------------------------------------------------------------------

inline float fmax_(float a, float b) { return std::fmax(a, b); }
inline float fmin_(float a, float b) { return std::fmin(a, b); }
inline float clampf_(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
inline float saturate_(float x) { return clampf_(x, 0.0f, 1.0f); }

// float -> int32 / uint32 truncating, saturating, NaN -> 0 (N3).
inline int32_t f2i(float x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}
inline uint32_t f2u(float x) {
    if (std::isnan(x) || x <= 0.0f) return 0u;
    if (x >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)x;
}
inline float u2f(uint32_t x) { return (float)x; }  // round to nearest even

struct f3 { float x, y, z; };
struct f4 { float x, y, z, w; };

// M * v for a column-major 4x4 (N1).
inline f4 mulv(const float *m, f4 v) {
    f4 r;
    r.x = ((m[0] * v.x + m[4] * v.y) + m[8] * v.z) + m[12] * v.w;
    r.y = ((m[1] * v.x + m[5] * v.y) + m[9] * v.z) + m[13] * v.w;
    r.z = ((m[2] * v.x + m[6] * v.y) + m[10] * v.z) + m[14] * v.w;
    r.w = ((m[3] * v.x + m[7] * v.y) + m[11] * v.z) + m[15] * v.w;
    return r;
}

inline void mat4mul(const float *a, const float *b, float *out) {
    float r[16];
    for (int c = 0; c < 4; ++c)
        for (int row = 0; row < 4; ++row)
            r[c * 4 + row] = ((a[0 * 4 + row] * b[c * 4 + 0] + a[1 * 4 + row] * b[c * 4 + 1]) +
                              a[2 * 4 + row] * b[c * 4 + 2]) +
                             a[3 * 4 + row] * b[c * 4 + 3];
    std::memcpy(out, r, sizeof(r));
}

// Project-written log2 (N5): x = m * 2^e with m in [sqrt(1/2), sqrt(2)),
// s = (m-1)/(m+1), ln(m) = 2 atanh(s) summed as the odd Taylor series of
// atanh through s^11 (Abramowitz & Stegun 4.1.27), log2 = e + ln(m)/ln(2).
float log2_contract(float x) {
    if (std::isnan(x)) return x;
    if (x < 0.0f) return std::numeric_limits<float>::quiet_NaN();
    if (x == 0.0f) return -std::numeric_limits<float>::infinity();
    if (std::isinf(x)) return x;
    uint32_t bits;
    std::memcpy(&bits, &x, 4);
    int e = (int)((bits >> 23) & 0xffu);
    if (e == 0) {  // subnormal: scale by 2^23 exactly
        float y = x * 8388608.0f;
        std::memcpy(&bits, &y, 4);
        e = (int)((bits >> 23) & 0xffu) - 23;
    }
    e -= 127;
    uint32_t mbits = (bits & 0x007fffffu) | 0x3f800000u;
    float m;
    std::memcpy(&m, &mbits, 4);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float s2 = s * s;
    float p = 0.0909090936f;      // 1/11
    p = p * s2 + 0.111111112f;    // 1/9
    p = p * s2 + 0.142857149f;    // 1/7
    p = p * s2 + 0.200000003f;    // 1/5
    p = p * s2 + 0.333333343f;    // 1/3
    p = p * s2 + 1.0f;
    const float t = s * p;        // atanh(s)
    const float l = t * 2.88539008f;  // 2/ln(2)
    return (float)e + l;
}

// ---------------------------------------------------------------------------
// Common.metal restatements
// ---------------------------------------------------------------------------

// depthToUintReverseZ / uintToDepthReverseZ (Common.metal:10-16).  The constant
// float(CR_MAX_DEPTH - 1u) rounds to 4294967296.0f.
// e^-x for x >= 0 (the coverage resolve's alpha), written for this project:
// Cody-Waite range reduction (Cody and Waite, Software Manual for the
// Elementary Functions, 1980): n = floor(x log2 e), r = (x - n ln2_hi) -
// n ln2_lo with ln2_hi exact in 15 bits, so n ln2_hi is exact; e^-r by its
// Taylor series to degree 9 (Horner, every operation rounded); an exact
// power-of-two scale 2^-n.  The kernels evaluate the same operations.
inline float exp_neg(float x) {
    if (x != x) return x;
    if (!(x > 0.0f)) return 1.0f;
    const float t = x * 1.44269504f;
    if (t >= 126.0f) return 0.0f;
    const float n = std::floor(t);
    const float r = (x - n * 0.693145751953125f) - n * 1.42860682e-06f;
    const float z = 0.0f - r;
    float p = 2.75573192e-06f;
    p = p * z + 2.48015873e-05f;
    p = p * z + 1.98412698e-04f;
    p = p * z + 1.38888889e-03f;
    p = p * z + 8.33333333e-03f;
    p = p * z + 4.16666667e-02f;
    p = p * z + 1.66666667e-01f;
    p = p * z + 0.5f;
    p = p * z + 1.0f;
    p = p * z + 1.0f;
    uint32_t bits = (uint32_t)(127 - (int)n) << 23;
    float scale;
    std::memcpy(&scale, &bits, 4);
    return p * scale;
}

inline uint32_t depth_to_uint(float z) { return f2u(saturate_(z) * 4294967296.0f); }
inline float uint_to_depth(uint32_t d) { return u2f(d) / 4294967296.0f; }

// hashUnit (Common.metal:190-197).
inline float hash_unit(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return u2f(x) * (1.0f / 4294967296.0f);
}

// pointFootprintRadius (Common.metal:18-61).
int footprint_radius(f3 point, const orc_file &file, const float *view, const float *proj,
                     int sw, int sh, const orc_config &cfg) {
    (void)sw;
    const f4 wp4 = mulv(file.world, f4{point.x, point.y, point.z, 1.0f});
    const f4 vp = mulv(view, f4{wp4.x, wp4.y, wp4.z, 1.0f});
    const float mn = cfg.minimumPointSize, mx = cfg.maximumPointSize;
    const float lo = fmax_(fmin_(mn, mx), 1.0f);
    const float hi = fmax_(fmax_(mn, mx), lo);
    const bool ortho = (proj[15] == 1.0f);
    float ps;
    if (cfg.pointSizeMode == 1) {
        const float focal = ((float)sh * 0.5f) * proj[5];
        if (ortho) {
            ps = (2.0f * cfg.pointSizeScale) * focal;
        } else {
            const float viewZ = fmax_(-vp.z, 0.000001f);
            ps = ((2.0f * cfg.pointSizeScale) * focal) / viewZ;
        }
    } else {
        if (ortho) {
            ps = cfg.pointSizeScale;
        } else {
            const float len = std::sqrt((vp.x * vp.x + vp.y * vp.y) + vp.z * vp.z);
            const float dist = fmax_(len, 0.000001f);
            ps = cfg.pointSizeScale / dist;
        }
    }
    if (!std::isfinite(ps)) ps = lo;
    ps = clampf_(ps, lo, hi);
    const int r = f2i(std::ceil(fmax_(ps - 1.0f, 0.0f) * 0.5f));
    return std::min(std::max(r, 0), 16);
}

// insidePointFootprint (Common.metal:63-71).
inline bool inside_footprint(int ox, int oy, int radius) {
    if (radius <= 0) return ox == 0 && oy == 0;
    const float px = (float)ox, py = (float)oy;
    const float r = (float)radius + 0.5f;
    return (px * px + py * py) <= r * r;
}

// decodePoint (Common.metal:89-117), batchSize (:81-83).
inline f3 decode_point(uint32_t i, const orc_batch &b, const orc_cloud &c, int level) {
    const float sx = fmax_(b.maxX - b.minX, 0.000001f);
    const float sy = fmax_(b.maxY - b.minY, 0.000001f);
    const float sz = fmax_(b.maxZ - b.minZ, 0.000001f);
    uint32_t x, y, z;
    float steps;
    const uint32_t lo = c.xyzLow[i];
    if (level == 0) {
        const uint32_t me = c.xyzMed[i], hi = c.xyzHigh[i];
        x = (((lo >> 0) & 1023u) << 20) | (((me >> 0) & 1023u) << 10) | ((hi >> 0) & 1023u);
        y = (((lo >> 10) & 1023u) << 20) | (((me >> 10) & 1023u) << 10) | ((hi >> 10) & 1023u);
        z = (((lo >> 20) & 1023u) << 20) | (((me >> 20) & 1023u) << 10) | ((hi >> 20) & 1023u);
        steps = 1073741824.0f;
    } else if (level == 1) {
        const uint32_t me = c.xyzMed[i];
        x = (((lo >> 0) & 1023u) << 10) | ((me >> 0) & 1023u);
        y = (((lo >> 10) & 1023u) << 10) | ((me >> 10) & 1023u);
        z = (((lo >> 20) & 1023u) << 10) | ((me >> 20) & 1023u);
        steps = 1048576.0f;
    } else {
        x = lo & 1023u;
        y = (lo >> 10) & 1023u;
        z = (lo >> 20) & 1023u;
        steps = 1024.0f;
    }
    const float qx = sx / steps, qy = sy / steps, qz = sz / steps;
    return f3{u2f(x) * qx + b.minX, u2f(y) * qy + b.minY, u2f(z) * qz + b.minZ};
}

struct plane { float nx, ny, nz, off; };

// makePlane (Common.metal:119-125).
inline plane make_plane(float x, float y, float z, float w) {
    const float len = fmax_(std::sqrt((x * x + y * y) + z * z), 0.000001f);
    return plane{x / len, y / len, z / len, w / len};
}

// intersectsFrustum (Common.metal:127-153); m[col*4+row].
bool intersects_frustum(const float *m, f3 mn, f3 mx) {
    auto M = [&](int c, int r) { return m[c * 4 + r]; };
    const plane planes[6] = {
        make_plane(M(0, 3) - M(0, 0), M(1, 3) - M(1, 0), M(2, 3) - M(2, 0), M(3, 3) - M(3, 0)),
        make_plane(M(0, 3) + M(0, 0), M(1, 3) + M(1, 0), M(2, 3) + M(2, 0), M(3, 3) + M(3, 0)),
        make_plane(M(0, 3) + M(0, 1), M(1, 3) + M(1, 1), M(2, 3) + M(2, 1), M(3, 3) + M(3, 1)),
        make_plane(M(0, 3) - M(0, 1), M(1, 3) - M(1, 1), M(2, 3) - M(2, 1), M(3, 3) - M(3, 1)),
        make_plane(M(0, 3) - M(0, 2), M(1, 3) - M(1, 2), M(2, 3) - M(2, 2), M(3, 3) - M(3, 2)),
        make_plane(M(0, 2), M(1, 2), M(2, 2), M(3, 2)),
    };
    for (int i = 0; i < 6; ++i) {
        const plane &p = planes[i];
        const float px = p.nx > 0.0f ? mx.x : mn.x;
        const float py = p.ny > 0.0f ? mx.y : mn.y;
        const float pz = p.nz > 0.0f ? mx.z : mn.z;
        if (((p.nx * px + p.ny * py) + p.nz * pz) + p.off < 0.0f) return false;
    }
    return true;
}

// pixelSizeOnScreen (Common.metal:155-170).
float pixel_size_on_screen(const orc_batch &b, const orc_file &file, const float *view,
                           const float *proj, int sw, int sh) {
    const f3 mn{b.minX, b.minY, b.minZ}, mx{b.maxX, b.maxY, b.maxZ};
    const f3 c{(mn.x + mx.x) * 0.5f, (mn.y + mx.y) * 0.5f, (mn.z + mx.z) * 0.5f};
    const float dx = mn.x - mx.x, dy = mn.y - mx.y, dz = mn.z - mx.z;
    const float radius = std::sqrt((dx * dx + dy * dy) + dz * dz);
    float vw[16];
    mat4mul(view, file.world, vw);
    const f4 vc = mulv(vw, f4{c.x, c.y, c.z, 1.0f});
    const f4 ve{vc.x + radius, vc.y + 0.0f, vc.z + 0.0f, vc.w + 0.0f};
    f4 pc = mulv(proj, vc);
    f4 pe = mulv(proj, ve);
    const float wc = fmax_(std::fabs(pc.w), 0.000001f);
    pc.x = pc.x / wc;
    pc.y = pc.y / wc;
    const float we = fmax_(std::fabs(pe.w), 0.000001f);
    pe.x = pe.x / we;
    pe.y = pe.y / we;
    const float W = (float)sw, H = (float)sh;
    const float scx = (W * (pc.x + 1.0f)) * 0.5f, scy = (H * (pc.y + 1.0f)) * 0.5f;
    const float sex = (W * (pe.x + 1.0f)) * 0.5f, sey = (H * (pe.y + 1.0f)) * 0.5f;
    const float ex = sex - scx, ey = sey - scy;
    return std::sqrt(ex * ex + ey * ey);
}

// precisionLevel thresholds (Common.metal:172-181, Cull/Shaders.metal:48-53).
inline int precision_level(float px) {
    if (px < 100.0f) return 4;
    if (px < 200.0f) return 3;
    if (px < 500.0f) return 2;
    if (px < 10000.0f) return 1;
    return 0;
}

// ---------------------------------------------------------------------------
// Cull (Cull/Shaders.metal:19-83), ordered.
// ---------------------------------------------------------------------------
bool cull_one(const orc_cloud &c, uint32_t gid, const orc_config &cfg, const float *view,
              const float *proj, int sw, int sh, orc_visible &out) {
    const orc_batch &b = c.batches[gid];
    if (b.state == 0) return false;
    const orc_file &file = c.files[b.fileIndex];
    if (cfg.enableFrustumCulling != 0) {
        if (!intersects_frustum(file.transformFrustum, f3{b.minX, b.minY, b.minZ},
                                f3{b.maxX, b.maxY, b.maxZ}))
            return false;
    }
    const float px = pixel_size_on_screen(b, file, view, proj, sw, sh);
    const int level = precision_level(px);
    // lodThresholdFromPixelSize (Common.metal:185-187): log2(max(px,1)/25) + 3 + bias.
    const float thr = (cfg.enableCLOD != 0)
                          ? fmax_(0.0f, (log2_contract(fmax_(px, 1.0f) / 25.0f) + 3.0f) +
                                            (float)cfg.lodBias)
                          : 99.0f;
    uint32_t active = b.numPoints;
    if (b.lodCum67 != 0u) {
        const int lmax = std::min(std::max(f2i(std::floor(thr + 0.5f)), 0), 7);
        const uint32_t words[4] = {b.lodCum01, b.lodCum23, b.lodCum45, b.lodCum67};
        const uint32_t word = words[lmax >> 1];
        active = (lmax & 1) ? (word >> 16) : (word & 0xffffu);
        active = std::min(active, b.numPoints);  // malformed counts stay inside the slot
    }
    if (active == 0u) return false;
    out.batchIndex = gid;
    out.level = level;
    out.lodThreshold = thr;
    out.activePoints = active;
    return true;
}

// ---------------------------------------------------------------------------
// Point traversal shared by depth / colour / nearest passes
// (DepthPass/Shaders.metal:58-115, ColorPass/Shaders.metal:58-93,
//  NearestDepth/Shaders.metal:56-90, NearestIndex/Shaders.metal:56-93).
// ---------------------------------------------------------------------------
struct projected {
    int px, py;     // pixel after the y flip
    float ndcz;
    uint32_t depth;
    int radius;
};

// Returns true when the point survives the dither, clip and screen tests.
// reject_z_le_zero: nearest passes reject ndc.z <= 0, HQS rejects ndc.z < 0.
inline bool project(const orc_cloud &c, const orc_batch &b, const orc_file &file,
                    const orc_visible &vb, uint32_t pointIndex, const orc_config &cfg,
                    const float *view, const float *proj, int sw, int sh, bool reject_z_le_zero,
                    projected &out) {
    const float pointLevel = u2f((uint32_t)c.levels[pointIndex] & 7u);
    const float dither = (cfg.enableLODDither != 0) ? hash_unit(pointIndex) : 0.5f;
    if (dither >= (vb.lodThreshold - pointLevel) + 0.5f) return false;
    const f3 p = decode_point(pointIndex, b, c, vb.level);
    const f4 clip = mulv(file.transform, f4{p.x, p.y, p.z, 1.0f});
    if (clip.w <= 0.0f) return false;
    const float nx = clip.x / clip.w, ny = clip.y / clip.w, nz = clip.z / clip.w;
    if (nx < -1.0f || ny < -1.0f || nx > 1.0f || ny > 1.0f) return false;
    if (reject_z_le_zero ? (nz <= 0.0f) : (nz < 0.0f)) return false;
    if (nz > 1.0f) return false;
    int px = f2i((nx * 0.5f + 0.5f) * (float)sw);
    int py = f2i((ny * 0.5f + 0.5f) * (float)sh);
    if (px < 0 || px >= sw || py < 0 || py >= sh) return false;
    py = sh - 1 - py;
    out.px = px;
    out.py = py;
    out.ndcz = nz;
    out.depth = depth_to_uint(nz);
    out.radius = footprint_radius(p, file, view, proj, sw, sh, cfg);
    return true;
}

inline void atomic_max_u32(uint32_t *p, uint32_t v, bool mt) {
    if (!mt) {
        if (v > *p) *p = v;
        return;
    }
    uint32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    while (v > cur &&
           !__atomic_compare_exchange_n(p, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
}
inline void atomic_min_u32(uint32_t *p, uint32_t v, bool mt) {
    if (!mt) {
        if (v < *p) *p = v;
        return;
    }
    uint32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    while (v < cur &&
           !__atomic_compare_exchange_n(p, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
}
inline void atomic_add_u32(uint32_t *p, uint32_t v, bool mt) {
    if (!mt)
        *p += v;
    else
        __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}

enum pass_kind { PASS_DEPTH, PASS_COLOR, PASS_NEAREST_DEPTH, PASS_NEAREST_INDEX };

struct pass_args {
    const orc_cloud *cloud;
    const orc_visible *vis;
    uint32_t nvis;
    const orc_config *cfg;
    const float *view, *proj;
    int sw, sh;
    uint32_t *depth;  // HQS depth plane or nearest depth plane
    uint32_t *accum;  // HQS r,g,b,count
    uint32_t *index;  // nearest index plane
    bool variant = false;  // HQS colour variants on (run_batch_variant)
};

inline float saturate_nan0(float x) { return fmin_(fmax_(x, 0.0f), 1.0f); }  // NaN -> 0

inline f4 attr(const float *a, uint32_t i) {
    if (!a) return f4{0.0f, 0.0f, 0.0f, 0.0f};
    return f4{a[4 * (size_t)i], a[4 * (size_t)i + 1], a[4 * (size_t)i + 2], a[4 * (size_t)i + 3]};
}

// The depth and colour passes with the colour variants on: displacement
// (DepthPass/Shaders.metal:63-71, ColorPass/Shaders.metal:70-77), tint mix and
// discard (ColorPass :116-140, DepthPass :56-60), coverage / motion-blur
// weighted-blended accumulation without a depth test, fixed point S = 4096
// (ColorPass :109-199).  One point at a time in the reference's order.
void run_batch_variant(const pass_args &a, pass_kind kind, uint32_t v, bool mt) {
    const orc_cloud &c = *a.cloud;
    const orc_visible &vb = a.vis[v];
    const orc_batch &b = c.batches[vb.batchIndex];
    const orc_file &file = c.files[b.fileIndex];
    const orc_config &cfg = *a.cfg;
    const int sw = a.sw, sh = a.sh;
    const bool coverage_mode = cfg.applyTint != 0 && cfg.tintAlphaIsCoverage != 0;
    const bool mb_on = cfg.motionBlur > 0.0f;
    const bool oit = coverage_mode || mb_on;
    for (uint32_t local = 0; local < vb.activePoints; ++local) {
        const uint32_t pi = b.firstPoint + local;
        const float pointLevel = u2f((uint32_t)c.levels[pi] & 7u);
        const float dither = (cfg.enableLODDither != 0) ? hash_unit(pi) : 0.5f;
        if (dither >= (vb.lodThreshold - pointLevel) + 0.5f) continue;
        if (kind == PASS_DEPTH && coverage_mode && attr(c.tints, pi).w < 0.0f) continue;
        const f3 base = decode_point(pi, b, c, vb.level);
        f3 p = base;
        if (cfg.applyDisplacement != 0) {
            const f4 d = attr(c.displacements, pi);
            p = f3{p.x + d.x, p.y + d.y, p.z + d.z};
            if (p.x != p.x || p.y != p.y || p.z != p.z) continue;
        }
        const f4 clip = mulv(file.transform, f4{p.x, p.y, p.z, 1.0f});
        if (clip.w <= 0.0f) continue;
        const float nx = clip.x / clip.w, ny = clip.y / clip.w, nz = clip.z / clip.w;
        if (nx < -1.0f || ny < -1.0f || nx > 1.0f || ny > 1.0f || nz < 0.0f || nz > 1.0f) continue;
        int px = f2i((nx * 0.5f + 0.5f) * (float)sw);
        int py = f2i((ny * 0.5f + 0.5f) * (float)sh);
        if (px < 0 || px >= sw || py < 0 || py >= sh) continue;
        py = sh - 1 - py;
        if (kind == PASS_DEPTH) {
            const uint32_t depth = depth_to_uint(nz);
            const int rad = footprint_radius(p, file, a.view, a.proj, sw, sh, cfg);
            for (int oy = -rad; oy <= rad; ++oy)
                for (int ox = -rad; ox <= rad; ++ox) {
                    if (!inside_footprint(ox, oy, rad)) continue;
                    const int tx = px + ox, ty = py + oy;
                    if (tx < 0 || tx >= sw || ty < 0 || ty >= sh) continue;
                    atomic_max_u32(&a.depth[(uint32_t)(ty * sw + tx)], depth, mt);
                }
            continue;
        }
        uint32_t color = c.colors[pi];
        if (cfg.colorizeChunks != 0)
            color = vb.batchIndex * 1234567u;
        else if (cfg.colorizeOverdraw != 0)
            color = 0x00010101u;
        uint32_t r = color & 0xffu, g = (color >> 8) & 0xffu, bl = (color >> 16) & 0xffu;
        float cov = 1.0f;
        if (cfg.applyTint != 0) {
            const f4 t = attr(c.tints, pi);
            if (t.w < 0.0f) continue;
            if (coverage_mode) {
                cov = saturate_nan0(1.0f - t.w);
            } else {
                const float w = saturate_nan0(t.w);
                const float k = 1.0f / 255.0f;
                const float ox = u2f(r) * k, oy = u2f(g) * k, oz = u2f(bl) * k;
                const float mx = ox + (saturate_nan0(t.x) - ox) * w;  // mix(orig, tint, w)
                const float my = oy + (saturate_nan0(t.y) - oy) * w;
                const float mz = oz + (saturate_nan0(t.z) - oz) * w;
                r = f2u(saturate_nan0(mx) * 255.0f + 0.5f);
                g = f2u(saturate_nan0(my) * 255.0f + 0.5f);
                bl = f2u(saturate_nan0(mz) * 255.0f + 0.5f);
            }
        }
        if (oit && cov <= 0.0f) continue;
        const int rad = footprint_radius(p, file, a.view, a.proj, sw, sh, cfg);
        int samples = 1;
        float stepx = 0.0f, stepy = 0.0f;
        if (mb_on) {
            f3 pp = base;
            if (cfg.applyDisplacement != 0) {
                const f4 d = attr(c.prevDisplacements ? c.prevDisplacements : c.displacements, pi);
                pp = f3{pp.x + d.x, pp.y + d.y, pp.z + d.z};
            }
            const f4 pc = mulv(file.prevTransform, f4{pp.x, pp.y, pp.z, 1.0f});
            if (pc.w > 0.0f) {
                const float pnx = pc.x / pc.w, pny = pc.y / pc.w;
                const int ppx = f2i((pnx * 0.5f + 0.5f) * (float)sw);
                const int ppy = sh - 1 - f2i((pny * 0.5f + 0.5f) * (float)sh);
                float vx = (float)((int64_t)px - (int64_t)ppx) * cfg.motionBlur;
                float vy = (float)((int64_t)py - (int64_t)ppy) * cfg.motionBlur;
                float len = std::sqrt(vx * vx + vy * vy);
                if (len > cfg.motionBlurMaxSpread) {
                    const float k = cfg.motionBlurMaxSpread / len;
                    vx = vx * k;
                    vy = vy * k;
                    len = cfg.motionBlurMaxSpread;
                }
                if (len > 0.75f) {
                    samples = std::min(std::max(f2i(std::ceil(len)), 1), cfg.motionBlurSamples);
                    samples = std::max(samples, 1);
                    const float den = (float)std::max(samples - 1, 1);
                    stepx = vx / den;
                    stepy = vy / den;
                }
            }
        }
        const float aN = cov / (float)samples;
        const float kS = 4096.0f, k255 = 1.0f / 255.0f;
        const uint32_t caR = f2u(((u2f(r) * k255) * aN) * kS + 0.5f);
        const uint32_t caG = f2u(((u2f(g) * k255) * aN) * kS + 0.5f);
        const uint32_t caB = f2u(((u2f(bl) * k255) * aN) * kS + 0.5f);
        const uint32_t caA = f2u(aN * kS + 0.5f);
        for (int s = 0; s < samples; ++s) {
            const int cx = px - f2i(std::round(stepx * (float)s));
            const int cy = py - f2i(std::round(stepy * (float)s));
            for (int oy = -rad; oy <= rad; ++oy)
                for (int ox = -rad; ox <= rad; ++ox) {
                    if (!inside_footprint(ox, oy, rad)) continue;
                    const int tx = cx + ox, ty = cy + oy;
                    if (tx < 0 || tx >= sw || ty < 0 || ty >= sh) continue;
                    const uint32_t pix = (uint32_t)(ty * sw + tx);
                    if (oit) {
                        atomic_add_u32(&a.accum[pix * 4 + 0], caR, mt);
                        atomic_add_u32(&a.accum[pix * 4 + 1], caG, mt);
                        atomic_add_u32(&a.accum[pix * 4 + 2], caB, mt);
                        atomic_add_u32(&a.accum[pix * 4 + 3], caA, mt);
                        continue;
                    }
                    const uint32_t closest = a.depth[pix];
                    if (closest == 0u) continue;
                    if (!(nz >= uint_to_depth(closest) * (1.0f - cfg.depthTolerance))) continue;
                    atomic_add_u32(&a.accum[pix * 4 + 0], r, mt);
                    atomic_add_u32(&a.accum[pix * 4 + 1], g, mt);
                    atomic_add_u32(&a.accum[pix * 4 + 2], bl, mt);
                    atomic_add_u32(&a.accum[pix * 4 + 3], 1u, mt);
                }
        }
    }
}

void run_batch(const pass_args &a, pass_kind kind, uint32_t v, bool mt) {
    if (a.variant) {
        run_batch_variant(a, kind, v, mt);
        return;
    }
    const orc_cloud &c = *a.cloud;
    const orc_visible &vb = a.vis[v];
    const orc_batch &b = c.batches[vb.batchIndex];
    const orc_file &file = c.files[b.fileIndex];
    const orc_config &cfg = *a.cfg;
    const bool nearest = (kind == PASS_NEAREST_DEPTH || kind == PASS_NEAREST_INDEX);
    for (uint32_t local = 0; local < vb.activePoints; ++local) {
        const uint32_t pointIndex = b.firstPoint + local;
        projected pr;
        if (!project(c, b, file, vb, pointIndex, cfg, a.view, a.proj, a.sw, a.sh, nearest, pr))
            continue;
        uint32_t r = 0, g = 0, bl = 0;
        if (kind == PASS_COLOR) {
            // ColorPass/Shaders.metal:95-104.
            uint32_t color = c.colors[pointIndex];
            if (cfg.colorizeChunks != 0)
                color = vb.batchIndex * 1234567u;
            else if (cfg.colorizeOverdraw != 0)
                color = 0x00010101u;
            r = color & 0xffu;
            g = (color >> 8) & 0xffu;
            bl = (color >> 16) & 0xffu;
        }
        const int rad = pr.radius;
        for (int oy = -rad; oy <= rad; ++oy) {
            for (int ox = -rad; ox <= rad; ++ox) {
                if (!inside_footprint(ox, oy, rad)) continue;
                const int tx = pr.px + ox, ty = pr.py + oy;
                if (tx < 0 || tx >= a.sw || ty < 0 || ty >= a.sh) continue;
                const uint32_t pix = (uint32_t)(ty * a.sw + tx);
                switch (kind) {
                case PASS_DEPTH:
                case PASS_NEAREST_DEPTH:
                    atomic_max_u32(&a.depth[pix], pr.depth, mt);
                    break;
                case PASS_COLOR: {
                    // ColorPass/Shaders.metal:201-214 (integer path).
                    const uint32_t closest = a.depth[pix];
                    if (closest == 0u) break;
                    const float closestDepth = uint_to_depth(closest);
                    if (!(pr.ndcz >= closestDepth * (1.0f - cfg.depthTolerance))) break;
                    atomic_add_u32(&a.accum[pix * 4 + 0], r, mt);
                    atomic_add_u32(&a.accum[pix * 4 + 1], g, mt);
                    atomic_add_u32(&a.accum[pix * 4 + 2], bl, mt);
                    atomic_add_u32(&a.accum[pix * 4 + 3], 1u, mt);
                    break;
                }
                case PASS_NEAREST_INDEX:
                    // NearestIndex/Shaders.metal:88-90.
                    if (pr.depth == a.depth[pix]) atomic_min_u32(&a.index[pix], pointIndex, mt);
                    break;
                }
            }
        }
    }
}

void run_pass(const pass_args &a, pass_kind kind, int threads) {
    if (threads <= 1 || a.nvis < 2) {
        for (uint32_t v = 0; v < a.nvis; ++v) run_batch(a, kind, v, false);
        return;
    }
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        pool.emplace_back([&]() {
            for (;;) {
                const uint32_t v = next.fetch_add(1);
                if (v >= a.nvis) break;
                run_batch(a, kind, v, true);
            }
        });
    }
    for (auto &th : pool) th.join();
}

// unorm8 texture write (N6).
inline uint8_t unorm8(float f) {
    const float x = clampf_(f * 255.0f, 0.0f, 255.0f);
    return (uint8_t)std::nearbyint(x);
}

// resolveUpdate (Resolve/Shaders.metal:13-57), count path.
void resolve_hqs(const uint32_t *depth, const uint32_t *accum, size_t npix, const float *bg,
                 uint8_t *img, float *dimg) {
    for (size_t p = 0; p < npix; ++p) {
        const uint32_t cnt = accum[p * 4 + 3];
        uint8_t *o = &img[p * 4];
        if (cnt == 0u) {
            o[0] = unorm8(bg[0]);
            o[1] = unorm8(bg[1]);
            o[2] = unorm8(bg[2]);
            o[3] = unorm8(0.0f);
            dimg[p] = 0.0f;
            continue;
        }
        const float inv = 1.0f / u2f(cnt);
        o[0] = unorm8((u2f(accum[p * 4 + 0]) * inv) / 255.0f);
        o[1] = unorm8((u2f(accum[p * 4 + 1]) * inv) / 255.0f);
        o[2] = unorm8((u2f(accum[p * 4 + 2]) * inv) / 255.0f);
        o[3] = unorm8(1.0f);
        dimg[p] = uint_to_depth(depth[p]);
    }
}

// resolveUpdate with coverageEnabled (Resolve/Shaders.metal:24-41): the
// weighted-blended average and alpha 1 - e^-(sum of alpha).
void resolve_coverage(const uint32_t *depth, const uint32_t *accum, size_t npix, const float *bg,
                      uint8_t *img, float *dimg) {
    for (size_t p = 0; p < npix; ++p) {
        const uint32_t a = accum[p * 4 + 3];
        uint8_t *o = &img[p * 4];
        if (a == 0u) {
            o[0] = unorm8(bg[0]);
            o[1] = unorm8(bg[1]);
            o[2] = unorm8(bg[2]);
            o[3] = unorm8(0.0f);
            dimg[p] = 0.0f;
            continue;
        }
        const float fa = u2f(a);
        o[0] = unorm8(u2f(accum[p * 4 + 0]) / fa);
        o[1] = unorm8(u2f(accum[p * 4 + 1]) / fa);
        o[2] = unorm8(u2f(accum[p * 4 + 2]) / fa);
        const float sum_a = fa * (1.0f / 4096.0f);
        o[3] = unorm8(saturate_nan0(1.0f - exp_neg(sum_a)));
        dimg[p] = uint_to_depth(depth[p]);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Exported API
// ---------------------------------------------------------------------------
extern "C" {

float orc_log2f(float x) { return log2_contract(x); }
float orc_exp_neg(float x) { return exp_neg(x); }
float orc_hash_unit(uint32_t x) { return hash_unit(x); }
uint32_t orc_depth_to_uint(float z) { return depth_to_uint(z); }
void orc_mat4_mul(const float a[16], const float b[16], float out[16]) { mat4mul(a, b, out); }

// updateFiles (ComputeRasteriserPointCloud.swift:493-504).
void orc_update_files(const orc_file *base, uint32_t n, const float vp[16], const float model[16],
                      const float *frustum, const float *prev_vp, orc_file *out) {
    for (uint32_t i = 0; i < n; ++i) {
        orc_file s = base[i];
        float world[16];
        mat4mul(model, base[i].world, world);
        mat4mul(vp, world, s.transform);
        mat4mul(frustum ? frustum : vp, world, s.transformFrustum);
        std::memcpy(s.world, world, sizeof(world));
        mat4mul(prev_vp ? prev_vp : vp, world, s.prevTransform);
        out[i] = s;
    }
}

uint32_t orc_cull(const orc_cloud *cloud, const orc_config *cfg, const float view[16],
                  const float proj[16], int width, int height, orc_visible *out, uint32_t cap) {
    uint32_t n = 0;
    for (uint32_t gid = 0; gid < cloud->batchCount; ++gid) {
        orc_visible v;
        if (cull_one(*cloud, gid, *cfg, view, proj, width, height, v)) {
            if (n < cap) out[n] = v;
            ++n;
        }
    }
    return n;
}

void orc_hole_fill(uint8_t *rgba, int w, int h, int iterations) {
    if (iterations <= 0 || w <= 0 || h <= 0) return;
    std::vector<uint8_t> src(rgba, rgba + (size_t)w * h * 4), dst(src.size());
    auto rd = [&](const std::vector<uint8_t> &img, int x, int y, int ch) {
        return u2f(img[((size_t)y * w + x) * 4 + ch]) / 255.0f;
    };
    for (int it = 0; it < iterations; ++it) {
        for (int y = 0; y < h; ++y) {
            for (int x = 0; x < w; ++x) {
                const size_t o = ((size_t)y * w + x) * 4;
                // HoleFill/Shaders.metal:21-47.
                if (rd(src, x, y, 3) >= 0.5f) {
                    std::memcpy(&dst[o], &src[o], 4);
                    continue;
                }
                float sr = 0.0f, sg = 0.0f, sb = 0.0f, cnt = 0.0f;
                for (int oy = -1; oy <= 1; ++oy) {
                    for (int ox = -1; ox <= 1; ++ox) {
                        if (ox == 0 && oy == 0) continue;
                        const int sx = x + ox, sy = y + oy;
                        if (sx < 0 || sx >= w || sy < 0 || sy >= h) continue;
                        if (rd(src, sx, sy, 3) >= 0.5f) {
                            sr = sr + rd(src, sx, sy, 0);
                            sg = sg + rd(src, sx, sy, 1);
                            sb = sb + rd(src, sx, sy, 2);
                            cnt = cnt + 1.0f;
                        }
                    }
                }
                if (cnt > 0.0f) {
                    dst[o + 0] = unorm8(sr / cnt);
                    dst[o + 1] = unorm8(sg / cnt);
                    dst[o + 2] = unorm8(sb / cnt);
                    dst[o + 3] = unorm8(1.0f);
                } else {
                    std::memcpy(&dst[o], &src[o], 4);
                }
            }
        }
        std::swap(src, dst);
    }
    std::memcpy(rgba, src.data(), src.size());
}

int orc_render(const orc_cloud *clouds, uint32_t nclouds, const orc_config *cfg,
               const float view[16], const float proj[16], int w, int h, uint32_t *depth_out,
               uint32_t *accum_out, uint32_t *ndepth_out, uint32_t *nindex_out, uint8_t *rgba,
               float *depthf, orc_visible *visible, uint32_t visible_stride,
               uint32_t *visible_count, int threads) {
    if (w <= 0 || h <= 0) return 1;
    const size_t npix = (size_t)w * h;
    std::vector<uint32_t> vcount(nclouds, 0);
    std::vector<std::vector<orc_visible>> vis(nclouds);
    // Resident clouds: at least one slot with state != 0 (residentBatchCount > 0).
    auto resident = [&](const orc_cloud &c) {
        for (uint32_t i = 0; i < c.batchCount; ++i)
            if (c.batches[i].state != 0) return true;
        return false;
    };
    auto cull_cloud = [&](uint32_t ci) {
        const orc_cloud &c = clouds[ci];
        vis[ci].resize(c.batchCount);
        vcount[ci] = orc_cull(&c, cfg, view, proj, w, h, vis[ci].data(), c.batchCount);
        vis[ci].resize(vcount[ci]);
    };

    std::vector<uint8_t> img(npix * 4);
    std::vector<float> dimg(npix, 0.0f);
    const float *bg = cfg->backgroundColor;

    if (cfg->mode == 0) {
        // encodeHighQualityAverage (ComputeRasteriser.swift:322-456): clear, then
        // cull / depth / colour phase-major over every resident cloud, then resolve.
        std::vector<uint32_t> depth(npix, 0u), accum(npix * 4, 0u);
        std::vector<uint32_t> order;
        for (uint32_t ci = 0; ci < nclouds; ++ci)
            if (resident(clouds[ci])) order.push_back(ci);
        for (uint32_t ci : order) cull_cloud(ci);
        // Colour variants (ComputeRasteriser.swift:229-253): coverage resolve
        // when translucent defocus or motion blur is on.
        const bool variant =
            cfg->applyDisplacement != 0 || cfg->applyTint != 0 || cfg->motionBlur > 0.0f;
        const bool coverage =
            (cfg->applyTint != 0 && cfg->tintAlphaIsCoverage != 0) || cfg->motionBlur > 0.0f;
        for (uint32_t ci : order) {
            pass_args a{&clouds[ci], vis[ci].data(), vcount[ci], cfg, view, proj, w, h,
                        depth.data(), accum.data(), nullptr};
            a.variant = variant;
            run_pass(a, PASS_DEPTH, threads);
        }
        for (uint32_t ci : order) {
            pass_args a{&clouds[ci], vis[ci].data(), vcount[ci], cfg, view, proj, w, h,
                        depth.data(), accum.data(), nullptr};
            a.variant = variant;
            run_pass(a, PASS_COLOR, threads);
        }
        if (coverage)
            resolve_coverage(depth.data(), accum.data(), npix, bg, img.data(), dimg.data());
        else
            resolve_hqs(depth.data(), accum.data(), npix, bg, img.data(), dimg.data());
        if (depth_out) std::memcpy(depth_out, depth.data(), npix * 4);
        if (accum_out) std::memcpy(accum_out, accum.data(), npix * 16);
    } else {
        // encodeNearestPoint (ComputeRasteriser.swift:483-522): first resident cloud.
        int first = -1;
        for (uint32_t ci = 0; ci < nclouds; ++ci)
            if (resident(clouds[ci])) {
                first = (int)ci;
                break;
            }
        if (first < 0) {
            // No resident cloud: the reference returns before any pass, leaving
            // the output untouched.  The oracle reports that with return code 2.
            if (visible_count)
                for (uint32_t ci = 0; ci < nclouds; ++ci) visible_count[ci] = 0;
            return 2;
        }
        std::vector<uint32_t> nd(npix, 0u), ni(npix, 0xffffffffu);  // clearWinnerUpdate
        cull_cloud((uint32_t)first);
        pass_args a{&clouds[first], vis[first].data(), vcount[first], cfg, view, proj, w, h,
                    nd.data(), nullptr, ni.data()};
        run_pass(a, PASS_NEAREST_DEPTH, threads);
        run_pass(a, PASS_NEAREST_INDEX, threads);
        // nearestResolveUpdate (NearestResolve/Shaders.metal:8-38).
        const uint32_t *colors = clouds[first].colors;
        for (size_t p = 0; p < npix; ++p) {
            uint8_t *o = &img[p * 4];
            if (nd[p] == 0u || ni[p] == 0xffffffffu) {
                o[0] = unorm8(bg[0]);
                o[1] = unorm8(bg[1]);
                o[2] = unorm8(bg[2]);
                o[3] = unorm8(0.0f);
                dimg[p] = 0.0f;
                continue;
            }
            const uint32_t c = colors[ni[p]];
            o[0] = unorm8(u2f(c & 0xffu) / 255.0f);
            o[1] = unorm8(u2f((c >> 8) & 0xffu) / 255.0f);
            o[2] = unorm8(u2f((c >> 16) & 0xffu) / 255.0f);
            o[3] = unorm8(1.0f);
            dimg[p] = uint_to_depth(nd[p]);
        }
        if (ndepth_out) std::memcpy(ndepth_out, nd.data(), npix * 4);
        if (nindex_out) std::memcpy(nindex_out, ni.data(), npix * 4);
    }
    orc_hole_fill(img.data(), w, h, cfg->holeFillIterations);
    if (rgba) std::memcpy(rgba, img.data(), npix * 4);
    if (depthf) std::memcpy(depthf, dimg.data(), npix * 4);
    if (visible_count)
        for (uint32_t ci = 0; ci < nclouds; ++ci) visible_count[ci] = vcount[ci];
    if (visible)
        for (uint32_t ci = 0; ci < nclouds; ++ci)
            for (uint32_t k = 0; k < vcount[ci] && k < visible_stride; ++k)
                visible[(size_t)ci * visible_stride + k] = vis[ci][k];
    return 0;
}

// One HQS stage of a frame split by points (cr_render_stages), in the order
// of encodeHighQualityAverage (ComputeRasteriser.swift:322-456): stage 1
// clears both planes, culls and runs the depth pass of every resident cloud;
// stage 2 culls and adds the colour pass of every resident cloud, tested
// against the given depth plane; stage 4 resolves the planes and hole-fills.
int orc_hqs_stage(const orc_cloud *clouds, uint32_t nclouds, const orc_config *cfg,
                  const float view[16], const float proj[16], int w, int h, uint32_t stage,
                  uint32_t *depth, uint32_t *accum, uint8_t *rgba, float *depthf, int threads) {
    if (w <= 0 || h <= 0 || cfg->mode != 0) return 1;
    const size_t npix = (size_t)w * h;
    auto resident = [&](const orc_cloud &c) {
        for (uint32_t i = 0; i < c.batchCount; ++i)
            if (c.batches[i].state != 0) return true;
        return false;
    };
    if (stage == 1 || stage == 2) {
        if (stage == 1) {
            std::fill(depth, depth + npix, 0u);
            std::fill(accum, accum + npix * 4, 0u);
        }
        for (uint32_t ci = 0; ci < nclouds; ++ci) {
            const orc_cloud &c = clouds[ci];
            if (!resident(c)) continue;
            std::vector<orc_visible> vis(c.batchCount);
            const uint32_t n = orc_cull(&c, cfg, view, proj, w, h, vis.data(), c.batchCount);
            pass_args a{&c, vis.data(), n, cfg, view, proj, w, h, depth, accum, nullptr};
            run_pass(a, stage == 1 ? PASS_DEPTH : PASS_COLOR, threads);
        }
        return 0;
    }
    if (stage != 4) return 1;
    std::vector<uint8_t> img(npix * 4);
    std::vector<float> dimg(npix, 0.0f);
    resolve_hqs(depth, accum, npix, cfg->backgroundColor, img.data(), dimg.data());
    orc_hole_fill(img.data(), w, h, cfg->holeFillIterations);
    if (rgba) std::memcpy(rgba, img.data(), npix * 4);
    if (depthf) std::memcpy(depthf, dimg.data(), npix * 4);
    return 0;
}

// Differentiable HQS colours in FP64 (reference for the FP32 path).  One
// view of one cloud: the HQS depth pass, then per-pixel FP64 sums of the
// learnable colours of the points that pass the colour pass's depth test
// (ColorPass/Shaders.metal:201-214, the same visible set as the integer
// path) and their count; image = sum / count (background where count = 0);
// loss = scale * sum over pixels and channels of (image - target)^2.
// Gradient: dL/dcolor_i = sum over the pixels p where point i is visible of
// 2 * scale * (image_p - target_p) / count_p.  Central differences: for
// each listed point and channel, the loss at colour +- h, evaluated over
// the loss terms that the point's colour changes (the pixels where it is
// visible), divided by 2h.  Multi-threaded over visible batches with
// per-thread planes; deterministic (per-thread planes are summed in order).
// grad and fd are added to (several views accumulate).
int orc_hqs_grad_f64(const orc_cloud *cloud, const orc_config *cfg, const float view[16],
                     const float proj[16], int w, int h, const double *colors,
                     const double *target, double scale, double *image, double *loss,
                     double *grad, const uint32_t *fd_points, uint32_t n_fd, double fd_h,
                     double *fd, int threads) {
    if (w <= 0 || h <= 0) return 1;
    const size_t npix = (size_t)w * h;
    const orc_cloud &c = *cloud;
    std::vector<orc_visible> vis(c.batchCount);
    const uint32_t nvis = orc_cull(&c, cfg, view, proj, w, h, vis.data(), c.batchCount);
    std::vector<uint32_t> depth(npix, 0u);
    pass_args a{&c, vis.data(), nvis, cfg, view, proj, w, h, depth.data(), nullptr, nullptr};
    run_pass(a, PASS_DEPTH, threads);
    const float keep = 1.0f - cfg->depthTolerance;
    // Calls f(pointIndex, pixel) for every (point, footprint pixel) that the
    // colour pass accumulates, batches [v0, v1).
    auto visit = [&](uint32_t v0, uint32_t v1, auto &&f) {
        for (uint32_t v = v0; v < v1; ++v) {
            const orc_visible &vb = vis[v];
            const orc_batch &b = c.batches[vb.batchIndex];
            const orc_file &file = c.files[b.fileIndex];
            for (uint32_t local = 0; local < vb.activePoints; ++local) {
                const uint32_t pi = b.firstPoint + local;
                projected pr;
                if (!project(c, b, file, vb, pi, *cfg, view, proj, w, h, false, pr)) continue;
                const int rad = pr.radius;
                for (int oy = -rad; oy <= rad; ++oy)
                    for (int ox = -rad; ox <= rad; ++ox) {
                        if (!inside_footprint(ox, oy, rad)) continue;
                        const int tx = pr.px + ox, ty = pr.py + oy;
                        if (tx < 0 || tx >= w || ty < 0 || ty >= h) continue;
                        const uint32_t pix = (uint32_t)(ty * w + tx);
                        const uint32_t closest = depth[pix];
                        if (closest == 0u) continue;
                        if (!(pr.ndcz >= uint_to_depth(closest) * keep)) continue;
                        f(pi, pix);
                    }
            }
        }
    };
    const int nt = std::max(1, std::min(threads, (int)std::max(nvis, 1u)));
    std::vector<std::vector<double>> sums(nt, std::vector<double>(npix * 3, 0.0));
    std::vector<std::vector<uint32_t>> counts(nt, std::vector<uint32_t>(npix, 0u));
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&, t]() {
                const uint32_t v0 = (uint32_t)((uint64_t)nvis * t / nt);
                const uint32_t v1 = (uint32_t)((uint64_t)nvis * (t + 1) / nt);
                visit(v0, v1, [&](uint32_t pi, uint32_t pix) {
                    for (int ch = 0; ch < 3; ++ch) sums[t][pix * 3 + ch] += colors[pi * 3 + ch];
                    counts[t][pix] += 1u;
                });
            });
        for (auto &th : pool) th.join();
    }
    std::vector<double> img(npix * 3), dl(npix * 3);
    std::vector<uint32_t> cnt(npix, 0u);
    double L = 0.0;
    for (size_t p = 0; p < npix; ++p) {
        for (int t = 0; t < nt; ++t) cnt[p] += counts[t][p];
        for (int ch = 0; ch < 3; ++ch) {
            double s = 0.0;
            for (int t = 0; t < nt; ++t) s += sums[t][p * 3 + ch];
            const double v = cnt[p] ? s / (double)cnt[p] : (double)cfg->backgroundColor[ch];
            img[p * 3 + ch] = v;
            const double d = v - target[p * 3 + ch];
            L += scale * d * d;
            dl[p * 3 + ch] = cnt[p] ? 2.0 * scale * d : 0.0;
        }
    }
    if (image) std::memcpy(image, img.data(), npix * 3 * sizeof(double));
    if (loss) *loss += L;
    std::vector<char> listed;
    std::vector<uint32_t> slot;
    if (fd && n_fd) {
        uint32_t maxp = 0;
        for (uint32_t k = 0; k < n_fd; ++k) maxp = std::max(maxp, fd_points[k]);
        listed.assign((size_t)maxp + 1, 0);
        slot.assign((size_t)maxp + 1, 0u);
        for (uint32_t k = 0; k < n_fd; ++k) {
            listed[fd_points[k]] = 1;
            slot[fd_points[k]] = k;
        }
    }
    visit(0, nvis, [&](uint32_t pi, uint32_t pix) {
        const double n = (double)cnt[pix];
        if (grad)
            for (int ch = 0; ch < 3; ++ch) grad[pi * 3 + ch] += dl[pix * 3 + ch] / n;
        if (fd && pi < listed.size() && listed[pi]) {
            for (int ch = 0; ch < 3; ++ch) {
                const double t = target[pix * 3 + ch], v = img[pix * 3 + ch];
                const double up = v + fd_h / n - t, dn = v - fd_h / n - t;
                fd[slot[pi] * 3 + ch] += scale * (up * up - dn * dn) / (2.0 * fd_h);
            }
        }
    });
    return 0;
}

// NearestPointCPUReference.render (NearestPointCPUReference.swift:16-81).
void orc_nearest_cpu_reference(const orc_cloud *cloud, int w, int h, const float view[16],
                               const float proj[16], int enable_frustum, uint32_t *depths,
                               uint32_t *indices) {
    const size_t npix = (size_t)std::max(w, 0) * (size_t)std::max(h, 0);
    for (size_t p = 0; p < npix; ++p) {
        depths[p] = 0u;
        indices[p] = 0xffffffffu;
    }
    if (w <= 0 || h <= 0) return;
    const orc_cloud &c = *cloud;
    for (uint32_t bi = 0; bi < c.batchCount; ++bi) {
        const orc_batch &b = c.batches[bi];
        const orc_file &file = c.files[b.fileIndex];
        if (enable_frustum &&
            !intersects_frustum(file.transformFrustum, f3{b.minX, b.minY, b.minZ},
                                f3{b.maxX, b.maxY, b.maxZ}))
            continue;
        const int level = precision_level(pixel_size_on_screen(b, file, view, proj, w, h));
        for (uint32_t local = 0; local < b.numPoints; ++local) {
            const uint32_t pi = b.firstPoint + local;
            const f3 p = decode_point(pi, b, c, level);
            const f4 clip = mulv(file.transform, f4{p.x, p.y, p.z, 1.0f});
            if (clip.w <= 0.0f) continue;
            const float nx = clip.x / clip.w, ny = clip.y / clip.w, nz = clip.z / clip.w;
            if (nx < -1.0f || nx > 1.0f || ny < -1.0f || ny > 1.0f || nz <= 0.0f || nz > 1.0f)
                continue;
            int px = f2i((nx * 0.5f + 0.5f) * (float)w);
            int py = f2i((ny * 0.5f + 0.5f) * (float)h);
            if (px < 0 || px >= w || py < 0 || py >= h) continue;
            py = h - 1 - py;
            const size_t pix = (size_t)py * w + px;
            const uint32_t d = depth_to_uint(nz);
            if (d > depths[pix]) {
                depths[pix] = d;
                indices[pix] = pi;
            } else if (d == depths[pix]) {
                indices[pix] = std::min(indices[pix], pi);
            }
        }
    }
}

// pickPointIndex read-back scan (ComputeRasteriser.swift:615-669).
int orc_pick_scan(const uint32_t *nindex, int w, int h, const float ndc[2], int radius,
                  uint32_t *out) {
    if (w <= 0 || h <= 0) return 0;
    const int px = std::min(std::max(f2i((ndc[0] * 0.5f + 0.5f) * (float)w), 0), w - 1);
    const int pyb = f2i((ndc[1] * 0.5f + 0.5f) * (float)h);
    const int py = std::min(std::max(h - 1 - pyb, 0), h - 1);
    const int r = std::max(0, radius);
    const int row0 = std::max(0, py - r), row1 = std::min(h - 1, py + r);
    long best_d = -1;
    uint32_t best = 0;
    const long r2 = (long)r * r;
    for (int y = row0; y <= row1; ++y) {
        const long dy = y - py;
        for (int x = std::max(0, px - r); x <= std::min(w - 1, px + r); ++x) {
            const long dx = x - px;
            const long d = dx * dx + dy * dy;
            if (d > r2 || (best_d >= 0 && d >= best_d)) continue;
            const uint32_t v = nindex[(size_t)y * w + x];
            if (v != 0xffffffffu) {
                best_d = d;
                best = v;
            }
        }
    }
    if (best_d < 0) return 0;
    *out = best;
    return 1;
}

}  // extern "C"
