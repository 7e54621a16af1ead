// cr_device.cuh — device-side pass math of the compute rasteriser.
//
// Every function restates one helper of the reference's shader library
// (Sources/SatinComputeRasteriser/Pipelines/Common.metal) under the numeric
// contract the CPU oracle also follows: the library is compiled with
// -fmad=false (no FMA contraction), IEEE division and square root, and a
// fixed left-to-right operation order.  float->int casts compile to
// cvt.rzi (truncate, saturate, NaN -> 0) and uint->float to cvt.rn.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cr/cr.h"

namespace crd {

// Programmatic dependent launch (sm_90+).  A kernel launched with
// programmatic stream serialisation may start while the kernel before it on
// the stream is still running; grid_wait() blocks until that kernel has
// completed and its memory is visible (a no-op for a normal launch), so
// every kernel calls it before touching memory the previous one writes.
// launch_dependents() lets the next kernel's launch begin.
__device__ __forceinline__ void grid_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

struct f3 {
    float x, y, z;
};
struct f4 {
    float x, y, z, w;
};

// M * v for a column-major 4x4: ((c0*x + c1*y) + c2*z) + c3*w per row.
__device__ __forceinline__ f4 mulv(const float *m, f4 v) {
    f4 r;
    r.x = ((m[0] * v.x + m[4] * v.y) + m[8] * v.z) + m[12] * v.w;
    r.y = ((m[1] * v.x + m[5] * v.y) + m[9] * v.z) + m[13] * v.w;
    r.z = ((m[2] * v.x + m[6] * v.y) + m[10] * v.z) + m[14] * v.w;
    r.w = ((m[3] * v.x + m[7] * v.y) + m[11] * v.z) + m[15] * v.w;
    return r;
}

// M * (p, 1): the w = 1 column enters as c3 * 1.
__device__ __forceinline__ f4 mulp(const float *m, float x, float y, float z) {
    f4 r;
    r.x = ((m[0] * x + m[4] * y) + m[8] * z) + m[12] * 1.0f;
    r.y = ((m[1] * x + m[5] * y) + m[9] * z) + m[13] * 1.0f;
    r.z = ((m[2] * x + m[6] * y) + m[10] * z) + m[14] * 1.0f;
    r.w = ((m[3] * x + m[7] * y) + m[11] * z) + m[15] * 1.0f;
    return r;
}

// Three IEEE single-precision quotients a/w, b/w, c/w that share one
// reciprocal, computed in double precision: r ~ 1/w from the single-precision
// reciprocal approximation refined by two Newton-Raphson steps in double
// (relative error below 2^-51), then q = RN32(RN64(a * r)).  The exact
// quotient of two floats lies at least 2^-49 |q| away from every midpoint
// between neighbouring floats (a * 2^k - m * w is a nonzero multiple of the
// unit of m * w for a midpoint m), while RN64(a * r) is within 2^-50 |q| of
// it, so rounding it to single precision gives the correctly rounded
// quotient, the same bits as a / w.  Outside |w| in [2^-125, 2^125] (and for
// NaN or infinite w) the plain divisions are used.
__device__ __forceinline__ void div3_shared(float a, float b, float c, float w, float &qa,
                                            float &qb, float &qc) {
    const float aw = fabsf(w);
    if (!(aw >= 2.3509887e-38f && aw <= 4.2535296e37f)) {
        qa = a / w;
        qb = b / w;
        qc = c / w;
        return;
    }
    float r0;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(w));
    const double wd = (double)w;
    double r = (double)r0;
    r = __fma_rn(r, __fma_rn(-wd, r, 1.0), r);
    r = __fma_rn(r, __fma_rn(-wd, r, 1.0), r);
    qa = __double2float_rn(__dmul_rn((double)a, r));
    qb = __double2float_rn(__dmul_rn((double)b, r));
    qc = __double2float_rn(__dmul_rn((double)c, r));
}

__device__ __forceinline__ void mat4mul(const float *a, const float *b, float *out) {
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int row = 0; row < 4; ++row)
            out[c * 4 + row] = ((a[0 * 4 + row] * b[c * 4 + 0] + a[1 * 4 + row] * b[c * 4 + 1]) +
                                a[2 * 4 + row] * b[c * 4 + 2]) +
                               a[3 * 4 + row] * b[c * 4 + 3];
}

// Project-written log2: x = m * 2^e with m in [sqrt(1/2), sqrt(2)),
// s = (m-1)/(m+1), ln(m) = 2 atanh(s) from the odd Taylor series of atanh
// through s^11 (Abramowitz & Stegun 4.1.27), log2(x) = e + ln(m)/ln(2).
// Used instead of a library log2 so the CPU oracle computes identical bits.
__device__ __forceinline__ float log2_contract(float x) {
    if (isnan(x)) return x;
    if (x < 0.0f) return __int_as_float(0x7fc00000);
    if (x == 0.0f) return __int_as_float(0xff800000);
    if (isinf(x)) return x;
    uint32_t bits = __float_as_uint(x);
    int e = (int)((bits >> 23) & 0xffu);
    if (e == 0) {
        const float y = x * 8388608.0f;
        bits = __float_as_uint(y);
        e = (int)((bits >> 23) & 0xffu) - 23;
    }
    e -= 127;
    float m = __uint_as_float((bits & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float s2 = s * s;
    float p = 0.0909090936f;
    p = p * s2 + 0.111111112f;
    p = p * s2 + 0.142857149f;
    p = p * s2 + 0.200000003f;
    p = p * s2 + 0.333333343f;
    p = p * s2 + 1.0f;
    const float t = s * p;
    const float l = t * 2.88539008f;
    return (float)e + l;
}

// depthToUintReverseZ / uintToDepthReverseZ (Common.metal:10-16):
// float(CR_MAX_DEPTH - 1u) rounds to 2^32; the conversion saturates at 1.0.
__device__ __forceinline__ uint32_t depth_to_uint(float z) {
    return (uint32_t)(fminf(fmaxf(z, 0.0f), 1.0f) * 4294967296.0f);
}
__device__ __forceinline__ float uint_to_depth(uint32_t d) { return (float)d / 4294967296.0f; }

// hashUnit (Common.metal:190-197).
__device__ __forceinline__ float hash_unit(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return (float)x * (1.0f / 4294967296.0f);
}

// Point-size inputs of pointFootprintRadius (Common.metal:18-61).
struct PointSize {
    int mode;
    float minimum, maximum, scale;
};

// pointFootprintRadius (Common.metal:18-61).
__device__ __forceinline__ int footprint_radius(float px, float py, float pz, const float *world,
                                                const float *view, const float *proj, int sh,
                                                const PointSize &ps_cfg) {
    const f4 wp = mulp(world, px, py, pz);
    const f4 vp = mulp(view, wp.x, wp.y, wp.z);
    const float lo = fmaxf(fminf(ps_cfg.minimum, ps_cfg.maximum), 1.0f);
    const float hi = fmaxf(fmaxf(ps_cfg.minimum, ps_cfg.maximum), lo);
    const bool ortho = (proj[15] == 1.0f);
    float ps;
    if (ps_cfg.mode == 1) {
        const float focal = ((float)sh * 0.5f) * proj[5];
        if (ortho) {
            ps = (2.0f * ps_cfg.scale) * focal;
        } else {
            const float viewZ = fmaxf(-vp.z, 0.000001f);
            ps = ((2.0f * ps_cfg.scale) * focal) / viewZ;
        }
    } else {
        if (ortho) {
            ps = ps_cfg.scale;
        } else {
            const float len = sqrtf((vp.x * vp.x + vp.y * vp.y) + vp.z * vp.z);
            ps = ps_cfg.scale / fmaxf(len, 0.000001f);
        }
    }
    if (!isfinite(ps)) ps = lo;
    ps = fminf(fmaxf(ps, lo), hi);
    const int r = (int)ceilf(fmaxf(ps - 1.0f, 0.0f) * 0.5f);
    return min(max(r, 0), 16);
}

// insidePointFootprint (Common.metal:63-71).
__device__ __forceinline__ bool inside_footprint(int ox, int oy, int radius) {
    if (radius <= 0) return ox == 0 && oy == 0;
    const float fx = (float)ox, fy = (float)oy;
    const float r = (float)radius + 0.5f;
    return (fx * fx + fy * fy) <= r * r;
}

// makePlane + intersectsFrustum (Common.metal:119-153), m[col*4+row].
__device__ __forceinline__ bool plane_rejects(float x, float y, float z, float w, f3 mn, f3 mx) {
    const float len = fmaxf(sqrtf((x * x + y * y) + z * z), 0.000001f);
    const float nx = x / len, ny = y / len, nz = z / len, off = w / len;
    const float px = nx > 0.0f ? mx.x : mn.x;
    const float py = ny > 0.0f ? mx.y : mn.y;
    const float pz = nz > 0.0f ? mx.z : mn.z;
    return ((nx * px + ny * py) + nz * pz) + off < 0.0f;
}

__device__ __forceinline__ bool intersects_frustum(const float *m, f3 mn, f3 mx) {
#define M_(c, r) m[(c) * 4 + (r)]
    if (plane_rejects(M_(0, 3) - M_(0, 0), M_(1, 3) - M_(1, 0), M_(2, 3) - M_(2, 0),
                      M_(3, 3) - M_(3, 0), mn, mx))
        return false;
    if (plane_rejects(M_(0, 3) + M_(0, 0), M_(1, 3) + M_(1, 0), M_(2, 3) + M_(2, 0),
                      M_(3, 3) + M_(3, 0), mn, mx))
        return false;
    if (plane_rejects(M_(0, 3) + M_(0, 1), M_(1, 3) + M_(1, 1), M_(2, 3) + M_(2, 1),
                      M_(3, 3) + M_(3, 1), mn, mx))
        return false;
    if (plane_rejects(M_(0, 3) - M_(0, 1), M_(1, 3) - M_(1, 1), M_(2, 3) - M_(2, 1),
                      M_(3, 3) - M_(3, 1), mn, mx))
        return false;
    if (plane_rejects(M_(0, 3) - M_(0, 2), M_(1, 3) - M_(1, 2), M_(2, 3) - M_(2, 2),
                      M_(3, 3) - M_(3, 2), mn, mx))
        return false;
    if (plane_rejects(M_(0, 2), M_(1, 2), M_(2, 2), M_(3, 2), mn, mx)) return false;
#undef M_
    return true;
}

// The per-file parts of the cull, computed once per file instead of once
// per batch (the same operations on the same inputs, so the same bits): the
// six normalised frustum planes of makePlane (nx, ny, nz, offset) and
// view * world for pixelSizeOnScreen.
struct FilePre {
    float plane[6][4];
    float vw[16];
};
__device__ __forceinline__ void plane_of(float x, float y, float z, float w, float *out) {
    const float len = fmaxf(sqrtf((x * x + y * y) + z * z), 0.000001f);
    out[0] = x / len;
    out[1] = y / len;
    out[2] = z / len;
    out[3] = w / len;
}
// Plane k (0..5) of the frustum matrix m, in intersects_frustum's order.
__device__ __forceinline__ void frustum_plane(const float *m, int k, float *out) {
#define M_(c, r) m[(c) * 4 + (r)]
    switch (k) {
    case 0: plane_of(M_(0, 3) - M_(0, 0), M_(1, 3) - M_(1, 0), M_(2, 3) - M_(2, 0), M_(3, 3) - M_(3, 0), out); break;
    case 1: plane_of(M_(0, 3) + M_(0, 0), M_(1, 3) + M_(1, 0), M_(2, 3) + M_(2, 0), M_(3, 3) + M_(3, 0), out); break;
    case 2: plane_of(M_(0, 3) + M_(0, 1), M_(1, 3) + M_(1, 1), M_(2, 3) + M_(2, 1), M_(3, 3) + M_(3, 1), out); break;
    case 3: plane_of(M_(0, 3) - M_(0, 1), M_(1, 3) - M_(1, 1), M_(2, 3) - M_(2, 1), M_(3, 3) - M_(3, 1), out); break;
    case 4: plane_of(M_(0, 3) - M_(0, 2), M_(1, 3) - M_(1, 2), M_(2, 3) - M_(2, 2), M_(3, 3) - M_(3, 2), out); break;
    default: plane_of(M_(0, 2), M_(1, 2), M_(2, 2), M_(3, 2), out); break;
    }
#undef M_
}
// intersects_frustum over precomputed planes.
__device__ __forceinline__ bool intersects_frustum_pre(const FilePre &f, f3 mn, f3 mx) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float nx = f.plane[k][0], ny = f.plane[k][1], nz = f.plane[k][2];
        const float px = nx > 0.0f ? mx.x : mn.x;
        const float py = ny > 0.0f ? mx.y : mn.y;
        const float pz = nz > 0.0f ? mx.z : mn.z;
        if (((nx * px + ny * py) + nz * pz) + f.plane[k][3] < 0.0f) return false;
    }
    return true;
}

// pixelSizeOnScreen (Common.metal:155-170).
__device__ __forceinline__ float pixel_size_on_screen_vw(const cr_raster_batch &b, const float *vw,
                                                         const float *proj, int sw, int sh);
__device__ __forceinline__ float pixel_size_on_screen(const cr_raster_batch &b, const float *world,
                                                      const float *view, const float *proj,
                                                      int sw, int sh) {
    float vw[16];
    mat4mul(view, world, vw);
    return pixel_size_on_screen_vw(b, vw, proj, sw, sh);
}
// pixelSizeOnScreen with view * world given.
__device__ __forceinline__ float pixel_size_on_screen_vw(const cr_raster_batch &b, const float *vw,
                                                         const float *proj, int sw, int sh) {
    const float cx = (b.minX + b.maxX) * 0.5f, cy = (b.minY + b.maxY) * 0.5f,
                cz = (b.minZ + b.maxZ) * 0.5f;
    const float dx = b.minX - b.maxX, dy = b.minY - b.maxY, dz = b.minZ - b.maxZ;
    const float radius = sqrtf((dx * dx + dy * dy) + dz * dz);
    const f4 vc = mulp(vw, cx, cy, cz);
    const f4 ve{vc.x + radius, vc.y + 0.0f, vc.z + 0.0f, vc.w + 0.0f};
    f4 pc = mulv(proj, vc);
    f4 pe = mulv(proj, ve);
    const float wc = fmaxf(fabsf(pc.w), 0.000001f);
    pc.x = pc.x / wc;
    pc.y = pc.y / wc;
    const float we = fmaxf(fabsf(pe.w), 0.000001f);
    pe.x = pe.x / we;
    pe.y = pe.y / we;
    const float W = (float)sw, H = (float)sh;
    const float scx = (W * (pc.x + 1.0f)) * 0.5f, scy = (H * (pc.y + 1.0f)) * 0.5f;
    const float sex = (W * (pe.x + 1.0f)) * 0.5f, sey = (H * (pe.y + 1.0f)) * 0.5f;
    const float ex = sex - scx, ey = sey - scy;
    return sqrtf(ex * ex + ey * ey);
}

// precisionLevel thresholds (Common.metal:172-181; Cull/Shaders.metal:48-53).
__device__ __forceinline__ int precision_level(float px) {
    if (px < 100.0f) return 4;
    if (px < 200.0f) return 3;
    if (px < 500.0f) return 2;
    if (px < 10000.0f) return 1;
    return 0;
}

// e^-x for x >= 0 (the coverage resolve's alpha), written for this project
// and evaluated by the oracle with the same operations: Cody-Waite range
// reduction (Cody and Waite, Software Manual for the Elementary Functions,
// 1980) n = floor(x log2 e), r = (x - n ln2_hi) - n ln2_lo with n ln2_hi
// exact; e^-r by its Taylor series to degree 9 (Horner, every operation
// rounded); an exact power-of-two scale 2^-n.
__device__ __forceinline__ float exp_neg(float x) {
    if (x != x) return x;
    if (!(x > 0.0f)) return 1.0f;
    const float t = __fmul_rn(x, 1.44269504f);
    if (t >= 126.0f) return 0.0f;
    const float n = floorf(t);
    const float r = __fsub_rn(__fsub_rn(x, __fmul_rn(n, 0.693145751953125f)),
                              __fmul_rn(n, 1.42860682e-06f));
    const float z = __fsub_rn(0.0f, r);
    float p = 2.75573192e-06f;
    p = __fadd_rn(__fmul_rn(p, z), 2.48015873e-05f);
    p = __fadd_rn(__fmul_rn(p, z), 1.98412698e-04f);
    p = __fadd_rn(__fmul_rn(p, z), 1.38888889e-03f);
    p = __fadd_rn(__fmul_rn(p, z), 8.33333333e-03f);
    p = __fadd_rn(__fmul_rn(p, z), 4.16666667e-02f);
    p = __fadd_rn(__fmul_rn(p, z), 1.66666667e-01f);
    p = __fadd_rn(__fmul_rn(p, z), 0.5f);
    p = __fadd_rn(__fmul_rn(p, z), 1.0f);
    p = __fadd_rn(__fmul_rn(p, z), 1.0f);
    const float scale = __uint_as_float((uint32_t)(127 - (int)n) << 23);
    return __fmul_rn(p, scale);
}

// unorm8 texture write (rint(clamp(f*255, 0, 255)), round half to even).
__device__ __forceinline__ uint32_t unorm8(float f) {
    return (uint32_t)rintf(fminf(fmaxf(f * 255.0f, 0.0f), 255.0f));
}

}  // namespace crd
