// synth.cu — seeded synthetic point clouds (the benchmark workloads), written
// on the device as 16-byte records {float x, y, z; uint32 rgba8}.
//
//   terrain  a 4 km x 4 km fractal heightfield: 2-D gradient noise (integer
//            lattice hash -> one of eight unit gradients, quintic fade),
//            summed over octaves with lacunarity 2 and gain 0.5, scaled to
//            the amplitude; a fraction of the points are uniform volumetric
//            outliers; colour = height ramp + per-channel normal noise
//            (Box-Muller with the project-written ln and cos below).
//   lattice  an n^3 lattice over [lo, hi]^3 with uniform jitter and uniform
//            RGB8 (alpha 255), the 1M-point cube workload at n = 100.
// Both are pure functions of (seed, point index), so any range of points can
// be generated independently and the cloud is identical for every caller.
// Every operation is rounded on its own (-fmad=false) and no math-library
// function is used, so a host restatement with the same operations produces
// bit-identical records.
#include <cmath>

#include "cr_internal.h"

namespace {

constexpr int kThreads = 256;

__host__ __device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x21f0aaadu;
    x ^= x >> 15;
    x *= 0x735a2d97u;
    x ^= x >> 15;
    return x;
}

__host__ __device__ __forceinline__ uint32_t hash3(uint32_t a, uint32_t b, uint32_t c) {
    return mix32(a ^ mix32(b ^ mix32(c + 0x9e3779b9u)));
}

__host__ __device__ __forceinline__ float unit(uint32_t h) {  // [0, 1)
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

__host__ __device__ __forceinline__ float grad_dot(uint32_t h, float x, float y) {
    const float d = 0.70710678f;
    switch (h & 7u) {
    case 0: return x;
    case 1: return -x;
    case 2: return y;
    case 3: return -y;
    case 4: return d * (x + y);
    case 5: return d * (x - y);
    case 6: return d * (-x + y);
    default: return -d * (x + y);
    }
}

__host__ __device__ __forceinline__ float fade(float t) {
    return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f);
}

__host__ __device__ float gradient_noise(float x, float y, uint32_t seed) {
    const float fx0 = floorf(x), fy0 = floorf(y);
    const int ix = (int)fx0, iy = (int)fy0;
    const float tx = x - fx0, ty = y - fy0;
    const float n00 = grad_dot(hash3((uint32_t)ix, (uint32_t)iy, seed), tx, ty);
    const float n10 = grad_dot(hash3((uint32_t)(ix + 1), (uint32_t)iy, seed), tx - 1.0f, ty);
    const float n01 = grad_dot(hash3((uint32_t)ix, (uint32_t)(iy + 1), seed), tx, ty - 1.0f);
    const float n11 =
        grad_dot(hash3((uint32_t)(ix + 1), (uint32_t)(iy + 1), seed), tx - 1.0f, ty - 1.0f);
    const float u = fade(tx), v = fade(ty);
    const float a = n00 + u * (n10 - n00);
    const float b = n01 + u * (n11 - n01);
    return a + v * (b - a);
}

__host__ __device__ float terrain_height(const cr_synth_terrain &t, float x, float y) {
    float sum = 0.0f, amp = 1.0f, freq = 1.0f / t.baseWavelength;
    for (int o = 0; o < t.octaves; ++o) {
        sum += amp * gradient_noise(x * freq, y * freq, (uint32_t)t.seed + 1013u * (uint32_t)o);
        amp *= t.gain;
        freq *= t.lacunarity;
    }
    return sum * t.amplitude;
}

__host__ __device__ __forceinline__ float height_bound(const cr_synth_terrain &t) {
    float s = 0.0f, amp = 1.0f;
    for (int o = 0; o < t.octaves; ++o) {
        s += amp;
        amp *= t.gain;
    }
    return s * t.amplitude;
}

// Natural log of u in (0, 1] for the colour noise, written for this project
// so that a host restatement evaluates identical bits: u = m 2^e with m in
// [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s), s = (m - 1)/(m + 1), by the odd
// series through s^11 (Abramowitz & Stegun 4.1.27), ln u = e ln 2 + ln m.
__device__ __forceinline__ float ln_unit(float u) {
    const uint32_t b = __float_as_uint(u);
    int e = (int)((b >> 23) & 0xffu) - 127;
    float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
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
    return (float)e * 0.693147182f + (s * p) * 2.0f;
}

// cos(2 pi u) for u in [0, 1), written for this project: q = the nearest
// quarter turn (u - q/4 is exact), then the Taylor series of cos (through
// r^8) or sin (through r^9) of the remainder r = 2 pi (u - q/4), |r| <= pi/4,
// with the quadrant's sign.
__device__ __forceinline__ float cos_2pi(float u) {
    const float q = floorf(u * 4.0f + 0.5f);
    const float d = u - q * 0.25f;
    const float r = d * 6.28318531f;
    const float r2 = r * r;
    float c = 2.48015873e-05f;
    c = c * r2 + -1.38888889e-03f;
    c = c * r2 + 4.16666667e-02f;
    c = c * r2 + -0.5f;
    c = c * r2 + 1.0f;
    float sn = 2.75573192e-06f;
    sn = sn * r2 + -1.98412698e-04f;
    sn = sn * r2 + 8.33333333e-03f;
    sn = sn * r2 + -1.66666667e-01f;
    sn = sn * r2 + 1.0f;
    sn = sn * r;
    switch ((int)q & 3) {
    case 0: return c;
    case 1: return -sn;
    case 2: return -c;
    default: return sn;
    }
}

__device__ __forceinline__ uint32_t clamp_byte(float v) {
    return (uint32_t)fminf(fmaxf(rintf(v), 0.0f), 255.0f);
}

__global__ void __launch_bounds__(kThreads)
    synth_terrain(cr_synth_terrain t, uint64_t first, uint64_t n, float4 *__restrict__ out) {
    const uint64_t k = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    if (k >= n) return;
    const uint64_t i = first + k;
    const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
    const uint32_t s = (uint32_t)t.seed ^ (uint32_t)(t.seed >> 32);
    const float x = unit(hash3(lo, hi, s ^ 0x1111u)) * t.extent;
    const float y = unit(hash3(lo, hi, s ^ 0x2222u)) * t.extent;
    const float hb = height_bound(t);
    float z;
    if (unit(hash3(lo, hi, s ^ 0x3333u)) < t.outlierFraction) {
        const float zr = hb + t.outlierMargin;
        z = -zr + unit(hash3(lo, hi, s ^ 0x4444u)) * (2.0f * zr);
    } else {
        z = terrain_height(t, x, y);
    }
    // Height ramp (low green -> high light grey) plus N(0, sigma) per channel
    // (Box-Muller from two hashes).
    const float r01 = fminf(fmaxf((z + hb) / (2.0f * hb), 0.0f), 1.0f);
    const float base[3] = {40.0f + 180.0f * r01, 110.0f + 110.0f * r01, 40.0f + 190.0f * r01};
    uint32_t rgb = 0;
    for (int c = 0; c < 3; ++c) {
        const float u1 = fmaxf(unit(hash3(lo, hi, s ^ (0x5555u + 2u * c))), 1e-7f);
        const float u2 = unit(hash3(lo, hi, s ^ (0x5556u + 2u * c)));
        const float g = sqrtf(-2.0f * ln_unit(u1)) * cos_2pi(u2);
        rgb |= clamp_byte(base[c] + t.colorNoiseSigma * g) << (8 * c);
    }
    out[k] = make_float4(x, y, z, __uint_as_float(rgb | 0xff000000u));
}

__global__ void __launch_bounds__(kThreads)
    synth_lattice(uint64_t seed, uint32_t n_axis, float lo, float hi, float jitter,
                  float4 *__restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    const uint64_t total = (uint64_t)n_axis * n_axis * n_axis;
    if (i >= total) return;
    const uint32_t ix = (uint32_t)(i % n_axis), iy = (uint32_t)((i / n_axis) % n_axis),
                   iz = (uint32_t)(i / ((uint64_t)n_axis * n_axis));
    const uint32_t s = (uint32_t)seed ^ (uint32_t)(seed >> 32);
    const float step = n_axis > 1 ? (hi - lo) / (float)(n_axis - 1) : 0.0f;
    const uint32_t li = (uint32_t)i, hi32 = (uint32_t)(i >> 32);
    const float jx = (unit(hash3(li, hi32, s ^ 0xa1u)) * 2.0f - 1.0f) * jitter;
    const float jy = (unit(hash3(li, hi32, s ^ 0xa2u)) * 2.0f - 1.0f) * jitter;
    const float jz = (unit(hash3(li, hi32, s ^ 0xa3u)) * 2.0f - 1.0f) * jitter;
    const uint32_t c = hash3(li, hi32, s ^ 0xa4u) & 0x00ffffffu;
    out[i] = make_float4(lo + step * (float)ix + jx, lo + step * (float)iy + jy,
                         lo + step * (float)iz + jz, __uint_as_float(c | 0xff000000u));
}

}  // namespace

extern "C" {

CR_API cr_status cr_synth_terrain_default(cr_synth_terrain *t) {
    if (!t) return cri::fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    t->seed = 0xC0FFEE02ull;
    t->extent = 4000.0f;
    t->amplitude = 200.0f;
    t->baseWavelength = 1500.0f;
    t->octaves = 6;
    t->lacunarity = 2.0f;
    t->gain = 0.5f;
    t->outlierFraction = 0.05f;
    t->outlierMargin = 50.0f;
    t->colorNoiseSigma = 10.0f;
    return CR_OK;
}

CR_API float cr_synth_terrain_height(const cr_synth_terrain *t, float x, float y) {
    return t ? terrain_height(*t, x, y) : 0.0f;
}

CR_API cr_status cr_synth_terrain_points(cr_context *ctx, const cr_synth_terrain *t, uint64_t first,
                                         uint64_t count, void *device_records) {
    if (!ctx || !t || (!device_records && count)) return cri::fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if (t->octaves < 1 || t->octaves > 16 || !(t->baseWavelength > 0.0f))
        return cri::fail(CR_ERR_INVALID_ARGUMENT, "bad terrain parameters");
    if (((uintptr_t)device_records & 15) != 0)
        return cri::fail(CR_ERR_INVALID_ARGUMENT, "records must be 16-byte aligned");
    if (count == 0) return CR_OK;
    cudaSetDevice(ctx->device);
    synth_terrain<<<(unsigned)((count + kThreads - 1) / kThreads), kThreads, 0, ctx->stream>>>(
        *t, first, count, static_cast<float4 *>(device_records));
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

CR_API cr_status cr_synth_lattice_points(cr_context *ctx, uint64_t seed, uint32_t n_axis, float lo,
                                         float hi, float jitter, void *device_records) {
    if (!ctx || (!device_records && n_axis)) return cri::fail(CR_ERR_INVALID_ARGUMENT, "null argument");
    if (((uintptr_t)device_records & 15) != 0)
        return cri::fail(CR_ERR_INVALID_ARGUMENT, "records must be 16-byte aligned");
    const uint64_t total = (uint64_t)n_axis * n_axis * n_axis;
    if (total == 0) return CR_OK;
    cudaSetDevice(ctx->device);
    synth_lattice<<<(unsigned)((total + kThreads - 1) / kThreads), kThreads, 0, ctx->stream>>>(
        seed, n_axis, lo, hi, jitter, static_cast<float4 *>(device_records));
    CR_CUDA(cudaGetLastError());
    return CR_OK;
}

}  // extern "C"
