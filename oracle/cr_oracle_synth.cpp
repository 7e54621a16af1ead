// cr_oracle_synth.cpp — CPU generators of the seeded synthetic clouds (test
// infrastructure).
//
// The benchmark workloads are synthetic: the 1M-point jittered lattice and the
// fractal heightfield with volumetric outliers.  The library generates them on
// the device; this file restates the same generators on the host so that the
// CPU side (the reference arm of the benchmark, the packer's parity check)
// builds its inputs without the library.  Every value is a pure function of
// (seed, point index) evaluated with the same operations in the same order
// (no FMA contraction, IEEE division and square root), and the colour noise
// uses the project-written ln and cos below instead of a math library, so the
// records are bit-identical to the device's.
#include "cr_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x21f0aaadu;
    x ^= x >> 15;
    x *= 0x735a2d97u;
    x ^= x >> 15;
    return x;
}

inline uint32_t hash3(uint32_t a, uint32_t b, uint32_t c) {
    return mix32(a ^ mix32(b ^ mix32(c + 0x9e3779b9u)));
}

inline float unit(uint32_t h) { return (float)(h >> 8) * (1.0f / 16777216.0f); }

inline float bits_f(uint32_t b) {
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}
inline uint32_t f_bits(float f) {
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return b;
}

float grad_dot(uint32_t h, float x, float y) {
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

inline float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }

float gradient_noise(float x, float y, uint32_t seed) {
    const float fx0 = std::floor(x), fy0 = std::floor(y);
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

float height_bound(const orc_terrain &t) {
    float s = 0.0f, amp = 1.0f;
    for (int o = 0; o < t.octaves; ++o) {
        s += amp;
        amp *= t.gain;
    }
    return s * t.amplitude;
}

// Natural log of u in (0, 1]: u = m 2^e with m in [sqrt(1/2), sqrt(2)),
// ln m = 2 atanh(s), s = (m - 1)/(m + 1), by the odd series through s^11
// (Abramowitz & Stegun 4.1.27), ln u = e ln 2 + ln m.
float ln_unit(float u) {
    uint32_t b = f_bits(u);
    int e = (int)((b >> 23) & 0xffu) - 127;
    float m = bits_f((b & 0x007fffffu) | 0x3f800000u);
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

// cos(2 pi u) for u in [0, 1): q = the nearest quarter turn (u - q/4 is exact,
// |r| <= pi/4 after scaling), then the Taylor series of cos (through r^8) or
// sin (through r^9) of the remainder, with the quadrant's sign.
float cos_2pi(float u) {
    const float q = std::floor(u * 4.0f + 0.5f);
    const float d = u - q * 0.25f;
    const float r = d * 6.28318531f;
    const float r2 = r * r;
    float c = 2.48015873e-05f;
    c = c * r2 + -1.38888889e-03f;
    c = c * r2 + 4.16666667e-02f;
    c = c * r2 + -0.5f;
    c = c * r2 + 1.0f;
    float s = 2.75573192e-06f;
    s = s * r2 + -1.98412698e-04f;
    s = s * r2 + 8.33333333e-03f;
    s = s * r2 + -1.66666667e-01f;
    s = s * r2 + 1.0f;
    s = s * r;
    switch ((int)q & 3) {
    case 0: return c;
    case 1: return -s;
    case 2: return -c;
    default: return s;
    }
}

inline uint32_t clamp_byte(float v) {
    return (uint32_t)std::fmin(std::fmax(std::rint(v), 0.0f), 255.0f);
}

void terrain_point(const orc_terrain &t, uint64_t i, float hb, float out[4]) {
    const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
    const uint32_t s = (uint32_t)t.seed ^ (uint32_t)(t.seed >> 32);
    const float x = unit(hash3(lo, hi, s ^ 0x1111u)) * t.extent;
    const float y = unit(hash3(lo, hi, s ^ 0x2222u)) * t.extent;
    float z;
    if (unit(hash3(lo, hi, s ^ 0x3333u)) < t.outlierFraction) {
        const float zr = hb + t.outlierMargin;
        z = -zr + unit(hash3(lo, hi, s ^ 0x4444u)) * (2.0f * zr);
    } else {
        z = orc_terrain_height(&t, x, y);
    }
    const float r01 = std::fmin(std::fmax((z + hb) / (2.0f * hb), 0.0f), 1.0f);
    const float base[3] = {40.0f + 180.0f * r01, 110.0f + 110.0f * r01, 40.0f + 190.0f * r01};
    uint32_t rgb = 0;
    for (uint32_t c = 0; c < 3; ++c) {
        const float u1 = std::fmax(unit(hash3(lo, hi, s ^ (0x5555u + 2u * c))), 1e-7f);
        const float u2 = unit(hash3(lo, hi, s ^ (0x5556u + 2u * c)));
        const float g = std::sqrt(-2.0f * ln_unit(u1)) * cos_2pi(u2);
        rgb |= clamp_byte(base[c] + t.colorNoiseSigma * g) << (8 * c);
    }
    out[0] = x;
    out[1] = y;
    out[2] = z;
    out[3] = bits_f(rgb | 0xff000000u);
}

template <typename F>
void parallel_for(uint64_t n, int threads, F f) {
    threads = std::max(1, threads);
    if (threads == 1 || n < 4096) {
        f(0, n);
        return;
    }
    std::vector<std::thread> pool;
    const uint64_t step = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const uint64_t a = std::min<uint64_t>(n, (uint64_t)t * step);
        const uint64_t b = std::min<uint64_t>(n, a + step);
        if (a < b) pool.emplace_back([=] { f(a, b); });
    }
    for (auto &th : pool) th.join();
}

}  // namespace

extern "C" {

float orc_terrain_height(const orc_terrain *t, float x, float y) {
    float sum = 0.0f, amp = 1.0f, freq = 1.0f / t->baseWavelength;
    for (int o = 0; o < t->octaves; ++o) {
        sum += amp * gradient_noise(x * freq, y * freq, (uint32_t)t->seed + 1013u * (uint32_t)o);
        amp *= t->gain;
        freq *= t->lacunarity;
    }
    return sum * t->amplitude;
}

int orc_synth_terrain(const orc_terrain *t, uint64_t first, uint64_t count, float *records,
                      int threads) {
    if (!t || (count && !records)) return 1;
    if (t->octaves < 1 || t->octaves > 16 || !(t->baseWavelength > 0.0f)) return 1;
    const float hb = height_bound(*t);
    parallel_for(count, threads, [&](uint64_t a, uint64_t b) {
        for (uint64_t k = a; k < b; ++k) terrain_point(*t, first + k, hb, records + 4 * k);
    });
    return 0;
}

int orc_synth_lattice(uint64_t seed, uint32_t n_axis, float lo, float hi, float jitter,
                      float *records, int threads) {
    const uint64_t total = (uint64_t)n_axis * n_axis * n_axis;
    if (total && !records) return 1;
    const uint32_t s = (uint32_t)seed ^ (uint32_t)(seed >> 32);
    const float step = n_axis > 1 ? (hi - lo) / (float)(n_axis - 1) : 0.0f;
    parallel_for(total, threads, [&](uint64_t a, uint64_t b) {
        for (uint64_t i = a; i < b; ++i) {
            const uint32_t ix = (uint32_t)(i % n_axis), iy = (uint32_t)((i / n_axis) % n_axis),
                           iz = (uint32_t)(i / ((uint64_t)n_axis * n_axis));
            const uint32_t li = (uint32_t)i, hi32 = (uint32_t)(i >> 32);
            const float jx = (unit(hash3(li, hi32, s ^ 0xa1u)) * 2.0f - 1.0f) * jitter;
            const float jy = (unit(hash3(li, hi32, s ^ 0xa2u)) * 2.0f - 1.0f) * jitter;
            const float jz = (unit(hash3(li, hi32, s ^ 0xa3u)) * 2.0f - 1.0f) * jitter;
            const uint32_t c = hash3(li, hi32, s ^ 0xa4u) & 0x00ffffffu;
            float *o = records + 4 * i;
            o[0] = lo + step * (float)ix + jx;
            o[1] = lo + step * (float)iy + jy;
            o[2] = lo + step * (float)iz + jz;
            o[3] = bits_f(c | 0xff000000u);
        }
    });
    return 0;
}

float orc_ln_unit(float u) { return ln_unit(u); }
float orc_cos_2pi(float u) { return cos_2pi(u); }

}  // extern "C"
