// cr_oracle_pack_util.h — arithmetic helpers shared by the single- and
// multi-threaded CPU packers of the oracle (test infrastructure): the
// reference's float->int conversions, Morton bit spreads and the bounds
// order (PackedPointCloudFixtures.swift:30-344).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace orcpack {

inline float fmax_(float a, float b) { return std::fmax(a, b); }
inline float fmin_(float a, float b) { return std::fmin(a, b); }
inline float clampf_(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
inline uint32_t f2u(float x) {
    if (std::isnan(x) || x <= 0.0f) return 0u;
    if (x >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)x;
}
inline int32_t f2i(float x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}

// mortonSpread10 (PackedPointCloudFixtures.swift:336-343).
inline uint32_t spread10(uint32_t v) {
    uint32_t x = v & 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// 21-bit spread into every third bit of a 63-bit word (same interleave rule).
inline uint64_t spread21(uint64_t v) {
    uint64_t x = v & 0x1fffffull;
    x = (x | (x << 32)) & 0x1f00000000ffffull;
    x = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

struct f3 { float x, y, z; };

// Bounds reductions order floats by their sign-flipped bit patterns (a total
// order with -0 below +0), so a serial loop and a parallel tree agree on the
// sign of a zero bound.
inline uint32_t flip(float f) {
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return b ^ ((b >> 31) ? 0xffffffffu : 0x80000000u);
}
inline float bmin_(float a, float b) { return flip(b) < flip(a) ? b : a; }
inline float bmax_(float a, float b) { return flip(b) > flip(a) ? b : a; }
inline f3 min3(f3 a, f3 b) { return f3{bmin_(a.x, b.x), bmin_(a.y, b.y), bmin_(a.z, b.z)}; }
inline f3 max3(f3 a, f3 b) { return f3{bmax_(a.x, b.x), bmax_(a.y, b.y), bmax_(a.z, b.z)}; }


}  // namespace orcpack
