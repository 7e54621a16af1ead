// cr_oracle_pack.cpp — CPU oracle of the point-cloud packer (test infrastructure).
//
// Restates PackedPointCloudFixtures.pack (Sources/SatinComputeRasteriser/
// PackedPointCloudFixtures.swift:30-344).  morton_bits = 10 is the reference's
// 30-bit key; morton_bits = 21 is the 63-bit key variant (21 bits per axis)
// with the same bounds, normalisation and tie order.
#include "cr_oracle.h"
#include "cr_oracle_pack_util.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

namespace {
using namespace orcpack;

// mortonOrder (PackedPointCloudFixtures.swift:218-239): key per point, then a
// stable sort of the indices by key (equal keys keep input order).
std::vector<uint32_t> morton_order(const std::vector<f3> &pos, f3 bmin, f3 bmax, int bits) {
    const size_t n = pos.size();
    const f3 ext{fmax_(bmax.x - bmin.x, 0.000001f), fmax_(bmax.y - bmin.y, 0.000001f),
                 fmax_(bmax.z - bmin.z, 0.000001f)};
    const float top = (bits == 21) ? 2097151.0f : 1023.0f;
    const f3 scale{top / ext.x, top / ext.y, top / ext.z};
    std::vector<uint64_t> keys(n);
    for (size_t i = 0; i < n; ++i) {
        const float nx = clampf_((pos[i].x - bmin.x) * scale.x, 0.0f, top);
        const float ny = clampf_((pos[i].y - bmin.y) * scale.y, 0.0f, top);
        const float nz = clampf_((pos[i].z - bmin.z) * scale.z, 0.0f, top);
        const uint32_t qx = f2u(nx), qy = f2u(ny), qz = f2u(nz);
        if (bits == 21)
            keys[i] = (spread21(qx) << 2) | (spread21(qy) << 1) | spread21(qz);
        else
            keys[i] = (uint64_t)((spread10(qx) << 2) | (spread10(qy) << 1) | spread10(qz));
    }
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    std::stable_sort(idx.begin(), idx.end(),
                     [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    return idx;
}

// computeLODLevels (PackedPointCloudFixtures.swift:245-334): per level,
// coarsest first, the first still-unassigned point (in sorted order) that
// lands in a not-yet-occupied voxel takes that level.
std::vector<uint8_t> lod_levels(const std::vector<f3> &pos, f3 bmin, f3 bmax, int L, int divs) {
    const size_t n = pos.size();
    const uint8_t maxLevel = (uint8_t)(L - 1);
    std::vector<uint8_t> lv(n, maxLevel);
    if (L <= 1) return lv;
    const f3 ext{fmax_(bmax.x - bmin.x, 0.000001f), fmax_(bmax.y - bmin.y, 0.000001f),
                 fmax_(bmax.z - bmin.z, 0.000001f)};
    const float longest = fmax_(ext.x, fmax_(ext.y, ext.z));
    const float baseVoxel = longest / (float)divs;
    // cellKey (:266-272): floor per axis, clamped at 0, 21 bits per axis.
    auto cell_key = [](float lx, float ly, float lz) -> uint64_t {
        const uint64_t cx = (uint64_t)std::max(0, f2i(std::floor(lx))) & 0x1fffffull;
        const uint64_t cy = (uint64_t)std::max(0, f2i(std::floor(ly))) & 0x1fffffull;
        const uint64_t cz = (uint64_t)std::max(0, f2i(std::floor(lz))) & 0x1fffffull;
        return (cx << 42) | (cy << 21) | cz;
    };
    // Open-addressing set with Fibonacci hashing (:293-331); the sentinel is
    // all ones, which no 63-bit key can equal.
    const uint64_t sentinel = ~0ull;
    size_t cap = 1;
    while (cap < n * 2) cap <<= 1;
    const size_t mask = cap - 1;
    int tz = 0;
    while ((1ull << tz) < cap) ++tz;
    const int shift = 64 - tz;
    std::vector<uint64_t> table(cap, sentinel);
    for (int level = 0; level < L - 1; ++level) {
        const float voxel = baseVoxel * std::pow(0.5f, (float)level);
        const float inv = 1.0f / fmax_(voxel, 0.000001f);
        if (level != 0) std::fill(table.begin(), table.end(), sentinel);
        for (size_t i = 0; i < n; ++i) {
            if (lv[i] != maxLevel) continue;
            const uint64_t key = cell_key((pos[i].x - bmin.x) * inv, (pos[i].y - bmin.y) * inv,
                                          (pos[i].z - bmin.z) * inv);
            size_t slot = (size_t)((key * 0x9E3779B97F4A7C15ull) >> shift);
            for (;;) {
                const uint64_t cur = table[slot];
                if (cur == sentinel) {
                    table[slot] = key;
                    lv[i] = (uint8_t)level;
                    break;
                }
                if (cur == key) break;
                slot = (slot + 1) & mask;
            }
        }
    }
    return lv;
}

}  // namespace

extern "C" int orc_pack(const float *positions, const float *colors_f32,
                        const uint32_t *colors_rgba8, uint64_t n, uint32_t ppb, int lod_levels_in,
                        int divs_in, int morton_bits, orc_batch *batches, uint32_t *xyz_low,
                        uint32_t *xyz_med, uint32_t *xyz_high, uint32_t *colors, uint8_t *levels,
                        uint32_t *source_indices, float *ordered_positions, float *bounds) {
    if (n == 0) return 0;
    if (ppb == 0 || ppb > 65535u) return 1;  // uint16 LOD prefix counts (:74)
    if (morton_bits != 10 && morton_bits != 21) return 1;
    std::vector<f3> pos(n);
    for (uint64_t i = 0; i < n; ++i)
        pos[i] = f3{positions[i * 3 + 0], positions[i * 3 + 1], positions[i * 3 + 2]};

    // Global bounds (:51-56).
    f3 bmin{3.4028235e38f, 3.4028235e38f, 3.4028235e38f};
    f3 bmax{-3.4028235e38f, -3.4028235e38f, -3.4028235e38f};
    for (const f3 &p : pos) {
        bmin = min3(bmin, p);
        bmax = max3(bmax, p);
    }

    std::vector<uint32_t> order = morton_order(pos, bmin, bmax, morton_bits);
    std::vector<f3> sorted(n);
    for (uint64_t i = 0; i < n; ++i) sorted[i] = pos[order[i]];
    const int L = std::max(1, std::min(lod_levels_in, 8));
    const int divs = std::max(1, divs_in);
    std::vector<uint8_t> lv = lod_levels(sorted, bmin, bmax, L, divs);

    // bucketSortBatchSlicesByLevel (:174-213): stable per-slice 8-bucket sort.
    for (uint64_t first = 0; first < n; first += ppb) {
        const uint64_t end = std::min<uint64_t>(first + ppb, n);
        uint32_t cursor[9] = {0};
        for (uint64_t i = first; i < end; ++i) cursor[(lv[i] & 7) + 1]++;
        for (int l = 1; l < 9; ++l) cursor[l] += cursor[l - 1];
        std::vector<uint64_t> perm(end - first);
        for (uint64_t i = first; i < end; ++i) perm[cursor[lv[i] & 7]++] = i;
        std::vector<uint32_t> o2(perm.size());
        std::vector<f3> p2(perm.size());
        std::vector<uint8_t> l2(perm.size());
        for (size_t j = 0; j < perm.size(); ++j) {
            o2[j] = order[perm[j]];
            p2[j] = sorted[perm[j]];
            l2[j] = lv[perm[j]];
        }
        for (size_t j = 0; j < perm.size(); ++j) {
            order[first + j] = o2[j];
            sorted[first + j] = p2[j];
            lv[first + j] = l2[j];
        }
    }

    // Per batch: AABB, 30-bit quantisation split into 3 x 10-bit chunks, LOD
    // cumulative counts (:89-143).
    uint64_t b = 0;
    for (uint64_t first = 0; first < n; first += ppb, ++b) {
        const uint64_t end = std::min<uint64_t>(first + ppb, n);
        f3 mn{3.4028235e38f, 3.4028235e38f, 3.4028235e38f};
        f3 mx{-3.4028235e38f, -3.4028235e38f, -3.4028235e38f};
        for (uint64_t i = first; i < end; ++i) {
            mn = min3(mn, sorted[i]);
            mx = max3(mx, sorted[i]);
        }
        const f3 size{fmax_(mx.x - mn.x, 0.000001f), fmax_(mx.y - mn.y, 0.000001f),
                      fmax_(mx.z - mn.z, 0.000001f)};
        for (uint64_t i = first; i < end; ++i) {
            // Float(computeRasteriserSteps30Bit - 1) rounds to 2^30 in f32.
            const float nx = clampf_((sorted[i].x - mn.x) / size.x, 0.0f, 0.99999994f);
            const float ny = clampf_((sorted[i].y - mn.y) / size.y, 0.0f, 0.99999994f);
            const float nz = clampf_((sorted[i].z - mn.z) / size.z, 0.0f, 0.99999994f);
            const uint32_t qx = f2u(nx * 1073741824.0f), qy = f2u(ny * 1073741824.0f),
                           qz = f2u(nz * 1073741824.0f);
            xyz_low[i] = ((qx >> 20) & 1023u) | (((qy >> 20) & 1023u) << 10) |
                         (((qz >> 20) & 1023u) << 20);
            xyz_med[i] = ((qx >> 10) & 1023u) | (((qy >> 10) & 1023u) << 10) |
                         (((qz >> 10) & 1023u) << 20);
            xyz_high[i] = (qx & 1023u) | ((qy & 1023u) << 10) | ((qz & 1023u) << 20);
        }
        orc_batch rb;
        std::memset(&rb, 0, sizeof(rb));
        rb.state = 1;
        rb.minX = mn.x;
        rb.minY = mn.y;
        rb.minZ = mn.z;
        rb.maxX = mx.x;
        rb.maxY = mx.y;
        rb.maxZ = mx.z;
        rb.numPoints = (uint32_t)(end - first);
        rb.firstPoint = (uint32_t)first;
        rb.fileIndex = 0;
        uint32_t cum[8] = {0};
        for (uint64_t i = first; i < end; ++i) cum[lv[i] & 7]++;
        for (int l = 1; l < 8; ++l) cum[l] += cum[l - 1];
        // setLODCumulativeCounts (ComputeRasteriserTypes.swift:214-223).
        rb.lodCum01 = cum[0] | (cum[1] << 16);
        rb.lodCum23 = cum[2] | (cum[3] << 16);
        rb.lodCum45 = cum[4] | (cum[5] << 16);
        rb.lodCum67 = cum[6] | (cum[7] << 16);
        batches[b] = rb;
    }

    // Colours in final order (:145-151): truncating clamp(c)*255 unless packed.
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t s = order[i];
        if (colors_rgba8) {
            colors[i] = colors_rgba8[s];
        } else {
            const float *c = &colors_f32[(size_t)s * 4];
            const uint32_t r = f2u(clampf_(c[0], 0.0f, 1.0f) * 255.0f);
            const uint32_t g = f2u(clampf_(c[1], 0.0f, 1.0f) * 255.0f);
            const uint32_t bl = f2u(clampf_(c[2], 0.0f, 1.0f) * 255.0f);
            const uint32_t a = f2u(clampf_(c[3], 0.0f, 1.0f) * 255.0f);
            colors[i] = r | (g << 8) | (bl << 16) | (a << 24);
        }
        levels[i] = lv[i];
        if (source_indices) source_indices[i] = s;
        if (ordered_positions) {
            ordered_positions[i * 3 + 0] = sorted[i].x;
            ordered_positions[i * 3 + 1] = sorted[i].y;
            ordered_positions[i * 3 + 2] = sorted[i].z;
        }
    }
    if (bounds) {
        bounds[0] = bmin.x;
        bounds[1] = bmin.y;
        bounds[2] = bmin.z;
        bounds[3] = bmax.x;
        bounds[4] = bmax.y;
        bounds[5] = bmax.z;
    }
    return 0;
}
