// cr_oracle_pack_mt.cpp — the oracle's CPU packer on several host threads
// (test infrastructure), bit-identical to orc_pack (cr_oracle_pack.cpp, which
// restates PackedPointCloudFixtures.pack, PackedPointCloudFixtures.swift:
// 30-344).  Used where the single-threaded pack would take minutes: the
// reference arm of the benchmark builds its 100M-point cloud with it, and the
// packer's parity check compares the GPU pack of a large cloud with it.
//
// Why each step gives the single-threaded result:
//  * bounds: min / max over a total order of the floats (sign-flipped bit
//    patterns) is associative and commutative;
//  * the stable sort by key: an LSD radix sort whose per-digit output
//    offsets are laid out digit-major, then by thread, over contiguous
//    per-thread input ranges, so equal keys keep their input order, as the
//    reference's stable sort does;
//  * the LOD claims: in sorted order, the first still-unassigned point of a
//    not-yet-occupied voxel takes the level; that point is the voxel's
//    unassigned point of smallest sorted index, which a concurrent table
//    finds with an atomic minimum per voxel;
//  * the per-batch level bucketing, AABB, quantisation and colours touch
//    one batch or one point at a time.
#include "cr_oracle.h"
#include "cr_oracle_pack_util.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

namespace {
using namespace orcpack;

// Runs f(t, begin, end) on `threads` contiguous ranges of [0, n), range t on
// thread t (ranges in thread order; the same split for the same n and threads).
template <typename F>
void pfor(int threads, uint64_t n, F f) {
    const uint64_t step = (n + threads - 1) / threads;
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) {
        const uint64_t a = std::min<uint64_t>(n, (uint64_t)t * step);
        const uint64_t b = std::min<uint64_t>(n, a + step);
        pool.emplace_back([=] { f(t, a, b); });
    }
    f(0, 0, std::min<uint64_t>(n, step));
    for (auto &th : pool) th.join();
}

// Stable LSD radix sort of (key, index) pairs by key, 11-bit digits over the
// key's `bits` low bits; a digit that all keys share is skipped.
void radix_sort(std::vector<uint64_t> &keys, std::vector<uint32_t> &idx, int bits, int threads) {
    constexpr int kDigit = 11;
    constexpr uint32_t kBuckets = 1u << kDigit;
    const uint64_t n = keys.size();
    std::vector<uint64_t> k2(n);
    std::vector<uint32_t> i2(n);
    std::vector<uint64_t> hist((size_t)threads * kBuckets);
    for (int shift = 0; shift < bits; shift += kDigit) {
        std::fill(hist.begin(), hist.end(), 0);
        pfor(threads, n, [&](int t, uint64_t a, uint64_t b) {
            uint64_t *h = &hist[(size_t)t * kBuckets];
            for (uint64_t i = a; i < b; ++i) ++h[(keys[i] >> shift) & (kBuckets - 1)];
        });
        bool constant = false;
        uint64_t run = 0;
        for (uint32_t d = 0; d < kBuckets; ++d) {
            uint64_t total = 0;
            for (int t = 0; t < threads; ++t) {
                const uint64_t c = hist[(size_t)t * kBuckets + d];
                hist[(size_t)t * kBuckets + d] = run;
                run += c;
                total += c;
            }
            if (total == n) constant = true;
        }
        if (constant) continue;
        pfor(threads, n, [&](int t, uint64_t a, uint64_t b) {
            uint64_t *off = &hist[(size_t)t * kBuckets];
            for (uint64_t i = a; i < b; ++i) {
                const uint64_t p = off[(keys[i] >> shift) & (kBuckets - 1)]++;
                k2[p] = keys[i];
                i2[p] = idx[i];
            }
        });
        keys.swap(k2);
        idx.swap(i2);
    }
}

// computeLODLevels (PackedPointCloudFixtures.swift:245-334) with the claims
// of each level resolved as a minimum sorted index per voxel.
std::vector<uint8_t> lod_levels_mt(const std::vector<f3> &pos, f3 bmin, f3 bmax, int L, int divs,
                                   int threads) {
    const uint64_t n = pos.size();
    const uint8_t maxLevel = (uint8_t)(L - 1);
    std::vector<uint8_t> lv(n, maxLevel);
    if (L <= 1) return lv;
    const f3 ext{fmax_(bmax.x - bmin.x, 0.000001f), fmax_(bmax.y - bmin.y, 0.000001f),
                 fmax_(bmax.z - bmin.z, 0.000001f)};
    const float longest = fmax_(ext.x, fmax_(ext.y, ext.z));
    const float baseVoxel = longest / (float)divs;
    auto cell_key = [](float lx, float ly, float lz) -> uint64_t {
        const uint64_t cx = (uint64_t)std::max(0, f2i(std::floor(lx))) & 0x1fffffull;
        const uint64_t cy = (uint64_t)std::max(0, f2i(std::floor(ly))) & 0x1fffffull;
        const uint64_t cz = (uint64_t)std::max(0, f2i(std::floor(lz))) & 0x1fffffull;
        return (cx << 42) | (cy << 21) | cz;
    };
    const uint64_t sentinel = ~0ull;
    std::vector<uint32_t> slot_of(n);
    for (int level = 0; level < L - 1; ++level) {
        const float voxel = baseVoxel * std::pow(0.5f, (float)level);
        const float inv = 1.0f / fmax_(voxel, 0.000001f);
        // Distinct voxels are at most the unassigned points and at most the
        // voxels of the bounding box; the table holds twice that.
        uint64_t unassigned = 0;
        for (uint64_t i = 0; i < n; ++i) unassigned += lv[i] == maxLevel;
        const double box = (std::floor((double)ext.x * inv) + 2.0) *
                           (std::floor((double)ext.y * inv) + 2.0) *
                           (std::floor((double)ext.z * inv) + 2.0);
        const uint64_t distinct =
            box < (double)unassigned ? (uint64_t)box : unassigned;
        uint64_t cap = 1024;
        while (cap < 2 * distinct) cap <<= 1;
        int tz = 0;
        while ((1ull << tz) < cap) ++tz;
        const int shift = 64 - tz;
        const uint64_t mask = cap - 1;
        std::unique_ptr<std::atomic<uint64_t>[]> tkeys(new std::atomic<uint64_t>[cap]);
        std::unique_ptr<std::atomic<uint32_t>[]> tmin(new std::atomic<uint32_t>[cap]);
        pfor(threads, cap, [&](int, uint64_t a, uint64_t b) {
            for (uint64_t s = a; s < b; ++s) {
                tkeys[s].store(sentinel, std::memory_order_relaxed);
                tmin[s].store(0xffffffffu, std::memory_order_relaxed);
            }
        });
        pfor(threads, n, [&](int, uint64_t a, uint64_t b) {
            for (uint64_t i = a; i < b; ++i) {
                if (lv[i] != maxLevel) continue;
                const uint64_t key = cell_key((pos[i].x - bmin.x) * inv, (pos[i].y - bmin.y) * inv,
                                              (pos[i].z - bmin.z) * inv);
                uint64_t slot = (key * 0x9E3779B97F4A7C15ull) >> shift;
                for (;;) {
                    uint64_t cur = tkeys[slot].load(std::memory_order_relaxed);
                    if (cur == sentinel &&
                        tkeys[slot].compare_exchange_strong(cur, key, std::memory_order_relaxed))
                        cur = key;
                    if (cur == key) break;
                    slot = (slot + 1) & mask;
                }
                uint32_t m = tmin[slot].load(std::memory_order_relaxed);
                while ((uint32_t)i < m &&
                       !tmin[slot].compare_exchange_weak(m, (uint32_t)i, std::memory_order_relaxed)) {
                }
                slot_of[i] = (uint32_t)slot;
            }
        });
        pfor(threads, n, [&](int, uint64_t a, uint64_t b) {
            for (uint64_t i = a; i < b; ++i)
                if (lv[i] == maxLevel &&
                    tmin[slot_of[i]].load(std::memory_order_relaxed) == (uint32_t)i)
                    lv[i] = (uint8_t)level;
        });
    }
    return lv;
}

}  // namespace

extern "C" int orc_pack_threads(const float *positions, const float *colors_f32,
                                const uint32_t *colors_rgba8, uint64_t n, uint32_t ppb,
                                int lod_levels_in, int divs_in, int morton_bits,
                                orc_batch *batches, uint32_t *xyz_low, uint32_t *xyz_med,
                                uint32_t *xyz_high, uint32_t *colors, uint8_t *levels,
                                uint32_t *source_indices, float *ordered_positions, float *bounds,
                                int threads) {
    if (n == 0) return 0;
    if (ppb == 0 || ppb > 65535u) return 1;
    if (morton_bits != 10 && morton_bits != 21) return 1;
    if (n >= (1ull << 32)) return 1;
    threads = std::max(1, std::min(threads, 256));
    std::vector<f3> pos(n);
    std::vector<f3> tmin((size_t)threads, f3{3.4028235e38f, 3.4028235e38f, 3.4028235e38f});
    std::vector<f3> tmax((size_t)threads, f3{-3.4028235e38f, -3.4028235e38f, -3.4028235e38f});
    pfor(threads, n, [&](int t, uint64_t a, uint64_t b) {
        f3 mn = tmin[t], mx = tmax[t];
        for (uint64_t i = a; i < b; ++i) {
            pos[i] = f3{positions[i * 3 + 0], positions[i * 3 + 1], positions[i * 3 + 2]};
            mn = min3(mn, pos[i]);
            mx = max3(mx, pos[i]);
        }
        tmin[t] = mn;
        tmax[t] = mx;
    });
    f3 bmin = tmin[0], bmax = tmax[0];
    for (int t = 1; t < threads; ++t) {
        bmin = min3(bmin, tmin[t]);
        bmax = max3(bmax, tmax[t]);
    }

    // mortonOrder (:218-239): keys, then the stable sort.
    std::vector<uint64_t> keys(n);
    std::vector<uint32_t> order(n);
    {
        const f3 ext{fmax_(bmax.x - bmin.x, 0.000001f), fmax_(bmax.y - bmin.y, 0.000001f),
                     fmax_(bmax.z - bmin.z, 0.000001f)};
        const int bits = morton_bits;
        const float top = (bits == 21) ? 2097151.0f : 1023.0f;
        const f3 scale{top / ext.x, top / ext.y, top / ext.z};
        pfor(threads, n, [&](int, uint64_t a, uint64_t b) {
            for (uint64_t i = a; i < b; ++i) {
                const float nx = clampf_((pos[i].x - bmin.x) * scale.x, 0.0f, top);
                const float ny = clampf_((pos[i].y - bmin.y) * scale.y, 0.0f, top);
                const float nz = clampf_((pos[i].z - bmin.z) * scale.z, 0.0f, top);
                const uint32_t qx = f2u(nx), qy = f2u(ny), qz = f2u(nz);
                keys[i] = bits == 21 ? (spread21(qx) << 2) | (spread21(qy) << 1) | spread21(qz)
                                     : (uint64_t)((spread10(qx) << 2) | (spread10(qy) << 1) |
                                                  spread10(qz));
                order[i] = (uint32_t)i;
            }
        });
        radix_sort(keys, order, bits == 21 ? 63 : 30, threads);
    }
    std::vector<uint64_t>().swap(keys);
    std::vector<f3> sorted(n);
    pfor(threads, n, [&](int, uint64_t a, uint64_t b) {
        for (uint64_t i = a; i < b; ++i) sorted[i] = pos[order[i]];
    });
    std::vector<f3>().swap(pos);
    const int L = std::max(1, std::min(lod_levels_in, 8));
    const int divs = std::max(1, divs_in);
    std::vector<uint8_t> lv = lod_levels_mt(sorted, bmin, bmax, L, divs, threads);

    // Per batch (:89-213): the stable level bucketing, AABB, quantisation and
    // cumulative level counts.
    const uint64_t nb = (n + ppb - 1) / ppb;
    pfor(threads, nb, [&](int, uint64_t b0, uint64_t b1) {
        std::vector<uint32_t> o2;
        std::vector<f3> p2;
        std::vector<uint8_t> l2;
        for (uint64_t b = b0; b < b1; ++b) {
            const uint64_t first = b * ppb, end = std::min<uint64_t>(first + ppb, n);
            const size_t m = (size_t)(end - first);
            uint32_t cursor[9] = {0};
            for (uint64_t i = first; i < end; ++i) cursor[(lv[i] & 7) + 1]++;
            for (int l = 1; l < 9; ++l) cursor[l] += cursor[l - 1];
            o2.resize(m);
            p2.resize(m);
            l2.resize(m);
            for (uint64_t i = first; i < end; ++i) {
                const uint32_t j = cursor[lv[i] & 7]++;
                o2[j] = order[i];
                p2[j] = sorted[i];
                l2[j] = lv[i];
            }
            std::copy(o2.begin(), o2.end(), order.begin() + first);
            std::copy(p2.begin(), p2.end(), sorted.begin() + first);
            std::copy(l2.begin(), l2.end(), lv.begin() + first);
            f3 mn{3.4028235e38f, 3.4028235e38f, 3.4028235e38f};
            f3 mx{-3.4028235e38f, -3.4028235e38f, -3.4028235e38f};
            for (uint64_t i = first; i < end; ++i) {
                mn = min3(mn, sorted[i]);
                mx = max3(mx, sorted[i]);
            }
            const f3 size{fmax_(mx.x - mn.x, 0.000001f), fmax_(mx.y - mn.y, 0.000001f),
                          fmax_(mx.z - mn.z, 0.000001f)};
            for (uint64_t i = first; i < end; ++i) {
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
            rb.numPoints = (uint32_t)m;
            rb.firstPoint = (uint32_t)first;
            rb.fileIndex = 0;
            uint32_t cum[8] = {0};
            for (uint64_t i = first; i < end; ++i) cum[lv[i] & 7]++;
            for (int l = 1; l < 8; ++l) cum[l] += cum[l - 1];
            rb.lodCum01 = cum[0] | (cum[1] << 16);
            rb.lodCum23 = cum[2] | (cum[3] << 16);
            rb.lodCum45 = cum[4] | (cum[5] << 16);
            rb.lodCum67 = cum[6] | (cum[7] << 16);
            batches[b] = rb;
        }
    });

    // Colours in final order (:145-151).
    pfor(threads, n, [&](int, uint64_t a, uint64_t b) {
        for (uint64_t i = a; i < b; ++i) {
            const uint32_t s = order[i];
            if (colors_rgba8) {
                colors[i] = colors_rgba8[s];
            } else {
                const float *c = &colors_f32[(size_t)s * 4];
                const uint32_t r = f2u(clampf_(c[0], 0.0f, 1.0f) * 255.0f);
                const uint32_t g = f2u(clampf_(c[1], 0.0f, 1.0f) * 255.0f);
                const uint32_t bl = f2u(clampf_(c[2], 0.0f, 1.0f) * 255.0f);
                const uint32_t al = f2u(clampf_(c[3], 0.0f, 1.0f) * 255.0f);
                colors[i] = r | (g << 8) | (bl << 16) | (al << 24);
            }
            levels[i] = lv[i];
            if (source_indices) source_indices[i] = s;
            if (ordered_positions) {
                ordered_positions[i * 3 + 0] = sorted[i].x;
                ordered_positions[i * 3 + 1] = sorted[i].y;
                ordered_positions[i * 3 + 2] = sorted[i].z;
            }
        }
    });
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
