// cr_pack.h — internal interface of the GPU packer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cr/cr.h"

// Grow-only scratch of the radix sort: look-back words (256 per 4096-key
// tile), the histograms and digit bases of up to 8 passes, one tile ticket
// counter per pass, and the epoch of the last pass (look-back words carry it).
struct RadixScratch {
    unsigned long long *lookback = nullptr;
    uint64_t cap_tiles = 0;
    uint32_t *hist = nullptr;
    uint32_t *bases = nullptr;
    uint32_t *tiles = nullptr;
    uint32_t epoch = 0;
};
void radix_scratch_free(RadixScratch &r);

// Stable sort of n (key, value) pairs by the low key_bits bits of the keys;
// the result is in (keys_alt, vals_alt) when *result_in_alt.  With
// vals_iota the values are the keys' input positions and `vals` is not read
// (the first pass makes them).  Synchronises once (the histograms are read
// back to skip constant digits).  A bounded wait that gives up stores
// kErrSortWait into *status.
template <typename K>
cr_status radix_sort_pairs(K *keys, uint32_t *vals, K *keys_alt, uint32_t *vals_alt, uint64_t n,
                           int key_bits, bool vals_iota, RadixScratch &rs, uint32_t *status,
                           int sm_count, cudaStream_t s, bool *result_in_alt);

// Grow-only device scratch of the packer, owned by the context (the
// reference's PackScratch, GPUPacker.swift:453-484).
struct PackScratch {
    uint64_t cap_points = 0;
    uint64_t cap_raw_bytes = 0;
    uint64_t cap_grid = 0;
    void *raw = nullptr;                    // staged host input
    float4 *pos = nullptr;                  // input x, y, z and RGBA8 bits in w
    void *keys[2] = {nullptr, nullptr};     // Morton keys (u32 or u64), ping-pong
    uint32_t *idx[2] = {nullptr, nullptr};  // sort payload, ping-pong
    float4 *sorted = nullptr;               // positions in Morton order
    uint8_t *lv_morton = nullptr;           // levels in Morton order
    uint8_t *lv_out = nullptr;              // levels in final order
    uint32_t *perm = nullptr;               // final order -> Morton position
    uint32_t *grid = nullptr;               // dense LOD occupancy grid
    RadixScratch radix;                     // the sort's look-back words and histograms
    uint32_t *bounds = nullptr;             // 6 flipped words: min xyz, max xyz
    uint32_t *src_idx = nullptr;            // final order -> input index
};

void pack_scratch_free(PackScratch &s);
