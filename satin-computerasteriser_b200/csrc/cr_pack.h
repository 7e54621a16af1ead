// cr_pack.h — internal interface of the GPU packer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cr/cr.h"

template <typename K>
cr_status radix_sort_pairs(K *keys, uint32_t *vals, K *keys_alt, uint32_t *vals_alt, uint64_t n,
                           int key_bits, uint32_t *hist, uint32_t *digit_total, cudaStream_t s,
                           bool *result_in_alt);
uint64_t radix_hist_words(uint64_t n);

// Grow-only device scratch of the packer, owned by the context (the
// reference's PackScratch, GPUPacker.swift:453-484).
struct PackScratch {
    uint64_t cap_points = 0;
    uint64_t cap_raw_bytes = 0;
    uint64_t cap_grid = 0;
    uint64_t cap_hist = 0;
    void *raw = nullptr;                    // staged host input
    float4 *pos = nullptr;                  // input x, y, z and RGBA8 bits in w
    void *keys[2] = {nullptr, nullptr};     // Morton keys (u32 or u64), ping-pong
    uint32_t *idx[2] = {nullptr, nullptr};  // sort payload, ping-pong
    float4 *sorted = nullptr;               // positions in Morton order
    uint8_t *lv_morton = nullptr;           // levels in Morton order
    uint8_t *lv_out = nullptr;              // levels in final order
    uint32_t *perm = nullptr;               // final order -> Morton position
    uint32_t *grid = nullptr;               // dense LOD occupancy grid
    uint32_t *hist = nullptr;               // radix histograms
    uint32_t *digit_total = nullptr;        // 256 digit totals
    uint32_t *bounds = nullptr;             // 6 flipped words: min xyz, max xyz
    uint32_t *src_idx = nullptr;            // final order -> input index
};

void pack_scratch_free(PackScratch &s);
