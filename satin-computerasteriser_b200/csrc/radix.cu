// radix.cu — stable LSD radix sort of (key, index) pairs for the packer.
//
// The reference packer (Pipelines/GPUPacker/Shaders.metal:134-215) sorts
// 30-bit Morton keys with four 8-bit passes, one *thread* per 1024-key tile
// walking the tile serially so histogram and scatter agree on order.  Here
// each pass is three kernels over 16384-key partitions, all threads busy:
//   upsweep  per-partition 256-bin histogram (per-warp sub-histograms in
//            shared memory), written digit-major;
//   scan     one CTA per digit turns its row into exclusive partition
//            offsets and the digit total;
//   scatter  each partition re-reads its keys in tiles of 4096, ranks them
//            among equal digits in input order (warp multisplit with
//            __match_any_sync, then scans over warps and digits), sorts the
//            tile by digit in shared memory and writes one coalesced run per
//            digit, so equal keys keep their input order (stable), as the
//            CPU's stable sort does.
// 32-bit keys (30-bit Morton) take 4 passes, 64-bit keys (63-bit Morton) 8.
#include <algorithm>

#include "cr_internal.h"
#include "cr_pack.h"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kPartition = 16384;

template <typename K>
__global__ void __launch_bounds__(kThreads)
    radix_upsweep(const K *__restrict__ keys, uint64_t n, int shift, uint32_t *__restrict__ hist,
                  uint32_t nparts) {
    __shared__ uint32_t sh[kWarps][256];
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kWarps * 256; i += kThreads) (&sh[0][0])[i] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kPartition;
    const uint64_t end = (base + kPartition < n) ? base + kPartition : n;
    for (uint64_t i = base + threadIdx.x; i < end; i += kThreads) {
        const uint32_t d = (uint32_t)(keys[i] >> shift) & 0xffu;
        atomicAdd(&sh[warp][d], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += kThreads) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += sh[w][d];
        hist[(size_t)d * nparts + blockIdx.x] = s;
    }
}

// One CTA per digit: exclusive scan of hist[d][0..nparts) in place, total out.
__global__ void __launch_bounds__(1024)
    radix_scan(uint32_t *__restrict__ hist, uint32_t nparts, uint32_t *__restrict__ digit_total) {
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t carry;
    uint32_t *row = hist + (size_t)blockIdx.x * nparts;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t c0 = 0; c0 < nparts; c0 += 1024) {
        const uint32_t i = c0 + threadIdx.x;
        const uint32_t v = i < nparts ? row[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t s = warp_sums[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            warp_sums[lane] = s;  // inclusive over warps
        }
        __syncthreads();
        const uint32_t before = (warp > 0 ? warp_sums[warp - 1] : 0u) + (x - v);
        if (i < nparts) row[i] = carry + before;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_sums[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) digit_total[blockIdx.x] = carry;
}

// Scatter of one pass, a partition per CTA in tiles of kTileKeys keys:
//   1. each warp takes 512 consecutive keys, 16 per lane in warp-striped
//      order (key j*32 + lane), and ranks them among equal digits with
//      __match_any_sync against running per-warp digit counts, in input
//      order (j, then lane);
//   2. per digit, exclusive scans over the warps and then over the digits
//      give each key its slot in a tile sorted by digit, stable;
//   3. the keys and values move to that slot in shared memory;
//   4. threads read the sorted tile in order and write each key to its
//      digit's running global offset: keys of one digit are consecutive in
//      shared memory and land at consecutive addresses (coalesced runs).
constexpr int kKeysPerLane = 16;
constexpr int kTileKeys = kThreads * kKeysPerLane;
static_assert(kPartition % kTileKeys == 0, "a partition is whole tiles");

template <typename K>
size_t scatter_smem_bytes() {
    return (size_t)kTileKeys * (sizeof(K) + sizeof(uint32_t)) +
           ((size_t)kWarps * 256 + 256 + 256) * sizeof(uint32_t);
}

template <typename K>
__global__ void __launch_bounds__(kThreads)
    radix_scatter(const K *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                  K *__restrict__ keys_out, uint32_t *__restrict__ vals_out, uint64_t n, int shift,
                  const uint32_t *__restrict__ hist, uint32_t nparts,
                  const uint32_t *__restrict__ digit_total) {
    extern __shared__ __align__(16) unsigned char smem[];
    K *skey = reinterpret_cast<K *>(smem);
    uint32_t *sval = reinterpret_cast<uint32_t *>(skey + kTileKeys);
    uint32_t *wcnt = sval + kTileKeys;        // [kWarps][256]
    uint32_t *offset = wcnt + kWarps * 256;   // running global offset per digit
    uint32_t *tbase = offset + 256;           // tile-local digit base
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    // Digit bases: exclusive scan of the 256 digit totals, plus this
    // partition's offset within each digit.
    {
        const uint32_t t = digit_total[threadIdx.x];
        tbase[threadIdx.x] = t;
        __syncthreads();
        for (int o = 1; o < 256; o <<= 1) {
            const uint32_t y = threadIdx.x >= (unsigned)o ? tbase[threadIdx.x - o] : 0u;
            __syncthreads();
            tbase[threadIdx.x] += y;
            __syncthreads();
        }
        offset[threadIdx.x] =
            tbase[threadIdx.x] - t + hist[(size_t)threadIdx.x * nparts + blockIdx.x];
    }
    const uint64_t pbase = (uint64_t)blockIdx.x * kPartition;
    for (uint32_t t0 = 0; t0 < kPartition; t0 += kTileKeys) {
        const uint64_t tile0 = pbase + t0;
        if (tile0 >= n) break;  // uniform across the CTA
        const uint32_t tile_n = (n - tile0 < (uint64_t)kTileKeys) ? (uint32_t)(n - tile0)
                                                                  : (uint32_t)kTileKeys;
        for (int i = threadIdx.x; i < kWarps * 256; i += kThreads) wcnt[i] = 0u;
        __syncthreads();
        // 1. Warp-level ranking in input order; a key's rank within its
        //    warp (< 512) and digit are kept packed, the key and value are
        //    read again (from L1 / L2) when they move.
        uint32_t rd[kKeysPerLane];
        uint32_t *wc = wcnt + warp * 256;
#pragma unroll
        for (int j = 0; j < kKeysPerLane; ++j) {
            const uint32_t li = (uint32_t)warp * (32 * kKeysPerLane) + (uint32_t)j * 32 + lane;
            const bool v = li < tile_n;
            const K key = v ? keys_in[tile0 + li] : K(0);
            const uint32_t d = v ? ((uint32_t)(key >> shift) & 0xffu) : 256u;
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            const uint32_t before = v ? wc[d] : 0u;
            rd[j] = (before + __popc(peers & lt)) | (d << 16);
            __syncwarp();
            if (v && (peers & lt) == 0u) wc[d] = before + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        // 2. Per digit: warp bases (exclusive over warps) and tile bases
        //    (exclusive over digits).
        const uint32_t dd = threadIdx.x;
        uint32_t total = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = wcnt[w * 256 + dd];
            wcnt[w * 256 + dd] = total;
            total += c;
        }
        tbase[dd] = total;
        __syncthreads();
        for (int o = 1; o < 256; o <<= 1) {
            const uint32_t y = dd >= (unsigned)o ? tbase[dd - o] : 0u;
            __syncthreads();
            tbase[dd] += y;
            __syncthreads();
        }
        tbase[dd] -= total;  // inclusive -> exclusive
        __syncthreads();
        // 3. Keys and values to their sorted slots in the tile.
#pragma unroll
        for (int j = 0; j < kKeysPerLane; ++j) {
            const uint32_t li = (uint32_t)warp * (32 * kKeysPerLane) + (uint32_t)j * 32 + lane;
            if (li < tile_n) {
                const uint32_t d = rd[j] >> 16;
                const uint32_t slot = tbase[d] + wcnt[warp * 256 + d] + (rd[j] & 0xffffu);
                skey[slot] = keys_in[tile0 + li];
                sval[slot] = vals_in[tile0 + li];
            }
        }
        __syncthreads();
        // 4. Coalesced runs per digit to the global output.
        for (uint32_t i = threadIdx.x; i < tile_n; i += kThreads) {
            const K k = skey[i];
            const uint32_t d = (uint32_t)(k >> shift) & 0xffu;
            const uint64_t dst = (uint64_t)offset[d] + (i - tbase[d]);
            if (dst < n) {  // always true when the histograms are consistent
                keys_out[dst] = k;
                vals_out[dst] = sval[i];
            }
        }
        __syncthreads();
        offset[dd] += total;
        __syncthreads();
    }
}

}  // namespace

template <typename K>
cr_status radix_sort_pairs(K *keys, uint32_t *vals, K *keys_alt, uint32_t *vals_alt, uint64_t n,
                           int key_bits, uint32_t *hist, uint32_t *digit_total, cudaStream_t s,
                           bool *result_in_alt) {
    *result_in_alt = false;
    if (n <= 1) return CR_OK;
    const uint32_t nparts = (uint32_t)((n + kPartition - 1) / kPartition);
    K *kin = keys, *kout = keys_alt;
    uint32_t *vin = vals, *vout = vals_alt;
    for (int shift = 0; shift < key_bits; shift += 8) {
        radix_upsweep<K><<<nparts, kThreads, 0, s>>>(kin, n, shift, hist, nparts);
        CR_CUDA(cudaGetLastError());
        radix_scan<<<256, 1024, 0, s>>>(hist, nparts, digit_total);
        CR_CUDA(cudaGetLastError());
        const size_t smem = scatter_smem_bytes<K>();
        CR_CUDA(cudaFuncSetAttribute(radix_scatter<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
        radix_scatter<K><<<nparts, kThreads, smem, s>>>(kin, vin, kout, vout, n, shift, hist, nparts,
                                                        digit_total);
        CR_CUDA(cudaGetLastError());
        std::swap(kin, kout);
        std::swap(vin, vout);
        *result_in_alt = !*result_in_alt;
    }
    return CR_OK;
}

uint64_t radix_hist_words(uint64_t n) { return 256ull * ((n + kPartition - 1) / kPartition); }

template cr_status radix_sort_pairs<uint32_t>(uint32_t *, uint32_t *, uint32_t *, uint32_t *,
                                              uint64_t, int, uint32_t *, uint32_t *, cudaStream_t,
                                              bool *);
template cr_status radix_sort_pairs<unsigned long long>(unsigned long long *, uint32_t *,
                                                        unsigned long long *, uint32_t *, uint64_t,
                                                        int, uint32_t *, uint32_t *, cudaStream_t,
                                                        bool *);
