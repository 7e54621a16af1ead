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
//   scatter  each partition re-reads its keys in rounds of 256; lanes rank
//            themselves among equal digits with __match_any_sync, warps are
//            ordered through shared memory, so equal keys keep their input
//            order (stable), as the CPU's stable sort does.
// 32-bit keys (30-bit Morton) take 4 passes, 64-bit keys (63-bit Morton) 8.
#include <algorithm>

#include "cr_internal.h"
#include "cr_pack.h"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kPartition = 16384;
constexpr int kRounds = kPartition / kThreads;

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

template <typename K>
__global__ void __launch_bounds__(kThreads)
    radix_scatter(const K *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                  K *__restrict__ keys_out, uint32_t *__restrict__ vals_out, uint64_t n, int shift,
                  const uint32_t *__restrict__ hist, uint32_t nparts,
                  const uint32_t *__restrict__ digit_total) {
    __shared__ uint32_t offset[256];       // running global offset per digit
    __shared__ uint32_t wcount[kWarps][256];
    __shared__ uint32_t scan_tmp[256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // Digit bases: exclusive scan of the 256 digit totals.
    {
        const uint32_t t = digit_total[threadIdx.x];
        scan_tmp[threadIdx.x] = t;
        __syncthreads();
        for (int o = 1; o < 256; o <<= 1) {
            const uint32_t y = threadIdx.x >= (unsigned)o ? scan_tmp[threadIdx.x - o] : 0u;
            __syncthreads();
            scan_tmp[threadIdx.x] += y;
            __syncthreads();
        }
        offset[threadIdx.x] =
            scan_tmp[threadIdx.x] - t + hist[(size_t)threadIdx.x * nparts + blockIdx.x];
    }
    for (int i = threadIdx.x; i < kWarps * 256; i += kThreads) (&wcount[0][0])[i] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kPartition;
    const uint32_t lt = (1u << lane) - 1u;
    for (int r = 0; r < kRounds; ++r) {
        const uint64_t i = base + (uint64_t)r * kThreads + threadIdx.x;
        if (base + (uint64_t)r * kThreads >= n) break;  // uniform across the CTA
        const bool v = i < n;
        K k = 0;
        uint32_t val = 0;
        if (v) {
            k = keys_in[i];
            val = vals_in[i];
        }
        const uint32_t d = v ? ((uint32_t)(k >> shift) & 0xffu) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & lt);
        if (v && rank == 0) wcount[warp][d] = __popc(peers);
        __syncthreads();
        uint32_t before = 0;
        if (v) {
            for (int w = 0; w < warp; ++w) before += wcount[w][d];
            const uint64_t dst = (uint64_t)offset[d] + before + rank;
            if (dst < n) {  // always true when the histograms are consistent
                keys_out[dst] = k;
                vals_out[dst] = val;
            }
        }
        __syncthreads();
        {
            uint32_t s = 0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                s += wcount[w][threadIdx.x];
                wcount[w][threadIdx.x] = 0;
            }
            offset[threadIdx.x] += s;
        }
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
        radix_scatter<K><<<nparts, kThreads, 0, s>>>(kin, vin, kout, vout, n, shift, hist, nparts,
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
