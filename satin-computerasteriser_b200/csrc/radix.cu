// radix.cu — stable LSD radix sort of (key, index) pairs for the packer.
//
// The reference packer (Pipelines/GPUPacker/Shaders.metal:134-215) sorts
// 30-bit Morton keys with four 8-bit passes, one *thread* per 1024-key tile
// walking the tile serially so histogram and scatter agree on order.  Here
// the sort reads the keys once for the histograms of every digit, then runs
// one kernel per 8-bit digit that reads each key and value once and writes
// them once (a single-sweep pass with decoupled look-back):
//   radix_histograms  one read of all keys: the 256-bin histogram of every
//                     digit position; the host reads them back, skips the
//                     passes whose digit is the same for every key and turns
//                     the rest into digit bases (exclusive scans);
//   radix_onesweep    per pass, 4096-key tiles taken in ticket order: a tile
//                     ranks its keys among equal digits in input order (warp
//                     multisplit with ballots, then scans over warps and
//                     digits), publishes its per-digit counts, sums the
//                     counts of the tiles before it per digit (look-back over
//                     their published counts and inclusive prefixes, a
//                     thread per digit), sorts the tile by digit in shared
//                     memory and writes one coalesced run per digit.  Equal
//                     keys keep their input order (stable), as the CPU's
//                     stable sort does.
// A tile waits only for tiles with smaller tickets, which started before it,
// so the waits end whatever the GPU schedules; each wait is nevertheless
// bounded (kLookbackLimit polls), after which the tile counts the missing
// predecessor as empty and stores kErrSortWait into the status word, which
// the host reports as CR_ERR_TIMEOUT.
#include <algorithm>
#include <cstring>
#include <vector>

#include "cr_internal.h"
#include "cr_pack.h"

namespace {

constexpr int kThreads = 256;  // one thread per digit in the per-digit phases
constexpr int kWarps = kThreads / 32;
constexpr int kKeysPerLane = 16;
constexpr int kTileKeys = kThreads * kKeysPerLane;  // 4096
constexpr uint32_t kLookbackLimit = 1u << 22;

// Look-back word of one (tile, digit): epoch (16 bits) | flag (2 bits) |
// count (46 bits).  Flag 1: the tile's own count; flag 2: the inclusive count
// over the tiles up to and including it.
constexpr unsigned long long kFlagAgg = 1ull, kFlagPrefix = 2ull;
__device__ __forceinline__ unsigned long long lookback_word(uint32_t epoch, unsigned long long flag,
                                                            unsigned long long count) {
    return ((unsigned long long)epoch << 48) | (flag << 46) | count;
}
// The look-back words carry their data (the counts) in the word itself, so
// relaxed loads and stores at GPU scope suffice (no other memory is read
// through them).
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ bool lookback_ready(unsigned long long v, uint32_t epoch) {
    return (uint32_t)(v >> 48) == epoch && ((v >> 46) & 3ull) != 0ull;
}
#ifndef CR_LOOKBACK_BATCH
#define CR_LOOKBACK_BATCH 8
#endif
constexpr int kLookbackBatch = CR_LOOKBACK_BATCH;  // predecessor words one round loads at once
// Per-warp digit counts and bases (at most kTileKeys) in 16 bits: 55.4 KB of
// shared memory and at most 64 registers let four sort CTAs share an SM.
using WarpCount = uint16_t;
constexpr int kSortBlocksPerSM = 4;

// Histograms of every 8-bit digit of the keys (grid-stride, per-CTA shared
// counts added to global memory once per CTA).
template <typename K>
__global__ void __launch_bounds__(kThreads)
    radix_histograms(const K *__restrict__ keys, uint64_t n, int passes,
                     uint32_t *__restrict__ hist) {
    __shared__ uint32_t sh[8 * 256];
    for (int i = threadIdx.x; i < passes * 256; i += kThreads) sh[i] = 0u;
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * kThreads) {
        const K k = keys[i];
        for (int p = 0; p < passes; ++p)
            atomicAdd(&sh[p * 256 + ((uint32_t)(k >> (8 * p)) & 0xffu)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kThreads)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// The values of a sort that ran no pass: their input positions.
__global__ void __launch_bounds__(kThreads) radix_iota(uint32_t *__restrict__ vals, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    if (i < n) vals[i] = (uint32_t)i;
}

// Inclusive warp scan.
__device__ __forceinline__ uint32_t warp_inclusive(uint32_t x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

template <typename K>
size_t onesweep_smem_bytes() {
    return (size_t)kTileKeys * (sizeof(K) + sizeof(uint32_t)) +
           (size_t)kWarps * 256 * sizeof(WarpCount) + (256 + 256 + 32) * sizeof(uint32_t);
}

// One pass: a tile of kTileKeys keys per CTA, in ticket order.
//   1. each warp takes 512 consecutive keys, 16 per lane in warp-striped order
//      (key j*32 + lane), and ranks them among equal digits (peer lanes found
//      by ballots) against running per-warp digit counts, in input order;
//   2. thread d: the tile's count of digit d (published at once) and the
//      exclusive bases of the warps;
//   3. exclusive scan over the digits gives each key its slot in a tile
//      sorted by digit; keys and values move there in shared memory; then
//      thread d sums the counts of the tiles before it (look-back) and
//      publishes the inclusive prefix;
//   4. threads read the sorted tile in order and write each key to its
//      digit's global offset: keys of one digit are consecutive in shared
//      memory and land at consecutive addresses (coalesced runs).
template <typename K, bool kIota>
__global__ void __launch_bounds__(kThreads, kSortBlocksPerSM)
    radix_onesweep(const K *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                   K *__restrict__ keys_out, uint32_t *__restrict__ vals_out, uint64_t n,
                   int shift, const uint32_t *__restrict__ digit_base,
                   unsigned long long *__restrict__ lookback, uint32_t epoch,
                   uint32_t *__restrict__ tile_counter, uint32_t *status) {
    extern __shared__ __align__(16) unsigned char smem[];
    K *skey = reinterpret_cast<K *>(smem);
    uint32_t *sval = reinterpret_cast<uint32_t *>(skey + kTileKeys);
    // [kWarps][256]: per-warp digit counts, then the warps' digit bases.
    WarpCount *wcnt = reinterpret_cast<WarpCount *>(sval + kTileKeys);
    // Global offset of the tile's run of each digit.
    uint32_t *offset = reinterpret_cast<uint32_t *>(wcnt + kWarps * 256);
    uint32_t *tbase = offset + 256;          // tile-local digit base
    uint32_t *misc = tbase + 256;            // [0] ticket, [1..8] warp sums of the digit scan
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    if (threadIdx.x == 0) misc[0] = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < kWarps * 256; i += kThreads) wcnt[i] = 0u;
    __syncthreads();
    const uint32_t tile = misc[0];
    const uint64_t tile0 = (uint64_t)tile * kTileKeys;
    const uint32_t tile_n =
        (n - tile0 < (uint64_t)kTileKeys) ? (uint32_t)(n - tile0) : (uint32_t)kTileKeys;
    // 1. Warp-level ranking in input order; a key's rank within its warp
    //    (< 512) and digit are kept packed, the key and value are read again
    //    (from L1 / L2) when they move.
    uint32_t rd[kKeysPerLane];
    WarpCount *wc = wcnt + warp * 256;
#pragma unroll
    for (int j = 0; j < kKeysPerLane; ++j) {
        const uint32_t li = (uint32_t)warp * (32 * kKeysPerLane) + (uint32_t)j * 32 + lane;
        const bool v = li < tile_n;
        const K key = v ? keys_in[tile0 + li] : K(0);
        const uint32_t d = v ? ((uint32_t)(key >> shift) & 0xffu) : 256u;
        // Lanes with the same digit (9 bits: the digit and the no-key flag):
        // the intersection, over the bits, of the lanes that agree with this
        // lane's bit.  (Nine ballots cost less than __match_any_sync when a
        // warp holds many distinct digits.)
        uint32_t peers = 0xffffffffu;
#pragma unroll
        for (int b = 0; b < 9; ++b) {
            const uint32_t m = __ballot_sync(0xffffffffu, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? m : ~m;
        }
        const uint32_t before = v ? wc[d] : 0u;
        rd[j] = (before + __popc(peers & lt)) | (d << 16);
        __syncwarp();
        if (v && (peers & lt) == 0u) wc[d] = (WarpCount)(before + __popc(peers));
        __syncwarp();
    }
    __syncthreads();
    // 2. Digit d = thread: the tile's count and the warps' exclusive bases.
    const uint32_t dd = threadIdx.x;
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const uint32_t c = wcnt[w * 256 + dd];
        wcnt[w * 256 + dd] = (WarpCount)total;
        total += c;
    }
    unsigned long long *my = lookback + (size_t)tile * 256 + dd;
    // Publish the tile's count first (tile 0: its prefix), so that the tiles
    // after it can go on while this one sorts its keys.
    st_relaxed64(my, lookback_word(epoch, tile == 0 ? kFlagPrefix : kFlagAgg, total));
    // 3. Exclusive scan of the tile's digit counts (a warp scan per 32
    //    digits, then over the warps).
    const uint32_t incl = warp_inclusive(total, lane);
    if (lane == 31) misc[1 + warp] = incl;
    __syncthreads();
    uint32_t wbase = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w)
        if (w < warp) wbase += misc[1 + w];
    tbase[dd] = wbase + incl - total;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kKeysPerLane; ++j) {
        const uint32_t li = (uint32_t)warp * (32 * kKeysPerLane) + (uint32_t)j * 32 + lane;
        if (li < tile_n) {
            const uint32_t d = rd[j] >> 16;
            const uint32_t slot = tbase[d] + wcnt[warp * 256 + d] + (rd[j] & 0xffffu);
            skey[slot] = keys_in[tile0 + li];
            sval[slot] = kIota ? (uint32_t)(tile0 + li) : vals_in[tile0 + li];
        }
    }
    // The look-back (thread d, digit d) over the tiles before this one, after
    // the tile-local work so that its waits overlap it.
    unsigned long long excl = 0;
    if (tile != 0) {
        // Look-back over the tiles before this one, kLookbackBatch words per
        // round (independent loads), newest first: add counts until a tile's
        // inclusive prefix; a word not yet published is polled (bounded).
        constexpr unsigned long long kCountMask = (1ull << 46) - 1ull;
        bool gave_up = false;
        int64_t t = (int64_t)tile - 1;
        while (t >= 0) {
            const int nb = t + 1 < kLookbackBatch ? (int)(t + 1) : kLookbackBatch;
            unsigned long long v[kLookbackBatch];
#pragma unroll
            for (int k = 0; k < kLookbackBatch; ++k)
                if (k < nb) v[k] = ld_relaxed64(lookback + (size_t)(t - k) * 256 + dd);
            // Add the batch's counts up to the first inclusive prefix (pf)
            // or the first word not yet published (nr).
            int nr = -1;
            bool pf = false;
#pragma unroll
            for (int k = 0; k < kLookbackBatch; ++k) {
                if (k < nb && nr < 0 && !pf) {
                    if (!lookback_ready(v[k], epoch)) {
                        nr = k;
                    } else {
                        excl += v[k] & kCountMask;
                        pf = ((v[k] >> 46) & 3ull) == kFlagPrefix;
                    }
                }
            }
            if (pf) break;
            if (nr < 0) {
                t -= nb;
                continue;
            }
            // Poll the unpublished predecessor, then carry on from the one
            // before it.
            const unsigned long long *w = lookback + (size_t)(t - nr) * 256 + dd;
            uint32_t polls = 0;
            unsigned long long x = ld_relaxed64(w);
            while (!lookback_ready(x, epoch) && ++polls < kLookbackLimit) {
                __nanosleep(32);
                x = ld_relaxed64(w);
            }
            if (!lookback_ready(x, epoch)) {
                gave_up = true;
                break;
            }
            excl += x & kCountMask;
            if (((x >> 46) & 3ull) == kFlagPrefix) break;
            t -= nr + 1;
        }
        if (gave_up && status) *(volatile uint32_t *)status = kErrSortWait;
        st_relaxed64(my, lookback_word(epoch, kFlagPrefix, excl + total));
    }
    offset[dd] = digit_base[dd] + (uint32_t)excl;
    __syncthreads();  // every digit's offset; the sorted tile complete
    // 4. Coalesced runs per digit to the global output.
    for (uint32_t i = threadIdx.x; i < tile_n; i += kThreads) {
        const K k = skey[i];
        const uint32_t d = (uint32_t)(k >> shift) & 0xffu;
        const uint64_t dst = (uint64_t)offset[d] + (i - tbase[d]);
        if (dst < n) {  // always true when the counts are consistent
            keys_out[dst] = k;
            vals_out[dst] = sval[i];
        }
    }
}

}  // namespace

void radix_scratch_free(RadixScratch &r) {
    void *ptrs[] = {r.lookback, r.hist, r.bases, r.tiles};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    r = RadixScratch{};
}

template <typename K>
cr_status radix_sort_pairs(K *keys, uint32_t *vals, K *keys_alt, uint32_t *vals_alt, uint64_t n,
                           int key_bits, bool vals_iota, RadixScratch &rs, uint32_t *status,
                           int sm_count, cudaStream_t s, bool *result_in_alt) {
    *result_in_alt = false;
    if (n <= 1) {
        if (vals_iota && n == 1) CR_CUDA(cudaMemsetAsync(vals, 0, sizeof(uint32_t), s));
        return CR_OK;
    }
    if (n >= (1ull << 32)) return cri::fail(CR_ERR_CAPACITY, "radix sort: at most 2^32 - 1 keys");
    const int passes = (key_bits + 7) / 8;
    const uint64_t ntiles = (n + kTileKeys - 1) / kTileKeys;
    // Scratch: look-back words (tiles x 256), histograms and bases (8 x 256),
    // tile tickets (one per pass).
    if (!rs.lookback || rs.cap_tiles < ntiles) {
        radix_scratch_free(rs);
        CR_CUDA(cudaMalloc((void **)&rs.lookback, ntiles * 256 * sizeof(unsigned long long)));
        CR_CUDA(cudaMalloc((void **)&rs.hist, 8 * 256 * sizeof(uint32_t)));
        CR_CUDA(cudaMalloc((void **)&rs.bases, 8 * 256 * sizeof(uint32_t)));
        CR_CUDA(cudaMalloc((void **)&rs.tiles, 8 * sizeof(uint32_t)));
        CR_CUDA(cudaMemsetAsync(rs.lookback, 0, ntiles * 256 * sizeof(unsigned long long), s));
        rs.cap_tiles = ntiles;
        rs.epoch = 0;
    }
    CR_CUDA(cudaMemsetAsync(rs.hist, 0, 8 * 256 * sizeof(uint32_t), s));
    CR_CUDA(cudaMemsetAsync(rs.tiles, 0, 8 * sizeof(uint32_t), s));
    const unsigned hgrid = (unsigned)std::min<uint64_t>((n + kThreads - 1) / kThreads,
                                                        (uint64_t)std::max(sm_count, 1) * 8);
    radix_histograms<K><<<hgrid, kThreads, 0, s>>>(keys, n, passes, rs.hist);
    CR_CUDA(cudaGetLastError());
    // The histograms on the host: skip the passes whose digit every key
    // shares, exclusive scans into the digit bases of the others.
    std::vector<uint32_t> hist(8 * 256), bases(8 * 256, 0u);
    CR_CUDA(cudaMemcpyAsync(hist.data(), rs.hist, passes * 256 * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    std::vector<int> run;
    for (int p = 0; p < passes; ++p) {
        uint32_t acc = 0;
        bool constant = false;
        for (int d = 0; d < 256; ++d) {
            bases[p * 256 + d] = acc;
            acc += hist[p * 256 + d];
            if (hist[p * 256 + d] == n) constant = true;
        }
        if (!constant) run.push_back(p);
    }
    CR_CUDA(cudaMemcpyAsync(rs.bases, bases.data(), passes * 256 * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s));
    const size_t smem = onesweep_smem_bytes<K>();
    for (auto *f : {radix_onesweep<K, false>, radix_onesweep<K, true>})
        CR_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (run.empty() && vals_iota) {
        radix_iota<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(vals, n);
        CR_CUDA(cudaGetLastError());
    }
    K *kin = keys, *kout = keys_alt;
    uint32_t *vin = vals, *vout = vals_alt;
    for (int p : run) {
        // A fresh epoch per pass, so the look-back words never need clearing;
        // after 65534 epochs the words are cleared once.
        if (++rs.epoch >= 0xffffu) {
            CR_CUDA(cudaMemsetAsync(rs.lookback, 0,
                                    rs.cap_tiles * 256 * sizeof(unsigned long long), s));
            rs.epoch = 1;
        }
        // The first pass of an index sort makes the indices (kIota).
        auto *kern = vals_iota && p == run.front() ? radix_onesweep<K, true>
                                                   : radix_onesweep<K, false>;
        kern<<<(unsigned)ntiles, kThreads, smem, s>>>(kin, vin, kout, vout, n, 8 * p,
                                                     rs.bases + p * 256, rs.lookback, rs.epoch,
                                                     rs.tiles + p, status);
        CR_CUDA(cudaGetLastError());
        std::swap(kin, kout);
        std::swap(vin, vout);
        *result_in_alt = !*result_in_alt;
    }
    return CR_OK;
}

template cr_status radix_sort_pairs<uint32_t>(uint32_t *, uint32_t *, uint32_t *, uint32_t *,
                                              uint64_t, int, bool, RadixScratch &, uint32_t *,
                                              int, cudaStream_t, bool *);
template cr_status radix_sort_pairs<unsigned long long>(unsigned long long *, uint32_t *,
                                                        unsigned long long *, uint32_t *, uint64_t,
                                                        int, bool, RadixScratch &, uint32_t *, int,
                                                        cudaStream_t, bool *);
