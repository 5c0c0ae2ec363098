// Stable LSD radix sort of (key, uint32 value) pairs, 8-bit digits.
//
// Per digit pass: (1) per-tile digit histograms, (2) a device-wide exclusive
// scan of the histograms in digit-major order gives every (digit, tile) its
// output offset, (3) each tile ranks its items stably — warps take 32
// consecutive items per round and rank equal digits with __match_any_sync —
// stages them in shared memory in digit order and writes them out in runs.
#pragma once

#include "scan.cuh"

namespace pb {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 8;                                 // items per lane
constexpr int kSortTile = kSortThreads * kSortRounds;          // 2048 items per tile
constexpr int kSortWarpItems = 32 * kSortRounds;               // 256 consecutive items per warp
constexpr unsigned kNoDigit = 256u;

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_histogram(const K* __restrict__ keys, int64_t count,
                                                                int shift, uint32_t* __restrict__ counts,
                                                                uint32_t tiles) {
    __shared__ uint32_t hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int k = threadIdx.x; k < kSortTile; k += kSortThreads) {
        int64_t i = base + k;
        if (i < count) atomicAdd(&hist[(unsigned)(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    counts[(int64_t)threadIdx.x * tiles + blockIdx.x] = hist[threadIdx.x];
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_scatter(const K* __restrict__ keys_in,
                                                              const uint32_t* __restrict__ vals_in,
                                                              K* __restrict__ keys_out,
                                                              uint32_t* __restrict__ vals_out, int64_t count,
                                                              int shift, const uint32_t* __restrict__ offsets,
                                                              uint32_t tiles) {
    __shared__ uint32_t warp_hist[kSortWarps][256];
    __shared__ uint32_t digit_start[256];
    __shared__ uint32_t warp_sums[32];
    __shared__ K s_keys[kSortTile];
    __shared__ uint32_t s_vals[kSortTile];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < kSortWarps * 256; k += kSortThreads) (&warp_hist[0][0])[k] = 0;
    __syncthreads();

    const int64_t tile_base = (int64_t)blockIdx.x * kSortTile;
    const int64_t warp_base = tile_base + (int64_t)warp * kSortWarpItems;
    const unsigned lt_mask = (1u << lane) - 1u;
    K key[kSortRounds];
    uint32_t val[kSortRounds];
    uint32_t rank[kSortRounds];
    unsigned dig[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        int64_t i = warp_base + r * 32 + lane;
        bool valid = i < count;
        key[r] = valid ? keys_in[i] : K(0);
        val[r] = valid ? vals_in[i] : 0u;
        unsigned d = valid ? ((unsigned)(key[r] >> shift) & 255u) : kNoDigit;
        dig[r] = d;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int leader = __ffs(peers) - 1;
        uint32_t before = 0;
        if (lane == leader && d != kNoDigit) {
            before = warp_hist[warp][d];
            warp_hist[warp][d] = before + __popc(peers);
        }
        before = __shfl_sync(0xffffffffu, before, leader);
        rank[r] = before + __popc(peers & lt_mask);
        __syncwarp();
    }
    __syncthreads();
    // Per digit: exclusive offsets of the warps, then the tile's digit totals.
    uint32_t digit_total = 0;
    {
        const unsigned d = threadIdx.x;  // kSortThreads == 256 digits
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t t = warp_hist[w][d];
            warp_hist[w][d] = run;
            run += t;
        }
        digit_total = run;
    }
    uint32_t tile_total;
    uint32_t start = block_exclusive_scan<uint32_t>(digit_total, warp_sums, tile_total);
    digit_start[threadIdx.x] = start;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        if (dig[r] == kNoDigit) continue;
        uint32_t pos = digit_start[dig[r]] + warp_hist[warp][dig[r]] + rank[r];
        s_keys[pos] = key[r];
        s_vals[pos] = val[r];
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < tile_total; j += kSortThreads) {
        K k = s_keys[j];
        unsigned d = (unsigned)(k >> shift) & 255u;
        int64_t out = (int64_t)offsets[(int64_t)d * tiles + blockIdx.x] + (j - digit_start[d]);
        keys_out[out] = k;
        vals_out[out] = s_vals[j];
    }
}

template <typename K>
void radix_carve(Workspace& ws, int64_t count) {
    int64_t tiles = (count + kSortTile - 1) / kSortTile;
    ws.take<uint32_t>(tiles * 256);
    scan_carve<uint32_t>(ws, tiles * 256);
}

// Sorts (keys, vals) by bits [0, bits) of the key, stably.  Ping-pongs between
// the primary and alternate buffers; *result_in_alt says where the result is.
template <typename K>
int radix_sort_pairs(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt, int64_t count, int bits,
                     bool* result_in_alt, Workspace& ws, cudaStream_t s) {
    *result_in_alt = false;
    if (count <= 1 || bits <= 0) return PB_OK;
    if (count > (int64_t)0xFFFFFFFFll) return fail(PB_ERR_INVALID, "radix sort: too many items");
    int64_t tiles = (count + kSortTile - 1) / kSortTile;
    uint32_t* counts = ws.take<uint32_t>(tiles * 256);
    if (!ws.fits()) return fail(PB_ERR_WORKSPACE, "radix sort workspace too small");
    K* src_k = keys;
    uint32_t* src_v = vals;
    K* dst_k = keys_alt;
    uint32_t* dst_v = vals_alt;
    for (int shift = 0; shift < bits; shift += 8) {
        radix_histogram<K><<<(unsigned)tiles, kSortThreads, 0, s>>>(src_k, count, shift, counts, (uint32_t)tiles);
        PB_CHECK_LAUNCH("radix_histogram");
        Workspace sub = ws;  // scan scratch is transient per pass
        PB_TRY(exclusive_scan<uint32_t>(counts, counts, tiles * 256, nullptr, sub, s));
        radix_scatter<K><<<(unsigned)tiles, kSortThreads, 0, s>>>(src_k, src_v, dst_k, dst_v, count, shift, counts,
                                                                  (uint32_t)tiles);
        PB_CHECK_LAUNCH("radix_scatter");
        K* tk = src_k; src_k = dst_k; dst_k = tk;
        uint32_t* tv = src_v; src_v = dst_v; dst_v = tv;
        *result_in_alt = !*result_in_alt;
    }
    return PB_OK;
}

}  // namespace pb
