// Device-wide exclusive prefix sum (reduce-then-scan, recursive over tiles).
#pragma once

#include "common.cuh"

namespace pb {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096 elements per block

// Exclusive scan of one value per thread across the block; returns the block total.
template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T value, T* warp_sums /*[32]*/, T& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    T inclusive = value;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, inclusive, o);
        if (lane >= o) inclusive += t;
    }
    if (lane == 31) warp_sums[warp] = inclusive;
    __syncthreads();
    if (warp == 0) {
        T w = lane < warps ? warp_sums[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < warps) warp_sums[lane] = wi - w;  // exclusive warp offsets
        if (lane == 31) warp_sums[31] = wi;          // block total (warps <= 31 used)
    }
    __syncthreads();
    total = warp_sums[31];
    T result = warp_sums[warp] + inclusive - value;
    __syncthreads();
    return result;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_tiles(const T* __restrict__ in, int64_t n,
                                                                 T* __restrict__ partial) {
    __shared__ T warp_sums[32];
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    T s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += in[base + k];
    T total;
    block_exclusive_scan<T>(s, warp_sums, total);
    if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// out[i] = offset(block) + exclusive sum within the block.  `in` may equal `out`.
template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_tiles(const T* in, T* out, int64_t n,
                                                          const T* __restrict__ block_offsets,
                                                          T* __restrict__ grand_total) {
    __shared__ T warp_sums[32];
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    T v[kScanItems];
    T s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : T(0);
        s += v[k];
    }
    T total;
    T run = block_exclusive_scan<T>(s, warp_sums, total);
    T off = block_offsets ? block_offsets[blockIdx.x] : T(0);
    run += off;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (grand_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *grand_total = off + total;
}

template <typename T>
void scan_carve(Workspace& ws, int64_t n) {
    while (n > kScanTile) {
        int64_t tiles = (n + kScanTile - 1) / kScanTile;
        ws.take<T>(tiles);
        n = tiles;
    }
}

template <typename T>
size_t scan_workspace(int64_t n) {
    return measure([&](Workspace& w) { scan_carve<T>(w, n); });
}

// Exclusive scan of in[0..n) into out (in-place allowed).  *grand_total (device,
// optional) receives the sum of all n inputs.  Scratch is carved from ws.
template <typename T>
int exclusive_scan(const T* in, T* out, int64_t n, T* grand_total, Workspace& ws, cudaStream_t s) {
    if (n <= 0) {
        if (grand_total) PB_CHECK_CUDA(cudaMemsetAsync(grand_total, 0, sizeof(T), s), "scan total");
        return PB_OK;
    }
    if (n <= kScanTile) {
        scan_tiles<T><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, grand_total);
        PB_CHECK_LAUNCH("scan_tiles");
        return PB_OK;
    }
    int64_t tiles = (n + kScanTile - 1) / kScanTile;
    T* partial = ws.take<T>(tiles);
    if (!ws.fits()) return fail(PB_ERR_WORKSPACE, "scan workspace too small");
    scan_reduce_tiles<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, partial);
    PB_CHECK_LAUNCH("scan_reduce_tiles");
    PB_TRY(exclusive_scan<T>(partial, partial, tiles, nullptr, ws, s));
    scan_tiles<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, partial, grand_total);
    PB_CHECK_LAUNCH("scan_tiles");
    return PB_OK;
}

}  // namespace pb
