// Active-cell count of the dual contour that allocates nothing.
//
// pb_dual_vertices_f64 in count mode needs a caller-provided workspace for its
// per-tile counts.  Some callers cannot provide one: code that runs where the
// device allocator must not be touched (cudaMalloc and cudaFree can block or
// synchronise the whole device, which a latency-critical serving loop or a
// host callback cannot afford), or foreign-language bindings that receive
// device buffers from another framework's pool and have no way to reserve
// extra device memory of their own.  This entry point keeps its scratch in a
// fixed array in the library's device memory instead.
//
// Scratch: kMaxTiles int64 tile counts (512 KiB), resident on every device that
// loads the library until the process exits.  One tile holds 2048 cells, so
// grids up to 134,217,728 cells are accepted: side n <= 513 (depth 9).
// Larger grids are rejected with PB_ERR_INVALID before anything is launched.
//
// Every call on a device shares the one array and leaves its contents behind;
// each call overwrites the tile slots it reads before reading them, so nothing
// has to start at zero.  Two calls whose work overlaps on the GPU (different
// streams, no ordering between them) race on the array and may return wrong
// counts: order such calls on one stream or synchronise between them.
//
// The first call on each device (and CUDA context) looks up the array's device
// address with cudaGetSymbolAddress while that device is current; make that
// first call before any stream capture.  The address is cached per (device,
// context): a call made under another context of the same device (one the
// caller created and made current with the driver API) looks it up again for
// that context.  cudaDeviceReset unloads the library's device memory; do not
// call this entry point on a device after resetting it in the same process.
#include <cuda.h>

#include <mutex>

#include "common.cuh"

namespace pb {
namespace noalloc {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int64_t kTile = kThreads * kItems;  // cells per tile
constexpr int64_t kMaxTiles = 65536;          // 512 KiB of int64 counts
constexpr int kMaxDevices = 64;

static __device__ __align__(256) long long g_tile_counts[kMaxTiles];

__device__ __forceinline__ int active(const double* __restrict__ f, int64_t i0, int64_t n, double iso) {
    const int64_t sy = n, sz = n * n;
    const int below = (f[i0] < iso) + (f[i0 + 1] < iso) + (f[i0 + sy] < iso) + (f[i0 + sy + 1] < iso) +
                      (f[i0 + sz] < iso) + (f[i0 + sz + 1] < iso) + (f[i0 + sz + sy] < iso) +
                      (f[i0 + sz + sy + 1] < iso);
    return below != 0 && below != 8;  // capi.mojo:884, :892
}

__global__ void __launch_bounds__(kThreads) count_tiles_kernel(const double* __restrict__ field, int64_t n, double iso,
                                                               long long* __restrict__ tiles) {
    __shared__ long long warp_sums[kThreads / 32];
    const int64_t cells = n - 1, total = cells * cells * cells;
    const int64_t base = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
    long long c = 0;
    for (int k = 0; k < kItems; ++k) {
        const int64_t i = base + k;
        if (i < total) {
            const int64_t x = i % cells, y = (i / cells) % cells, z = i / (cells * cells);
            c += active(field, (z * n + y) * n + x, n, iso);
        }
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < kThreads / 32; ++w) t += warp_sums[w];
        tiles[blockIdx.x] = t;  // every slot read below is written first by this call
    }
}

__global__ void __launch_bounds__(kThreads) sum_tiles_kernel(const long long* __restrict__ tiles, int64_t count,
                                                             int64_t* __restrict__ out) {
    __shared__ long long warp_sums[kThreads / 32];
    long long c = 0;
    for (int64_t i = threadIdx.x; i < count; i += kThreads) c += tiles[i];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < kThreads / 32; ++w) t += warp_sums[w];
        *out = t;
    }
}

typedef CUresult (*CtxGetCurrent)(CUcontext*);

// The driver's cuCtxGetCurrent, fetched through the runtime (the library does
// not link libcuda directly).
static CtxGetCurrent ctx_get_current() {
    static CtxGetCurrent fn = [] {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<CtxGetCurrent>(ptr);
        return (CtxGetCurrent) nullptr;
    }();
    return fn;
}

// Device address of g_tile_counts on the current device, looked up once per
// device and context.  A thread with no current context gets the device's
// primary context from the runtime's first symbol lookup.
static int scratch_address(long long** out) {
    static std::mutex mu;
    static long long* addresses[kMaxDevices] = {};
    static CUcontext contexts[kMaxDevices] = {};
    int dev = 0;
    PB_CHECK_CUDA(cudaGetDevice(&dev), "dual count (no alloc): cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(PB_ERR_DEVICE, "dual count (no alloc): device index %d", dev);
    CtxGetCurrent get = ctx_get_current();
    if (!get) return fail(PB_ERR_CUDA, "dual count (no alloc): cuCtxGetCurrent is unavailable");
    std::lock_guard<std::mutex> lock(mu);
    CUcontext ctx = nullptr;
    if (get(&ctx) != CUDA_SUCCESS) return fail(PB_ERR_CUDA, "dual count (no alloc): cuCtxGetCurrent failed");
    if (ctx && addresses[dev] && contexts[dev] == ctx) {
        *out = addresses[dev];
        return PB_OK;
    }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_tile_counts);
    if (e != cudaSuccess || !p) return cuda_fail(e, "dual count (no alloc): cudaGetSymbolAddress");
    if (!ctx && (get(&ctx) != CUDA_SUCCESS || !ctx))
        return fail(PB_ERR_CUDA, "dual count (no alloc): no current context after the symbol lookup");
    addresses[dev] = static_cast<long long*>(p);
    contexts[dev] = ctx;
    *out = addresses[dev];
    return PB_OK;
}

}  // namespace noalloc
}  // namespace pb

using namespace pb;

extern "C" int pb_dual_vertex_count_f64_noalloc(const double* field, int64_t n, double iso, int64_t* count,
                                                void* stream) {
    using namespace pb::noalloc;
    if (!field || !count) return fail(PB_ERR_INVALID, "dual count (no alloc): null buffer");
    if (n < 2) return fail(PB_ERR_INVALID, "dual count (no alloc): n must be >= 2 (got %lld)", (long long)n);
    // n is bounded before the cell count is formed, so the product cannot overflow.
    if (n > 4097)
        return fail(PB_ERR_INVALID,
                    "dual count (no alloc): n = %lld exceeds the fixed scratch (n <= 513); use "
                    "pb_dual_vertices_f64 with a workspace for larger grids",
                    (long long)n);
    const int64_t cells = n - 1;
    const int64_t tiles = (cells * cells * cells + kTile - 1) / kTile;
    if (tiles > kMaxTiles)
        return fail(PB_ERR_INVALID,
                    "dual count (no alloc): n = %lld needs %lld tile slots but the fixed scratch holds %lld "
                    "(n <= 513); use pb_dual_vertices_f64 with a workspace for larger grids",
                    (long long)n, (long long)tiles, (long long)kMaxTiles);
    long long* scratch = nullptr;
    PB_TRY(scratch_address(&scratch));
    cudaStream_t s = (cudaStream_t)stream;
    count_tiles_kernel<<<(unsigned)tiles, kThreads, 0, s>>>(field, n, iso, scratch);
    PB_CHECK_LAUNCH("count_tiles_kernel");
    sum_tiles_kernel<<<1, kThreads, 0, s>>>(scratch, tiles, count);
    PB_CHECK_LAUNCH("sum_tiles_kernel");
    return PB_OK;
}
