// Shared helpers for the sm_100a kernels of the screened-Poisson path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/poisson_b200.h"
#include "checked.cuh"

namespace pb {

// Sets the thread-local message returned by pb_last_error() and passes the code through.
int fail(int code, const char* fmt, ...);

// Maps a CUDA error (from a launch or an API call) to PB_ERR_CUDA with its text.
int cuda_fail(cudaError_t err, const char* where);

// Counts every kernel this library launches (read by pb_launch_count()).
void count_launch();

// The autotuned value of a launch parameter (PB_TUNE_*) for grid side n, or
// `fallback` when none is set (pb_tune_set).
int64_t tuned(int param, int64_t n, int64_t fallback);

#define PB_CHECK_LAUNCH(where)                                   \
    do {                                                         \
        ::pb::count_launch();                                    \
        cudaError_t e_ = cudaGetLastError();                     \
        if (e_ != cudaSuccess) return ::pb::cuda_fail(e_, where); \
    } while (0)

#define PB_CHECK_CUDA(call, where)                               \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return ::pb::cuda_fail(e_, where); \
    } while (0)

#define PB_TRY(expr)              \
    do {                          \
        int s_ = (expr);          \
        if (s_ != PB_OK) return s_; \
    } while (0)

constexpr int kSMs = 148;  // B200: 148 SMs on two dies

__host__ __device__ __forceinline__ int64_t grid_index(int64_t x, int64_t y, int64_t z, int64_t n) {
    return (z * n + y) * n + x;
}

// Unsigned 32-bit division by an invariant divisor d as a multiply-high and
// shifts (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, round-up variant): with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1, n / d = (t + ((n - t) >> 1)) >> (l - 1)
// where t = mulhi(m, n), exact for every 32-bit n and 2 <= d < 2^32.
struct FastDiv {
    uint32_t d = 1, m = 0, s = 0;
    FastDiv() = default;
    explicit FastDiv(uint32_t divisor) : d(divisor) {
        if (d >= 2) {
            int l = 0;
            while ((1ull << l) < d) ++l;
            m = (uint32_t)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
            s = (uint32_t)(l - 1);
        }
    }
    __device__ __forceinline__ uint32_t div(uint32_t n) const {
        if (d == 1) return n;
        const uint32_t t = __umulhi(m, n);
        return (t + ((n - t) >> 1)) >> s;
    }
};

inline unsigned blocks_for(int64_t items, int threads) {
    int64_t b = (items + threads - 1) / threads;
    return (unsigned)(b < 1 ? 1 : b);
}

// A caller-provided scratch buffer carved into aligned pieces.
struct Workspace {
    char* base;
    size_t size;
    size_t used;
    __host__ Workspace(void* p, size_t s) : base((char*)p), size(s), used(0) {}
    template <typename T>
    __host__ T* take(size_t count) {
        size_t off = (used + 255) & ~size_t(255);
        used = off + count * sizeof(T);
        return base ? (T*)(base + off) : nullptr;
    }
    __host__ bool fits() const { return used <= size; }
};

// Bytes a sequence of `take` calls needs (run the same carving with base = null).
template <typename F>
size_t measure(F&& carve) {
    Workspace w(nullptr, 0);
    carve(w);
    return w.used + 256;
}

}  // namespace pb
