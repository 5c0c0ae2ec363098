// Error reporting, version and device check for the C ABI.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <utility>

#include "common.cuh"

namespace pb {

static thread_local char g_last_error[512] = "";
static std::atomic<long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int fail(int code, const char* fmt, ...) {
    va_list args;
    va_start(args, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, args);
    va_end(args);
    return code;
}

int cuda_fail(cudaError_t err, const char* where) {
    return fail(PB_ERR_CUDA, "%s: %s (%s)", where, cudaGetErrorString(err), cudaGetErrorName(err));
}

// Launch parameters chosen by the autotuner, per (parameter, grid side); read
// by the host launchers, which fall back to their built-in choice when unset.
static std::mutex g_tune_mu;
static std::map<std::pair<int64_t, int64_t>, int64_t> g_tune;

int64_t tuned(int param, int64_t n, int64_t fallback) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find({(int64_t)param, n});
    return it == g_tune.end() ? fallback : it->second;
}

}  // namespace pb

#ifdef PB_CHECKED
namespace pb {
__device__ unsigned long long g_check_word = 0;
}
#endif

extern "C" int pb_checked_build(void) {
#ifdef PB_CHECKED
    return 1;
#else
    return 0;
#endif
}

extern "C" int pb_check_status(uint64_t* word, int clear) {
    if (!word) return pb::fail(PB_ERR_INVALID, "check status: null output");
    *word = 0;
#ifdef PB_CHECKED
    unsigned long long w = 0;
    PB_CHECK_CUDA(cudaMemcpyFromSymbol(&w, pb::g_check_word, sizeof(w)), "check status: read");
    *word = w;
    if (clear) {
        const unsigned long long zero = 0;
        PB_CHECK_CUDA(cudaMemcpyToSymbol(pb::g_check_word, &zero, sizeof(zero)), "check status: clear");
    }
#else
    (void)clear;
#endif
    return PB_OK;
}

extern "C" const char* pb_last_error(void) { return pb::g_last_error; }

extern "C" int pb_version(void) { return 10000; }

extern "C" long long pb_launch_count(void) { return pb::g_launches.load(std::memory_order_relaxed); }

extern "C" int pb_note_launches(long long count) {
    if (count > 0) pb::g_launches.fetch_add(count, std::memory_order_relaxed);
    return 0;
}

extern "C" int pb_init(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return pb::cuda_fail(e, "pb_init: cudaSetDevice");
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return pb::cuda_fail(e, "pb_init: cudaGetDeviceProperties");
    if (prop.major != 10)
        return pb::fail(PB_ERR_DEVICE, "pb_init: device %d is sm_%d%d; this library is built for sm_100a", device,
                        prop.major, prop.minor);
    return PB_OK;
}

extern "C" int pb_tune_set(int64_t param, int64_t n, int64_t value) {
    if (param < 0 || param >= PB_TUNE_PARAMS || n < 2 || n > 4097 || value < 0 || value > 4097)
        return pb::fail(PB_ERR_INVALID, "tune set: bad parameter, side or value");
    std::lock_guard<std::mutex> lock(pb::g_tune_mu);
    if (value == 0) pb::g_tune.erase({param, n});
    else pb::g_tune[{param, n}] = value;
    return PB_OK;
}

extern "C" int64_t pb_tune_get(int64_t param, int64_t n) { return pb::tuned((int)param, n, 0); }

extern "C" int pb_tune_clear(void) {
    std::lock_guard<std::mutex> lock(pb::g_tune_mu);
    pb::g_tune.clear();
    return PB_OK;
}
