// Error reporting, version and device check for the C ABI.
#include <atomic>
#include <cstdarg>
#include <cstdio>

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

}  // namespace pb

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
