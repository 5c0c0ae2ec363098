// Weighted iso-value (src/capi.mojo:746-795): sum_i w_i * trilinear(field, p_i)
// / sum_i w_i with w_i = |n_i| (confidence) or 1.  Per-point terms are exact
// restatements (compiled with -fmad=false); the two sums use a fixed-shape
// tree (warp shuffles, then per-block partials summed in block order), so the
// result is deterministic and differs from the serial sum by rounding only.
#include "common.cuh"

namespace pb {

constexpr int kIsoThreads = 256;

__device__ __forceinline__ double iso_norm3(double x, double y, double z) {  // capi.mojo:51-59
    double scale = fmax(fabs(x), fmax(fabs(y), fabs(z)));
    if (scale == 0.0) return 0.0;
    double sx = x / scale, sy = y / scale, sz = z / scale;
    return scale * sqrt(sx * sx + sy * sy + sz * sz);
}

__device__ __forceinline__ void iso_cell(double p, int64_t res, int64_t& i, double& f) {  // capi.mojo:771-779
    double g = p * (double)res;
    int64_t t = (int64_t)g;
    i = t < 0 ? 0 : (t > res - 1 ? res - 1 : t);
    double m = g - (double)i;
    m = m > 0.0 ? m : 0.0;
    f = m < 1.0 ? m : 1.0;
}

__device__ __forceinline__ void block_sum2(double& a, double& b, double* sa, double* sb) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sa[warp] = a;
        sb[warp] = b;
    }
    __syncthreads();
    if (warp == 0) {
        const int warps = blockDim.x >> 5;
        a = lane < warps ? sa[lane] : 0.0;
        b = lane < warps ? sb[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
    }
}

__global__ void __launch_bounds__(kIsoThreads) iso_partial_kernel(const double* __restrict__ field,
                                                                  const double* __restrict__ points,
                                                                  const double* __restrict__ normals, int64_t count,
                                                                  int64_t n, int confidence,
                                                                  double* __restrict__ partial) {
    __shared__ double sa[32], sb[32];
    const int64_t res = n - 1;
    double value_sum = 0.0, weight_sum = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < count; p += (int64_t)gridDim.x * blockDim.x) {
        const double w = confidence ? iso_norm3(normals[3 * p], normals[3 * p + 1], normals[3 * p + 2]) : 1.0;
        int64_t ix, iy, iz;
        double fx, fy, fz;
        iso_cell(points[3 * p], res, ix, fx);
        iso_cell(points[3 * p + 1], res, iy, fy);
        iso_cell(points[3 * p + 2], res, iz, fz);
        double value = 0.0;
        for (int dz = 0; dz < 2; ++dz) {
            const double wz = dz == 1 ? fz : 1.0 - fz;
            for (int dy = 0; dy < 2; ++dy) {
                const double wy = dy == 1 ? fy : 1.0 - fy;
                for (int dx = 0; dx < 2; ++dx) {
                    const double wx = dx == 1 ? fx : 1.0 - fx;
                    value += field[grid_index(ix + dx, iy + dy, iz + dz, n)] * wx * wy * wz;
                }
            }
        }
        value_sum += value * w;
        weight_sum += w;
    }
    block_sum2(value_sum, weight_sum, sa, sb);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = value_sum;
        partial[2 * blockIdx.x + 1] = weight_sum;
    }
}

__global__ void __launch_bounds__(kIsoThreads) iso_finish_kernel(const double* __restrict__ partial, int blocks,
                                                                 double* __restrict__ iso) {
    __shared__ double sa[32], sb[32];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) {
        a += partial[2 * i];
        b += partial[2 * i + 1];
    }
    block_sum2(a, b, sa, sb);
    if (threadIdx.x == 0) *iso = b > 0.0 ? a / b : 0.0;
}

static unsigned iso_blocks(int64_t count) {
    int64_t b = (count + kIsoThreads - 1) / kIsoThreads;
    const int64_t cap = (int64_t)kSMs * 8;
    if (b > cap) b = cap;
    return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace pb

using namespace pb;

extern "C" size_t pb_iso_value_workspace_size(int64_t point_count) {
    return (size_t)iso_blocks(point_count) * 2 * sizeof(double) + 256;
}

extern "C" int pb_iso_value_f64(const double* field, const double* points, const double* normals, int64_t point_count,
                                int64_t n, int64_t confidence, double* iso, void* workspace, size_t workspace_bytes,
                                void* stream) {
    if (n < 2) return fail(PB_ERR_INVALID, "iso value: n must be >= 2");
    if (point_count < 0) return fail(PB_ERR_INVALID, "iso value: negative point_count");
    if (!field || !iso || (point_count && (!points || !normals))) return fail(PB_ERR_INVALID, "iso value: null buffer");
    if (!workspace || workspace_bytes < pb_iso_value_workspace_size(point_count))
        return fail(PB_ERR_WORKSPACE, "iso value: workspace needs %zu bytes", pb_iso_value_workspace_size(point_count));
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned blocks = iso_blocks(point_count);
    double* partial = (double*)workspace;
    iso_partial_kernel<<<blocks, kIsoThreads, 0, s>>>(field, points, normals, point_count, n, (int)confidence, partial);
    PB_CHECK_LAUNCH("iso_partial_kernel");
    iso_finish_kernel<<<1, kIsoThreads, 0, s>>>(partial, (int)blocks, iso);
    PB_CHECK_LAUNCH("iso_finish_kernel");
    return PB_OK;
}
