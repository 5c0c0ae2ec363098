// Input preparation and output mapping for reconstruct() on the device.
//
// Reference: python/mojo_poissonrecon/core.py:73-83 (_valid_oriented_rows),
// :377-385 (_normalize), :425 (vertices * width + origin).  Rows with a
// non-finite coordinate or a zero / non-finite normal are dropped, keeping the
// order of the rest; the bounding box of the kept points gives the unit-cube
// map.  Min/max are exact, and each coordinate is mapped with the same two
// roundings as NumPy (compiled with -fmad=false), so the results are
// bit-identical to the reference's NumPy code.
#include <math.h>

#include "scan.cuh"

namespace pb {

// A kept row: finite point and normal, and max |n_k| > 0.  (The reference also
// requires the scaled squared norm to be finite and positive; with a finite
// non-zero maximum the scaled components lie in [-1, 1] with one at +-1, so
// that test always holds.)
__device__ __forceinline__ bool row_valid(const double* p, const double* nrm) {
    bool finite = isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]) && isfinite(nrm[0]) && isfinite(nrm[1]) &&
                  isfinite(nrm[2]);
    double s = fmax(fabs(nrm[0]), fmax(fabs(nrm[1]), fabs(nrm[2])));
    return finite && s > 0.0;
}

__global__ void valid_flags_kernel(const double* __restrict__ points, const double* __restrict__ normals,
                                   int64_t count, uint32_t* __restrict__ flags) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) flags[i] = row_valid(points + 3 * i, normals + 3 * i) ? 1u : 0u;
}

__global__ void compact_rows_kernel(const double* __restrict__ points, const double* __restrict__ normals,
                                    int64_t count, const uint32_t* __restrict__ rank, double* __restrict__ out_points,
                                    double* __restrict__ out_normals) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const double* p = points + 3 * i;
    const double* nrm = normals + 3 * i;
    if (!row_valid(p, nrm)) return;
    const int64_t j = rank[i];
    out_points[3 * j] = p[0];
    out_points[3 * j + 1] = p[1];
    out_points[3 * j + 2] = p[2];
    out_normals[3 * j] = nrm[0];
    out_normals[3 * j + 1] = nrm[1];
    out_normals[3 * j + 2] = nrm[2];
}

// Per-block min/max of each axis over the first *kept rows.
__global__ void bbox_partial_kernel(const double* __restrict__ points, const uint32_t* __restrict__ kept,
                                    double* __restrict__ partial) {
    __shared__ double lo[3][32], hi[3][32];
    const int64_t count = *kept;
    double l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        for (int k = 0; k < 3; ++k) {
            const double v = points[3 * i + k];
            l[k] = fmin(l[k], v);
            h[k] = fmax(h[k], v);
        }
    for (int k = 0; k < 3; ++k)
        for (int o = 16; o > 0; o >>= 1) {
            l[k] = fmin(l[k], __shfl_down_sync(0xffffffffu, l[k], o));
            h[k] = fmax(h[k], __shfl_down_sync(0xffffffffu, h[k], o));
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 3; ++k) {
            lo[k][warp] = l[k];
            hi[k][warp] = h[k];
        }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
            for (int k = 0; k < 3; ++k) {
                l[k] = fmin(l[k], lo[k][w]);
                h[k] = fmax(h[k], hi[k][w]);
            }
        for (int k = 0; k < 3; ++k) {
            partial[6 * blockIdx.x + k] = l[k];
            partial[6 * blockIdx.x + 3 + k] = h[k];
        }
    }
}

// map[0..2] = origin, map[3] = width (core.py:377-385).  Min and max are exact
// in any order, so the block-parallel reduction gives the serial result.
__global__ void bbox_finish_kernel(const double* __restrict__ partial, int blocks, double scale,
                                   double* __restrict__ map) {
    __shared__ double lo[3][32], hi[3][32];
    double l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int b = threadIdx.x; b < blocks; b += blockDim.x)
        for (int k = 0; k < 3; ++k) {
            l[k] = fmin(l[k], partial[6 * b + k]);
            h[k] = fmax(h[k], partial[6 * b + 3 + k]);
        }
    for (int k = 0; k < 3; ++k)
        for (int o = 16; o > 0; o >>= 1) {
            l[k] = fmin(l[k], __shfl_down_sync(0xffffffffu, l[k], o));
            h[k] = fmax(h[k], __shfl_down_sync(0xffffffffu, h[k], o));
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 3; ++k) {
            lo[k][warp] = l[k];
            hi[k][warp] = h[k];
        }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
        for (int k = 0; k < 3; ++k) {
            l[k] = fmin(l[k], lo[k][w]);
            h[k] = fmax(h[k], hi[k][w]);
        }
    double extent = fmax(h[0] - l[0], fmax(h[1] - l[1], h[2] - l[2]));
    double width = extent * scale;
    if (!isfinite(width) || !(width > 0.0)) width = 1.0;
    for (int k = 0; k < 3; ++k) {
        const double center = 0.5 * (l[k] + h[k]);
        map[k] = center - 0.5 * width;
    }
    map[3] = width;
}

__global__ void normalize_kernel(double* __restrict__ points, const uint32_t* __restrict__ kept,
                                 const double* __restrict__ map) {
    const int64_t count = (int64_t)*kept * 3;
    const double width = map[3];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        points[i] = (points[i] - map[i % 3]) / width;
}

__global__ void unit_cube_check_kernel(const double* __restrict__ points, int64_t count, int* __restrict__ outside) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < 3 * count; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = points[i];
        if (v < 0.0 || v > 1.0) *outside = 1;
    }
}

__global__ void map_vertices_kernel(double* __restrict__ v, int64_t count, const double* __restrict__ map) {
    const double width = map[3];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < 3 * count; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = v[i] * width + map[i % 3];
}

__global__ void store_kept_kernel(const uint32_t* __restrict__ kept, int64_t* __restrict__ out) { *out = *kept; }

static unsigned capped_blocks(int64_t items) {
    int64_t b = (items + 255) / 256;
    if (b > (int64_t)kSMs * 8) b = (int64_t)kSMs * 8;
    return (unsigned)(b < 1 ? 1 : b);
}

static size_t prep_ws_bytes(int64_t count) {
    return measure([&](Workspace& w) {
        w.take<uint32_t>(count + 1);
        w.take<uint32_t>(1);
        w.take<double>(6 * (size_t)capped_blocks(count));
        scan_carve<uint32_t>(w, count);
    });
}

}  // namespace pb

using namespace pb;

extern "C" size_t pb_prepare_workspace_size(int64_t point_count) {
    return prep_ws_bytes(point_count < 1 ? 1 : point_count);
}

// Keeps the valid rows of (points, normals) in order, writes their number to
// *kept (device int64) and, when scale > 0, maps the kept points into the unit
// cube in place (map[0..2] = origin, map[3] = width, device doubles).
extern "C" int pb_prepare_points_f64(const double* points, const double* normals, int64_t point_count, double scale,
                                     double* out_points, double* out_normals, int64_t* kept, double* map,
                                     void* workspace, size_t workspace_bytes, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (point_count < 1 || point_count >= (int64_t)0xFFFFFFFFll)
        return fail(PB_ERR_INVALID, "prepare: point_count must be in [1, 2^32)");
    if (!points || !normals || !out_points || !out_normals || !kept || (scale > 0.0 && !map))
        return fail(PB_ERR_INVALID, "prepare: null buffer");
    const size_t need = prep_ws_bytes(point_count);
    if (!workspace || workspace_bytes < need) return fail(PB_ERR_WORKSPACE, "prepare: workspace needs %zu bytes", need);
    Workspace w(workspace, workspace_bytes);
    uint32_t* rank = w.take<uint32_t>(point_count + 1);
    uint32_t* total = w.take<uint32_t>(1);
    const unsigned pb_blocks = capped_blocks(point_count);
    double* partial = w.take<double>(6 * (size_t)pb_blocks);
    valid_flags_kernel<<<blocks_for(point_count, 256), 256, 0, s>>>(points, normals, point_count, rank);
    PB_CHECK_LAUNCH("valid_flags_kernel");
    PB_TRY(exclusive_scan<uint32_t>(rank, rank, point_count, total, w, s));
    compact_rows_kernel<<<blocks_for(point_count, 256), 256, 0, s>>>(points, normals, point_count, rank, out_points,
                                                                      out_normals);
    PB_CHECK_LAUNCH("compact_rows_kernel");
    store_kept_kernel<<<1, 1, 0, s>>>(total, kept);
    PB_CHECK_LAUNCH("store_kept_kernel");
    if (scale > 0.0) {
        bbox_partial_kernel<<<pb_blocks, 256, 0, s>>>(out_points, total, partial);
        PB_CHECK_LAUNCH("bbox_partial_kernel");
        bbox_finish_kernel<<<1, 256, 0, s>>>(partial, (int)pb_blocks, scale, map);
        PB_CHECK_LAUNCH("bbox_finish_kernel");
        normalize_kernel<<<capped_blocks(3 * point_count), 256, 0, s>>>(out_points, total, map);
        PB_CHECK_LAUNCH("normalize_kernel");
    }
    return PB_OK;
}

// *outside (device int) is set to 1 if any coordinate lies outside [0, 1]
// (core.py:225-227); the caller zeroes it first.
extern "C" int pb_unit_cube_check_f64(const double* points, int64_t point_count, int* outside, void* stream) {
    if (point_count < 0 || !outside || (point_count && !points)) return fail(PB_ERR_INVALID, "unit cube check: bad args");
    if (!point_count) return PB_OK;
    unit_cube_check_kernel<<<capped_blocks(3 * point_count), 256, 0, (cudaStream_t)stream>>>(points, point_count,
                                                                                            outside);
    PB_CHECK_LAUNCH("unit_cube_check_kernel");
    return PB_OK;
}

// vertices = vertices * width + origin (core.py:425), map as written by pb_prepare_points_f64.
extern "C" int pb_map_vertices_f64(double* vertices, int64_t vertex_count, const double* map, void* stream) {
    if (vertex_count < 0 || !map || (vertex_count && !vertices)) return fail(PB_ERR_INVALID, "map vertices: bad args");
    if (!vertex_count) return PB_OK;
    map_vertices_kernel<<<capped_blocks(3 * vertex_count), 256, 0, (cudaStream_t)stream>>>(vertices, vertex_count, map);
    PB_CHECK_LAUNCH("map_vertices_kernel");
    return PB_OK;
}
