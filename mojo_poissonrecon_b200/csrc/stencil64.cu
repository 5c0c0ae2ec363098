// FP64 grid operators of the screened-Poisson multigrid, bit-exact with the
// reference (src/capi.mojo:228-742).  Grids are dense [z][y][x], side n.
//
// Compiled with -fmad=false: no multiply-add is fused, so every result rounds
// exactly as the reference's scalar code does.  Per-node work is independent
// (red-black colouring makes each colour's updates read only the other
// colour), so parallel execution does not change any bit.
#include "common.cuh"

namespace pb {

// ---- assemble (capi.mojo:228-279) -------------------------------------------
__global__ void assemble_kernel(const double* __restrict__ vx, const double* __restrict__ vy,
                                const double* __restrict__ vz, const double* __restrict__ screen,
                                double* __restrict__ rhs, int64_t n, FastDiv dn, double point_weight,
                                double target) {
    const int64_t total = n * n * n;
    const bool small = total <= 0xFFFFFFFFll;  // coordinates by 32-bit invariant division
    const double h_inv = (double)(n - 1);
    const double h_inv2 = h_inv * h_inv;
    const double half_h = 0.5 * h_inv;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int64_t x, y, z;
        if (small) {
            const uint32_t i32 = (uint32_t)idx, row = dn.div(i32), zz = dn.div(row);
            x = i32 - row * (uint32_t)n;
            y = row - zz * (uint32_t)n;
            z = zz;
        } else {
            x = idx % n;
            y = (idx / n) % n;
            z = idx / (n * n);
        }
        const int64_t sy = n, sz = n * n;
        double div = 0.0;
        if (x == 0) div += (vx[idx + 1] - vx[idx]) * h_inv;
        else if (x == n - 1) div += (vx[idx] - vx[idx - 1]) * h_inv;
        else div += (vx[idx + 1] - vx[idx - 1]) * half_h;
        if (y == 0) div += (vy[idx + sy] - vy[idx]) * h_inv;
        else if (y == n - 1) div += (vy[idx] - vy[idx - sy]) * h_inv;
        else div += (vy[idx + sy] - vy[idx - sy]) * half_h;
        if (z == 0) div += (vz[idx + sz] - vz[idx]) * h_inv;
        else if (z == n - 1) div += (vz[idx] - vz[idx - sz]) * h_inv;
        else div += (vz[idx + sz] - vz[idx - sz]) * half_h;
        const double screening = point_weight * screen[idx] * h_inv2;
        rhs[idx] = -div + screening * target;
    }
}

// Neumann 6-neighbour sum in the order x-, x+, y-, y+, z-, z+ (capi.mojo:282-306).
__device__ __forceinline__ double neighbour_sum(const double* __restrict__ v, int64_t idx, int64_t x, int64_t y,
                                                int64_t z, int64_t n, int& degree) {
    double s = 0.0;
    int d = 0;
    const int64_t sy = n, sz = n * n;
    if (x > 0) { s += v[idx - 1]; ++d; }
    if (x + 1 < n) { s += v[idx + 1]; ++d; }
    if (y > 0) { s += v[idx - sy]; ++d; }
    if (y + 1 < n) { s += v[idx + sy]; ++d; }
    if (z > 0) { s += v[idx - sz]; ++d; }
    if (z + 1 < n) { s += v[idx + sz]; ++d; }
    degree = d;
    return s;
}

// ---- one colour of red-black Gauss-Seidel (capi.mojo:310-410) ---------------
// Thread (k, y, z) updates x = ((y+z+colour)&1) + 2k.
__global__ void relax_colour_kernel(double* __restrict__ sol, const double* __restrict__ rhs,
                                    const double* __restrict__ screen, int64_t n, double point_weight, int colour) {
    const int64_t half = (n + 1) / 2;
    const int64_t total = half * n * n;
    const double h_inv = (double)(n - 1);
    const double h_inv2 = h_inv * h_inv;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = t % half, row = t / half;
        const int64_t y = row % n, z = row / n;
        const int64_t x = ((y + z + colour) & 1) + 2 * k;
        if (x >= n) continue;
        const int64_t idx = (z * n + y) * n + x;
        int degree;
        const double s = neighbour_sum(sol, idx, x, y, z, n, degree);
        const double screening = point_weight * screen[idx] * h_inv2;
        const double diagonal = (double)degree * h_inv2 + screening;
        PB_GUARD(idx, n * n * n, kSiteRelax64)
        if (diagonal > 1.0e-30) sol[idx] = (rhs[idx] + s * h_inv2) / diagonal;
    }
}

// ---- residual (capi.mojo:413-553) with per-block sums of squares --------------
constexpr int kNormThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* shared /*[32]*/) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) shared[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        r = lane < (int)(blockDim.x >> 5) ? shared[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;  // valid in thread 0
}

__global__ void __launch_bounds__(kNormThreads) residual_kernel(const double* __restrict__ sol,
                                                                const double* __restrict__ rhs,
                                                                const double* __restrict__ screen,
                                                                double* __restrict__ res, int64_t n,
                                                                double point_weight, double* __restrict__ partial) {
    __shared__ double shared[32];
    const int64_t total = n * n * n;
    const double h_inv = (double)(n - 1);
    const double h_inv2 = h_inv * h_inv;
    double sq = 0.0;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = idx % n, y = (idx / n) % n, z = idx / (n * n);
        int degree;
        const double s = neighbour_sum(sol, idx, x, y, z, n, degree);
        const double screening = point_weight * screen[idx] * h_inv2;
        const double applied = ((double)degree * h_inv2 + screening) * sol[idx] - s * h_inv2;
        const double r = rhs[idx] - applied;
        res[idx] = r;
        sq += r * r;
    }
    const double b = block_sum(sq, shared);
    if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

// Sums the per-block partials in a fixed order (deterministic) and takes sqrt.
__global__ void __launch_bounds__(kNormThreads) finish_norm_kernel(const double* __restrict__ partial, int count,
                                                                   double* __restrict__ norm, int take_sqrt) {
    __shared__ double shared[32];
    double v = 0.0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) v += partial[i];
    const double b = block_sum(v, shared);
    if (threadIdx.x == 0) *norm = take_sqrt ? sqrt(b) : b;
}

// Per-block sums of squares of a flat array.
__global__ void __launch_bounds__(kNormThreads) sumsq_kernel(const double* __restrict__ v, int64_t count,
                                                             double* __restrict__ partial) {
    __shared__ double shared[32];
    double sq = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        sq += v[i] * v[i];
    const double b = block_sum(sq, shared);
    if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

// ---- restriction (capi.mojo:557-673) ----------------------------------------
__global__ void restrict_kernel(const double* __restrict__ fine, double* __restrict__ coarse, int64_t fine_n) {
    const int64_t cn = (fine_n + 1) / 2;
    const int64_t total = cn * cn * cn;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = idx % cn, y = (idx / cn) % cn, z = idx / (cn * cn);
        double sum = 0.0, weight = 0.0;
        for (int oz = -1; oz <= 1; ++oz) {
            const int64_t zz = 2 * z + oz;
            if (zz < 0 || zz >= fine_n) continue;
            const double wz = oz == 0 ? 2.0 : 1.0;
            for (int oy = -1; oy <= 1; ++oy) {
                const int64_t yy = 2 * y + oy;
                if (yy < 0 || yy >= fine_n) continue;
                const double wy = oy == 0 ? 2.0 : 1.0;
                const double* row = fine + (zz * fine_n + yy) * fine_n;
                for (int ox = -1; ox <= 1; ++ox) {
                    const int64_t xx = 2 * x + ox;
                    if (xx < 0 || xx >= fine_n) continue;
                    const double wx = ox == 0 ? 2.0 : 1.0;
                    const double w = wx * wy * wz;
                    sum += row[xx] * w;
                    weight += w;
                }
            }
        }
        coarse[idx] = sum / weight;
    }
}

// ---- prolongation (capi.mojo:677-742) ---------------------------------------
__global__ void prolong_add_kernel(const double* __restrict__ c, double* __restrict__ fine, int64_t fine_n) {
    const int64_t cn = (fine_n + 1) / 2;
    const int64_t total = fine_n * fine_n * fine_n;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = idx % fine_n, y = (idx / fine_n) % fine_n, z = idx / (fine_n * fine_n);
        const int64_t x0 = x / 2, y0 = y / 2, z0 = z / 2;
        const int64_t x1 = x0 + 1 < cn - 1 ? x0 + 1 : cn - 1;
        const int64_t y1 = y0 + 1 < cn - 1 ? y0 + 1 : cn - 1;
        const int64_t z1 = z0 + 1 < cn - 1 ? z0 + 1 : cn - 1;
        const double tx = (x & 1) ? 0.5 : 0.0, ty = (y & 1) ? 0.5 : 0.0, tz = (z & 1) ? 0.5 : 0.0;
        const double c000 = c[grid_index(x0, y0, z0, cn)], c100 = c[grid_index(x1, y0, z0, cn)];
        const double c010 = c[grid_index(x0, y1, z0, cn)], c110 = c[grid_index(x1, y1, z0, cn)];
        const double c001 = c[grid_index(x0, y0, z1, cn)], c101 = c[grid_index(x1, y0, z1, cn)];
        const double c011 = c[grid_index(x0, y1, z1, cn)], c111 = c[grid_index(x1, y1, z1, cn)];
        const double c00 = c000 * (1.0 - tx) + c100 * tx;
        const double c10 = c010 * (1.0 - tx) + c110 * tx;
        const double c01 = c001 * (1.0 - tx) + c101 * tx;
        const double c11 = c011 * (1.0 - tx) + c111 * tx;
        const double c0 = c00 * (1.0 - ty) + c10 * ty;
        const double c1 = c01 * (1.0 - ty) + c11 * ty;
        fine[idx] += c0 * (1.0 - tz) + c1 * tz;
    }
}

// Elementwise helpers used by the host orchestration (core.py:255 divides the
// density by samples_per_node; core.py:269 multiplies restricted screens by 4).
__global__ void scale_kernel(double* __restrict__ v, int64_t count, double factor) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = v[i] * factor;
}

__global__ void divide_kernel(double* __restrict__ v, int64_t count, double divisor) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = v[i] / divisor;
}

__global__ void fill_kernel(double* __restrict__ v, int64_t count, double value) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = value;
}

// Grid of a grid-stride launch: enough blocks to fill 148 SMs several times over.
static unsigned stride_blocks(int64_t items, int threads) {
    int64_t b = (items + threads - 1) / threads;
    const int64_t cap = (int64_t)kSMs * 16;
    if (b > cap) b = cap;
    return (unsigned)(b < 1 ? 1 : b);
}

static int check_n(int64_t n, const char* what) {
    if (n < 2) return fail(PB_ERR_INVALID, "%s: n must be >= 2 (got %lld)", what, (long long)n);
    if (n > 4097) return fail(PB_ERR_INVALID, "%s: n must be <= 4097", what);
    return PB_OK;
}

unsigned residual_blocks(int64_t n) { return stride_blocks(n * n * n, kNormThreads); }

}  // namespace pb

using namespace pb;

extern "C" int pb_assemble_f64(const double* vx, const double* vy, const double* vz, const double* screen, double* rhs,
                               int64_t n, double point_weight, double target_value, void* stream) {
    PB_TRY(check_n(n, "assemble"));
    if (!vx || !vy || !vz || !screen || !rhs) return fail(PB_ERR_INVALID, "assemble: null buffer");
    assemble_kernel<<<stride_blocks(n * n * n, 256), 256, 0, (cudaStream_t)stream>>>(
        vx, vy, vz, screen, rhs, n, FastDiv((uint32_t)n), point_weight, target_value);
    PB_CHECK_LAUNCH("assemble_kernel");
    return PB_OK;
}

extern "C" int pb_relax_f64(double* solution, const double* rhs, const double* screen, int64_t n, double point_weight,
                            int64_t iterations, void* stream) {
    PB_TRY(check_n(n, "relax"));
    if (!solution || !rhs || !screen) return fail(PB_ERR_INVALID, "relax: null buffer");
    if (iterations < 0) return fail(PB_ERR_INVALID, "relax: negative iterations");
    const unsigned blocks = stride_blocks(((n + 1) / 2) * n * n, 256);
    for (int64_t it = 0; it < iterations; ++it)
        for (int colour = 0; colour < 2; ++colour) {
            relax_colour_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(solution, rhs, screen, n, point_weight,
                                                                           colour);
            PB_CHECK_LAUNCH("relax_colour_kernel");
        }
    return PB_OK;
}

extern "C" size_t pb_residual_workspace_size(int64_t n) {
    if (n < 2) n = 2;
    return (size_t)residual_blocks(n) * sizeof(double) + 256;
}

extern "C" int pb_residual_f64(const double* solution, const double* rhs, const double* screen, double* residual,
                               int64_t n, double point_weight, double* norm, void* workspace, size_t workspace_bytes,
                               void* stream) {
    PB_TRY(check_n(n, "residual"));
    if (!solution || !rhs || !screen || !residual || !norm) return fail(PB_ERR_INVALID, "residual: null buffer");
    const unsigned blocks = residual_blocks(n);
    if (!workspace || workspace_bytes < pb_residual_workspace_size(n))
        return fail(PB_ERR_WORKSPACE, "residual: workspace needs %zu bytes", pb_residual_workspace_size(n));
    double* partial = (double*)workspace;
    cudaStream_t s = (cudaStream_t)stream;
    residual_kernel<<<blocks, kNormThreads, 0, s>>>(solution, rhs, screen, residual, n, point_weight, partial);
    PB_CHECK_LAUNCH("residual_kernel");
    finish_norm_kernel<<<1, kNormThreads, 0, s>>>(partial, (int)blocks, norm, 1);
    PB_CHECK_LAUNCH("finish_norm_kernel");
    return PB_OK;
}

// *norm (device) = ||values||_2 over `count` doubles; the workspace of
// pb_residual_workspace_size(n) suffices for count <= n^3.
extern "C" int pb_norm_f64(const double* values, int64_t count, double* norm, void* workspace, size_t workspace_bytes,
                           void* stream) {
    if (count < 1 || !values || !norm) return fail(PB_ERR_INVALID, "norm: bad args");
    const unsigned blocks = stride_blocks(count, kNormThreads);
    if (!workspace || workspace_bytes < (size_t)blocks * sizeof(double))
        return fail(PB_ERR_WORKSPACE, "norm: workspace needs %zu bytes", (size_t)blocks * sizeof(double));
    cudaStream_t s = (cudaStream_t)stream;
    sumsq_kernel<<<blocks, kNormThreads, 0, s>>>(values, count, (double*)workspace);
    PB_CHECK_LAUNCH("sumsq_kernel");
    finish_norm_kernel<<<1, kNormThreads, 0, s>>>((const double*)workspace, (int)blocks, norm, 1);
    PB_CHECK_LAUNCH("finish_norm_kernel");
    return PB_OK;
}

extern "C" int pb_restrict_f64(const double* fine, double* coarse, int64_t fine_n, void* stream) {
    PB_TRY(check_n(fine_n, "restrict"));
    if (!fine || !coarse) return fail(PB_ERR_INVALID, "restrict: null buffer");
    const int64_t cn = (fine_n + 1) / 2;
    restrict_kernel<<<stride_blocks(cn * cn * cn, 256), 256, 0, (cudaStream_t)stream>>>(fine, coarse, fine_n);
    PB_CHECK_LAUNCH("restrict_kernel");
    return PB_OK;
}

extern "C" int pb_prolong_add_f64(const double* coarse, double* fine, int64_t fine_n, void* stream) {
    PB_TRY(check_n(fine_n, "prolong"));
    if (!fine || !coarse) return fail(PB_ERR_INVALID, "prolong: null buffer");
    prolong_add_kernel<<<stride_blocks(fine_n * fine_n * fine_n, 256), 256, 0, (cudaStream_t)stream>>>(coarse, fine,
                                                                                                      fine_n);
    PB_CHECK_LAUNCH("prolong_add_kernel");
    return PB_OK;
}

extern "C" int pb_scale_f64(double* values, int64_t count, double factor, void* stream) {
    if (count < 0 || (count && !values)) return fail(PB_ERR_INVALID, "scale: bad buffer");
    if (!count) return PB_OK;
    scale_kernel<<<stride_blocks(count, 256), 256, 0, (cudaStream_t)stream>>>(values, count, factor);
    PB_CHECK_LAUNCH("scale_kernel");
    return PB_OK;
}

extern "C" int pb_divide_f64(double* values, int64_t count, double divisor, void* stream) {
    if (count < 0 || (count && !values)) return fail(PB_ERR_INVALID, "divide: bad buffer");
    if (!count) return PB_OK;
    divide_kernel<<<stride_blocks(count, 256), 256, 0, (cudaStream_t)stream>>>(values, count, divisor);
    PB_CHECK_LAUNCH("divide_kernel");
    return PB_OK;
}

extern "C" int pb_fill_f64(double* values, int64_t count, double value, void* stream) {
    if (count < 0 || (count && !values)) return fail(PB_ERR_INVALID, "fill: bad buffer");
    if (!count) return PB_OK;
    fill_kernel<<<stride_blocks(count, 256), 256, 0, (cudaStream_t)stream>>>(values, count, value);
    PB_CHECK_LAUNCH("fill_kernel");
    return PB_OK;
}
