// FP32 multigrid level 0 and the FP64 defect of the refined solvers.
//
// The reference solves A x = b with FP64 V-cycles (src/capi.mojo:310-742,
// python/mojo_poissonrecon/core.py:141-193).  The refined solvers keep x in
// FP64 and precondition with FP32 V-cycles on A e = r.  Level 0 of those
// cycles uses the reference's operator in the padded FP32 layout
// (level32.cuh): ghosts are zero, so a 6-neighbour sum over the padded array
// equals the reference's Neumann sum over in-grid neighbours, and the degree
// term lives in the stored diagonal D = (deg + pw*screen) * (n-1)^2.  The
// coarse levels are Galerkin operators (mg27.cu).
#include "batch.cuh"
#include "common.cuh"
#include "level32.cuh"

namespace pb {

// ---- level set-up: D, 1/D and the prolongation weights from the FP64 screen ----
// weights (may be null): s = 1 on nodes of the coarse grid (all coordinates
// even), else deg (n-1)^2 / D (mg27.cu).
__global__ void __launch_bounds__(256) level_setup_kernel(const double* __restrict__ screen, Geom g, double pw,
                                                          float* __restrict__ D, float* __restrict__ invD,
                                                          float* __restrict__ weights) {
    const int n = g.n;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
    if (x >= n || y >= n) return;
    const double h = (double)(n - 1), h2 = h * h;
    const int deg = (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
    const double d = (double)deg * h2 + pw * screen[((int64_t)z * n + y) * n + x] * h2;
    const int64_t p = g.at(x, y, z);
    D[p] = (float)d;
    invD[p] = (float)(1.0 / d);
    if (weights) weights[p] = ((x | y | z) & 1) ? (float)((double)deg * h2 / d) : 1.0f;
}

// ---- FP64 defect with the fused update x_new = x_old + e ------------------------
// r32 = (float)(b - A x_new) into the padded level-0 rhs, ||b - A x_new||^2 per block.
// Block-wide sum (valid in linear thread 0) for 1-D, 2-D or 3-D blocks.
__device__ __forceinline__ double warp_block_sum(double v, double* shared) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int warps = (blockDim.x * blockDim.y * blockDim.z) >> 5;
    if (lane == 0) shared[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        r = lane < warps ? shared[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
}

// A block owns 256 consecutive (x, y) columns of a plane (one 32-bit division
// per thread; full warps on 2^k + 1 sides) and a z range; rows are read
// coalesced, and the z-neighbours of consecutive planes stay in L1/L2.
constexpr int kDefThreads = 256, kDefZ = 16;

template <bool UPDATE>
__global__ void __launch_bounds__(kDefThreads) defect_tile_kernel(
    const double* __restrict__ x_old, const float* __restrict__ e, double* __restrict__ x_new,
    const double* __restrict__ b, const double* __restrict__ screen, Geom g, double pw, float* __restrict__ r32,
    double* __restrict__ r64, double* __restrict__ partial) {
    __shared__ double shared[32];
    const int n = g.n;
    const unsigned t = blockIdx.x * kDefThreads + threadIdx.x;
    const int y = t < (unsigned)(n * n) ? (int)(t / (unsigned)n) : n, x = (int)(t - (unsigned)y * n);
    const int z0 = blockIdx.y * kDefZ, z1 = min(n, z0 + kDefZ);
    const double h = (double)(n - 1), h2 = h * h;
    const int64_t nn = (int64_t)n * n;
    double sq = 0.0;
    if (x < n && y < n) {
        const int degxy = (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n);
        for (int z = z0; z < z1; ++z) {
            const int64_t i = (int64_t)z * nn + (int64_t)y * n + x;
            const int64_t p = g.at(x, y, z);
            auto val = [&](int64_t di, int64_t dp) -> double {
                double v = x_old[i + di];
                if (UPDATE) v += (double)e[p + dp];
                return v;
            };
            double s = 0.0;
            if (x > 0) s += val(-1, -1);
            if (x + 1 < n) s += val(1, 1);
            if (y > 0) s += val(-n, -g.P);
            if (y + 1 < n) s += val(n, g.P);
            if (z > 0) s += val(-nn, -g.plane);
            if (z + 1 < n) s += val(nn, g.plane);
            const int deg = degxy + (z > 0) + (z + 1 < n);
            const double xc = val(0, 0);
            if (UPDATE) x_new[i] = xc;
            const double applied = ((double)deg * h2 + pw * screen[i] * h2) * xc - s * h2;
            const double r = b[i] - applied;
            r32[p] = (float)r;
            if (r64) r64[i] = r;
            sq += r * r;
        }
    }
    const double total = warp_block_sum(sq, shared);
    if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = total;
}

__global__ void sum_partials_kernel(const double* __restrict__ partial, int count, double* __restrict__ out) {
    __shared__ double shared[32];
    double v = 0.0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) v += partial[i];
    const double t = warp_block_sum(v, shared);
    if (threadIdx.x == 0) *out = t;
}

// ---- level-0 residual fused with the scaled restriction -------------------------
// coarse_rhs = P^T (s (rhs - A e)) / 8 (mg27.cu) without writing the fine
// residual.  A block owns a 64 x 4 tile of coarse (x, y) and marches coarse z.
// The fine residual of the tile's region (fine x from 2 xc0 - 4, 136 columns;
// fine y from 2 yc0 - 1, 9 rows), already multiplied by the prolongation weight
// s, is computed four x at a time (float4 loads of e, rhs, D and s; the row
// starts stay 16-byte aligned) into a five-plane ring in shared memory, plane
// 2zc+1 being reused as plane 2(zc+1)-1 of the next coarse plane; five slots
// let each coarse plane pass a single barrier.  Out-of-grid
// ring entries are zero, so the restriction sums all 27 entries with weights
// (1,2,1)^3 / 64.
constexpr int kRrCX = 64, kRrCY = 4, kRrCZ = 4;  // coarse tile and planes per block (measured: 8 -> 4, 108 -> 90 us)
constexpr int kRrRing = 5;                        // fine planes held in shared memory
constexpr int kRrFX = 2 * kRrCX + 8, kRrFY = 2 * kRrCY + 1;  // 136 x 9 fine nodes
constexpr int kRrGroups = kRrFX / 4;                            // float4 groups per ring row
constexpr int kRrThreads = 256;

// PAIRED: the two fine planes of a coarse plane are computed in one loop over
// their 612 float4 items (three rounds of 256 threads instead of two rounds per
// plane, 80 % of the lanes busy instead of 60 %); each item's arithmetic is the
// same, so the results are too.  THREADS = 320 (tuning variant 3, paired):
// the 612 items in two rounds (96 % busy); the first 256 threads restrict.
template <bool PAIRED, int THREADS = kRrThreads>
__device__ __forceinline__ void residual_restrict32_body(const float* __restrict__ e, const float* __restrict__ rhs,
                                                         const float* __restrict__ D, const float* __restrict__ w,
                                                         Geom gf, float h2, float* __restrict__ coarse, Geom gc,
                                                         int cz, int bx, int by, int bz) {
    __shared__ __align__(16) float ring[kRrRing][kRrFY][kRrFX];
    const int fn = gf.n, cn = gc.n;
    const int xc0 = bx * kRrCX, yc0 = by * kRrCY;
    const int zc0 = bz * cz, zc1 = min(cn, zc0 + cz);
    const int fx0 = 2 * xc0 - 4, fy0 = 2 * yc0 - 1;
    const int tid = threadIdx.x;
    constexpr int kItems = kRrFY * kRrGroups;
    auto fine_item = [&](int f, int i) {  // s-weighted residual of one float4 of fine plane f
        float(*dst)[kRrFX] = ring[(f + kRrRing) % kRrRing];
        {
            const int ly = i / kRrGroups, g = i - ly * kRrGroups;
            const int x = fx0 + 4 * g, y = fy0 + ly;
            float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
            if (f >= 0 && f < fn && y >= 0 && y < fn && x >= 0 && x < fn) {
                const int64_t p = gf.at(x, y, f);
                const float4 c = *reinterpret_cast<const float4*>(e + p);
                const float4 ym = *reinterpret_cast<const float4*>(e + p - gf.P);
                const float4 yp = *reinterpret_cast<const float4*>(e + p + gf.P);
                const float4 zm = *reinterpret_cast<const float4*>(e + p - gf.plane);
                const float4 zp = *reinterpret_cast<const float4*>(e + p + gf.plane);
                const float4 b = *reinterpret_cast<const float4*>(rhs + p);
                const float4 d = *reinterpret_cast<const float4*>(D + p);
                const float4 s = *reinterpret_cast<const float4*>(w + p);
                const float l = e[p - 1], rr = e[p + 4];
                const float s0 = l + c.y + ym.x + yp.x + zm.x + zp.x;
                const float s1 = c.x + c.z + ym.y + yp.y + zm.y + zp.y;
                const float s2 = c.y + c.w + ym.z + yp.z + zm.z + zp.z;
                const float s3 = c.z + rr + ym.w + yp.w + zm.w + zp.w;
                // lanes at x >= fn lie on ghosts or padding, where s and D are zero: mask them explicitly
                r.x = s.x * (b.x - (d.x * c.x - s0 * h2));
                r.y = x + 1 < fn ? s.y * (b.y - (d.y * c.y - s1 * h2)) : 0.f;
                r.z = x + 2 < fn ? s.z * (b.z - (d.z * c.z - s2 * h2)) : 0.f;
                r.w = x + 3 < fn ? s.w * (b.w - (d.w * c.w - s3 * h2)) : 0.f;
            }
            *reinterpret_cast<float4*>(&dst[ly][4 * g]) = r;
        }
    };
    auto fine_plane = [&](int f) {
        for (int i = tid; i < kItems; i += THREADS) fine_item(f, i);
    };
    fine_plane(2 * zc0 - 1);
    for (int zc = zc0; zc < zc1; ++zc) {
        if (PAIRED) {
            for (int j = tid; j < 2 * kItems; j += THREADS) {
                const int second = j >= kItems;
                fine_item(2 * zc + second, j - second * kItems);
            }
        } else {
            fine_plane(2 * zc);
            fine_plane(2 * zc + 1);
        }
        __syncthreads();
        {
            const int cy = tid / kRrCX, cx = tid - cy * kRrCX;  // 256 threads = the 64 x 4 coarse tile
            const int xc = xc0 + cx, yc = yc0 + cy;
            if (cy < kRrCY && xc < cn && yc < cn) {
                float sum = 0.0f;
#pragma unroll
                for (int oz = -1; oz <= 1; ++oz) {
                    const int zz = 2 * zc + oz;
#pragma unroll
                    for (int oy = -1; oy <= 1; ++oy) {
                        const float* row = ring[(zz + kRrRing) % kRrRing][2 * cy + 1 + oy];
#pragma unroll
                        for (int ox = -1; ox <= 1; ++ox)
                            sum += row[2 * cx + 4 + ox] * (float)((ox ? 1 : 2) * (oy ? 1 : 2) * (oz ? 1 : 2));
                    }
                }
                coarse[gc.at(xc, yc, zc)] = sum * (1.0f / 64.0f);
            }
        }
        // no second barrier: the next coarse plane writes fine planes 2zc+2 and
        // 2zc+3, whose slots (mod 5) differ from the three read here, and the one
        // after it rewrites these only after all threads pass its first barrier
    }
}

__global__ void __launch_bounds__(kRrThreads) residual_restrict32_kernel(const float* __restrict__ e,
                                                                          const float* __restrict__ rhs,
                                                                          const float* __restrict__ D,
                                                                          const float* __restrict__ w, Geom gf,
                                                                          float h2, float* __restrict__ coarse,
                                                                          Geom gc, int cz) {
    residual_restrict32_body<false>(e, rhs, D, w, gf, h2, coarse, gc, cz, blockIdx.x, blockIdx.y, blockIdx.z);
}

__global__ void __launch_bounds__(kRrThreads) residual_restrict32_paired_kernel(const float* __restrict__ e,
                                                                                 const float* __restrict__ rhs,
                                                                                 const float* __restrict__ D,
                                                                                 const float* __restrict__ w, Geom gf,
                                                                                 float h2, float* __restrict__ coarse,
                                                                                 Geom gc, int cz) {
    residual_restrict32_body<true>(e, rhs, D, w, gf, h2, coarse, gc, cz, blockIdx.x, blockIdx.y, blockIdx.z);
}

__global__ void __launch_bounds__(320) residual_restrict32_paired320_kernel(const float* __restrict__ e,
                                                                          const float* __restrict__ rhs,
                                                                          const float* __restrict__ D,
                                                                          const float* __restrict__ w, Geom gf,
                                                                          float h2, float* __restrict__ coarse,
                                                                          Geom gc, int cz) {
    residual_restrict32_body<true, 320>(e, rhs, D, w, gf, h2, coarse, gc, cz, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Grouped (batch.cuh): ptr[0] e, ptr[1] rhs, ptr[2] D, ptr[3] weights, ptr[4] coarse rhs.
__global__ void __launch_bounds__(kRrThreads) residual_restrict32_grouped_kernel(
    const batch::GridDesc* __restrict__ descs, int count, const int* __restrict__ flags) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    const int n = (int)d.n;
    residual_restrict32_body<false>((const float*)d.ptr[0], (const float*)d.ptr[1], (const float*)d.ptr[2],
                             (const float*)d.ptr[3], geom(n), (float)((n - 1) * (n - 1)), (float*)d.ptr[4],
                             geom((n + 1) / 2), (int)d.aux[0], bx, by, bz);
}


static dim3 defect_grid(int n) {
    return dim3((n * n + kDefThreads - 1) / kDefThreads, (n + kDefZ - 1) / kDefZ);
}

unsigned defect_blocks(int n) {
    const dim3 g = defect_grid(n);
    return g.x * g.y * g.z;
}

}  // namespace pb

using namespace pb;

extern "C" int pb_level_geometry(int64_t n, int64_t* pitch, int64_t* padded_count) {
    if (n < 2 || n > 4097) return fail(PB_ERR_INVALID, "level geometry: n must be in [2, 4097]");
    if (pitch) *pitch = pitch_of((int)n);
    if (padded_count) *padded_count = padded_size((int)n);
    return PB_OK;
}

extern "C" int pb_level_setup_f32(const double* screen, int64_t n, double point_weight, float* D, float* invD,
                                  float* weights, void* stream) {
    if (n < 2 || n > 4097 || !screen || !D || !invD) return fail(PB_ERR_INVALID, "level setup: bad args");
    const dim3 block(32, 8), grid(((int)n + 31) / 32, ((int)n + 7) / 8, (int)n);
    level_setup_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(screen, geom((int)n), point_weight, D, invD,
                                                                 weights);
    PB_CHECK_LAUNCH("level_setup_kernel");
    return PB_OK;
}

extern "C" size_t pb_defect_workspace_size(int64_t n) { return (size_t)defect_blocks((int)(n < 2 ? 2 : n)) * 8 + 256; }

extern "C" int pb_defect_f64(const double* x_old, const float* e, double* x_new, const double* rhs,
                             const double* screen, int64_t n, double point_weight, float* r32, double* r64,
                             double* norm2, void* workspace, size_t workspace_bytes, void* stream) {
    if (n < 2 || n > 4097 || !x_old || !rhs || !screen || !r32 || !norm2) return fail(PB_ERR_INVALID, "defect: bad args");
    if (e && !x_new) return fail(PB_ERR_INVALID, "defect: update needs x_new");
    if (e && x_new == x_old) return fail(PB_ERR_INVALID, "defect: x_new must not alias x_old");
    const unsigned blocks = defect_blocks((int)n);
    if (!workspace || workspace_bytes < (size_t)blocks * 8) return fail(PB_ERR_WORKSPACE, "defect: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    double* partial = (double*)workspace;
    const dim3 grid = defect_grid((int)n), block(kDefThreads);
    if (e)
        defect_tile_kernel<true><<<grid, block, 0, s>>>(x_old, e, x_new, rhs, screen, geom((int)n), point_weight, r32,
                                                        r64, partial);
    else
        defect_tile_kernel<false><<<grid, block, 0, s>>>(x_old, nullptr, nullptr, rhs, screen, geom((int)n),
                                                         point_weight, r32, r64, partial);
    PB_CHECK_LAUNCH("defect_tile_kernel");
    sum_partials_kernel<<<1, 1024, 0, s>>>(partial, (int)blocks, norm2);
    PB_CHECK_LAUNCH("sum_partials_kernel");
    return PB_OK;
}

// coarse_rhs (side (n+1)/2) = P^T (s (rhs - A e)) / 8 on level 0 (side n, diagonal D, weights s).
extern "C" int pb_residual_restrict_f32(const float* e, const float* rhs, const float* D, const float* weights,
                                        float* coarse_rhs, int64_t n, void* stream) {
    if (n < 3 || n > 4097 || !e || !rhs || !D || !weights || !coarse_rhs)
        return fail(PB_ERR_INVALID, "residual_restrict: bad args");
    const int cn = (int)((n + 1) / 2);
    const float h2 = (float)((n - 1) * (n - 1));
    const int cz = (int)tuned(PB_TUNE_RESTRICT_PLANES, n, kRrCZ);
    const dim3 grid((cn + kRrCX - 1) / kRrCX, (cn + kRrCY - 1) / kRrCY, (cn + cz - 1) / cz);
    const int64_t variant = tuned(PB_TUNE_RESTRICT_VARIANT, n, 0);
    auto kernel = variant == 1 ? residual_restrict32_paired_kernel
                  : variant == 3 ? residual_restrict32_paired320_kernel
                                 : residual_restrict32_kernel;
    kernel<<<grid, variant == 3 ? 320 : kRrThreads, 0, (cudaStream_t)stream>>>(e, rhs, D, weights, geom((int)n), h2,
                                                                               coarse_rhs, geom(cn), cz);
    PB_CHECK_LAUNCH("residual_restrict32_kernel");
    return PB_OK;
}


// ---- grouped launches (batch.cuh) ----------------------------------------------------

namespace pb {
namespace batch {

int describe_residual_restrict32(GridDesc& d) {
    const int n = (int)d.n;
    if (n < 3 || n > 4097 || !d.ptr[0] || !d.ptr[1] || !d.ptr[2] || !d.ptr[3] || !d.ptr[4])
        return fail(PB_ERR_INVALID, "batch residual_restrict32: bad args");
    const int cn = (n + 1) / 2;
    d.gx = (cn + kRrCX - 1) / kRrCX;
    d.gy = (cn + kRrCY - 1) / kRrCY;
    const int cz = (int)tuned(PB_TUNE_RESTRICT_PLANES, n, kRrCZ);
    d.gz = (cn + cz - 1) / cz;
    d.aux[0] = cz;
    return PB_OK;
}

int launch_residual_restrict32(const GridDesc* descs, int count, int64_t blocks, const int* flags, cudaStream_t s) {
    residual_restrict32_grouped_kernel<<<(unsigned)blocks, kRrThreads, 0, s>>>(descs, count, flags);
    PB_CHECK_LAUNCH("residual_restrict32_grouped_kernel");
    return PB_OK;
}

}  // namespace batch
}  // namespace pb
