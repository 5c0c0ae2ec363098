// FP32 multigrid inside an FP64 defect-correction loop.
//
// The reference solves A x = b with FP64 V-cycles (src/capi.mojo:310-742,
// python/mojo_poissonrecon/core.py:141-193).  Here the FP64 iterate x is
// refined by corrections e from FP32 V-cycles on A e = r, r = b - A x taken in
// FP64.  The operator, smoother, transfers and cycle shape are the
// reference's; only the precision of the inner cycle changes.
//
// FP32 level layout ("padded"): side n grid stored with a one-node ghost
// layer of zeros on every face, x offset 4, row pitch P (multiple of 8):
//   index(x, y, z) = ((z+1)*(n+2) + (y+1))*P + (x+4),  x,y,z in [-1, n].
// Ghosts stay zero, so a 6-neighbour sum over the padded array equals the
// reference's Neumann sum over in-grid neighbours; the degree term lives in
// the stored diagonal D = (deg + pw*screen) * (n-1)^2.
#include "common.cuh"

namespace pb {

struct Geom {
    int n;          // grid side
    int P;          // row pitch (floats)
    int64_t plane;  // (n+2)*P
    __host__ __device__ __forceinline__ int64_t at(int x, int y, int z) const {
        return ((int64_t)(z + 1) * (n + 2) + (y + 1)) * P + (x + 4);
    }
};

__host__ __device__ inline int pitch_of(int n) { return ((n + 5) + 7) & ~7; }
inline Geom geom(int n) { return Geom{n, pitch_of(n), (int64_t)(n + 2) * pitch_of(n)}; }
inline int64_t padded_size(int n) { return (int64_t)(n + 2) * geom(n).plane; }

// ---- level set-up: D and 1/D from the FP64 screen (dense layout) --------------
__global__ void level_setup_kernel(const double* __restrict__ screen, Geom g, double pw, float* __restrict__ D,
                                   float* __restrict__ invD) {
    const int n = g.n;
    const int64_t total = (int64_t)n * n * n;
    const double h = (double)(n - 1), h2 = h * h;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((int64_t)n * n));
        const int deg = (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
        const double d = (double)deg * h2 + pw * screen[i] * h2;
        const int64_t p = g.at(x, y, z);
        D[p] = (float)d;
        invD[p] = (float)(1.0 / d);
    }
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

// Tiled variant: a block owns a 64 x 4 (x, y) tile and a z range; coordinates
// come from the launch shape (no 64-bit division per node), rows are read
// coalesced, and the z-neighbours of consecutive planes stay in L1/L2.
constexpr int kDefTX = 64, kDefTY = 4, kDefZ = 16;

template <bool UPDATE>
__global__ void __launch_bounds__(kDefTX* kDefTY) defect_tile_kernel(
    const double* __restrict__ x_old, const float* __restrict__ e, double* __restrict__ x_new,
    const double* __restrict__ b, const double* __restrict__ screen, Geom g, double pw, float* __restrict__ r32,
    double* __restrict__ r64, double* __restrict__ partial) {
    __shared__ double shared[32];
    const int n = g.n;
    const int x = blockIdx.x * kDefTX + threadIdx.x;
    const int y = blockIdx.y * kDefTY + threadIdx.y;
    const int z0 = blockIdx.z * kDefZ, z1 = min(n, z0 + kDefZ);
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
    const double t = warp_block_sum(sq, shared);
    if (threadIdx.x == 0 && threadIdx.y == 0)
        partial[(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
}

__global__ void sum_partials_kernel(const double* __restrict__ partial, int count, double* __restrict__ out) {
    __shared__ double shared[32];
    double v = 0.0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) v += partial[i];
    const double t = warp_block_sum(v, shared);
    if (threadIdx.x == 0) *out = t;
}

// Trilinear prolongation of the coarse correction at fine node (x, y, z)
// (capi.mojo:677-742 in FP32).
__device__ __forceinline__ float prolong_at(const float* __restrict__ c, const Geom& gc, int x, int y, int z) {
    const int x0 = x >> 1, y0 = y >> 1, z0 = z >> 1;
    const int x1 = min(x0 + 1, gc.n - 1), y1 = min(y0 + 1, gc.n - 1), z1 = min(z0 + 1, gc.n - 1);
    const float tx = (x & 1) ? 0.5f : 0.0f, ty = (y & 1) ? 0.5f : 0.0f, tz = (z & 1) ? 0.5f : 0.0f;
    const float c00 = c[gc.at(x0, y0, z0)] * (1.f - tx) + c[gc.at(x1, y0, z0)] * tx;
    const float c10 = c[gc.at(x0, y1, z0)] * (1.f - tx) + c[gc.at(x1, y1, z0)] * tx;
    const float c01 = c[gc.at(x0, y0, z1)] * (1.f - tx) + c[gc.at(x1, y0, z1)] * tx;
    const float c11 = c[gc.at(x0, y1, z1)] * (1.f - tx) + c[gc.at(x1, y1, z1)] * tx;
    const float c0 = c00 * (1.f - ty) + c10 * ty;
    const float c1 = c01 * (1.f - ty) + c11 * ty;
    return c0 * (1.f - tz) + c1 * tz;
}

// ---- FP32 residual fused with full-weighting restriction -----------------------
// coarse_rhs = restrict(rhs - A e) (capi.mojo:413-470 then :557-673, in FP32)
// without writing the fine residual.  A block owns a 32 x 4 tile of coarse
// (x, y) and marches coarse z; fine residual planes of the tile plus a halo of
// one (65 x 9 nodes) are computed into a three-plane ring in shared memory,
// plane 2zc+1 being reused as plane 2(zc+1)-1 of the next coarse plane.  The
// restriction weights (1,2,1)^3 over in-grid fine nodes, normalised by their
// sum, as in the reference.
constexpr int kRrCX = 32, kRrCY = 4, kRrCZ = 8;
constexpr int kRrFX = 2 * kRrCX + 1, kRrFY = 2 * kRrCY + 1;  // 65 x 9 fine nodes
constexpr int kRrThreads = 256;

__global__ void __launch_bounds__(kRrThreads) residual_restrict32_kernel(const float* __restrict__ e,
                                                                          const float* __restrict__ rhs,
                                                                          const float* __restrict__ D, Geom gf,
                                                                          float h2, float* __restrict__ coarse,
                                                                          Geom gc) {
    __shared__ float ring[3][kRrFY][kRrFX + 3];
    const int fn = gf.n, cn = gc.n;
    const int xc0 = blockIdx.x * kRrCX, yc0 = blockIdx.y * kRrCY;
    const int zc0 = blockIdx.z * kRrCZ, zc1 = min(cn, zc0 + kRrCZ);
    const int fx0 = 2 * xc0 - 1, fy0 = 2 * yc0 - 1;
    const int tid = threadIdx.x;
    auto fine_plane = [&](int f) {  // residual of fine plane f over the tile region
        float(*dst)[kRrFX + 3] = ring[(f + 3) % 3];
        for (int i = tid; i < kRrFY * kRrFX; i += kRrThreads) {
            const int ly = i / kRrFX, lx = i - ly * kRrFX;
            const int x = fx0 + lx, y = fy0 + ly;
            float r = 0.0f;
            if (f >= 0 && f < fn && x >= 0 && x < fn && y >= 0 && y < fn) {
                const int64_t p = gf.at(x, y, f);
                const float sum = e[p - 1] + e[p + 1] + e[p - gf.P] + e[p + gf.P] + e[p - gf.plane] + e[p + gf.plane];
                r = rhs[p] - (D[p] * e[p] - sum * h2);
            }
            dst[ly][lx] = r;
        }
    };
    fine_plane(2 * zc0 - 1);
    for (int zc = zc0; zc < zc1; ++zc) {
        fine_plane(2 * zc);
        fine_plane(2 * zc + 1);
        __syncthreads();
        if (tid < kRrCX * kRrCY) {
            const int cy = tid / kRrCX, cx = tid - cy * kRrCX;
            const int xc = xc0 + cx, yc = yc0 + cy;
            if (xc < cn && yc < cn) {
                float sum = 0.0f, wsum = 0.0f;
                for (int oz = -1; oz <= 1; ++oz) {
                    const int zz = 2 * zc + oz;
                    if (zz < 0 || zz >= fn) continue;
                    const float wz = oz == 0 ? 2.f : 1.f;
                    for (int oy = -1; oy <= 1; ++oy) {
                        const int yy = 2 * yc + oy;
                        if (yy < 0 || yy >= fn) continue;
                        const float wy = oy == 0 ? 2.f : 1.f;
                        const float* row = ring[(zz + 3) % 3][2 * cy + 1 + oy];
                        for (int ox = -1; ox <= 1; ++ox) {
                            const int xx = 2 * xc + ox;
                            if (xx < 0 || xx >= fn) continue;
                            const float w = (ox == 0 ? 2.f : 1.f) * wy * wz;
                            sum += row[2 * cx + 1 + ox] * w;
                            wsum += w;
                        }
                    }
                }
                coarse[gc.at(xc, yc, zc)] = sum / wsum;
            }
        }
        __syncthreads();  // the ring slots of planes 2zc-1 and 2zc are rewritten next
    }
}

// ---- all levels with n <= kCoarseN in one block ---------------------------------
// The reference's recursion below that size (V(3,3), 40 sweeps at n = 3) with
// __syncthreads between colour passes; arrays stay in the padded layout.
constexpr int kCoarseN = 17;
constexpr int kCoarseThreads = 1024;
constexpr int kMaxLevels = 8;

struct CoarseLevels {
    int count;
    Geom g[kMaxLevels];
    float* e[kMaxLevels];
    float* rhs[kMaxLevels];
    float* res[kMaxLevels];
    const float* D[kMaxLevels];
    const float* invD[kMaxLevels];
};

__device__ void coarse_relax(const CoarseLevels& L, int l, int iters) {
    const Geom g = L.g[l];
    const int n = g.n;
    const float h2 = (float)(n - 1) * (float)(n - 1);
    float* e = L.e[l];
    const float* rhs = L.rhs[l];
    const float* invD = L.invD[l];
    const int total = n * n * n;
    for (int it = 0; it < iters; ++it)
        for (int colour = 0; colour < 2; ++colour) {
            for (int i = threadIdx.x; i < total; i += blockDim.x) {
                const int x = i % n, y = (i / n) % n, z = i / (n * n);
                if (((x + y + z) & 1) != colour) continue;
                const int64_t p = g.at(x, y, z);
                const float s = e[p - 1] + e[p + 1] + e[p - g.P] + e[p + g.P] + e[p - g.plane] + e[p + g.plane];
                e[p] = (rhs[p] + s * h2) * invD[p];
            }
            __syncthreads();
        }
}

__global__ void __launch_bounds__(kCoarseThreads) coarse_cycle_kernel(CoarseLevels L, int pre, int post, int coarsest) {
    // descend
    for (int l = 0; l < L.count; ++l) {
        const Geom g = L.g[l];
        const int n = g.n;
        // e = 0 on the interior (ghosts are already zero)
        for (int i = threadIdx.x; i < n * n * n; i += blockDim.x) {
            const int x = i % n, y = (i / n) % n, z = i / (n * n);
            L.e[l][g.at(x, y, z)] = 0.0f;
        }
        __syncthreads();
        if (l == L.count - 1) {
            coarse_relax(L, l, coarsest);
            break;
        }
        coarse_relax(L, l, pre);
        const float h2 = (float)(n - 1) * (float)(n - 1);
        for (int i = threadIdx.x; i < n * n * n; i += blockDim.x) {
            const int x = i % n, y = (i / n) % n, z = i / (n * n);
            const int64_t p = g.at(x, y, z);
            const float* e = L.e[l];
            const float s = e[p - 1] + e[p + 1] + e[p - g.P] + e[p + g.P] + e[p - g.plane] + e[p + g.plane];
            L.res[l][p] = L.rhs[l][p] - (L.D[l][p] * e[p] - s * h2);
        }
        __syncthreads();
        const Geom gc = L.g[l + 1];
        const int cn = gc.n;
        for (int i = threadIdx.x; i < cn * cn * cn; i += blockDim.x) {
            const int x = i % cn, y = (i / cn) % cn, z = i / (cn * cn);
            float sum = 0.0f, wsum = 0.0f;
            for (int oz = -1; oz <= 1; ++oz) {
                const int zz = 2 * z + oz;
                if (zz < 0 || zz >= n) continue;
                for (int oy = -1; oy <= 1; ++oy) {
                    const int yy = 2 * y + oy;
                    if (yy < 0 || yy >= n) continue;
                    for (int ox = -1; ox <= 1; ++ox) {
                        const int xx = 2 * x + ox;
                        if (xx < 0 || xx >= n) continue;
                        const float w = (ox == 0 ? 2.f : 1.f) * (oy == 0 ? 2.f : 1.f) * (oz == 0 ? 2.f : 1.f);
                        sum += L.res[l][g.at(xx, yy, zz)] * w;
                        wsum += w;
                    }
                }
            }
            L.rhs[l + 1][gc.at(x, y, z)] = sum / wsum;
        }
        __syncthreads();
    }
    // ascend
    for (int l = L.count - 2; l >= 0; --l) {
        const Geom g = L.g[l], gc = L.g[l + 1];
        const int n = g.n;
        for (int i = threadIdx.x; i < n * n * n; i += blockDim.x) {
            const int x = i % n, y = (i / n) % n, z = i / (n * n);
            L.e[l][g.at(x, y, z)] += prolong_at(L.e[l + 1], gc, x, y, z);
        }
        __syncthreads();
        coarse_relax(L, l, post);
    }
}

static unsigned stride_grid(int64_t items, int threads, int per_sm = 16) {
    int64_t b = (items + threads - 1) / threads;
    const int64_t cap = (int64_t)kSMs * per_sm;
    if (b > cap) b = cap;
    return (unsigned)(b < 1 ? 1 : b);
}

static dim3 defect_grid(int n) {
    return dim3((n + kDefTX - 1) / kDefTX, (n + kDefTY - 1) / kDefTY, (n + kDefZ - 1) / kDefZ);
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
                                  void* stream) {
    if (n < 2 || n > 4097 || !screen || !D || !invD) return fail(PB_ERR_INVALID, "level setup: bad args");
    level_setup_kernel<<<stride_grid(n * n * n, 256), 256, 0, (cudaStream_t)stream>>>(screen, geom((int)n),
                                                                                     point_weight, D, invD);
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
    const dim3 grid = defect_grid((int)n), block(kDefTX, kDefTY);
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

// coarse_rhs (side (n+1)/2) = full-weighting restriction of rhs - A e on side n.
extern "C" int pb_residual_restrict_f32(const float* e, const float* rhs, const float* D, float* coarse_rhs,
                                        int64_t n, void* stream) {
    if (n < 3 || n > 4097 || !e || !rhs || !D || !coarse_rhs) return fail(PB_ERR_INVALID, "residual_restrict: bad args");
    const int cn = (int)((n + 1) / 2);
    const float h2 = (float)((n - 1) * (n - 1));
    const dim3 grid((cn + kRrCX - 1) / kRrCX, (cn + kRrCY - 1) / kRrCY, (cn + kRrCZ - 1) / kRrCZ);
    residual_restrict32_kernel<<<grid, kRrThreads, 0, (cudaStream_t)stream>>>(e, rhs, D, geom((int)n), h2,
                                                                              coarse_rhs, geom(cn));
    PB_CHECK_LAUNCH("residual_restrict32_kernel");
    return PB_OK;
}

// Levels with side <= 17 in one block.  Arrays of `count` levels, finest first,
// each in the padded layout; rhs[0] holds the restricted residual from above.
extern "C" int pb_coarse_cycle_f32(int64_t count, const int64_t* sizes, float* const* e, float* const* rhs,
                                   float* const* res, const float* const* D, const float* const* invD, int64_t pre,
                                   int64_t post, int64_t coarsest_sweeps, void* stream) {
    if (count < 1 || count > kMaxLevels || !sizes || !e || !rhs || !res || !D || !invD)
        return fail(PB_ERR_INVALID, "coarse cycle: bad args");
    CoarseLevels L;
    L.count = (int)count;
    for (int l = 0; l < count; ++l) {
        if (sizes[l] < 2 || sizes[l] > kCoarseN || (l && sizes[l] != (sizes[l - 1] + 1) / 2))
            return fail(PB_ERR_INVALID, "coarse cycle: bad level sizes");
        L.g[l] = geom((int)sizes[l]);
        L.e[l] = e[l];
        L.rhs[l] = rhs[l];
        L.res[l] = res[l];
        L.D[l] = D[l];
        L.invD[l] = invD[l];
    }
    coarse_cycle_kernel<<<1, kCoarseThreads, 0, (cudaStream_t)stream>>>(L, (int)pre, (int)post, (int)coarsest_sweeps);
    PB_CHECK_LAUNCH("coarse_cycle_kernel");
    return PB_OK;
}
