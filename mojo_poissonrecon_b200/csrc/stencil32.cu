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

// ---- fused red-black sweep, out of place -------------------------------------
// Colour 0 = (x+y+z) even, updated first (capi.mojo:403-405).  A block owns an
// (x, y) tile and a z range and marches z with a three-plane ring of input
// values (halo 2) and of updated colour-0 values (halo 1): at step t it loads
// input plane t+1, updates colour 0 on plane t, then colour 1 on plane t-1 and
// writes plane t-1.  Input modes: ZERO_IN (e = 0), PROLONG (e_in + trilinear
// prolongation of the coarse correction, capi.mojo:677-742, fused into the load).
constexpr int kTX = 64;          // tile width (the last x tile may hold kTX + 1 columns)
constexpr int kTY = 8;           // tile height (the last y tile may hold kTY + 1 rows)
constexpr int kSX = kTX + 1 + 4; // shared row length for the input ring (halo 2)
constexpr int kSY = kTY + 1 + 4;
constexpr int kRX = kTX + 1 + 2; // colour-0 ring (halo 1)
constexpr int kRY = kTY + 1 + 2;
constexpr int kSweepThreads = 256;

struct Tile {
    int x0, x1, y0, y1;  // interior [x0, x1) x [y0, y1)
};

__device__ __forceinline__ Tile tile_of(int n, int bx, int by) {
    const int ntx = (n - 1) / kTX > 0 ? (n - 1) / kTX : 1;
    const int nty = (n - 1) / kTY > 0 ? (n - 1) / kTY : 1;
    Tile t;
    t.x0 = bx * kTX;
    t.x1 = bx == ntx - 1 ? n : t.x0 + kTX;
    t.y0 = by * kTY;
    t.y1 = by == nty - 1 ? n : t.y0 + kTY;
    return t;
}

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

template <int MODE>  // 0 = plain input, 1 = zero input, 2 = input + prolongation
__global__ void __launch_bounds__(kSweepThreads) rb_sweep_kernel(const float* __restrict__ e_in,
                                                                 float* __restrict__ e_out,
                                                                 const float* __restrict__ rhs,
                                                                 const float* __restrict__ invD,
                                                                 const float* __restrict__ coarse, Geom g, Geom gc,
                                                                 float h2, int z_chunk) {
    __shared__ float in_ring[3][kSY][kSX];
    __shared__ float red_ring[3][kRY][kRX];
    const int n = g.n;
    const Tile T = tile_of(n, blockIdx.x, blockIdx.y);
    const int zb = blockIdx.z * z_chunk;
    const int ze = min(n, zb + z_chunk);
    const int W = T.x1 - T.x0, H = T.y1 - T.y0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = kSweepThreads / 32;

    auto load_plane = [&](int z) {
        float(*dst)[kSX] = in_ring[(z + 3) % 3];
        for (int ly = warp; ly < H + 4; ly += warps) {
            const int y = T.y0 - 2 + ly;
            for (int lx = lane; lx < W + 4; lx += 32) {
                const int x = T.x0 - 2 + lx;
                float v = 0.0f;
                if (MODE != 1 && z >= 0 && z < n && x >= 0 && x < n && y >= 0 && y < n) {
                    v = e_in[g.at(x, y, z)];
                    if (MODE == 2) v += prolong_at(coarse, gc, x, y, z);
                }
                dst[ly][lx] = v;
            }
        }
    };
    // colour-0 nodes of plane z on the halo-1 region
    auto red_plane = [&](int z) {
        float(*dst)[kRX] = red_ring[(z + 3) % 3];
        const float(*cm)[kSX] = in_ring[(z + 2) % 3];
        const float(*cc)[kSX] = in_ring[(z + 3) % 3];
        const float(*cp)[kSX] = in_ring[(z + 4) % 3];
        for (int ly = warp; ly < H + 2; ly += warps) {
            const int y = T.y0 - 1 + ly;
            for (int lx = lane; lx < W + 2; lx += 32) {
                const int x = T.x0 - 1 + lx;
                float v = 0.0f;
                if (z >= 0 && z < n && x >= 0 && x < n && y >= 0 && y < n && ((x + y + z) & 1) == 0) {
                    const int sy = ly + 1, sx = lx + 1;
                    const float s = cc[sy][sx - 1] + cc[sy][sx + 1] + cc[sy - 1][sx] + cc[sy + 1][sx] + cm[sy][sx] +
                                    cp[sy][sx];
                    const int64_t p = g.at(x, y, z);
                    v = (rhs[p] + s * h2) * invD[p];
                }
                dst[ly][lx] = v;
            }
        }
    };
    // colour-1 nodes of plane z on the interior, and the output plane
    auto black_plane = [&](int z) {
        const float(*rm)[kRX] = red_ring[(z + 2) % 3];
        const float(*rc)[kRX] = red_ring[(z + 3) % 3];
        const float(*rp)[kRX] = red_ring[(z + 4) % 3];
        for (int ly = warp; ly < H; ly += warps) {
            const int y = T.y0 + ly;
            for (int lx = lane; lx < W; lx += 32) {
                const int x = T.x0 + lx;
                const int sy = ly + 1, sx = lx + 1;
                const int64_t p = g.at(x, y, z);
                float v;
                if (((x + y + z) & 1) == 0) {
                    v = rc[sy][sx];
                } else {
                    const float s = rc[sy][sx - 1] + rc[sy][sx + 1] + rc[sy - 1][sx] + rc[sy + 1][sx] + rm[sy][sx] +
                                    rp[sy][sx];
                    v = (rhs[p] + s * h2) * invD[p];
                }
                e_out[p] = v;
            }
        }
    };

    // Ring discipline: load(t+1) overwrites plane t-2, last read by red(t-1);
    // red(t) overwrites colour-0 plane t-3, last read by black(t-2).  The two
    // barriers per step separate exactly those pairs.
    load_plane(zb - 2);
    load_plane(zb - 1);
    load_plane(zb);
    __syncthreads();
    red_plane(zb - 1);  // zero outside the grid
    __syncthreads();
    for (int t = zb; t <= ze; ++t) {
        load_plane(t + 1);
        __syncthreads();
        red_plane(t);
        __syncthreads();
        if (t - 1 >= zb) black_plane(t - 1);
    }
}

// ---- FP32 residual (padded) and full-weighting restriction -------------------
__global__ void residual32_kernel(const float* __restrict__ e, const float* __restrict__ rhs,
                                  const float* __restrict__ D, Geom g, float h2, float* __restrict__ res) {
    const int n = g.n;
    const int64_t total = (int64_t)n * n * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((int64_t)n * n));
        const int64_t p = g.at(x, y, z);
        const float s = e[p - 1] + e[p + 1] + e[p - g.P] + e[p + g.P] + e[p - g.plane] + e[p + g.plane];
        res[p] = rhs[p] - (D[p] * e[p] - s * h2);
    }
}

// capi.mojo:557-673 in FP32 on the padded layout: weights (1,2,1)^3 over the
// in-grid fine nodes, normalised by their sum.
__global__ void restrict32_kernel(const float* __restrict__ fine, Geom gf, float* __restrict__ coarse, Geom gc) {
    const int cn = gc.n, fn = gf.n;
    const int64_t total = (int64_t)cn * cn * cn;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % cn), y = (int)((i / cn) % cn), z = (int)(i / ((int64_t)cn * cn));
        float sum = 0.0f, wsum = 0.0f;
        for (int oz = -1; oz <= 1; ++oz) {
            const int zz = 2 * z + oz;
            if (zz < 0 || zz >= fn) continue;
            const float wz = oz == 0 ? 2.f : 1.f;
            for (int oy = -1; oy <= 1; ++oy) {
                const int yy = 2 * y + oy;
                if (yy < 0 || yy >= fn) continue;
                const float wy = oy == 0 ? 2.f : 1.f;
                const float* row = fine + gf.at(0, yy, zz);
                for (int ox = -1; ox <= 1; ++ox) {
                    const int xx = 2 * x + ox;
                    if (xx < 0 || xx >= fn) continue;
                    const float w = (ox == 0 ? 2.f : 1.f) * wy * wz;
                    sum += row[xx] * w;
                    wsum += w;
                }
            }
        }
        coarse[gc.at(x, y, z)] = sum / wsum;
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

static dim3 sweep_grid(int n, int z_chunk) {
    const int ntx = (n - 1) / kTX > 0 ? (n - 1) / kTX : 1;
    const int nty = (n - 1) / kTY > 0 ? (n - 1) / kTY : 1;
    return dim3(ntx, nty, (n + z_chunk - 1) / z_chunk);
}

// One fused red-black sweep e_out <- sweep(e_in).  mode 0: e_in as is; 1: e_in
// taken as zero (e_in may be NULL); 2: e_in + prolongation of `coarse` (side
// (n+1)/2).  The grid side must satisfy n = 2^k + 1 or n <= kTX + 1.
extern "C" int pb_sweep_f32(const float* e_in, float* e_out, const float* rhs, const float* invD, const float* coarse,
                            int64_t n, int64_t mode, int64_t z_chunk, void* stream) {
    if (n < 2 || n > 4097 || !e_out || !rhs || !invD || (mode != 1 && !e_in) || (mode == 2 && !coarse) || mode < 0 ||
        mode > 2)
        return fail(PB_ERR_INVALID, "sweep: bad args");
    if (e_in == e_out) return fail(PB_ERR_INVALID, "sweep: out of place only");
    const int ntx = (int)((n - 1) / kTX > 0 ? (n - 1) / kTX : 1);
    const int nty = (int)((n - 1) / kTY > 0 ? (n - 1) / kTY : 1);
    if (n - (int64_t)(ntx - 1) * kTX > kTX + 1 || n - (int64_t)(nty - 1) * kTY > kTY + 1)
        return fail(PB_ERR_INVALID, "sweep: n = %lld does not tile (needs n = 2^k + 1)", (long long)n);
    if (z_chunk < 1) z_chunk = 32;
    const Geom g = geom((int)n);
    const Geom gc = geom((int)((n + 1) / 2));
    const float h2 = (float)((n - 1) * (n - 1));
    const dim3 grid = sweep_grid((int)n, (int)z_chunk);
    cudaStream_t s = (cudaStream_t)stream;
    if (mode == 0)
        rb_sweep_kernel<0><<<grid, kSweepThreads, 0, s>>>(e_in, e_out, rhs, invD, nullptr, g, gc, h2, (int)z_chunk);
    else if (mode == 1)
        rb_sweep_kernel<1><<<grid, kSweepThreads, 0, s>>>(nullptr, e_out, rhs, invD, nullptr, g, gc, h2, (int)z_chunk);
    else
        rb_sweep_kernel<2><<<grid, kSweepThreads, 0, s>>>(e_in, e_out, rhs, invD, coarse, g, gc, h2, (int)z_chunk);
    PB_CHECK_LAUNCH("rb_sweep_kernel");
    return PB_OK;
}

extern "C" int pb_residual_f32(const float* e, const float* rhs, const float* D, float* res, int64_t n, void* stream) {
    if (n < 2 || n > 4097 || !e || !rhs || !D || !res) return fail(PB_ERR_INVALID, "residual32: bad args");
    const float h2 = (float)((n - 1) * (n - 1));
    residual32_kernel<<<stride_grid(n * n * n, 256), 256, 0, (cudaStream_t)stream>>>(e, rhs, D, geom((int)n), h2, res);
    PB_CHECK_LAUNCH("residual32_kernel");
    return PB_OK;
}

extern "C" int pb_restrict_f32(const float* fine, float* coarse, int64_t fine_n, void* stream) {
    if (fine_n < 3 || fine_n > 4097 || !fine || !coarse) return fail(PB_ERR_INVALID, "restrict32: bad args");
    const int cn = (int)((fine_n + 1) / 2);
    restrict32_kernel<<<stride_grid((int64_t)cn * cn * cn, 256), 256, 0, (cudaStream_t)stream>>>(
        fine, geom((int)fine_n), coarse, geom(cn));
    PB_CHECK_LAUNCH("restrict32_kernel");
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
