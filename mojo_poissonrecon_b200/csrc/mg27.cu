// Galerkin coarse levels of the FP32 preconditioner.
//
// The reference's coarse levels rediscretise the operator (screen restricted
// and scaled by 4 per level, python/mojo_poissonrecon/core.py:267-269) and
// transfer with trilinear prolongation and boundary-normalised full weighting
// (src/capi.mojo:557-742).  The screening term pw*screen is concentrated on a
// thin shell of nodes around the samples, where it outweighs the Laplacian by
// one to two orders of magnitude; across that shell a trilinear coarse
// correction is wrong by O(1), and the reference-shaped cycle reduces the
// residual by only about 0.35 per cycle even with an exact coarse solve.  The
// FP32 preconditioner keeps the reference's fine operator and red-black
// smoother on level 0 and replaces the coarse side:
//   prolongation  P_s = S P, P trilinear, S = diag(s) with s_i = 1 where the
//                 fine node coincides with a coarse node, else
//                 s_i = (sum_{j != i} -a_ij) / a_ii  (deg / (deg + pw*screen)
//                 on level 0): a correction is damped where screening
//                 dominates the row;
//   restriction   R = P_s^T / 8 (full weighting scaled by s, not renormalised);
//   coarse ops    A_c = R A P_s (Galerkin), 27-point and symmetric;
//   coarsest      the 3^3 level solved exactly with its inverse.
// That cycle reduces the residual by about 0.03-0.05 per cycle independent of
// depth.  The FP64 outer loop still measures convergence with the reference's
// operator, so the answer is the reference's to the requested tolerance.
//
// Smoothing on 27-point levels: red-black ordered, same-colour couplings
// taken from the previous iterate (two passes per sweep, e_prev -> e_next,
// no in-place race); levels of side > 9 with their couplings packed per colour
// (see "packed 27-point levels" below), the smaller ones in one block.
//
// Storage of a 27-point level: 14 coefficient planes in the padded layout
// (level32.cuh), plane stride = padded_size(n); plane 0 the diagonal, planes
// 1..13 the couplings to the 13 "forward" neighbours J+K (K.z > 0; or K.z == 0
// and K.y > 0; or K = (1,0,0)).  The coupling to a backward neighbour J-K is
// plane k(K) at J-K (symmetry).  Ghost entries are zero.
#include <cuda_fp16.h>

#include "batch.cuh"
#include "common.cuh"
#include "level32.cuh"

namespace pb {

__host__ __device__ constexpr bool is_forward(int dx, int dy, int dz) {
    return dz > 0 || (dz == 0 && (dy > 0 || (dy == 0 && dx > 0)));
}
__host__ __device__ constexpr int fwd_index(int dx, int dy, int dz) {
    return dz == 1 ? 1 + (dy + 1) * 3 + (dx + 1) : (dy == 1 ? 10 + (dx + 1) : 13);
}
__host__ __device__ constexpr float wt(int d) { return d == 0 ? 1.0f : 0.5f; }

__device__ __forceinline__ int64_t offset_of(const Geom& g, int dx, int dy, int dz) {
    return (int64_t)dx + (int64_t)dy * g.P + (int64_t)dz * g.plane;
}

// a(J, J+K) for the node at padded index p.
__device__ __forceinline__ float coupling(const float* __restrict__ c, int64_t cs, const Geom& g, int64_t p, int dx,
                                          int dy, int dz) {
    if (dx == 0 && dy == 0 && dz == 0) return c[p];
    if (is_forward(dx, dy, dz)) return c[fwd_index(dx, dy, dz) * cs + p];
    return c[fwd_index(-dx, -dy, -dz) * cs + p + offset_of(g, dx, dy, dz)];
}

__device__ __forceinline__ bool inside(int x, int y, int z, int n) {
    return (unsigned)x < (unsigned)n && (unsigned)y < (unsigned)n && (unsigned)z < (unsigned)n;
}

// Node of this thread on a level of side m, threads flattened over each plane's
// (x, y) (blockIdx.x) with the plane in blockIdx.y: full warps on 2^k + 1 sides.
// False past the plane's last node.
__device__ __forceinline__ bool plane_node(int m, int& x, int& y, int& z) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (unsigned)(m * m)) return false;
    y = (int)(t / (unsigned)m);
    x = (int)(t - (unsigned)y * m);
    z = blockIdx.y;
    return true;
}

inline dim3 plane_grid(int m, int threads) { return dim3((m * m + threads - 1) / threads, m); }

// ---- Galerkin product A_c = P_s^T A P_s / 8 from level 0 ------------------------
// One thread per coarse node J streams once over the fine nodes i = 2J + o of
// J's support (27) and their 7-point stencil neighbours j = i + K, and
// scatters the product p_iJ a_ij s_j into the stored entries A_c[J, J+m]
// (m = 0 or forward) whose column support holds j, with weight P(d - 2m),
// d = o + K.  Every index and weight is resolved at compile time, so the 14
// sums stay in registers.  (From a 27-point level the product is separable:
// see the x, y, z stages below.)
__device__ __forceinline__ void scatter14(float v, int dx, int dy, int dz, float* acc) {
#pragma unroll
    for (int mz = -1; mz <= 1; ++mz)
#pragma unroll
        for (int my = -1; my <= 1; ++my)
#pragma unroll
            for (int mx = -1; mx <= 1; ++mx) {
                const int ex = dx - 2 * mx, ey = dy - 2 * my, ez = dz - 2 * mz;
                if (ex < -1 || ex > 1 || ey < -1 || ey > 1 || ez < -1 || ez > 1) continue;
                const bool centre = mx == 0 && my == 0 && mz == 0;
                if (!centre && !is_forward(mx, my, mz)) continue;
                acc[centre ? 0 : fwd_index(mx, my, mz)] += v * (wt(ex) * wt(ey) * wt(ez));
            }
}

// The sums for one coarse node below level 0: `D` is the level-0 diagonal
// (couplings -h2 to in-grid face neighbours), S its prolongation weights.
// INTERIOR: every i and j of J lies in the grid (no bounds tests).
template <bool INTERIOR>
__device__ __forceinline__ void galerkin7_sums(const float* __restrict__ D, const float* __restrict__ S,
                                               const Geom& gf, float h2, int xc, int yc, int zc, float* acc) {
    const int fn = gf.n;
#pragma unroll
    for (int oz = -1; oz <= 1; ++oz)
#pragma unroll
        for (int oy = -1; oy <= 1; ++oy)
#pragma unroll
            for (int ox = -1; ox <= 1; ++ox) {
                const int xi = 2 * xc + ox, yi = 2 * yc + oy, zi = 2 * zc + oz;
                if (!INTERIOR && !inside(xi, yi, zi, fn)) continue;
                const int64_t pi = gf.at(xi, yi, zi);
                const float si = wt(ox) * wt(oy) * wt(oz) * S[pi];
#pragma unroll
                for (int kz = -1; kz <= 1; ++kz)
#pragma unroll
                    for (int ky = -1; ky <= 1; ++ky)
#pragma unroll
                        for (int kx = -1; kx <= 1; ++kx) {
                            if ((kx != 0) + (ky != 0) + (kz != 0) > 1) continue;  // 7-point stencil
                            if (!INTERIOR && !inside(xi + kx, yi + ky, zi + kz, fn)) continue;
                            const float a = (kx == 0 && ky == 0 && kz == 0) ? D[pi] : -h2;
                            scatter14(si * a * S[pi + offset_of(gf, kx, ky, kz)], ox + kx, oy + ky, oz + kz, acc);
                        }
            }
}

__device__ __forceinline__ void galerkin_store(const float* acc, float* __restrict__ cc, int64_t cs, const Geom& gc,
                                               int xc, int yc, int zc) {
    const int64_t p = gc.at(xc, yc, zc);
    cc[p] = acc[0] * 0.125f;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx)
                if (is_forward(dx, dy, dz)) {
                    const int k = fwd_index(dx, dy, dz);
                    cc[k * cs + p] = inside(xc + dx, yc + dy, zc + dz, gc.n) ? acc[k] * 0.125f : 0.0f;
                }
}

// Level 0 as the fine level: interior coarse nodes take the branch-free sums.
__global__ void __launch_bounds__(128) galerkin7_kernel(const float* __restrict__ D, const float* __restrict__ S,
                                                        Geom gf, float h2, float* __restrict__ cc, int64_t cs,
                                                        Geom gc) {
    const int cn = gc.n;
    int xc, yc, zc;
    if (!plane_node(cn, xc, yc, zc)) return;
    float acc[14];
#pragma unroll
    for (int k = 0; k < 14; ++k) acc[k] = 0.0f;
    if (xc >= 1 && yc >= 1 && zc >= 1 && xc <= cn - 2 && yc <= cn - 2 && zc <= cn - 2)
        galerkin7_sums<true>(D, S, gf, h2, xc, yc, zc, acc);
    else
        galerkin7_sums<false>(D, S, gf, h2, xc, yc, zc, acc);
    galerkin_store(acc, cc, cs, gc, xc, yc, zc);
}

// ---- separable product for a 27-point fine level ---------------------------------
// P is the tensor product of 1D linear interpolation (coarse M -> fine j with
// weight 1 at j = 2M and 1/2 at j = 2M +- 1), so P^T (S A S) P / 8 contracts
// one axis at a time: x, then y, then z.  Each stage maps fine positions 2M +
// a (a in {-1, 0, 1}) and their offsets d to coarse offsets m with weights
// P(a) P(a + d - 2m), keeping the other two axes' offsets, and takes 81
// products per output node against the direct sum's 27 x 27 per coarse node
// scattered over 14 entries.  Stages x and y write full 27-entry stencils,
// entry e = (oz+1)*9 + (oy+1)*3 + (ox+1), as 27 planes of a dense grid into
// scratch, a slab of fine z-planes at a time; stage z writes the 14 stored
// planes.  Out-of-grid fine nodes and neighbours contribute nothing.
__host__ __device__ constexpr float wt1(int d) { return d == 0 ? 1.0f : (d == 1 || d == -1 ? 0.5f : 0.0f); }

// Stage x: node (I, y, z) of the grid cn x fn x (slab of fine z from zlo);
// entry (m, dy, dz) = sum over a, dx of P(a) s_i a(i, j) s_j P(a + dx - 2m),
// i = (2I + a, y, z), j = i + (dx, dy, dz).
__global__ void __launch_bounds__(128) galerkin_x_kernel(const float* __restrict__ c, int64_t cs,
                                                         const float* __restrict__ S, Geom gf, int cn, int zlo,
                                                         float* __restrict__ out, int64_t ps) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;  // flattened over (I, y)
    const int fn = gf.n;
    if (t >= (unsigned)(cn * fn)) return;
    const int y = (int)(t / (unsigned)cn), I = (int)(t - (unsigned)y * cn);
    const int z = zlo + blockIdx.y;
    const int64_t o = ((int64_t)blockIdx.y * fn + y) * cn + I;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
            float acc[3] = {0.0f, 0.0f, 0.0f};
            if (inside(0, y + dy, z + dz, fn)) {
#pragma unroll
                for (int a = -1; a <= 1; ++a) {
                    const int xi = 2 * I + a;
                    if (xi < 0 || xi >= fn) continue;
                    const int64_t pi = gf.at(xi, y, z);
                    const float si = wt1(a) * S[pi];
#pragma unroll
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (xi + dx < 0 || xi + dx >= fn) continue;
                        const float t = si * coupling(c, cs, gf, pi, dx, dy, dz) * S[pi + offset_of(gf, dx, dy, dz)];
#pragma unroll
                        for (int m = -1; m <= 1; ++m)
                            if (wt1(a + dx - 2 * m) != 0.0f) acc[m + 1] += t * wt1(a + dx - 2 * m);
                    }
                }
            }
#pragma unroll
            for (int m = -1; m <= 1; ++m) out[((dz + 1) * 9 + (dy + 1) * 3 + (m + 1)) * ps + o] = acc[m + 1];
        }
}

// Stage y: node (I, J, z) of cn x cn x slab from stage x's cn x fn x slab.
__global__ void __launch_bounds__(128) galerkin_y_kernel(const float* __restrict__ in, int64_t pin, int fn, int cn,
                                                         float* __restrict__ out, int64_t pout) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;  // flattened over (I, J)
    if (t >= (unsigned)(cn * cn)) return;
    const int J = (int)(t / (unsigned)cn), I = (int)(t - (unsigned)J * cn);
    const int zr = blockIdx.y;
    const int64_t o = ((int64_t)zr * cn + J) * cn + I;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int m = -1; m <= 1; ++m) {
            float acc[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int b = -1; b <= 1; ++b) {
                const int yj = 2 * J + b;
                if (yj < 0 || yj >= fn) continue;
                const int64_t q = ((int64_t)zr * fn + yj) * cn + I;
#pragma unroll
                for (int dy = -1; dy <= 1; ++dy) {
                    const float v = wt1(b) * in[((dz + 1) * 9 + (dy + 1) * 3 + (m + 1)) * pin + q];
#pragma unroll
                    for (int my = -1; my <= 1; ++my)
                        if (wt1(b + dy - 2 * my) != 0.0f) acc[my + 1] += v * wt1(b + dy - 2 * my);
                }
            }
#pragma unroll
            for (int my = -1; my <= 1; ++my) out[((dz + 1) * 9 + (my + 1) * 3 + (m + 1)) * pout + o] = acc[my + 1];
        }
}

// Stage z: coarse node (I, J, K), K in [k0, k1), from stage y's slab (fine z
// from zlo, nz planes); the diagonal and the 13 forward couplings / 8 into the
// 14 planes, zero where the coarse neighbour lies outside the grid.
__global__ void __launch_bounds__(128) galerkin_z_kernel(const float* __restrict__ in, int64_t pin, int fn, int zlo,
                                                         int k0, float* __restrict__ cc, int64_t cs, Geom gc) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;  // flattened over (I, J)
    const int cn = gc.n;
    if (t >= (unsigned)(cn * cn)) return;
    const int J = (int)(t / (unsigned)cn), I = (int)(t - (unsigned)J * cn);
    const int K = k0 + blockIdx.y;
    const int64_t p = gc.at(I, J, K);
#pragma unroll
    for (int my = -1; my <= 1; ++my)
#pragma unroll
        for (int m = -1; m <= 1; ++m) {
            float acc[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int c = -1; c <= 1; ++c) {
                const int zf = 2 * K + c;
                if (zf < 0 || zf >= fn) continue;
                const int64_t q = ((int64_t)(zf - zlo) * cn + J) * cn + I;
#pragma unroll
                for (int dz = -1; dz <= 1; ++dz) {
                    const float v = wt1(c) * in[((dz + 1) * 9 + (my + 1) * 3 + (m + 1)) * pin + q];
#pragma unroll
                    for (int mz = -1; mz <= 1; ++mz)
                        if (wt1(c + dz - 2 * mz) != 0.0f) acc[mz + 1] += v * wt1(c + dz - 2 * mz);
                }
            }
#pragma unroll
            for (int mz = -1; mz <= 1; ++mz) {
                const bool centre = m == 0 && my == 0 && mz == 0;
                if (!centre && !is_forward(m, my, mz)) continue;
                const float val = inside(I + m, J + my, K + mz, cn) ? acc[mz + 1] * 0.125f : 0.0f;
                cc[(centre ? 0 : fwd_index(m, my, mz)) * cs + p] = val;
            }
        }
}

// A 7-point level (diagonal D, off-diagonals -h2 inside the grid) as 14 planes.
__global__ void level7_to_27_kernel(const float* __restrict__ D, Geom g, float h2, float* __restrict__ c, int64_t cs) {
    const int n = g.n;
    int x, y, z;
    if (!plane_node(n, x, y, z)) return;
    const int64_t p = g.at(x, y, z);
    c[p] = D[p];
#pragma unroll
    for (int k = 1; k <= 13; ++k) c[k * cs + p] = 0.0f;
    c[fwd_index(1, 0, 0) * cs + p] = x + 1 < n ? -h2 : 0.0f;
    c[fwd_index(0, 1, 0) * cs + p] = y + 1 < n ? -h2 : 0.0f;
    c[fwd_index(0, 0, 1) * cs + p] = z + 1 < n ? -h2 : 0.0f;
}

// 1/a_JJ and the prolongation weight s_J of a 27-point level.
__global__ void level27_finish_kernel(const float* __restrict__ c, int64_t cs, Geom g, float* __restrict__ invD,
                                      float* __restrict__ fac) {
    const int n = g.n;
    int x, y, z;
    if (!plane_node(n, x, y, z)) return;
    const int64_t p = g.at(x, y, z);
    float off = 0.0f;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx)
                if (dx || dy || dz) off -= coupling(c, cs, g, p, dx, dy, dz);
    const float d = c[p];
    invD[p] = 1.0f / d;
    float s = 1.0f;
    if ((x | y | z) & 1) s = fminf(fmaxf(off / d, 0.0f), 1.0f);
    fac[p] = s;
}

// ---- 27-point smoothing, residual, transfers ------------------------------------
// coarse[J] = sum_o w(o)/64 res[2J+o], w = prod (2 on the axis, 1 off it);
// out-of-grid fine nodes are ghosts holding zero.
__device__ __forceinline__ void restrict27_body(const float* __restrict__ res, Geom gf, float* __restrict__ coarse,
                                                Geom gc, int bx, int by) {
    const unsigned t = bx * blockDim.x + threadIdx.x;
    if (t >= (unsigned)(gc.n * gc.n)) return;
    const int y = (int)(t / (unsigned)gc.n), x = (int)(t - (unsigned)y * gc.n), z = by;
    const int64_t p = gf.at(2 * x, 2 * y, 2 * z);
    float s = 0.0f;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx)
                s += res[p + offset_of(gf, dx, dy, dz)] * (float)((dx ? 1 : 2) * (dy ? 1 : 2) * (dz ? 1 : 2));
    coarse[gc.at(x, y, z)] = s * (1.0f / 64.0f);
}

__global__ void __launch_bounds__(256) restrict27_kernel(const float* __restrict__ res, Geom gf,
                                                         float* __restrict__ coarse, Geom gc) {
    restrict27_body(res, gf, coarse, gc, blockIdx.x, blockIdx.y);
}

// ---- packed 27-point levels: per-colour FP16 couplings --------------------------
// A colour pass over the 14-plane storage reads its nodes' forward coupling
// planes with stride 2 and the backward couplings at neighbours: about 140
// bytes per node and sweep from DRAM on the 129^3 level.  Packed, each colour's nodes are
// numbered compactly (row (y, z), i-th node of the colour: x = 2i + ((y+z+c)&1),
// compact index (z*n + y)*Pc + i, Pc = (n+1)/2) and hold their 26 couplings
// divided by the diagonal, c_K = -a(J, J+K) / a(J, J), in FP16 (|c_K| <= 1),
// node-major: 32 halves (64 bytes, the last 6 zero) per node, coupling k =
// offset index over (dz, dy, dx) in lexicographic order with the centre
// skipped, read as four 16-byte loads; and 1/a(J, J) in FP32.  Relaxation and residual of the level both
// use the rounded couplings, so the level's operator stays one operator:
//   e_new(J) = invD(J) rhs(J) + sum_K c_K e(J+K)
//   r(J)     = rhs(J) - (e(J) - sum_K c_K e(J+K)) / invD(J)
// The rounding (relative 2^-11) changes the preconditioner only; convergence is
// measured with the reference's FP64 operator.
__host__ __device__ constexpr int packed_index(int dx, int dy, int dz) {
    const int k = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
    return k < 13 ? k : k - 1;  // the centre (13) is not stored
}

constexpr int kPackedStride = 32;  // halves per node

struct Packed {
    int n, Pc;
    int64_t cs;  // compact nodes per colour = n * n * Pc
    __host__ __device__ __forceinline__ int64_t at(int i, int y, int z) const { return ((int64_t)z * n + y) * Pc + i; }
};

__host__ __device__ inline Packed packed_of(int n) {
    Packed p;
    p.n = n;
    p.Pc = (n + 1) / 2;
    p.cs = (int64_t)n * n * p.Pc;
    return p;
}

__global__ void __launch_bounds__(256) pack27_kernel(const float* __restrict__ c, int64_t cs, Geom g, Packed pk,
                                                     __half* __restrict__ h0, __half* __restrict__ h1,
                                                     float* __restrict__ i0, float* __restrict__ i1) {
    const int n = g.n;
    int x, y, z;
    if (!plane_node(n, x, y, z)) return;
    const int colour = (x + y + z) & 1;
    const int64_t q = pk.at(x >> 1, y, z);
    const int64_t p = g.at(x, y, z);
    const float inv = 1.0f / c[p];
    (colour ? i1 : i0)[q] = inv;
    __align__(16) __half v[kPackedStride];
#pragma unroll
    for (int k = 26; k < kPackedStride; ++k) v[k] = __float2half_rn(0.0f);
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                if (!(dx || dy || dz)) continue;
                v[packed_index(dx, dy, dz)] = __float2half_rn(-coupling(c, cs, g, p, dx, dy, dz) * inv);
            }
    uint4* dst = reinterpret_cast<uint4*>((colour ? h1 : h0) + q * kPackedStride);
    const uint4* src = reinterpret_cast<const uint4*>(v);
#pragma unroll
    for (int k = 0; k < 4; ++k) dst[k] = src[k];
}

// The 26 couplings of compact node q, as floats.
__device__ __forceinline__ void load_couplings(const __half* __restrict__ h, int64_t q, float* c) {
    const uint4* src = reinterpret_cast<const uint4*>(h + q * kPackedStride);
    __align__(16) __half v[kPackedStride];
    uint4* d = reinterpret_cast<uint4*>(v);
#pragma unroll
    for (int k = 0; k < 4; ++k) d[k] = src[k];
#pragma unroll
    for (int k = 0; k < 26; ++k) c[k] = __half2float(v[k]);
}

// One colour pass on a packed level: nodes of colour COLOUR get
// invD rhs + sum_K c_K e(J+K), neighbours of the other colour read from `next`
// when COLOUR == 1 (updated by pass 0), everything else from `prev` (zero when
// ZERO).
template <int COLOUR, bool ZERO>
__device__ __forceinline__ void relax27p_body(const float* __restrict__ prev, float* next,
                                              const float* __restrict__ rhs, const __half* __restrict__ h,
                                              const float* __restrict__ inv, Geom g, Packed pk, int bx, int by) {
    // threads flattened over the plane's compact (i, y) nodes: full warps on odd rows
    const unsigned t = bx * blockDim.x + threadIdx.x;
    const int n = g.n, z = by;
    if (t >= (unsigned)(pk.Pc * n)) return;
    const int y = (int)(t / (unsigned)pk.Pc), i = (int)(t - (unsigned)y * pk.Pc);
    const int x = 2 * i + ((y + z + COLOUR) & 1);
    if (x >= n) return;
    const int64_t p = g.at(x, y, z), q = pk.at(i, y, z);
    float cf[26];
    load_couplings(h, q, cf);
    float s = 0.0f;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                if (!(dx || dy || dz)) continue;
                const bool other = ((dx + dy + dz) & 1) != 0;
                if (ZERO && !(COLOUR == 1 && other)) continue;
                const int64_t o = p + offset_of(g, dx, dy, dz);
                const float v = (COLOUR == 1 && other) ? next[o] : prev[o];
                s += cf[packed_index(dx, dy, dz)] * v;
            }
    next[p] = inv[q] * rhs[p] + s;
}

template <int COLOUR, bool ZERO>
__global__ void __launch_bounds__(256) relax27p_kernel(const float* __restrict__ prev, float* next,
                                                       const float* __restrict__ rhs, const __half* __restrict__ h,
                                                       const float* __restrict__ inv, Geom g, Packed pk) {
    relax27p_body<COLOUR, ZERO>(prev, next, rhs, h, inv, g, pk, blockIdx.x, blockIdx.y);
}

// The same colour pass with the neighbour planes staged in shared memory.  A
// block owns 32 compact columns (64 x) by 8 rows of the colour's nodes and
// marches `tz` planes; each plane of `prev` (and, for the colour-1 pass, the
// colour-0 values of `next`) over the tile and its one-node halo is loaded
// once, coalesced, into a ring of four planes, so a node reads its 26
// neighbours from shared memory instead of 26 gathers.  Out-of-grid halo
// entries read zero, as the ghosts do.  Same values, same summation order:
// results are bit-identical to relax27p_kernel.
constexpr int kTPi = 32, kTPy = 8, kTPRing = 4;
constexpr int kTPW = 2 * kTPi + 4, kTPH = kTPy + 2;  // staged x from 2 i0 - 2, y from y0 - 1

template <int COLOUR, bool ZERO>
__global__ void __launch_bounds__(kTPi* kTPy) relax27p_tiled_kernel(const float* __restrict__ prev, float* next,
                                                                    const float* __restrict__ rhs,
                                                                    const __half* __restrict__ h,
                                                                    const float* __restrict__ inv, Geom g, Packed pk,
                                                                    int tz) {
    constexpr bool kPrev = !ZERO, kNext = COLOUR == 1;
    __shared__ float sp[kPrev ? kTPRing : 1][kTPH][kTPW];
    __shared__ float sn[kNext ? kTPRing : 1][kTPH][kTPW];
    const int n = g.n;
    const int i0 = blockIdx.x * kTPi, y0 = blockIdx.y * kTPy;
    const int z0 = blockIdx.z * tz, z1 = min(n, z0 + tz);
    const int tid = threadIdx.x, ti = tid % kTPi, ty = tid / kTPi;
    const int xs0 = 2 * i0 - 2, ys0 = y0 - 1;
    auto stage = [&](int z) {  // plane z (>= -1) into ring slot (z + 1) % kTPRing
        const int slot = (z + 1) % kTPRing;
        for (int k = tid; k < kTPH * kTPW; k += kTPi * kTPy) {
            const int ry = k / kTPW, rx = k - ry * kTPW;
            const int x = xs0 + rx, y = ys0 + ry;
            const bool ok = x >= -1 && x <= n && y >= -1 && y <= n && z <= n;
            const int64_t o = ok ? g.at(x, y, z) : 0;
            if (kPrev) sp[kPrev ? slot : 0][ry][rx] = ok ? prev[o] : 0.0f;
            if (kNext) sn[kNext ? slot : 0][ry][rx] = ok && ((x + y + z) & 1) != COLOUR ? next[o] : 0.0f;
        }
    };
    if (kPrev || kNext) {
        stage(z0 - 1);
        stage(z0);
    }
    const int i = i0 + ti, y = y0 + ty;
    for (int z = z0; z < z1; ++z) {
        if (kPrev || kNext) {
            if (z + 1 <= n) stage(z + 1);  // into the slot of plane z - 3, last read before the previous barrier
            __syncthreads();
        }
        if (i >= pk.Pc || y >= n) continue;
        const int x = 2 * i + ((y + z + COLOUR) & 1);
        if (x >= n) continue;
        const int64_t p = g.at(x, y, z), q = pk.at(i, y, z);
        float cf[26];
        load_couplings(h, q, cf);
        float s = 0.0f;
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!(dx || dy || dz)) continue;
                    const bool other = ((dx + dy + dz) & 1) != 0;
                    if (ZERO && !(COLOUR == 1 && other)) continue;
                    const int sl = (z + dz + 1) % kTPRing, ry = ty + 1 + dy, rx = x + dx - xs0;
                    const float v = (COLOUR == 1 && other) ? sn[kNext ? sl : 0][ry][rx] : sp[kPrev ? sl : 0][ry][rx];
                    s += cf[packed_index(dx, dy, dz)] * v;
                }
        next[p] = inv[q] * rhs[p] + s;
    }
}

// res = s (rhs - A e) on a packed level, one thread per node.
__device__ __forceinline__ void residual27p_body(const float* __restrict__ e, const float* __restrict__ rhs,
                                                 const __half* __restrict__ h0, const __half* __restrict__ h1,
                                                 const float* __restrict__ i0, const float* __restrict__ i1,
                                                 const float* __restrict__ fac, Geom g, Packed pk,
                                                 float* __restrict__ res, int bx, int by) {
    const unsigned t = bx * blockDim.x + threadIdx.x;  // flattened over the plane's (x, y)
    const int n = g.n, z = by;
    if (t >= (unsigned)(n * n)) return;
    const int y = (int)(t / (unsigned)n), x = (int)(t - (unsigned)y * n);
    const int colour = (x + y + z) & 1;
    const __half* __restrict__ h = colour ? h1 : h0;
    const int64_t p = g.at(x, y, z), q = pk.at(x >> 1, y, z);
    float cf[26];
    load_couplings(h, q, cf);
    float s = 0.0f;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                if (!(dx || dy || dz)) continue;
                s += cf[packed_index(dx, dy, dz)] * e[p + offset_of(g, dx, dy, dz)];
            }
    const float inv = colour ? i1[q] : i0[q];
    res[p] = fac[p] * (rhs[p] - (e[p] - s) / inv);
}

__global__ void __launch_bounds__(256) residual27p_kernel(const float* __restrict__ e, const float* __restrict__ rhs,
                                                          const __half* __restrict__ h0,
                                                          const __half* __restrict__ h1,
                                                          const float* __restrict__ i0, const float* __restrict__ i1,
                                                          const float* __restrict__ fac, Geom g, Packed pk,
                                                          float* __restrict__ res) {
    residual27p_body(e, rhs, h0, h1, i0, i1, fac, g, pk, res, blockIdx.x, blockIdx.y);
}

// The packed residual with e's planes staged in shared memory: a block owns a
// 64 x 4 tile of nodes (both colours) and marches `tz` planes with a ring of
// four planes of e over the tile and its halo; same values and order as
// residual27p_kernel, so bit-identical results.
constexpr int kTRx = 64, kTRy = 4;
constexpr int kTRW = kTRx + 4, kTRH = kTRy + 2;  // staged x from x0 - 2, y from y0 - 1

__global__ void __launch_bounds__(kTRx* kTRy) residual27p_tiled_kernel(
    const float* __restrict__ e, const float* __restrict__ rhs, const __half* __restrict__ h0,
    const __half* __restrict__ h1, const float* __restrict__ i0, const float* __restrict__ i1,
    const float* __restrict__ fac, Geom g, Packed pk, float* __restrict__ res, int tz) {
    __shared__ float se[kTPRing][kTRH][kTRW];
    const int n = g.n;
    const int x0 = blockIdx.x * kTRx, y0 = blockIdx.y * kTRy;
    const int z0 = blockIdx.z * tz, z1 = min(n, z0 + tz);
    const int tid = threadIdx.x, tx = tid % kTRx, ty = tid / kTRx;
    const int xs0 = x0 - 2, ys0 = y0 - 1;
    auto stage = [&](int z) {
        const int slot = (z + 1) % kTPRing;
        for (int k = tid; k < kTRH * kTRW; k += kTRx * kTRy) {
            const int ry = k / kTRW, rx = k - ry * kTRW;
            const int x = xs0 + rx, y = ys0 + ry;
            const bool ok = x >= -1 && x <= n && y >= -1 && y <= n && z <= n;
            se[slot][ry][rx] = ok ? e[g.at(x, y, z)] : 0.0f;
        }
    };
    stage(z0 - 1);
    stage(z0);
    const int x = x0 + tx, y = y0 + ty;
    for (int z = z0; z < z1; ++z) {
        if (z + 1 <= n) stage(z + 1);
        __syncthreads();
        if (x >= n || y >= n) continue;
        const int colour = (x + y + z) & 1;
        const __half* __restrict__ h = colour ? h1 : h0;
        const int64_t p = g.at(x, y, z), q = pk.at(x >> 1, y, z);
        float cf[26];
        load_couplings(h, q, cf);
        float s = 0.0f;
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!(dx || dy || dz)) continue;
                    s += cf[packed_index(dx, dy, dz)] * se[(z + dz + 1) % kTPRing][ty + 1 + dy][tx + 2 + dx];
                }
        const float inv = colour ? i1[q] : i0[q];
        res[p] = fac[p] * (rhs[p] - (se[(z + 1) % kTPRing][ty + 1][tx + 2] - s) / inv);
    }
}

// ---- exact solve on the 3^3 level -----------------------------------------------
// The 27 x 27 operator of the coarsest level inverted once per set-up by one
// warp: FP64 Gauss-Jordan without pivoting (the Galerkin operator is
// symmetric positive definite), lane i owning row i; stored FP64 row-major and
// applied in FP64 (the coarsest-level solve stays in double precision).
constexpr int kInvN = 27;

__global__ void __launch_bounds__(32) coarse_inverse_kernel(const float* __restrict__ c, int64_t cs, Geom g,
                                                            double* __restrict__ inv) {
    __shared__ double a[kInvN][kInvN + 1];
    const int lane = threadIdx.x;
    if (lane < kInvN) {
        const int x = lane % 3, y = (lane / 3) % 3, z = lane / 9;
        const int64_t p = g.at(x, y, z);
        for (int j = 0; j < kInvN; ++j) a[lane][j] = 0.0;
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx)
                    if (inside(x + dx, y + dy, z + dz, 3))
                        a[lane][lane + dx + 3 * dy + 9 * dz] = (double)coupling(c, cs, g, p, dx, dy, dz);
    }
    __syncwarp();
    for (int k = 0; k < kInvN; ++k) {
        const double inv_piv = 1.0 / a[k][k];
        __syncwarp();
        if (lane < kInvN) a[k][lane] = lane == k ? inv_piv : a[k][lane] * inv_piv;  // row k / pivot, in parallel
        __syncwarp();
        if (lane < kInvN && lane != k) {
            const double f = a[lane][k];
            a[lane][k] = 0.0;
            for (int j = 0; j < kInvN; ++j) a[lane][j] -= f * a[k][j];
        }
        __syncwarp();
    }
    if (lane < kInvN)
        for (int j = 0; j < kInvN; ++j) inv[lane * kInvN + j] = a[lane][j];
}

// ---- levels of side <= 9 in one block, from shared memory -------------------------
// The first level of side <= 9 and those below it (9, 5, 3) run in one block.
// Their operators do not change during a solve, so set-up writes them once
// into a compact image (pb_coarse27_image_f32): per level above the last, the
// 27 couplings of every node (offsets (dz, dy, dx) in lexicographic order, zero
// outside the grid), 1/diagonal and the prolongation weights, node-major; then
// the 3^3 inverse (FP64).  Each cycle copies the image into shared memory and keeps e,
// rhs and the residual of every level there in padded cubes ((n+2)^3 floats,
// zero ghosts), so global memory sees only the first level's rhs and its
// correction.
constexpr int kC27N = 9;
constexpr int kC27Threads = 1024;
constexpr int kC27MaxLevels = 3;  // 9, 5, 3
static_assert(kC27N * kC27N * kC27N <= kC27Threads, "one node per thread on the largest level");

__host__ __device__ inline int round4(int v) { return (v + 3) & ~3; }
__host__ __device__ inline int cube_size(int n) { return (n + 2) * (n + 2) * (n + 2); }

// Float offsets of the image sections and of the shared work cubes (after the image).
struct CoarseLayout {
    int count;
    int n[kC27MaxLevels];
    int coef[kC27MaxLevels], invD[kC27MaxLevels], fac[kC27MaxLevels], inverse;
    int image;  // floats of the image (a multiple of 4)
    int e[kC27MaxLevels], rhs[kC27MaxLevels], res[kC27MaxLevels];
    int total;  // floats of shared memory
};

__host__ __device__ inline CoarseLayout coarse_layout(int count, const int* sizes) {
    CoarseLayout c{};
    c.count = count;
    int off = 0;
    for (int l = 0; l < count; ++l) {
        const int n = sizes[l], N = n * n * n;
        c.n[l] = n;
        if (l == count - 1) break;  // the last level keeps its inverse only
        c.coef[l] = off;
        off += round4(27 * N);
        c.invD[l] = off;
        off += round4(N);
        c.fac[l] = off;
        off += round4(N);
    }
    c.inverse = off;  // 16-byte aligned: doubles
    off += round4(2 * kInvN * kInvN);
    c.image = off;
    for (int l = 0; l < count; ++l) {
        const int m = round4(cube_size(sizes[l]));
        c.e[l] = off;
        c.rhs[l] = off + m;
        c.res[l] = off + 2 * m;
        off += 3 * m;
    }
    c.total = off;
    return c;
}

__device__ __forceinline__ int cube_at(int x, int y, int z, int n) { return ((z + 1) * (n + 2) + (y + 1)) * (n + 2) + (x + 1); }

__device__ __forceinline__ void unflatten(int i, int n, int& x, int& y, int& z) {
    x = i % n;
    y = (i / n) % n;
    z = i / (n * n);
}

// sum over the 27 (or 26) offsets of a_K e[J+K], in the couplings' order.
__device__ __forceinline__ float stencil_cube(const float* a, const float* e, int c, int n, bool skip_centre) {
    const int sy = n + 2, sz = (n + 2) * (n + 2);
    float s = 0.0f;
    int k = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx, ++k) {
                if (skip_centre && !(dx || dy || dz)) continue;
                s += a[k] * e[c + dx + dy * sy + dz * sz];
            }
    return s;
}

// One node's couplings, 1/diagonal and weight into the image (set-up).
__global__ void coarse_image_kernel(const float* __restrict__ c, int64_t cs, Geom g, const float* __restrict__ invD,
                                    const float* __restrict__ fac, float* __restrict__ coef_out,
                                    float* __restrict__ invD_out, float* __restrict__ fac_out) {
    const int n = g.n, N = n * n * n;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int x, y, z;
    unflatten(i, n, x, y, z);
    const int64_t p = g.at(x, y, z);
    int k = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx, ++k)
                coef_out[27 * i + k] = inside(x + dx, y + dy, z + dz, n) ? coupling(c, cs, g, p, dx, dy, dz) : 0.0f;
    invD_out[i] = invD[p];
    fac_out[i] = fac[p];
}

// Red-black ordered sweeps in place on a cube: each colour's new values are
// computed from the current iterate and written after a barrier, so
// same-colour neighbours are read from the previous iterate, as the
// multi-block colour passes do.
__device__ void cube_relax(const float* cf, const float* invD, const float* rhs, float* e, int n, int iters) {
    const int N = n * n * n, i = threadIdx.x;
    int x = 0, y = 0, z = 0;
    if (i < N) unflatten(i, n, x, y, z);
    const int c = cube_at(x, y, z, n);
    for (int it = 0; it < iters; ++it)
        for (int colour = 0; colour < 2; ++colour) {
            const bool mine = i < N && ((x + y + z) & 1) == colour;
            float v = 0.0f;
            if (mine) v = (rhs[c] - stencil_cube(cf + 27 * i, e, c, n, true)) * invD[i];
            __syncthreads();
            if (mine) e[c] = v;
            __syncthreads();
        }
}

__device__ __forceinline__ void coarse27_body(const float4* __restrict__ image, const CoarseLayout& lay,
                                              const float* __restrict__ rhs0, float* __restrict__ e0, Geom g0,
                                              int pre, int post, int inner) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    const int tid = threadIdx.x;
    for (int i = tid; i < lay.image / 4; i += kC27Threads) smem4[i] = image[i];
    for (int i = lay.image + tid; i < lay.total; i += kC27Threads) sm[i] = 0.0f;
    __syncthreads();
    {
        const int n = lay.n[0];
        if (tid < n * n * n) {
            int x, y, z;
            unflatten(tid, n, x, y, z);
            sm[lay.rhs[0] + cube_at(x, y, z, n)] = rhs0[g0.at(x, y, z)];
        }
    }
    __syncthreads();
    const int count = lay.count;
    for (int l = 0; l < count; ++l) {
        const int n = lay.n[l];
        float* e = sm + lay.e[l];
        const float* rhs = sm + lay.rhs[l];
        if (l == count - 1) {  // side 3: e = A^-1 rhs
            if (tid < kInvN) {
                const double* inv = reinterpret_cast<const double*>(sm + lay.inverse);
                double v = 0.0;
                for (int j = 0; j < kInvN; ++j)
                    v += inv[tid * kInvN + j] * (double)rhs[cube_at(j % 3, (j / 3) % 3, j / 9, 3)];
                e[cube_at(tid % 3, (tid / 3) % 3, tid / 9, 3)] = (float)v;
            }
            __syncthreads();
            break;
        }
        const float* cf = sm + lay.coef[l];
        cube_relax(cf, sm + lay.invD[l], rhs, e, n, l == 0 ? pre : inner);  // e starts at zero
        float* res = sm + lay.res[l];
        if (tid < n * n * n) {
            int x, y, z;
            unflatten(tid, n, x, y, z);
            const int c = cube_at(x, y, z, n);
            res[c] = sm[lay.fac[l] + tid] * (rhs[c] - stencil_cube(cf + 27 * tid, e, c, n, false));
        }
        __syncthreads();
        const int cn = lay.n[l + 1], sy = n + 2, sz = (n + 2) * (n + 2);
        if (tid < cn * cn * cn) {
            int x, y, z;
            unflatten(tid, cn, x, y, z);
            const int c = cube_at(2 * x, 2 * y, 2 * z, n);
            float s = 0.0f;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx)
                        s += res[c + dx + dy * sy + dz * sz] * (float)((dx ? 1 : 2) * (dy ? 1 : 2) * (dz ? 1 : 2));
            sm[lay.rhs[l + 1] + cube_at(x, y, z, cn)] = s * (1.0f / 64.0f);
        }
        __syncthreads();
    }
    for (int l = count - 2; l >= 0; --l) {
        const int n = lay.n[l], cn = lay.n[l + 1];
        float* e = sm + lay.e[l];
        const float* ec = sm + lay.e[l + 1];
        if (tid < n * n * n) {
            int x, y, z;
            unflatten(tid, n, x, y, z);
            // trilinear: the mean of the 8 corners, a corner repeated on even axes
            const int x0 = x >> 1, y0 = y >> 1, z0 = z >> 1;
            const int x1 = x0 + (x & 1), y1 = y0 + (y & 1), z1 = z0 + (z & 1);
            const float v = 0.125f * (ec[cube_at(x0, y0, z0, cn)] + ec[cube_at(x1, y0, z0, cn)] +
                                      ec[cube_at(x0, y1, z0, cn)] + ec[cube_at(x1, y1, z0, cn)] +
                                      ec[cube_at(x0, y0, z1, cn)] + ec[cube_at(x1, y0, z1, cn)] +
                                      ec[cube_at(x0, y1, z1, cn)] + ec[cube_at(x1, y1, z1, cn)]);
            e[cube_at(x, y, z, n)] += sm[lay.fac[l] + tid] * v;
        }
        __syncthreads();
        cube_relax(sm + lay.coef[l], sm + lay.invD[l], sm + lay.rhs[l], e, n, l == 0 ? post : inner);
    }
    const int n = lay.n[0];
    if (tid < n * n * n) {
        int x, y, z;
        unflatten(tid, n, x, y, z);
        e0[g0.at(x, y, z)] = sm[lay.e[0] + cube_at(x, y, z, n)];
    }
}

__global__ void __launch_bounds__(kC27Threads) coarse27_kernel(const float4* __restrict__ image, CoarseLayout lay,
                                                               const float* __restrict__ rhs0,
                                                               float* __restrict__ e0, Geom g0, int pre, int post,
                                                               int inner) {
    coarse27_body(image, lay, rhs0, e0, g0, pre, post, inner);
}

// ---- grouped launches (batch.cuh) ----------------------------------------------------

// relax27p: ptr[0] e_prev (null: from zero), ptr[1] e_next, ptr[2] rhs, ptr[3] h0, ptr[4] h1, ptr[5] inv0,
// ptr[6] inv1.  Colour COLOUR of every grid.
template <int COLOUR, bool ZERO>
__global__ void __launch_bounds__(256) relax27p_grouped_kernel(const batch::GridDesc* __restrict__ descs, int count,
                                                               const int* __restrict__ flags) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    const int n = (int)d.n;
    relax27p_body<COLOUR, ZERO>((const float*)d.ptr[0], (float*)d.ptr[1], (const float*)d.ptr[2],
                                (const __half*)d.ptr[3 + COLOUR], (const float*)d.ptr[5 + COLOUR], geom(n),
                                packed_of(n), bx, by);
}

// residual27p: ptr[0] e, ptr[1] rhs, ptr[2] h0, ptr[3] h1, ptr[4] inv0, ptr[5] inv1, ptr[6] weights, ptr[7] res.
__global__ void __launch_bounds__(256) residual27p_grouped_kernel(const batch::GridDesc* __restrict__ descs,
                                                                  int count, const int* __restrict__ flags) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    const int n = (int)d.n;
    residual27p_body((const float*)d.ptr[0], (const float*)d.ptr[1], (const __half*)d.ptr[2],
                     (const __half*)d.ptr[3], (const float*)d.ptr[4], (const float*)d.ptr[5], (const float*)d.ptr[6],
                     geom(n), packed_of(n), (float*)d.ptr[7], bx, by);
}

// restrict27: ptr[0] fine residual, ptr[1] coarse rhs; d.n is the fine side.
__global__ void __launch_bounds__(256) restrict27_grouped_kernel(const batch::GridDesc* __restrict__ descs, int count,
                                                                 const int* __restrict__ flags) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    const int n = (int)d.n;
    restrict27_body((const float*)d.ptr[0], geom(n), (float*)d.ptr[1], geom((n + 1) / 2), bx, by);
}

// coarse27: one block per cloud; ptr[0] image, ptr[1] rhs, ptr[2] e; d.n the first level's side (9, 5 or 3
// levels below it); aux[0..2] pre, post, inner.  Every grid of one launch has the same side.
__global__ void __launch_bounds__(kC27Threads) coarse27_grouped_kernel(const batch::GridDesc* __restrict__ descs,
                                                                       int count, const int* __restrict__ flags,
                                                                       CoarseLayout lay) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    coarse27_body((const float4*)d.ptr[0], lay, (const float*)d.ptr[1], (float*)d.ptr[2], geom((int)d.n),
                  (int)d.aux[0], (int)d.aux[1], (int)d.aux[2]);
}


}  // namespace pb

using namespace pb;

static bool level_side_ok(int64_t n) { return n >= 3 && n <= 4097 && ((n - 1) & (n - 2)) == 0; }

// Scratch floats of the separable product for a slab of kp coarse planes:
// stage x (cn x fn x nz) and stage y (cn x cn x nz), 27 planes each, nz =
// 2 kp + 1 fine planes.
static int64_t galerkin_slab_floats(int fn, int kp) {
    const int cn = (fn + 1) / 2;
    const int64_t nz = 2 * (int64_t)kp + 1;
    return 27 * ((int64_t)cn * fn + (int64_t)cn * cn) * nz;
}

// Scratch bytes for the whole level in one slab (any size down to one coarse
// plane, galerkin_slab_floats(fn, 1) * 4 bytes, works in more slabs); 0 for
// a 7-point fine level.
extern "C" size_t pb_galerkin_workspace_size(int64_t fine_n, int fine_is_7pt) {
    if (!level_side_ok(fine_n) || fine_is_7pt) return 0;
    return (size_t)galerkin_slab_floats((int)fine_n, (int)((fine_n + 1) / 2)) * sizeof(float) + 256;
}

// Coarse 27-point operator (14 planes, plane stride padded_size(cn)) of the
// level below a fine level of side fine_n with prolongation weights
// fine_weights.  fine_is_7pt: `fine` is the level-0 diagonal D (couplings
// -(n-1)^2, direct sum, no scratch); otherwise `fine` holds 14 planes and the
// separable stages run over slabs of coarse planes that fit the workspace.
extern "C" int pb_galerkin_f32(const float* fine, int64_t fine_n, int fine_is_7pt, const float* fine_weights,
                               float* coarse, void* workspace, size_t workspace_bytes, void* stream) {
    if (!level_side_ok(fine_n) || !fine || !coarse || !fine_weights) return fail(PB_ERR_INVALID, "galerkin: bad args");
    const int fn = (int)fine_n, cn = (fn + 1) / 2;
    const Geom gf = geom(fn), gc = geom(cn);
    cudaStream_t s = (cudaStream_t)stream;
    if (fine_is_7pt) {
        const float h2 = (float)(fn - 1) * (float)(fn - 1);
        galerkin7_kernel<<<plane_grid(cn, 128), 128, 0, s>>>(fine, fine_weights, gf, h2, coarse, padded_size(cn),
                                                                gc);
        PB_CHECK_LAUNCH("galerkin7_kernel");
        return PB_OK;
    }
    const int64_t have = workspace ? (int64_t)(workspace_bytes / sizeof(float)) : 0;
    if (have < galerkin_slab_floats(fn, 1))
        return fail(PB_ERR_WORKSPACE, "galerkin: workspace needs at least %lld bytes",
                    (long long)(galerkin_slab_floats(fn, 1) * (int64_t)sizeof(float)));
    int kp = cn;
    while (kp > 1 && galerkin_slab_floats(fn, kp) > have) kp = (kp + 1) / 2;
    float* bx = static_cast<float*>(workspace);
    for (int k0 = 0; k0 < cn; k0 += kp) {
        const int k1 = min(cn, k0 + kp);
        const int zlo = max(0, 2 * k0 - 1), zhi = min(fn, 2 * k1);
        const int nz = zhi - zlo;
        const int64_t px = (int64_t)cn * fn * nz, py = (int64_t)cn * cn * nz;
        float* by = bx + 27 * px;
        galerkin_x_kernel<<<dim3((cn * fn + 127) / 128, nz), 128, 0, s>>>(fine, padded_size(fn), fine_weights, gf,
                                                                          cn, zlo, bx, px);
        PB_CHECK_LAUNCH("galerkin_x_kernel");
        galerkin_y_kernel<<<dim3((cn * cn + 127) / 128, nz), 128, 0, s>>>(bx, px, fn, cn, by, py);
        PB_CHECK_LAUNCH("galerkin_y_kernel");
        galerkin_z_kernel<<<dim3((cn * cn + 127) / 128, k1 - k0), 128, 0, s>>>(by, py, fn, zlo, k0, coarse,
                                                                              padded_size(cn), gc);
        PB_CHECK_LAUNCH("galerkin_z_kernel");
    }
    return PB_OK;
}

// 14 planes of a 7-point level (diagonal D, off-diagonals -(n-1)^2).
extern "C" int pb_level27_from7_f32(const float* D, int64_t n, float* coef, void* stream) {
    if (!level_side_ok(n) || !D || !coef) return fail(PB_ERR_INVALID, "level27 from 7: bad args");
    level7_to_27_kernel<<<plane_grid((int)n, 128), 128, 0, (cudaStream_t)stream>>>(
        D, geom((int)n), (float)(n - 1) * (float)(n - 1), coef, padded_size((int)n));
    PB_CHECK_LAUNCH("level7_to_27_kernel");
    return PB_OK;
}

// invD = 1 / diagonal and the prolongation weights of a 27-point level.
extern "C" int pb_level27_finish_f32(const float* coef, int64_t n, float* invD, float* weights, void* stream) {
    if (!level_side_ok(n) || !coef || !invD || !weights) return fail(PB_ERR_INVALID, "level27 finish: bad args");
    level27_finish_kernel<<<plane_grid((int)n, 128), 128, 0, (cudaStream_t)stream>>>(
        coef, padded_size((int)n), geom((int)n), invD, weights);
    PB_CHECK_LAUNCH("level27_finish_kernel");
    return PB_OK;
}

// Inverse (27 x 27, FP32 row-major) of a 27-point level of side 3.
extern "C" int pb_coarse_inverse_f64(const float* coef, int64_t n, double* inverse, void* stream) {
    if (n != 3 || !coef || !inverse) return fail(PB_ERR_INVALID, "coarse inverse: side must be 3");
    coarse_inverse_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(coef, padded_size(3), geom(3), inverse);
    PB_CHECK_LAUNCH("coarse_inverse_kernel");
    return PB_OK;
}

static int coarse_sizes(int64_t count, const int64_t* sizes, int* out) {
    if (count < 1 || count > kC27MaxLevels || !sizes) return fail(PB_ERR_INVALID, "coarse27: 1 to 3 levels");
    for (int l = 0; l < count; ++l) {
        if (!level_side_ok(sizes[l]) || sizes[l] > kC27N || (l && sizes[l] != (sizes[l - 1] + 1) / 2))
            return fail(PB_ERR_INVALID, "coarse27: level sides must halve from <= 9 down to 3");
        out[l] = (int)sizes[l];
    }
    if (sizes[count - 1] != 3) return fail(PB_ERR_INVALID, "coarse27: the last level must have side 3");
    return PB_OK;
}

// Bytes of the image of levels `sizes` (finest first, side <= 9 halving to 3).
extern "C" size_t pb_coarse27_image_size(int64_t count, const int64_t* sizes) {
    int sz[kC27MaxLevels];
    if (coarse_sizes(count, sizes, sz) != PB_OK) return 0;
    return (size_t)coarse_layout((int)count, sz).image * sizeof(float);
}

// The image the single-block cycle reads: per level but the last, couplings
// (from its 14 planes), 1/diagonal and prolongation weights; then the 3^3
// inverse (FP64, from pb_coarse_inverse_f64).  image: 16-byte aligned.
extern "C" int pb_coarse27_image_f32(int64_t count, const int64_t* sizes, const float* const* coef,
                                     const float* const* invD, const float* const* weights, const double* inverse,
                                     float* image, size_t image_bytes, void* stream) {
    int sz[kC27MaxLevels];
    PB_TRY(coarse_sizes(count, sizes, sz));
    if (!coef || !invD || !weights || !inverse || !image || (reinterpret_cast<uintptr_t>(image) & 15))
        return fail(PB_ERR_INVALID, "coarse27 image: bad args");
    const CoarseLayout lay = coarse_layout((int)count, sz);
    if (image_bytes < (size_t)lay.image * sizeof(float)) return fail(PB_ERR_WORKSPACE, "coarse27 image: too small");
    cudaStream_t s = (cudaStream_t)stream;
    for (int l = 0; l + 1 < count; ++l) {
        if (!coef[l] || !invD[l] || !weights[l]) return fail(PB_ERR_INVALID, "coarse27 image: null level array");
        const int N = sz[l] * sz[l] * sz[l];
        coarse_image_kernel<<<(N + 255) / 256, 256, 0, s>>>(coef[l], padded_size(sz[l]), geom(sz[l]), invD[l],
                                                            weights[l], image + lay.coef[l], image + lay.invD[l],
                                                            image + lay.fac[l]);
        PB_CHECK_LAUNCH("coarse_image_kernel");
    }
    PB_CHECK_CUDA(cudaMemcpyAsync(image + lay.inverse, inverse, sizeof(double) * kInvN * kInvN,
                                  cudaMemcpyDeviceToDevice, s),
                  "coarse27 image inverse");
    return PB_OK;
}

// Levels of side <= 9 in one block from their image: V(pre, post) on the
// first, `inner` sweeps each way on the others, the last (side 3) solved with
// its inverse.  rhs: the first level's right-hand side (padded layout); e
// receives its correction (padded layout; ghosts untouched).
extern "C" int pb_coarse27_cycle_f32(int64_t count, const int64_t* sizes, const float* image, const float* rhs,
                                     float* e, int64_t pre, int64_t post, int64_t inner, void* stream) {
    int sz[kC27MaxLevels];
    PB_TRY(coarse_sizes(count, sizes, sz));
    if (!image || !rhs || !e || (reinterpret_cast<uintptr_t>(image) & 15))
        return fail(PB_ERR_INVALID, "coarse27 cycle: bad args");
    if (pre < 0 || post < 0 || inner < 0 || pre > 64 || post > 64 || inner > 64)
        return fail(PB_ERR_INVALID, "coarse27 cycle: sweep counts must be in [0, 64]");
    const CoarseLayout lay = coarse_layout((int)count, sz);
    const size_t smem = (size_t)lay.total * sizeof(float);
    PB_CHECK_CUDA(cudaFuncSetAttribute(coarse27_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                  "coarse27 smem");
    coarse27_kernel<<<1, kC27Threads, smem, (cudaStream_t)stream>>>(reinterpret_cast<const float4*>(image), lay,
                                                                     rhs, e, geom(sz[0]), (int)pre, (int)post,
                                                                     (int)inner);
    PB_CHECK_LAUNCH("coarse27_kernel");
    return PB_OK;
}

// ---- packed levels ----------------------------------------------------------------
// Bytes of one colour's packed couplings (32 FP16 per node) and of its 1/diagonal.
extern "C" int pb_packed27_size(int64_t n, int64_t* coupling_bytes, int64_t* inverse_bytes) {
    if (!level_side_ok(n)) return fail(PB_ERR_INVALID, "packed27 size: bad side");
    const Packed pk = packed_of((int)n);
    if (coupling_bytes) *coupling_bytes = kPackedStride * pk.cs * (int64_t)sizeof(__half);
    if (inverse_bytes) *inverse_bytes = pk.cs * (int64_t)sizeof(float);
    return PB_OK;
}

// Packs a 27-point level (14 planes): per colour c, couplings h_c and 1/diagonal inv_c.
extern "C" int pb_pack27_f32(const float* coef, int64_t n, void* h0, void* h1, float* inv0, float* inv1,
                             void* stream) {
    if (!level_side_ok(n) || !coef || !h0 || !h1 || !inv0 || !inv1) return fail(PB_ERR_INVALID, "pack27: bad args");
    pack27_kernel<<<plane_grid((int)n, 256), 256, 0, (cudaStream_t)stream>>>(
        coef, padded_size((int)n), geom((int)n), packed_of((int)n), (__half*)h0, (__half*)h1, inv0, inv1);
    PB_CHECK_LAUNCH("pack27_kernel");
    return PB_OK;
}

// One red-black ordered sweep e_next <- S(e_prev) on a packed level (e_prev null: from zero).
extern "C" int pb_relax27p_f32(const float* e_prev, float* e_next, const float* rhs, const void* h0, const void* h1,
                               const float* inv0, const float* inv1, int64_t n, void* stream) {
    if (!level_side_ok(n) || !e_next || !rhs || !h0 || !h1 || !inv0 || !inv1 || e_prev == e_next)
        return fail(PB_ERR_INVALID, "relax27p: bad args");
    cudaStream_t s = (cudaStream_t)stream;
    const Geom g = geom((int)n);
    const Packed pk = packed_of((int)n);
    const dim3 block(256);
    const dim3 grid((pk.Pc * (int)n + 255) / 256, (int)n);
    const __half *a = (const __half*)h0, *b = (const __half*)h1;
    if (tuned(PB_TUNE_RELAX27_VARIANT, n, 0) == 1) {  // shared-memory staged neighbours
        const int tiles = ((pk.Pc + kTPi - 1) / kTPi) * (((int)n + kTPy - 1) / kTPy);
        const int64_t want = 2LL * 8 * kSMs;  // about two waves of 8 resident blocks per SM
        int tz = (int)(((int64_t)n * tiles + want - 1) / want);
        tz = tz < 2 ? 2 : (tz > 16 ? 16 : tz);
        const dim3 tg((pk.Pc + kTPi - 1) / kTPi, ((int)n + kTPy - 1) / kTPy, ((int)n + tz - 1) / tz);
        if (e_prev) {
            relax27p_tiled_kernel<0, false><<<tg, kTPi * kTPy, 0, s>>>(e_prev, e_next, rhs, a, inv0, g, pk, tz);
            PB_CHECK_LAUNCH("relax27p_tiled_kernel");
            relax27p_tiled_kernel<1, false><<<tg, kTPi * kTPy, 0, s>>>(e_prev, e_next, rhs, b, inv1, g, pk, tz);
        } else {
            relax27p_kernel<0, true><<<grid, block, 0, s>>>(nullptr, e_next, rhs, a, inv0, g, pk);  // no neighbours
            PB_CHECK_LAUNCH("relax27p_kernel");
            relax27p_tiled_kernel<1, true><<<tg, kTPi * kTPy, 0, s>>>(nullptr, e_next, rhs, b, inv1, g, pk, tz);
        }
        PB_CHECK_LAUNCH("relax27p_tiled_kernel");
        return PB_OK;
    }
    if (e_prev) {
        relax27p_kernel<0, false><<<grid, block, 0, s>>>(e_prev, e_next, rhs, a, inv0, g, pk);
        PB_CHECK_LAUNCH("relax27p_kernel");
        relax27p_kernel<1, false><<<grid, block, 0, s>>>(e_prev, e_next, rhs, b, inv1, g, pk);
    } else {
        relax27p_kernel<0, true><<<grid, block, 0, s>>>(nullptr, e_next, rhs, a, inv0, g, pk);
        PB_CHECK_LAUNCH("relax27p_kernel");
        relax27p_kernel<1, true><<<grid, block, 0, s>>>(nullptr, e_next, rhs, b, inv1, g, pk);
    }
    PB_CHECK_LAUNCH("relax27p_kernel");
    return PB_OK;
}

// res = weights * (rhs - A e) with the packed operator, then coarse_rhs = P^T res / 8.
extern "C" int pb_residual_restrict27p_f32(const float* e, const float* rhs, const void* h0, const void* h1,
                                           const float* inv0, const float* inv1, const float* weights, int64_t n,
                                           float* res, float* coarse_rhs, void* stream) {
    if (!level_side_ok(n) || n < 5 || !e || !rhs || !h0 || !h1 || !inv0 || !inv1 || !weights || !res || !coarse_rhs)
        return fail(PB_ERR_INVALID, "residual_restrict27p: bad args");
    cudaStream_t s = (cudaStream_t)stream;
    const int fn = (int)n, cn = (fn + 1) / 2;
    if (tuned(PB_TUNE_RESIDUAL27_VARIANT, n, 0) == 1) {  // shared-memory staged e planes
        const int tiles = ((fn + kTRx - 1) / kTRx) * ((fn + kTRy - 1) / kTRy);
        const int64_t want = 2LL * 8 * kSMs;
        int tz = (int)(((int64_t)fn * tiles + want - 1) / want);
        tz = tz < 2 ? 2 : (tz > 16 ? 16 : tz);
        const dim3 tg((fn + kTRx - 1) / kTRx, (fn + kTRy - 1) / kTRy, (fn + tz - 1) / tz);
        residual27p_tiled_kernel<<<tg, kTRx * kTRy, 0, s>>>(e, rhs, (const __half*)h0, (const __half*)h1, inv0, inv1,
                                                           weights, geom(fn), packed_of(fn), res, tz);
        PB_CHECK_LAUNCH("residual27p_tiled_kernel");
    } else {
        residual27p_kernel<<<dim3((fn * fn + 255) / 256, fn), 256, 0, s>>>(
            e, rhs, (const __half*)h0, (const __half*)h1, inv0, inv1, weights, geom(fn), packed_of(fn), res);
        PB_CHECK_LAUNCH("residual27p_kernel");
    }
    restrict27_kernel<<<plane_grid(cn, 256), 256, 0, s>>>(res, geom(fn), coarse_rhs, geom(cn));
    PB_CHECK_LAUNCH("restrict27_kernel");
    return PB_OK;
}

// ---- grouped launches (batch.cuh) ----------------------------------------------------

namespace pb {
namespace batch {

int describe_relax27p(GridDesc& d, bool zero) {
    const int n = (int)d.n;
    if (!level_side_ok(n) || (!zero && !d.ptr[0]) || !d.ptr[1] || !d.ptr[2] || !d.ptr[3] || !d.ptr[4] || !d.ptr[5] ||
        !d.ptr[6] || d.ptr[0] == d.ptr[1])
        return fail(PB_ERR_INVALID, "batch relax27p: bad args");
    const Packed pk = packed_of(n);
    d.gx = (pk.Pc * n + 255) / 256;
    d.gy = n;
    d.gz = 1;
    return PB_OK;
}

int launch_relax27p(const GridDesc* descs, int count, int64_t blocks, bool zero, const int* flags, cudaStream_t s) {
    if (zero) {
        relax27p_grouped_kernel<0, true><<<(unsigned)blocks, 256, 0, s>>>(descs, count, flags);
        PB_CHECK_LAUNCH("relax27p_grouped_kernel");
        relax27p_grouped_kernel<1, true><<<(unsigned)blocks, 256, 0, s>>>(descs, count, flags);
    } else {
        relax27p_grouped_kernel<0, false><<<(unsigned)blocks, 256, 0, s>>>(descs, count, flags);
        PB_CHECK_LAUNCH("relax27p_grouped_kernel");
        relax27p_grouped_kernel<1, false><<<(unsigned)blocks, 256, 0, s>>>(descs, count, flags);
    }
    PB_CHECK_LAUNCH("relax27p_grouped_kernel");
    return PB_OK;
}

int describe_residual27p(GridDesc& d) {
    const int n = (int)d.n;
    for (int k = 0; k < 8; ++k)
        if (!d.ptr[k]) return fail(PB_ERR_INVALID, "batch residual27p: bad args");
    if (!level_side_ok(n) || n < 5) return fail(PB_ERR_INVALID, "batch residual27p: bad side");
    d.gx = (n * n + 255) / 256;
    d.gy = n;
    d.gz = 1;
    return PB_OK;
}

int launch_residual27p(const GridDesc* descs, int count, int64_t blocks, const int* flags, cudaStream_t s) {
    residual27p_grouped_kernel<<<(unsigned)blocks, 256, 0, s>>>(descs, count, flags);
    PB_CHECK_LAUNCH("residual27p_grouped_kernel");
    return PB_OK;
}

int describe_restrict27(GridDesc& d) {
    const int n = (int)d.n;
    if (!level_side_ok(n) || n < 5 || !d.ptr[0] || !d.ptr[1]) return fail(PB_ERR_INVALID, "batch restrict27: bad args");
    const int cn = (n + 1) / 2;
    d.gx = (cn * cn + 255) / 256;
    d.gy = cn;
    d.gz = 1;
    return PB_OK;
}

int launch_restrict27(const GridDesc* descs, int count, int64_t blocks, const int* flags, cudaStream_t s) {
    restrict27_grouped_kernel<<<(unsigned)blocks, 256, 0, s>>>(descs, count, flags);
    PB_CHECK_LAUNCH("restrict27_grouped_kernel");
    return PB_OK;
}

int describe_coarse27(GridDesc& d) {
    const int n = (int)d.n;
    if (!level_side_ok(n) || n > kC27N || !d.ptr[0] || !d.ptr[1] || !d.ptr[2] ||
        (reinterpret_cast<uintptr_t>(d.ptr[0]) & 15))
        return fail(PB_ERR_INVALID, "batch coarse27: bad args");
    if (d.aux[0] < 0 || d.aux[1] < 0 || d.aux[2] < 0 || d.aux[0] > 64 || d.aux[1] > 64 || d.aux[2] > 64)
        return fail(PB_ERR_INVALID, "batch coarse27: sweep counts must be in [0, 64]");
    d.gx = d.gy = d.gz = 1;
    return PB_OK;
}

int launch_coarse27(const GridDesc* descs, int count, int64_t blocks, int first_side, const int* flags,
                    cudaStream_t s) {
    int sz[kC27MaxLevels];
    int levels = 0;
    for (int m = first_side; levels < kC27MaxLevels; m = (m + 1) / 2) {
        sz[levels++] = m;
        if (m == 3) break;
    }
    if (sz[levels - 1] != 3) return fail(PB_ERR_INVALID, "batch coarse27: first side must be 9, 5 or 3");
    const CoarseLayout lay = coarse_layout(levels, sz);
    const size_t smem = (size_t)lay.total * sizeof(float);
    PB_CHECK_CUDA(cudaFuncSetAttribute(coarse27_grouped_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                  "batch coarse27 smem");
    coarse27_grouped_kernel<<<(unsigned)blocks, kC27Threads, smem, s>>>(descs, count, flags, lay);
    PB_CHECK_LAUNCH("coarse27_grouped_kernel");
    return PB_OK;
}

}  // namespace batch
}  // namespace pb

// ---- a whole hierarchy's set-up in one call ---------------------------------------
// The sequence Hierarchy32.setup issues level by level, from one host call:
// level 0 from the screen, each coarser level's Galerkin operator from the one
// above, finish, and the packing of every packed level right after the product
// that reads it for the last time; then the 3^3 inverse and the coarse image.
// Same launches in the same order as the separate entry points.
extern "C" int pb_hierarchy_setup_f32(int64_t levels, const int64_t* sides, const void* const* arrays,
                                      int64_t first_coarse, const double* screen, double point_weight,
                                      void* galerkin_ws, size_t galerkin_bytes, double* inverse, float* image,
                                      size_t image_bytes, void* stream) {
    constexpr int A = PB_LEVEL_ARRAYS;
    if (levels < 2 || levels > 13 || !sides || !arrays || !screen || !inverse || !image || first_coarse < 0 ||
        first_coarse >= levels)
        return fail(PB_ERR_INVALID, "hierarchy setup: bad args");
    for (int64_t l = 0; l < levels; ++l) {
        if (!level_side_ok(sides[l]) || (l && sides[l] != (sides[l - 1] + 1) / 2))
            return fail(PB_ERR_INVALID, "hierarchy setup: level sides must halve from a 2^k + 1 side down to 3");
        if (!arrays[l * A + 1] || !arrays[l * A + 2] || (l && !arrays[l * A + 3]))
            return fail(PB_ERR_INVALID, "hierarchy setup: level %lld misses invD, weights or coef", (long long)l);
    }
    if (sides[levels - 1] != 3) return fail(PB_ERR_INVALID, "hierarchy setup: the last level must have side 3");
    auto D = [&](int64_t l) { return (float*)arrays[l * A + 0]; };
    auto invD = [&](int64_t l) { return (float*)arrays[l * A + 1]; };
    auto W = [&](int64_t l) { return (float*)arrays[l * A + 2]; };
    auto coef = [&](int64_t l) { return (float*)arrays[l * A + 3]; };
    auto packed = [&](int64_t l) { return arrays[l * A + 4] != nullptr; };
    const bool seven = coef(0) == nullptr;
    if (!D(0)) return fail(PB_ERR_INVALID, "hierarchy setup: level 0 needs D");
    if (seven && first_coarse == 0)
        return fail(PB_ERR_INVALID, "hierarchy setup: a 7-point level 0 cannot be part of the coarse cycle");
    PB_TRY(pb_level_setup_f32(screen, sides[0], point_weight, D(0), invD(0), W(0), stream));
    if (!seven) {
        PB_TRY(pb_level27_from7_f32(D(0), sides[0], coef(0), stream));
        PB_TRY(pb_level27_finish_f32(coef(0), sides[0], invD(0), W(0), stream));
    }
    for (int64_t l = 1; l < levels; ++l) {
        const bool fine7 = l == 1 && seven;
        PB_TRY(pb_galerkin_f32(fine7 ? D(0) : coef(l - 1), sides[l - 1], fine7 ? 1 : 0, W(l - 1), coef(l),
                               galerkin_ws, galerkin_bytes, stream));
        PB_TRY(pb_level27_finish_f32(coef(l), sides[l], invD(l), W(l), stream));
        if (packed(l - 1))
            PB_TRY(pb_pack27_f32(coef(l - 1), sides[l - 1], (void*)arrays[(l - 1) * A + 4],
                                 (void*)arrays[(l - 1) * A + 5], (float*)arrays[(l - 1) * A + 6],
                                 (float*)arrays[(l - 1) * A + 7], stream));
    }
    PB_TRY(pb_coarse_inverse_f64(coef(levels - 1), 3, inverse, stream));
    const int64_t tail = levels - first_coarse;
    const float* tc[kC27MaxLevels];
    const float* ti[kC27MaxLevels];
    const float* tw[kC27MaxLevels];
    if (tail < 1 || tail > kC27MaxLevels) return fail(PB_ERR_INVALID, "hierarchy setup: 1 to 3 levels of side <= 9");
    for (int64_t k = 0; k < tail; ++k) {
        tc[k] = coef(first_coarse + k);
        ti[k] = invD(first_coarse + k);
        tw[k] = W(first_coarse + k);
    }
    return pb_coarse27_image_f32(tail, sides + first_coarse, tc, ti, tw, inverse, image, image_bytes, stream);
}
