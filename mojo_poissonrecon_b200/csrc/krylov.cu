// FP64 flexible conjugate gradients, FCG(1), around the FP32 V-cycle.
//
// The reference solves A x = b by repeating V-cycles (python/mojo_poissonrecon/
// core.py:274-285).  Used as a preconditioner z = M(r) inside a Krylov loop
// the V-cycle needs fewer applications.  Because M is an FP32 V-cycle (not a
// fixed symmetric operator), the flexible form is used: each direction is
// A-orthogonalised against the previous one only.
//
//   r = b - A x;  repeat:  z = M(r)
//                          p = z - beta p_prev,   beta  = (z, A p_prev) / (p_prev, A p_prev)
//                          x += alpha p,          alpha = (p, r) / (p, A p)
//                          r = b - A x            (the true residual, FP64)
//
// Two passes per iteration.  Pass 1 is one stencil pass over z giving
// (z, Az), (Az, p_prev) = (z, A p_prev) (A is symmetric), (z, r) and
// (p_prev, r); beta, (p, Ap) = (z,Az) - 2 beta (z,A p_prev) + beta^2 (p_prev,A p_prev)
// and alpha follow without forming q = A p.  Pass 2 writes p and x + alpha p
// and recomputes r = b - A x from them (neighbours formed on the fly), so the
// residual never drifts from the iterate and no final residual pass is needed.
// x and p alternate between two buffers by iteration parity (flags[1], on the
// device), so every iteration launches the same kernels on the same pointers
// and can be captured once in a graph.  x, b and the screening are FP64 and
// dense; z and r32 (the FP32 padded copy of r that the next V-cycle reads) are
// padded FP32; the direction p is stored in FP32 (dense): x moves along the
// unrounded z - beta p_prev, the stored copy only orthogonalises the next
// direction, and the residual is recomputed from x in FP64 every iteration,
// so the rounding perturbs alpha and beta by ~1e-7 relative and never the
// measured residual.
#include "batch.cuh"
#include "common.cuh"

namespace pb {
namespace fcg {

// pass 1: 256 (x, y) columns per block; both passes kTZ planes deep unless the
// autotuner chose otherwise (measured: 16 -> 24, pass 1 82 -> 78 us).  Partial
// sums are sized for the shallowest depth a launch may use, kMinTZ.
constexpr int kTZ = 24, kMinTZ = 8, kThreads = 256;

// Pass 2 tile: 32 x 8 nodes per block, kTZ planes deep.
constexpr int kUX = 32, kUY = 8, kUThreads = kUX * kUY;
static_assert(2 * (kUX + kUY) <= kUThreads, "one halo node per thread");

struct Pad {  // padded FP32 layout of the multigrid levels
    int n, P;
    int64_t plane;
    __device__ __forceinline__ int64_t at(int x, int y, int z) const {
        return checked_at(((int64_t)(z + 1) * (n + 2) + (y + 1)) * P + (x + 4), (int64_t)(n + 2) * plane, kSitePad);
    }
};

__device__ __forceinline__ int lin_tid() { return threadIdx.y * blockDim.x + threadIdx.x; }

// Sums K values over the block; results valid in linear thread 0.
template <int K>
__device__ __forceinline__ void block_sums(double (&v)[K], double (*shared)[32]) {
    const int tid = lin_tid(), lane = tid & 31, warp = tid >> 5;
    const int warps = (blockDim.x * blockDim.y) >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) shared[k][warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            v[k] = lane < warps ? shared[k][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        }
    }
}

__device__ __forceinline__ int64_t block_index() {
    return ((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
}

// Pass 1: per-block (z, Az), (Az, p_prev), (z, r32), (p_prev, r32); flags[1]
// (iterations done) selects p_prev = p[it & 1]; flags[0] != 0 on the first step.
// Each thread marches down its column with z of planes k - 1 and k in
// registers; the ghosts of the padded z are zero, so the 6-neighbour sum needs
// no tests.  Compiled for 4 resident blocks per SM (64 registers), which keeps
// more loads in flight than the occupancy-first default.
// TZC > 0: the planes per block as a compile-time constant (the built-in kTZ),
// which lets the compiler unroll the z march; 0: the runtime tz.
template <int TZC>
__device__ __forceinline__ void direction_sums_body(const float* __restrict__ z, Pad g, const float* __restrict__ p0,
                                                    const float* __restrict__ p1, const float* __restrict__ r32,
                                                    const double* __restrict__ screen, double pw,
                                                    const int* __restrict__ flags, double* __restrict__ part, int tz,
                                                    int bx, int by, int64_t block) {
    __shared__ double shared[4][32];
    const int n = g.n;
    const unsigned t = bx * kThreads + threadIdx.x;  // flattened over the plane's (x, y): full warps
    const int y = t < (unsigned)(n * n) ? (int)(t / (unsigned)n) : n, x = (int)(t - (unsigned)y * n);
    const int tzv = TZC > 0 ? TZC : tz;
    const int z0 = by * tzv, z1 = min(n, z0 + tzv);
    const double h = (double)(n - 1), h2 = h * h;
    const bool first = flags[0] != 0;
    const float* __restrict__ pp = (flags[1] & 1) ? p1 : p0;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (x < n && y < n) {
        const int degxy = (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n);
        const int64_t nn = (int64_t)n * n;
        int64_t i = (int64_t)z0 * nn + (int64_t)y * n + x, c = g.at(x, y, z0);
        float zb = z[c - g.plane], zm = z[c];
        for (int k = z0; k < z1; ++k, i += nn, c += g.plane) {
            const float za = z[c + g.plane];  // the ghost plane past the last
            const double s = (double)z[c - 1] + (double)z[c + 1] + (double)z[c - g.P] + (double)z[c + g.P] +
                             (double)zb + (double)za;
            const double zc = (double)zm;
            zb = zm;
            zm = za;
            const int deg = degxy + (k > 0) + (k + 1 < n);
            const double az = ((double)deg * h2 + pw * screen[i] * h2) * zc - s * h2;
            const double rc = (double)r32[c];
            v[0] += zc * az;
            v[2] += zc * rc;
            if (!first) {
                const double pv = (double)pp[i];
                v[1] += az * pv;
                v[3] += pv * rc;
            }
        }
    }
    block_sums<4>(v, shared);
    if (lin_tid() == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) part[4 * block + k] = v[k];
}

// MINB: resident blocks per SM the compiler must allow (register budget); the
// autotuner picks among the compiled variants (PB_TUNE_FCG_DIRECTION_VARIANT).
template <int MINB, int TZC>
__global__ void __launch_bounds__(kThreads, MINB) direction_sums_kernel(const float* __restrict__ z, Pad g,
                                                                     const float* __restrict__ p0,
                                                                     const float* __restrict__ p1,
                                                                     const float* __restrict__ r32,
                                                                     const double* __restrict__ screen, double pw,
                                                                     const int* __restrict__ flags,
                                                                     double* __restrict__ part, int tz) {
    direction_sums_body<TZC>(z, g, p0, p1, r32, screen, pw, flags, part, tz, blockIdx.x, blockIdx.y, block_index());
}

// Sums pass 1's partials (fixed order) and forms the step's scalars:
//   scal[0] (p, Ap) (the previous direction's on entry)   scal[1] beta
//   scal[2] alpha   scal[3] (p, r)
__device__ __forceinline__ void direction_finish_body(const double* __restrict__ part, int blocks,
                                                      const int* __restrict__ flags, double* __restrict__ scal) {
    __shared__ double shared[4][32];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < blocks; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] += part[4 * (int64_t)b + k];
    block_sums<4>(v, shared);
    if (threadIdx.x != 0) return;
    const double zz = v[0], zq = v[1], zr = v[2], pr = v[3];
    const bool first = flags[0] != 0;
    const double pap_prev = scal[0];
    const double beta = first || !(pap_prev > 0.0) ? 0.0 : zq / pap_prev;
    const double pap = first ? zz : zz - 2.0 * beta * zq + beta * beta * pap_prev;
    const double prn = first ? zr : zr - beta * pr;
    scal[0] = pap;
    scal[1] = beta;
    scal[2] = pap > 0.0 ? prn / pap : 0.0;
    scal[3] = prn;
}

__global__ void direction_finish_kernel(const double* __restrict__ part, int blocks, const int* __restrict__ flags,
                                        double* __restrict__ scal) {
    direction_finish_body(part, blocks, flags, scal);
}

// Halo node of thread tid for a tile at (bx, by): rows by - 1 and by + kUY,
// columns bx - 1 and bx + kUX; (sx, sy) its slot in the shared tile.
struct Halo {
    int hx = -1, hy = -1, sx = 0, sy = 0;
    bool has = false;
    __device__ Halo(int tid, int bx, int by) {
        if (tid < 2 * kUX) {
            hx = bx + (tid % kUX);
            hy = tid < kUX ? by - 1 : by + kUY;
            sx = tid % kUX + 1;
            sy = tid < kUX ? 0 : kUY + 1;
            has = true;
        } else if (tid < 2 * kUX + 2 * kUY) {
            const int j = tid - 2 * kUX;
            hy = by + (j % kUY);
            hx = j < kUY ? bx - 1 : bx + kUX;
            sy = j % kUY + 1;
            sx = j < kUY ? 0 : kUX + 1;
            has = true;
        }
    }
    __device__ bool inside(int n) const { return has && hx >= 0 && hx < n && hy >= 0 && hy < n; }
};

// Pass 2: p_new = z - beta p_prev, x_new = x + alpha p_new, r = b - A x_new
// (neighbour values of x_new formed on the fly), r32 = (float) r, per-block
// ||r||^2.  Buffers by parity: p_prev = p[it & 1] -> p_new = p[(it+1) & 1],
// x = x[it & 1] -> x_new = x[(it+1) & 1].
//
// A 32 x 8 tile marches down z: the new iterate of plane k over the tile and
// its one-node halo goes to shared memory once (two tiles by plane parity, so
// one barrier per plane), the column's planes k - 1 and k + 1 stay in
// registers (about 7 global loads per node instead of 23 with every neighbour
// formed from memory).  Nodes outside the domain hold 0 and
// the neighbour sum adds x-, x+, y-, y+, z-, z+ in that order.
template <int TZC>
__device__ __forceinline__ void update_residual_body(const float* __restrict__ z, Pad g, float* p0, float* p1,
                                                     double* x0, double* x1, const double* __restrict__ b,
                                                     const double* __restrict__ screen, double pw,
                                                     const double* __restrict__ scal, const int* __restrict__ flags,
                                                     float* __restrict__ r32, double* __restrict__ part, int tz,
                                                     int tile_x, int tile_y, int tile_z, int64_t block) {
    __shared__ double tiles[2][kUY + 2][kUX + 2];  // by plane parity: one barrier per plane
    __shared__ double shared[1][32];
    const int n = g.n;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kUX + tx;
    const int bx = tile_x * kUX, by = tile_y * kUY;
    const int x = bx + tx, y = by + ty;
    const int tzv = TZC > 0 ? TZC : tz;
    const int z0 = tile_z * tzv, z1 = min(n, z0 + tzv);
    const double h = (double)(n - 1), h2 = h * h;
    const int odd = flags[1] & 1;
    const bool first = flags[0] != 0;
    const float* __restrict__ pp = odd ? p1 : p0;
    float* __restrict__ pn = odd ? p0 : p1;
    const double* __restrict__ xc = odd ? x1 : x0;
    double* __restrict__ xn = odd ? x0 : x1;
    const double beta = first ? 0.0 : scal[1], alpha = scal[2];
    const int64_t nn = (int64_t)n * n;
    auto dir_at = [&](int64_t ii, int64_t cc) -> double {
        double val = (double)z[cc];
        if (!first) val -= beta * (double)pp[ii];
        return val;
    };
    const Halo hl(tid, bx, by);
    const bool halo_in = hl.inside(n);
    int64_t hi = 0, hc = 0;
    if (halo_in) {
        hi = (int64_t)z0 * nn + (int64_t)hl.hy * n + hl.hx;
        hc = g.at(hl.hx, hl.hy, z0);
    }
    const bool inside = x < n && y < n;
    int64_t i = 0, c = 0;
    double dm = 0.0, xm = 0.0, xb = 0.0;
    if (inside) {
        i = (int64_t)z0 * nn + (int64_t)y * n + x;
        c = g.at(x, y, z0);
        dm = dir_at(i, c);
        xm = xc[i] + alpha * dm;
        xb = z0 > 0 ? xc[i - nn] + alpha * dir_at(i - nn, c - g.plane) : 0.0;
    }
    const int degxy = (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n);
    double v[1] = {0.0};
    for (int k = z0; k < z1; ++k) {
        const double hv = halo_in ? xc[hi] + alpha * dir_at(hi, hc) : 0.0;
        const bool up = k + 1 < n;
        double da = 0.0, xa = 0.0, bi = 0.0, sc = 0.0;
        if (inside) {
            if (up) {
                da = dir_at(i + nn, c + g.plane);
                xa = xc[i + nn] + alpha * da;
            }
            bi = b[i];
            sc = screen[i];
        }
        // plane k - 2's reads of this tile ended before plane k - 1's barrier
        double(*tile)[kUX + 2] = tiles[k & 1];
        tile[ty + 1][tx + 1] = inside ? xm : 0.0;
        if (hl.has) tile[hl.sy][hl.sx] = hv;
        __syncthreads();
        if (inside) {
            double s = 0.0;
            s += tile[ty + 1][tx];
            s += tile[ty + 1][tx + 2];
            s += tile[ty][tx + 1];
            s += tile[ty + 2][tx + 1];
            s += xb;
            s += xa;
            const int deg = degxy + (k > 0) + up;
            PB_GUARD(i, nn * n, kSiteFcgStore) {
                pn[i] = (float)dm;
                xn[i] = xm;
            }
            const double r = bi - (((double)deg * h2 + pw * sc * h2) * xm - s * h2);
            PB_GUARD(c, (int64_t)(n + 2) * g.plane, kSiteFcgStore)
            r32[c] = (float)r;
            v[0] += r * r;
            i += nn;
            c += g.plane;
        }
        xb = xm;
        xm = xa;
        dm = da;
        hi += nn;
        hc += g.plane;
    }
    block_sums<1>(v, shared);
    if (lin_tid() == 0) part[block] = v[0];
}

// ---- pass 2 with the next planes prefetched by cp.async -------------------------
// The same arithmetic as update_residual_body, in the same order.  Each
// thread copies the values it will read of plane k + RING - 1 (its x, z, p, b
// and screen, and its halo node's x, z, p) into its own shared-memory slots
// with cp.async while it works on plane k, so RING - 1 planes of loads are in
// flight per thread without holding registers; a thread only reads its own
// slots, so cp.async.wait_group suffices (the tile of new iterates keeps its
// barrier).  RING = 3 by default, 4 as a tuning variant.
constexpr int kRing = 3;

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int TZC, int RING = kRing>
__device__ __forceinline__ void update_residual_prefetch_body(
    const float* __restrict__ z, Pad g, float* p0, float* p1, double* x0, double* x1, const double* __restrict__ b,
    const double* __restrict__ screen, double pw, const double* __restrict__ scal, const int* __restrict__ flags,
    float* __restrict__ r32, double* __restrict__ part, int tz, int tile_x, int tile_y, int tile_z, int64_t block) {
    static_assert(RING >= 3 && RING <= 4, "two or three planes in flight");
    __shared__ double tiles[2][kUY + 2][kUX + 2];
    __shared__ double shared[1][32];
    constexpr int kHalo = 2 * (kUX + kUY);     // the threads tid < kHalo own a halo node
    __shared__ double rd[RING][3][kUThreads];  // own x, b, screen
    __shared__ double hd[RING][kHalo];         // halo x
    __shared__ float rf[RING][2][kUThreads];   // own z, p
    __shared__ float hf[RING][2][kHalo];       // halo z, p
    const int n = g.n;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kUX + tx;
    const int bx = tile_x * kUX, by = tile_y * kUY;
    const int x = bx + tx, y = by + ty;
    const int tzv = TZC > 0 ? TZC : tz;
    const int z0 = tile_z * tzv, z1 = min(n, z0 + tzv);
    const double h = (double)(n - 1), h2 = h * h;
    const int odd = flags[1] & 1;
    const bool first = flags[0] != 0;
    const float* __restrict__ pp = odd ? p1 : p0;
    float* __restrict__ pn = odd ? p0 : p1;
    const double* __restrict__ xc = odd ? x1 : x0;
    double* __restrict__ xn = odd ? x0 : x1;
    const double beta = first ? 0.0 : scal[1], alpha = scal[2];
    const int64_t nn = (int64_t)n * n;
    auto dir_at = [&](int64_t ii, int64_t cc) -> double {
        double val = (double)z[cc];
        if (!first) val -= beta * (double)pp[ii];
        return val;
    };
    auto dir_of = [&](float zv, float pv) -> double {  // dir_at from prefetched values
        double val = (double)zv;
        if (!first) val -= beta * (double)pv;
        return val;
    };
    const Halo hl(tid, bx, by);
    const bool halo_in = hl.inside(n);
    const bool inside = x < n && y < n;
    const int64_t i0 = inside ? (int64_t)z0 * nn + (int64_t)y * n + x : 0;
    const int64_t c0 = inside ? g.at(x, y, z0) : 0;
    const int64_t hi0 = halo_in ? (int64_t)z0 * nn + (int64_t)hl.hy * n + hl.hx : 0;
    const int64_t hc0 = halo_in ? g.at(hl.hx, hl.hy, z0) : 0;
    auto issue = [&](int p) {  // plane p's values into slot p % RING, one commit group
        const int sl = p % RING;
        const int64_t dz = p - z0;
        if (inside && p < n && p <= z1) {  // own x, z, p of planes z0 .. z1 (z1: the last plane's upper neighbour)
            const int64_t ip = i0 + dz * nn, cq = c0 + dz * g.plane;
            cp_async8(&rd[sl][0][tid], xc + ip);
            cp_async4(&rf[sl][0][tid], z + cq);
            if (!first) cp_async4(&rf[sl][1][tid], pp + ip);
            if (p < z1) {
                cp_async8(&rd[sl][1][tid], b + ip);
                cp_async8(&rd[sl][2][tid], screen + ip);
            }
        }
        if (halo_in && p < z1) {
            const int64_t hp = hi0 + dz * nn, hq = hc0 + dz * g.plane;
            cp_async8(&hd[sl][tid], xc + hp);
            cp_async4(&hf[sl][0][tid], z + hq);
            if (!first) cp_async4(&hf[sl][1][tid], pp + hp);
        }
        cp_commit();
    };
    issue(z0);
    issue(z0 + 1);
    if (RING == 4) issue(z0 + 2);
    cp_wait<RING - 2>();
    double dm = 0.0, xm = 0.0, xb = 0.0;
    if (inside) {
        const int sl = z0 % RING;
        dm = dir_of(rf[sl][0][tid], rf[sl][1][tid]);
        xm = rd[sl][0][tid] + alpha * dm;
        xb = z0 > 0 ? xc[i0 - nn] + alpha * dir_at(i0 - nn, c0 - g.plane) : 0.0;
    }
    int64_t i = i0, c = c0;
    const int degxy = (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n);
    double v[1] = {0.0};
    for (int k = z0; k < z1; ++k) {
        issue(k + RING - 1);  // into the slot of plane k - 1, read by this thread alone in the previous step
        cp_wait<RING - 2>();  // planes up to k + 1 have landed
        const int sk = k % RING, sn = (k + 1) % RING;
        const double hv = halo_in ? hd[sk][tid] + alpha * dir_of(hf[sk][0][tid], hf[sk][1][tid]) : 0.0;
        const bool up = k + 1 < n;
        double da = 0.0, xa = 0.0, bi = 0.0, sc = 0.0;
        if (inside) {
            if (up) {
                da = dir_of(rf[sn][0][tid], rf[sn][1][tid]);
                xa = rd[sn][0][tid] + alpha * da;
            }
            bi = rd[sk][1][tid];
            sc = rd[sk][2][tid];
        }
        double(*tile)[kUX + 2] = tiles[k & 1];
        tile[ty + 1][tx + 1] = inside ? xm : 0.0;
        if (hl.has) tile[hl.sy][hl.sx] = hv;
        __syncthreads();
        if (inside) {
            double s = 0.0;
            s += tile[ty + 1][tx];
            s += tile[ty + 1][tx + 2];
            s += tile[ty][tx + 1];
            s += tile[ty + 2][tx + 1];
            s += xb;
            s += xa;
            const int deg = degxy + (k > 0) + up;
            PB_GUARD(i, nn * n, kSiteFcgStore) {
                pn[i] = (float)dm;
                xn[i] = xm;
            }
            const double r = bi - (((double)deg * h2 + pw * sc * h2) * xm - s * h2);
            PB_GUARD(c, (int64_t)(n + 2) * g.plane, kSiteFcgStore)
            r32[c] = (float)r;
            v[0] += r * r;
            i += nn;
            c += g.plane;
        }
        xb = xm;
        xm = xa;
        dm = da;
    }
    cp_wait<0>();
    block_sums<1>(v, shared);
    if (lin_tid() == 0) part[block] = v[0];
}

template <int TZC, int RING = kRing>
__global__ void __launch_bounds__(kUThreads) update_residual_prefetch_kernel(
    const float* __restrict__ z, Pad g, float* p0, float* p1, double* x0, double* x1, const double* __restrict__ b,
    const double* __restrict__ screen, double pw, const double* __restrict__ scal, const int* __restrict__ flags,
    float* __restrict__ r32, double* __restrict__ part, int tz) {
    update_residual_prefetch_body<TZC, RING>(z, g, p0, p1, x0, x1, b, screen, pw, scal, flags, r32, part, tz,
                                             blockIdx.x, blockIdx.y, blockIdx.z, block_index());
}

// MINB as above (PB_TUNE_FCG_UPDATE_VARIANT; the default 5 matches a 48-register budget).
template <int MINB, int TZC>
__global__ void __launch_bounds__(kUThreads, MINB) update_residual_kernel(
    const float* __restrict__ z, Pad g, float* p0, float* p1, double* x0, double* x1, const double* __restrict__ b,
    const double* __restrict__ screen, double pw, const double* __restrict__ scal, const int* __restrict__ flags,
    float* __restrict__ r32, double* __restrict__ part, int tz) {
    update_residual_body<TZC>(z, g, p0, p1, x0, x1, b, screen, pw, scal, flags, r32, part, tz, blockIdx.x, blockIdx.y,
                         blockIdx.z, block_index());
}

// out[0] = sum over blocks of part[b] (fixed order).
__device__ __forceinline__ void sum_body(const double* __restrict__ part, int blocks, double* __restrict__ out) {
    __shared__ double shared[1][32];
    double v[1] = {0.0};
    for (int b = threadIdx.x; b < blocks; b += blockDim.x) v[0] += part[b];
    block_sums<1>(v, shared);
    if (threadIdx.x == 0) out[0] = v[0];
}

__global__ void sum_kernel(const double* __restrict__ part, int blocks, double* __restrict__ out) {
    sum_body(part, blocks, out);
}

// End of one iteration: record ||r||^2, count it, clear the first-step flag
// and, inside a graph, set the WHILE condition: continue while
// ||r||^2 > target2 and fewer than min(max_iter, ctrl[1]) iterations have run.
//   flags[0] first-step flag, flags[1] iterations; ctrl[0] = target2, ctrl[1] = cap.
__global__ void loop_kernel(cudaGraphConditionalHandle handle, int use_handle, const double* __restrict__ scal,
                            const double* __restrict__ ctrl, int* __restrict__ flags, int max_iter,
                            double* __restrict__ history) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int it = flags[1] + 1;
    flags[1] = it;
    flags[0] = 0;
    const double r2 = scal[4];
    if (history && it <= max_iter) history[it - 1] = r2;
    const bool more = r2 > ctrl[0] && it < max_iter && (double)it < ctrl[1];
    if (use_handle) cudaGraphSetConditional(handle, more ? 1u : 0u);
}

static int direction_planes(int n) {
    const int64_t tz = tuned(PB_TUNE_FCG_DIRECTION_PLANES, n, kTZ);
    return tz < kMinTZ ? kMinTZ : (int)tz;
}
static int update_planes(int n) {
    const int64_t tz = tuned(PB_TUNE_FCG_UPDATE_PLANES, n, kTZ);
    return tz < kMinTZ ? kMinTZ : (int)tz;
}
static dim3 flat_grid_of(int n, int tz) { return dim3((n * n + kThreads - 1) / kThreads, (n + tz - 1) / tz); }
static dim3 tile_grid_of(int n, int tz) {
    return dim3((n + kUX - 1) / kUX, (n + kUY - 1) / kUY, (n + tz - 1) / tz);
}
static unsigned count(dim3 g) { return g.x * g.y * g.z; }
static unsigned blocks_of(int n) {  // the most either pass can launch (kMinTZ planes per block)
    const unsigned a = count(flat_grid_of(n, kMinTZ)), t = count(tile_grid_of(n, kMinTZ));
    return a > t ? a : t;
}
__host__ __device__ inline Pad pad_of(int n) {
    const int P = ((n + 5) + 7) & ~7;
    return Pad{n, P, (int64_t)(n + 2) * P};
}

// ---- grouped launches over a batch of clouds (batch.cuh) --------------------------
// Per cloud c: flags + 4c (first step, iterations, active), scal + 8c, its own
// partial-sum area.  The point weight travels as the bits of a double in aux[0].

__device__ __forceinline__ double aux_double(int64_t bits) { return __longlong_as_double((long long)bits); }

// ptr[0] z, ptr[1] p0, ptr[2] p1, ptr[3] r32, ptr[4] screen, ptr[5] partials.
__global__ void __launch_bounds__(kThreads, 4) direction_sums_grouped_kernel(const batch::GridDesc* __restrict__ descs,
                                                                             int count, const int* __restrict__ flags) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    direction_sums_body<kTZ>((const float*)d.ptr[0], pad_of((int)d.n), (const float*)d.ptr[1], (const float*)d.ptr[2],
                        (const float*)d.ptr[3], (const double*)d.ptr[4], aux_double(d.aux[0]),
                        flags + d.cloud * batch::kFlagStride, (double*)d.ptr[5], (int)d.aux[1], bx, by,
                        bx + d.gx * (int64_t)by);
}

// One block per cloud: ptr[0] partials, ptr[1] the cloud's scalars; aux[0] pass-1 blocks.
__global__ void direction_finish_grouped_kernel(const batch::GridDesc* __restrict__ descs, int count,
                                                const int* __restrict__ flags) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    direction_finish_body((const double*)d.ptr[0], (int)d.aux[0], flags + d.cloud * batch::kFlagStride,
                          (double*)d.ptr[1]);
}

// ptr[0] z, ptr[1] p0, ptr[2] p1, ptr[3] x0, ptr[4] x1, ptr[5] b, ptr[6] screen, ptr[7] r32, ptr[8] the
// cloud's scalars, ptr[9] partials.
__global__ void __launch_bounds__(kUThreads, 4) update_residual_grouped_kernel(const batch::GridDesc* __restrict__ descs,
                                                                            int count, const int* __restrict__ flags) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    update_residual_prefetch_body<kTZ>((const float*)d.ptr[0], pad_of((int)d.n), (float*)d.ptr[1], (float*)d.ptr[2],
                         (double*)d.ptr[3], (double*)d.ptr[4], (const double*)d.ptr[5], (const double*)d.ptr[6],
                         aux_double(d.aux[0]), (const double*)d.ptr[8], flags + d.cloud * batch::kFlagStride,
                         (float*)d.ptr[7], (double*)d.ptr[9], (int)d.aux[1], bx, by, bz,
                         bx + d.gx * ((int64_t)by + d.gy * bz));
}

// One block per cloud: ptr[0] partials, ptr[1] output (the cloud's scal + 4); aux[0] blocks.
__global__ void sum_grouped_kernel(const batch::GridDesc* __restrict__ descs, int count,
                                   const int* __restrict__ flags) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    sum_body((const double*)d.ptr[0], (int)d.aux[0], (double*)d.ptr[1]);
}

// End of one batch iteration, every active cloud: record ||r||^2, count the
// iteration, clear the first-step flag, and keep the cloud active while
// ||r||^2 > target2 and fewer than min(max_iter, cap) iterations have run.  The
// WHILE condition (inside a graph) continues while any cloud is active.
__global__ void __launch_bounds__(1024) loop_batch_kernel(cudaGraphConditionalHandle handle, int use_handle,
                                                          const double* __restrict__ scal,
                                                          const double* __restrict__ ctrl, int* __restrict__ flags,
                                                          int clouds, int max_iter, double* __restrict__ history) {
    int any = 0;
    for (int c = threadIdx.x; c < clouds; c += blockDim.x) {
        int* f = flags + (int64_t)c * batch::kFlagStride;
        if (!f[batch::kFlagActive]) continue;
        const int it = f[batch::kFlagIter] + 1;
        f[batch::kFlagIter] = it;
        f[batch::kFlagFirst] = 0;
        const double r2 = scal[(int64_t)c * batch::kScalStride + 4];
        if (history && it <= max_iter) history[(int64_t)c * max_iter + it - 1] = r2;
        const double* ct = ctrl + (int64_t)c * batch::kCtrlStride;
        const bool more = r2 > ct[0] && it < max_iter && (double)it < ct[1];
        f[batch::kFlagActive] = more ? 1 : 0;
        any |= more ? 1 : 0;
    }
    any = __syncthreads_or(any);
    if (use_handle && threadIdx.x == 0) cudaGraphSetConditional(handle, any ? 1u : 0u);
}

}  // namespace fcg

namespace batch {

int describe_fcg_direction(GridDesc& d) {
    const int n = (int)d.n;
    for (int k = 0; k < 6; ++k)
        if (!d.ptr[k]) return fail(PB_ERR_INVALID, "batch fcg direction: bad args");
    if (n < 2 || n > 4097 || d.ptr[1] == d.ptr[2]) return fail(PB_ERR_INVALID, "batch fcg direction: bad args");
    const int tz = fcg::kTZ;  // grouped launches keep the built-in planes per block
    const dim3 g = fcg::flat_grid_of(n, tz);
    d.gx = g.x;
    d.gy = g.y;
    d.gz = 1;
    d.aux[1] = tz;
    return PB_OK;
}

int describe_fcg_update(GridDesc& d) {
    const int n = (int)d.n;
    for (int k = 0; k < 10; ++k)
        if (!d.ptr[k]) return fail(PB_ERR_INVALID, "batch fcg update: bad args");
    if (n < 2 || n > 4097 || d.ptr[1] == d.ptr[2] || d.ptr[3] == d.ptr[4])
        return fail(PB_ERR_INVALID, "batch fcg update: bad args");
    const int tz = fcg::kTZ;
    const dim3 g = fcg::tile_grid_of(n, tz);
    d.gx = g.x;
    d.gy = g.y;
    d.gz = g.z;
    d.aux[1] = tz;
    return PB_OK;
}

int describe_fcg_reduce(GridDesc& d) {
    if (!d.ptr[0] || !d.ptr[1] || d.aux[0] < 1) return fail(PB_ERR_INVALID, "batch fcg reduce: bad args");
    d.gx = d.gy = d.gz = 1;
    return PB_OK;
}

// Partial-sum doubles one cloud of side n needs (both FCG passes).
int64_t fcg_partials(int n) { return (int64_t)fcg::blocks_of(n) * 4; }
int64_t fcg_direction_blocks(int n) { return fcg::count(fcg::flat_grid_of(n, fcg::kTZ)); }
int64_t fcg_update_blocks(int n) { return fcg::count(fcg::tile_grid_of(n, fcg::kTZ)); }

int launch_fcg(int kind, const GridDesc* descs, int count, int64_t blocks, const int* flags, cudaStream_t s) {
    switch (kind) {
        case 0:
            fcg::direction_sums_grouped_kernel<<<(unsigned)blocks, fcg::kThreads, 0, s>>>(descs, count, flags);
            PB_CHECK_LAUNCH("direction_sums_grouped_kernel");
            return PB_OK;
        case 1:
            fcg::direction_finish_grouped_kernel<<<(unsigned)blocks, 1024, 0, s>>>(descs, count, flags);
            PB_CHECK_LAUNCH("direction_finish_grouped_kernel");
            return PB_OK;
        case 2:
            fcg::update_residual_grouped_kernel<<<(unsigned)blocks, dim3(fcg::kUX, fcg::kUY), 0, s>>>(descs, count,
                                                                                                      flags);
            PB_CHECK_LAUNCH("update_residual_grouped_kernel");
            return PB_OK;
        case 3:
            fcg::sum_grouped_kernel<<<(unsigned)blocks, 1024, 0, s>>>(descs, count, flags);
            PB_CHECK_LAUNCH("sum_grouped_kernel");
            return PB_OK;
    }
    return fail(PB_ERR_INVALID, "batch fcg: unknown kind %d", kind);
}

int launch_loop_batch(unsigned long long handle, const double* scal, const double* ctrl, int* flags, int clouds,
                      int max_iter, double* history, cudaStream_t s) {
    fcg::loop_batch_kernel<<<1, 1024, 0, s>>>((cudaGraphConditionalHandle)handle, handle != 0, scal, ctrl, flags,
                                              clouds, max_iter, history);
    PB_CHECK_LAUNCH("loop_batch_kernel");
    return PB_OK;
}

}  // namespace batch
}  // namespace pb

using namespace pb;

extern "C" size_t pb_fcg_workspace_size(int64_t n) {
    if (n < 2) n = 2;
    return (size_t)fcg::blocks_of((int)n) * 4 * sizeof(double) + 256;
}

static int fcg_check(int64_t n, size_t workspace_bytes, const void* workspace) {
    if (!workspace || workspace_bytes < (size_t)pb::fcg::blocks_of((int)n) * 4 * sizeof(double))
        return fail(PB_ERR_WORKSPACE, "fcg: workspace needs %zu bytes", pb_fcg_workspace_size(n));
    return PB_OK;
}

// FCG(1) pass 1 after the preconditioner produced z (padded FP32): the step's
// scalars into scal[0..3] (scal[0] holds the previous (p, Ap) on entry).
// p0/p1: the two dense FP32 direction buffers, p_prev = p[flags[1] & 1];
// r32: the padded FP32 residual the preconditioner read.
extern "C" int pb_fcg_direction_f64(const float* z, const float* p0, const float* p1, const float* r32,
                                    const double* screen, int64_t n, double point_weight, double* scal,
                                    const int* flags, void* workspace, size_t workspace_bytes, void* stream) {
    using namespace pb::fcg;
    if (n < 2 || n > 4097 || !z || !p0 || !p1 || p0 == p1 || !r32 || !screen || !scal || !flags)
        return fail(PB_ERR_INVALID, "fcg direction: bad args");
    PB_TRY(fcg_check(n, workspace_bytes, workspace));
    double* part = (double*)workspace;
    cudaStream_t s = (cudaStream_t)stream;
    const int tz = direction_planes((int)n);
    const dim3 grid = flat_grid_of((int)n, tz);
    const bool fixed = tz == kTZ;
    auto dir = fixed ? direction_sums_kernel<4, kTZ> : direction_sums_kernel<4, 0>;
    switch (tuned(PB_TUNE_FCG_DIRECTION_VARIANT, n, 0)) {
        case 1: dir = fixed ? direction_sums_kernel<6, kTZ> : direction_sums_kernel<6, 0>; break;
        case 2: dir = fixed ? direction_sums_kernel<8, kTZ> : direction_sums_kernel<8, 0>; break;
        default: break;
    }
    dir<<<grid, kThreads, 0, s>>>(z, pad_of((int)n), p0, p1, r32, screen, point_weight, flags, part, tz);
    PB_CHECK_LAUNCH("fcg direction_sums_kernel");
    direction_finish_kernel<<<1, 1024, 0, s>>>(part, (int)count(grid), flags, scal);
    PB_CHECK_LAUNCH("fcg direction_finish_kernel");
    return PB_OK;
}

// FCG(1) pass 2: p_new, x_new = x + alpha p_new and the true residual
// r = b - A x_new into r32, scal[4] = ||r||^2.  Iterate and direction buffers
// alternate by parity of flags[1]: x[it & 1] -> x[(it+1) & 1].
extern "C" int pb_fcg_update_f64(const float* z, float* p0, float* p1, double* x0, double* x1, const double* b,
                                 const double* screen, float* r32, int64_t n, double point_weight, double* scal,
                                 const int* flags, void* workspace, size_t workspace_bytes, void* stream) {
    using namespace pb::fcg;
    if (n < 2 || n > 4097 || !z || !p0 || !p1 || p0 == p1 || !x0 || !x1 || x0 == x1 || !b || !screen || !r32 ||
        !scal || !flags)
        return fail(PB_ERR_INVALID, "fcg update: bad args");
    PB_TRY(fcg_check(n, workspace_bytes, workspace));
    double* part = (double*)workspace;
    cudaStream_t s = (cudaStream_t)stream;
    const int tz = update_planes((int)n);
    const dim3 grid = tile_grid_of((int)n, tz);
    const bool fixed = tz == kTZ;
    auto upd = fixed ? update_residual_kernel<5, kTZ> : update_residual_kernel<5, 0>;
    switch (tuned(PB_TUNE_FCG_UPDATE_VARIANT, n, 0)) {
        case 1: upd = fixed ? update_residual_kernel<6, kTZ> : update_residual_kernel<6, 0>; break;
        case 2: upd = fixed ? update_residual_kernel<8, kTZ> : update_residual_kernel<8, 0>; break;
        case 3: upd = fixed ? update_residual_prefetch_kernel<kTZ> : update_residual_prefetch_kernel<0>; break;
        case 4: upd = fixed ? update_residual_prefetch_kernel<kTZ, 4> : update_residual_prefetch_kernel<0, 4>; break;
        default: break;
    }
    upd<<<grid, dim3(kUX, kUY), 0, s>>>(z, pad_of((int)n), p0, p1, x0, x1, b, screen, point_weight, scal, flags,
                                        r32, part, tz);
    PB_CHECK_LAUNCH("fcg update_residual_kernel");
    sum_kernel<<<1, 1024, 0, s>>>(part, (int)count(grid), scal + 4);
    PB_CHECK_LAUNCH("fcg sum_kernel");
    return PB_OK;
}

// ---- device-driven iteration: a CUDA graph with a WHILE conditional node ------
// pb_loop_capture_begin creates a graph holding one WHILE node and starts
// capturing `stream` into its body; the caller then queues one iteration (its
// last launch being pb_loop_condition with the returned handle) and calls
// pb_loop_capture_end, which instantiates the graph.  Each pb_graph_launch then
// runs iterations on the device until the condition kernel says stop — no
// host synchronisation per iteration.  The condition starts at 1 on every launch.
extern "C" int pb_loop_capture_begin(void* stream, void** graph_out, unsigned long long* handle_out) {
    if (!graph_out || !handle_out) return fail(PB_ERR_INVALID, "loop capture: null output");
    cudaGraph_t graph = nullptr;
    PB_CHECK_CUDA(cudaGraphCreate(&graph, 0), "cudaGraphCreate");
    cudaGraphConditionalHandle handle;
    cudaError_t e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_fail(e, "cudaGraphConditionalHandleCreate");
    }
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, graph, nullptr, 0, &params);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_fail(e, "cudaGraphAddNode (while)");
    }
    cudaGraph_t body = params.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph((cudaStream_t)stream, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_fail(e, "cudaStreamBeginCaptureToGraph");
    }
    *graph_out = graph;
    *handle_out = (unsigned long long)handle;
    return PB_OK;
}

// Queues the end-of-iteration kernel (see loop_kernel).  handle = 0: eager use
// outside a graph (no condition is set).
extern "C" int pb_loop_condition(unsigned long long handle, const double* scal, const double* ctrl, int* flags,
                                 int64_t max_iter, double* history, void* stream) {
    if (!scal || !ctrl || !flags || max_iter < 1) return fail(PB_ERR_INVALID, "loop condition: bad args");
    pb::fcg::loop_kernel<<<1, 32, 0, (cudaStream_t)stream>>>((cudaGraphConditionalHandle)handle, handle != 0, scal,
                                                            ctrl, flags, (int)max_iter, history);
    PB_CHECK_LAUNCH("loop_kernel");
    return PB_OK;
}

extern "C" int pb_loop_capture_end(void* stream, void* graph, void** exec_out) {
    if (!graph || !exec_out) return fail(PB_ERR_INVALID, "loop capture end: bad args");
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture((cudaStream_t)stream, &captured);
    if (e != cudaSuccess) {
        cudaGraphDestroy((cudaGraph_t)graph);
        return cuda_fail(e, "cudaStreamEndCapture");
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, (cudaGraph_t)graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy((cudaGraph_t)graph);
        return cuda_fail(e, "cudaGraphInstantiate");
    }
    *exec_out = exec;
    return PB_OK;
}

extern "C" int pb_graph_launch(void* exec, void* stream) {
    if (!exec) return fail(PB_ERR_INVALID, "graph launch: null graph");
    PB_CHECK_CUDA(cudaGraphLaunch((cudaGraphExec_t)exec, (cudaStream_t)stream), "cudaGraphLaunch");
    return PB_OK;
}

extern "C" int pb_graph_destroy(void* exec, void* graph) {
    if (exec) cudaGraphExecDestroy((cudaGraphExec_t)exec);
    if (graph) cudaGraphDestroy((cudaGraph_t)graph);
    return PB_OK;
}

// Adds launches that ran inside graphs (known to the host only afterwards) to
// the library's launch count.
extern "C" int pb_note_launches(long long count);
