// TMA-staged fused red-black sweep on the padded FP32 layout (sm_100a).
//
// Same update as capi.mojo:310-410 for one iteration (colour 0 then colour 1)
// in FP32, out of place.  A block owns an (x, y) tile of up to 65 x 17 nodes
// and a z range.  One thread issues cp.async.bulk.tensor loads of whole plane
// boxes (72 x 21 floats: the tile plus a halo of 2, x origin aligned to 16
// bytes) of e_in, rhs and 1/D into a ring of kSlots slots, each guarded by an
// mbarrier, kSlots-1 planes ahead of the plane being updated; all threads then
// compute out of shared memory.  Out-of-grid nodes read as zero (ghost layer
// or TMA zero fill) and 1/D is zero there, so colour-0 values at halo nodes
// outside the grid come out zero without branches.
//
// Waits are bounded: a barrier that does not complete within ~1 s of SM clock
// sets *status = 1 and the block stops issuing work, after draining its own
// outstanding copies (also bounded).
#include <cuda.h>

#include "common.cuh"

namespace pb {

namespace tma {

constexpr int kTX = 64;                 // interior tile width (last x tile: 65)
constexpr int kTY = 16;                 // interior tile height (last y tile: 17)
constexpr int kBoxX = 72;               // kTX + 1 + halo 2 + 2, rounded to 16 B; x origin = x0 - 4
constexpr int kBoxY = kTY + 1 + 4;      // 21
constexpr int kRedX = 68;               // colour-0 ring row stride (>= kTX + 1 + 2)
constexpr int kRedY = kTY + 1 + 2;      // 19
constexpr int kSlots = 5;
constexpr int kThreads = 256;
constexpr int kBoxFloats = kBoxX * kBoxY;  // 1512 floats = 6048 bytes land per box
constexpr int kPlane = 1536;               // slot stride: 6144 bytes keeps every box 128-byte aligned
constexpr long long kWaitCycles = 2000000000ll;

struct Smem {
    float slot[kSlots][3][kPlane];      // [slot][e, rhs, invD][row * kBoxX + col]
    float red[3][kRedY][kRedX];
    unsigned long long bar[kSlots];
};

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(unsigned long long* b) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(b)) : "memory");
}

__device__ __forceinline__ void bar_expect(unsigned long long* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool bar_test(unsigned long long* b, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ bool bar_wait(unsigned long long* b, uint32_t parity) {
    const long long start = clock64();
    while (!bar_test(b, parity))
        if (clock64() - start > kWaitCycles) return false;
    return true;
}

__device__ __forceinline__ void load_box(float* dst, const CUtensorMap* map, int x, int y, int z,
                                         unsigned long long* b) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(saddr(b))
        : "memory");
}

struct Params {
    int n, P;
    int64_t plane;
    int ntx, nty, z_chunk;
    float h2;
    float* e_out;
    int* status;
};

template <bool ZERO_IN>
__global__ void __launch_bounds__(kThreads, 2)
    sweep_kernel(const __grid_constant__ CUtensorMap map_e, const __grid_constant__ CUtensorMap map_rhs,
                 const __grid_constant__ CUtensorMap map_invD, Params p) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // TMA destinations must be 128-byte aligned: align the carve-out base.
    const uint32_t raw = saddr(smem_raw);
    Smem& S = *reinterpret_cast<Smem*>(smem_raw + (((raw + 127u) & ~127u) - raw));
    const int n = p.n;
    const int bx = blockIdx.x, by = blockIdx.y;
    const int x0 = bx * kTX, y0 = by * kTY;
    const int W = (bx == p.ntx - 1 ? n : x0 + kTX) - x0;
    const int H = (by == p.nty - 1 ? n : y0 + kTY) - y0;
    const int zb = blockIdx.z * p.z_chunk;
    const int ze = min(n, zb + p.z_chunk);
    const int zfirst = zb - 2, zlast = ze + 1;  // planes read by this block
    const int tid = threadIdx.x;
    const uint32_t bytes = (ZERO_IN ? 2u : 3u) * kBoxFloats * 4u;

    if (tid == 0) {
        for (int s = 0; s < kSlots; ++s) bar_init(&S.bar[s]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    auto issue = [&](int z) {  // thread 0 only
        const int k = z - zfirst, s = k % kSlots;
        bar_expect(&S.bar[s], bytes);
        // box origin in storage coordinates: x = x0 - 4 + 4, y = (y0 - 2) + 1, z = z + 1
        if (!ZERO_IN) load_box(S.slot[s][0], &map_e, x0, y0 - 1, z + 1, &S.bar[s]);
        load_box(S.slot[s][1], &map_rhs, x0, y0 - 1, z + 1, &S.bar[s]);
        load_box(S.slot[s][2], &map_invD, x0, y0 - 1, z + 1, &S.bar[s]);
    };
    auto slot_of = [&](int z) { return (z - zfirst) % kSlots; };
    auto parity_of = [&](int z) { return (uint32_t)(((z - zfirst) / kSlots) & 1); };

    int issued = zfirst;  // next plane to issue
    if (tid == 0)
        for (; issued <= zlast && issued < zfirst + kSlots; ++issued) issue(issued);

    // Planes zfirst and zfirst + 1 must be resident before the first colour-0
    // step.  Every give-up decision is made block-wide (__syncthreads_and) so
    // that no thread leaves the loop while others wait at a barrier.
    bool ok = bar_wait(&S.bar[slot_of(zfirst)], parity_of(zfirst));
    ok = bar_wait(&S.bar[slot_of(zfirst + 1)], parity_of(zfirst + 1)) && ok;
    ok = __syncthreads_and(ok);

    for (int t = zb - 1; t <= ze && ok; ++t) {
        const bool arrived = bar_wait(&S.bar[slot_of(t + 1)], parity_of(t + 1));
        // colour 0 on plane t over the tile plus a halo of 1 (all reads stay
        // inside the ring, so a late plane only gives unused values)
        {
            const float* em = S.slot[slot_of(t - 1)][0];
            const float* ec = S.slot[slot_of(t)][0];
            const float* ep = S.slot[slot_of(t + 1)][0];
            const float* rhs = S.slot[slot_of(t)][1];
            const float* inv = S.slot[slot_of(t)][2];
            float(*red)[kRedX] = S.red[(t + 3) % 3];
            const int rows = H + 2, pairs = (W + 3) / 2;
            for (int i = tid; i < rows * 34; i += kThreads) {
                const int ly = i / 34, k = i - ly * 34;
                if (k >= pairs) continue;
                const int y = y0 - 1 + ly;
                const int lx = 2 * k + ((1 + y + t) & 1);  // x = x0 - 1 + lx has x + y + t even
                if (lx >= W + 2) continue;
                const int c = (ly + 1) * kBoxX + lx + 3;
                float v = 0.0f;
                if (!ZERO_IN) {
                    const float s = ec[c - 1] + ec[c + 1] + ec[c - kBoxX] + ec[c + kBoxX] + em[c] + ep[c];
                    v = (rhs[c] + s * p.h2) * inv[c];
                } else {
                    v = rhs[c] * inv[c];
                }
                red[ly][lx] = v;
            }
        }
        ok = __syncthreads_and(arrived);
        if (!ok) break;
        // colour 1 on plane t - 1 over the tile, and its output rows
        if (t - 1 >= zb) {
            const int z = t - 1;
            const float* rhs = S.slot[slot_of(z)][1];
            const float* inv = S.slot[slot_of(z)][2];
            const float(*rm)[kRedX] = S.red[(z + 2) % 3];
            const float(*rc)[kRedX] = S.red[(z + 3) % 3];
            const float(*rp)[kRedX] = S.red[(z + 4) % 3];
            const int pairs = (W + 1) / 2;
            for (int i = tid; i < H * 33; i += kThreads) {
                const int ly = i / 33, k = i - ly * 33;
                if (k >= pairs) continue;
                const int y = y0 + ly;
                const int lx = 2 * k;
                float out[2];
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int x = x0 + lx + j;
                    const int ry = ly + 1, rx = lx + j + 1;
                    if (((x + y + z) & 1) == 0) {
                        out[j] = rc[ry][rx];
                    } else {
                        const float s = rc[ry][rx - 1] + rc[ry][rx + 1] + rc[ry - 1][rx] + rc[ry + 1][rx] +
                                        rm[ry][rx] + rp[ry][rx];
                        const int c = (ly + 2) * kBoxX + lx + j + 4;
                        out[j] = (rhs[c] + s * p.h2) * inv[c];
                    }
                }
                float* dst = p.e_out + ((int64_t)(z + 1) * (n + 2) + (y + 1)) * p.P + (x0 + lx + 4);
                if (lx + 1 < W) {
                    *reinterpret_cast<float2*>(dst) = make_float2(out[0], out[1]);
                } else {
                    dst[0] = out[0];
                }
            }
        }
        __syncthreads();  // slot of plane t - 1 and colour-0 plane t - 2 are free now
        if (tid == 0 && issued <= zlast) issue(issued++);
    }
    if (!ok) {
        if (tid == 0) {
            atomicExch(p.status, 1);
            // drain: the copies still in flight (at most the last kSlots issued)
            // must land before the block exits; each wait is bounded too
            for (int z = max(zfirst, issued - kSlots); z < issued; ++z)
                (void)bar_wait(&S.bar[slot_of(z)], parity_of(z));
        }
        __syncthreads();
    }
}

// ---- version 2: in-place colour-0 updates on float4 column groups -------------
// The state ring holds e for planes t-2 .. t+3.  Colour 0 of plane t is
// updated in place (float4 groups of 4 columns, 18 groups per 72-column box
// row); colour 1 of plane t-1 is computed into registers and written out with
// the colour-0 values of the same group as one float4 store.  A colour-0
// update reads only colour-1 nodes and vice versa, so in-place stores never
// change a value another thread of the same phase reads.  For a group at box
// row br on plane t (colour 0) or t-1 (colour 1), the updated columns are
// j = s and s + 2 with s = (br + t) & 1, because x0 and y0 are even.
constexpr int kGroups = kBoxX / 4;  // 18

// Geometry of one v2 configuration: tile height TY (the last y tile holds
// TY + 1 rows), SLOTS planes in the ring (SLOTS - 4 planes of prefetch).
template <int TY, int SLOTS>
struct Geo2 {
    static constexpr int kBoxRows = TY + 1 + 4;
    static constexpr int kBox = kBoxX * kBoxRows;
    static constexpr int kStride = (kBox + 31) / 32 * 32;  // 128-byte aligned slot arrays
    struct Smem {
        float slot[SLOTS][3][kStride];
        unsigned long long bar[SLOTS];
    };
};

__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }

template <bool ZERO_IN, int TY, int SLOTS>
__global__ void __launch_bounds__(kThreads, 2)
    sweep_v2_kernel(const __grid_constant__ CUtensorMap map_e, const __grid_constant__ CUtensorMap map_rhs,
                    const __grid_constant__ CUtensorMap map_invD, Params p) {
    using G = Geo2<TY, SLOTS>;
    constexpr int kSlots2 = SLOTS;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = saddr(smem_raw);
    typename G::Smem& S = *reinterpret_cast<typename G::Smem*>(smem_raw + (((raw + 127u) & ~127u) - raw));
    const int n = p.n;
    const int bx = blockIdx.x, by = blockIdx.y;
    const int x0 = bx * kTX, y0 = by * TY;
    const int W = (bx == p.ntx - 1 ? n : x0 + kTX) - x0;
    const int H = (by == p.nty - 1 ? n : y0 + TY) - y0;
    const int zb = blockIdx.z * p.z_chunk;
    const int ze = min(n, zb + p.z_chunk);
    const int zfirst = zb - 2, zlast = ze + 1;
    const int tid = threadIdx.x;
    const uint32_t bytes = (ZERO_IN ? 2u : 3u) * G::kBox * 4u;
    const float h2 = p.h2;

    if (tid == 0) {
        for (int s = 0; s < kSlots2; ++s) bar_init(&S.bar[s]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    auto slot_of = [&](int z) { return (z - zfirst) % kSlots2; };
    auto parity_of = [&](int z) { return (uint32_t)(((z - zfirst) / kSlots2) & 1); };
    auto issue = [&](int z) {
        const int s = slot_of(z);
        bar_expect(&S.bar[s], bytes);
        if (!ZERO_IN) load_box(S.slot[s][0], &map_e, x0, y0 - 1, z + 1, &S.bar[s]);
        load_box(S.slot[s][1], &map_rhs, x0, y0 - 1, z + 1, &S.bar[s]);
        load_box(S.slot[s][2], &map_invD, x0, y0 - 1, z + 1, &S.bar[s]);
    };
    int issued = zfirst;
    if (tid == 0)
        for (; issued <= zlast && issued < zfirst + kSlots2; ++issued) issue(issued);

    bool ok = bar_wait(&S.bar[slot_of(zfirst)], parity_of(zfirst));
    ok = bar_wait(&S.bar[slot_of(zfirst + 1)], parity_of(zfirst + 1)) && ok;
    ok = __syncthreads_and(ok);

    const int itemsA = (H + 2) * kGroups;
    const int groupsB = (W + 3) / 4;  // groups 1 .. groupsB cover box columns 4 .. W+3
    const int itemsB = H * groupsB;
    for (int t = zb - 1; t <= ze && ok; ++t) {
        const bool arrived = bar_wait(&S.bar[slot_of(t + 1)], parity_of(t + 1));
        {  // colour 0 of plane t on box rows 1 .. H+2, columns 3 .. W+4
            float* e = S.slot[slot_of(t)][0];
            const float* em = S.slot[slot_of(t - 1)][0];
            const float* ep = S.slot[slot_of(t + 1)][0];
            const float* rhs = S.slot[slot_of(t)][1];
            const float* inv = S.slot[slot_of(t)][2];
            for (int i = tid; i < itemsA; i += kThreads) {
                const int br = 1 + i / kGroups, g = i - (br - 1) * kGroups;
                const int base = br * kBoxX + 4 * g;
                const int s = (br + t) & 1;
                const float4 r4 = lds4(rhs + base), i4 = lds4(inv + base);
                float4 c = lds4(e + base);
                float v[4];
                if (ZERO_IN) {
                    v[0] = r4.x * i4.x; v[1] = r4.y * i4.y; v[2] = r4.z * i4.z; v[3] = r4.w * i4.w;
                } else {
                    const float4 u = lds4(e + base - kBoxX), d = lds4(e + base + kBoxX);
                    const float4 zm = lds4(em + base), zp = lds4(ep + base);
                    const float L = g > 0 ? e[base - 1] : 0.0f;
                    const float R = g < kGroups - 1 ? e[base + 4] : 0.0f;
                    v[0] = (r4.x + (L + c.y + u.x + d.x + zm.x + zp.x) * h2) * i4.x;
                    v[1] = (r4.y + (c.x + c.z + u.y + d.y + zm.y + zp.y) * h2) * i4.y;
                    v[2] = (r4.z + (c.y + c.w + u.z + d.z + zm.z + zp.z) * h2) * i4.z;
                    v[3] = (r4.w + (c.z + R + u.w + d.w + zm.w + zp.w) * h2) * i4.w;
                }
                const int b0 = 4 * g;
                float cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const bool upd = ((j & 1) == s) && (b0 + j >= 3) && (b0 + j < W + 5);
                    cc[j] = upd ? v[j] : cc[j];
                }
                *reinterpret_cast<float4*>(e + base) = make_float4(cc[0], cc[1], cc[2], cc[3]);
            }
        }
        ok = __syncthreads_and(arrived);
        if (!ok) break;
        if (t - 1 >= zb) {  // colour 1 of plane t-1 on the tile, written with colour 0
            const int z = t - 1;
            const float* e = S.slot[slot_of(z)][0];
            const float* em = S.slot[slot_of(z - 1)][0];
            const float* ep = S.slot[slot_of(z + 1)][0];
            const float* rhs = S.slot[slot_of(z)][1];
            const float* inv = S.slot[slot_of(z)][2];
            for (int i = tid; i < itemsB; i += kThreads) {
                const int r = i / groupsB;
                const int g = 1 + (i - r * groupsB);
                const int br = r + 2;
                const int base = br * kBoxX + 4 * g;
                const int s = (br + t) & 1;
                const float4 c = lds4(e + base), u = lds4(e + base - kBoxX), d = lds4(e + base + kBoxX);
                const float4 zm = lds4(em + base), zp = lds4(ep + base);
                const float4 r4 = lds4(rhs + base), i4 = lds4(inv + base);
                const float L = e[base - 1];
                const float R = g < kGroups - 1 ? e[base + 4] : 0.0f;
                float v[4];
                v[0] = (r4.x + (L + c.y + u.x + d.x + zm.x + zp.x) * h2) * i4.x;
                v[1] = (r4.y + (c.x + c.z + u.y + d.y + zm.y + zp.y) * h2) * i4.y;
                v[2] = (r4.z + (c.y + c.w + u.z + d.z + zm.z + zp.z) * h2) * i4.z;
                v[3] = (r4.w + (c.z + R + u.w + d.w + zm.w + zp.w) * h2) * i4.w;
                float o[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) o[j] = ((j & 1) == s) ? v[j] : o[j];
                float* dst = p.e_out + ((int64_t)(z + 1) * (n + 2) + (y0 - 1 + br)) * p.P + (x0 + 4 * g);
                const int valid = W + 4 - 4 * g;  // columns of this group inside the tile
                if (valid >= 4) {
                    *reinterpret_cast<float4*>(dst) = make_float4(o[0], o[1], o[2], o[3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        if (j < valid) dst[j] = o[j];
                }
            }
        }
        __syncthreads();  // plane t-2 is no longer read
        if (tid == 0 && t - 2 >= zfirst && issued <= zlast) issue(issued++);
    }
    if (!ok) {
        if (tid == 0) {
            atomicExch(p.status, 1);
            for (int z = max(zfirst, issued - kSlots2); z < issued; ++z)
                (void)bar_wait(&S.bar[slot_of(z)], parity_of(z));
        }
        __syncthreads();
    }
}

typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiled encoder() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(ptr);
    }
    return fn;
}

// 3D map over a padded level: dims (P, n+2, n+2) floats, box (72, rows, 1).
static int make_map(CUtensorMap* map, const float* base, int n, int P, int rows) {
    EncodeTiled enc = encoder();
    if (!enc) return fail(PB_ERR_CUDA, "sweep: cuTensorMapEncodeTiled is unavailable");
    if (reinterpret_cast<uintptr_t>(base) & 15) return fail(PB_ERR_INVALID, "sweep: arrays must be 16-byte aligned");
    const cuuint64_t dims[3] = {(cuuint64_t)P, (cuuint64_t)(n + 2), (cuuint64_t)(n + 2)};
    const cuuint64_t strides[2] = {(cuuint64_t)P * 4, (cuuint64_t)P * (n + 2) * 4};
    const cuuint32_t box[3] = {kBoxX, (cuuint32_t)rows, 1};
    const cuuint32_t estride[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estride,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(PB_ERR_CUDA, "sweep: cuTensorMapEncodeTiled failed (%d)", (int)r);
    return PB_OK;
}

}  // namespace tma

// ---- prolongation add on the padded layout (capi.mojo:677-742 in FP32) -------
__global__ void prolong_add32_kernel(const float* __restrict__ c, float* __restrict__ f, int n, int P, int cn,
                                     int cP) {
    const int64_t total = (int64_t)n * n * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((int64_t)n * n));
        const int x0 = x >> 1, y0 = y >> 1, z0 = z >> 1;
        const int x1 = min(x0 + 1, cn - 1), y1 = min(y0 + 1, cn - 1), z1 = min(z0 + 1, cn - 1);
        const float tx = (x & 1) ? 0.5f : 0.f, ty = (y & 1) ? 0.5f : 0.f, tz = (z & 1) ? 0.5f : 0.f;
        auto C = [&](int a, int b, int d) { return c[((int64_t)(d + 1) * (cn + 2) + (b + 1)) * cP + (a + 4)]; };
        const float c00 = C(x0, y0, z0) * (1.f - tx) + C(x1, y0, z0) * tx;
        const float c10 = C(x0, y1, z0) * (1.f - tx) + C(x1, y1, z0) * tx;
        const float c01 = C(x0, y0, z1) * (1.f - tx) + C(x1, y0, z1) * tx;
        const float c11 = C(x0, y1, z1) * (1.f - tx) + C(x1, y1, z1) * tx;
        const float v = (c00 * (1.f - ty) + c10 * ty) * (1.f - tz) + (c01 * (1.f - ty) + c11 * ty) * tz;
        f[((int64_t)(z + 1) * (n + 2) + (y + 1)) * P + (x + 4)] += v;
    }
}

}  // namespace pb

using namespace pb;

static int pitch_for(int n) { return ((n + 5) + 7) & ~7; }

// One TMA-staged fused sweep.  n = 2^k + 1 >= 33 (smaller levels use the
// single-block coarse kernel).  mode 0: from e_in; mode 1: from zero.
// z_chunk <= 0 picks one that fills the 148 SMs with two blocks each.
// *status (device int) is set to 1 if a bounded wait gave up.
template <typename K>
static int launch_sweep(K kernel, size_t smem, int ty, int n, int z_chunk, cudaStream_t s, const float* e_in,
                        const float* rhs, const float* invD, pb::tma::Params prm) {
    using namespace pb::tma;
    const int P = prm.P;
    prm.nty = (n - 1) / ty > 0 ? (n - 1) / ty : 1;
    const int tiles = prm.ntx * prm.nty;
    int per_sm = (int)((228 * 1024) / (smem + 1024));
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 2) per_sm = 2 + (per_sm > 2);  // register file: at most 3 blocks of 256 threads
    if (z_chunk <= 0) {
        const int want = per_sm * kSMs;
        int chunks = want / tiles > 1 ? want / tiles : 1;
        z_chunk = (n + chunks - 1) / chunks;
        if (z_chunk < 4) z_chunk = 4;
    }
    prm.z_chunk = z_chunk;
    CUtensorMap me, mr, mi;
    const int rows = ty + 5;
    PB_TRY(make_map(&mr, rhs, n, P, rows));
    PB_TRY(make_map(&mi, invD, n, P, rows));
    PB_TRY(make_map(&me, e_in ? e_in : rhs, n, P, rows));
    const dim3 grid(prm.ntx, prm.nty, (n + z_chunk - 1) / z_chunk);
    PB_CHECK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                  "sweep_tma smem");
    kernel<<<grid, kThreads, smem, s>>>(me, mr, mi, prm);
    PB_CHECK_LAUNCH("sweep_tma kernel");
    return PB_OK;
}

template <int TY, int SLOTS>
static int launch_v2(bool zero_in, int n, int z_chunk, cudaStream_t s, const float* e_in, const float* rhs,
                     const float* invD, const pb::tma::Params& prm) {
    using namespace pb::tma;
    const size_t smem = sizeof(typename Geo2<TY, SLOTS>::Smem) + 128;
    return zero_in ? launch_sweep(sweep_v2_kernel<true, TY, SLOTS>, smem, TY, n, z_chunk, s, nullptr, rhs, invD, prm)
                   : launch_sweep(sweep_v2_kernel<false, TY, SLOTS>, smem, TY, n, z_chunk, s, e_in, rhs, invD, prm);
}

// Bits 8..15 of `mode` select a tile-height / ring-depth configuration of the
// kernel (0: 16 rows, 6 slots — the default); bit 2 selects the first TMA
// version.  Both are there for tuning runs.
extern "C" int pb_sweep_tma_f32(const float* e_in, float* e_out, const float* rhs, const float* invD, int64_t n,
                                int64_t mode, int64_t z_chunk, int* status, void* stream) {
    using namespace pb::tma;
    const bool legacy = (mode & 4) != 0;
    const int variant = (int)((mode >> 8) & 0xff);
    mode &= 3;
    if (n < 33 || n > 4097 || ((n - 1) & (n - 2)) || !e_out || !rhs || !invD || !status || (mode == 0 && !e_in) ||
        mode > 1 || variant > 5)
        return fail(PB_ERR_INVALID, "sweep_tma: bad args (n must be 2^k + 1 >= 33)");
    if (e_in == e_out) return fail(PB_ERR_INVALID, "sweep_tma: out of place only");
    const int N = (int)n;
    Params prm;
    prm.n = N;
    prm.P = pitch_for(N);
    prm.plane = (int64_t)(N + 2) * prm.P;
    prm.ntx = (N - 1) / kTX > 0 ? (N - 1) / kTX : 1;
    prm.nty = 1;
    prm.z_chunk = 0;
    prm.h2 = (float)((N - 1) * (N - 1));
    prm.e_out = e_out;
    prm.status = status;
    cudaStream_t s = (cudaStream_t)stream;
    const bool zero = mode == 1;
    if (legacy) {
        const size_t smem = sizeof(Smem) + 128;
        return zero ? launch_sweep(sweep_kernel<true>, smem, kTY, N, (int)z_chunk, s, nullptr, rhs, invD, prm)
                    : launch_sweep(sweep_kernel<false>, smem, kTY, N, (int)z_chunk, s, e_in, rhs, invD, prm);
    }
    switch (variant) {
        case 1: return launch_v2<16, 8>(zero, N, (int)z_chunk, s, e_in, rhs, invD, prm);
        case 2: return launch_v2<8, 6>(zero, N, (int)z_chunk, s, e_in, rhs, invD, prm);
        case 3: return launch_v2<8, 8>(zero, N, (int)z_chunk, s, e_in, rhs, invD, prm);
        case 4: return launch_v2<8, 10>(zero, N, (int)z_chunk, s, e_in, rhs, invD, prm);
        case 5: return launch_v2<16, 7>(zero, N, (int)z_chunk, s, e_in, rhs, invD, prm);
        default: return launch_v2<16, 6>(zero, N, (int)z_chunk, s, e_in, rhs, invD, prm);
    }
}

// fine += trilinear prolongation of coarse (side (n+1)/2), padded layouts.
extern "C" int pb_prolong_add_f32(const float* coarse, float* fine, int64_t fine_n, void* stream) {
    if (fine_n < 3 || fine_n > 4097 || !coarse || !fine) return fail(PB_ERR_INVALID, "prolong32: bad args");
    const int n = (int)fine_n, cn = (n + 1) / 2;
    int64_t blocks = ((int64_t)n * n * n + 255) / 256;
    if (blocks > kSMs * 16) blocks = kSMs * 16;
    prolong_add32_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(coarse, fine, n, pitch_for(n), cn,
                                                                             pitch_for(cn));
    PB_CHECK_LAUNCH("prolong_add32_kernel");
    return PB_OK;
}
