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

// 3D map over a padded level: dims (P, n+2, n+2) floats, box (72, 21, 1).
static int make_map(CUtensorMap* map, const float* base, int n, int P) {
    EncodeTiled enc = encoder();
    if (!enc) return fail(PB_ERR_CUDA, "sweep: cuTensorMapEncodeTiled is unavailable");
    if (reinterpret_cast<uintptr_t>(base) & 15) return fail(PB_ERR_INVALID, "sweep: arrays must be 16-byte aligned");
    const cuuint64_t dims[3] = {(cuuint64_t)P, (cuuint64_t)(n + 2), (cuuint64_t)(n + 2)};
    const cuuint64_t strides[2] = {(cuuint64_t)P * 4, (cuuint64_t)P * (n + 2) * 4};
    const cuuint32_t box[3] = {kBoxX, kBoxY, 1};
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
extern "C" int pb_sweep_tma_f32(const float* e_in, float* e_out, const float* rhs, const float* invD, int64_t n,
                                int64_t mode, int64_t z_chunk, int* status, void* stream) {
    using namespace pb::tma;
    if (n < 33 || n > 4097 || ((n - 1) & (n - 2)) || !e_out || !rhs || !invD || !status || (mode == 0 && !e_in) ||
        mode < 0 || mode > 1)
        return fail(PB_ERR_INVALID, "sweep_tma: bad args (n must be 2^k + 1 >= 33)");
    if (e_in == e_out) return fail(PB_ERR_INVALID, "sweep_tma: out of place only");
    const int N = (int)n, P = pitch_for(N);
    Params prm;
    prm.n = N;
    prm.P = P;
    prm.plane = (int64_t)(N + 2) * P;
    prm.ntx = (N - 1) / kTX > 0 ? (N - 1) / kTX : 1;
    prm.nty = (N - 1) / kTY > 0 ? (N - 1) / kTY : 1;
    const int tiles = prm.ntx * prm.nty;
    if (z_chunk <= 0) {
        const int want = 2 * kSMs;
        int chunks = want / tiles > 1 ? want / tiles : 1;
        z_chunk = (N + chunks - 1) / chunks;
        if (z_chunk < 4) z_chunk = 4;
    }
    prm.z_chunk = (int)z_chunk;
    prm.h2 = (float)((N - 1) * (N - 1));
    prm.e_out = e_out;
    prm.status = status;
    CUtensorMap me, mr, mi;
    PB_TRY(make_map(&mr, rhs, N, P));
    PB_TRY(make_map(&mi, invD, N, P));
    PB_TRY(make_map(&me, mode == 1 ? rhs : e_in, N, P));
    const dim3 grid(prm.ntx, prm.nty, (N + prm.z_chunk - 1) / prm.z_chunk);
    const size_t smem = sizeof(Smem) + 128;
    cudaStream_t s = (cudaStream_t)stream;
    if (mode == 1) {
        static bool attr1 = false;
        if (!attr1) {
            PB_CHECK_CUDA(cudaFuncSetAttribute(sweep_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                          "sweep_tma smem");
            attr1 = true;
        }
        sweep_kernel<true><<<grid, kThreads, smem, s>>>(me, mr, mi, prm);
    } else {
        static bool attr0 = false;
        if (!attr0) {
            PB_CHECK_CUDA(cudaFuncSetAttribute(sweep_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                          "sweep_tma smem");
            attr0 = true;
        }
        sweep_kernel<false><<<grid, kThreads, smem, s>>>(me, mr, mi, prm);
    }
    PB_CHECK_LAUNCH("sweep_tma kernel");
    return PB_OK;
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
