// TMA-staged fused red-black sweep on the padded FP32 layout (sm_100a).
//
// Same update as capi.mojo:310-410 for one iteration (colour 0 then colour 1)
// in FP32, out of place.  A block owns an (x, y) tile of up to 65 x 17 nodes
// and a z range, and marches z.  One thread issues cp.async.bulk.tensor loads
// of whole plane boxes (72 x 21 floats: the tile plus a halo of 2, x origin
// aligned to 16 bytes) of e_in, rhs and 1/D into a ring of kSlots slots, each
// guarded by an mbarrier, three planes ahead of the plane being updated.
// Each thread owns one float4 column group of the box for the whole march and
// keeps its planes in registers (see sweep_kernel); shared memory serves only
// the in-plane neighbours.  Out-of-grid nodes read as zero (ghost layer or TMA
// zero fill) and 1/D is zero there, so colour-0 values at halo nodes outside
// the grid come out zero without branches.
//
// Waits are bounded: a barrier that does not complete within ~1 s of SM clock
// sets *status = 1 and the block stops issuing work, after draining its own
// outstanding copies (also bounded).
#include <cuda.h>

#include "batch.cuh"
#include "common.cuh"

namespace pb {

namespace tma {

constexpr int kTX = 64;                 // interior tile width (last x tile: 65)
constexpr int kTY = 16;                 // interior tile height (last y tile: 17)
constexpr int kBoxX = 72;               // kTX + 1 + halo 2 + 2, rounded to 16 B; x origin = x0 - 4
constexpr int kBoxY = kTY + 1 + 4;      // 21
#ifndef PB_SWEEP_SLOTS
#define PB_SWEEP_SLOTS 5
#endif
#ifndef PB_SWEEP_MIN_BLOCKS
#define PB_SWEEP_MIN_BLOCKS 2
#endif
constexpr int kSlots = PB_SWEEP_SLOTS;  // planes t-1 .. t+3
constexpr long long kWaitCycles = 2000000000ll;

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

constexpr int kGroups = kBoxX / 4;  // 18 float4 column groups per box row

// Shared-memory ring of SLOTS planes: box of e, rhs and 1/D per plane.
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

// Each thread owns one float4 column group (box row br, group g: box columns
// 4g .. 4g+3) for the whole z range and keeps in registers the input of planes
// t-1, t and t+1, the colour-0-updated values of planes t-2 and t-1, and rhs
// and 1/D of planes t-1 and t.  At step t it updates colour 0 of plane t in
// place (float4 store back into the slot, read by the neighbours' colour-1
// updates), then colour 1 of plane t-1, written out together with that
// plane's colour-0 values as one float4.  A colour-0 update reads only
// colour-1 nodes and vice versa, so concurrent in-place stores never change a
// value another thread of the same phase uses.  Because x0 and y0 are even,
// the updated columns of a group on box row br are j = s and s + 2 with
// s = (br + t) & 1 in both phases.
constexpr int kThreads = 352;  // 19 box rows x 18 groups = 342 work items, one per thread
// SPLIT mapping: threads 0..191 take the odd box rows 1..19 (180 items) and
// threads 192..383 the even rows 2..18 (162 items), so every warp's rows share
// one parity, s is warp-uniform, and each phase computes only the two lanes it
// updates (the others are selected away in the default mapping).
constexpr int kSplitHalf = 192, kSplitThreads = 2 * kSplitHalf;
static_assert(10 * kGroups <= kSplitHalf && 9 * kGroups <= kSplitHalf, "one item per thread");

// The sweep of tile (bx, by) and z chunk bz; the maps may live in kernel
// parameters (single grid) or in global memory (grouped launches).
// ONE_BAR: the ring slot of plane t - 2 is refilled right after plane t's first
// barrier (plane t - 2 was last read by the previous step's colour-1 pass), so
// the barrier at the end of each step goes; needs SLOTS >= 4 (plane t + 1,
// waited for at step t, is issued at step t + 3 - SLOTS).
template <bool ZERO_IN, int SLOTS, bool SPLIT = false, bool ONE_BAR = false>
__device__ __forceinline__ void sweep_body(const CUtensorMap* map_e, const CUtensorMap* map_rhs,
                                           const CUtensorMap* map_invD, const Params& p, int bx, int by, int bz) {
    static_assert(!ONE_BAR || SLOTS >= 4, "the early refill needs four ring slots");
    constexpr int TY = kTY;
    using G = Geo2<TY, SLOTS>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = saddr(smem_raw);
    typename G::Smem& S = *reinterpret_cast<typename G::Smem*>(smem_raw + (((raw + 127u) & ~127u) - raw));
    const int n = p.n;
    const int x0 = bx * kTX, y0 = by * TY;
    const int W = (bx == p.ntx - 1 ? n : x0 + kTX) - x0;
    const int H = (by == p.nty - 1 ? n : y0 + TY) - y0;
    const int zb = bz * p.z_chunk;
    const int ze = min(n, zb + p.z_chunk);
    const int zfirst = zb - 2, zlast = ze + 1;
    const int tid = threadIdx.x;
    const uint32_t bytes = (ZERO_IN ? 2u : 3u) * G::kBox * 4u;
    const float h2 = p.h2;

    if (tid == 0) {
        for (int s = 0; s < SLOTS; ++s) bar_init(&S.bar[s]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto slot_of = [&](int z) { return (z - zfirst) % SLOTS; };
    auto parity_of = [&](int z) { return (uint32_t)(((z - zfirst) / SLOTS) & 1); };
    auto issue = [&](int z) {
        const int s = slot_of(z);
        bar_expect(&S.bar[s], bytes);
        if (!ZERO_IN) load_box(S.slot[s][0], map_e, x0, y0 - 1, z + 1, &S.bar[s]);
        load_box(S.slot[s][1], map_rhs, x0, y0 - 1, z + 1, &S.bar[s]);
        load_box(S.slot[s][2], map_invD, x0, y0 - 1, z + 1, &S.bar[s]);
    };
    int issued = zfirst;
    if (tid == 0)
        for (; issued <= zlast && issued < zfirst + SLOTS; ++issued) issue(issued);

    // this thread's work item (rows past the box: no work, barriers only)
    int br, g;
    if (SPLIT) {
        const bool odd = tid < kSplitHalf;
        const int item = odd ? tid : tid - kSplitHalf, r = item / kGroups;
        br = (odd ? 1 : 2) + 2 * r;
        g = item - r * kGroups;
    } else {
        br = 1 + tid / kGroups;
        g = tid - (br - 1) * kGroups;
    }
    const bool has_a = br <= H + 2;                                       // colour-0 region rows 1 .. H+2
    const bool has_b = br >= 2 && br <= H + 1 && g >= 1 && g <= (W + 3) / 4;  // output rows and groups
    const int base = br * kBoxX + 4 * g;
    const int b0 = 4 * g;
    bool upd_ok[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) upd_ok[j] = (b0 + j >= 3) && (b0 + j < W + 5);
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);

    bool ok = bar_wait(&S.bar[slot_of(zfirst)], parity_of(zfirst));
    ok = bar_wait(&S.bar[slot_of(zfirst + 1)], parity_of(zfirst + 1)) && ok;
    ok = __syncthreads_and(ok);

    // registers: e at t-1 (input), e at t (input); updated colour-0 planes t-2, t-1
    float4 e_prev = zero4, e_cur = zero4;
    if (!ZERO_IN && has_a && ok) {
        e_prev = lds4(S.slot[slot_of(zb - 2)][0] + base);
        e_cur = lds4(S.slot[slot_of(zb - 1)][0] + base);
    }
    float4 r_prev = zero4, i_prev = zero4, red_prev2 = zero4, red_prev = zero4;

    for (int t = zb - 1; t <= ze && ok; ++t) {
        const bool arrived = bar_wait(&S.bar[slot_of(t + 1)], parity_of(t + 1));
        float4 red_cur = zero4, r_cur = zero4, i_cur = zero4, e_next = zero4;
        if (has_a) {  // colour 0 of plane t
            const float* e = S.slot[slot_of(t)][0];
            r_cur = lds4(S.slot[slot_of(t)][1] + base);
            i_cur = lds4(S.slot[slot_of(t)][2] + base);
            const int s = (br + t) & 1;
            float v[4];
            if (ZERO_IN) {
                v[0] = r_cur.x * i_cur.x; v[1] = r_cur.y * i_cur.y; v[2] = r_cur.z * i_cur.z; v[3] = r_cur.w * i_cur.w;
            } else if (SPLIT) {  // s is warp-uniform: only the updated lanes
                e_next = lds4(S.slot[slot_of(t + 1)][0] + base);
                const float4 u = lds4(e + base - kBoxX), d = lds4(e + base + kBoxX);
                const float4 c = e_cur, zm = e_prev, zp = e_next;
                if (s == 0) {
                    const float L = g > 0 ? e[base - 1] : 0.0f;
                    v[0] = (r_cur.x + (L + c.y + u.x + d.x + zm.x + zp.x) * h2) * i_cur.x;
                    v[2] = (r_cur.z + (c.y + c.w + u.z + d.z + zm.z + zp.z) * h2) * i_cur.z;
                    v[1] = v[3] = 0.0f;
                } else {
                    const float R = g < kGroups - 1 ? e[base + 4] : 0.0f;
                    v[1] = (r_cur.y + (c.x + c.z + u.y + d.y + zm.y + zp.y) * h2) * i_cur.y;
                    v[3] = (r_cur.w + (c.z + R + u.w + d.w + zm.w + zp.w) * h2) * i_cur.w;
                    v[0] = v[2] = 0.0f;
                }
            } else {
                e_next = lds4(S.slot[slot_of(t + 1)][0] + base);
                const float4 u = lds4(e + base - kBoxX), d = lds4(e + base + kBoxX);
                const float L = g > 0 ? e[base - 1] : 0.0f;
                const float R = g < kGroups - 1 ? e[base + 4] : 0.0f;
                const float4 c = e_cur, zm = e_prev, zp = e_next;
                v[0] = (r_cur.x + (L + c.y + u.x + d.x + zm.x + zp.x) * h2) * i_cur.x;
                v[1] = (r_cur.y + (c.x + c.z + u.y + d.y + zm.y + zp.y) * h2) * i_cur.y;
                v[2] = (r_cur.z + (c.y + c.w + u.z + d.z + zm.z + zp.z) * h2) * i_cur.z;
                v[3] = (r_cur.w + (c.z + R + u.w + d.w + zm.w + zp.w) * h2) * i_cur.w;
            }
            float cc[4] = {e_cur.x, e_cur.y, e_cur.z, e_cur.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) cc[j] = ((j & 1) == s && upd_ok[j]) ? v[j] : cc[j];
            red_cur = make_float4(cc[0], cc[1], cc[2], cc[3]);
            *reinterpret_cast<float4*>(S.slot[slot_of(t)][0] + base) = red_cur;
            if (ONE_BAR) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // before a TMA refill
        }
        ok = __syncthreads_and(arrived);
        if (!ok) break;
        if (ONE_BAR && tid == 0 && t - 2 >= zfirst && issued <= zlast) issue(issued++);  // into plane t-2's slot
        if (has_b && t - 1 >= zb) {  // colour 1 of plane t-1, written out with its colour 0
            const int z = t - 1;
            const float* e = S.slot[slot_of(z)][0];
            const float4 u = lds4(e + base - kBoxX), d = lds4(e + base + kBoxX);
            const float4 c = red_prev, zm = red_prev2, zp = red_cur;
            const int s = (br + t) & 1;
            float v[4];
            if (SPLIT) {  // s is warp-uniform: only the updated lanes
                if (s == 0) {
                    const float L = e[base - 1];
                    v[0] = (r_prev.x + (L + c.y + u.x + d.x + zm.x + zp.x) * h2) * i_prev.x;
                    v[2] = (r_prev.z + (c.y + c.w + u.z + d.z + zm.z + zp.z) * h2) * i_prev.z;
                    v[1] = v[3] = 0.0f;
                } else {
                    const float R = g < kGroups - 1 ? e[base + 4] : 0.0f;
                    v[1] = (r_prev.y + (c.x + c.z + u.y + d.y + zm.y + zp.y) * h2) * i_prev.y;
                    v[3] = (r_prev.w + (c.z + R + u.w + d.w + zm.w + zp.w) * h2) * i_prev.w;
                    v[0] = v[2] = 0.0f;
                }
            } else {
                const float L = e[base - 1];
                const float R = g < kGroups - 1 ? e[base + 4] : 0.0f;
                v[0] = (r_prev.x + (L + c.y + u.x + d.x + zm.x + zp.x) * h2) * i_prev.x;
                v[1] = (r_prev.y + (c.x + c.z + u.y + d.y + zm.y + zp.y) * h2) * i_prev.y;
                v[2] = (r_prev.z + (c.y + c.w + u.z + d.z + zm.z + zp.z) * h2) * i_prev.z;
                v[3] = (r_prev.w + (c.z + R + u.w + d.w + zm.w + zp.w) * h2) * i_prev.w;
            }
            float o[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) o[j] = ((j & 1) == s) ? v[j] : o[j];
            const int64_t oi = ((int64_t)(z + 1) * (n + 2) + (y0 - 1 + br)) * p.P + (x0 + 4 * g);
            float* dst = p.e_out + oi;
            const int valid = W + 4 - 4 * g;
            PB_GUARD(oi + (valid < 4 ? valid : 4) - 1, (int64_t)(n + 2) * p.plane, kSiteSweepStore)
            if (valid >= 4) {
                *reinterpret_cast<float4*>(dst) = make_float4(o[0], o[1], o[2], o[3]);
            } else {
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    if (j < valid) dst[j] = o[j];
            }
        }
        red_prev2 = red_prev;
        red_prev = red_cur;
        r_prev = r_cur;
        i_prev = i_cur;
        e_prev = e_cur;
        e_cur = e_next;
        if (!ONE_BAR) {
            __syncthreads();  // plane t-1 is no longer read
            if (tid == 0 && t - 1 >= zfirst && issued <= zlast) issue(issued++);
        }
    }
    if (!ok) {
        if (tid == 0) {
            atomicExch(p.status, 1);
            for (int z = max(zfirst, issued - SLOTS); z < issued; ++z)
                (void)bar_wait(&S.bar[slot_of(z)], parity_of(z));
        }
        __syncthreads();
    }
}

// SLOTS planes in the shared ring (at least 3: planes t-1, t, t+1), MINB
// resident blocks per SM the register budget must allow; the autotuner picks
// among the compiled pairs (PB_TUNE_SWEEP_VARIANT).
template <bool ZERO_IN, int SLOTS, int MINB, bool SPLIT = false, bool ONE_BAR = false>
__global__ void __launch_bounds__(SPLIT ? kSplitThreads : kThreads, MINB)
    sweep_kernel(const __grid_constant__ CUtensorMap map_e, const __grid_constant__ CUtensorMap map_rhs,
                 const __grid_constant__ CUtensorMap map_invD, Params p) {
    sweep_body<ZERO_IN, SLOTS, SPLIT, ONE_BAR>(&map_e, &map_rhs, &map_invD, p, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Grouped: one launch over the level-0 sweeps of many clouds (batch.cuh).
// Descriptor operands: map[0..2] = e_in, rhs, 1/D; ptr[0] = e_out, ptr[1] =
// status word; aux[0] = z chunk.
template <bool ZERO_IN, int SLOTS>
__global__ void __launch_bounds__(kThreads, PB_SWEEP_MIN_BLOCKS)
    sweep_grouped_kernel(const batch::GridDesc* __restrict__ descs, int count, const int* __restrict__ flags) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    Params p;
    p.n = (int)d.n;
    p.P = ((p.n + 5) + 7) & ~7;
    p.plane = (int64_t)(p.n + 2) * p.P;
    p.ntx = (int)d.gx;
    p.nty = (int)d.gy;
    p.z_chunk = (int)d.aux[0];
    p.h2 = (float)((p.n - 1) * (p.n - 1));
    p.e_out = (float*)d.ptr[0];
    p.status = (int*)d.ptr[1];
    sweep_body<ZERO_IN, SLOTS>(&d.map[0], &d.map[1], &d.map[2], p, bx, by, bz);
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

// ---- level-0 residual with the scaled restriction, planes staged by TMA ----------
// The arithmetic of residual_restrict32_kernel (stencil32.cu) on the same 64 x 4
// coarse tile and z march, with its inputs brought in by cp.async.bulk.tensor
// instead of per-thread float4 loads: per fine plane one box of e (144 x 11:
// the 136 x 9 residual region and a one-node halo, x origin aligned to 16 B)
// and one box each of rhs, D and s (136 x 9), into a ring of four planes, two
// planes ahead of the plane being computed, each slot guarded by an mbarrier.
// Every thread reads its float4 groups from shared memory; the residual ring
// keeps planes 2zc-1 .. 2zc+1 for the restriction.  Per node and per coarse
// node the same expressions in the same order: bit-identical results.  Waits
// are bounded as in the sweep (status word, drain, stop).
constexpr int kRCX = 64, kRCY = 4;
constexpr int kRFX = 2 * kRCX + 8, kRFY = 2 * kRCY + 1;  // 136 x 9 residuals: fine x from 2 xc0 - 4, y from 2 yc0 - 1
constexpr int kREX = kRFX + 8, kREY = kRFY + 2;          // 144 x 11 of e: fine x from 2 xc0 - 8, y from 2 yc0 - 2
constexpr int kRSlots = 4;
constexpr int kRRes = 3;  // residual planes 2zc-1 .. 2zc+1
constexpr int kRThreads = 320;  // one float4 item of a fine plane per thread (306 items); 256 restrict
static_assert(kRFY * (kRFX / 4) <= kRThreads && kRCX * kRCY <= kRThreads, "one round per plane");
constexpr int kREStride = (kREX * kREY + 31) / 32 * 32;  // 128-byte aligned boxes
constexpr int kRFStride = (kRFX * kRFY + 31) / 32 * 32;
constexpr uint32_t kREBytes = kREX * kREY * 4, kRFBytes = kRFX * kRFY * 4;

struct RSmem {
    float e[kRSlots][kREStride];
    float rhs[kRSlots][kRFStride];
    float d[kRSlots][kRFStride];
    float w[kRSlots][kRFStride];
    float res[kRRes][kRFY][kRFX];
    unsigned long long bar[kRSlots];
};

__global__ void __launch_bounds__(kRThreads, 2)
    residual_restrict_tma_kernel(const __grid_constant__ CUtensorMap map_e, const __grid_constant__ CUtensorMap map_b,
                                 const __grid_constant__ CUtensorMap map_d, const __grid_constant__ CUtensorMap map_w,
                                 int fn, int cn, int cz, float h2, float* __restrict__ coarse, int cP,
                                 int* __restrict__ status) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = saddr(smem_raw);
    RSmem& S = *reinterpret_cast<RSmem*>(smem_raw + (((raw + 127u) & ~127u) - raw));
    const int xc0 = blockIdx.x * kRCX, yc0 = blockIdx.y * kRCY;
    const int zc0 = blockIdx.z * cz, zc1 = min(cn, zc0 + cz);
    const int fx0 = 2 * xc0 - 4, fy0 = 2 * yc0 - 1;
    const int pe0 = 2 * zc0 - 2, pe1 = 2 * zc1;  // e planes read; rhs, D, s for pe0 + 1 .. pe1 - 1
    const int tid = threadIdx.x;
    auto slot_of = [&](int p) { return (p - pe0) % kRSlots; };
    auto parity_of = [&](int p) { return (uint32_t)(((p - pe0) / kRSlots) & 1); };
    auto issue = [&](int p) {
        const int sl = slot_of(p);
        const bool inner = p > pe0 && p < pe1;
        bar_expect(&S.bar[sl], kREBytes + (inner ? 3 * kRFBytes : 0));
        load_box(S.e[sl], &map_e, 2 * xc0 - 4, 2 * yc0 - 1, p + 1, &S.bar[sl]);
        if (inner) {
            load_box(S.rhs[sl], &map_b, 2 * xc0, 2 * yc0, p + 1, &S.bar[sl]);
            load_box(S.d[sl], &map_d, 2 * xc0, 2 * yc0, p + 1, &S.bar[sl]);
            load_box(S.w[sl], &map_w, 2 * xc0, 2 * yc0, p + 1, &S.bar[sl]);
        }
    };
    if (tid == 0) {
        for (int k = 0; k < kRSlots; ++k) bar_init(&S.bar[k]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int issued = pe0;
    if (tid == 0)
        for (; issued <= pe1 && issued < pe0 + kRSlots; ++issued) issue(issued);
    bool ok = bar_wait(&S.bar[slot_of(pe0)], parity_of(pe0));
    ok = bar_wait(&S.bar[slot_of(pe0 + 1)], parity_of(pe0 + 1)) && ok;
    ok = __syncthreads_and(ok);
    for (int f = pe0 + 1; f < pe1 && ok; ++f) {
        ok = __syncthreads_and(bar_wait(&S.bar[slot_of(f + 1)], parity_of(f + 1)));
        if (!ok) break;
        {  // s-weighted residual of fine plane f (residual_restrict32_body's expressions)
            const float* ec = S.e[slot_of(f)];
            const float* em = S.e[slot_of(f - 1)];
            const float* ep = S.e[slot_of(f + 1)];
            const float* bb = S.rhs[slot_of(f)];
            const float* dd = S.d[slot_of(f)];
            const float* ww = S.w[slot_of(f)];
            float(*dst)[kRFX] = S.res[(f + kRRes) % kRRes];
            constexpr int kGroups = kRFX / 4;
            for (int i = tid; i < kRFY * kGroups; i += kRThreads) {
                const int ly = i / kGroups, g = i - ly * kGroups;
                const int x = fx0 + 4 * g, y = fy0 + ly;
                float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
                if (f >= 0 && f < fn && y >= 0 && y < fn && x >= 0 && x < fn) {
                    const int q = (ly + 1) * kREX + 4 * g + 4, k = ly * kRFX + 4 * g;
                    const float4 c = *reinterpret_cast<const float4*>(ec + q);
                    const float4 ym = *reinterpret_cast<const float4*>(ec + q - kREX);
                    const float4 yp = *reinterpret_cast<const float4*>(ec + q + kREX);
                    const float4 zm = *reinterpret_cast<const float4*>(em + q);
                    const float4 zp = *reinterpret_cast<const float4*>(ep + q);
                    const float4 b = *reinterpret_cast<const float4*>(bb + k);
                    const float4 d = *reinterpret_cast<const float4*>(dd + k);
                    const float4 sw = *reinterpret_cast<const float4*>(ww + k);
                    const float l = ec[q - 1], rr = ec[q + 4];
                    const float s0 = l + c.y + ym.x + yp.x + zm.x + zp.x;
                    const float s1 = c.x + c.z + ym.y + yp.y + zm.y + zp.y;
                    const float s2 = c.y + c.w + ym.z + yp.z + zm.z + zp.z;
                    const float s3 = c.z + rr + ym.w + yp.w + zm.w + zp.w;
                    r.x = sw.x * (b.x - (d.x * c.x - s0 * h2));
                    r.y = x + 1 < fn ? sw.y * (b.y - (d.y * c.y - s1 * h2)) : 0.f;
                    r.z = x + 2 < fn ? sw.z * (b.z - (d.z * c.z - s2 * h2)) : 0.f;
                    r.w = x + 3 < fn ? sw.w * (b.w - (d.w * c.w - s3 * h2)) : 0.f;
                }
                *reinterpret_cast<float4*>(&dst[ly][4 * g]) = r;
            }
        }
        __syncthreads();  // plane f's residual complete; e of plane f - 1 read for the last time
        if (f > pe0 + 1 && (f & 1)) {  // f = 2 zc + 1 with zc >= zc0: restrict coarse plane zc
            const int zc = (f - 1) / 2;
            const int cy = tid / kRCX, cx = tid - cy * kRCX;
            const int xc = xc0 + cx, yc = yc0 + cy;
            if (cy < kRCY && xc < cn && yc < cn) {
                float sum = 0.0f;
#pragma unroll
                for (int oz = -1; oz <= 1; ++oz) {
                    const int zz = 2 * zc + oz;
#pragma unroll
                    for (int oy = -1; oy <= 1; ++oy) {
                        const float* row = S.res[(zz + kRRes) % kRRes][2 * cy + 1 + oy];
#pragma unroll
                        for (int ox = -1; ox <= 1; ++ox)
                            sum += row[2 * cx + 4 + ox] * (float)((ox ? 1 : 2) * (oy ? 1 : 2) * (oz ? 1 : 2));
                    }
                }
                coarse[((int64_t)(zc + 1) * (cn + 2) + (yc + 1)) * cP + (xc + 4)] = sum * (1.0f / 64.0f);
            }
            // plane 2zc+2 (the slot of 2zc-1) is written after the next step's barrier
        }
        if (tid == 0 && issued <= pe1) {  // into the slot of plane f - 1, read for the last time above
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(issued++);
        }
    }
    if (!ok) {
        if (tid == 0) {
            atomicExch(status, 1);
            for (int p = max(pe0, issued - kRSlots); p < issued; ++p) (void)bar_wait(&S.bar[slot_of(p)], parity_of(p));
        }
        __syncthreads();
    }
}

// A 3D map over a padded level with a box of `width` x `rows` x 1 floats.
static int make_box_map(CUtensorMap* map, const float* base, int n, int P, int width, int rows) {
    EncodeTiled enc = encoder();
    if (!enc) return fail(PB_ERR_CUDA, "tma: cuTensorMapEncodeTiled is unavailable");
    if (reinterpret_cast<uintptr_t>(base) & 15) return fail(PB_ERR_INVALID, "tma: arrays must be 16-byte aligned");
    const cuuint64_t dims[3] = {(cuuint64_t)P, (cuuint64_t)(n + 2), (cuuint64_t)(n + 2)};
    const cuuint64_t strides[2] = {(cuuint64_t)P * 4, (cuuint64_t)P * (n + 2) * 4};
    const cuuint32_t box[3] = {(cuuint32_t)width, (cuuint32_t)rows, 1};
    const cuuint32_t estride[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estride,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(PB_ERR_CUDA, "tma: cuTensorMapEncodeTiled failed (%d)", (int)r);
    return PB_OK;
}

}  // namespace tma

// ---- scaled prolongation add on the padded layout -------------------------------
// fine += s * trilinear(coarse) (the P_s of mg27.cu; trilinear as in
// capi.mojo:677-742), s the fine level's prolongation weights.
// A thread owns four consecutive fine x (one float4 of e and of s; x offset 4
// keeps them 16-byte aligned), a block 256 consecutive (group, y) slots of a
// plane and `tz` fine planes (up to kProTZ, fewer on small levels so that the grid still fills
// the GPU: the planes of a block run one after another).  The four fine nodes of a thread share three coarse values per
// coarse row: fine x = 4k + j lies on coarse 2k + j/2 (even j) or between
// 2k + j/2 and the next (odd j).  Fine x >= n (ghost and padding) is never
// written.
constexpr int kProTX = 32, kProTY = 8, kProTZ = 16;

__device__ __forceinline__ void prolong_add32_body(const float* __restrict__ c, float* __restrict__ f,
                                                   const float* __restrict__ w, int n, int P, int cn, int cP, int tz,
                                                   int row, int bx, int by) {
    // threads flattened over the plane's (float4 group, y), `row` threads per y:
    // the group count on short rows (full warps), a whole number of warps on
    // long ones (a warp's coarse reads stay on one row)
    const unsigned t = bx * (kProTX * kProTY) + threadIdx.x;
    const int groups = (n + 3) / 4;
    const int y = (int)(t / (unsigned)row), k = (int)(t - (unsigned)y * row);
    if (y >= n || k >= groups) return;
    const int x = 4 * k;
    const int z0 = by * tz, z1 = min(n, z0 + tz);
    const int ya = y >> 1, yb = min(ya + 1, cn - 1);
    const float ty = (y & 1) ? 0.5f : 0.f;
    const int64_t cplane = (int64_t)(cn + 2) * cP;
    // coarse row ya, columns 2k .. 2k+2 (offset 4); column 2k+2 <= cn + 1 stays inside the padded row
    const float* ca = c + (int64_t)(ya + 1) * cP + (2 * k + 4);
    const int64_t dy = (int64_t)(yb - ya) * cP;
    const int valid = min(4, n - x);
    for (int z = z0; z < z1; ++z) {
        const int za = z >> 1, zb = min(za + 1, cn - 1);
        const float wz = (z & 1) ? 0.5f : 0.f;
        const float* c0 = ca + (int64_t)(za + 1) * cplane;
        const float* c1 = ca + (int64_t)(zb + 1) * cplane;
        float q[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float a0 = c0[i] * (1.f - ty) + c0[dy + i] * ty;
            const float a1 = c1[i] * (1.f - ty) + c1[dy + i] * ty;
            q[i] = a0 * (1.f - wz) + a1 * wz;
        }
        // x interpolation: t = 0 on even x, 1/2 on odd x (coarse 2k + 2 only weighs odd x < n - 1)
        const float v0 = q[0], v1 = q[0] * 0.5f + q[1] * 0.5f, v2 = q[1], v3 = q[1] * 0.5f + q[2] * 0.5f;
        const int64_t p = ((int64_t)(z + 1) * (n + 2) + (y + 1)) * P + (x + 4);
        PB_GUARD(p + (valid < 4 ? valid : 4) - 1, (int64_t)(n + 2) * (n + 2) * P, kSiteProlong)
        if (valid == 4) {
            float4 e = *reinterpret_cast<const float4*>(f + p);
            const float4 s = *reinterpret_cast<const float4*>(w + p);
            e.x += s.x * v0;
            e.y += s.y * v1;
            e.z += s.z * v2;
            e.w += s.w * v3;
            *reinterpret_cast<float4*>(f + p) = e;
        } else {
            const float v[4] = {v0, v1, v2, v3};
#pragma unroll
            for (int j = 0; j < 3; ++j)
                if (j < valid) f[p + j] += w[p + j] * v[j];
        }
    }
}

__global__ void __launch_bounds__(kProTX* kProTY) prolong_add32_kernel(const float* __restrict__ c,
                                                                       float* __restrict__ f,
                                                                       const float* __restrict__ w, int n, int P,
                                                                       int cn, int cP, int tz, int row) {
    prolong_add32_body(c, f, w, n, P, cn, cP, tz, row, blockIdx.x, blockIdx.y);
}

// Grouped (batch.cuh): ptr[0] = coarse, ptr[1] = fine, ptr[2] = weights;
// aux[0] = planes per block, aux[1] = threads per row.
__global__ void __launch_bounds__(kProTX* kProTY) prolong_add32_grouped_kernel(const batch::GridDesc* __restrict__ descs,
                                                                               int count,
                                                                               const int* __restrict__ flags) {
    int bx, by, bz;
    const batch::GridDesc& d = batch::locate(descs, count, blockIdx.x, bx, by, bz);
    if (!batch::cloud_active(flags, d.cloud)) return;
    const int n = (int)d.n, cn = (n + 1) / 2;
    prolong_add32_body((const float*)d.ptr[0], (float*)d.ptr[1], (const float*)d.ptr[2], n, ((n + 5) + 7) & ~7, cn,
                       ((cn + 5) + 7) & ~7, (int)d.aux[0], (int)d.aux[1], bx, by);
}

}  // namespace pb

using namespace pb;

static int pitch_for(int n) { return ((n + 5) + 7) & ~7; }

// One TMA-staged fused sweep.  n = 2^k + 1 >= 33 (smaller levels use the
// single-block coarse kernel).  mode 0: from e_in; mode 1: from zero.
// z_chunk <= 0 picks one that puts two blocks on each of the 148 SMs.
// *status (device int) is set to 1 if a bounded wait gave up.
extern "C" int pb_sweep_tma_f32(const float* e_in, float* e_out, const float* rhs, const float* invD, int64_t n,
                                int64_t mode, int64_t z_chunk, int* status, void* stream) {
    using namespace pb::tma;
    if (n < 33 || n > 4097 || ((n - 1) & (n - 2)) || !e_out || !rhs || !invD || !status || (mode == 0 && !e_in) ||
        mode < 0 || mode > 1)
        return fail(PB_ERR_INVALID, "sweep_tma: bad args (n must be 2^k + 1 >= 33)");
    if (e_in == e_out) return fail(PB_ERR_INVALID, "sweep_tma: out of place only");
    const int N = (int)n;
    Params prm;
    prm.n = N;
    prm.P = pitch_for(N);
    prm.plane = (int64_t)(N + 2) * prm.P;
    prm.ntx = (N - 1) / kTX > 0 ? (N - 1) / kTX : 1;
    prm.nty = (N - 1) / kTY > 0 ? (N - 1) / kTY : 1;
    const int tiles = prm.ntx * prm.nty;
    // ring slots and resident blocks per SM: (5, 2) built in, (4, 3) and (3, 3) as
    // variants 1 and 2; variants 3, 4 and 5: the SPLIT mapping with (5, 2), (6, 2),
    // (4, 3); variants 6, 7 and 8: the same with ONE_BAR
    const int64_t variant = tuned(PB_TUNE_SWEEP_VARIANT, n, 0);
    const int64_t v3 = variant >= 6 ? variant - 3 : variant;
    const int ring = v3 == 1 || v3 == 5 ? 4 : v3 == 2 ? 3 : v3 == 4 ? 6 : kSlots;
    const int per_sm = v3 == 1 || v3 == 2 || v3 == 5 ? 3 : PB_SWEEP_MIN_BLOCKS;
    if (z_chunk <= 0) z_chunk = tuned(PB_TUNE_SWEEP_Z_CHUNK, n, 0);
    if (z_chunk <= 0) {
        // c chunks per tile: minimise waves x (planes per chunk + the 4 planes a
        // chunk loads beyond its range), waves = ceil(tiles c / (resident blocks x
        // 148 SMs)).  At 257^3 with 2 blocks per SM this picks c = 9 (two waves,
        // 66 us a sweep) over the one-wave c = 4 (70 us, 40 of 296 slots idle);
        // measured on B200.
        const int64_t slots = (int64_t)per_sm * kSMs;
        int64_t best = -1;
        int chosen = 1;
        for (int c = 1; c <= N; ++c) {
            const int zc = (N + c - 1) / c;
            if (zc < 4) break;
            const int64_t cost = ((int64_t)tiles * c + slots - 1) / slots * (zc + 4);
            if (best < 0 || cost < best) {
                best = cost;
                chosen = c;
            }
        }
        z_chunk = (N + chosen - 1) / chosen;
    }
    prm.z_chunk = (int)z_chunk;
    prm.h2 = (float)((N - 1) * (N - 1));
    prm.e_out = e_out;
    prm.status = status;
    CUtensorMap me, mr, mi;
    PB_TRY(make_map(&mr, rhs, N, prm.P, kBoxY));
    PB_TRY(make_map(&mi, invD, N, prm.P, kBoxY));
    PB_TRY(make_map(&me, mode == 1 ? rhs : e_in, N, prm.P, kBoxY));
    const dim3 grid(prm.ntx, prm.nty, (N + prm.z_chunk - 1) / prm.z_chunk);
    cudaStream_t s = (cudaStream_t)stream;
    const bool split = variant >= 3 && variant <= 8;
    auto launch = [&](auto kernel, size_t smem) -> int {
        PB_CHECK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                      "sweep_tma smem");
        kernel<<<grid, split ? kSplitThreads : kThreads, smem, s>>>(me, mr, mi, prm);
        PB_CHECK_LAUNCH("sweep_tma kernel");
        return PB_OK;
    };
    const size_t s5 = sizeof(Geo2<kTY, kSlots>::Smem) + 128, s4 = sizeof(Geo2<kTY, 4>::Smem) + 128,
                 s3 = sizeof(Geo2<kTY, 3>::Smem) + 128;
    if (variant == 3)
        return mode == 1 ? launch(sweep_kernel<true, 5, 2, true>, sizeof(Geo2<kTY, 5>::Smem) + 128)
                         : launch(sweep_kernel<false, 5, 2, true>, sizeof(Geo2<kTY, 5>::Smem) + 128);
    if (variant == 4)
        return mode == 1 ? launch(sweep_kernel<true, 6, 2, true>, sizeof(Geo2<kTY, 6>::Smem) + 128)
                         : launch(sweep_kernel<false, 6, 2, true>, sizeof(Geo2<kTY, 6>::Smem) + 128);
    if (variant == 5)
        return mode == 1 ? launch(sweep_kernel<true, 4, 3, true>, s4) : launch(sweep_kernel<false, 4, 3, true>, s4);
    if (variant == 6)
        return mode == 1 ? launch(sweep_kernel<true, 5, 2, true, true>, s5)
                         : launch(sweep_kernel<false, 5, 2, true, true>, s5);
    if (variant == 7)
        return mode == 1 ? launch(sweep_kernel<true, 6, 2, true, true>, sizeof(Geo2<kTY, 6>::Smem) + 128)
                         : launch(sweep_kernel<false, 6, 2, true, true>, sizeof(Geo2<kTY, 6>::Smem) + 128);
    if (variant == 8)
        return mode == 1 ? launch(sweep_kernel<true, 4, 3, true, true>, s4)
                         : launch(sweep_kernel<false, 4, 3, true, true>, s4);
    if (ring == 4)
        return mode == 1 ? launch(sweep_kernel<true, 4, 3>, s4) : launch(sweep_kernel<false, 4, 3>, s4);
    if (ring == 3)
        return mode == 1 ? launch(sweep_kernel<true, 3, 3>, s3) : launch(sweep_kernel<false, 3, 3>, s3);
    return mode == 1 ? launch(sweep_kernel<true, kSlots, PB_SWEEP_MIN_BLOCKS>, s5)
                     : launch(sweep_kernel<false, kSlots, PB_SWEEP_MIN_BLOCKS>, s5);
}

// fine += s * trilinear(coarse) (coarse side (n+1)/2), padded layouts, s the
// fine level's prolongation weights.
extern "C" int pb_prolong_fac_f32(const float* coarse, float* fine, const float* weights, int64_t fine_n,
                                  void* stream) {
    if (fine_n < 3 || fine_n > 4097 || !coarse || !fine || !weights) return fail(PB_ERR_INVALID, "prolong32: bad args");
    const int n = (int)fine_n, cn = (n + 1) / 2;
    const int groups = (n + 3) / 4;
    const int row = groups < 64 ? groups : (groups + 31) / 32 * 32;  // measured: 257^3 keeps whole-warp rows
    const int gxy = (row * n + kProTX * kProTY - 1) / (kProTX * kProTY);
    // planes per block: as many as keep at least 4 blocks per SM, at most kProTZ
    const int64_t fill = (int64_t)gxy * n / (4 * kSMs);
    const int tz = (int)tuned(PB_TUNE_PROLONG_PLANES, n, fill < 1 ? 1 : (fill > kProTZ ? kProTZ : fill));
    const dim3 grid(gxy, (n + tz - 1) / tz);
    prolong_add32_kernel<<<grid, kProTX * kProTY, 0, (cudaStream_t)stream>>>(coarse, fine, weights, n, pitch_for(n),
                                                                              cn, pitch_for(cn), tz, row);
    PB_CHECK_LAUNCH("prolong_add32_kernel");
    return PB_OK;
}

// ---- grouped launches (batch.cuh) ----------------------------------------------------

namespace pb {
namespace batch {

// Level-0 sweep of one grid: ptr[0] e_in (ignored from zero), ptr[1] e_out,
// ptr[2] rhs, ptr[3] 1/D, ptr[4] status word; z_chunk <= 0: whole planes.
int describe_sweep(GridDesc& d, bool zero_in, int64_t z_chunk) {
    using namespace pb::tma;
    const int N = (int)d.n;
    if (N < 33 || N > 4097 || ((N - 1) & (N - 2)))
        return fail(PB_ERR_INVALID, "batch sweep: side must be 2^k + 1 >= 33 (got %d)", N);
    const float* e_in = (const float*)d.ptr[0];
    const float* rhs = (const float*)d.ptr[2];
    const float* invD = (const float*)d.ptr[3];
    if ((!zero_in && !e_in) || !d.ptr[1] || !rhs || !invD || !d.ptr[4] || e_in == d.ptr[1])
        return fail(PB_ERR_INVALID, "batch sweep: bad operands");
    const int P = pitch_for(N);
    PB_TRY(make_map(&d.map[0], zero_in ? rhs : e_in, N, P, kBoxY));
    PB_TRY(make_map(&d.map[1], rhs, N, P, kBoxY));
    PB_TRY(make_map(&d.map[2], invD, N, P, kBoxY));
    const int zc = z_chunk <= 0 || z_chunk > N ? N : (int)z_chunk;
    d.gx = (N - 1) / kTX > 0 ? (N - 1) / kTX : 1;
    d.gy = (N - 1) / kTY > 0 ? (N - 1) / kTY : 1;
    d.gz = (N + zc - 1) / zc;
    d.aux[0] = zc;
    d.ptr[0] = d.ptr[1];  // e_out, as the grouped kernel reads it
    d.ptr[1] = d.ptr[4];  // status
    return PB_OK;
}

int launch_sweep(const GridDesc* descs, int count, int64_t blocks, bool zero_in, const int* flags, cudaStream_t s) {
    using namespace pb::tma;
    const size_t smem = sizeof(Geo2<kTY, kSlots>::Smem) + 128;
    auto go = [&](auto kernel) -> int {
        PB_CHECK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                      "batch sweep smem");
        kernel<<<(unsigned)blocks, kThreads, smem, s>>>(descs, count, flags);
        PB_CHECK_LAUNCH("sweep_grouped_kernel");
        return PB_OK;
    };
    return zero_in ? go(sweep_grouped_kernel<true, kSlots>) : go(sweep_grouped_kernel<false, kSlots>);
}

// fine += s * trilinear(coarse): ptr[0] coarse, ptr[1] fine, ptr[2] weights.
int describe_prolong32(GridDesc& d) {
    const int n = (int)d.n;
    if (n < 3 || n > 4097 || !d.ptr[0] || !d.ptr[1] || !d.ptr[2]) return fail(PB_ERR_INVALID, "batch prolong: bad args");
    const int groups = (n + 3) / 4;
    const int row = groups < 64 ? groups : (groups + 31) / 32 * 32;
    const int gxy = (row * n + kProTX * kProTY - 1) / (kProTX * kProTY);
    const int tz = (int)tuned(PB_TUNE_PROLONG_PLANES, n, n < kProTZ ? n : kProTZ);
    d.gx = gxy;
    d.gy = (n + tz - 1) / tz;
    d.gz = 1;
    d.aux[0] = tz;
    d.aux[1] = row;
    return PB_OK;
}

int launch_prolong32(const GridDesc* descs, int count, int64_t blocks, const int* flags, cudaStream_t s) {
    prolong_add32_grouped_kernel<<<(unsigned)blocks, kProTX * kProTY, 0, s>>>(descs, count, flags);
    PB_CHECK_LAUNCH("prolong_add32_grouped_kernel");
    return PB_OK;
}

}  // namespace batch
}  // namespace pb

// Level 0: coarse_rhs = P^T (s (rhs - A e)) / 8 with the fine planes staged by
// TMA (same results as pb_residual_restrict_f32).  *status (device int) is set
// to 1 if a bounded wait gave up.
extern "C" int pb_residual_restrict_tma_f32(const float* e, const float* rhs, const float* D, const float* weights,
                                            float* coarse_rhs, int64_t n, int* status, void* stream) {
    using namespace pb::tma;
    if (n < 33 || n > 4097 || ((n - 1) & (n - 2)) || !e || !rhs || !D || !weights || !coarse_rhs || !status)
        return fail(PB_ERR_INVALID, "residual_restrict_tma: bad args (n must be 2^k + 1 >= 33)");
    const int fn = (int)n, cn = (fn + 1) / 2;
    const int P = pitch_for(fn);
    CUtensorMap me, mb, md, mw;
    PB_TRY(make_box_map(&me, e, fn, P, kREX, kREY));
    PB_TRY(make_box_map(&mb, rhs, fn, P, kRFX, kRFY));
    PB_TRY(make_box_map(&md, D, fn, P, kRFX, kRFY));
    PB_TRY(make_box_map(&mw, weights, fn, P, kRFX, kRFY));
    int cz = (int)tuned(PB_TUNE_RESTRICT_PLANES, n, 4);
    if (cz < 1) cz = 1;
    const dim3 grid((cn + kRCX - 1) / kRCX, (cn + kRCY - 1) / kRCY, (cn + cz - 1) / cz);
    const size_t smem = sizeof(RSmem) + 128;
    PB_CHECK_CUDA(cudaFuncSetAttribute(residual_restrict_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem),
                  "residual_restrict_tma smem");
    residual_restrict_tma_kernel<<<grid, kRThreads, smem, (cudaStream_t)stream>>>(
        me, mb, md, mw, fn, cn, cz, (float)((fn - 1) * (fn - 1)), coarse_rhs, pitch_for(cn), status);
    PB_CHECK_LAUNCH("residual_restrict_tma_kernel");
    return PB_OK;
}
