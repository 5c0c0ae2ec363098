// C ABI of the grouped launches (batch.cuh): a batch of clouds solved with one
// launch per step of the V-cycle and of FCG(1) for all of them.
//
// pb_batch_describe fills a host buffer of GridDesc (one per grid, first
// blocks as running sums in the given order); the caller copies it to device
// memory it owns (64-byte aligned) once, and pb_batch_launch then queues the
// step over those grids as often as needed (inside a captured graph too).
#include <cstring>

#include "batch.cuh"

namespace pb {
namespace batch {

int describe_sweep(GridDesc& d, bool zero_in, int64_t z_chunk);
int launch_sweep(const GridDesc* descs, int count, int64_t blocks, bool zero_in, const int* flags, cudaStream_t s);
int describe_prolong32(GridDesc& d);
int launch_prolong32(const GridDesc* descs, int count, int64_t blocks, const int* flags, cudaStream_t s);
int describe_residual_restrict32(GridDesc& d);
int launch_residual_restrict32(const GridDesc* descs, int count, int64_t blocks, const int* flags, cudaStream_t s);
int describe_relax27p(GridDesc& d, bool zero);
int launch_relax27p(const GridDesc* descs, int count, int64_t blocks, bool zero, const int* flags, cudaStream_t s);
int describe_residual27p(GridDesc& d);
int launch_residual27p(const GridDesc* descs, int count, int64_t blocks, const int* flags, cudaStream_t s);
int describe_restrict27(GridDesc& d);
int launch_restrict27(const GridDesc* descs, int count, int64_t blocks, const int* flags, cudaStream_t s);
int describe_coarse27(GridDesc& d);
int launch_coarse27(const GridDesc* descs, int count, int64_t blocks, int first_side, const int* flags,
                    cudaStream_t s);
int describe_fcg_direction(GridDesc& d);
int describe_fcg_update(GridDesc& d);
int describe_fcg_reduce(GridDesc& d);
int launch_fcg(int kind, const GridDesc* descs, int count, int64_t blocks, const int* flags, cudaStream_t s);
int launch_loop_batch(unsigned long long handle, const double* scal, const double* ctrl, int* flags, int clouds,
                      int max_iter, double* history, cudaStream_t s);
int64_t fcg_partials(int n);
int64_t fcg_direction_blocks(int n);
int64_t fcg_update_blocks(int n);

}  // namespace batch
}  // namespace pb

using namespace pb;
using namespace pb::batch;

extern "C" size_t pb_batch_desc_bytes(int64_t count) {
    return count < 0 ? 0 : (size_t)count * sizeof(GridDesc);
}

extern "C" int64_t pb_batch_fcg_partials(int64_t n) {
    if (n < 2 || n > 4097) return -1;
    return fcg_partials((int)n);
}

extern "C" int64_t pb_batch_fcg_blocks(int64_t n, int64_t pass) {
    if (n < 2 || n > 4097) return -1;
    return pass == 0 ? fcg_direction_blocks((int)n) : fcg_update_blocks((int)n);
}

extern "C" int pb_batch_describe(int kind, int64_t count, const int64_t* clouds, const int64_t* sides,
                                 const void* const* ptrs, const int64_t* aux, int64_t z_chunk, void* desc_host,
                                 size_t desc_bytes, int64_t* blocks_out) {
    if (count < 1 || count > (1 << 20) || !clouds || !sides || !ptrs || !desc_host || !blocks_out)
        return fail(PB_ERR_INVALID, "batch describe: bad args");
    if (desc_bytes < pb_batch_desc_bytes(count))
        return fail(PB_ERR_WORKSPACE, "batch describe: descriptor buffer needs %zu bytes", pb_batch_desc_bytes(count));
    if (reinterpret_cast<uintptr_t>(desc_host) % alignof(GridDesc))
        return fail(PB_ERR_INVALID, "batch describe: descriptor buffer must be 64-byte aligned");
    GridDesc* out = static_cast<GridDesc*>(desc_host);
    int64_t blocks = 0;
    for (int64_t i = 0; i < count; ++i) {
        GridDesc d;
        memset(&d, 0, sizeof(d));
        d.n = sides[i];
        d.cloud = clouds[i];
        if (d.cloud < 0) return fail(PB_ERR_INVALID, "batch describe: negative cloud index");
        for (int k = 0; k < kPtrs; ++k) d.ptr[k] = ptrs[i * kPtrs + k];
        if (aux)
            for (int k = 0; k < 4; ++k) d.aux[k] = aux[i * 4 + k];
        int st = PB_OK;
        switch (kind) {
            case PB_BATCH_SWEEP: st = describe_sweep(d, false, z_chunk); break;
            case PB_BATCH_SWEEP_ZERO: st = describe_sweep(d, true, z_chunk); break;
            case PB_BATCH_PROLONG32: st = describe_prolong32(d); break;
            case PB_BATCH_RESIDUAL_RESTRICT32: st = describe_residual_restrict32(d); break;
            case PB_BATCH_RELAX27P: st = describe_relax27p(d, false); break;
            case PB_BATCH_RELAX27P_ZERO: st = describe_relax27p(d, true); break;
            case PB_BATCH_RESIDUAL27P: st = describe_residual27p(d); break;
            case PB_BATCH_RESTRICT27: st = describe_restrict27(d); break;
            case PB_BATCH_COARSE27:
                st = describe_coarse27(d);
                if (st == PB_OK && i > 0 && d.n != out[0].n)
                    st = fail(PB_ERR_INVALID, "batch coarse27: every grid of a launch needs the same side");
                break;
            case PB_BATCH_FCG_DIRECTION:
            case PB_BATCH_FCG_UPDATE:
                st = kind == PB_BATCH_FCG_DIRECTION ? describe_fcg_direction(d) : describe_fcg_update(d);
                break;
            case PB_BATCH_FCG_DIRECTION_FINISH:
            case PB_BATCH_FCG_SUM: st = describe_fcg_reduce(d); break;
            default: st = fail(PB_ERR_INVALID, "batch describe: unknown kind %d", kind);
        }
        if (st != PB_OK) return st;
        d.block0 = blocks;
        blocks += d.gx * d.gy * d.gz;
        if (blocks > 0x7fffffffLL) return fail(PB_ERR_INVALID, "batch describe: more than 2^31 - 1 blocks");
        out[i] = d;
    }
    *blocks_out = blocks;
    return PB_OK;
}

extern "C" int pb_batch_launch(int kind, const void* desc_device, int64_t count, int64_t blocks, const int* flags,
                               int64_t first_side, void* stream) {
    if (!desc_device || count < 1 || blocks < 1 || blocks > 0x7fffffffLL || !flags)
        return fail(PB_ERR_INVALID, "batch launch: bad args");
    if (reinterpret_cast<uintptr_t>(desc_device) % alignof(GridDesc))
        return fail(PB_ERR_INVALID, "batch launch: descriptors must be 64-byte aligned");
    const GridDesc* d = static_cast<const GridDesc*>(desc_device);
    const int c = (int)count;
    cudaStream_t s = (cudaStream_t)stream;
    switch (kind) {
        case PB_BATCH_SWEEP: return launch_sweep(d, c, blocks, false, flags, s);
        case PB_BATCH_SWEEP_ZERO: return launch_sweep(d, c, blocks, true, flags, s);
        case PB_BATCH_PROLONG32: return launch_prolong32(d, c, blocks, flags, s);
        case PB_BATCH_RESIDUAL_RESTRICT32: return launch_residual_restrict32(d, c, blocks, flags, s);
        case PB_BATCH_RELAX27P: return launch_relax27p(d, c, blocks, false, flags, s);
        case PB_BATCH_RELAX27P_ZERO: return launch_relax27p(d, c, blocks, true, flags, s);
        case PB_BATCH_RESIDUAL27P: return launch_residual27p(d, c, blocks, flags, s);
        case PB_BATCH_RESTRICT27: return launch_restrict27(d, c, blocks, flags, s);
        case PB_BATCH_COARSE27: return launch_coarse27(d, c, blocks, (int)first_side, flags, s);
        case PB_BATCH_FCG_DIRECTION: return launch_fcg(0, d, c, blocks, flags, s);
        case PB_BATCH_FCG_DIRECTION_FINISH: return launch_fcg(1, d, c, blocks, flags, s);
        case PB_BATCH_FCG_UPDATE: return launch_fcg(2, d, c, blocks, flags, s);
        case PB_BATCH_FCG_SUM: return launch_fcg(3, d, c, blocks, flags, s);
    }
    return fail(PB_ERR_INVALID, "batch launch: unknown kind %d", kind);
}

extern "C" int pb_batch_loop_condition(unsigned long long handle, const double* scal, const double* ctrl, int* flags,
                                       int64_t clouds, int64_t max_iter, double* history, void* stream) {
    if (!scal || !ctrl || !flags || clouds < 1 || clouds > (1 << 20) || max_iter < 1)
        return fail(PB_ERR_INVALID, "batch loop condition: bad args");
    return launch_loop_batch(handle, scal, ctrl, flags, (int)clouds, (int)max_iter, history, (cudaStream_t)stream);
}
