// Oriented points from a triangle mesh, bit-identical to the reference's loop.
//
// Reference: python/mojo_poissonrecon/core.py:429-451.  Per face (a, b, c) in
// order: cross = (v_b - v_a) x (v_c - v_a) (NumPy's cross: each product
// rounded, then the difference); a face whose cross is finite with a positive
// squared length adds cross to the normals of a, b and c, in that order, and
// marks them referenced.  Then length = sqrt((n_x^2 + n_y^2) + n_z^2); vertices
// that are referenced with a finite positive length are kept, in vertex order,
// with normal / length.
//
// Additions in the same order as the loop: every valid face emits three
// records (key = vertex, value = 3 face + corner); a stable radix sort groups
// them by vertex keeping face (and corner) order; one thread per vertex adds
// its contributions in that order, starting from zero.  Face indices outside
// [0, vertex_count) are not dereferenced: they set an error flag the host reads.
//
// Compiled with -fmad=false: every product and sum rounds as written.
#include "radix_sort.cuh"

namespace pb {
namespace mesh {

constexpr int kT = 256;

__global__ void face_records_kernel(const double* __restrict__ v, int64_t nv, const int64_t* __restrict__ faces,
                                    int64_t nf, uint32_t sentinel, uint32_t* __restrict__ keys,
                                    uint32_t* __restrict__ vals, double* __restrict__ cross,
                                    int* __restrict__ bad_index) {
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int64_t a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
    bool valid = false;
    double cx = 0.0, cy = 0.0, cz = 0.0;
    if (a < 0 || a >= nv || b < 0 || b >= nv || c < 0 || c >= nv) {
        atomicExch(bad_index, 1);
    } else {
        const double u0 = v[3 * b] - v[3 * a], u1 = v[3 * b + 1] - v[3 * a + 1], u2 = v[3 * b + 2] - v[3 * a + 2];
        const double w0 = v[3 * c] - v[3 * a], w1 = v[3 * c + 1] - v[3 * a + 1], w2 = v[3 * c + 2] - v[3 * a + 2];
        cx = u1 * w2 - u2 * w1;
        cy = u2 * w0 - u0 * w2;
        cz = u0 * w1 - u1 * w0;
        // squared length > 0: no cancellation among squares, so the order of their sum is immaterial
        valid = isfinite(cx) && isfinite(cy) && isfinite(cz) && (cx * cx + cy * cy + cz * cz) > 0.0;
    }
    cross[3 * f] = cx;
    cross[3 * f + 1] = cy;
    cross[3 * f + 2] = cz;
    const int64_t corner[3] = {a, b, c};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        keys[3 * f + k] = valid ? (uint32_t)corner[k] : sentinel;
        vals[3 * f + k] = (uint32_t)(3 * f + k);
    }
}

// Run heads (first record of each vertex's run, sentinel runs excluded),
// compacted in record order so the sums take one thread per run, full warps.
__global__ void head_flags_kernel(const uint32_t* __restrict__ keys, int64_t records, uint32_t sentinel,
                                  uint32_t* __restrict__ flag) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= records) return;
    const uint32_t vert = keys[j];
    flag[j] = vert != sentinel && (j == 0 || keys[j - 1] != vert);
}

__global__ void heads_kernel(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ rank, int64_t records,
                             uint32_t* __restrict__ heads) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < records && flag[j]) heads[rank[j]] = (uint32_t)j;
}

// One thread per run of records with the same vertex: the vertex's summed
// normal (zero-initialised), in face order; referenced[v] = 1.
__global__ void vertex_sums_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                                   int64_t records, const uint32_t* __restrict__ heads,
                                   const uint32_t* __restrict__ head_count, const double* __restrict__ cross,
                                   double* __restrict__ normals, uint32_t* __restrict__ referenced) {
    const uint32_t runs = *head_count;
    for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < runs; h += gridDim.x * blockDim.x) {
        const int64_t j = heads[h];
        const uint32_t vert = keys[j];
        double x = 0.0, y = 0.0, z = 0.0;
        for (int64_t k = j; k < records && keys[k] == vert; ++k) {
            const int64_t f = vals[k] / 3;
            x += cross[3 * f];
            y += cross[3 * f + 1];
            z += cross[3 * f + 2];
        }
        normals[3 * (int64_t)vert] = x;
        normals[3 * (int64_t)vert + 1] = y;
        normals[3 * (int64_t)vert + 2] = z;
        referenced[vert] = 1;
    }
}

// keep[v] (in place over referenced[v]) and the vertex's length.
__global__ void keep_flags_kernel(const double* __restrict__ normals, int64_t nv, uint32_t* __restrict__ keep,
                                  double* __restrict__ length) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const double x = normals[3 * i], y = normals[3 * i + 1], z = normals[3 * i + 2];
    const double len = sqrt((x * x + y * y) + z * z);
    length[i] = len;
    keep[i] = keep[i] && len > 0.0 && isfinite(len);
}

__global__ void emit_kernel(const double* __restrict__ v, const double* __restrict__ normals,
                            const double* __restrict__ length, const uint32_t* __restrict__ keep,
                            const uint32_t* __restrict__ rank, int64_t nv, double* __restrict__ out_points,
                            double* __restrict__ out_normals) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv || !keep[i]) return;
    const int64_t o = rank[i];
    const double len = length[i];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        out_points[3 * o + k] = v[3 * i + k];
        out_normals[3 * o + k] = normals[3 * i + k] / len;
    }
}

__global__ void store_kept_count_kernel(const uint32_t* __restrict__ total, const int* __restrict__ bad,
                                        int64_t* __restrict__ out) {
    out[0] = *total;
    out[1] = *bad;
}

struct Work {
    uint32_t *keys, *keys_alt, *vals, *vals_alt, *keep, *rank, *total;
    uint32_t *flag, *head_rank, *heads, *head_count;
    double *cross, *normals, *length;
    int* bad;
};

inline Work carve(Workspace& w, int64_t nv, int64_t nf) {
    Work o;
    const int64_t records = 3 * nf;
    o.keys = w.take<uint32_t>(records);
    o.keys_alt = w.take<uint32_t>(records);
    o.vals = w.take<uint32_t>(records);
    o.vals_alt = w.take<uint32_t>(records);
    o.cross = w.take<double>(3 * nf);
    o.normals = w.take<double>(3 * nv);
    o.length = w.take<double>(nv);
    o.keep = w.take<uint32_t>(nv + 1);
    o.rank = w.take<uint32_t>(nv + 1);
    o.total = w.take<uint32_t>(1);
    o.bad = w.take<int>(1);
    o.flag = w.take<uint32_t>(records);
    o.head_rank = w.take<uint32_t>(records);
    o.heads = w.take<uint32_t>(records);
    o.head_count = w.take<uint32_t>(1);
    return o;
}

inline size_t ws_bytes(int64_t nv, int64_t nf) {
    return measure([&](Workspace& w) {
        carve(w, nv, nf);
        radix_carve<uint32_t>(w, 3 * nf);
        scan_carve<uint32_t>(w, nv);
        scan_carve<uint32_t>(w, 3 * nf);
    });
}

inline int bit_width(uint64_t v) {
    int b = 0;
    while (v) {
        ++b;
        v >>= 1;
    }
    return b;
}

}  // namespace mesh
}  // namespace pb

using namespace pb;

extern "C" size_t pb_mesh_normals_workspace_size(int64_t vertex_count, int64_t face_count) {
    return mesh::ws_bytes(vertex_count < 1 ? 1 : vertex_count, face_count < 1 ? 1 : face_count);
}

// Pass 1 of oriented_points_from_mesh (core.py:429-451): counts[0] = kept
// vertices, counts[1] = 1 if a face index lies outside [0, vertex_count)
// (device int64[2]).  Leaves the per-vertex state in the workspace for
// pb_mesh_normals_emit_f64 (same arguments and workspace, called next).
extern "C" int pb_mesh_normals_count_f64(const double* vertices, int64_t vertex_count, const int64_t* faces,
                                         int64_t face_count, int64_t* counts, void* workspace,
                                         size_t workspace_bytes, void* stream) {
    using namespace pb::mesh;
    cudaStream_t s = (cudaStream_t)stream;
    if (vertex_count < 0 || vertex_count >= (int64_t)0xFFFFFFFFll || face_count < 0 ||
        3 * face_count >= (int64_t)0xFFFFFFFFll || !counts || (vertex_count && !vertices) || (face_count && !faces))
        return fail(PB_ERR_INVALID, "mesh normals: bad args");
    const size_t need = ws_bytes(vertex_count < 1 ? 1 : vertex_count, face_count < 1 ? 1 : face_count);
    if (!workspace || workspace_bytes < need)
        return fail(PB_ERR_WORKSPACE, "mesh normals: workspace needs %zu bytes", need);
    Workspace w(workspace, workspace_bytes);
    Work o = carve(w, vertex_count, face_count);
    PB_CHECK_CUDA(cudaMemsetAsync(o.bad, 0, sizeof(int), s), "mesh normals flag");
    PB_CHECK_CUDA(cudaMemsetAsync(o.keep, 0, sizeof(uint32_t) * (vertex_count + 1), s), "mesh normals keep");
    if (vertex_count)
        PB_CHECK_CUDA(cudaMemsetAsync(o.normals, 0, sizeof(double) * 3 * vertex_count, s), "mesh normals zero");
    const uint32_t sentinel = (uint32_t)vertex_count;
    if (face_count) {
        face_records_kernel<<<blocks_for(face_count, kT), kT, 0, s>>>(vertices, vertex_count, faces, face_count,
                                                                     sentinel, o.keys, o.vals, o.cross, o.bad);
        PB_CHECK_LAUNCH("face_records_kernel");
        bool in_alt = false;
        Workspace sort_ws = w;
        PB_TRY(radix_sort_pairs<uint32_t>(o.keys, o.vals, o.keys_alt, o.vals_alt, 3 * face_count,
                                          bit_width(sentinel), &in_alt, sort_ws, s));
        const uint32_t* keys = in_alt ? o.keys_alt : o.keys;
        const int64_t records = 3 * face_count;
        head_flags_kernel<<<blocks_for(records, kT), kT, 0, s>>>(keys, records, sentinel, o.flag);
        PB_CHECK_LAUNCH("head_flags_kernel");
        Workspace head_ws = w;
        PB_TRY(exclusive_scan<uint32_t>(o.flag, o.head_rank, records, o.head_count, head_ws, s));
        heads_kernel<<<blocks_for(records, kT), kT, 0, s>>>(o.flag, o.head_rank, records, o.heads);
        PB_CHECK_LAUNCH("heads_kernel");
        vertex_sums_kernel<<<8 * kSMs, kT, 0, s>>>(keys, in_alt ? o.vals_alt : o.vals, records, o.heads,
                                                   o.head_count, o.cross, o.normals, o.keep);
        PB_CHECK_LAUNCH("vertex_sums_kernel");
    }
    if (vertex_count) {
        keep_flags_kernel<<<blocks_for(vertex_count, kT), kT, 0, s>>>(o.normals, vertex_count, o.keep, o.length);
        PB_CHECK_LAUNCH("keep_flags_kernel");
    }
    Workspace scan_ws = w;
    PB_TRY(exclusive_scan<uint32_t>(o.keep, o.rank, vertex_count, o.total, scan_ws, s));
    store_kept_count_kernel<<<1, 1, 0, s>>>(o.total, o.bad, counts);
    PB_CHECK_LAUNCH("store_kept_count_kernel");
    return PB_OK;
}

// Pass 2: the kept vertices and their unit normals, in vertex order
// (out_points and out_normals: counts[0] x 3).
extern "C" int pb_mesh_normals_emit_f64(const double* vertices, int64_t vertex_count, const int64_t* faces,
                                        int64_t face_count, double* out_points, double* out_normals,
                                        void* workspace, size_t workspace_bytes, void* stream) {
    using namespace pb::mesh;
    (void)faces;
    if (vertex_count < 0 || face_count < 0 || (vertex_count && (!vertices || !out_points || !out_normals)))
        return fail(PB_ERR_INVALID, "mesh normals emit: bad args");
    const size_t need = ws_bytes(vertex_count < 1 ? 1 : vertex_count, face_count < 1 ? 1 : face_count);
    if (!workspace || workspace_bytes < need)
        return fail(PB_ERR_WORKSPACE, "mesh normals: workspace needs %zu bytes", need);
    if (!vertex_count) return PB_OK;
    Workspace w(workspace, workspace_bytes);
    Work o = carve(w, vertex_count, face_count);
    emit_kernel<<<blocks_for(vertex_count, kT), kT, 0, (cudaStream_t)stream>>>(
        vertices, o.normals, o.length, o.keep, o.rank, vertex_count, out_points, out_normals);
    PB_CHECK_LAUNCH("emit_kernel");
    return PB_OK;
}
