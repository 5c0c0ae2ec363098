// Two-pass dual contouring (surface nets), order-preserving.
//
// Reference: src/capi.mojo:798-1129.  The reference numbers active cells
// serially in z,y,x order and emits quads in three serial sweeps (x-edges,
// y-edges, z-edges, each in z,y,x order).  Here both orders come from stream
// compaction: (1) per-tile counts, (2) an exclusive scan of the tile counts,
// (3) each tile recomputes its flags, scans them within the block and writes
// element i at (tile offset + rank).  Ids, vertex order and face order are
// therefore identical to the serial reference; vertex coordinates are exact
// restatements (compiled with -fmad=false).
#include "scan.cuh"

namespace pb {

constexpr int kDualThreads = 256;
constexpr int kDualItems = 8;
constexpr int kDualTile = kDualThreads * kDualItems;

struct IsoArg {
    double value;
    const double* ptr;
    __device__ __forceinline__ double get() const { return ptr ? *ptr : value; }
};

__device__ __forceinline__ bool cell_active(const double* __restrict__ f, int64_t x, int64_t y, int64_t z, int64_t n,
                                            double iso) {
    const int64_t i0 = (z * n + y) * n + x;
    const int64_t sy = n, sz = n * n;
    int below = (f[i0] < iso) + (f[i0 + 1] < iso) + (f[i0 + sy] < iso) + (f[i0 + sy + 1] < iso) +
                (f[i0 + sz] < iso) + (f[i0 + sz + 1] < iso) + (f[i0 + sz + sy] < iso) + (f[i0 + sz + sy + 1] < iso);
    return below != 0 && below != 8;
}

__global__ void __launch_bounds__(kDualThreads) cell_count_kernel(const double* __restrict__ field, int64_t n,
                                                                  IsoArg iso_arg, int64_t* __restrict__ tile_counts) {
    __shared__ int64_t warp_sums[32];
    const int64_t cells = n - 1;
    const int64_t total = cells * cells * cells;
    const double iso = iso_arg.get();
    const int64_t base = (int64_t)blockIdx.x * kDualTile + (int64_t)threadIdx.x * kDualItems;
    int64_t c = 0;
#pragma unroll
    for (int k = 0; k < kDualItems; ++k) {
        const int64_t i = base + k;
        if (i < total) {
            const int64_t x = i % cells, y = (i / cells) % cells, z = i / (cells * cells);
            c += cell_active(field, x, y, z, n, iso);
        }
    }
    int64_t t;
    block_exclusive_scan<int64_t>(c, warp_sums, t);
    if (threadIdx.x == 0) tile_counts[blockIdx.x] = t;
}

// capi.mojo:812-836
__device__ __forceinline__ int edge_root(double v0, double v1, double iso, double x0, double y0, double z0, double x1,
                                         double y1, double z1, double& sx, double& sy, double& sz) {
    if ((v0 < iso) == (v1 < iso)) return 0;
    double t = (iso - v0) / (v1 - v0);
    t = t > 0.0 ? t : 0.0;
    t = t < 1.0 ? t : 1.0;
    sx = sx + x0 + (x1 - x0) * t;
    sy = sy + y0 + (y1 - y0) * t;
    sz = sz + z0 + (z1 - z0) * t;
    return 1;
}

__global__ void __launch_bounds__(kDualThreads) vertex_emit_kernel(const double* __restrict__ field,
                                                                   const double* __restrict__ density, int64_t n,
                                                                   IsoArg iso_arg,
                                                                   const int64_t* __restrict__ tile_offsets,
                                                                   int64_t capacity, int64_t* __restrict__ cell_map,
                                                                   double* __restrict__ vertices,
                                                                   double* __restrict__ vertex_density) {
    __shared__ int64_t warp_sums[32];
    const int64_t cells = n - 1;
    const int64_t total = cells * cells * cells;
    const double iso = iso_arg.get();
    const int64_t base = (int64_t)blockIdx.x * kDualTile + (int64_t)threadIdx.x * kDualItems;
    unsigned active = 0;
    int64_t c = 0;
#pragma unroll
    for (int k = 0; k < kDualItems; ++k) {
        const int64_t i = base + k;
        if (i < total) {
            const int64_t x = i % cells, y = (i / cells) % cells, z = i / (cells * cells);
            if (cell_active(field, x, y, z, n, iso)) {
                active |= 1u << k;
                ++c;
            }
        }
    }
    int64_t t;
    int64_t id = tile_offsets[blockIdx.x] + block_exclusive_scan<int64_t>(c, warp_sums, t);
    const double cells_d = (double)cells;
    for (int k = 0; k < kDualItems; ++k) {
        const int64_t i = base + k;
        if (i >= total) break;
        if (!(active & (1u << k))) {
            cell_map[i] = -1;
            continue;
        }
        if (id >= capacity) {  // capi.mojo:961-963: past capacity, the cell keeps 0
            cell_map[i] = 0;
            ++id;
            continue;
        }
        const int64_t x = i % cells, y = (i / cells) % cells, z = i / (cells * cells);
        double v[8];
#pragma unroll
        for (int corner = 0; corner < 8; ++corner)
            v[corner] = field[grid_index(x + (corner & 1), y + ((corner >> 1) & 1), z + ((corner >> 2) & 1), n)];
        double sx = 0.0, sy = 0.0, sz = 0.0;
        int roots = 0;
        // x-edges, y-edges, z-edges; within each, (a, b) in row-major order (capi.mojo:968-1023).
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int c0 = 2 * a + 4 * b;
                roots += edge_root(v[c0], v[c0 + 1], iso, 0.0, (double)a, (double)b, 1.0, (double)a, (double)b, sx, sy, sz);
            }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int c0 = a + 4 * b;
                roots += edge_root(v[c0], v[c0 + 2], iso, (double)a, 0.0, (double)b, (double)a, 1.0, (double)b, sx, sy, sz);
            }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int c0 = a + 2 * b;
                roots += edge_root(v[c0], v[c0 + 4], iso, (double)a, (double)b, 0.0, (double)a, (double)b, 1.0, sx, sy, sz);
            }
        const double inv_roots = 1.0 / (double)roots;
        vertices[3 * id] = ((double)x + sx * inv_roots) / cells_d;
        vertices[3 * id + 1] = ((double)y + sy * inv_roots) / cells_d;
        vertices[3 * id + 2] = ((double)z + sz * inv_roots) / cells_d;
        double dsum = 0.0;
#pragma unroll
        for (int corner = 0; corner < 8; ++corner)
            dsum += density[grid_index(x + (corner & 1), y + ((corner >> 1) & 1), z + ((corner >> 2) & 1), n)];
        vertex_density[id] = dsum * 0.125;
        cell_map[i] = id;
        ++id;
    }
}

// Edge e of the three sweeps (capi.mojo:1090-1128).  Each sweep has
// cells*(cells-1)^2 edges; returns the quad's four cells (cell indices) and
// whether the edge changes sign, with v0 < iso for the orientation.
__device__ __forceinline__ bool edge_quad(const double* __restrict__ f, const int64_t* __restrict__ cm, int64_t n,
                                          double iso, int64_t e, int64_t per_sweep, int64_t q[4], bool& reverse) {
    const int64_t cells = n - 1;
    const int sweep = (int)(e / per_sweep);
    const int64_t local = e - (int64_t)sweep * per_sweep;
    int64_t x, y, z;
    const int64_t cm1 = cells - 1;
    double v0, v1;
    if (sweep == 0) {  // z in [1,cells), y in [1,cells), x in [0,cells)
        x = local % cells;
        y = 1 + (local / cells) % cm1;
        z = 1 + local / (cells * cm1);
        v0 = f[grid_index(x, y, z, n)];
        v1 = f[grid_index(x + 1, y, z, n)];
    } else if (sweep == 1) {  // z in [1,cells), y in [0,cells), x in [1,cells)
        x = 1 + local % cm1;
        y = (local / cm1) % cells;
        z = 1 + local / (cm1 * cells);
        v0 = f[grid_index(x, y, z, n)];
        v1 = f[grid_index(x, y + 1, z, n)];
    } else {  // z in [0,cells), y in [1,cells), x in [1,cells)
        x = 1 + local % cm1;
        y = 1 + (local / cm1) % cm1;
        z = local / (cm1 * cm1);
        v0 = f[grid_index(x, y, z, n)];
        v1 = f[grid_index(x, y, z + 1, n)];
    }
    if ((v0 < iso) == (v1 < iso)) return false;
    reverse = v0 < iso;
    if (sweep == 0) {
        q[0] = grid_index(x, y - 1, z - 1, cells);
        q[1] = grid_index(x, y, z - 1, cells);
        q[2] = grid_index(x, y, z, cells);
        q[3] = grid_index(x, y - 1, z, cells);
    } else if (sweep == 1) {
        q[0] = grid_index(x - 1, y, z - 1, cells);
        q[1] = grid_index(x - 1, y, z, cells);
        q[2] = grid_index(x, y, z, cells);
        q[3] = grid_index(x, y, z - 1, cells);
    } else {
        q[0] = grid_index(x - 1, y - 1, z, cells);
        q[1] = grid_index(x, y - 1, z, cells);
        q[2] = grid_index(x, y, z, cells);
        q[3] = grid_index(x - 1, y, z, cells);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        q[k] = cm[q[k]];
        if (q[k] < 0) return false;  // capi.mojo:1055-1056
    }
    return true;
}

__global__ void __launch_bounds__(kDualThreads) face_count_kernel(const double* __restrict__ field,
                                                                  const int64_t* __restrict__ cm, int64_t n,
                                                                  IsoArg iso_arg, int64_t per_sweep,
                                                                  int64_t* __restrict__ tile_counts) {
    __shared__ int64_t warp_sums[32];
    const int64_t total = 3 * per_sweep;
    const double iso = iso_arg.get();
    const int64_t base = (int64_t)blockIdx.x * kDualTile + (int64_t)threadIdx.x * kDualItems;
    int64_t c = 0;
    for (int k = 0; k < kDualItems; ++k) {
        const int64_t e = base + k;
        if (e >= total) break;
        int64_t q[4];
        bool rev;
        c += edge_quad(field, cm, n, iso, e, per_sweep, q, rev);
    }
    int64_t t;
    block_exclusive_scan<int64_t>(c, warp_sums, t);
    if (threadIdx.x == 0) tile_counts[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kDualThreads) face_emit_kernel(const double* __restrict__ field,
                                                                 const int64_t* __restrict__ cm, int64_t n,
                                                                 IsoArg iso_arg, int64_t per_sweep,
                                                                 const int64_t* __restrict__ tile_offsets,
                                                                 int64_t capacity, int64_t* __restrict__ faces) {
    __shared__ int64_t warp_sums[32];
    const int64_t total = 3 * per_sweep;
    const double iso = iso_arg.get();
    const int64_t base = (int64_t)blockIdx.x * kDualTile + (int64_t)threadIdx.x * kDualItems;
    int64_t q[kDualItems][4];
    unsigned emit = 0, rev = 0;
    int64_t c = 0;
#pragma unroll
    for (int k = 0; k < kDualItems; ++k) {
        const int64_t e = base + k;
        bool r = false;
        if (e < total && edge_quad(field, cm, n, iso, e, per_sweep, q[k], r)) {
            emit |= 1u << k;
            if (r) rev |= 1u << k;
            ++c;
        }
    }
    int64_t t;
    int64_t quad = tile_offsets[blockIdx.x] + block_exclusive_scan<int64_t>(c, warp_sums, t);
#pragma unroll
    for (int k = 0; k < kDualItems; ++k) {
        if (!(emit & (1u << k))) continue;
        const int64_t fc = 2 * quad;
        if (fc + 2 <= capacity) {  // capi.mojo:1057-1071
            int64_t* out = faces + 3 * fc;
            const int64_t a = q[k][0], b = q[k][1], cc = q[k][2], d = q[k][3];
            if (rev & (1u << k)) {
                out[0] = a; out[1] = d; out[2] = cc; out[3] = a; out[4] = cc; out[5] = b;
            } else {
                out[0] = a; out[1] = b; out[2] = cc; out[3] = a; out[4] = cc; out[5] = d;
            }
        }
        ++quad;
    }
}

__global__ void double_count_kernel(int64_t* __restrict__ count) { *count = 2 * *count; }

static int64_t tiles_of(int64_t items) { return (items + kDualTile - 1) / kDualTile; }

static size_t dual_ws_bytes(int64_t n) {
    const int64_t cells = n - 1;
    const int64_t vt = tiles_of(cells * cells * cells);
    const int64_t ft = tiles_of(3 * cells * (cells - 1) * (cells - 1));
    const int64_t tiles = vt > ft ? vt : ft;
    return measure([&](Workspace& w) {
        w.take<int64_t>(tiles);
        scan_carve<int64_t>(w, tiles);
    });
}

static int dual_vertices(const double* field, const double* density, int64_t n, IsoArg iso, int64_t* cell_map,
                         double* vertices, double* vertex_density, int64_t capacity, int64_t* count, void* workspace,
                         size_t workspace_bytes, cudaStream_t s) {
    if (n < 2 || n > 4097) return fail(PB_ERR_INVALID, "dual vertices: n must be in [2, 4097]");
    if (!field || !count) return fail(PB_ERR_INVALID, "dual vertices: null buffer");
    if (capacity > 0 && (!density || !cell_map || !vertices || !vertex_density))
        return fail(PB_ERR_INVALID, "dual vertices: null output buffer");
    const size_t need = dual_ws_bytes(n);
    if (!workspace || workspace_bytes < need) return fail(PB_ERR_WORKSPACE, "dual: workspace needs %zu bytes", need);
    Workspace w(workspace, workspace_bytes);
    const int64_t cells = n - 1;
    const int64_t total = cells * cells * cells;
    const int64_t tiles = tiles_of(total);
    int64_t* tile_counts = w.take<int64_t>(tiles);
    cell_count_kernel<<<(unsigned)tiles, kDualThreads, 0, s>>>(field, n, iso, tile_counts);
    PB_CHECK_LAUNCH("cell_count_kernel");
    PB_TRY(exclusive_scan<int64_t>(tile_counts, tile_counts, tiles, count, w, s));
    if (capacity > 0) {
        vertex_emit_kernel<<<(unsigned)tiles, kDualThreads, 0, s>>>(field, density, n, iso, tile_counts, capacity,
                                                                    cell_map, vertices, vertex_density);
        PB_CHECK_LAUNCH("vertex_emit_kernel");
    }
    return PB_OK;
}

static int dual_faces(const double* field, int64_t n, IsoArg iso, const int64_t* cell_map, int64_t* faces,
                      int64_t capacity, int64_t* count, void* workspace, size_t workspace_bytes, cudaStream_t s) {
    if (n < 2 || n > 4097) return fail(PB_ERR_INVALID, "dual faces: n must be in [2, 4097]");
    if (!field || !count || !cell_map) return fail(PB_ERR_INVALID, "dual faces: null buffer");
    if (capacity > 0 && !faces) return fail(PB_ERR_INVALID, "dual faces: null faces");
    const size_t need = dual_ws_bytes(n);
    if (!workspace || workspace_bytes < need) return fail(PB_ERR_WORKSPACE, "dual: workspace needs %zu bytes", need);
    const int64_t cells = n - 1;
    const int64_t per_sweep = cells * (cells - 1) * (cells - 1);
    if (per_sweep == 0) {
        PB_CHECK_CUDA(cudaMemsetAsync(count, 0, sizeof(int64_t), s), "dual faces count");
        return PB_OK;
    }
    Workspace w(workspace, workspace_bytes);
    const int64_t tiles = tiles_of(3 * per_sweep);
    int64_t* tile_counts = w.take<int64_t>(tiles);
    face_count_kernel<<<(unsigned)tiles, kDualThreads, 0, s>>>(field, cell_map, n, iso, per_sweep, tile_counts);
    PB_CHECK_LAUNCH("face_count_kernel");
    PB_TRY(exclusive_scan<int64_t>(tile_counts, tile_counts, tiles, count, w, s));
    if (capacity > 0) {
        face_emit_kernel<<<(unsigned)tiles, kDualThreads, 0, s>>>(field, cell_map, n, iso, per_sweep, tile_counts,
                                                                  capacity, faces);
        PB_CHECK_LAUNCH("face_emit_kernel");
    }
    double_count_kernel<<<1, 1, 0, s>>>(count);  // two triangles per quad
    PB_CHECK_LAUNCH("double_count_kernel");
    return PB_OK;
}

}  // namespace pb

using namespace pb;

extern "C" size_t pb_dual_workspace_size(int64_t n) { return dual_ws_bytes(n < 2 ? 2 : n); }

extern "C" int pb_dual_vertices_f64(const double* field, const double* density, int64_t n, double iso,
                                    int64_t* cell_map, double* vertices, double* vertex_density, int64_t capacity,
                                    int64_t* count, void* workspace, size_t workspace_bytes, void* stream) {
    return dual_vertices(field, density, n, IsoArg{iso, nullptr}, cell_map, vertices, vertex_density, capacity, count,
                         workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int pb_dual_vertices_f64_isoptr(const double* field, const double* density, int64_t n, const double* iso,
                                           int64_t* cell_map, double* vertices, double* vertex_density,
                                           int64_t capacity, int64_t* count, void* workspace, size_t workspace_bytes,
                                           void* stream) {
    if (!iso) return fail(PB_ERR_INVALID, "dual vertices: null iso pointer");
    return dual_vertices(field, density, n, IsoArg{0.0, iso}, cell_map, vertices, vertex_density, capacity, count,
                         workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int pb_dual_faces_f64(const double* field, int64_t n, double iso, const int64_t* cell_map, int64_t* faces,
                                 int64_t capacity, int64_t* count, void* workspace, size_t workspace_bytes,
                                 void* stream) {
    return dual_faces(field, n, IsoArg{iso, nullptr}, cell_map, faces, capacity, count, workspace, workspace_bytes,
                      (cudaStream_t)stream);
}

extern "C" int pb_dual_faces_f64_isoptr(const double* field, int64_t n, const double* iso, const int64_t* cell_map,
                                        int64_t* faces, int64_t capacity, int64_t* count, void* workspace,
                                        size_t workspace_bytes, void* stream) {
    if (!iso) return fail(PB_ERR_INVALID, "dual faces: null iso pointer");
    return dual_faces(field, n, IsoArg{0.0, iso}, cell_map, faces, capacity, count, workspace, workspace_bytes,
                      (cudaStream_t)stream);
}
