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

// Vertex of active cell (x, y, z): the mean of its edge roots (capi.mojo:964-1033),
// and the mean density of its corners.
__device__ __forceinline__ void cell_vertex(const double* __restrict__ field, const double* __restrict__ density,
                                            int64_t n, int64_t x, int64_t y, int64_t z, double iso, double cells_d,
                                            double* __restrict__ out, double* __restrict__ dens) {
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
    out[0] = ((double)x + sx * inv_roots) / cells_d;
    out[1] = ((double)y + sy * inv_roots) / cells_d;
    out[2] = ((double)z + sz * inv_roots) / cells_d;
    double dsum = 0.0;
#pragma unroll
    for (int corner = 0; corner < 8; ++corner)
        dsum += density[grid_index(x + (corner & 1), y + ((corner >> 1) & 1), z + ((corner >> 2) & 1), n)];
    *dens = dsum * 0.125;
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
        cell_vertex(field, density, n, x, y, z, iso, cells_d, vertices + 3 * id, vertex_density + id);
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


// ---- extraction for reconstruct(): sign bits and rank structures ----------------
// Same output, order and arithmetic as the two-pass kernels above, but the
// passes over all cells and edges read a bit per node (field < iso) instead of
// the FP64 field, and vertex ids are ranks in a bit array of active cells
// (prefix sum per 32-cell word + popcount) instead of a dense cell map.  Only
// active cells read field and density values.  Sides up to 1025 (32-bit
// node, cell and per-sweep edge indices).
namespace fast {

constexpr int kT = 256;
constexpr int64_t kMaxSide = 1025;

__device__ __forceinline__ uint32_t bit_at(const uint32_t* __restrict__ bits, uint32_t i) {
    return (bits[i >> 5] >> (i & 31)) & 1u;
}
__device__ __forceinline__ uint32_t lanes_below(uint32_t word, uint32_t b) { return __popc(word & ((1u << b) - 1u)); }

// bits: bit b of word w = (field[32w + b] < iso).
__global__ void __launch_bounds__(kT) sign_bits_kernel(const double* __restrict__ field, uint32_t nodes, IsoArg iso_arg,
                                                       uint32_t* __restrict__ bits) {
    const double iso = iso_arg.get();
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i - lane < nodes; i += stride) {
        const uint32_t m = __ballot_sync(0xffffffffu, i < nodes && field[i] < iso);
        if (lane == 0) bits[i >> 5] = m;
    }
}

// active cells (corners on both sides, capi.mojo:946-960) as bits, and the
// popcount of each 32-cell word (scanned in place into the word's first id).
__global__ void __launch_bounds__(kT) cell_words_kernel(const uint32_t* __restrict__ bits, uint32_t n, FastDiv dc,
                                                        uint32_t cells3, uint32_t* __restrict__ active,
                                                        uint32_t* __restrict__ counts) {
    const uint32_t c = n - 1, nn = n * n, lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i - lane < cells3; i += stride) {
        bool a = false;
        if (i < cells3) {
            const uint32_t ci = (uint32_t)i, t = dc.div(ci), x = ci - t * c, z = dc.div(t), y = t - z * c;
            const uint32_t i0 = (z * n + y) * n + x;
            const uint32_t below = bit_at(bits, i0) + bit_at(bits, i0 + 1) + bit_at(bits, i0 + n) +
                                   bit_at(bits, i0 + n + 1) + bit_at(bits, i0 + nn) + bit_at(bits, i0 + nn + 1) +
                                   bit_at(bits, i0 + nn + n) + bit_at(bits, i0 + nn + n + 1);
            a = below != 0 && below != 8;
        }
        const uint32_t m = __ballot_sync(0xffffffffu, a);
        if (lane == 0) {
            active[i >> 5] = m;
            counts[i >> 5] = __popc(m);
        }
    }
}

// Edge `local` of sweep s (capi.mojo:1090-1128): its lower node; sweep order z, y, x.
struct SideDiv {  // the cell count per axis c and c - 1, as invariant divisors
    uint32_t c;
    FastDiv dc, dm;
};

__device__ __forceinline__ void sweep_edge(int s, uint32_t local, const SideDiv& sd, uint32_t& x, uint32_t& y,
                                           uint32_t& z) {
    const uint32_t c = sd.c, cm1 = c - 1;
    if (s == 0) {  // x-edges: z, y in [1, c), x in [0, c)
        const uint32_t t = sd.dc.div(local), u = sd.dm.div(t);
        x = local - t * c;
        y = 1 + (t - u * cm1);
        z = 1 + u;
    } else if (s == 1) {  // y-edges: z in [1, c), y in [0, c), x in [1, c)
        const uint32_t t = sd.dm.div(local), u = sd.dc.div(t);
        x = 1 + (local - t * cm1);
        y = t - u * c;
        z = 1 + u;
    } else {  // z-edges: z in [0, c), y, x in [1, c)
        const uint32_t t = sd.dm.div(local), u = sd.dm.div(t);
        x = 1 + (local - t * cm1);
        y = 1 + (t - u * cm1);
        z = u;
    }
}

// Sign-changing edges of the three sweeps as bits (word w of sweep s at
// s * words + w) and per-word popcounts.  An interior edge that changes sign
// lies on four active cells, so it always yields a quad.
__global__ void __launch_bounds__(kT) edge_words_kernel(const uint32_t* __restrict__ bits, uint32_t n, SideDiv sd,
                                                        uint32_t per_sweep, uint32_t words,
                                                        uint32_t* __restrict__ fwords, uint32_t* __restrict__ counts) {
    const int s = blockIdx.y;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t step = s == 0 ? 1u : (s == 1 ? n : n * n);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e - lane < per_sweep; e += stride) {
        bool a = false;
        if (e < per_sweep) {
            uint32_t x, y, z;
            sweep_edge(s, (uint32_t)e, sd, x, y, z);
            const uint32_t i0 = (z * n + y) * n + x;
            a = bit_at(bits, i0) != bit_at(bits, i0 + step);
        }
        const uint32_t m = __ballot_sync(0xffffffffu, a);
        if (lane == 0) {
            fwords[(uint64_t)s * words + (e >> 5)] = m;
            counts[(uint64_t)s * words + (e >> 5)] = __popc(m);
        }
    }
}

__global__ void store_counts_kernel(const uint32_t* __restrict__ totals, int64_t* __restrict__ counts) {
    counts[0] = totals[0];
    counts[1] = 2 * (int64_t)totals[1];  // two triangles per quad
}

// One thread per 32-cell word: each active cell's vertex at id = its rank.
__global__ void __launch_bounds__(kT) vertex_words_kernel(const double* __restrict__ field,
                                                          const double* __restrict__ density, uint32_t n, FastDiv dc,
                                                          IsoArg iso_arg, const uint32_t* __restrict__ active,
                                                          const uint32_t* __restrict__ first, uint32_t cell_words,
                                                          double* __restrict__ vertices,
                                                          double* __restrict__ vertex_density) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= cell_words) return;
    uint32_t m = active[w];
    if (!m) return;
    const double iso = iso_arg.get();
    const uint32_t c = n - 1;
    const double cells_d = (double)c;
    uint32_t id = first[w];
    while (m) {
        const uint32_t b = __ffs(m) - 1;
        m &= m - 1;
        const uint32_t ci = 32 * w + b, t = dc.div(ci), x = ci - t * c, z = dc.div(t), y = t - z * c;
        cell_vertex(field, density, n, x, y, z, iso, cells_d, vertices + 3 * (int64_t)id, vertex_density + id);
        ++id;
    }
}

__device__ __forceinline__ int64_t cell_id(const uint32_t* __restrict__ active, const uint32_t* __restrict__ first,
                                           uint32_t ci) {
    return (int64_t)first[ci >> 5] + lanes_below(active[ci >> 5], ci & 31);
}

// One thread per 32-edge word: each sign-changing edge's two triangles at
// quad = its rank (capi.mojo:1040-1071).
__global__ void __launch_bounds__(kT) face_words_kernel(const uint32_t* __restrict__ bits, uint32_t n, SideDiv sd,
                                                        uint32_t words, const uint32_t* __restrict__ fwords,
                                                        const uint32_t* __restrict__ ffirst,
                                                        const uint32_t* __restrict__ active,
                                                        const uint32_t* __restrict__ first,
                                                        int64_t* __restrict__ faces) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= words) return;
    const int s = blockIdx.y;
    uint32_t m = fwords[(uint64_t)s * words + w];
    if (!m) return;
    const uint32_t c = n - 1;
    int64_t quad = ffirst[(uint64_t)s * words + w];
    while (m) {
        const uint32_t b = __ffs(m) - 1;
        m &= m - 1;
        uint32_t x, y, z;
        sweep_edge(s, 32 * w + b, sd, x, y, z);
        const bool reverse = bit_at(bits, (z * n + y) * n + x) != 0;
        uint32_t q[4];
        if (s == 0) {
            q[0] = (uint32_t)grid_index(x, y - 1, z - 1, c);
            q[1] = (uint32_t)grid_index(x, y, z - 1, c);
            q[2] = (uint32_t)grid_index(x, y, z, c);
            q[3] = (uint32_t)grid_index(x, y - 1, z, c);
        } else if (s == 1) {
            q[0] = (uint32_t)grid_index(x - 1, y, z - 1, c);
            q[1] = (uint32_t)grid_index(x - 1, y, z, c);
            q[2] = (uint32_t)grid_index(x, y, z, c);
            q[3] = (uint32_t)grid_index(x, y, z - 1, c);
        } else {
            q[0] = (uint32_t)grid_index(x - 1, y - 1, z, c);
            q[1] = (uint32_t)grid_index(x, y - 1, z, c);
            q[2] = (uint32_t)grid_index(x, y, z, c);
            q[3] = (uint32_t)grid_index(x - 1, y, z, c);
        }
        const int64_t a = cell_id(active, first, q[0]), bb = cell_id(active, first, q[1]);
        const int64_t cc = cell_id(active, first, q[2]), d = cell_id(active, first, q[3]);
        int64_t* out = faces + 6 * quad;
        if (reverse) {
            out[0] = a; out[1] = d; out[2] = cc; out[3] = a; out[4] = cc; out[5] = bb;
        } else {
            out[0] = a; out[1] = bb; out[2] = cc; out[3] = a; out[4] = cc; out[5] = d;
        }
        ++quad;
    }
}

inline uint64_t words_of(uint64_t items) { return (items + 31) / 32; }

// Arrays carved from the workspace, identically in count and emit.
struct Layout {
    uint32_t n, c, nodes, cells3, cell_words, per_sweep, words;
    uint32_t *bits, *active, *first, *fwords, *ffirst, *totals;
    void* base;
    size_t bytes, used;
    Workspace scratch() const {  // the scan scratch after the arrays
        Workspace w(base, bytes);
        w.used = used;
        return w;
    }
};

template <class W>
void carve(W& w, uint64_t nodes, uint64_t cell_words, uint64_t words, uint32_t** out) {
    out[0] = w.template take<uint32_t>(words_of(nodes));
    out[1] = w.template take<uint32_t>(cell_words);
    out[2] = w.template take<uint32_t>(cell_words + 1);
    out[3] = w.template take<uint32_t>(3 * words + 1);
    out[4] = w.template take<uint32_t>(3 * words + 1);
    out[5] = w.template take<uint32_t>(2);
}

inline Layout layout(int64_t n, void* base, size_t bytes) {
    Layout L{};
    L.n = (uint32_t)n;
    L.c = (uint32_t)(n - 1);
    L.nodes = (uint32_t)(n * n * n);
    L.cells3 = L.c * L.c * L.c;
    L.cell_words = (uint32_t)words_of(L.cells3);
    L.per_sweep = L.c == 0 ? 0 : L.c * (L.c - 1) * (L.c - 1);
    L.words = (uint32_t)words_of(L.per_sweep);
    Workspace w(base, bytes);
    uint32_t* p[6];
    carve(w, L.nodes, L.cell_words, L.words, p);
    L.bits = p[0];
    L.active = p[1];
    L.first = p[2];
    L.fwords = p[3];
    L.ffirst = p[4];
    L.totals = p[5];
    L.base = base;
    L.bytes = bytes;
    L.used = w.used;
    return L;
}

inline size_t workspace_bytes(int64_t n) {
    return measure([&](Workspace& w) {
        const uint64_t c = n - 1, nodes = (uint64_t)n * n * n, cells3 = c * c * c;
        const uint64_t per_sweep = c == 0 ? 0 : c * (c - 1) * (c - 1);
        const uint64_t cw = words_of(cells3), fw = words_of(per_sweep);
        uint32_t* p[6];
        carve(w, nodes, cw, fw, p);
        scan_carve<uint32_t>(w, (int64_t)(cw > 3 * fw ? cw : 3 * fw));
    });
}

inline unsigned grid_for(uint64_t items) {
    uint64_t b = (items + kT - 1) / kT;
    const uint64_t cap = (uint64_t)kSMs * 16;
    return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace fast

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

// ---- extraction for reconstruct() (no counterpart in the reference's C API) ----
extern "C" size_t pb_extract_workspace_size(int64_t n) { return fast::workspace_bytes(n < 2 ? 2 : n); }

// Counts of the mesh extract_isosurface(field, iso) would give (capi.mojo:
// 798-1129): counts[0] = vertices, counts[1] = triangles (device int64[2]).
// Leaves in the workspace the state pb_extract_emit_f64 needs: call emit next
// with the same field, side, iso and workspace.  Sides 2..1025.
extern "C" int pb_extract_count_f64(const double* field, int64_t n, const double* iso, int64_t* counts,
                                    void* workspace, size_t workspace_bytes, void* stream) {
    if (n < 2 || n > fast::kMaxSide || !field || !iso || !counts) return fail(PB_ERR_INVALID, "extract count: bad args");
    if (!workspace || workspace_bytes < fast::workspace_bytes(n))
        return fail(PB_ERR_WORKSPACE, "extract: workspace needs %zu bytes", fast::workspace_bytes(n));
    cudaStream_t s = (cudaStream_t)stream;
    fast::Layout L = fast::layout(n, workspace, workspace_bytes);
    const IsoArg ia{0.0, iso};
    fast::sign_bits_kernel<<<fast::grid_for(L.nodes), fast::kT, 0, s>>>(field, L.nodes, ia, L.bits);
    PB_CHECK_LAUNCH("sign_bits_kernel");
    const FastDiv dc(L.n - 1);
    const fast::SideDiv sd{L.n - 1, dc, FastDiv(L.n - 2)};
    fast::cell_words_kernel<<<fast::grid_for(L.cells3), fast::kT, 0, s>>>(L.bits, L.n, dc, L.cells3, L.active,
                                                                           L.first);
    PB_CHECK_LAUNCH("cell_words_kernel");
    Workspace scan_ws = L.scratch();
    PB_TRY(exclusive_scan<uint32_t>(L.first, L.first, L.cell_words, L.totals, scan_ws, s));
    if (L.per_sweep) {
        fast::edge_words_kernel<<<dim3(fast::grid_for(L.per_sweep), 3), fast::kT, 0, s>>>(L.bits, L.n, sd,
                                                                                           L.per_sweep, L.words,
                                                                                           L.fwords, L.ffirst);
        PB_CHECK_LAUNCH("edge_words_kernel");
        Workspace scan_ws2 = L.scratch();
        PB_TRY(exclusive_scan<uint32_t>(L.ffirst, L.ffirst, 3 * (int64_t)L.words, L.totals + 1, scan_ws2, s));
    } else {
        PB_CHECK_CUDA(cudaMemsetAsync(L.totals + 1, 0, sizeof(uint32_t), s), "extract face total");
    }
    fast::store_counts_kernel<<<1, 1, 0, s>>>(L.totals, counts);
    PB_CHECK_LAUNCH("store_counts_kernel");
    return PB_OK;
}

// Emits the counted mesh: vertices (counts[0] x 3), vertex_density
// (counts[0]), faces (counts[1] x 3), in the reference's order, bit-identical
// to pb_dual_vertices_f64 / pb_dual_faces_f64.  vertices (with
// vertex_density) or faces may be NULL when their count is 0; they are then
// not written.
extern "C" int pb_extract_emit_f64(const double* field, const double* density, int64_t n, const double* iso,
                                   double* vertices, double* vertex_density, int64_t* faces, void* workspace,
                                   size_t workspace_bytes, void* stream) {
    if (n < 2 || n > fast::kMaxSide || !field || !iso || (vertices && (!density || !vertex_density)))
        return fail(PB_ERR_INVALID, "extract emit: bad args");
    if (!workspace || workspace_bytes < fast::workspace_bytes(n))
        return fail(PB_ERR_WORKSPACE, "extract: workspace needs %zu bytes", fast::workspace_bytes(n));
    cudaStream_t s = (cudaStream_t)stream;
    fast::Layout L = fast::layout(n, workspace, workspace_bytes);
    const IsoArg ia{0.0, iso};
    if (vertices) {
        fast::vertex_words_kernel<<<(L.cell_words + fast::kT - 1) / fast::kT, fast::kT, 0, s>>>(
            field, density, L.n, FastDiv(L.n - 1), ia, L.active, L.first, L.cell_words, vertices, vertex_density);
        PB_CHECK_LAUNCH("vertex_words_kernel");
    }
    if (faces && L.per_sweep) {
        fast::face_words_kernel<<<dim3((L.words + fast::kT - 1) / fast::kT, 3), fast::kT, 0, s>>>(
            L.bits, L.n, fast::SideDiv{L.n - 1, FastDiv(L.n - 1), FastDiv(L.n - 2)}, L.words, L.fwords, L.ffirst,
            L.active, L.first, faces);
        PB_CHECK_LAUNCH("face_words_kernel");
    }
    return PB_OK;
}
