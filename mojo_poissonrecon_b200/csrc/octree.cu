// Morton codes and the breadth-first flat octree on the device.
//
// Reference: src/capi.mojo:62-99 (codes), python/mojo_poissonrecon/core.py:86-127
// (per-level np.unique, breadth-first concatenation, parent/child links,
// point_leaf).  Here: leaf codes are radix-sorted once; because a level-l code
// is the leaf code shifted right by 3*(depth-l), the sorted leaf order is also
// sorted order at every level.  For sorted position i, L_i = the shallowest
// level at which its code differs from position i-1 (0 for i = 0, depth+1 for
// an identical leaf).  Position i starts a new level-l node iff L_i <= l, so a
// prefix count of (L_i <= l) numbers the level's nodes in ascending code
// order — exactly np.unique's order — and the level-(l-1) count at the same
// position is the parent.
#include "radix_sort.cuh"

namespace pb {

// Per-level child index chain, capi.mojo:72-99 (integer conversion truncates
// toward zero, then clamps to [0, 2^level - 1]).
__device__ __forceinline__ int64_t level_cell(double v, int64_t scale) {
    int64_t i = (int64_t)(v * (double)scale);
    if (i < 0) i = 0;
    if (i >= scale) i = scale - 1;
    return i;
}

__global__ void octree_codes_kernel(const double* __restrict__ points, int64_t count, int depth,
                                    int64_t* __restrict__ codes) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    double x = points[3 * i], y = points[3 * i + 1], z = points[3 * i + 2];
    int64_t code = 0;
    int64_t* out = codes + i * (depth + 1);
    out[0] = 0;
    for (int d = 0; d < depth; ++d) {
        int64_t scale = (int64_t)1 << (d + 1);
        int64_t child = (level_cell(x, scale) & 1) | ((level_cell(y, scale) & 1) << 1) |
                        ((level_cell(z, scale) & 1) << 2);
        code = (code << 3) | child;
        out[d + 1] = code;
    }
}

__global__ void leaf_keys_kernel(const double* __restrict__ points, int64_t count, int depth,
                                 uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    double x = points[3 * i], y = points[3 * i + 1], z = points[3 * i + 2];
    uint64_t code = 0;
    for (int d = 0; d < depth; ++d) {
        int64_t scale = (int64_t)1 << (d + 1);
        uint64_t child = (uint64_t)((level_cell(x, scale) & 1) | ((level_cell(y, scale) & 1) << 1) |
                                    ((level_cell(z, scale) & 1) << 2));
        code = (code << 3) | child;
    }
    keys[i] = code;
    vals[i] = (uint32_t)i;
}

// L_i and its histogram (bins 0..depth+1).
__global__ void split_level_kernel(const uint64_t* __restrict__ keys, int64_t count, int depth,
                                   uint8_t* __restrict__ split, unsigned long long* __restrict__ hist) {
    __shared__ unsigned int local[32];
    if (threadIdx.x < 32) local[threadIdx.x] = 0;
    __syncthreads();
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        int level;
        if (i == 0) {
            level = 0;
        } else {
            uint64_t diff = keys[i] ^ keys[i - 1];
            if (diff == 0) {
                level = depth + 1;
            } else {
                int high_bit = 63 - __clzll((long long)diff);
                level = depth - high_bit / 3;
            }
        }
        split[i] = (uint8_t)level;
        atomicAdd(&local[level], 1u);
    }
    __syncthreads();
    if (threadIdx.x < depth + 2 && local[threadIdx.x]) atomicAdd(&hist[threadIdx.x], (unsigned long long)local[threadIdx.x]);
}

// Nodes at level l = sorted positions with L_i <= l (a running sum of the histogram).
__global__ void level_counts_kernel(const unsigned long long* __restrict__ hist, int depth,
                                    int64_t* __restrict__ level_counts) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int64_t run = 0;
    for (int l = 0; l <= depth; ++l) {
        run += (int64_t)hist[l];
        level_counts[l] = run;
    }
}

__global__ void level_flags_kernel(const uint8_t* __restrict__ split, int64_t count, int level,
                                   uint32_t* __restrict__ flags) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) flags[i] = split[i] <= level ? 1u : 0u;
}

__device__ __forceinline__ int64_t level_offset(const int64_t* level_counts, int level) {
    int64_t off = 0;
    for (int l = 0; l < level; ++l) off += level_counts[l];
    return off;
}

// One level of the flat octree.  rank_cur/rank_prev: exclusive prefix counts
// of the level-l / level-(l-1) node starts over sorted positions.
__global__ void emit_level_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ perm,
                                  const uint8_t* __restrict__ split, int64_t count, int depth, int level,
                                  const int64_t* __restrict__ level_counts,
                                  const uint32_t* __restrict__ rank_cur, const uint32_t* __restrict__ rank_prev,
                                  int64_t* __restrict__ node_depth, int64_t* __restrict__ morton,
                                  int64_t* __restrict__ parent, int64_t* __restrict__ child_start,
                                  int64_t* __restrict__ child_count, int64_t* __restrict__ point_leaf) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int s = split[i];
    const int64_t off = level_offset(level_counts, level);
    if (level == depth) {
        // Every sorted position belongs to the leaf node that its last start opened.
        int64_t leaf_rank = (int64_t)rank_cur[i] + (s <= level ? 1 : 0) - 1;
        point_leaf[perm[i]] = off + leaf_rank;
    }
    if (s > level) return;
    const int64_t node = off + rank_cur[i];
    morton[node] = (int64_t)(keys[i] >> (3 * (depth - level)));
    node_depth[node] = level;
    child_start[node] = -1;
    child_count[node] = 0;
    if (level == 0) {
        parent[node] = -1;
        return;
    }
    const int64_t prev_off = level_offset(level_counts, level - 1);
    const int64_t p = prev_off + (int64_t)rank_prev[i] + (s <= level - 1 ? 1 : 0) - 1;
    parent[node] = p;
    if (s <= level - 1) child_start[p] = node;  // first child of a parent that starts here
    atomicAdd((unsigned long long*)&child_count[p], 1ull);
}

struct OctreeWork {
    uint64_t *keys, *keys_alt;
    uint32_t *vals, *vals_alt;
    uint8_t* split;
    uint32_t *rank_a, *rank_b;
    unsigned long long* hist;
};

static OctreeWork octree_carve(Workspace& w, int64_t count) {
    OctreeWork o;
    o.keys = w.take<uint64_t>(count);
    o.keys_alt = w.take<uint64_t>(count);
    o.vals = w.take<uint32_t>(count);
    o.vals_alt = w.take<uint32_t>(count);
    o.split = w.take<uint8_t>(count);
    o.rank_a = w.take<uint32_t>(count);
    o.rank_b = w.take<uint32_t>(count);
    o.hist = w.take<unsigned long long>(32);
    return o;
}

static size_t octree_ws_bytes(int64_t count) {
    return measure([&](Workspace& w) {
        octree_carve(w, count);
        Workspace a = w;
        radix_carve<uint64_t>(a, count);
        Workspace b = w;
        scan_carve<uint32_t>(b, count);
        w.used = a.used > b.used ? a.used : b.used;
    });
}

static int check_octree_args(int64_t count, int64_t depth) {
    if (count < 1) return fail(PB_ERR_INVALID, "octree: point_count must be >= 1 (got %lld)", (long long)count);
    if (count > 0xFFFFFFFFll) return fail(PB_ERR_INVALID, "octree: point_count must be < 2^32");
    if (depth < 0 || depth > 19) return fail(PB_ERR_INVALID, "octree: depth must be between 0 and 19");
    return PB_OK;
}

}  // namespace pb

using namespace pb;

extern "C" int pb_octree_codes_f64(const double* points, int64_t point_count, int64_t depth, int64_t* codes,
                                   void* stream) {
    if (point_count < 0) return fail(PB_ERR_INVALID, "octree codes: negative point_count");
    if (depth < 0 || depth > 19) return fail(PB_ERR_INVALID, "octree codes: depth must be between 0 and 19");
    if (point_count == 0) return PB_OK;
    if (!points || !codes) return fail(PB_ERR_INVALID, "octree codes: null buffer");
    octree_codes_kernel<<<blocks_for(point_count, 256), 256, 0, (cudaStream_t)stream>>>(points, point_count,
                                                                                        (int)depth, codes);
    PB_CHECK_LAUNCH("octree_codes_kernel");
    return PB_OK;
}

extern "C" size_t pb_octree_workspace_size(int64_t point_count, int64_t depth) {
    (void)depth;
    return octree_ws_bytes(point_count < 1 ? 1 : point_count);
}

extern "C" int pb_octree_count(const double* points, int64_t point_count, int64_t depth, int64_t* level_counts,
                               void* workspace, size_t workspace_bytes, void* stream) {
    PB_TRY(check_octree_args(point_count, depth));
    if (!points || !level_counts) return fail(PB_ERR_INVALID, "octree count: null buffer");
    if (!workspace || workspace_bytes < octree_ws_bytes(point_count))
        return fail(PB_ERR_WORKSPACE, "octree count: workspace needs %zu bytes", octree_ws_bytes(point_count));
    cudaStream_t s = (cudaStream_t)stream;
    Workspace w(workspace, workspace_bytes);
    OctreeWork o = octree_carve(w, point_count);
    const unsigned blocks = blocks_for(point_count, 256);
    leaf_keys_kernel<<<blocks, 256, 0, s>>>(points, point_count, (int)depth, o.keys, o.vals);
    PB_CHECK_LAUNCH("leaf_keys_kernel");
    bool in_alt = false;
    Workspace sort_ws = w;
    PB_TRY(radix_sort_pairs<uint64_t>(o.keys, o.vals, o.keys_alt, o.vals_alt, point_count, (int)(3 * depth), &in_alt,
                                      sort_ws, s));
    const uint64_t* keys = in_alt ? o.keys_alt : o.keys;
    PB_CHECK_CUDA(cudaMemsetAsync(o.hist, 0, 32 * sizeof(unsigned long long), s), "octree hist");
    split_level_kernel<<<blocks, 256, 0, s>>>(keys, point_count, (int)depth, o.split, o.hist);
    PB_CHECK_LAUNCH("split_level_kernel");
    level_counts_kernel<<<1, 32, 0, s>>>(o.hist, (int)depth, level_counts);
    PB_CHECK_LAUNCH("level_counts_kernel");
    return PB_OK;
}

extern "C" int pb_octree_emit(int64_t point_count, int64_t depth, const int64_t* level_counts, int64_t node_count,
                              int64_t* node_depth, int64_t* morton, int64_t* parent, int64_t* child_start,
                              int64_t* child_count, int64_t* point_leaf, void* workspace, size_t workspace_bytes,
                              void* stream) {
    PB_TRY(check_octree_args(point_count, depth));
    if (!level_counts || !node_depth || !morton || !parent || !child_start || !child_count || !point_leaf)
        return fail(PB_ERR_INVALID, "octree emit: null buffer");
    if (node_count < depth + 1) return fail(PB_ERR_INVALID, "octree emit: node_count too small");
    if (!workspace || workspace_bytes < octree_ws_bytes(point_count))
        return fail(PB_ERR_WORKSPACE, "octree emit: workspace needs %zu bytes", octree_ws_bytes(point_count));
    cudaStream_t s = (cudaStream_t)stream;
    Workspace w(workspace, workspace_bytes);
    OctreeWork o = octree_carve(w, point_count);
    const int passes = (int)((3 * depth + 7) / 8);
    const bool in_alt = point_count > 1 && (passes & 1);
    const uint64_t* keys = in_alt ? o.keys_alt : o.keys;
    const uint32_t* perm = in_alt ? o.vals_alt : o.vals;
    const unsigned blocks = blocks_for(point_count, 256);
    uint32_t* prev = o.rank_a;
    uint32_t* cur = o.rank_b;
    for (int level = 0; level <= depth; ++level) {
        level_flags_kernel<<<blocks, 256, 0, s>>>(o.split, point_count, level, cur);
        PB_CHECK_LAUNCH("level_flags_kernel");
        Workspace scan_ws = w;
        PB_TRY(exclusive_scan<uint32_t>(cur, cur, point_count, nullptr, scan_ws, s));
        emit_level_kernel<<<blocks, 256, 0, s>>>(keys, perm, o.split, point_count, (int)depth, level, level_counts, cur,
                                                 prev, node_depth, morton, parent, child_start, child_count,
                                                 point_leaf);
        PB_CHECK_LAUNCH("emit_level_kernel");
        uint32_t* t = prev;
        prev = cur;
        cur = t;
    }
    return PB_OK;
}
