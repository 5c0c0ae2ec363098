// Two-pass trilinear splat, bit-identical to the serial reference.
//
// Reference: src/capi.mojo:104-224.  The reference adds each sample's eight
// corner weights into the grids in point order; floating-point addition is not
// associative, so atomics would change the last bits.  Here every (point,
// corner) pair becomes a record keyed by its grid node; a stable radix sort
// groups the records by node while keeping point order inside each group; one
// thread then adds a node's contributions in that order, starting from the
// node's current value — the same additions, in the same order, as the
// reference.  Pass 2 reuses the sorted order (both passes address the same
// eight nodes per sample).
//
// Compiled with -fmad=false: every product and sum rounds as written.
#include "radix_sort.cuh"

namespace pb {

__device__ __forceinline__ double norm3(double x, double y, double z) {  // capi.mojo:51-59
    double scale = fmax(fabs(x), fmax(fabs(y), fabs(z)));
    if (scale == 0.0) return 0.0;
    double sx = x / scale, sy = y / scale, sz = z / scale;
    return scale * sqrt(sx * sx + sy * sy + sz * sz);
}

__device__ __forceinline__ double clamp01(double v) {  // min(max(v, 0), 1)
    double m = v > 0.0 ? v : 0.0;
    return m < 1.0 ? m : 1.0;
}

// Pass-1 base cell and fractions (capi.mojo:139-162).
__device__ __forceinline__ void pass1_cell(double p, int64_t res, int64_t& i, double& f) {
    double g = p * (double)res;
    i = (int64_t)g;
    if (i < 0) i = 0;
    if (i >= res) {
        i = res - 1;
        g = (double)res;
    }
    f = g - (double)i;
}

// Pass-2 / iso-value base cell and fractions (capi.mojo:187-195, :771-779).
__device__ __forceinline__ void pass2_cell(double p, int64_t res, int64_t& i, double& f) {
    double g = p * (double)res;
    int64_t t = (int64_t)g;
    i = t < 0 ? 0 : (t > res - 1 ? res - 1 : t);
    f = clamp01(g - (double)i);
}

// Records: key = grid node (or the sentinel n^3 for a rejected sample), value =
// point*8 + corner, corner = dz*4 + dy*2 + dx; weight[record] = pass-1 weight.
// One thread per record (the eight threads of a point repeat its cell
// arithmetic), so each array is written with coalesced stores.
__global__ void splat_records_kernel(const double* __restrict__ points, const double* __restrict__ normals,
                                     int64_t count, int64_t n, int confidence, uint32_t* __restrict__ keys,
                                     uint32_t* __restrict__ vals, double* __restrict__ weight,
                                     unsigned long long* __restrict__ accepted) {
    __shared__ unsigned int block_accepted;
    if (threadIdx.x == 0) block_accepted = 0;
    __syncthreads();
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < 8 * count) {
        const int64_t p = r >> 3;
        const int c = (int)(r & 7), dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
        const int64_t res = n - 1;
        double nx = normals[3 * p], ny = normals[3 * p + 1], nz = normals[3 * p + 2];
        double length = norm3(nx, ny, nz);
        vals[r] = (uint32_t)r;
        if (length <= 0.0) {  // capi.mojo:132-133
            keys[r] = (uint32_t)(n * n * n);
            weight[r] = 0.0;
        } else {
            double sw = confidence ? length : 1.0;
            int64_t ix, iy, iz;
            double fx, fy, fz;
            pass1_cell(points[3 * p], res, ix, fx);
            pass1_cell(points[3 * p + 1], res, iy, fy);
            pass1_cell(points[3 * p + 2], res, iz, fz);
            const double wz = dz == 1 ? fz : 1.0 - fz;
            const double wy = dy == 1 ? fy : 1.0 - fy;
            const double wx = dx == 1 ? fx : 1.0 - fx;
            keys[r] = (uint32_t)grid_index(ix + dx, iy + dy, iz + dz, n);
            weight[r] = wx * wy * wz * sw;
            if (c == 0) atomicAdd(&block_accepted, 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && block_accepted) atomicAdd(accepted, (unsigned long long)block_accepted);
}

// Runs of records with the same node are consumed kRun at a time: the keys
// of the next kRun records are loaded together and the run's length within
// them counted, then their values and gathered weights are loaded together,
// and only then added, one after another in record order.  The additions are
// exactly the serial ones; only the loads overlap.
constexpr int kRun = 8;

__device__ __forceinline__ int run_length(const uint32_t* __restrict__ keys, int64_t k, int64_t records,
                                          uint32_t node) {
    uint32_t kk[kRun];
#pragma unroll
    for (int t = 0; t < kRun; ++t) kk[t] = k + t < records ? keys[k + t] : node + 1;
    int m = 0;
    bool run = true;
#pragma unroll
    for (int t = 0; t < kRun; ++t) {
        run = run && kk[t] == node;
        m += run;
    }
    return m;
}

// Pass 1 (capi.mojo:171-172): density += 2w, screen += w, per node in point order.
// The gathers of a run's values (weight[vals[k]], the sample's unit normal) are
// done first for every record at once, one thread per record, into arrays in
// sorted record order (gather_weights_kernel, gather_vectors_kernel); a run's
// head then reads its values contiguously.  Products are rounded where the
// serial loop rounds them, so the sums are unchanged bit for bit.
__global__ void gather_weights_kernel(const uint32_t* __restrict__ vals, int64_t records,
                                      const double* __restrict__ weight, double* __restrict__ out) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < records) out[k] = weight[vals[k]];
}

// (u_x w, u_y w, u_z w) of each record, w its vector weight, u its sample's unit normal.
__global__ void gather_vectors_kernel(const uint32_t* __restrict__ vals, int64_t records,
                                      const double* __restrict__ weight, const double* __restrict__ unit_normals,
                                      double* __restrict__ px, double* __restrict__ py, double* __restrict__ pz) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= records) return;
    const uint32_t r = vals[k];
    const double vw = weight[r];
    const double* u = unit_normals + 3 * (int64_t)(r >> 3);
    px[k] = u[0] * vw;
    py[k] = u[1] * vw;
    pz[k] = u[2] * vw;
}

// Run heads: the first record of each node's run (sentinel runs excluded),
// compacted in record order so the run sums below take one thread per run
// with full warps (one thread per record left ~2 of 32 lanes busy).
__global__ void run_head_flags_kernel(const uint32_t* __restrict__ keys, int64_t records, uint32_t sentinel,
                                      uint32_t* __restrict__ flag) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= records) return;
    const uint32_t node = keys[j];
    flag[j] = node != sentinel && (j == 0 || keys[j - 1] != node);
}

__global__ void run_heads_kernel(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ rank,
                                 int64_t records, uint32_t* __restrict__ heads) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < records && flag[j]) heads[rank[j]] = (uint32_t)j;
}

__global__ void splat_density_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ heads,
                                     const uint32_t* __restrict__ head_count, int64_t records,
                                     const double* __restrict__ gathered, double* __restrict__ density,
                                     double* __restrict__ screen) {
    const uint32_t runs = *head_count;
    for (uint32_t hd = blockIdx.x * blockDim.x + threadIdx.x; hd < runs; hd += gridDim.x * blockDim.x) {
        const int64_t j = heads[hd];
        const uint32_t node = keys[j];
        double d = density[node], s = screen[node];
        for (int64_t k = j;; k += kRun) {
            const int m = run_length(keys, k, records, node);
            double w[kRun];
#pragma unroll
            for (int t = 0; t < kRun; ++t) w[t] = t < m ? gathered[k + t] : 0.0;
#pragma unroll
            for (int t = 0; t < kRun; ++t)
                if (t < m) {
                    d += 2.0 * w[t];
                    s += w[t];
                }
            if (m < kRun) break;
        }
        density[node] = d;
        screen[node] = s;
    }
}

// Pass 2, per sample (capi.mojo:176-209): local density from the pass-1 grid,
// the density factor, and per-record vector weights w * res / factor.
__global__ void splat_vector_weights_kernel(const double* __restrict__ points, const double* __restrict__ normals,
                                            int64_t count, int64_t n, int confidence, double samples_per_node,
                                            const double* __restrict__ density, double* __restrict__ weight,
                                            double* __restrict__ unit_normals) {
    // each warp's 32 x 8 weights go through shared memory so the stores are
    // contiguous; records of points that set none keep their pass-1 weight
    __shared__ double staged[256 / 32][32 * 8];
    __shared__ unsigned char written[256 / 32][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    written[warp][lane] = 0;
    bool active = p < count;
    double nx = 0.0, ny = 0.0, nz = 0.0, length = 0.0;
    if (active) {
        nx = normals[3 * p];
        ny = normals[3 * p + 1];
        nz = normals[3 * p + 2];
        length = norm3(nx, ny, nz);
        active = length > 0.0;  // capi.mojo:181-182
    }
    if (active) {
        const int64_t res = n - 1;
        double sw = confidence ? length : 1.0;
        unit_normals[3 * p] = nx / length;
        unit_normals[3 * p + 1] = ny / length;
        unit_normals[3 * p + 2] = nz / length;
        int64_t ix, iy, iz;
        double fx, fy, fz;
        pass2_cell(points[3 * p], res, ix, fx);
        pass2_cell(points[3 * p + 1], res, iy, fy);
        pass2_cell(points[3 * p + 2], res, iz, fz);
        double local = 0.0;
        for (int dz = 0; dz < 2; ++dz) {
            double wz = dz == 1 ? fz : 1.0 - fz;
            for (int dy = 0; dy < 2; ++dy) {
                double wy = dy == 1 ? fy : 1.0 - fy;
                for (int dx = 0; dx < 2; ++dx) {
                    double wx = dx == 1 ? fx : 1.0 - fx;
                    local += density[grid_index(ix + dx, iy + dy, iz + dz, n)] * wx * wy * wz;
                }
            }
        }
        double q = local / samples_per_node;
        double factor = 1.0 > q ? 1.0 : q;
        for (int dz = 0; dz < 2; ++dz) {
            double wz = dz == 1 ? fz : 1.0 - fz;
            for (int dy = 0; dy < 2; ++dy) {
                double wy = dy == 1 ? fy : 1.0 - fy;
                for (int dx = 0; dx < 2; ++dx) {
                    double wx = dx == 1 ? fx : 1.0 - fx;
                    double w = wx * wy * wz * sw;
                    staged[warp][lane * 8 + dz * 4 + dy * 2 + dx] = w * (double)res / factor;
                }
            }
        }
        written[warp][lane] = 1;
    }
    __syncwarp();
    const int64_t r0 = ((int64_t)blockIdx.x * blockDim.x + warp * 32) * 8;  // the warp's first record
    for (int e = lane; e < 32 * 8; e += 32)
        if (written[warp][e >> 3]) weight[r0 + e] = staged[warp][e];
}

// Pass 2 (capi.mojo:221-223): V -= n_hat * vector_weight, per node in point order.
__global__ void splat_vector_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ heads,
                                    const uint32_t* __restrict__ head_count, int64_t records,
                                    const double* __restrict__ px, const double* __restrict__ py,
                                    const double* __restrict__ pz, double* __restrict__ vx,
                                    double* __restrict__ vy, double* __restrict__ vz) {
    const uint32_t runs = *head_count;
    for (uint32_t hd = blockIdx.x * blockDim.x + threadIdx.x; hd < runs; hd += gridDim.x * blockDim.x) {
        const int64_t j = heads[hd];
        const uint32_t node = keys[j];
        double ax = vx[node], ay = vy[node], az = vz[node];
        for (int64_t k = j;; k += kRun) {
            const int m = run_length(keys, k, records, node);
            double qx[kRun], qy[kRun], qz[kRun];
#pragma unroll
            for (int t = 0; t < kRun; ++t) {
                qx[t] = t < m ? px[k + t] : 0.0;
                qy[t] = t < m ? py[k + t] : 0.0;
                qz[t] = t < m ? pz[k + t] : 0.0;
            }
#pragma unroll
            for (int t = 0; t < kRun; ++t)
                if (t < m) {  // V -= n_hat * w: the product was rounded by the gather, as here
                    ax -= qx[t];
                    ay -= qy[t];
                    az -= qz[t];
                }
            if (m < kRun) break;
        }
        vx[node] = ax;
        vy[node] = ay;
        vz[node] = az;
    }
}

// ---- auxiliary attributes (upstream PoissonRecon's colour interpolation) --------
// Each sample's k attributes are splatted with its pass-1 weights w (the
// screening weights), per node in record order: planes 0 .. k-1 of `grids`
// hold sum w a_c, plane k holds sum w.  One thread per run, one channel at a
// time (deterministic sums).
__global__ void attribute_runs_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                                      const uint32_t* __restrict__ heads, const uint32_t* __restrict__ head_count,
                                      int64_t records, const double* __restrict__ weight,
                                      const double* __restrict__ attributes, int channels, int64_t plane,
                                      double* __restrict__ grids) {
    const uint32_t runs = *head_count;
    for (uint32_t hd = blockIdx.x * blockDim.x + threadIdx.x; hd < runs; hd += gridDim.x * blockDim.x) {
        const int64_t j = heads[hd];
        const uint32_t node = keys[j];
        for (int c = 0; c <= channels; ++c) {
            double sum = 0.0;
            for (int64_t k = j; k < records && keys[k] == node; ++k) {
                const uint32_t r = vals[k];
                const double w = weight[r];
                sum += c < channels ? w * attributes[(int64_t)(r >> 3) * channels + c] : w;
            }
            grids[c * plane + node] = sum;
        }
    }
}

// Per vertex (world coordinates, mapped to the unit cube by `map` = (min x, y,
// z, width)): the ratio of the trilinear interpolants of sum w a_c and sum w
// over its cell (zero where no sample's weight reaches the cell).
__global__ void sample_attributes_kernel(const double* __restrict__ vertices, int64_t count,
                                         const double* __restrict__ map, int64_t n, const double* __restrict__ grids,
                                         int channels, double* __restrict__ out) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= count) return;
    const int64_t res = n - 1, plane = n * n * n;
    int64_t ix[3];
    double f[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double u = (vertices[3 * v + a] - map[a]) / map[3];
        pass2_cell(u, res, ix[a], f[a]);
    }
    double den = 0.0;
    for (int c = 0; c <= channels; ++c) {
        double num = 0.0;
        for (int dz = 0; dz < 2; ++dz) {
            const double wz = dz == 1 ? f[2] : 1.0 - f[2];
            for (int dy = 0; dy < 2; ++dy) {
                const double wy = dy == 1 ? f[1] : 1.0 - f[1];
                for (int dx = 0; dx < 2; ++dx) {
                    const double wx = dx == 1 ? f[0] : 1.0 - f[0];
                    num += grids[c * plane + grid_index(ix[0] + dx, ix[1] + dy, ix[2] + dz, n)] * wx * wy * wz;
                }
            }
        }
        if (c == channels) den = num;
        else out[v * channels + c] = num;
    }
    for (int c = 0; c < channels; ++c) out[v * channels + c] = den > 0.0 ? out[v * channels + c] / den : 0.0;
}

__global__ void store_count_kernel(const unsigned long long* __restrict__ src, int64_t* __restrict__ dst) {
    *dst = (int64_t)*src;
}

struct SplatWork {
    uint32_t *keys, *keys_alt, *vals, *vals_alt;
    double* weight;
    double *gx, *gy, *gz;  // gathered values in sorted record order
    uint32_t *flag, *rank, *heads, *head_count;  // run heads in record order
    double* unit_normals;
    unsigned long long* accepted;
};

static SplatWork splat_carve(Workspace& w, int64_t count) {
    SplatWork o;
    const int64_t records = count * 8;
    o.keys = w.take<uint32_t>(records);
    o.keys_alt = w.take<uint32_t>(records);
    o.vals = w.take<uint32_t>(records);
    o.vals_alt = w.take<uint32_t>(records);
    o.weight = w.take<double>(records);
    o.gx = w.take<double>(records);
    o.gy = w.take<double>(records);
    o.gz = w.take<double>(records);
    o.flag = w.take<uint32_t>(records);
    o.rank = w.take<uint32_t>(records);
    o.heads = w.take<uint32_t>(records);
    o.head_count = w.take<uint32_t>(1);
    o.unit_normals = w.take<double>(count * 3);
    o.accepted = w.take<unsigned long long>(1);
    return o;
}

static size_t splat_ws_bytes(int64_t count) {
    return measure([&](Workspace& w) {
        splat_carve(w, count);
        radix_carve<uint32_t>(w, count * 8);
        scan_carve<uint32_t>(w, count * 8);
    });
}

static int bit_width(uint64_t v) {
    int b = 0;
    while (v) {
        ++b;
        v >>= 1;
    }
    return b;
}

}  // namespace pb

using namespace pb;

extern "C" size_t pb_splat_workspace_size(int64_t point_count, int64_t n) {
    (void)n;
    return splat_ws_bytes(point_count < 1 ? 1 : point_count);
}

extern "C" int pb_splat_f64(const double* points, const double* normals, int64_t point_count, int64_t n,
                            int64_t confidence, double* density, double* vx, double* vy, double* vz, double* screen,
                            double samples_per_node, int64_t* accepted, void* workspace, size_t workspace_bytes,
                            void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (n < 2) return fail(PB_ERR_INVALID, "splat: n must be >= 2");
    if (n * n * n >= (int64_t)0x7FFFFFFF) return fail(PB_ERR_INVALID, "splat: n^3 must be < 2^31");
    if (point_count < 0 || point_count * 8 >= (int64_t)0xFFFFFFFFll)
        return fail(PB_ERR_INVALID, "splat: point_count must be in [0, 2^29)");
    if (!accepted || !density || !vx || !vy || !vz || !screen) return fail(PB_ERR_INVALID, "splat: null buffer");
    if (point_count == 0) {
        PB_CHECK_CUDA(cudaMemsetAsync(accepted, 0, sizeof(int64_t), s), "splat accepted");
        return PB_OK;
    }
    if (!points || !normals) return fail(PB_ERR_INVALID, "splat: null points/normals");
    const size_t need = splat_ws_bytes(point_count);
    if (!workspace || workspace_bytes < need) return fail(PB_ERR_WORKSPACE, "splat: workspace needs %zu bytes", need);
    Workspace w(workspace, workspace_bytes);
    SplatWork o = splat_carve(w, point_count);
    const int64_t records = point_count * 8;
    const uint32_t sentinel = (uint32_t)(n * n * n);
    PB_CHECK_CUDA(cudaMemsetAsync(o.accepted, 0, sizeof(unsigned long long), s), "splat accepted");
    splat_records_kernel<<<blocks_for(8 * point_count, 256), 256, 0, s>>>(points, normals, point_count, n,
                                                                          (int)confidence, o.keys, o.vals, o.weight,
                                                                          o.accepted);
    PB_CHECK_LAUNCH("splat_records_kernel");
    bool in_alt = false;
    PB_TRY(radix_sort_pairs<uint32_t>(o.keys, o.vals, o.keys_alt, o.vals_alt, records, bit_width(sentinel), &in_alt,
                                      w, s));
    const uint32_t* keys = in_alt ? o.keys_alt : o.keys;
    const uint32_t* vals = in_alt ? o.vals_alt : o.vals;
    run_head_flags_kernel<<<blocks_for(records, 256), 256, 0, s>>>(keys, records, sentinel, o.flag);
    PB_CHECK_LAUNCH("run_head_flags_kernel");
    PB_TRY(exclusive_scan<uint32_t>(o.flag, o.rank, records, o.head_count, w, s));
    run_heads_kernel<<<blocks_for(records, 256), 256, 0, s>>>(o.flag, o.rank, records, o.heads);
    PB_CHECK_LAUNCH("run_heads_kernel");
    const unsigned run_blocks = 8 * kSMs;  // grid-stride over the runs (their count stays on the device)
    gather_weights_kernel<<<blocks_for(records, 256), 256, 0, s>>>(vals, records, o.weight, o.gx);
    PB_CHECK_LAUNCH("gather_weights_kernel");
    splat_density_kernel<<<run_blocks, 256, 0, s>>>(keys, o.heads, o.head_count, records, o.gx, density, screen);
    PB_CHECK_LAUNCH("splat_density_kernel");
    splat_vector_weights_kernel<<<blocks_for(point_count, 256), 256, 0, s>>>(
        points, normals, point_count, n, (int)confidence, samples_per_node, density, o.weight, o.unit_normals);
    PB_CHECK_LAUNCH("splat_vector_weights_kernel");
    gather_vectors_kernel<<<blocks_for(records, 256), 256, 0, s>>>(vals, records, o.weight, o.unit_normals, o.gx,
                                                                    o.gy, o.gz);
    PB_CHECK_LAUNCH("gather_vectors_kernel");
    splat_vector_kernel<<<run_blocks, 256, 0, s>>>(keys, o.heads, o.head_count, records, o.gx, o.gy, o.gz, vx, vy,
                                                    vz);
    PB_CHECK_LAUNCH("splat_vector_kernel");
    store_count_kernel<<<1, 1, 0, s>>>(o.accepted, accepted);
    PB_CHECK_LAUNCH("store_count_kernel");
    return PB_OK;
}

namespace pb {

struct AttrWork {
    uint32_t *keys, *keys_alt, *vals, *vals_alt, *flag, *rank, *heads, *head_count;
    double* weight;
    unsigned long long* accepted;
};

static AttrWork attr_carve(Workspace& w, int64_t count) {
    AttrWork o;
    const int64_t records = count * 8;
    o.keys = w.take<uint32_t>(records);
    o.keys_alt = w.take<uint32_t>(records);
    o.vals = w.take<uint32_t>(records);
    o.vals_alt = w.take<uint32_t>(records);
    o.flag = w.take<uint32_t>(records);
    o.rank = w.take<uint32_t>(records);
    o.heads = w.take<uint32_t>(records);
    o.head_count = w.take<uint32_t>(1);
    o.weight = w.take<double>(records);
    o.accepted = w.take<unsigned long long>(1);
    return o;
}

static size_t attr_ws_bytes(int64_t count) {
    return measure([&](Workspace& w) {
        attr_carve(w, count);
        radix_carve<uint32_t>(w, count * 8);
        scan_carve<uint32_t>(w, count * 8);
    });
}

}  // namespace pb

extern "C" size_t pb_splat_attributes_workspace_size(int64_t point_count) {
    return attr_ws_bytes(point_count < 1 ? 1 : point_count);
}

// Auxiliary attributes of unit-cube samples (points, normals as for
// pb_splat_f64; attributes: point_count x channels, row-major): grids (channels
// + 1 planes of n^3, overwritten) get sum w a_c per node and, in the last
// plane, sum w, with w the samples' pass-1 weights, summed in sample order.
extern "C" int pb_splat_attributes_f64(const double* points, const double* normals, int64_t point_count, int64_t n,
                                       int64_t confidence, const double* attributes, int64_t channels,
                                       double* grids, void* workspace, size_t workspace_bytes, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (n < 2 || n * n * n >= (int64_t)0x7FFFFFFF) return fail(PB_ERR_INVALID, "splat attributes: bad n");
    if (point_count < 0 || point_count * 8 >= (int64_t)0xFFFFFFFFll || channels < 1 || channels > 64 || !grids)
        return fail(PB_ERR_INVALID, "splat attributes: bad sizes");
    PB_CHECK_CUDA(cudaMemsetAsync(grids, 0, sizeof(double) * (size_t)(channels + 1) * (size_t)(n * n * n), s),
                  "splat attributes zero");
    if (point_count == 0) return PB_OK;
    if (!points || !normals || !attributes) return fail(PB_ERR_INVALID, "splat attributes: null input");
    const size_t need = attr_ws_bytes(point_count);
    if (!workspace || workspace_bytes < need)
        return fail(PB_ERR_WORKSPACE, "splat attributes: workspace needs %zu bytes", need);
    Workspace w(workspace, workspace_bytes);
    AttrWork o = attr_carve(w, point_count);
    const int64_t records = point_count * 8;
    const uint32_t sentinel = (uint32_t)(n * n * n);
    PB_CHECK_CUDA(cudaMemsetAsync(o.accepted, 0, sizeof(unsigned long long), s), "splat attributes accepted");
    splat_records_kernel<<<blocks_for(records, 256), 256, 0, s>>>(points, normals, point_count, n, (int)confidence,
                                                                  o.keys, o.vals, o.weight, o.accepted);
    PB_CHECK_LAUNCH("splat_records_kernel");
    bool in_alt = false;
    PB_TRY(radix_sort_pairs<uint32_t>(o.keys, o.vals, o.keys_alt, o.vals_alt, records, bit_width(sentinel), &in_alt,
                                      w, s));
    const uint32_t* keys = in_alt ? o.keys_alt : o.keys;
    const uint32_t* vals = in_alt ? o.vals_alt : o.vals;
    run_head_flags_kernel<<<blocks_for(records, 256), 256, 0, s>>>(keys, records, sentinel, o.flag);
    PB_CHECK_LAUNCH("run_head_flags_kernel");
    PB_TRY(exclusive_scan<uint32_t>(o.flag, o.rank, records, o.head_count, w, s));
    run_heads_kernel<<<blocks_for(records, 256), 256, 0, s>>>(o.flag, o.rank, records, o.heads);
    PB_CHECK_LAUNCH("run_heads_kernel");
    attribute_runs_kernel<<<8 * kSMs, 256, 0, s>>>(keys, vals, o.heads, o.head_count, records, o.weight, attributes,
                                                   (int)channels, n * n * n, grids);
    PB_CHECK_LAUNCH("attribute_runs_kernel");
    return PB_OK;
}

// Attribute values at mesh vertices (world coordinates; map = the (min x, y, z,
// width) that took the samples to the unit cube): out (vertex_count x
// channels) from the grids of pb_splat_attributes_f64.
extern "C" int pb_sample_attributes_f64(const double* vertices, int64_t vertex_count, const double* map, int64_t n,
                                        const double* grids, int64_t channels, double* out, void* stream) {
    if (n < 2 || vertex_count < 0 || channels < 1 || channels > 64 || !map || !grids ||
        (vertex_count && (!vertices || !out)))
        return fail(PB_ERR_INVALID, "sample attributes: bad args");
    if (!vertex_count) return PB_OK;
    sample_attributes_kernel<<<blocks_for(vertex_count, 256), 256, 0, (cudaStream_t)stream>>>(
        vertices, vertex_count, map, n, grids, (int)channels, out);
    PB_CHECK_LAUNCH("sample_attributes_kernel");
    return PB_OK;
}
