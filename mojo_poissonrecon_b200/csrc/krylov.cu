// FP64 flexible conjugate gradients, FCG(1), around the FP32 V-cycle.
//
// The reference solves A x = b by repeating V-cycles (python/mojo_poissonrecon/
// core.py:274-285).  Used as a preconditioner z = M(r) inside a Krylov loop the
// same V-cycle needs far fewer applications: on the benchmark torus at depth 7
// FCG(1) reaches ||r|| / ||b|| <= 1e-8 in 12 cycles where plain repetition
// needs 27.  Because M is a V-cycle in FP32 (not a fixed symmetric operator),
// the flexible form is used: each direction is A-orthogonalised against the
// previous one only.
//
//   r = b - A x;  repeat:  z = M(r)
//                          p = z - beta p_prev,   beta = (z, q_prev) / (p_prev, q_prev)
//                          q = A p,               alpha = (p, r) / (p, q)
//                          x += alpha p;  r -= alpha q
//
// All vectors are FP64 except z (the FP32 V-cycle's padded output) and r32
// (the FP32 copy of r the next V-cycle reads).  The scalars stay on the device:
// each kernel reads the sums the previous one produced, so an iteration needs
// no host synchronisation; the host reads ||r||^2 only to decide when to stop.
#include "common.cuh"

namespace pb {
namespace fcg {

constexpr int kTX = 64, kTY = 4, kTZ = 16, kThreads = kTX * kTY;

struct Pad {  // padded FP32 layout of the multigrid levels
    int n, P;
    int64_t plane;
    __device__ __forceinline__ int64_t at(int x, int y, int z) const {
        return ((int64_t)(z + 1) * (n + 2) + (y + 1)) * P + (x + 4);
    }
};

__device__ __forceinline__ int lin_tid() { return threadIdx.y * blockDim.x + threadIdx.x; }

// Sums up to 3 values over the block; results valid in linear thread 0.
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

// (z, q_prev) per block.
__global__ void __launch_bounds__(kThreads) dot_zq_kernel(const float* __restrict__ z, Pad g,
                                                          const double* __restrict__ q, double* __restrict__ part) {
    __shared__ double shared[1][32];
    const int n = g.n;
    const int x = blockIdx.x * kTX + threadIdx.x, y = blockIdx.y * kTY + threadIdx.y;
    const int z0 = blockIdx.z * kTZ, z1 = min(n, z0 + kTZ);
    double v[1] = {0.0};
    if (x < n && y < n)
        for (int k = z0; k < z1; ++k)
            v[0] += (double)z[g.at(x, y, k)] * q[((int64_t)k * n + y) * n + x];
    block_sums<1>(v, shared);
    if (lin_tid() == 0) part[block_index()] = v[0];
}

// p = z - beta p_prev (beta from the device sums; p = z on the first step),
// q = A p, and per-block (p, q) and (p, r).
template <bool FIRST>
__global__ void __launch_bounds__(kThreads) direction_kernel(const float* __restrict__ zc, Pad g,
                                                             const double* __restrict__ p_prev,
                                                             const double* __restrict__ scal,
                                                             const double* __restrict__ screen,
                                                             const double* __restrict__ r, double pw,
                                                             double* __restrict__ p, double* __restrict__ q,
                                                             double* __restrict__ part) {
    __shared__ double shared[2][32];
    const int n = g.n;
    const int x = blockIdx.x * kTX + threadIdx.x, y = blockIdx.y * kTY + threadIdx.y;
    const int z0 = blockIdx.z * kTZ, z1 = min(n, z0 + kTZ);
    const double h = (double)(n - 1), h2 = h * h;
    // scal[0] = (z, q_prev); scal[2] still holds (p_prev, q_prev) from the previous step
    const double beta = FIRST ? 0.0 : scal[0] / scal[2];
    const int64_t nn = (int64_t)n * n;
    double v[2] = {0.0, 0.0};
    if (x < n && y < n) {
        const int degxy = (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n);
        for (int k = z0; k < z1; ++k) {
            const int64_t i = (int64_t)k * nn + (int64_t)y * n + x;
            const int64_t c = g.at(x, y, k);
            auto pv = [&](int64_t di, int64_t dc) -> double {
                double val = (double)zc[c + dc];
                if (!FIRST) val -= beta * p_prev[i + di];
                return val;
            };
            double s = 0.0;
            if (x > 0) s += pv(-1, -1);
            if (x + 1 < n) s += pv(1, 1);
            if (y > 0) s += pv(-n, -g.P);
            if (y + 1 < n) s += pv(n, g.P);
            if (k > 0) s += pv(-nn, -g.plane);
            if (k + 1 < n) s += pv(nn, g.plane);
            const int deg = degxy + (k > 0) + (k + 1 < n);
            const double pc = pv(0, 0);
            const double qc = ((double)deg * h2 + pw * screen[i] * h2) * pc - s * h2;
            p[i] = pc;
            q[i] = qc;
            v[0] += pc * qc;
            v[1] += pc * r[i];
        }
    }
    block_sums<2>(v, shared);
    if (lin_tid() == 0) {
        part[2 * block_index()] = v[0];
        part[2 * block_index() + 1] = v[1];
    }
}

// x += alpha p, r -= alpha q (alpha = scal[3] / scal[2]), r32 = (float) r, per-block ||r||^2.
__global__ void __launch_bounds__(kThreads) update_kernel(double* __restrict__ x, double* __restrict__ r,
                                                          const double* __restrict__ p,
                                                          const double* __restrict__ q,
                                                          const double* __restrict__ scal, float* __restrict__ r32,
                                                          Pad g, double* __restrict__ part) {
    __shared__ double shared[1][32];
    const int n = g.n;
    const int xx = blockIdx.x * kTX + threadIdx.x, y = blockIdx.y * kTY + threadIdx.y;
    const int z0 = blockIdx.z * kTZ, z1 = min(n, z0 + kTZ);
    const double alpha = scal[3] / scal[2];  // (p, r) / (p, q)
    double v[1] = {0.0};
    if (xx < n && y < n)
        for (int k = z0; k < z1; ++k) {
            const int64_t i = ((int64_t)k * n + y) * n + xx;
            x[i] += alpha * p[i];
            const double rn = r[i] - alpha * q[i];
            r[i] = rn;
            r32[g.at(xx, y, k)] = (float)rn;
            v[0] += rn * rn;
        }
    block_sums<1>(v, shared);
    if (lin_tid() == 0) part[block_index()] = v[0];
}

// out[k] = sum over blocks of part[stride * b + k], k < count (fixed order).
__global__ void finish_kernel(const double* __restrict__ part, int blocks, int stride, int count,
                              double* __restrict__ out) {
    __shared__ double shared[3][32];
    double v[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < blocks; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (k < count) v[k] += part[(int64_t)stride * b + k];
    block_sums<3>(v, shared);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (k < count) out[k] = v[k];
}

// ---- graph-friendly form: one iteration touches the same buffers every time ----
// p = first ? z : z - beta p, in place (pointwise), beta = scal[0] / scal[2];
// flags[0] != 0 marks the first step.
__global__ void __launch_bounds__(kThreads) newdir_kernel(const float* __restrict__ zc, Pad g,
                                                          double* __restrict__ p, const double* __restrict__ scal,
                                                          const int* __restrict__ flags) {
    const int n = g.n;
    const int x = blockIdx.x * kTX + threadIdx.x, y = blockIdx.y * kTY + threadIdx.y;
    if (x >= n || y >= n) return;
    const int z0 = blockIdx.z * kTZ, z1 = min(n, z0 + kTZ);
    const bool first = flags[0] != 0;
    const double beta = first ? 0.0 : scal[0] / scal[2];
    for (int k = z0; k < z1; ++k) {
        const int64_t i = ((int64_t)k * n + y) * n + x;
        const double zv = (double)zc[g.at(x, y, k)];
        p[i] = first ? zv : zv - beta * p[i];
    }
}

// q = A p and per-block (p, q), (p, r).
__global__ void __launch_bounds__(kThreads) matvec_kernel(const double* __restrict__ p, int n,
                                                          const double* __restrict__ screen,
                                                          const double* __restrict__ r, double pw,
                                                          double* __restrict__ q, double* __restrict__ part) {
    __shared__ double shared[2][32];
    const int x = blockIdx.x * kTX + threadIdx.x, y = blockIdx.y * kTY + threadIdx.y;
    const int z0 = blockIdx.z * kTZ, z1 = min(n, z0 + kTZ);
    const double h = (double)(n - 1), h2 = h * h;
    const int64_t nn = (int64_t)n * n;
    double v[2] = {0.0, 0.0};
    if (x < n && y < n) {
        const int degxy = (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n);
        for (int k = z0; k < z1; ++k) {
            const int64_t i = (int64_t)k * nn + (int64_t)y * n + x;
            double s = 0.0;
            if (x > 0) s += p[i - 1];
            if (x + 1 < n) s += p[i + 1];
            if (y > 0) s += p[i - n];
            if (y + 1 < n) s += p[i + n];
            if (k > 0) s += p[i - nn];
            if (k + 1 < n) s += p[i + nn];
            const int deg = degxy + (k > 0) + (k + 1 < n);
            const double pc = p[i];
            const double qc = ((double)deg * h2 + pw * screen[i] * h2) * pc - s * h2;
            q[i] = qc;
            v[0] += pc * qc;
            v[1] += pc * r[i];
        }
    }
    block_sums<2>(v, shared);
    if (lin_tid() == 0) {
        part[2 * block_index()] = v[0];
        part[2 * block_index() + 1] = v[1];
    }
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

static dim3 grid_of(int n) { return dim3((n + kTX - 1) / kTX, (n + kTY - 1) / kTY, (n + kTZ - 1) / kTZ); }
static unsigned blocks_of(int n) {
    const dim3 g = grid_of(n);
    return g.x * g.y * g.z;
}
static Pad pad_of(int n) {
    const int P = ((n + 5) + 7) & ~7;
    return Pad{n, P, (int64_t)(n + 2) * P};
}

}  // namespace fcg
}  // namespace pb

using namespace pb;

extern "C" size_t pb_fcg_workspace_size(int64_t n) {
    if (n < 2) n = 2;
    return (size_t)fcg::blocks_of((int)n) * 2 * sizeof(double) + 256;
}

// One FCG(1) step after the preconditioner produced z (padded FP32):
//   scal (device, 5 doubles): [0] (z, q_prev)  [2] (p, q)  [3] (p, r)
//                             [4] ||r||^2 after the step  ([1] unused)
// p_prev -> p and q are dense FP64; on the first step p_prev may be NULL.
// Writes x, r (FP64), r32 (padded FP32 copy of r) and scal[0..4]; p_prev and p
// must differ (the direction is formed from neighbours of p_prev).
extern "C" int pb_fcg_step_f64(const float* z, const double* p_prev, double* p, double* q, double* x, double* r,
                               float* r32, const double* screen, int64_t n, double point_weight, double* scal,
                               int64_t first, void* workspace, size_t workspace_bytes, void* stream) {
    using namespace pb::fcg;
    if (n < 2 || n > 4097 || !z || !p || !q || !x || !r || !r32 || !screen || !scal || (!first && !p_prev))
        return fail(PB_ERR_INVALID, "fcg step: bad args");
    if (p == p_prev) return fail(PB_ERR_INVALID, "fcg step: p must not alias p_prev");
    const unsigned blocks = blocks_of((int)n);
    if (!workspace || workspace_bytes < (size_t)blocks * 2 * sizeof(double))
        return fail(PB_ERR_WORKSPACE, "fcg step: workspace needs %zu bytes", pb_fcg_workspace_size(n));
    double* part = (double*)workspace;
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid = grid_of((int)n), block(kTX, kTY);
    const Pad g = pad_of((int)n);
    if (!first) {
        dot_zq_kernel<<<grid, block, 0, s>>>(z, g, q, part);  // q still holds q_prev here
        PB_CHECK_LAUNCH("fcg dot_zq_kernel");
        finish_kernel<<<1, 1024, 0, s>>>(part, (int)blocks, 1, 1, scal + 0);
        PB_CHECK_LAUNCH("fcg finish_kernel");
        direction_kernel<false><<<grid, block, 0, s>>>(z, g, p_prev, scal, screen, r, point_weight, p, q, part);
    } else {
        direction_kernel<true><<<grid, block, 0, s>>>(z, g, nullptr, scal, screen, r, point_weight, p, q, part);
    }
    PB_CHECK_LAUNCH("fcg direction_kernel");
    finish_kernel<<<1, 1024, 0, s>>>(part, (int)blocks, 2, 2, scal + 2);
    PB_CHECK_LAUNCH("fcg finish_kernel");
    update_kernel<<<grid, block, 0, s>>>(x, r, p, q, scal, r32, g, part);
    PB_CHECK_LAUNCH("fcg update_kernel");
    finish_kernel<<<1, 1024, 0, s>>>(part, (int)blocks, 1, 1, scal + 4);
    PB_CHECK_LAUNCH("fcg finish_kernel");
    return PB_OK;
}

// Graph-friendly FCG(1) step: the direction is updated in place (pointwise),
// then q = A p, alpha, and the x / r update; flags[0] selects the first step.
// Every call touches the same buffers, so the step can be captured in a graph.
extern "C" int pb_fcg_step_inplace_f64(const float* z, double* p, double* q, double* x, double* r, float* r32,
                                       const double* screen, int64_t n, double point_weight, double* scal,
                                       const int* flags, void* workspace, size_t workspace_bytes, void* stream) {
    using namespace pb::fcg;
    if (n < 2 || n > 4097 || !z || !p || !q || !x || !r || !r32 || !screen || !scal || !flags)
        return fail(PB_ERR_INVALID, "fcg step: bad args");
    const unsigned blocks = blocks_of((int)n);
    if (!workspace || workspace_bytes < (size_t)blocks * 2 * sizeof(double))
        return fail(PB_ERR_WORKSPACE, "fcg step: workspace needs %zu bytes", pb_fcg_workspace_size(n));
    double* part = (double*)workspace;
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid = grid_of((int)n), block(kTX, kTY);
    const Pad g = pad_of((int)n);
    dot_zq_kernel<<<grid, block, 0, s>>>(z, g, q, part);  // q holds q_prev (ignored on the first step)
    PB_CHECK_LAUNCH("fcg dot_zq_kernel");
    finish_kernel<<<1, 1024, 0, s>>>(part, (int)blocks, 1, 1, scal + 0);
    PB_CHECK_LAUNCH("fcg finish_kernel");
    newdir_kernel<<<grid, block, 0, s>>>(z, g, p, scal, flags);
    PB_CHECK_LAUNCH("fcg newdir_kernel");
    matvec_kernel<<<grid, block, 0, s>>>(p, (int)n, screen, r, point_weight, q, part);
    PB_CHECK_LAUNCH("fcg matvec_kernel");
    finish_kernel<<<1, 1024, 0, s>>>(part, (int)blocks, 2, 2, scal + 2);
    PB_CHECK_LAUNCH("fcg finish_kernel");
    update_kernel<<<grid, block, 0, s>>>(x, r, p, q, scal, r32, g, part);
    PB_CHECK_LAUNCH("fcg update_kernel");
    finish_kernel<<<1, 1024, 0, s>>>(part, (int)blocks, 1, 1, scal + 4);
    PB_CHECK_LAUNCH("fcg finish_kernel");
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
