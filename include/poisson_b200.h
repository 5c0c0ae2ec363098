/*
 * poisson_b200 — C ABI of the B200 (sm_100a) screened-Poisson reconstruction kernels.
 *
 * Drop-in boundary for mojo-poissonrecon's native library.  The reference
 * binds eleven `mpr_*` symbols through ctypes (python/mojo_poissonrecon/
 * _lib.py:20-32) over caller-owned NumPy buffers.  Every function here keeps
 * the argument order and meaning of the symbol it replaces, with four changes
 * that a GPU boundary needs:
 *
 *   - buffers are DEVICE pointers (e.g. torch.Tensor.data_ptr()), C-contiguous,
 *     [z][y][x] row-major grids of side n (index (z*n + y)*n + x);
 *   - each call is asynchronous on the given cudaStream_t (passed as void*;
 *     NULL = the legacy default stream) and returns an int status (PB_OK = 0);
 *   - values the reference returns (accepted count, residual norm, iso-value,
 *     vertex/face counts) are written to a DEVICE int64/double the caller
 *     passes, so no call synchronises the host;
 *   - functions that need scratch take a caller-owned device workspace whose
 *     size the matching *_workspace_size() reports.  Like the reference
 *     (README.md:84-95) the library never allocates or retains memory.
 *
 * Errors: a non-zero status leaves a message in pb_last_error() (thread-local).
 * Arguments are validated on the host before any launch (PB_ERR_INVALID).
 */
#ifndef POISSON_B200_H
#define POISSON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PB_OK = 0,
    PB_ERR_INVALID = 1,   /* bad size, null pointer, unsupported argument */
    PB_ERR_CUDA = 2,      /* a CUDA launch or API call failed */
    PB_ERR_WORKSPACE = 3, /* workspace missing or smaller than *_workspace_size() */
    PB_ERR_DEVICE = 4,    /* no usable sm_100 device */
    PB_ERR_TIMEOUT = 5    /* a bounded wait gave up */
};

/* Message of the last failing call on this host thread ("" if none). */
const char *pb_last_error(void);
/* ABI version, major*10000 + minor*100 + patch. */
int pb_version(void);
/* Number of kernels this library has launched in the process so far. */
long long pb_launch_count(void);
/* 1 in the checked build (libpoisson_b200_checked.so, compiled with
 * -DPB_CHECKED), 0 otherwise.  No counterpart in the reference. */
int pb_checked_build(void);
/* The checked build's device error word: 0, or (site << 56) | index of the
 * first padded index or guarded store found outside its array (the access was
 * redirected to index 0 or skipped).  clear != 0 resets it.  Synchronous.  The
 * normal build reports 0. */
int pb_check_status(uint64_t *word, int clear);

/* Replaces mpr_parallel_init (_lib.py:21; capi.mojo:36-38): selects `device`
 * and checks it is an sm_100 part.  Optional; every call works without it. */
int pb_init(int device);

/* ---- octree (a1, a2) ------------------------------------------------------ */

/* mpr_octree_codes_f64 (_lib.py:22; capi.mojo:62-99): codes[i*(depth+1)+l] is
 * point i's Morton child-index chain down to level l (codes[i*(depth+1)] = 0).
 * 0 <= depth <= 19.  Bit-exact. */
int pb_octree_codes_f64(const double *points, int64_t point_count, int64_t depth,
                        int64_t *codes, void *stream);

/* build_octree (core.py:86-127) on the device, in two phases sharing one
 * workspace.  pb_octree_count sorts the leaf codes and writes the number of
 * distinct codes per level to level_counts[0..depth] (device int64).  After
 * the caller has read them and allocated node_count = sum(level_counts)
 * entries per node array, pb_octree_emit fills the breadth-first flat octree:
 * depth, morton, parent (-1 at the root), child_start (-1 for leaves),
 * child_count, and point_leaf[point_count].  Bit-exact with the reference.
 * 1 <= point_count, 0 <= depth <= 19. */
size_t pb_octree_workspace_size(int64_t point_count, int64_t depth);
int pb_octree_count(const double *points, int64_t point_count, int64_t depth,
                    int64_t *level_counts, void *workspace, size_t workspace_bytes, void *stream);
int pb_octree_emit(int64_t point_count, int64_t depth, const int64_t *level_counts,
                   int64_t node_count, int64_t *node_depth, int64_t *morton, int64_t *parent,
                   int64_t *child_start, int64_t *child_count, int64_t *point_leaf,
                   void *workspace, size_t workspace_bytes, void *stream);

/* ---- splat and assembly (a5-a7) ----------------------------------------- */

/* mpr_splat_f64 (_lib.py:23; capi.mojo:104-224): adds the two-pass trilinear
 * splat into density, screen, vx, vy, vz (callers zero them first, as the
 * reference does) and writes the accepted-sample count to *accepted (device).
 * Each grid node sums its contributions in point order, exactly as the serial
 * reference does, so the grids are bit-identical to it.  n >= 2,
 * n^3 < 2^31, 8*point_count < 2^32. */
size_t pb_splat_workspace_size(int64_t point_count, int64_t n);
int pb_splat_f64(const double *points, const double *normals, int64_t point_count, int64_t n,
                 int64_t confidence, double *density, double *vx, double *vy, double *vz,
                 double *screen, double samples_per_node, int64_t *accepted,
                 void *workspace, size_t workspace_bytes, void *stream);
/* Auxiliary attribute interpolation (no counterpart in the reference, which
 * lists it among upstream PoissonRecon features it leaves out, README.md:31-36):
 * per-sample attributes (point_count x channels, row-major FP64) of unit-cube
 * samples splatted with the samples' pass-1 weights w, summed per node in
 * sample order: grids (channels + 1 planes of n^3, overwritten) get sum w a_c
 * and, last, sum w.  Then the values at mesh vertices (world coordinates, `map`
 * = the (min x, y, z, width) of pb_prepare_points_f64): the ratio of the
 * trilinear interpolants of sum w a_c and sum w over the vertex's cell, 0
 * where no weight reaches it.  1 <= channels <= 64. */
size_t pb_splat_attributes_workspace_size(int64_t point_count);
int pb_splat_attributes_f64(const double *points, const double *normals, int64_t point_count, int64_t n,
                            int64_t confidence, const double *attributes, int64_t channels, double *grids,
                            void *workspace, size_t workspace_bytes, void *stream);
int pb_sample_attributes_f64(const double *vertices, int64_t vertex_count, const double *map, int64_t n,
                             const double *grids, int64_t channels, double *out, void *stream);

/* mpr_assemble_f64 (_lib.py:24; capi.mojo:228-279):
 * rhs = -div(V) + point_weight * screen * (n-1)^2 * target_value. Bit-exact. */
int pb_assemble_f64(const double *vx, const double *vy, const double *vz, const double *screen,
                    double *rhs, int64_t n, double point_weight, double target_value,
                    void *stream);

/* ---- multigrid operators, FP64 (a9-a12) ------------------------------------ */

/* mpr_relax_f64 (_lib.py:25; capi.mojo:310-410): `iterations` red-black
 * Gauss-Seidel sweeps in place.  Bit-exact. */
int pb_relax_f64(double *solution, const double *rhs, const double *screen, int64_t n,
                 double point_weight, int64_t iterations, void *stream);

/* mpr_residual_f64 (_lib.py:26; capi.mojo:474-553): residual = rhs - A x
 * (bit-exact) and *norm = ||residual||_2 (device; summation order differs
 * from the serial reference by rounding only). */
size_t pb_residual_workspace_size(int64_t n);
int pb_residual_f64(const double *solution, const double *rhs, const double *screen,
                    double *residual, int64_t n, double point_weight, double *norm,
                    void *workspace, size_t workspace_bytes, void *stream);

/* ||values||_2 into *norm (device) — the scale of the relative residual
 * ||rhs - A x|| / ||rhs|| that the tolerance-driven solves stop on (the
 * reference runs a fixed number of cycles and has no such loop). */
int pb_norm_f64(const double *values, int64_t count, double *norm, void *workspace,
                size_t workspace_bytes, void *stream);

/* mpr_restrict_f64 (_lib.py:27; capi.mojo:557-673): boundary-normalised full
 * weighting onto coarse_n = (fine_n+1)/2.  Bit-exact. */
int pb_restrict_f64(const double *fine, double *coarse, int64_t fine_n, void *stream);

/* mpr_prolong_add_f64 (_lib.py:28; capi.mojo:677-742): fine += trilinear(coarse).
 * Bit-exact. */
int pb_prolong_add_f64(const double *coarse, double *fine, int64_t fine_n, void *stream);

/* ---- iso-value (a14) -------------------------------------------------------- */

/* mpr_iso_value_f64 (_lib.py:29; capi.mojo:746-795): *iso (device) = weighted
 * mean of the trilinear field at the samples (0 when the weights sum to 0). */
size_t pb_iso_value_workspace_size(int64_t point_count);
int pb_iso_value_f64(const double *field, const double *points, const double *normals,
                     int64_t point_count, int64_t n, int64_t confidence, double *iso,
                     void *workspace, size_t workspace_bytes, void *stream);

/* ---- dual contouring (a15-a17) ------------------------------------------------ */

/* mpr_dual_vertices_f64 (_lib.py:30; capi.mojo:841-1041).  capacity <= 0:
 * count the active cells into *count (device); cell_map, vertices and
 * vertex_density are not touched.  capacity > 0: cell_map[(n-1)^3] gets the
 * vertex id of each active cell in z,y,x order (-1 for inactive cells; active
 * cells past `capacity` keep 0, as in the reference), the first `capacity`
 * vertices and their densities are written, and *count gets the total.
 * Topology and coordinates are bit-exact.
 * The _isoptr variant reads the iso-value from device memory instead. */
size_t pb_dual_workspace_size(int64_t n);
int pb_dual_vertices_f64(const double *field, const double *density, int64_t n, double iso,
                         int64_t *cell_map, double *vertices, double *vertex_density,
                         int64_t capacity, int64_t *count, void *workspace,
                         size_t workspace_bytes, void *stream);
int pb_dual_vertices_f64_isoptr(const double *field, const double *density, int64_t n,
                                const double *iso, int64_t *cell_map, double *vertices,
                                double *vertex_density, int64_t capacity, int64_t *count,
                                void *workspace, size_t workspace_bytes, void *stream);

/* Active-cell count of pb_dual_vertices_f64's count mode, for callers that
 * cannot allocate device memory (no workspace argument).  No counterpart in
 * the reference: its count mode writes into the caller's scratch buffer.
 * Scratch is a fixed 512 KiB array in the library's device memory, so
 * n <= 513; larger grids get PB_ERR_INVALID.  The first call on a device
 * (and on each further context of it) looks the array up: make it before any
 * stream capture.  Calls that overlap on the GPU share the array and race.
 * Do not call it on a device after cudaDeviceReset in the same process. */
int pb_dual_vertex_count_f64_noalloc(const double *field, int64_t n, double iso, int64_t *count,
                                     void *stream);

/* mpr_dual_faces_f64 (_lib.py:31; capi.mojo:1076-1129): two triangles per
 * sign-changing interior edge (x-edges, then y-edges, then z-edges, each in
 * z,y,x order); faces are written while 2 more fit in `capacity`; *count
 * (device) gets the total.  Bit-exact. */
int pb_dual_faces_f64(const double *field, int64_t n, double iso, const int64_t *cell_map,
                      int64_t *faces, int64_t capacity, int64_t *count, void *workspace,
                      size_t workspace_bytes, void *stream);
int pb_dual_faces_f64_isoptr(const double *field, int64_t n, const double *iso,
                             const int64_t *cell_map, int64_t *faces, int64_t capacity,
                             int64_t *count, void *workspace, size_t workspace_bytes,
                             void *stream);

/* ---- FP32 inner multigrid for FP64 defect correction ----------------------------
 * No counterpart in the reference, which solves in FP64 only (capi.mojo:310-742).
 * FP32 level arrays use a padded layout: side n with a zero ghost layer on
 * every face, x offset 4, row pitch P = pb_level_geometry(n):
 *   index(x, y, z) = ((z+1)*(n+2) + (y+1))*P + (x+4),   x, y, z in [-1, n].
 * Callers allocate them zero-filled; kernels write interior nodes only. */
int pb_level_geometry(int64_t n, int64_t *pitch, int64_t *padded_count);
/* D = (degree + pw*screen)*(n-1)^2 and 1/D per node from the dense FP64 screen;
 * weights (may be NULL): the prolongation weights s of the FP32 cycle, 1 on
 * nodes of the coarse grid, else degree*(n-1)^2 / D. */
int pb_level_setup_f32(const double *screen, int64_t n, double point_weight, float *D, float *invD,
                       float *weights, void *stream);
/* r32 = b - A x in FP64 (dense x, b, screen; r32 padded), *norm2 = ||b - A x||^2,
 * and the FP64 residual into r64 when it is not NULL.  With e != NULL the
 * iterate is first updated: x_new = x_old + e (written). */
size_t pb_defect_workspace_size(int64_t n);
int pb_defect_f64(const double *x_old, const float *e, double *x_new, const double *rhs,
                  const double *screen, int64_t n, double point_weight, float *r32, double *r64,
                  double *norm2, void *workspace, size_t workspace_bytes, void *stream);
/* FP64 flexible conjugate gradients, FCG(1), preconditioned by the FP32
 * V-cycle, in two passes per iteration (no counterpart in the reference, which
 * repeats V-cycles, core.py:274-285).  Device scalars scal[0..4]: (p, Ap),
 * beta, alpha, (p, r), ||b - A x||^2; flags[0] != 0 on the first step,
 * flags[1] = iterations done, whose parity selects the buffers: directions
 * p[it & 1] -> p[(it+1) & 1] (dense FP32), iterates x[it & 1] -> x[(it+1) & 1]
 * (dense FP64).  Every iteration touches the same pointers, so one can be
 * captured in a graph. */
size_t pb_fcg_workspace_size(int64_t n);
/* Pass 1, after z = M(r32): beta, (p, Ap) and alpha from one stencil pass over z. */
int pb_fcg_direction_f64(const float *z, const float *p0, const float *p1, const float *r32,
                         const double *screen, int64_t n, double point_weight, double *scal, const int *flags,
                         void *workspace, size_t workspace_bytes, void *stream);
/* Pass 2: p, x += alpha p and the true residual b - A x into r32 (padded FP32),
 * ||b - A x||^2 into scal[4]. */
int pb_fcg_update_f64(const float *z, float *p0, float *p1, double *x0, double *x1, const double *b,
                      const double *screen, float *r32, int64_t n, double point_weight, double *scal,
                      const int *flags, void *workspace, size_t workspace_bytes, void *stream);
/* One red-black Gauss-Seidel sweep (colour 0 then colour 1), out of place,
 * with TMA-staged planes (n = 2^k + 1 >= 33): mode 0 from e_in, mode 1 from
 * zero (e_in unused).  z_chunk <= 0 picks one.  A bounded wait that gives up
 * sets *status (device int) to 1. */
int pb_sweep_tma_f32(const float *e_in, float *e_out, const float *rhs, const float *invD, int64_t n,
                     int64_t mode, int64_t z_chunk, int *status, void *stream);
/* fine += s * trilinear(coarse) (coarse side (n+1)/2), padded layouts, s the
 * prolongation weights of the fine level (pb_level_setup_f32 for level 0,
 * pb_level27_finish_f32 below).  Replaces mpr_prolong_add_f64
 * (capi.mojo:677-742) inside the FP32 cycle. */
int pb_prolong_fac_f32(const float *coarse, float *fine, const float *weights, int64_t fine_n, void *stream);
/* Device-driven iteration (no counterpart in the reference).  Begin: a graph
 * with one WHILE conditional node; `stream` is captured into its body until
 * pb_loop_capture_end, which instantiates it.  The body's last launch must be
 * pb_loop_condition(handle, ...): it counts the iteration (flags[1]), clears
 * flags[0], records scal[4] in history[iteration-1] (if not NULL) and keeps
 * looping while scal[4] > ctrl[0] and fewer than min(max_iter, ctrl[1])
 * iterations ran (max_iter also bounds history).
 * handle = 0 runs the same bookkeeping eagerly.  Every pb_graph_launch runs
 * the loop to completion on the device. */
int pb_loop_capture_begin(void *stream, void **graph, unsigned long long *handle);
int pb_loop_condition(unsigned long long handle, const double *scal, const double *ctrl, int *flags,
                      int64_t max_iter, double *history, void *stream);
int pb_loop_capture_end(void *stream, void *graph, void **exec);
int pb_graph_launch(void *exec, void *stream);
int pb_graph_destroy(void *exec, void *graph);
/* Adds launches that ran inside graphs to pb_launch_count(). */
int pb_note_launches(long long count);

/* Extraction for reconstruct(): the mesh pb_dual_vertices_f64 +
 * pb_dual_faces_f64 give (same vertices, densities and faces, same order,
 * bit-identical), from sign bits and rank structures instead of a dense cell
 * map (no counterpart in the reference, whose extraction is
 * capi.mojo:798-1129).  Count first (counts[0] = vertices, counts[1] =
 * triangles, device int64), then emit with the same field, side, iso and
 * workspace; emit's vertices (with vertex_density) or faces may be NULL when
 * their count is 0 and are then not written.  Sides 2..1025. */
size_t pb_extract_workspace_size(int64_t n);
int pb_extract_count_f64(const double *field, int64_t n, const double *iso, int64_t *counts, void *workspace,
                         size_t workspace_bytes, void *stream);
int pb_extract_emit_f64(const double *field, const double *density, int64_t n, const double *iso, double *vertices,
                        double *vertex_density, int64_t *faces, void *workspace, size_t workspace_bytes,
                        void *stream);

/* oriented_points_from_mesh (core.py:429-451) on the device, bit-identical to
 * the reference's per-face loop: count first (counts[0] = kept vertices,
 * counts[1] = 1 if a face index lies outside [0, vertex_count); device
 * int64[2]), then emit the kept vertices and their unit area-weighted normals
 * in vertex order with the same arguments and workspace. */
size_t pb_mesh_normals_workspace_size(int64_t vertex_count, int64_t face_count);
int pb_mesh_normals_count_f64(const double *vertices, int64_t vertex_count, const int64_t *faces,
                              int64_t face_count, int64_t *counts, void *workspace, size_t workspace_bytes,
                              void *stream);
int pb_mesh_normals_emit_f64(const double *vertices, int64_t vertex_count, const int64_t *faces, int64_t face_count,
                             double *out_points, double *out_normals, void *workspace, size_t workspace_bytes,
                             void *stream);

/* ---- FP32 preconditioner levels (no counterpart in the reference) ----------
 * The reference's V-cycle (core.py:141-193) rediscretises coarse levels; the
 * FP32 preconditioner of the refined solvers uses Galerkin coarse levels
 * A_c = P_s^T A P_s / 8 with the screening-scaled prolongation P_s = S P.
 * 27-point levels store 14 planes (plane stride = padded count of the level):
 * the diagonal, then the couplings to the 13 forward neighbours. */

/* Level 0: coarse_rhs (side (n+1)/2) = P^T (s (rhs - A e)) / 8 with A the
 * reference's operator (diagonal D) and s its weights, without writing the
 * fine residual. */
int pb_residual_restrict_f32(const float *e, const float *rhs, const float *D, const float *weights,
                             float *coarse_rhs, int64_t n, void *stream);
/* The same result, bit for bit, with the fine planes of e, rhs, D and weights
 * staged in shared memory by TMA (a four-plane ring two planes ahead, one
 * mbarrier per plane); sides 2^k + 1 >= 33.  The FP32 cycle calls it in place
 * of pb_residual_restrict_f32 where RESTRICT_VARIANT is 2.  A bounded wait
 * that gives up sets *status (device int) to 1. */
int pb_residual_restrict_tma_f32(const float *e, const float *rhs, const float *D, const float *weights,
                                 float *coarse_rhs, int64_t n, int *status, void *stream);
/* 14 planes of the Galerkin operator of the level below a level of side
 * fine_n with prolongation weights fine_weights: from level 0 (fine_is_7pt
 * != 0, `fine` = D; no workspace) or from 14 planes, one axis at a time over
 * slabs of coarse planes that fit the workspace.  pb_galerkin_workspace_size
 * gives the bytes for a single slab; smaller workspaces work down to the size
 * of one coarse plane's slab (the call reports it when too small). */
size_t pb_galerkin_workspace_size(int64_t fine_n, int fine_is_7pt);
int pb_galerkin_f32(const float *fine, int64_t fine_n, int fine_is_7pt, const float *fine_weights,
                    float *coarse, void *workspace, size_t workspace_bytes, void *stream);
/* 14 planes of a 7-point level (diagonal D, off-diagonals -(n-1)^2). */
int pb_level27_from7_f32(const float *D, int64_t n, float *coef, void *stream);
/* invD = 1 / diagonal and the prolongation weights of a 27-point level. */
int pb_level27_finish_f32(const float *coef, int64_t n, float *invD, float *weights, void *stream);
/* Packed 27-point levels: per colour c, the 26 couplings divided by the
 * diagonal, -a(J, J+K) / a(J, J), in FP16 (h_c, 32 halves per node, node-major)
 * and 1/a(J, J) in FP32 (inv_c), over the colour's nodes numbered compactly;
 * sizes in bytes from pb_packed27_size.  Relaxation and residual of a packed level both use
 * the rounded couplings. */
int pb_packed27_size(int64_t n, int64_t *coupling_bytes, int64_t *inverse_bytes);
int pb_pack27_f32(const float *coef, int64_t n, void *h0, void *h1, float *inv0, float *inv1, void *stream);
/* One red-black ordered sweep e_next <- S(e_prev) on a packed level, the
 * same-colour couplings from e_prev (e_prev NULL: from zero). */
int pb_relax27p_f32(const float *e_prev, float *e_next, const float *rhs, const void *h0, const void *h1,
                    const float *inv0, const float *inv1, int64_t n, void *stream);
/* res = weights * (rhs - A e) on a packed level, then coarse_rhs = P^T res / 8. */
int pb_residual_restrict27p_f32(const float *e, const float *rhs, const void *h0, const void *h1,
                                const float *inv0, const float *inv1, const float *weights, int64_t n,
                                float *res, float *coarse_rhs, void *stream);
/* Inverse (27 x 27, FP64 row-major, by FP64 Gauss-Jordan) of the 27-point level
 * of side 3; the single-block cycle applies it in FP64. */
int pb_coarse_inverse_f64(const float *coef, int64_t n, double *inverse, void *stream);
/* Levels of side <= 9 (sizes: count levels halving down to 3, finest first)
 * run in one block from a compact image written at set-up: per level but the
 * last, the 27 couplings of each node, 1/diagonal and prolongation weights
 * (host arrays of device pointers to each level's 14 planes, invD and
 * weights), then the 3^3 inverse (FP64).  image: 16-byte aligned, of
 * pb_coarse27_image_size bytes (0 for invalid sizes). */
size_t pb_coarse27_image_size(int64_t count, const int64_t *sizes);
int pb_coarse27_image_f32(int64_t count, const int64_t *sizes, const float *const *coef,
                          const float *const *invD, const float *const *weights, const double *inverse,
                          float *image, size_t image_bytes, void *stream);
/* The V-cycle over those levels in shared memory: (pre, post) sweeps on the
 * first, `inner` each way on the others, the last solved with its inverse.
 * rhs: the first level's right-hand side (padded layout); e receives its
 * correction. */
int pb_coarse27_cycle_f32(int64_t count, const int64_t *sizes, const float *image, const float *rhs, float *e,
                          int64_t pre, int64_t post, int64_t inner, void *stream);

/* A whole preconditioner hierarchy's set-up from one call: the launches of
 * pb_level_setup_f32 (level 0 from the FP64 screen; for a 27-point level 0 also
 * pb_level27_from7_f32 and pb_level27_finish_f32), then per level l >= 1
 * pb_galerkin_f32 from level l-1, pb_level27_finish_f32, and pb_pack27_f32 of
 * level l-1 when it is packed; pb_coarse_inverse_f64 of the last level and
 * pb_coarse27_image_f32 of the levels from first_coarse on — in that order, so
 * the results are those of the separate calls.  arrays: PB_LEVEL_ARRAYS device
 * pointers per level, in the order D, invD, weights, coef, h0, h1, inv0, inv1
 * (D on level 0 only; coef NULL for a 7-point level 0; the packed four NULL on
 * levels that are not packed).  No counterpart in the reference, whose coarse
 * levels are rediscretised per cycle (core.py:267-269). */
enum { PB_LEVEL_ARRAYS = 8 };
int pb_hierarchy_setup_f32(int64_t levels, const int64_t *sides, const void *const *arrays, int64_t first_coarse,
                           const double *screen, double point_weight, void *galerkin_ws, size_t galerkin_bytes,
                           double *inverse, float *image, size_t image_bytes, void *stream);

/* ---- batches of clouds: one grouped launch per solver step ------------------
 * No counterpart in the reference, which solves one cloud at a time and level
 * by level (core.py:141-193, driven per cycle at :270-287).  A grouped launch
 * runs one step of the FP32 V-cycle or of FCG(1) over many (cloud, level)
 * grids of any side at once.  The caller describes the grids once:
 * pb_batch_describe writes `count` descriptors (pb_batch_desc_bytes(count)
 * bytes, 64-byte aligned, host memory) from, per grid, its cloud index, side,
 * PB_BATCH_PTRS operand pointers (kind-specific order below, unused slots
 * NULL) and 4 kind-specific integers (aux, may be NULL: zeros), and reports
 * the launch's total blocks.  The caller copies the descriptors to device
 * memory it owns (64-byte aligned) and pb_batch_launch queues the step over
 * them as often as needed, inside a captured graph too.
 *
 * Per-cloud state, indexed by the cloud index: flags int[4] (first step,
 * iterations done, active, unused), scalars double[8] (as pb_fcg_*), loop
 * control double[2] (target ||r||^2, iteration cap).  Every block of a cloud
 * whose active flag is 0 returns at once, so converged clouds stay as they
 * are while the others iterate.
 *
 * Operands per kind (p = padded FP32 level arrays, d = dense):
 *   SWEEP / SWEEP_ZERO     e_in (ignored from zero), e_out, rhs, 1/D, status word;
 *                          z_chunk <= 0: whole planes per block (sides 2^k + 1 >= 33)
 *   PROLONG32              coarse, fine, weights               (pb_prolong_fac_f32)
 *   RESIDUAL_RESTRICT32    e, rhs, D, weights, coarse rhs      (pb_residual_restrict_f32)
 *   RELAX27P / _ZERO       e_prev, e_next, rhs, h0, h1, inv0, inv1   (pb_relax27p_f32)
 *   RESIDUAL27P            e, rhs, h0, h1, inv0, inv1, weights, res
 *   RESTRICT27             fine res, coarse rhs (side = the fine side)
 *   COARSE27               image, rhs, e; aux = pre, post, inner; one block per
 *                          grid, every grid of the launch of the same first side
 *                          (pass it as first_side to pb_batch_launch)
 *   FCG_DIRECTION          z, p0, p1, r32, screen (d), partials; aux[0] = point
 *                          weight as the bits of a double
 *   FCG_DIRECTION_FINISH   partials, the cloud's scalars; aux[0] = the cloud's
 *                          pb_batch_fcg_blocks(n, 0)
 *   FCG_UPDATE             z, p0, p1, x0, x1, b, screen, r32, the cloud's scalars,
 *                          partials; aux[0] = point weight bits
 *   FCG_SUM                partials, the cloud's scalars + 4; aux[0] =
 *                          pb_batch_fcg_blocks(n, 1)
 * Partials: pb_batch_fcg_partials(n) doubles per cloud. */
enum {
    PB_BATCH_SWEEP = 0,
    PB_BATCH_SWEEP_ZERO = 1,
    PB_BATCH_PROLONG32 = 2,
    PB_BATCH_RESIDUAL_RESTRICT32 = 3,
    PB_BATCH_RELAX27P = 4,
    PB_BATCH_RELAX27P_ZERO = 5,
    PB_BATCH_RESIDUAL27P = 6,
    PB_BATCH_RESTRICT27 = 7,
    PB_BATCH_COARSE27 = 8,
    PB_BATCH_FCG_DIRECTION = 9,
    PB_BATCH_FCG_DIRECTION_FINISH = 10,
    PB_BATCH_FCG_UPDATE = 11,
    PB_BATCH_FCG_SUM = 12,
    PB_BATCH_PTRS = 12
};
size_t pb_batch_desc_bytes(int64_t count);
int64_t pb_batch_fcg_partials(int64_t n);
int64_t pb_batch_fcg_blocks(int64_t n, int64_t pass);
int pb_batch_describe(int kind, int64_t count, const int64_t *clouds, const int64_t *sides,
                      const void *const *ptrs, const int64_t *aux, int64_t z_chunk, void *desc_host,
                      size_t desc_bytes, int64_t *blocks);
int pb_batch_launch(int kind, const void *desc_device, int64_t count, int64_t blocks, const int *flags,
                    int64_t first_side, void *stream);
/* End of one batch iteration (the last launch of a captured WHILE body, as
 * pb_loop_condition for one cloud): for every active cloud, count the
 * iteration, clear its first-step flag, record scal[4] in
 * history[cloud*max_iter + iteration-1] (history may be NULL) and keep it
 * active while scal[4] > ctrl[0] and fewer than min(max_iter, ctrl[1])
 * iterations ran; the loop continues while any cloud is active. */
int pb_batch_loop_condition(unsigned long long handle, const double *scal, const double *ctrl, int *flags,
                            int64_t clouds, int64_t max_iter, double *history, void *stream);

/* ---- launch parameters chosen by an autotuner (no counterpart in the reference,
 * whose launch shape is the fixed GRID_Z_CHUNK / PARALLEL_GRID_THRESHOLD of
 * capi.mojo:9-10) ----------------------------------------------------------------
 * A host-side table per (parameter, grid side n); a launcher reads it when it
 * chooses its launch shape and uses its built-in choice where no value is set.
 *   SWEEP_Z_CHUNK          planes per block of pb_sweep_tma_f32 when its z_chunk <= 0
 *   RESTRICT_PLANES        coarse planes per block of pb_residual_restrict_f32 (default 4)
 *   PROLONG_PLANES         fine planes per block of pb_prolong_fac_f32
 *   FCG_DIRECTION_PLANES   planes per block of pb_fcg_direction_f64 (default 24, at least 8)
 *   FCG_UPDATE_PLANES      planes per block of pb_fcg_update_f64 (default 24, at least 8)
 *   FCG_DIRECTION_VARIANT  register budget of pb_fcg_direction_f64: 0 = 4 resident
 *                          blocks per SM, 1 = 6, 2 = 8
 *   RESTRICT_VARIANT       pb_residual_restrict_f32: 1 = both fine planes of a coarse
 *                          plane in one loop over their items; 2 = the FP32 cycle
 *                          calls pb_residual_restrict_tma_f32 instead; 3 = as 1 with
 *                          320 threads per block
 *   RELAX27_VARIANT        pb_relax27p_f32 (per level side): 1 = the neighbour planes
 *                          staged in shared memory
 *   RESIDUAL27_VARIANT     pb_residual_restrict27p_f32 (per level side): 1 = the
 *                          residual with e's planes staged in shared memory
 *   SWEEP_VARIANT          pb_sweep_tma_f32: 0 = a 5-plane shared ring with 2 resident
 *                          blocks per SM, 1 = 4 planes with 3 blocks, 2 = 3 planes with 3;
 *                          3, 4, 5 = each warp's box rows of one parity, so a phase
 *                          computes only the lanes it updates: (5 planes, 2 blocks),
 *                          (6, 2), (4, 3); 6, 7, 8 = the same with one barrier per
 *                          plane (a ring slot refilled one step earlier)
 *   FCG_UPDATE_VARIANT     pb_fcg_update_f64: 0 = 5 resident blocks per SM,
 *                          1 = 6 resident blocks per SM, 2 = 8, 3 = the next two planes
 *                          prefetched into shared memory by cp.async, 4 = three planes
 * The plane counts also apply to the grouped launches described after they are
 * set.  value 0 clears an entry.  Results do not depend on these values, except
 * the FCG passes' planes per block: they shape the inner products' partial-sum
 * trees, so another value changes results by rounding. */
enum {
    PB_TUNE_SWEEP_Z_CHUNK = 0,
    PB_TUNE_RESTRICT_PLANES = 1,
    PB_TUNE_PROLONG_PLANES = 2,
    PB_TUNE_FCG_DIRECTION_PLANES = 3,
    PB_TUNE_FCG_UPDATE_PLANES = 4,
    PB_TUNE_FCG_DIRECTION_VARIANT = 5,
    PB_TUNE_FCG_UPDATE_VARIANT = 6,
    PB_TUNE_SWEEP_VARIANT = 7,
    PB_TUNE_RESTRICT_VARIANT = 8,
    PB_TUNE_RELAX27_VARIANT = 9,
    PB_TUNE_RESIDUAL27_VARIANT = 10,
    PB_TUNE_PARAMS = 11
};
int pb_tune_set(int64_t param, int64_t n, int64_t value);
int64_t pb_tune_get(int64_t param, int64_t n);
int pb_tune_clear(void);

/* ---- host-orchestration helpers (core.py steps done on the device) ---------- */

/* core.py:73-83 + :377-385: keep the rows of (points, normals) with a finite
 * point and a finite non-zero normal, in order, into out_points/out_normals;
 * *kept (device int64) = their number.  scale > 0: also map the kept points
 * into the unit cube in place, map[0..2] = origin, map[3] = width (device).
 * Bit-identical to the reference's NumPy arithmetic. */
size_t pb_prepare_workspace_size(int64_t point_count);
int pb_prepare_points_f64(const double *points, const double *normals, int64_t point_count, double scale,
                          double *out_points, double *out_normals, int64_t *kept, double *map,
                          void *workspace, size_t workspace_bytes, void *stream);
/* core.py:225-227: *outside (device int, zeroed by the caller) = 1 if any
 * coordinate lies outside [0, 1]. */
int pb_unit_cube_check_f64(const double *points, int64_t point_count, int *outside, void *stream);
/* core.py:425: vertices = vertices * map[3] + map[0..2]. */
int pb_map_vertices_f64(double *vertices, int64_t vertex_count, const double *map, void *stream);
/* core.py:255 (density /= samples_per_node), :269 (screen * 4), :270/:287 (fill). */
int pb_divide_f64(double *values, int64_t count, double divisor, void *stream);
int pb_scale_f64(double *values, int64_t count, double factor, void *stream);
int pb_fill_f64(double *values, int64_t count, double value, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* POISSON_B200_H */
