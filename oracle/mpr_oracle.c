/*
 * CPU ORACLE — test infrastructure only, never part of the product path.
 *
 * A plain-C restatement of the eleven native kernels of mojo-poissonrecon
 * (src/capi.mojo).  It exports the same `mpr_*` C symbols with the same
 * argument lists as the reference's ctypes table (python/mojo_poissonrecon/
 * _lib.py:20-32), so the reference's own Python orchestration and tests can
 * load it in place of the Mojo library.  Only tests/, __graft_entry__.smoke()
 * and bench.py (its CPU-baseline and reference legs) may load this library.
 *
 * Arithmetic follows capi.mojo operation for operation: the same summation
 * orders, the same clamps and the same association of products.  Build with
 * -ffp-contract=off so that no multiply-add is fused (the GPU kernels use
 * explicitly rounded FP64 operations to match).
 *
 * Parallelism: grid stencils (relax, residual, restrict, prolong, assemble,
 * dual-cell marking) are element-independent per colour / per pass, so the
 * optional OpenMP loops below leave every result bit-identical to the serial
 * run.  Order-dependent sums (splat, iso-value, residual norm, vertex id
 * assignment, faces) stay serial, exactly as in the reference.
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>

typedef int64_t I;

#define GRID_Z_CHUNK 4 /* capi.mojo:10 */

static inline I grid_index(I x, I y, I z, I n) { return (z * n + y) * n + x; } /* capi.mojo:42 */
static inline I cell_index(I x, I y, I z, I c) { return (z * c + y) * c + x; } /* capi.mojo:47 */

/* capi.mojo:51-59 — overflow-safe Euclidean length. */
static inline double norm3(double x, double y, double z) {
    double ax = fabs(x), ay = fabs(y), az = fabs(z);
    double m = ay > az ? ay : az;
    double scale = ax > m ? ax : m;
    if (scale == 0.0) return 0.0;
    double sx = x / scale, sy = y / scale, sz = z / scale;
    return scale * sqrt(sx * sx + sy * sy + sz * sz);
}

static inline I clampi(I v, I lo, I hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline double clampd(double v, double lo, double hi) {
    /* min(max(v, lo), hi) as in capi.mojo:193-195 */
    double m = v > lo ? v : lo;
    return m < hi ? m : hi;
}

/* capi.mojo:36-38 — the reference's runtime hook; nothing to initialise. */
I mpr_parallel_init(void) { return 0; }

/* The reference's loader registers this at exit (_lib.py:84-89). */
void KGEN_CompilerRT_AsyncRT_ReleaseCPUDevice(I device) { (void)device; }

/* capi.mojo:62-99 — per point, per level, the 3-bit child index chain. */
void mpr_octree_codes_f64(I points_address, I point_count, I depth, I codes_address) {
    const double *points = (const double *)(intptr_t)points_address;
    int64_t *codes = (int64_t *)(intptr_t)codes_address;
#pragma omp parallel for schedule(static) if (point_count > 65536)
    for (I i = 0; i < point_count; ++i) {
        double x = points[3 * i], y = points[3 * i + 1], z = points[3 * i + 2];
        int64_t code = 0;
        codes[i * (depth + 1)] = 0;
        for (I d = 0; d < depth; ++d) {
            I scale = (I)1 << (d + 1);
            I ix = (I)(x * (double)scale), iy = (I)(y * (double)scale), iz = (I)(z * (double)scale);
            if (ix < 0) ix = 0;
            if (iy < 0) iy = 0;
            if (iz < 0) iz = 0;
            if (ix >= scale) ix = scale - 1;
            if (iy >= scale) iy = scale - 1;
            if (iz >= scale) iz = scale - 1;
            I child = (ix & 1) | ((iy & 1) << 1) | ((iz & 1) << 2);
            code = (code << 3) | child;
            codes[i * (depth + 1) + d + 1] = code;
        }
    }
}

/* capi.mojo:104-224 — two-pass trilinear splat (density/screen, then the
 * density-normalised vector field).  Returns the number of accepted samples. */
I mpr_splat_f64(I points_address, I normals_address, I point_count, I n, I confidence,
                I density_address, I vx_address, I vy_address, I vz_address,
                I screen_address, double samples_per_node) {
    const double *points = (const double *)(intptr_t)points_address;
    const double *normals = (const double *)(intptr_t)normals_address;
    double *density = (double *)(intptr_t)density_address;
    double *vx = (double *)(intptr_t)vx_address;
    double *vy = (double *)(intptr_t)vy_address;
    double *vz = (double *)(intptr_t)vz_address;
    double *screen = (double *)(intptr_t)screen_address;
    I resolution = n - 1;
    I accepted = 0;
    /* pass 1: capi.mojo:127-173 */
    for (I p = 0; p < point_count; ++p) {
        double nx = normals[3 * p], ny = normals[3 * p + 1], nz = normals[3 * p + 2];
        double length = norm3(nx, ny, nz);
        if (length <= 0.0) continue;
        double sample_weight = confidence != 0 ? length : 1.0;
        double gx = points[3 * p] * (double)resolution;
        double gy = points[3 * p + 1] * (double)resolution;
        double gz = points[3 * p + 2] * (double)resolution;
        I ix = (I)gx, iy = (I)gy, iz = (I)gz;
        if (ix < 0) ix = 0;
        if (iy < 0) iy = 0;
        if (iz < 0) iz = 0;
        if (ix >= resolution) { ix = resolution - 1; gx = (double)resolution; }
        if (iy >= resolution) { iy = resolution - 1; gy = (double)resolution; }
        if (iz >= resolution) { iz = resolution - 1; gz = (double)resolution; }
        double fx = gx - (double)ix, fy = gy - (double)iy, fz = gz - (double)iz;
        for (int dz = 0; dz < 2; ++dz) {
            double wz = dz == 1 ? fz : 1.0 - fz;
            for (int dy = 0; dy < 2; ++dy) {
                double wy = dy == 1 ? fy : 1.0 - fy;
                for (int dx = 0; dx < 2; ++dx) {
                    double wx = dx == 1 ? fx : 1.0 - fx;
                    double w = wx * wy * wz * sample_weight;
                    I idx = grid_index(ix + dx, iy + dy, iz + dz, n);
                    density[idx] += 2.0 * w;
                    screen[idx] += w;
                }
            }
        }
        accepted += 1;
    }
    /* pass 2: capi.mojo:175-223 */
    for (I p = 0; p < point_count; ++p) {
        double nx = normals[3 * p], ny = normals[3 * p + 1], nz = normals[3 * p + 2];
        double length = norm3(nx, ny, nz);
        if (length <= 0.0) continue;
        double sample_weight = confidence != 0 ? length : 1.0;
        nx /= length;
        ny /= length;
        nz /= length;
        double gx = points[3 * p] * (double)resolution;
        double gy = points[3 * p + 1] * (double)resolution;
        double gz = points[3 * p + 2] * (double)resolution;
        I ix = clampi((I)gx, 0, resolution - 1);
        I iy = clampi((I)gy, 0, resolution - 1);
        I iz = clampi((I)gz, 0, resolution - 1);
        double fx = clampd(gx - (double)ix, 0.0, 1.0);
        double fy = clampd(gy - (double)iy, 0.0, 1.0);
        double fz = clampd(gz - (double)iz, 0.0, 1.0);
        double local_density = 0.0;
        for (int dz = 0; dz < 2; ++dz) {
            double wz = dz == 1 ? fz : 1.0 - fz;
            for (int dy = 0; dy < 2; ++dy) {
                double wy = dy == 1 ? fy : 1.0 - fy;
                for (int dx = 0; dx < 2; ++dx) {
                    double wx = dx == 1 ? fx : 1.0 - fx;
                    local_density += density[grid_index(ix + dx, iy + dy, iz + dz, n)] * wx * wy * wz;
                }
            }
        }
        double q = local_density / samples_per_node;
        double density_factor = 1.0 > q ? 1.0 : q; /* max(1.0, q) */
        for (int dz = 0; dz < 2; ++dz) {
            double wz = dz == 1 ? fz : 1.0 - fz;
            for (int dy = 0; dy < 2; ++dy) {
                double wy = dy == 1 ? fy : 1.0 - fy;
                for (int dx = 0; dx < 2; ++dx) {
                    double wx = dx == 1 ? fx : 1.0 - fx;
                    double w = wx * wy * wz * sample_weight;
                    I idx = grid_index(ix + dx, iy + dy, iz + dz, n);
                    double vector_weight = w * (double)resolution / density_factor;
                    vx[idx] -= nx * vector_weight;
                    vy[idx] -= ny * vector_weight;
                    vz[idx] -= nz * vector_weight;
                }
            }
        }
    }
    return accepted;
}

/* capi.mojo:228-279 — rhs = -div(V) + point_weight * screen * h^-2 * target. */
void mpr_assemble_f64(I vx_address, I vy_address, I vz_address, I screen_address,
                      I rhs_address, I n, double point_weight, double target_value) {
    const double *vx = (const double *)(intptr_t)vx_address;
    const double *vy = (const double *)(intptr_t)vy_address;
    const double *vz = (const double *)(intptr_t)vz_address;
    const double *screen = (const double *)(intptr_t)screen_address;
    double *rhs = (double *)(intptr_t)rhs_address;
    double h_inv = (double)(n - 1);
    double h_inv2 = h_inv * h_inv;
#pragma omp parallel for schedule(static) if (n * n * n >= 262144)
    for (I z = 0; z < n; ++z)
        for (I y = 0; y < n; ++y)
            for (I x = 0; x < n; ++x) {
                I idx = grid_index(x, y, z, n);
                double div = 0.0;
                if (x == 0) div += (vx[grid_index(1, y, z, n)] - vx[idx]) * h_inv;
                else if (x == n - 1) div += (vx[idx] - vx[grid_index(x - 1, y, z, n)]) * h_inv;
                else div += (vx[grid_index(x + 1, y, z, n)] - vx[grid_index(x - 1, y, z, n)]) * (0.5 * h_inv);
                if (y == 0) div += (vy[grid_index(x, 1, z, n)] - vy[idx]) * h_inv;
                else if (y == n - 1) div += (vy[idx] - vy[grid_index(x, y - 1, z, n)]) * h_inv;
                else div += (vy[grid_index(x, y + 1, z, n)] - vy[grid_index(x, y - 1, z, n)]) * (0.5 * h_inv);
                if (z == 0) div += (vz[grid_index(x, y, 1, n)] - vz[idx]) * h_inv;
                else if (z == n - 1) div += (vz[idx] - vz[grid_index(x, y, z - 1, n)]) * h_inv;
                else div += (vz[grid_index(x, y, z + 1, n)] - vz[grid_index(x, y, z - 1, n)]) * (0.5 * h_inv);
                double screening = point_weight * screen[idx] * h_inv2;
                rhs[idx] = -div + screening * target_value;
            }
}

/* capi.mojo:282-306 — Neumann 6-neighbour sum in the order x-,x+,y-,y+,z-,z+. */
static inline double stencil_sum_and_degree(const double *v, I x, I y, I z, I n, I *degree) {
    double s = 0.0;
    I d = 0;
    if (x > 0) { s += v[grid_index(x - 1, y, z, n)]; d += 1; }
    if (x + 1 < n) { s += v[grid_index(x + 1, y, z, n)]; d += 1; }
    if (y > 0) { s += v[grid_index(x, y - 1, z, n)]; d += 1; }
    if (y + 1 < n) { s += v[grid_index(x, y + 1, z, n)]; d += 1; }
    if (z > 0) { s += v[grid_index(x, y, z - 1, n)]; d += 1; }
    if (z + 1 < n) { s += v[grid_index(x, y, z + 1, n)]; d += 1; }
    *degree = d;
    return s;
}

/* capi.mojo:310-410 — red-black Gauss-Seidel, colour (x+y+z)&1, in place.
 * The diagonal guard (> 1e-30) is applied at every node, as the reference's
 * own test does (tests/test_kernels.py:157-161); the Mojo vector path omits it
 * for interior x, which only differs when the diagonal is not positive (a
 * negative screen or point weight). */
void mpr_relax_f64(I solution_address, I rhs_address, I screen_address, I n,
                   double point_weight, I iterations) {
    double *x = (double *)(intptr_t)solution_address;
    const double *rhs = (const double *)(intptr_t)rhs_address;
    const double *screen = (const double *)(intptr_t)screen_address;
    double h_inv = (double)(n - 1);
    double h_inv2 = h_inv * h_inv;
    for (I it = 0; it < iterations; ++it)
        for (I color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static) if (n * n * n >= 262144)
            for (I z = 0; z < n; ++z)
                for (I y = 0; y < n; ++y)
                    for (I xx = ((y + z + color) & 1); xx < n; xx += 2) {
                        I idx = grid_index(xx, y, z, n);
                        I degree;
                        double s = stencil_sum_and_degree(x, xx, y, z, n, &degree);
                        double screening = point_weight * screen[idx] * h_inv2;
                        double diagonal = (double)degree * h_inv2 + screening;
                        if (diagonal > 1.0e-30) x[idx] = (rhs[idx] + s * h_inv2) / diagonal;
                    }
        }
}

/* capi.mojo:413-553 — r = rhs - A x; returns the absolute L2 norm of r.
 * The norm's summation order cannot follow the Mojo build exactly: it sums
 * SIMD lanes whose width depends on the host CPU. */
double mpr_residual_f64(I solution_address, I rhs_address, I screen_address,
                        I residual_address, I n, double point_weight) {
    const double *x = (const double *)(intptr_t)solution_address;
    const double *rhs = (const double *)(intptr_t)rhs_address;
    const double *screen = (const double *)(intptr_t)screen_address;
    double *r = (double *)(intptr_t)residual_address;
    double h_inv = (double)(n - 1);
    double h_inv2 = h_inv * h_inv;
#pragma omp parallel for schedule(static) if (n * n * n >= 262144)
    for (I z = 0; z < n; ++z)
        for (I y = 0; y < n; ++y)
            for (I xx = 0; xx < n; ++xx) {
                I idx = grid_index(xx, y, z, n);
                I degree;
                double s = stencil_sum_and_degree(x, xx, y, z, n, &degree);
                double screening = point_weight * screen[idx] * h_inv2;
                double applied = ((double)degree * h_inv2 + screening) * x[idx] - s * h_inv2;
                r[idx] = rhs[idx] - applied;
            }
    /* Neumaier-compensated sum of squares: deterministic and within about one
     * ulp of the exact sum, so it sits as close to NumPy's norm as the Mojo
     * SIMD-lane sum (tests/test_kernels.py:142 allows 2e-15 relative). */
    double sq = 0.0, comp = 0.0;
    I size = n * n * n;
    for (I i = 0; i < size; ++i) {
        double term = r[i] * r[i];
        double t = sq + term;
        comp += fabs(sq) >= fabs(term) ? (sq - t) + term : (term - t) + sq;
        sq = t;
    }
    return sqrt(sq + comp);
}

/* capi.mojo:557-673 — boundary-normalised full weighting, weights (1,2,1)^3,
 * accumulated in (oz, oy, ox) order.  Every product is by a power of two, so
 * the Mojo vector and scalar paths give the same bits as this loop. */
void mpr_restrict_f64(I fine_address, I coarse_address, I fine_n) {
    const double *fine = (const double *)(intptr_t)fine_address;
    double *coarse = (double *)(intptr_t)coarse_address;
    I coarse_n = (fine_n + 1) / 2;
#pragma omp parallel for schedule(static) if (coarse_n * coarse_n * coarse_n >= 262144)
    for (I z = 0; z < coarse_n; ++z)
        for (I y = 0; y < coarse_n; ++y)
            for (I x = 0; x < coarse_n; ++x) {
                double sum = 0.0, weight = 0.0;
                for (I oz = -1; oz <= 1; ++oz) {
                    I zz = 2 * z + oz;
                    if (zz < 0 || zz >= fine_n) continue;
                    double wz = oz == 0 ? 2.0 : 1.0;
                    for (I oy = -1; oy <= 1; ++oy) {
                        I yy = 2 * y + oy;
                        if (yy < 0 || yy >= fine_n) continue;
                        double wy = oy == 0 ? 2.0 : 1.0;
                        for (I ox = -1; ox <= 1; ++ox) {
                            I xx = 2 * x + ox;
                            if (xx < 0 || xx >= fine_n) continue;
                            double wx = ox == 0 ? 2.0 : 1.0;
                            double w = wx * wy * wz;
                            sum += fine[grid_index(xx, yy, zz, fine_n)] * w;
                            weight += w;
                        }
                    }
                }
                coarse[grid_index(x, y, z, coarse_n)] = sum / weight;
            }
}

/* capi.mojo:677-742 — fine += trilinear(coarse), t in {0, 1/2} per axis. */
void mpr_prolong_add_f64(I coarse_address, I fine_address, I fine_n) {
    const double *c = (const double *)(intptr_t)coarse_address;
    double *fine = (double *)(intptr_t)fine_address;
    I cn = (fine_n + 1) / 2;
#pragma omp parallel for schedule(static) if (fine_n * fine_n * fine_n >= 262144)
    for (I z = 0; z < fine_n; ++z) {
        I z0 = z / 2, z1 = z0 + 1 < cn - 1 ? z0 + 1 : cn - 1;
        double tz = (z & 1) ? 0.5 : 0.0;
        for (I y = 0; y < fine_n; ++y) {
            I y0 = y / 2, y1 = y0 + 1 < cn - 1 ? y0 + 1 : cn - 1;
            double ty = (y & 1) ? 0.5 : 0.0;
            for (I x = 0; x < fine_n; ++x) {
                I x0 = x / 2, x1 = x0 + 1 < cn - 1 ? x0 + 1 : cn - 1;
                double tx = (x & 1) ? 0.5 : 0.0;
                double c000 = c[grid_index(x0, y0, z0, cn)], c100 = c[grid_index(x1, y0, z0, cn)];
                double c010 = c[grid_index(x0, y1, z0, cn)], c110 = c[grid_index(x1, y1, z0, cn)];
                double c001 = c[grid_index(x0, y0, z1, cn)], c101 = c[grid_index(x1, y0, z1, cn)];
                double c011 = c[grid_index(x0, y1, z1, cn)], c111 = c[grid_index(x1, y1, z1, cn)];
                double c00 = c000 * (1.0 - tx) + c100 * tx;
                double c10 = c010 * (1.0 - tx) + c110 * tx;
                double c01 = c001 * (1.0 - tx) + c101 * tx;
                double c11 = c011 * (1.0 - tx) + c111 * tx;
                double c0 = c00 * (1.0 - ty) + c10 * ty;
                double c1 = c01 * (1.0 - ty) + c11 * ty;
                fine[grid_index(x, y, z, fine_n)] += c0 * (1.0 - tz) + c1 * tz;
            }
        }
    }
}

/* capi.mojo:746-795 — (confidence-)weighted mean of the trilinear field at the samples. */
double mpr_iso_value_f64(I field_address, I points_address, I normals_address,
                         I point_count, I n, I confidence) {
    const double *field = (const double *)(intptr_t)field_address;
    const double *points = (const double *)(intptr_t)points_address;
    const double *normals = (const double *)(intptr_t)normals_address;
    I resolution = n - 1;
    double value_sum = 0.0, weight_sum = 0.0;
    for (I p = 0; p < point_count; ++p) {
        double weight = confidence != 0 ? norm3(normals[3 * p], normals[3 * p + 1], normals[3 * p + 2]) : 1.0;
        double gx = points[3 * p] * (double)resolution;
        double gy = points[3 * p + 1] * (double)resolution;
        double gz = points[3 * p + 2] * (double)resolution;
        I ix = clampi((I)gx, 0, resolution - 1);
        I iy = clampi((I)gy, 0, resolution - 1);
        I iz = clampi((I)gz, 0, resolution - 1);
        double fx = clampd(gx - (double)ix, 0.0, 1.0);
        double fy = clampd(gy - (double)iy, 0.0, 1.0);
        double fz = clampd(gz - (double)iz, 0.0, 1.0);
        double value = 0.0;
        for (int dz = 0; dz < 2; ++dz) {
            double wz = dz == 1 ? fz : 1.0 - fz;
            for (int dy = 0; dy < 2; ++dy) {
                double wy = dy == 1 ? fy : 1.0 - fy;
                for (int dx = 0; dx < 2; ++dx) {
                    double wx = dx == 1 ? fx : 1.0 - fx;
                    value += field[grid_index(ix + dx, iy + dy, iz + dz, n)] * wx * wy * wz;
                }
            }
        }
        value_sum += value * weight;
        weight_sum += weight;
    }
    return weight_sum > 0.0 ? value_sum / weight_sum : 0.0;
}

static inline double corner_value(const double *f, I x, I y, I z, I n, int corner) { /* capi.mojo:798-809 */
    return f[grid_index(x + (corner & 1), y + ((corner >> 1) & 1), z + ((corner >> 2) & 1), n)];
}

static inline int cell_active(const double *f, I x, I y, I z, I n, double iso) {
    int below = 0;
    for (int c = 0; c < 8; ++c) below += corner_value(f, x, y, z, n, c) < iso;
    return below != 0 && below != 8;
}

/* capi.mojo:812-836 */
static inline int add_edge_root(double v0, double v1, double iso, double x0, double y0, double z0,
                                double x1, double y1, double z1, double *sx, double *sy, double *sz) {
    if ((v0 < iso) == (v1 < iso)) return 0;
    double t = (iso - v0) / (v1 - v0);
    t = clampd(t, 0.0, 1.0);
    *sx = *sx + x0 + (x1 - x0) * t;
    *sy = *sy + y0 + (y1 - y0) * t;
    *sz = *sz + z0 + (z1 - z0) * t;
    return 1;
}

/* capi.mojo:841-1041 — dual (surface-nets) vertices.  capacity <= 0: count
 * active cells, writing per-z-chunk counts into the scratch buffer.  Otherwise
 * mark cells, then assign vertex ids serially in z,y,x cell order. */
I mpr_dual_vertices_f64(I field_address, I density_address, I n, double iso,
                        I cell_map_address, I vertices_address, I vertex_density_address,
                        I capacity) {
    const double *field = (const double *)(intptr_t)field_address;
    I cells = n - 1;
    I count = 0;
    if (capacity <= 0) {
        int64_t *counts = (int64_t *)(intptr_t)cell_map_address;
        I tasks = (cells + GRID_Z_CHUNK - 1) / GRID_Z_CHUNK;
#pragma omp parallel for schedule(static) if (cells * cells * cells >= 262144)
        for (I t = 0; t < tasks; ++t) {
            int64_t local = 0;
            I z_end = (t + 1) * GRID_Z_CHUNK < cells ? (t + 1) * GRID_Z_CHUNK : cells;
            for (I z = t * GRID_Z_CHUNK; z < z_end; ++z)
                for (I y = 0; y < cells; ++y)
                    for (I x = 0; x < cells; ++x) local += cell_active(field, x, y, z, n, iso);
            counts[t] = local;
        }
        for (I t = 0; t < tasks; ++t) count += counts[t];
        return count;
    }
    const double *density = (const double *)(intptr_t)density_address;
    int64_t *cell_map = (int64_t *)(intptr_t)cell_map_address;
    double *vertices = (double *)(intptr_t)vertices_address;
    double *vertex_density = (double *)(intptr_t)vertex_density_address;
#pragma omp parallel for schedule(static) if (cells * cells * cells >= 262144)
    for (I z = 0; z < cells; ++z)
        for (I y = 0; y < cells; ++y)
            for (I x = 0; x < cells; ++x)
                cell_map[cell_index(x, y, z, cells)] = cell_active(field, x, y, z, n, iso) ? 0 : -1;
    for (I z = 0; z < cells; ++z)
        for (I y = 0; y < cells; ++y)
            for (I x = 0; x < cells; ++x) {
                if (cell_map[cell_index(x, y, z, cells)] < 0) continue;
                double values[8];
                for (int c = 0; c < 8; ++c) values[c] = corner_value(field, x, y, z, n, c);
                if (count >= capacity) { count += 1; continue; }
                double sx = 0.0, sy = 0.0, sz = 0.0;
                I roots = 0;
                for (int axis = 0; axis < 3; ++axis)
                    for (int a = 0; a < 2; ++a)
                        for (int b = 0; b < 2; ++b) {
                            int c0, c1;
                            double x0, y0, z0, x1, y1, z1;
                            if (axis == 0) {
                                c0 = 2 * a + 4 * b; c1 = c0 + 1;
                                x0 = 0.0; y0 = (double)a; z0 = (double)b; x1 = 1.0; y1 = y0; z1 = z0;
                            } else if (axis == 1) {
                                c0 = a + 4 * b; c1 = c0 + 2;
                                x0 = (double)a; y0 = 0.0; z0 = (double)b; x1 = x0; y1 = 1.0; z1 = z0;
                            } else {
                                c0 = a + 2 * b; c1 = c0 + 4;
                                x0 = (double)a; y0 = (double)b; z0 = 0.0; x1 = x0; y1 = y0; z1 = 1.0;
                            }
                            roots += add_edge_root(values[c0], values[c1], iso, x0, y0, z0, x1, y1, z1, &sx, &sy, &sz);
                        }
                double inv_roots = 1.0 / (double)roots;
                vertices[3 * count] = ((double)x + sx * inv_roots) / (double)cells;
                vertices[3 * count + 1] = ((double)y + sy * inv_roots) / (double)cells;
                vertices[3 * count + 2] = ((double)z + sz * inv_roots) / (double)cells;
                double dsum = 0.0;
                for (int c = 0; c < 8; ++c) dsum += corner_value(density, x, y, z, n, c);
                vertex_density[count] = dsum * 0.125;
                cell_map[cell_index(x, y, z, cells)] = count;
                count += 1;
            }
    return count;
}

/* capi.mojo:1044-1072 */
static inline I emit_quad(int64_t *faces, I face_count, I capacity, int64_t a, int64_t b,
                          int64_t c, int64_t d, int reverse) {
    if (a < 0 || b < 0 || c < 0 || d < 0) return face_count;
    if (face_count + 2 <= capacity) {
        int64_t *f = faces + 3 * face_count;
        if (reverse) { f[0] = a; f[1] = d; f[2] = c; f[3] = a; f[4] = c; f[5] = b; }
        else { f[0] = a; f[1] = b; f[2] = c; f[3] = a; f[4] = c; f[5] = d; }
    }
    return face_count + 2;
}

/* capi.mojo:1076-1129 — quads across sign-changing interior edges, swept as
 * x-edges, then y-edges, then z-edges, each in z,y,x order. */
I mpr_dual_faces_f64(I field_address, I n, double iso, I cell_map_address, I faces_address,
                     I capacity) {
    const double *field = (const double *)(intptr_t)field_address;
    const int64_t *cm = (const int64_t *)(intptr_t)cell_map_address;
    int64_t *faces = (int64_t *)(intptr_t)faces_address;
    I cells = n - 1;
    I fc = 0;
    for (I z = 1; z < cells; ++z)
        for (I y = 1; y < cells; ++y)
            for (I x = 0; x < cells; ++x) {
                double v0 = field[grid_index(x, y, z, n)], v1 = field[grid_index(x + 1, y, z, n)];
                if ((v0 < iso) != (v1 < iso))
                    fc = emit_quad(faces, fc, capacity, cm[cell_index(x, y - 1, z - 1, cells)],
                                   cm[cell_index(x, y, z - 1, cells)], cm[cell_index(x, y, z, cells)],
                                   cm[cell_index(x, y - 1, z, cells)], v0 < iso);
            }
    for (I z = 1; z < cells; ++z)
        for (I y = 0; y < cells; ++y)
            for (I x = 1; x < cells; ++x) {
                double v0 = field[grid_index(x, y, z, n)], v1 = field[grid_index(x, y + 1, z, n)];
                if ((v0 < iso) != (v1 < iso))
                    fc = emit_quad(faces, fc, capacity, cm[cell_index(x - 1, y, z - 1, cells)],
                                   cm[cell_index(x - 1, y, z, cells)], cm[cell_index(x, y, z, cells)],
                                   cm[cell_index(x, y, z - 1, cells)], v0 < iso);
            }
    for (I z = 0; z < cells; ++z)
        for (I y = 1; y < cells; ++y)
            for (I x = 1; x < cells; ++x) {
                double v0 = field[grid_index(x, y, z, n)], v1 = field[grid_index(x, y, z + 1, n)];
                if ((v0 < iso) != (v1 < iso))
                    fc = emit_quad(faces, fc, capacity, cm[cell_index(x - 1, y - 1, z, cells)],
                                   cm[cell_index(x, y - 1, z, cells)], cm[cell_index(x, y, z, cells)],
                                   cm[cell_index(x - 1, y, z, cells)], v0 < iso);
            }
    return fc;
}

/* Thread count actually used by the OpenMP loops (1 in a serial build). */
I mpr_oracle_threads(void) {
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}
