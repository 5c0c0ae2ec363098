"""CPU ORACLE driver — test infrastructure only, never part of the product path.

Restates the reference's host orchestration (python/mojo_poissonrecon/core.py)
over the C oracle library in this directory (mpr_oracle.c, which restates
src/capi.mojo).  Used by tests/ as the checker, by __graft_entry__.smoke() and
by bench.py's CPU-baseline and reference legs.  It reads nothing from the
reference checkout, so it runs wherever the oracle library was built.

Beyond the reference it adds one loop the reference does not have: iterate
V-cycles until the relative residual ||b - A x|| / ||b|| reaches a tolerance
(`tol`), the stopping rule of the benchmark workloads.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_I = ctypes.c_int64
_F = ctypes.c_double
# Same argument lists as the reference's ctypes table (_lib.py:20-32).
_SIGNATURES = {
    "mpr_parallel_init": ([], _I),
    "mpr_octree_codes_f64": ([_I, _I, _I, _I], None),
    "mpr_splat_f64": ([_I] * 10 + [_F], _I),
    "mpr_assemble_f64": ([_I, _I, _I, _I, _I, _I, _F, _F], None),
    "mpr_relax_f64": ([_I, _I, _I, _I, _F, _I], None),
    "mpr_residual_f64": ([_I, _I, _I, _I, _I, _F], _F),
    "mpr_restrict_f64": ([_I, _I, _I], None),
    "mpr_prolong_add_f64": ([_I, _I, _I], None),
    "mpr_iso_value_f64": ([_I, _I, _I, _I, _I, _I], _F),
    "mpr_dual_vertices_f64": ([_I, _I, _I, _F, _I, _I, _I, _I], _I),
    "mpr_dual_faces_f64": ([_I, _I, _F, _I, _I, _I], _I),
    "mpr_oracle_threads": ([], _I),
}
_LIBS: dict[bool, ctypes.CDLL] = {}


def lib(threaded: bool = False) -> ctypes.CDLL:
    """The serial oracle, or its OpenMP build (bit-identical results)."""
    if threaded not in _LIBS:
        name = "liboracle_mpr_omp.so" if threaded else "liboracle_mpr.so"
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C {HERE}`")
        cdll = ctypes.CDLL(path)
        for fn_name, (argtypes, restype) in _SIGNATURES.items():
            fn = getattr(cdll, fn_name)
            fn.argtypes = argtypes
            fn.restype = restype
        _LIBS[threaded] = cdll
    return _LIBS[threaded]


def _a(array: np.ndarray) -> int:
    assert array.flags.c_contiguous and array.dtype in (np.float64, np.int64)
    return int(array.ctypes.data)


@dataclass
class OracleTree:
    depth: np.ndarray
    morton: np.ndarray
    parent: np.ndarray
    child_start: np.ndarray
    child_count: np.ndarray
    point_leaf: np.ndarray


@dataclass
class OracleSolution:
    field: np.ndarray
    density: np.ndarray
    screen: np.ndarray
    rhs: np.ndarray
    iso_value: float
    residual_norm: float
    octree: OracleTree | None
    cycles_run: int = 0
    relative_residual: float = float("nan")


@dataclass
class OracleMesh:
    vertices: np.ndarray
    faces: np.ndarray
    density: np.ndarray
    iso_value: float = 0.0
    residual_norm: float = 0.0


def octree_codes(points: np.ndarray, depth: int, threaded: bool = False) -> np.ndarray:
    points = np.ascontiguousarray(points, dtype=np.float64)
    codes = np.empty((len(points), depth + 1), dtype=np.int64)
    if len(points):
        lib(threaded).mpr_octree_codes_f64(_a(points), len(points), depth, _a(codes))
    return codes


def build_octree(points: np.ndarray, depth: int, threaded: bool = False) -> OracleTree:
    """core.py:86-127: per-level sorted unique codes, breadth-first, with
    parent / first-child / child-count links and each point's leaf node."""
    if not len(points):
        zero = np.zeros(1, np.int64)
        return OracleTree(zero, zero.copy(), np.full(1, -1, np.int64), np.full(1, -1, np.int64),
                          zero.copy(), np.empty(0, np.int64))
    codes = octree_codes(points, depth, threaded)
    per_level = []
    leaf_inverse = None
    for level in range(depth + 1):
        uniq, inverse = np.unique(codes[:, level], return_inverse=True)
        per_level.append(uniq)
        leaf_inverse = inverse
    sizes = [len(u) for u in per_level]
    starts = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    morton = np.concatenate(per_level).astype(np.int64)
    depths = np.repeat(np.arange(depth + 1, dtype=np.int64), sizes)
    parent = np.full(len(morton), -1, np.int64)
    child_start = np.full(len(morton), -1, np.int64)
    child_count = np.zeros(len(morton), np.int64)
    for level in range(1, depth + 1):
        # Each child's parent code is its own code without the last 3 bits;
        # parents are sorted, so a binary search finds their positions.
        child_codes = per_level[level]
        local_parent = np.searchsorted(per_level[level - 1], child_codes >> 3)
        nodes = starts[level] + np.arange(len(child_codes), dtype=np.int64)
        parents = starts[level - 1] + local_parent
        parent[nodes] = parents
        counts = np.bincount(local_parent, minlength=len(per_level[level - 1]))
        child_count[starts[level - 1]: starts[level]] = counts
        first = np.full(len(per_level[level - 1]), -1, np.int64)
        # children of one parent are contiguous; the first occurrence wins.
        seen = np.r_[True, local_parent[1:] != local_parent[:-1]]
        first[local_parent[seen]] = nodes[seen]
        child_start[starts[level - 1]: starts[level]] = first
    point_leaf = np.asarray(leaf_inverse, dtype=np.int64).reshape(-1) + starts[depth]
    return OracleTree(depths, morton, parent, child_start, child_count, point_leaf)


def restrict(fine: np.ndarray, threaded: bool = False) -> np.ndarray:
    cn = (fine.shape[0] + 1) // 2
    coarse = np.empty((cn, cn, cn))
    lib(threaded).mpr_restrict_f64(_a(fine), _a(coarse), fine.shape[0])
    return coarse


def _v_cycle(level, sol, rhs, scr, res, pw, pre, post, L):
    """core.py:141-193: recursive V(pre, post) with 40 sweeps at n <= 3."""
    n = sol[level].shape[0]
    if n <= 3:
        L.mpr_relax_f64(_a(sol[level]), _a(rhs[level]), _a(scr[level]), n, pw, 40)
        return
    L.mpr_relax_f64(_a(sol[level]), _a(rhs[level]), _a(scr[level]), n, pw, pre)
    L.mpr_residual_f64(_a(sol[level]), _a(rhs[level]), _a(scr[level]), _a(res[level]), n, pw)
    L.mpr_restrict_f64(_a(res[level]), _a(rhs[level + 1]), n)
    sol[level + 1].fill(0.0)
    _v_cycle(level + 1, sol, rhs, scr, res, pw, pre, post, L)
    L.mpr_prolong_add_f64(_a(sol[level + 1]), _a(sol[level]), n)
    L.mpr_relax_f64(_a(sol[level]), _a(rhs[level]), _a(scr[level]), n, pw, post)


def splat_and_assemble(points, normals, depth, point_weight, confidence, samples_per_node,
                       threaded=False):
    """core.py:228-265: zeroed grids, two-pass splat, density /= spn, RHS."""
    L = lib(threaded)
    n = (1 << depth) + 1
    density, vx, vy, vz, screen, rhs = (np.zeros((n, n, n)) for _ in range(6))
    if len(points):
        accepted = L.mpr_splat_f64(_a(points), _a(normals), len(points), n, int(confidence),
                                   _a(density), _a(vx), _a(vy), _a(vz), _a(screen),
                                   samples_per_node)
        if accepted != len(points):
            raise RuntimeError(f"oracle splat accepted {accepted} of {len(points)} samples")
        density /= samples_per_node
        L.mpr_assemble_f64(_a(vx), _a(vy), _a(vz), _a(screen), _a(rhs), n, point_weight, 0.5)
    return density, screen, rhs


def solve(points, normals, *, depth=6, point_weight=4.0, confidence=False, cycles=4,
          samples_per_node=1.5, tol=None, max_cycles=100, threaded=False, octree=True):
    """core.py:196-306 on already-validated unit-cube points.

    tol=None: exactly `cycles` V-cycles (the reference).  tol=t: V-cycles until
    ||rhs - A x||_2 / ||rhs||_2 <= t (at most max_cycles)."""
    L = lib(threaded)
    points = np.ascontiguousarray(points, dtype=np.float64)
    normals = np.ascontiguousarray(normals, dtype=np.float64)
    tree = build_octree(points, depth, threaded) if octree else None
    density, screen, rhs = splat_and_assemble(points, normals, depth, point_weight, confidence,
                                              samples_per_node, threaded)
    screens = [screen]
    while screens[-1].shape[0] > 3:
        screens.append(restrict(screens[-1], threaded) * 4.0)
    sol = [np.full_like(s, 0.5) for s in screens]
    rhs_levels = [np.zeros_like(s) for s in screens]
    res = [np.empty_like(s) for s in screens]
    rhs_levels[0][...] = rhs
    n = rhs.shape[0]
    cycles_run = 0
    rel = float("nan")
    if len(points):
        rhs_norm = float(np.sqrt(np.dot(rhs.ravel(), rhs.ravel())))
        if tol is None:
            for _ in range(cycles):
                _v_cycle(0, sol, rhs_levels, screens, res, point_weight, 3, 3, L)
            cycles_run = cycles
        else:
            while cycles_run < max_cycles:
                _v_cycle(0, sol, rhs_levels, screens, res, point_weight, 3, 3, L)
                cycles_run += 1
                norm = L.mpr_residual_f64(_a(sol[0]), _a(rhs), _a(screen), _a(res[0]), n,
                                          point_weight)
                rel = norm / rhs_norm if rhs_norm > 0 else 0.0
                if rel <= tol:
                    break
    else:
        sol[0].fill(0.0)
    residual_norm = L.mpr_residual_f64(_a(sol[0]), _a(rhs), _a(screen), _a(res[0]), n,
                                       point_weight)
    if len(points):
        rhs_norm = float(np.sqrt(np.dot(rhs.ravel(), rhs.ravel())))
        rel = residual_norm / rhs_norm if rhs_norm > 0 else 0.0
    iso = (L.mpr_iso_value_f64(_a(sol[0]), _a(points), _a(normals), len(points), n,
                               int(confidence)) if len(points) else 0.0)
    return OracleSolution(sol[0], density, screen, rhs, float(iso), float(residual_norm), tree,
                          cycles_run, rel)


def extract(field, iso_value=0.0, density=None, threaded=False) -> OracleMesh:
    """core.py:309-374: count, then emit vertices; count, then emit faces."""
    L = lib(threaded)
    field = np.ascontiguousarray(field, dtype=np.float64)
    density = np.zeros_like(field) if density is None else np.ascontiguousarray(density, np.float64)
    n = field.shape[0]
    cells = n - 1
    scratch = np.empty((cells + 3) // 4, np.int64)
    dummy_f = np.zeros(1)
    dummy_i = np.zeros(1, np.int64)
    count = L.mpr_dual_vertices_f64(_a(field), _a(density), n, iso_value, _a(scratch),
                                    _a(dummy_f), _a(dummy_f), 0)
    if count == 0:
        return OracleMesh(np.empty((0, 3)), np.empty((0, 3), np.int64), np.empty(0), iso_value)
    vertices = np.empty((count, 3))
    vdens = np.empty(count)
    cell_map = np.empty(cells**3, np.int64)
    written = L.mpr_dual_vertices_f64(_a(field), _a(density), n, iso_value, _a(cell_map),
                                      _a(vertices), _a(vdens), count)
    assert written == count
    fcount = L.mpr_dual_faces_f64(_a(field), n, iso_value, _a(cell_map), _a(dummy_i), 0)
    faces = np.empty((fcount, 3), np.int64)
    if fcount:
        L.mpr_dual_faces_f64(_a(field), n, iso_value, _a(cell_map), _a(faces), fcount)
    return OracleMesh(vertices, faces, vdens, iso_value)


def normalize(points: np.ndarray, scale: float):
    """core.py:377-385: bounding-box centre, widest extent times `scale`."""
    lo, hi = points.min(axis=0), points.max(axis=0)
    width = float(np.max(hi - lo)) * scale
    if not np.isfinite(width) or width <= 0:
        width = 1.0
    origin = 0.5 * (lo + hi) - 0.5 * width
    return np.ascontiguousarray((points - origin) / width), origin, width


def valid_rows(points: np.ndarray, normals: np.ndarray) -> np.ndarray:
    """core.py:73-83: finite rows with a non-zero, non-overflowing normal."""
    finite = np.isfinite(points).all(axis=1) & np.isfinite(normals).all(axis=1)
    scale = np.max(np.abs(normals), axis=1)
    rows = finite & (scale > 0)
    norm2 = np.zeros(len(normals))
    scaled = normals[rows] / scale[rows, None]
    norm2[rows] = np.einsum("ij,ij->i", scaled, scaled)
    return rows & np.isfinite(norm2) & (norm2 > 0)


def reconstruct(points, normals, *, depth=6, point_weight=4.0, confidence=False, cycles=4,
                scale=1.1, samples_per_node=1.5, tol=None, max_cycles=100, threaded=False,
                octree=True) -> OracleMesh:
    """core.py:388-426."""
    points = np.ascontiguousarray(points, dtype=np.float64)
    normals = np.ascontiguousarray(normals, dtype=np.float64)
    keep = valid_rows(points, normals)
    points, normals = points[keep], normals[keep]
    if not len(points):
        return OracleMesh(np.empty((0, 3)), np.empty((0, 3), np.int64), np.empty(0))
    unit, origin, width = normalize(points, scale)
    sol = solve(unit, normals, depth=depth, point_weight=point_weight, confidence=confidence,
                cycles=cycles, samples_per_node=samples_per_node, tol=tol,
                max_cycles=max_cycles, threaded=threaded, octree=octree)
    mesh = extract(sol.field, sol.iso_value, sol.density, threaded)
    return OracleMesh(np.ascontiguousarray(mesh.vertices * width + origin), mesh.faces,
                      mesh.density, sol.iso_value, sol.residual_norm)
