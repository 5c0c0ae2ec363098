"""Screened Poisson surface reconstruction on a B200 — the drop-in public API.

Same names, signatures, defaults, dataclasses, array shapes, [z, y, x] grid
layout, error types and messages as python/mojo_poissonrecon/core.py, so code
written against the reference runs unchanged.  Inputs may be NumPy arrays
(as in the reference) or torch tensors (CPU, pinned or CUDA); outputs are
NumPy arrays, or CUDA tensors with ``device_out=True``.

Extensions (keyword-only, defaults keep the reference's behaviour):
``precision`` ("fp64" | "fp32_refined" | "fp32_defect"), ``tol`` (stop on the relative
residual instead of a fixed cycle count), ``max_cycles``, ``device_out``.
The depth cap is lifted from 8 to 10.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _native as nat
from . import _sync, _trace, solver
from ._convert import f64, i64

MAX_DEPTH = 10
PINNED_LIMIT = 1 << 30  # bytes; larger results are copied to pageable memory
# fp32_refined: FP64 FCG(1) preconditioned by FP32 V-cycles; fp32_defect: plain
# FP64 defect correction x += V(r) with FP32 V-cycles.
PRECISIONS = ("fp64", "fp32_refined", "fp32_defect")


@dataclass(frozen=True)
class FlatOctree:
    depth: np.ndarray
    morton: np.ndarray
    parent: np.ndarray
    child_start: np.ndarray
    child_count: np.ndarray
    point_leaf: np.ndarray

    @property
    def node_count(self) -> int:
        return int(self.depth.shape[0])


@dataclass(frozen=True)
class GridSolution:
    field: np.ndarray
    density: np.ndarray
    screen: np.ndarray
    rhs: np.ndarray
    iso_value: float
    residual_norm: float
    octree: FlatOctree | None
    cycles: int = 0
    relative_residual: float = float("nan")
    precision: str = "fp64"


@dataclass(frozen=True)
class Mesh:
    vertices: np.ndarray
    faces: np.ndarray
    density: np.ndarray
    iso_value: float = 0.0
    residual_norm: float = 0.0

    @property
    def is_empty(self) -> bool:
        return self.vertices.shape[0] == 0


# ---- validation (core.py:50-83, 207-227) --------------------------------------

def _points(values):
    result = f64(values)
    if result.ndim != 2 or result.shape[1] != 3:
        raise ValueError("points must have shape (n, 3)")
    return result


def _integer_parameter(name: str, value) -> int:
    if isinstance(value, (bool, np.bool_)) or not isinstance(value, (int, np.integer)):
        raise TypeError(f"{name} must be an integer")
    return int(value)


def _finite_parameter(name: str, value) -> float:
    try:
        result = float(value)
    except (TypeError, ValueError, OverflowError) as error:
        raise TypeError(f"{name} must be a real number") from error
    if not np.isfinite(result):
        raise ValueError(f"{name} must be finite")
    return result


def _precision(value: str) -> str:
    if value not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}")
    return value


def _tolerance(tol) -> float | None:
    if tol is None:
        return None
    tol = _finite_parameter("tol", tol)
    if tol <= 0:
        raise ValueError("tol must be positive")
    return tol


class _Context:
    """Per-call device state: the device, a workspace and the stream handle."""

    def __init__(self):
        self.device = nat.require_cuda()
        self.lib = nat.lib()
        self.ws = nat.Workspace(self.device)
        self.stream = nat.stream_handle()

    def check(self, status: int, what: str) -> None:
        nat.check(status, what)


def _to_device(array, device: torch.device) -> torch.Tensor:
    if isinstance(array, torch.Tensor):
        return array.to(device=device, dtype=torch.float64, non_blocking=True).contiguous()
    return torch.from_numpy(np.ascontiguousarray(array, dtype=np.float64)).to(device, non_blocking=True)


def _host_all(tensors, device_out: bool) -> list:
    """Results to NumPy: asynchronous copies into ONE pinned buffer on the
    current stream (64-byte aligned slices, one pinned allocation however many
    arrays), one synchronisation for all (pageable .cpu() copies are several
    times slower and synchronise each).  Arrays above PINNED_LIMIT bytes (the
    grids of deep solves) use pageable copies.  The returned arrays are views
    of the shared buffer, which lives as long as any of them."""
    if device_out:
        return list(tensors)
    slots, total = [], 0
    for t in tensors:
        nbytes = t.numel() * t.element_size()
        if t.is_cuda and 0 < nbytes <= PINNED_LIMIT:
            slots.append(total)
            total += (nbytes + 63) // 64 * 64
        else:
            slots.append(-1)
    buf = None
    if total:
        try:
            buf = torch.empty(total, dtype=torch.uint8, pin_memory=True)
        except RuntimeError:  # page-locked memory refused: pageable copies instead
            slots = [-1] * len(slots)
    out = []
    for t, off in zip(tensors, slots):
        if off >= 0:
            h = buf[off:off + t.numel() * t.element_size()].view(t.dtype).view(t.shape)
            h.copy_(t, non_blocking=True)
            out.append(h)
        else:
            out.append(t.cpu())
    _sync.wait("result copies")
    torch.cuda.current_stream().synchronize()
    return [h.numpy() for h in out]


def _prepare(ctx: _Context, points: torch.Tensor, normals: torch.Tensor, scale: float):
    """Valid rows (core.py:73-83), optionally mapped to the unit cube (:377-385).
    Returns (points, normals, kept, map) with the kept rows only."""
    count = points.shape[0]
    out_p = torch.empty_like(points)
    out_n = torch.empty_like(normals)
    kept = torch.empty(1, dtype=torch.int64, device=ctx.device)
    fmap = torch.empty(4, dtype=torch.float64, device=ctx.device)
    ptr, size = ctx.ws.get(ctx.lib.pb_prepare_workspace_size(count))
    ctx.check(ctx.lib.pb_prepare_points_f64(points.data_ptr(), normals.data_ptr(), count, scale, out_p.data_ptr(),
                                            out_n.data_ptr(), kept.data_ptr(), fmap.data_ptr(), ptr, size,
                                            ctx.stream), "prepare points")
    _sync.wait("prepare points")
    k = int(kept.item())
    return out_p[:k], out_n[:k], k, fmap


# ---- octree (core.py:86-127) ---------------------------------------------------

def _octree_device(ctx: _Context, points: torch.Tensor, depth: int) -> dict:
    count = points.shape[0]
    L = ctx.lib
    if count == 0:
        z = torch.zeros(1, dtype=torch.int64, device=ctx.device)
        m1 = torch.full((1,), -1, dtype=torch.int64, device=ctx.device)
        return dict(depth=z, morton=z.clone(), parent=m1, child_start=m1.clone(), child_count=z.clone(),
                    point_leaf=torch.empty(0, dtype=torch.int64, device=ctx.device))
    ws = nat.Workspace(ctx.device)  # kept alive across the two phases
    ptr, size = ws.get(L.pb_octree_workspace_size(count, depth))
    counts = torch.empty(depth + 1, dtype=torch.int64, device=ctx.device)
    ctx.check(L.pb_octree_count(points.data_ptr(), count, depth, counts.data_ptr(), ptr, size, ctx.stream),
              "octree count")
    nodes = int(counts.sum().item())
    arrays = {k: torch.empty(nodes, dtype=torch.int64, device=ctx.device)
              for k in ("depth", "morton", "parent", "child_start", "child_count")}
    arrays["point_leaf"] = torch.empty(count, dtype=torch.int64, device=ctx.device)
    ctx.check(L.pb_octree_emit(count, depth, counts.data_ptr(), nodes, arrays["depth"].data_ptr(),
                               arrays["morton"].data_ptr(), arrays["parent"].data_ptr(),
                               arrays["child_start"].data_ptr(), arrays["child_count"].data_ptr(),
                               arrays["point_leaf"].data_ptr(), ptr, size, ctx.stream), "octree emit")
    return arrays


def _octree_out(arrays: dict, device_out: bool) -> FlatOctree:
    return FlatOctree(*_host_all([arrays[k] for k in
                                  ("depth", "morton", "parent", "child_start", "child_count", "point_leaf")],
                                 device_out))


def build_octree(points, depth: int = 6, *, device_out: bool = False) -> FlatOctree:
    """Build a compact breadth-first Morton octree over unit-cube points."""
    points = _points(points)
    depth = _integer_parameter("depth", depth)
    if not 0 <= depth <= 19:
        raise ValueError("depth must be between 0 and 19")
    ctx = _Context()
    dpts = _to_device(points, ctx.device)
    if dpts.shape[0]:
        bad = (~torch.isfinite(dpts)).any() | (dpts < 0).any() | (dpts > 1).any()
        if bool(bad):
            raise ValueError("octree points must be finite and inside [0, 1]^3")
    return _octree_out(_octree_device(ctx, dpts, depth), device_out)


# ---- solve (core.py:196-306) ---------------------------------------------------

def _splat_assemble(ctx: _Context, points: torch.Tensor, normals: torch.Tensor, depth: int, point_weight: float,
                    confidence: bool, samples_per_node: float):
    L = ctx.lib
    n = (1 << depth) + 1
    count = points.shape[0]
    grids = {k: torch.empty((n, n, n), dtype=torch.float64, device=ctx.device)
             for k in ("density", "vx", "vy", "vz", "screen", "rhs")}
    # the splat accumulates into zeroed grids (core.py:229-236); assembly writes every rhs node
    for k in ("density", "vx", "vy", "vz", "screen") if count else grids:
        ctx.check(L.pb_fill_f64(grids[k].data_ptr(), n ** 3, 0.0, ctx.stream), "zero grid")
    accepted = torch.zeros(1, dtype=torch.int64, device=ctx.device)
    if count:
        ptr, size = ctx.ws.get(L.pb_splat_workspace_size(count, n))
        ctx.check(L.pb_splat_f64(points.data_ptr(), normals.data_ptr(), count, n, int(confidence),
                                 grids["density"].data_ptr(), grids["vx"].data_ptr(), grids["vy"].data_ptr(),
                                 grids["vz"].data_ptr(), grids["screen"].data_ptr(), samples_per_node,
                                 accepted.data_ptr(), ptr, size, ctx.stream), "splat")
        ctx.check(L.pb_divide_f64(grids["density"].data_ptr(), n ** 3, samples_per_node, ctx.stream), "divide")
        ctx.check(L.pb_assemble_f64(grids["vx"].data_ptr(), grids["vy"].data_ptr(), grids["vz"].data_ptr(),
                                    grids["screen"].data_ptr(), grids["rhs"].data_ptr(), n, point_weight, 0.5,
                                    ctx.stream), "assemble")
    for k in ("vx", "vy", "vz"):
        del grids[k]
    return grids, accepted


def _iso_value(ctx: _Context, field: torch.Tensor, points: torch.Tensor, normals: torch.Tensor,
               confidence: bool) -> torch.Tensor:
    iso = torch.zeros(1, dtype=torch.float64, device=ctx.device)
    count = points.shape[0]
    if count:
        ptr, size = ctx.ws.get(ctx.lib.pb_iso_value_workspace_size(count))
        ctx.check(ctx.lib.pb_iso_value_f64(field.data_ptr(), points.data_ptr(), normals.data_ptr(), count,
                                           field.shape[0], int(confidence), iso.data_ptr(), ptr, size, ctx.stream),
                  "iso value")
    return iso


def _solve_device(ctx: _Context, points: torch.Tensor, normals: torch.Tensor, *, depth: int, point_weight: float,
                  confidence: bool, cycles: int, samples_per_node: float, precision: str, tol, max_cycles: int,
                  octree: bool, refine_method: str = "fcg"):
    with _trace.stage("octree"):
        tree = _octree_device(ctx, points, depth) if octree else None
    with _trace.stage("splat"):
        grids, accepted = _splat_assemble(ctx, points, normals, depth, point_weight, confidence, samples_per_node)
    ctx.ws = nat.Workspace(ctx.device)  # the splat's scratch (GBs at 20M points) is not needed past here
    count = points.shape[0]
    with _trace.stage("solve"):
        if precision == "fp64":
            field, stats = solver.solve_fp64(grids["rhs"], grids["screen"], point_weight, ctx.ws, cycles=cycles,
                                             tol=tol, max_cycles=max_cycles, has_points=count > 0)
        else:
            from . import solver32
            field, stats = solver32.solve_refined(grids["rhs"], grids["screen"], point_weight, ctx.ws,
                                                  tol=1e-8 if tol is None else tol, max_cycles=max_cycles,
                                                  has_points=count > 0,
                                                  method="defect" if precision == "fp32_defect" else refine_method)
    with _trace.stage("iso"):
        iso = _iso_value(ctx, field, points, normals, confidence)
    if count and int(accepted.item()) != count:
        raise RuntimeError(f"splat accepted {int(accepted.item())} of {count} validated samples")
    return field, grids, iso, stats, tree


def solve_screened_poisson(
    points,
    normals,
    *,
    depth: int = 6,
    point_weight: float = 4.0,
    confidence: bool = False,
    cycles: int = 4,
    samples_per_node: float = 1.5,
    precision: str = "fp64",
    tol: float | None = None,
    max_cycles: int = 200,
    device_out: bool = False,
) -> GridSolution:
    """Build the octree, splat samples, and solve the screened Poisson system."""
    points = _points(points)
    normals = _points(normals)
    if tuple(points.shape) != tuple(normals.shape):
        raise ValueError("points and normals must have the same shape")
    depth = _integer_parameter("depth", depth)
    cycles = _integer_parameter("cycles", cycles)
    max_cycles = _integer_parameter("max_cycles", max_cycles)
    point_weight = _finite_parameter("point_weight", point_weight)
    samples_per_node = _finite_parameter("samples_per_node", samples_per_node)
    precision = _precision(precision)
    tol = _tolerance(tol)
    if not 2 <= depth <= MAX_DEPTH:
        raise ValueError(f"depth must be between 2 and {MAX_DEPTH}")
    if cycles < 1:
        raise ValueError("cycles must be positive")
    if point_weight < 0 or samples_per_node <= 0:
        raise ValueError("point_weight must be non-negative and samples_per_node positive")
    ctx = _Context()
    dp = _to_device(points, ctx.device)
    dn = _to_device(normals, ctx.device)
    if dp.shape[0]:
        dp, dn, count, _ = _prepare(ctx, dp, dn, 0.0)
        if count:
            outside = torch.zeros(1, dtype=torch.int32, device=ctx.device)
            ctx.check(ctx.lib.pb_unit_cube_check_f64(dp.data_ptr(), count, outside.data_ptr(), ctx.stream),
                      "unit cube check")
            if int(outside.item()):
                raise ValueError("solver points must be inside [0, 1]^3")
    field, grids, iso, stats, tree = _solve_device(
        ctx, dp, dn, depth=depth, point_weight=point_weight, confidence=confidence, cycles=cycles,
        samples_per_node=samples_per_node, precision=precision, tol=tol, max_cycles=max_cycles, octree=True)
    out = _host_all([field, grids["density"], grids["screen"], grids["rhs"], iso], device_out)
    iso_value = float(out[4][0])
    return GridSolution(out[0], out[1], out[2], out[3], iso_value, float(stats.residual_norm),
                        _octree_out(tree, device_out), stats.cycles, stats.relative_residual, precision)


# ---- extraction (core.py:309-374) --------------------------------------------

EXTRACT_FAST_MAX_SIDE = 1025


def _extract_device(ctx: _Context, field: torch.Tensor, density: torch.Tensor, iso: torch.Tensor):
    """Dual contouring on device tensors; returns (vertices, faces, vdens).

    Sides up to 1025 use the bit-array extraction (count, one host read of the
    two counts, emit); larger ones the reference-shaped two-pass entry points.
    Both give the reference's mesh (capi.mojo:798-1129) bit for bit."""
    L = ctx.lib
    n = field.shape[0]
    if n <= EXTRACT_FAST_MAX_SIDE:
        ptr, size = ctx.ws.get(L.pb_extract_workspace_size(n))
        counts = torch.empty(2, dtype=torch.int64, device=ctx.device)
        ctx.check(L.pb_extract_count_f64(field.data_ptr(), n, iso.data_ptr(), counts.data_ptr(), ptr, size,
                                         ctx.stream), "extract count")
        _sync.wait("extract count")
        nv, nf = (int(v) for v in counts.cpu())
        vertices = torch.empty((nv, 3), dtype=torch.float64, device=ctx.device)
        vdens = torch.empty(nv, dtype=torch.float64, device=ctx.device)
        faces = torch.empty((nf, 3), dtype=torch.int64, device=ctx.device)
        if nv:
            ctx.check(L.pb_extract_emit_f64(field.data_ptr(), density.data_ptr(), n, iso.data_ptr(),
                                            vertices.data_ptr(), vdens.data_ptr(), faces.data_ptr() if nf else None,
                                            ptr, size, ctx.stream), "extract emit")
        return vertices, faces, vdens
    cells = n - 1
    ptr, size = ctx.ws.get(L.pb_dual_workspace_size(n))
    count = torch.zeros(1, dtype=torch.int64, device=ctx.device)
    ctx.check(L.pb_dual_vertices_f64_isoptr(field.data_ptr(), density.data_ptr(), n, iso.data_ptr(), None, None,
                                            None, 0, count.data_ptr(), ptr, size, ctx.stream), "dual count")
    nv = int(count.item())
    if nv < 0 or nv > cells ** 3:
        raise RuntimeError(f"invalid dual vertex count: {nv}")
    if nv == 0:
        empty = torch.empty((0, 3), dtype=torch.float64, device=ctx.device)
        return empty, torch.empty((0, 3), dtype=torch.int64, device=ctx.device), torch.empty(
            0, dtype=torch.float64, device=ctx.device)
    vertices = torch.empty((nv, 3), dtype=torch.float64, device=ctx.device)
    vdens = torch.empty(nv, dtype=torch.float64, device=ctx.device)
    cell_map = torch.empty(cells ** 3, dtype=torch.int64, device=ctx.device)
    ctx.check(L.pb_dual_vertices_f64_isoptr(field.data_ptr(), density.data_ptr(), n, iso.data_ptr(),
                                            cell_map.data_ptr(), vertices.data_ptr(), vdens.data_ptr(), nv,
                                            count.data_ptr(), ptr, size, ctx.stream), "dual vertices")
    fcount = torch.zeros(1, dtype=torch.int64, device=ctx.device)
    ctx.check(L.pb_dual_faces_f64_isoptr(field.data_ptr(), n, iso.data_ptr(), cell_map.data_ptr(), None, 0,
                                         fcount.data_ptr(), ptr, size, ctx.stream), "dual face count")
    pair = torch.stack([count, fcount]).cpu()
    if int(pair[0]) != nv:
        raise RuntimeError("dual vertex count changed between extraction passes")
    nf = int(pair[1])
    if nf < 0 or nf > 6 * cells ** 3:
        raise RuntimeError(f"invalid dual face count: {nf}")
    faces = torch.empty((nf, 3), dtype=torch.int64, device=ctx.device)
    if nf:
        ctx.check(L.pb_dual_faces_f64_isoptr(field.data_ptr(), n, iso.data_ptr(), cell_map.data_ptr(),
                                             faces.data_ptr(), nf, fcount.data_ptr(), ptr, size, ctx.stream),
                  "dual faces")
    del cell_map
    return vertices, faces, vdens


def extract_isosurface(field, *, iso_value: float = 0.0, density=None, device_out: bool = False) -> Mesh:
    """Extract a triangle mesh from a cubic scalar grid on the dual grid."""
    field = f64(field)
    if field.ndim != 3 or len(set(tuple(field.shape))) != 1 or field.shape[0] < 2:
        raise ValueError("field must be a cubic array with side length >= 2")
    iso_value = _finite_parameter("iso_value", iso_value)

    def all_finite(values) -> bool:
        if isinstance(values, np.ndarray):
            return bool(np.isfinite(values).all())
        return bool(torch.isfinite(values).all())

    if not all_finite(field):
        raise ValueError("field and iso_value must be finite")
    if density is not None:
        density = f64(density)
        if tuple(density.shape) != tuple(field.shape):
            raise ValueError("density must have the same shape as field")
        if not all_finite(density):
            raise ValueError("density must be finite")
    ctx = _Context()
    dfield = _to_device(field, ctx.device)
    ddens = torch.zeros_like(dfield) if density is None else _to_device(density, ctx.device)
    iso = torch.full((1,), iso_value, dtype=torch.float64, device=ctx.device)
    v, f, d = _extract_device(ctx, dfield, ddens, iso)
    return Mesh(*_host_all([v, f, d], device_out), iso_value)


# ---- reconstruct (core.py:388-455) ----------------------------------------------

def reconstruct(
    points,
    normals,
    *,
    depth: int = 6,
    point_weight: float = 4.0,
    confidence: bool = False,
    cycles: int = 4,
    scale: float = 1.1,
    samples_per_node: float = 1.5,
    precision: str = "fp64",
    tol: float | None = None,
    max_cycles: int = 200,
    device_out: bool = False,
) -> Mesh:
    """Reconstruct a watertight surface from oriented points."""
    points = _points(points)
    normals = _points(normals)
    if tuple(points.shape) != tuple(normals.shape):
        raise ValueError("points and normals must have the same shape")
    scale = _finite_parameter("scale", scale)
    if scale <= 1.0:
        raise ValueError("scale must be greater than 1")
    depth = _integer_parameter("depth", depth)
    cycles = _integer_parameter("cycles", cycles)
    max_cycles = _integer_parameter("max_cycles", max_cycles)
    point_weight = _finite_parameter("point_weight", point_weight)
    samples_per_node = _finite_parameter("samples_per_node", samples_per_node)
    precision = _precision(precision)
    tol = _tolerance(tol)
    if not 2 <= depth <= MAX_DEPTH:
        raise ValueError(f"depth must be between 2 and {MAX_DEPTH}")
    if cycles < 1:
        raise ValueError("cycles must be positive")
    if point_weight < 0 or samples_per_node <= 0:
        raise ValueError("point_weight must be non-negative and samples_per_node positive")

    def empty() -> Mesh:
        if device_out:
            dev = nat.require_cuda()
            return Mesh(torch.empty((0, 3), dtype=torch.float64, device=dev),
                        torch.empty((0, 3), dtype=torch.int64, device=dev),
                        torch.empty(0, dtype=torch.float64, device=dev))
        return Mesh(np.empty((0, 3), np.float64), np.empty((0, 3), np.int64), np.empty(0))

    if points.shape[0] == 0:
        return empty()
    ctx = _Context()
    with _trace.stage("prepare"):
        dp, dn, count, fmap = _prepare(ctx, _to_device(points, ctx.device), _to_device(normals, ctx.device), scale)
    if count == 0:
        return empty()
    # The reference also builds the octree here and discards it; it feeds no output.
    field, grids, iso, stats, _ = _solve_device(
        ctx, dp, dn, depth=depth, point_weight=point_weight, confidence=confidence, cycles=cycles,
        samples_per_node=samples_per_node, precision=precision, tol=tol, max_cycles=max_cycles, octree=False)
    with _trace.stage("extract"):
        vertices, faces, vdens = _extract_device(ctx, field, grids["density"], iso)
        ctx.check(ctx.lib.pb_map_vertices_f64(vertices.data_ptr(), vertices.shape[0], fmap.data_ptr(),
                                              ctx.stream), "map vertices")
    with _trace.stage("copy-out"):
        v, f, d, iso_h = _host_all([vertices, faces, vdens, iso], device_out)
    return Mesh(v, f, d, float(iso_h[0]), float(stats.residual_norm))


# ---- mesh input (core.py:429-455) -------------------------------------------

def _oriented_points_device(vertices, faces) -> tuple[torch.Tensor, torch.Tensor]:
    """core.py:429-451 on the device (csrc/mesh.cu): referenced vertices and their
    area-weighted unit normals, bit-identical to the reference's per-face loop."""
    vertices = _points(vertices)
    faces = i64(faces)
    if faces.ndim != 2 or faces.shape[1] != 3:
        raise ValueError("faces must have shape (m, 3)")
    if isinstance(faces, np.ndarray) and len(faces) and (faces.min() < 0 or faces.max() >= len(vertices)):
        raise ValueError("face index out of range")  # device inputs are checked by the kernel
    if len(faces) == 0 or len(vertices) == 0:  # nothing is referenced: no device work
        empty = torch.empty((0, 3), dtype=torch.float64)
        return empty, empty.clone()
    ctx = _Context()
    dv = _to_device(vertices, ctx.device)
    df = faces.to(ctx.device).contiguous() if isinstance(faces, torch.Tensor) else \
        torch.from_numpy(np.ascontiguousarray(faces)).to(ctx.device)
    nv, nf = dv.shape[0], df.shape[0]
    L = ctx.lib
    ptr, size = ctx.ws.get(L.pb_mesh_normals_workspace_size(nv, nf))
    counts = torch.empty(2, dtype=torch.int64, device=ctx.device)
    ctx.check(L.pb_mesh_normals_count_f64(dv.data_ptr() if nv else None, nv, df.data_ptr() if nf else None, nf,
                                          counts.data_ptr(), ptr, size, ctx.stream), "mesh normals count")
    kept, bad = (int(c) for c in counts.cpu())
    if bad:
        raise ValueError("face index out of range")
    points = torch.empty((kept, 3), dtype=torch.float64, device=ctx.device)
    normals = torch.empty((kept, 3), dtype=torch.float64, device=ctx.device)
    if kept:
        ctx.check(L.pb_mesh_normals_emit_f64(dv.data_ptr(), nv, df.data_ptr() if nf else None, nf,
                                             points.data_ptr(), normals.data_ptr(), ptr, size, ctx.stream),
                  "mesh normals emit")
    return points, normals


def oriented_points_from_mesh(vertices, faces):
    """Return referenced vertices and area-weighted normals from a triangle mesh."""
    points, normals = _oriented_points_device(vertices, faces)
    return points.cpu().numpy(), normals.cpu().numpy()


def reconstruct_mesh(vertices, faces, **kwargs) -> Mesh:
    points, normals = _oriented_points_device(vertices, faces)
    return reconstruct(points, normals, **kwargs)
