"""Auxiliary attribute interpolation onto reconstructed meshes.

Upstream PoissonRecon carries per-sample attributes (colours, typically) onto
the output mesh; the reference leaves this out (README.md:31-36).  Here each
sample's attributes are splatted on the device with the sample's pass-1
weights w (the screening weights of `reconstruct` at the same depth and
scale), summed per grid node in sample order, and a mesh vertex takes the
ratio of the trilinear interpolants of sum w a and sum w over its cell
(csrc/splat.cu: pb_splat_attributes_f64, pb_sample_attributes_f64).
"""

from __future__ import annotations

import numpy as np
import torch

from . import core
from ._convert import f64


def interpolate_attributes(points, normals, attributes, vertices, *, depth: int = 6, confidence: bool = False,
                           scale: float = 1.1, device_out: bool = False):
    """Values of per-point `attributes` ((n,) or (n, k) for n points) at mesh
    `vertices` ((m, 3), world coordinates, e.g. `reconstruct(points, normals,
    depth=depth, scale=scale).vertices`).  Returns (m,) or (m, k) float64 (CUDA
    tensors with device_out=True); 0 at a vertex whose cell no sample's weight
    reaches.  Every (point, normal) row must be valid (finite point, finite
    non-zero normal) so that attributes stay aligned with the samples."""
    points = core._points(points)
    normals = core._points(normals)
    if tuple(points.shape) != tuple(normals.shape):
        raise ValueError("points and normals must have the same shape")
    values = f64(attributes)
    one_d = values.ndim == 1
    if one_d:
        values = values.reshape(-1, 1)
    if values.ndim != 2 or values.shape[0] != points.shape[0] or not 1 <= values.shape[1] <= 64:
        raise ValueError("attributes must have shape (n,) or (n, k) with n points and 1 <= k <= 64")
    vertices = core._points(vertices)
    depth = core._integer_parameter("depth", depth)
    if not 2 <= depth <= core.MAX_DEPTH:
        raise ValueError(f"depth must be between 2 and {core.MAX_DEPTH}")
    scale = core._finite_parameter("scale", scale)
    if scale <= 1.0:
        raise ValueError("scale must be greater than 1")
    channels, nv = int(values.shape[1]), int(vertices.shape[0])

    ctx = core._Context()
    L = ctx.lib
    if points.shape[0] == 0:
        raise ValueError("no points to interpolate from")
    dp, dn, count, fmap = core._prepare(ctx, core._to_device(points, ctx.device), core._to_device(normals, ctx.device),
                                        scale)
    if count != points.shape[0]:
        raise ValueError(f"{points.shape[0] - count} (point, normal) rows are invalid; drop them (and their "
                         "attributes) first")
    n = (1 << depth) + 1
    grids = torch.empty((channels + 1, n, n, n), dtype=torch.float64, device=ctx.device)
    attrs = core._to_device(values, ctx.device)
    ptr, size = ctx.ws.get(L.pb_splat_attributes_workspace_size(count))
    ctx.check(L.pb_splat_attributes_f64(dp.data_ptr(), dn.data_ptr(), count, n, int(bool(confidence)),
                                        attrs.data_ptr(), channels, grids.data_ptr(), ptr, size, ctx.stream),
              "splat attributes")
    verts = core._to_device(vertices, ctx.device)
    out = torch.empty((nv, channels), dtype=torch.float64, device=ctx.device)
    ctx.check(L.pb_sample_attributes_f64(verts.data_ptr() if nv else None, nv, fmap.data_ptr(), n, grids.data_ptr(),
                                         channels, out.data_ptr() if nv else None, ctx.stream),
              "sample attributes")
    result = core._host_all([out], device_out)[0]
    if one_d:
        result = result[:, 0] if device_out else np.ascontiguousarray(result[:, 0])
    return result
