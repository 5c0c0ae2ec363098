"""Auxiliary attribute interpolation (mojo_poissonrecon_b200/attributes.py,
csrc/splat.cu) against a NumPy restatement of its definition: per-sample
attributes splatted with the pass-1 weights (capi.mojo:139-172's cell and
weights), summed per node in sample order, and sampled at the vertices as the
ratio of the trilinear interpolants of sum w a and sum w.  The restatement runs
the same FP64 operations in the same order on the device's unit-cube points,
so the tolerance is 1e-12 relative (the sums agree to rounding)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda")


def _norm3(x, y, z):
    scale = max(abs(x), abs(y), abs(z))
    if scale == 0.0:
        return 0.0
    sx, sy, sz = x / scale, y / scale, z / scale
    return scale * np.sqrt(sx * sx + sy * sy + sz * sz)


def _cell1(p, res):  # pass-1 cell and fraction
    g = p * res
    i = int(g)
    if i < 0:
        i = 0
    if i >= res:
        i, g = res - 1, float(res)
    return i, g - i


def _cell2(p, res):  # pass-2 cell and fraction, clamped
    g = p * res
    i = min(max(int(g), 0), res - 1)
    return i, min(max(g - i, 0.0), 1.0)


def restated(unit_points, normals, attrs, vertices, fmap, n, confidence):
    res = n - 1
    k = attrs.shape[1]
    grids = np.zeros((k + 1, n * n * n))
    for p in range(len(unit_points)):
        sw = _norm3(*normals[p]) if confidence else 1.0
        (ix, fx), (iy, fy), (iz, fz) = (_cell1(unit_points[p, a], res) for a in range(3))
        for dz in range(2):
            wz = fz if dz else 1.0 - fz
            for dy in range(2):
                wy = fy if dy else 1.0 - fy
                for dx in range(2):
                    wx = fx if dx else 1.0 - fx
                    w = wx * wy * wz * sw
                    node = ((iz + dz) * n + iy + dy) * n + ix + dx
                    for c in range(k):
                        grids[c, node] += w * attrs[p, c]
                    grids[k, node] += w
    out = np.zeros((len(vertices), k))
    for v in range(len(vertices)):
        cells = [_cell2((vertices[v, a] - fmap[a]) / fmap[3], res) for a in range(3)]
        (ix, fx), (iy, fy), (iz, fz) = cells
        acc = np.zeros(k + 1)
        for c in range(k + 1):
            for dz in range(2):
                wz = fz if dz else 1.0 - fz
                for dy in range(2):
                    wy = fy if dy else 1.0 - fy
                    for dx in range(2):
                        wx = fx if dx else 1.0 - fx
                        acc[c] += grids[c, ((iz + dz) * n + iy + dy) * n + ix + dx] * wx * wy * wz
        out[v] = acc[:k] / acc[k] if acc[k] > 0 else 0.0
    return out


@pytest.mark.parametrize("confidence", [False, True])
def test_matches_restatement(cuda, confidence):
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import core, workloads

    pts, nrm = workloads.sphere(1500, seed=5)
    rng = np.random.default_rng(6)
    nrm = nrm * rng.uniform(0.5, 2.0, size=(len(nrm), 1))  # confidence weights differ per sample
    attrs = np.column_stack([pts[:, 0] * 100.0, rng.random(len(pts))])
    depth = 4
    mesh = mpr.reconstruct(pts, nrm, depth=depth, confidence=confidence)
    got = mpr.interpolate_attributes(pts, nrm, attrs, mesh.vertices, depth=depth, confidence=confidence)
    ctx = core._Context()
    dp, dn, count, fmap = core._prepare(ctx, core._to_device(pts, cuda), core._to_device(nrm, cuda), 1.1)
    want = restated(dp.cpu().numpy(), dn.cpu().numpy(), attrs, mesh.vertices, fmap.cpu().numpy(),
                    (1 << depth) + 1, confidence)
    assert got.shape == want.shape == (len(mesh.vertices), 2)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_constant_attribute_and_shapes(cuda):
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.sphere(2000, seed=7)
    mesh = mpr.reconstruct(pts, nrm, depth=5)
    got = mpr.interpolate_attributes(pts, nrm, np.full(len(pts), 3.25), mesh.vertices, depth=5)
    assert got.shape == (len(mesh.vertices),)
    reached = got != 0.0  # vertices whose cell some sample's weight reaches
    assert reached.mean() > 0.9
    assert np.abs(got[reached] - 3.25).max() <= 1e-12
    dev = mpr.interpolate_attributes(pts, nrm, np.full(len(pts), 3.25), mesh.vertices, depth=5, device_out=True)
    assert dev.is_cuda and torch.equal(dev.cpu(), torch.from_numpy(got))


def test_rejects_invalid_rows_and_shapes(cuda):
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.sphere(200, seed=8)
    bad = nrm.copy()
    bad[3] = 0.0
    with pytest.raises(ValueError):
        mpr.interpolate_attributes(pts, bad, np.ones(200), pts, depth=4)
    with pytest.raises(ValueError):
        mpr.interpolate_attributes(pts, nrm, np.ones(199), pts, depth=4)
    with pytest.raises(ValueError):
        mpr.interpolate_attributes(pts, nrm, np.ones((200, 65)), pts, depth=4)
