"""End-to-end parity of the public API on the GPU against the golden fixtures
made by the reference's own orchestration (tests/golden/pipeline_small.npz)
and against the CPU oracle.

FP64 mode at a fixed cycle count is bit-identical to the reference for the
field, density, screen, rhs and octree; the iso-value is a parallel sum and
agrees within 1e-12 relative (the north-star bar is 1e-9); mesh topology is
then identical and vertices agree within 1e-12."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_sphere_config_small_bit_exact(golden_pipeline):
    import mojo_poissonrecon_b200 as mpr

    g = golden_pipeline
    sol = mpr.solve_screened_poisson(g["sphere_unit_points"], g["sphere_points"], depth=5, cycles=5)
    for k in ("field", "density", "screen", "rhs"):
        assert np.array_equal(getattr(sol, k), g[f"sphere_{k}"]), k
    assert sol.iso_value == pytest.approx(float(g["sphere_iso"]), rel=1e-12)
    assert sol.residual_norm == pytest.approx(float(g["sphere_residual_norm"]), rel=1e-12)
    for k in ("depth", "morton", "parent", "child_start", "child_count", "point_leaf"):
        assert np.array_equal(getattr(sol.octree, k), g[f"sphere_octree_{k}"]), k


@pytest.mark.parametrize("case", ["sphere", "ellipsoid"])
def test_reconstruct_matches_golden_mesh(golden_pipeline, case):
    import mojo_poissonrecon_b200 as mpr

    g = golden_pipeline
    if case == "sphere":
        mesh = mpr.reconstruct(g["sphere_points"], g["sphere_points"], depth=5, cycles=5)
    else:
        mesh = mpr.reconstruct(g["ellipsoid_points"], g["ellipsoid_normals"], depth=4, cycles=3, confidence=True,
                               point_weight=2.0)
    assert np.array_equal(mesh.faces, g[f"{case}_mesh_faces"])
    assert np.allclose(mesh.vertices, g[f"{case}_mesh_vertices"], rtol=0, atol=1e-12)
    assert np.allclose(mesh.density, g[f"{case}_mesh_density"], rtol=0, atol=1e-12)
    assert mesh.iso_value == pytest.approx(float(g[f"{case}_mesh_iso"]), rel=1e-12)
    assert mesh.residual_norm == pytest.approx(float(g[f"{case}_mesh_residual_norm"]), rel=1e-12)


def test_tolerance_mode_matches_oracle(oracle):
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.torus(20_000, seed=11)
    keep = oracle.valid_rows(pts, nrm)
    unit, _, _ = oracle.normalize(pts[keep], 1.1)
    want = oracle.solve(unit, nrm[keep], depth=6, confidence=True, tol=1e-8, max_cycles=80, octree=False)
    got = mpr.solve_screened_poisson(unit, nrm[keep], depth=6, confidence=True, tol=1e-8, max_cycles=80)
    assert got.relative_residual <= 1e-8
    assert got.cycles == want.cycles_run
    assert np.array_equal(got.field, want.field)
    assert got.iso_value == pytest.approx(want.iso_value, rel=1e-12)


def test_empty_and_invalid_inputs():
    import mojo_poissonrecon_b200 as mpr

    empty = mpr.reconstruct(np.empty((0, 3)), np.empty((0, 3)))
    assert empty.is_empty and empty.faces.shape == (0, 3)
    pts = np.array([[0.1, 0.2, 0.3], [np.nan, 0, 0]])
    nrm = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    assert mpr.reconstruct(pts, nrm).is_empty  # every row dropped
    sol = mpr.solve_screened_poisson(pts, nrm, depth=3)
    assert not sol.field.any() and sol.iso_value == 0.0 and sol.residual_norm == 0.0
    assert sol.octree.node_count == 1
    with pytest.raises(ValueError, match="inside"):
        mpr.solve_screened_poisson(np.array([[1.5, 0.5, 0.5]]), np.array([[1.0, 0, 0]]))
    with pytest.raises(ValueError, match="finite"):
        mpr.build_octree(np.array([[np.nan, 0.5, 0.5]]))


def test_single_point_and_minimum_depth(oracle):
    import mojo_poissonrecon_b200 as mpr

    pts = np.array([[0.3, 0.6, 0.9]])
    nrm = np.array([[0.0, 0.0, 2.5]])
    for conf in (False, True):
        got = mpr.solve_screened_poisson(pts, nrm, depth=2, cycles=2, confidence=conf)
        want = oracle.solve(pts, nrm, depth=2, cycles=2, confidence=conf)
        assert np.array_equal(got.field, want.field)
        assert got.iso_value == pytest.approx(want.iso_value, rel=1e-13)


def test_watertight_sphere_like_reference():
    """tests/test_reconstruction.py:65-83 on the GPU path."""
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    points, _ = workloads.sphere(1200, seed=2)
    mesh = mpr.reconstruct(points, points, depth=5, cycles=5)
    edges = np.sort(np.concatenate([mesh.faces[:, [0, 1]], mesh.faces[:, [1, 2]], mesh.faces[:, [2, 0]]]), axis=1)
    _, counts = np.unique(edges, axis=0, return_counts=True)
    assert np.all(counts == 2)
    ext = mesh.vertices.max(axis=0) - mesh.vertices.min(axis=0)
    assert ext.max() / ext.min() < 1.04
    vol = abs(np.einsum("ij,ij->i", mesh.vertices[mesh.faces[:, 0]],
                        np.cross(mesh.vertices[mesh.faces[:, 1]], mesh.vertices[mesh.faces[:, 2]])).sum() / 6)
    assert vol == pytest.approx(4 * np.pi / 3, rel=0.04)
    assert mesh.residual_norm / np.linalg.norm(points) < 0.2


def test_reconstruct_mesh_nonempty():
    import mojo_poissonrecon_b200 as mpr

    v = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=np.float64)
    f = np.array([[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4], [2, 0, 5], [1, 2, 5], [3, 1, 5], [0, 3, 5]])
    mesh = mpr.reconstruct_mesh(v, f, depth=3, cycles=2)
    assert not mesh.is_empty and mesh.faces.shape[1] == 3


def test_device_out_returns_cuda_tensors():
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    pts, _ = workloads.sphere(500, seed=1)
    host = mpr.reconstruct(pts, pts, depth=4)
    devm = mpr.reconstruct(torch.from_numpy(pts).cuda(), torch.from_numpy(pts).cuda(), depth=4, device_out=True)
    assert devm.vertices.is_cuda and devm.faces.dtype == torch.int64
    assert np.array_equal(devm.faces.cpu().numpy(), host.faces)
    assert np.array_equal(devm.vertices.cpu().numpy(), host.vertices)


def test_repeatable_bits():
    """Same input twice gives the same bits (no atomics on any float path)."""
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.torus(30_000, seed=5)
    a = mpr.reconstruct(pts, nrm, depth=6, confidence=True)
    b = mpr.reconstruct(pts, nrm, depth=6, confidence=True)
    assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.faces, b.faces)
    assert a.iso_value == b.iso_value
