"""oriented_points_from_mesh / reconstruct_mesh on the device (csrc/mesh.cu)
against the reference's per-face loop (core.py:429-451, restated below):
identical arrays, bit for bit."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import mojo_poissonrecon_b200 as mpr  # noqa: E402


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


EMPTY = (np.empty((0, 3)), np.empty((0, 3), dtype=np.int64), 0)
SINGLE = (np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0]]), np.array([[0, 1, 2]]), 3)
DUPLICATE = (np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 0]]), np.array([[0, 1, 2], [3, 1, 2]]), 4)
ZERO_AREA = (np.array([[0.0, 0, 0], [1, 0, 0], [2, 0, 0]]), np.array([[0, 1, 2]]), 0)
NON_MANIFOLD = (np.array([[0.0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, -1, 0], [0.5, 0, 1]]),
                np.array([[0, 1, 2], [1, 0, 3], [0, 1, 4]]), 5)
UNREFERENCED = (np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [9, 9, 9]]), np.array([[0, 1, 2]]), 3)


@pytest.mark.parametrize("vertices,faces,expected", [EMPTY, SINGLE, DUPLICATE, ZERO_AREA, NON_MANIFOLD, UNREFERENCED],
                         ids=["empty", "single", "duplicate", "zero-area", "non-manifold", "unreferenced"])
def test_degenerate_mesh_preprocessing(vertices, faces, expected):
    points, normals = mpr.oriented_points_from_mesh(vertices, faces)
    assert len(points) == expected and points.shape == normals.shape
    assert np.isfinite(normals).all()
    if expected:
        assert np.allclose(np.linalg.norm(normals, axis=1), 1.0)


def test_mesh_normals_are_area_weighted():
    vertices = np.array([[0, 0, 0], [2, 0, 0], [0, 2, 0], [0, 0, 1]], dtype=np.float64)
    faces = np.array([[0, 1, 2], [0, 3, 1]], dtype=np.int64)
    points, normals = mpr.oriented_points_from_mesh(vertices, faces)
    origin = np.flatnonzero(np.all(points == vertices[0], axis=1))[0]
    assert np.allclose(normals[origin], [0.0, 1 / np.sqrt(5), 2 / np.sqrt(5)])


def _reference_loop(vertices, faces):
    """The per-face loop of core.py:429-450, restated for the bit comparison."""
    normals = np.zeros_like(vertices)
    referenced = np.zeros(len(vertices), dtype=bool)
    for a, b, c in faces:
        cross = np.cross(vertices[b] - vertices[a], vertices[c] - vertices[a])
        if np.isfinite(cross).all() and np.dot(cross, cross) > 0:
            normals[a] += cross
            normals[b] += cross
            normals[c] += cross
            referenced[[a, b, c]] = True
    lengths = np.linalg.norm(normals, axis=1)
    keep = referenced & (lengths > 0) & np.isfinite(lengths)
    normals[keep] /= lengths[keep, None]
    return vertices[keep], normals[keep]


def test_mesh_normals_bit_identical_to_per_face_loop():
    rng = np.random.default_rng(1)
    v = rng.normal(size=(300, 3))
    f = rng.integers(0, 300, size=(2000, 3))
    f[5] = [4, 4, 9]
    p1, n1 = mpr.oriented_points_from_mesh(v, f)
    p2, n2 = _reference_loop(v, f)
    assert np.array_equal(p1, p2) and np.array_equal(n1, n2)


def test_mesh_normals_bit_identical_on_a_closed_mesh():
    """A sphere mesh from the library's own reconstruction: every vertex referenced."""
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.sphere(3000, seed=0)
    mesh = mpr.reconstruct(pts, nrm, depth=5)
    p1, n1 = mpr.oriented_points_from_mesh(mesh.vertices, mesh.faces)
    p2, n2 = _reference_loop(mesh.vertices, mesh.faces)
    assert len(p1) == len(mesh.vertices)
    assert np.array_equal(p1, p2) and np.array_equal(n1, n2)


def test_device_inputs_and_out_of_range_faces():
    v = torch.rand(10, 3, dtype=torch.float64, device="cuda")
    f = torch.tensor([[0, 1, 2], [3, 4, 5]], device="cuda")
    p1, n1 = mpr.oriented_points_from_mesh(v, f)
    p2, n2 = _reference_loop(v.cpu().numpy(), f.cpu().numpy())
    assert np.array_equal(p1, p2) and np.array_equal(n1, n2)
    with pytest.raises(ValueError, match="face index out of range"):
        mpr.oriented_points_from_mesh(v, torch.tensor([[0, 1, 10]], device="cuda"))


def test_reconstruct_mesh_matches_points_path():
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.sphere(3000, seed=0)
    mesh = mpr.reconstruct(pts, nrm, depth=5)
    a = mpr.reconstruct_mesh(mesh.vertices, mesh.faces, depth=5)
    p, n = mpr.oriented_points_from_mesh(mesh.vertices, mesh.faces)
    b = mpr.reconstruct(p, n, depth=5)
    assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.faces, b.faces)
