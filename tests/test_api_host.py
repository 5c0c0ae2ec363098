"""Host-side behaviour of the public API that needs no GPU: validation errors
(tests/test_kernels.py:91-103, :198-208 of the reference), the conversion
guards, and mesh preprocessing (tests/test_reconstruction.py:86-179)."""

import numpy as np
import pytest

import mojo_poissonrecon_b200 as mpr
from mojo_poissonrecon_b200._convert import addr, f64, i64


def test_public_names_match_reference():
    for name in ("FlatOctree", "GridSolution", "Mesh", "build", "build_octree", "extract_isosurface",
                 "oriented_points_from_mesh", "reconstruct", "reconstruct_mesh", "solve_screened_poisson"):
        assert hasattr(mpr, name)


def test_conversions_reject_narrowing_and_bad_buffers():
    import torch

    with pytest.raises(TypeError, match="complex"):
        f64(np.array([1 + 2j]))
    with pytest.raises(TypeError, match="real numbers"):
        f64(["1.0"])
    with pytest.raises(ValueError, match="exactly"):
        f64(np.array([2**53 + 1], dtype=np.int64))
    with pytest.raises(ValueError, match="finite integers"):
        i64(np.array([1.5]))
    with pytest.raises(TypeError, match="dtype"):
        addr(torch.ones(3, dtype=torch.float32))
    with pytest.raises(TypeError, match="CUDA"):
        addr(np.ones(3))


def test_public_validation_rejects_unsafe_values():
    points = np.array([[0.25, 0.25, 0.25]])
    normals = np.array([[1.0, 0.0, 0.0]])
    with pytest.raises(TypeError, match="depth"):
        mpr.solve_screened_poisson(points, normals, depth=2.5)
    with pytest.raises(ValueError, match="finite"):
        mpr.solve_screened_poisson(points, normals, point_weight=np.nan)
    with pytest.raises(ValueError, match="density must be finite"):
        mpr.extract_isosurface(np.zeros((2, 2, 2)), density=np.full((2, 2, 2), np.nan))
    with pytest.raises(ValueError, match="greater than 1"):
        mpr.reconstruct(points, normals, scale=1.0)
    with pytest.raises(ValueError, match="depth must be between 2 and 10"):
        mpr.solve_screened_poisson(points, normals, depth=11)
    with pytest.raises(ValueError, match="cycles"):
        mpr.solve_screened_poisson(points, normals, cycles=0)
    with pytest.raises(ValueError, match="precision"):
        mpr.solve_screened_poisson(points, normals, precision="fp16")
    with pytest.raises(ValueError, match="tol"):
        mpr.solve_screened_poisson(points, normals, tol=-1.0)
    with pytest.raises(ValueError, match="shape"):
        mpr.reconstruct(np.zeros((3, 2)), np.zeros((3, 2)))
    with pytest.raises(ValueError, match="same shape"):
        mpr.reconstruct(np.zeros((3, 3)), np.zeros((4, 3)))
    with pytest.raises(ValueError, match="cubic"):
        mpr.extract_isosurface(np.zeros((2, 3, 2)))
    with pytest.raises(ValueError, match="between 0 and 19"):
        mpr.build_octree(points, 20)


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


def test_empty_mesh_reconstructs_to_empty_without_gpu():
    assert mpr.reconstruct_mesh(EMPTY[0], EMPTY[1]).is_empty
