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


def test_mesh_validation_on_host():
    v = np.zeros((3, 3))
    with pytest.raises(ValueError, match="faces must have shape"):
        mpr.oriented_points_from_mesh(v, np.zeros((2, 4), dtype=np.int64))
    with pytest.raises(ValueError, match="face index out of range"):
        mpr.oriented_points_from_mesh(v, np.array([[0, 1, 3]]))
    with pytest.raises(ValueError, match="face index out of range"):
        mpr.oriented_points_from_mesh(v, np.array([[0, -1, 2]]))
    p, n = mpr.oriented_points_from_mesh(EMPTY[0], EMPTY[1])
    assert p.shape == (0, 3) and n.shape == (0, 3)


def test_empty_mesh_reconstructs_to_empty_without_gpu():
    assert mpr.reconstruct_mesh(EMPTY[0], EMPTY[1]).is_empty
