"""Pins the CPU oracle (oracle/mpr_oracle.c + oracle/pipeline.py) against the
golden vectors made from the reference (tests/golden/make_golden.py), with the
reference tests' own tolerances (tests/test_kernels.py)."""

import ctypes

import numpy as np
import pytest


def _a(x):
    return int(x.ctypes.data)


def test_octree_codes_exact(oracle, golden_kernels):
    pts = golden_kernels["octree_points"]
    assert np.array_equal(oracle.octree_codes(pts, 7), golden_kernels["octree_codes_d7"])


@pytest.mark.parametrize(
    "tag,points,normals,n,conf,spn",
    [
        ("hand_n5_conf", "splat_hand_points", "splat_hand_normals", 5, True, 1.0),
        ("rand_n9_conf", "splat_rand_points", "splat_rand_normals", 9, True, 1.5),
        ("rand_n17_plain", "splat_rand_points", "splat_rand_normals", 17, False, 1.5),
    ],
)
def test_splat_and_assemble_match_numpy_translation(oracle, golden_kernels, tag, points, normals, n, conf, spn):
    g = golden_kernels
    p, nrm = g[points], g[normals]
    L = oracle.lib()
    grids = [np.zeros((n, n, n)) for _ in range(5)]
    density, vx, vy, vz, screen = grids
    accepted = L.mpr_splat_f64(_a(p), _a(nrm), len(p), n, int(conf), *(_a(x) for x in grids), spn)
    assert accepted == len(p)
    rhs = np.zeros((n, n, n))
    L.mpr_assemble_f64(_a(vx), _a(vy), _a(vz), _a(screen), _a(rhs), n, 4.0, 0.5)
    # tests/test_kernels.py:41-43 tolerances; the vector field is compared the same way.
    assert np.allclose(density, g[f"splat_{tag}_density"], rtol=0, atol=2e-15)
    assert np.allclose(screen, g[f"splat_{tag}_screen"], rtol=0, atol=2e-15)
    for k, v in (("vx", vx), ("vy", vy), ("vz", vz)):
        ref = g[f"splat_{tag}_{k}"]
        assert np.allclose(v, ref, rtol=1e-14, atol=1e-14 * max(1.0, np.abs(ref).max()))
    assert np.allclose(rhs, g[f"splat_{tag}_rhs"], rtol=0, atol=2e-13 * max(1.0, np.abs(rhs).max() / 100))


def test_confidence_known_sums(oracle):
    # tests/test_kernels.py:46-58 known answers.
    pts = np.array([[0.25, 0.25, 0.25], [0.75, 0.75, 0.75]])
    nrm = np.array([[1.0, 0.0, 0.0], [0.0, 2.0, 0.0]])
    plain = oracle.solve(pts, nrm, depth=2, cycles=1, confidence=False, samples_per_node=1.0)
    weighted = oracle.solve(pts, nrm, depth=2, cycles=1, confidence=True, samples_per_node=1.0)
    assert plain.density.sum() == 4.0 and weighted.density.sum() == 6.0
    assert plain.screen.sum() == 2.0 and weighted.screen.sum() == 3.0


@pytest.mark.parametrize("n", [9, 17])
def test_restrict_matches_numpy_translation(oracle, golden_kernels, n):
    fine = golden_kernels[f"restrict_{n}_fine"]
    assert np.allclose(oracle.restrict(fine), golden_kernels[f"restrict_{n}_coarse"], rtol=0, atol=2e-16)


@pytest.mark.parametrize("n", [9, 17])
def test_residual_and_relax_match_numpy_stencils(oracle, golden_kernels, n):
    g = golden_kernels
    sol, rhs, scr = g[f"stencil_{n}_solution"], g[f"stencil_{n}_rhs"], g[f"stencil_{n}_screen"]
    L = oracle.lib()
    res = np.empty_like(sol)
    norm = L.mpr_residual_f64(_a(sol), _a(rhs), _a(scr), _a(res), n, 4.0)
    assert np.allclose(res, g[f"stencil_{n}_residual"], rtol=2e-15, atol=3e-11)
    assert norm == pytest.approx(np.linalg.norm(g[f"stencil_{n}_residual"]), rel=2e-15)
    relaxed = sol.copy()
    L.mpr_relax_f64(_a(relaxed), _a(rhs), _a(scr), n, 4.0, 1)
    assert np.allclose(relaxed, g[f"stencil_{n}_relaxed"], rtol=0, atol=2e-15)


def test_prolong_and_iso_known_answers(oracle):
    # tests/test_kernels.py:67-88.
    L = oracle.lib()
    coarse = np.arange(125, dtype=np.float64).reshape(5, 5, 5)
    fine = np.zeros((9, 9, 9))
    L.mpr_prolong_add_f64(_a(coarse), _a(fine), 9)
    assert np.array_equal(fine[::2, ::2, ::2], coarse)
    assert fine[1, 1, 1] == pytest.approx(coarse[:2, :2, :2].mean())
    pts = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5], [1.0, 1.0, 1.0]])
    nrm = np.ones_like(pts)
    iso = L.mpr_iso_value_f64(_a(fine), _a(pts), _a(nrm), 3, 9, 0)
    assert iso == pytest.approx(np.mean([fine[0, 0, 0], fine[4, 4, 4], fine[8, 8, 8]]))


@pytest.mark.parametrize("case,iso", [("sphere13", 0.0), ("noisy10", 0.1)])
def test_dual_contour_matches_numpy_translation(oracle, golden_kernels, case, iso):
    g = golden_kernels
    mesh = oracle.extract(g[f"dual_{case}_field"], iso)
    assert np.allclose(mesh.vertices, g[f"dual_{case}_vertices"], rtol=0, atol=4e-16)
    assert np.array_equal(mesh.faces, g[f"dual_{case}_faces"])


def test_dual_vertex_count_matches_numpy(oracle):
    # tests/test_kernels.py:168-185 at n = 14 and 65.
    L = oracle.lib()
    for n in (14, 65):
        field = np.random.default_rng(n).normal(size=(n, n, n))
        below = field < 0.0
        cnt = sum(below[dz:dz + n - 1, dy:dy + n - 1, dx:dx + n - 1]
                  for dz in range(2) for dy in range(2) for dx in range(2))
        expected = np.count_nonzero((cnt != 0) & (cnt != 8))
        scratch = np.empty((n - 1 + 3) // 4, np.int64)
        dummy = np.zeros(1)
        assert L.mpr_dual_vertices_f64(_a(field), _a(field), n, 0.0, _a(scratch), _a(dummy), _a(dummy), 0) == expected


def test_pipeline_reproduces_reference_orchestration(oracle, golden_pipeline):
    """oracle/pipeline.py (a restatement of core.py) gives the same bits as the
    reference's own core.py driving the same native oracle."""
    g = golden_pipeline
    sol = oracle.solve(g["sphere_unit_points"], g["sphere_points"], depth=5, cycles=5)
    for k in ("field", "density", "screen", "rhs"):
        assert np.array_equal(getattr(sol, k), g[f"sphere_{k}"]), k
    assert sol.iso_value == g["sphere_iso"] and sol.residual_norm == g["sphere_residual_norm"]
    for k in ("depth", "morton", "parent", "child_start", "child_count", "point_leaf"):
        assert np.array_equal(getattr(sol.octree, k), g[f"sphere_octree_{k}"]), k
    mesh = oracle.reconstruct(g["sphere_points"], g["sphere_points"], depth=5, cycles=5)
    assert np.array_equal(mesh.vertices, g["sphere_mesh_vertices"])
    assert np.array_equal(mesh.faces, g["sphere_mesh_faces"])
    mesh = oracle.reconstruct(g["ellipsoid_points"], g["ellipsoid_normals"], depth=4, cycles=3, confidence=True,
                              point_weight=2.0)
    assert np.array_equal(mesh.vertices, g["ellipsoid_mesh_vertices"])
    assert np.array_equal(mesh.faces, g["ellipsoid_mesh_faces"])
    assert mesh.iso_value == g["ellipsoid_mesh_iso"]


def test_octree_matches_numpy_translation(oracle, golden_kernels):
    # tests/test_kernels.py:10-21 on the golden points.
    pts = golden_kernels["octree_points"]
    expected = golden_kernels["octree_codes_d7"]
    tree = oracle.build_octree(pts, 7)
    for d in range(8):
        assert np.array_equal(tree.morton[tree.depth == d], np.unique(expected[:, d]))
    assert np.array_equal(tree.morton[tree.point_leaf], expected[:, -1])
    assert np.array_equal(tree.morton[tree.parent[tree.depth > 0]], tree.morton[tree.depth > 0] >> 3)


def test_openmp_build_is_bit_identical(oracle):
    pts = np.random.default_rng(4).random((3000, 3))
    nrm = np.random.default_rng(5).normal(size=(3000, 3))
    a = oracle.solve(pts, nrm, depth=6, cycles=2, threaded=False)
    b = oracle.solve(pts, nrm, depth=6, cycles=2, threaded=True)
    assert np.array_equal(a.field, b.field) and a.iso_value == b.iso_value


def test_tolerance_loop_reaches_target(oracle, golden_pipeline):
    g = golden_pipeline
    sol = oracle.solve(g["sphere_unit_points"], g["sphere_points"], depth=5, tol=1e-8, max_cycles=60)
    assert sol.relative_residual <= 1e-8
    assert 5 < sol.cycles_run < 60


def test_planted_mistake_is_caught(oracle, golden_kernels):
    """A checker that cannot fail proves nothing: perturb one oracle output by
    one ulp (on the CPU) and confirm the exact comparison notices."""
    fine = golden_kernels["restrict_9_fine"]
    coarse = oracle.restrict(fine)
    coarse[2, 2, 2] = np.nextafter(coarse[2, 2, 2], np.inf)
    assert not np.array_equal(coarse, oracle.restrict(fine))
