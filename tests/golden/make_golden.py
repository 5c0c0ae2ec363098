"""Generate the golden fixtures in this directory from the reference itself.

Run in a checkout that has the reference mounted (default /root/reference):

    make -C oracle && python tests/golden/make_golden.py [/path/to/reference]

Sources of truth, per fixture:

* `kernels_numpy.npz` — outputs of the reference's NumPy translations
  (python/mojo_poissonrecon/_reference.py: octree_codes :8-18, splat :21-87,
  assemble :90-124, restrict :127-155, dual_isosurface :158-249) and of the
  NumPy stencils in the reference's tests (tests/test_kernels.py:106-165),
  all on seeded inputs.  Independent of any native code.
* `pipeline_small.npz` — the reference's own orchestration (core.py:
  build_octree :86-127, solve_screened_poisson :196-306, extract_isosurface
  :309-374, reconstruct :388-426) with the CPU oracle library standing in for
  the Mojo library (the reference's test suite passes against it; see
  oracle/run_reference_tests.py).  Inputs: the 2,000-point unit-sphere cloud
  from seed 0 (README.md:62-72) at depth 5 with 5 V-cycles, and a 400-point
  confidence-weighted ellipsoid cloud at depth 4.

The fixtures are committed; tests read them without the reference present.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))


def _stencil_sum_degree(values):
    # tests/test_kernels.py:106-121, restated.
    neighbor_sum = np.zeros_like(values)
    degree = np.zeros(values.shape, dtype=np.int64)
    neighbor_sum[:, :, 1:] += values[:, :, :-1]
    degree[:, :, 1:] += 1
    neighbor_sum[:, :, :-1] += values[:, :, 1:]
    degree[:, :, :-1] += 1
    neighbor_sum[:, 1:, :] += values[:, :-1, :]
    degree[:, 1:, :] += 1
    neighbor_sum[:, :-1, :] += values[:, 1:, :]
    degree[:, :-1, :] += 1
    neighbor_sum[1:, :, :] += values[:-1, :, :]
    degree[1:, :, :] += 1
    neighbor_sum[:-1, :, :] += values[1:, :, :]
    degree[:-1, :, :] += 1
    return neighbor_sum, degree


def sphere_cloud(count: int, seed: int) -> np.ndarray:
    """README.md:62-72 / bench/bench.py:34-41 sphere sampling."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, count)
    theta = rng.uniform(0.0, 2.0 * np.pi, count)
    r = np.sqrt(1.0 - z * z)
    return np.ascontiguousarray(np.column_stack((r * np.cos(theta), r * np.sin(theta), z)))


def kernels_numpy(ref) -> dict:
    out = {}
    # Octree codes (exact): the reference test's seed-3 case plus edge points.
    pts = np.random.default_rng(3).random((200, 3))
    pts = np.vstack([pts, [[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.5, 0.5, 0.5], [1.0, 0.0, 0.25]]])
    out["octree_points"] = pts
    out["octree_codes_d7"] = ref.octree_codes(pts, 7)

    # Splat + assemble: the reference test's hand case (confidence) and a seeded cloud.
    hand_p = np.array([[0.15, 0.25, 0.35], [0.8, 0.7, 0.6], [1.0, 0.5, 0.0]])
    hand_n = np.array([[2.0, 0.0, 0.0], [0.0, -3.0, 0.0], [0.0, 0.0, 4.0]])
    rng = np.random.default_rng(5)
    rand_p = rng.random((300, 3))
    rand_n = rng.normal(size=(300, 3))
    out["splat_hand_points"], out["splat_hand_normals"] = hand_p, hand_n
    out["splat_rand_points"], out["splat_rand_normals"] = rand_p, rand_n
    for tag, p, nrm, n, conf, spn in (
        ("hand_n5_conf", hand_p, hand_n, 5, True, 1.0),
        ("rand_n9_conf", rand_p, rand_n, 9, True, 1.5),
        ("rand_n17_plain", rand_p, rand_n, 17, False, 1.5),
    ):
        density, vx, vy, vz, screen = ref.splat(p, nrm, n, conf, samples_per_node=spn)
        out[f"splat_{tag}_density"] = density
        out[f"splat_{tag}_vx"] = vx
        out[f"splat_{tag}_vy"] = vy
        out[f"splat_{tag}_vz"] = vz
        out[f"splat_{tag}_screen"] = screen
        out[f"splat_{tag}_rhs"] = ref.assemble(vx, vy, vz, screen, 4.0)

    # Restriction (seed 11 as tests/test_kernels.py:61-64, plus 17^3).
    for n, seed in ((9, 11), (17, 12)):
        fine = np.random.default_rng(seed).normal(size=(n, n, n))
        out[f"restrict_{n}_fine"] = fine
        out[f"restrict_{n}_coarse"] = ref.restrict(fine)

    # Residual and one red-black sweep (tests/test_kernels.py:124-165).
    for n in (9, 17):
        rng = np.random.default_rng(n)
        solution = rng.normal(size=(n, n, n))
        rhs = rng.normal(size=(n, n, n))
        screen = rng.random((n, n, n))
        h_inv2 = float((n - 1) ** 2)
        neighbor_sum, degree = _stencil_sum_degree(solution)
        residual = rhs - ((degree * h_inv2 + 4.0 * screen * h_inv2) * solution - neighbor_sum * h_inv2)
        relaxed = solution.copy()
        parity = np.indices((n, n, n)).sum(axis=0) & 1
        for color in range(2):
            nsum, deg = _stencil_sum_degree(relaxed)
            diagonal = deg * h_inv2 + 4.0 * screen * h_inv2
            mask = (parity == color) & (diagonal > 1.0e-30)
            relaxed[mask] = (rhs[mask] + nsum[mask] * h_inv2) / diagonal[mask]
        out[f"stencil_{n}_solution"] = solution
        out[f"stencil_{n}_rhs"] = rhs
        out[f"stencil_{n}_screen"] = screen
        out[f"stencil_{n}_residual"] = residual
        out[f"stencil_{n}_relaxed"] = relaxed

    # Dual contouring: the 13^3 sphere SDF (tests/test_kernels.py:188-195) and a noisy field.
    axis = np.linspace(0.0, 1.0, 13)
    z, y, x = np.meshgrid(axis, axis, axis, indexing="ij")
    sphere = (x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2 - 0.3**2
    out["dual_sphere13_field"] = sphere
    v, f = ref.dual_isosurface(sphere, 0.0)
    out["dual_sphere13_vertices"], out["dual_sphere13_faces"] = v, f
    noisy = np.random.default_rng(9).normal(size=(10, 10, 10))
    out["dual_noisy10_field"] = noisy
    v, f = ref.dual_isosurface(noisy, 0.1)
    out["dual_noisy10_vertices"], out["dual_noisy10_faces"] = v, f
    return out


def pipeline(mpr) -> dict:
    out = {}
    pts = sphere_cloud(2000, 0)
    out["sphere_points"] = pts
    # Solve on the normalised cloud exactly as reconstruct() would (core.py:412).
    unit, origin, width = mpr.core._normalize(pts, 1.1)
    sol = mpr.solve_screened_poisson(unit, pts, depth=5, cycles=5)
    out["sphere_unit_points"] = unit
    for name in ("field", "density", "screen", "rhs"):
        out[f"sphere_{name}"] = getattr(sol, name)
    out["sphere_iso"] = np.float64(sol.iso_value)
    out["sphere_residual_norm"] = np.float64(sol.residual_norm)
    for name in ("depth", "morton", "parent", "child_start", "child_count", "point_leaf"):
        out[f"sphere_octree_{name}"] = getattr(sol.octree, name)
    mesh = mpr.reconstruct(pts, pts, depth=5, cycles=5)
    out["sphere_mesh_vertices"] = mesh.vertices
    out["sphere_mesh_faces"] = mesh.faces
    out["sphere_mesh_density"] = mesh.density
    out["sphere_mesh_iso"] = np.float64(mesh.iso_value)
    out["sphere_mesh_residual_norm"] = np.float64(mesh.residual_norm)

    # Confidence-weighted ellipsoid at depth 4 (normals scaled by U(0.5, 1.5)).
    rng = np.random.default_rng(21)
    u = rng.normal(size=(400, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    axes = np.array([0.9, 0.5, 0.35])
    p = u * axes
    nrm = u / axes
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm *= rng.uniform(0.5, 1.5, size=(400, 1))
    out["ellipsoid_points"], out["ellipsoid_normals"] = p, nrm
    mesh = mpr.reconstruct(p, nrm, depth=4, cycles=3, confidence=True, point_weight=2.0)
    out["ellipsoid_mesh_vertices"] = mesh.vertices
    out["ellipsoid_mesh_faces"] = mesh.faces
    out["ellipsoid_mesh_density"] = mesh.density
    out["ellipsoid_mesh_iso"] = np.float64(mesh.iso_value)
    out["ellipsoid_mesh_residual_norm"] = np.float64(mesh.residual_norm)
    return out


def main(argv: list[str]) -> None:
    reference = argv[1] if len(argv) > 1 else "/root/reference"
    sys.path.insert(0, os.path.join(reference, "python"))
    sys.dont_write_bytecode = True
    from run_reference_tests import install_oracle

    import mojo_poissonrecon as mpr
    from mojo_poissonrecon import _reference

    install_oracle(os.path.join(REPO, "oracle", "liboracle_mpr.so"))
    np.savez_compressed(os.path.join(HERE, "kernels_numpy.npz"), **kernels_numpy(_reference))
    np.savez_compressed(os.path.join(HERE, "pipeline_small.npz"), **pipeline(mpr))
    for name in ("kernels_numpy.npz", "pipeline_small.npz"):
        print(name, os.path.getsize(os.path.join(HERE, name)), "bytes")


if __name__ == "__main__":
    main(sys.argv)
